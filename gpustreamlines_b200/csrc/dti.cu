// The steps before tracking that the reference runs on the host through DIPY
// (run_gpu_streamlines.py:289-314): the DTI fit for the FA stopping map and
// the random seeds from a mask.
//
// FA: per voxel, weighted least squares on log signals (the WLS method of
// dipy.reconst.dti, after Salvador et al. 2005 / Chung et al. 2006): an OLS
// fit beta0 = pinv(X) y, weights w = exp(X beta0), then the fit of
// (w * X) beta = w * y through the 7x7 normal equations (Cholesky, double);
// D from beta[1..6], eigenvalues of the symmetric 3x3 by the trigonometric
// closed form, clipped at 0; FA = sqrt(3/2) |lambda - mean| / |lambda|.
// One thread per voxel, double precision, design matrix in shared memory.
//
// Seeds: voxels whose mask value exceeds a threshold are listed in order
// (CUB select), then seed i takes voxel floor(u0 * n_voxels) and the jitter
// (u1, u2, u3) - 0.5, u in [0, 1) with 24 bits, from Philox stream (key =
// seed, subsequence = i): the
// distribution of dipy.tracking.utils.random_seeds_from_mask
// (seed_count_per_voxel=False), with a counter-based generator.
#include <cuda_runtime.h>

#include <cmath>
#include <cub/cub.cuh>
#include <vector>

#include "philox.cuh"

namespace csl {

constexpr int kDtiMaxT = 512;

__global__ void dti_fa_kernel(const float *__restrict__ dwi, long long nvox, int T, const double *__restrict__ Xg,
                              const double *__restrict__ Pg, const float *__restrict__ mask, double min_signal,
                              float *__restrict__ fa) {
    extern __shared__ double sm[];
    double *X = sm;          // [T][7]
    double *Pm = sm + 7 * T;  // [7][T]
    for (int e = threadIdx.x; e < 7 * T; e += blockDim.x) {
        X[e] = Xg[e];
        Pm[e] = Pg[e];
    }
    __syncthreads();
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nvox;
         v += (long long)gridDim.x * blockDim.x) {
        if (mask && !(mask[v] > 0.0f)) {
            fa[v] = 0.0f;
            continue;
        }
        const float *s = dwi + v * T;
        double b0[7] = {0, 0, 0, 0, 0, 0, 0};
        for (int t = 0; t < T; t++) {
            const double y = log(fmax((double)s[t], min_signal));
#pragma unroll
            for (int k = 0; k < 7; k++) b0[k] += Pm[k * T + t] * y;
        }
        double A[28] = {0};  // packed lower triangle of X^T W^2 X
        double r[7] = {0, 0, 0, 0, 0, 0, 0};
        for (int t = 0; t < T; t++) {
            const double *x = X + 7 * t;
            double pred = 0;
#pragma unroll
            for (int k = 0; k < 7; k++) pred += x[k] * b0[k];
            const double w = exp(pred);
            const double w2 = w * w;
            const double y = log(fmax((double)s[t], min_signal));
            int q = 0;
#pragma unroll
            for (int i = 0; i < 7; i++) {
                r[i] += w2 * x[i] * y;
#pragma unroll
                for (int j = 0; j <= i; j++) A[q++] += w2 * x[i] * x[j];
            }
        }
        // Cholesky of the packed 7x7 (row i starts at i(i+1)/2)
        double Lm[7][7];
        bool ok = true;
        for (int i = 0; i < 7 && ok; i++) {
            for (int j = 0; j <= i; j++) {
                double sum = A[i * (i + 1) / 2 + j];
                for (int k = 0; k < j; k++) sum -= Lm[i][k] * Lm[j][k];
                if (i == j) {
                    if (!(sum > 0)) {
                        ok = false;
                        break;
                    }
                    Lm[i][i] = sqrt(sum);
                } else {
                    Lm[i][j] = sum / Lm[j][j];
                }
            }
        }
        double beta[7];
        if (ok) {
            double z[7];
            for (int i = 0; i < 7; i++) {
                double sum = r[i];
                for (int k = 0; k < i; k++) sum -= Lm[i][k] * z[k];
                z[i] = sum / Lm[i][i];
            }
            for (int i = 6; i >= 0; i--) {
                double sum = z[i];
                for (int k = i + 1; k < 7; k++) sum -= Lm[k][i] * beta[k];
                beta[i] = sum / Lm[i][i];
            }
        } else {
            for (int k = 0; k < 7; k++) beta[k] = b0[k];
        }
        // eigenvalues of D = [[b1 b4 b5] [b4 b2 b6] [b5 b6 b3]]
        const double a11 = beta[1], a22 = beta[2], a33 = beta[3], a12 = beta[4], a13 = beta[5], a23 = beta[6];
        const double p1 = a12 * a12 + a13 * a13 + a23 * a23;
        double e1, e2, e3;
        if (p1 == 0.0) {
            e1 = a11;
            e2 = a22;
            e3 = a33;
        } else {
            const double q = (a11 + a22 + a33) / 3.0;
            const double p2 = (a11 - q) * (a11 - q) + (a22 - q) * (a22 - q) + (a33 - q) * (a33 - q) + 2.0 * p1;
            const double p = sqrt(p2 / 6.0);
            const double b11 = (a11 - q) / p, b22 = (a22 - q) / p, b33 = (a33 - q) / p;
            const double b12 = a12 / p, b13 = a13 / p, b23 = a23 / p;
            double rr = (b11 * (b22 * b33 - b23 * b23) - b12 * (b12 * b33 - b23 * b13) + b13 * (b12 * b23 - b22 * b13)) / 2.0;
            rr = rr < -1.0 ? -1.0 : (rr > 1.0 ? 1.0 : rr);
            const double phi = acos(rr) / 3.0;
            e1 = q + 2.0 * p * cos(phi);
            e3 = q + 2.0 * p * cos(phi + 2.0943951023931957);
            e2 = 3.0 * q - e1 - e3;
        }
        e1 = fmax(e1, 0.0);
        e2 = fmax(e2, 0.0);
        e3 = fmax(e3, 0.0);
        const double md = (e1 + e2 + e3) / 3.0;
        const double num = sqrt((e1 - md) * (e1 - md) + (e2 - md) * (e2 - md) + (e3 - md) * (e3 - md));
        const double den = sqrt(e1 * e1 + e2 * e2 + e3 * e3);
        double f = den > 0 ? sqrt(1.5) * num / den : 0.0;
        f = f < 0 ? 0 : (f > 1 ? 1 : f);
        fa[v] = (float)f;
    }
}

struct AboveThreshold {
    const float *m;
    float thr;
    __device__ __forceinline__ bool operator()(const long long &i) const { return m[i] > thr; }
};

__global__ void seeds_kernel(const long long *__restrict__ vox, const long long *__restrict__ nvox_d, int Y, int Z,
                             long long n, unsigned long long seed, float *__restrict__ out) {
    const long long nv = *nvox_d;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        Philox g;
        g.init(seed, (unsigned long long)i, 0);
        const uint32_t w0 = g.next(), w1 = g.next(), w2 = g.next(), w3 = g.next();
        long long k = (long long)(((unsigned long long)w0 * (unsigned long long)nv) >> 32);
        if (nv <= 0) k = 0;
        const long long v = nv > 0 ? vox[k] : 0;
        const long long x = v / ((long long)Y * Z), y = (v / Z) % Y, z = v % Z;
        // jitter in [-0.5, 0.5): 24-bit uniforms in [0, 1), exact in float32
        const float s24 = 5.9604644775390625e-08f;  // 2^-24
        // (the sum is rounded to float32; a value that rounds up to the
        // voxel's upper face is moved one ulp down, so the seed stays in it)
        const long long c[3] = {x, y, z};
        const uint32_t wj[3] = {w1, w2, w3};
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const float base = (float)c[a];
            float f = base + ((float)(wj[a] >> 8) * s24 - 0.5f);
            if (f >= base + 0.5f) f = nextafterf(base + 0.5f, -INFINITY);
            out[3 * i + a] = f;
        }
    }
}

}  // namespace csl

using namespace csl;

// Host: DTI design matrix X [T x 7] (columns 1, -b gx^2, -b gy^2, -b gz^2,
// -2b gx gy, -2b gx gz, -2b gy gz) and its pseudo-inverse (X^T X)^-1 X^T.
static bool dti_design(const double *bvals, const double *bvecs, int T, std::vector<double> &X,
                       std::vector<double> &P) {
    X.assign((size_t)T * 7, 0.0);
    for (int t = 0; t < T; t++) {
        const double b = bvals[t], gx = bvecs[3 * t], gy = bvecs[3 * t + 1], gz = bvecs[3 * t + 2];
        const double row[7] = {1.0, -b * gx * gx, -b * gy * gy, -b * gz * gz, -2 * b * gx * gy, -2 * b * gx * gz,
                               -2 * b * gy * gz};
        for (int k = 0; k < 7; k++) X[(size_t)t * 7 + k] = row[k];
    }
    double M[7][14];
    for (int i = 0; i < 7; i++)
        for (int j = 0; j < 14; j++) M[i][j] = 0.0;
    for (int i = 0; i < 7; i++) {
        for (int j = 0; j < 7; j++)
            for (int t = 0; t < T; t++) M[i][j] += X[(size_t)t * 7 + i] * X[(size_t)t * 7 + j];
        M[i][7 + i] = 1.0;
    }
    for (int c = 0; c < 7; c++) {  // Gauss-Jordan with partial pivoting
        int piv = c;
        for (int r = c + 1; r < 7; r++)
            if (std::fabs(M[r][c]) > std::fabs(M[piv][c])) piv = r;
        if (std::fabs(M[piv][c]) < 1e-300) return false;
        if (piv != c)
            for (int j = 0; j < 14; j++) std::swap(M[c][j], M[piv][j]);
        const double d = M[c][c];
        for (int j = 0; j < 14; j++) M[c][j] /= d;
        for (int r = 0; r < 7; r++)
            if (r != c) {
                const double f = M[r][c];
                for (int j = 0; j < 14; j++) M[r][j] -= f * M[c][j];
            }
    }
    P.assign((size_t)7 * T, 0.0);
    for (int k = 0; k < 7; k++)
        for (int t = 0; t < T; t++) {
            double s = 0;
            for (int j = 0; j < 7; j++) s += M[k][7 + j] * X[(size_t)t * 7 + j];
            P[(size_t)k * T + t] = s;
        }
    return true;
}

extern "C" int csl_dti_fa(const float *dwi_dev, long long nvox, int T, const double *bvals, const double *bvecs,
                          const float *mask_dev, double min_signal, float *fa_dev, void *stream) {
    if (!dwi_dev || !fa_dev || !bvals || !bvecs || nvox < 0 || T < 7 || T > kDtiMaxT || !(min_signal > 0))
        return -1;
    if (nvox == 0) return 0;
    std::vector<double> X, P;
    if (!dti_design(bvals, bvecs, T, X, P)) return -1;
    cudaStream_t st = (cudaStream_t)stream;
    double *d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(double) * 14 * T);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d, X.data(), sizeof(double) * 7 * T, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d + 7 * T, P.data(), sizeof(double) * 7 * T, cudaMemcpyHostToDevice, st);
    const int smem = (int)(sizeof(double) * 14 * T);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(dti_fa_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) {
        dti_fa_kernel<<<2048, 128, smem, st>>>(dwi_dev, nvox, T, d, d + 7 * T, mask_dev, min_signal, fa_dev);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (d) cudaFree(d);
    return e == cudaSuccess ? 0 : -2;
}

extern "C" int csl_seeds_from_mask(const float *mask_dev, int X, int Y, int Z, float threshold, long long n,
                                   unsigned long long seed, float *seeds_dev, long long *nvox_out, void *stream) {
    if (!mask_dev || !seeds_dev || X <= 0 || Y <= 0 || Z <= 0 || n < 0) return -1;
    cudaStream_t st = (cudaStream_t)stream;
    const long long nv = (long long)X * Y * Z;
    long long *vox = nullptr;
    long long *cnt = nullptr;
    void *tmp = nullptr;
    size_t tmpb = 0;
    cub::CountingInputIterator<long long> it(0);
    AboveThreshold pred{mask_dev, threshold};
    cudaError_t e = cub::DeviceSelect::If(nullptr, tmpb, it, (long long *)nullptr, (long long *)nullptr, nv, pred, st);
    if (e == cudaSuccess) e = cudaMalloc(&vox, sizeof(long long) * (nv + 1));
    if (e == cudaSuccess) e = cudaMalloc(&cnt, sizeof(long long));
    if (e == cudaSuccess) e = cudaMalloc(&tmp, tmpb > 0 ? tmpb : 1);
    if (e == cudaSuccess) e = cub::DeviceSelect::If(tmp, tmpb, it, vox, cnt, nv, pred, st);
    long long hcnt = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hcnt, cnt, sizeof(long long), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess && hcnt == 0 && n > 0) e = cudaErrorInvalidValue;
    if (e == cudaSuccess && n > 0) {
        seeds_kernel<<<1024, 256, 0, st>>>(vox, cnt, Y, Z, n, seed, seeds_dev);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (vox) cudaFree(vox);
    if (cnt) cudaFree(cnt);
    if (tmp) cudaFree(tmp);
    if (nvox_out) *nvox_out = hcnt;
    if (e == cudaErrorInvalidValue && hcnt == 0) return -1;
    return e == cudaSuccess ? 0 : -2;
}
