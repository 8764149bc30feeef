// Learned direction proposal: a 48 -> 128 -> 128 -> 128 -> 40 MLP with SiLU
// whose 40 outputs parameterise an 8-component von Mises-Fisher mixture on
// the sphere (per component: 3 mean, 1 concentration, 1 weight logit).  The
// input is the 45 interpolated SH coefficients plus the incoming direction.
//
// Training kernels (FP32): a tiled GEMM with either operand transposed (the
// forward product X W^T, the input gradient dZ W and the weight gradient
// dZ^T X), bias + SiLU forward and backward, the column sums of dZ for the
// bias gradients, the mixture negative log-likelihood with its gradient, and
// Adam.  Inference: one fused kernel, all weights in shared memory
// (transposed so that the lanes of a warp read consecutive outputs), one warp
// per sample.
#include <cuda_runtime.h>

#include <cmath>

namespace csl {

constexpr int kMlpIn = 48, kMlpHid = 128, kMlpOut = 40, kMlpComp = 8;

// ---- C[M x N] = op(A) op(B) (+ beta C); row-major; op = transpose when T*
template <bool TA, bool TB>
__global__ void __launch_bounds__(256) mlp_gemm_kernel(int M, int N, int K, const float *__restrict__ A, int lda,
                                                       const float *__restrict__ B, int ldb, float *__restrict__ C,
                                                       int ldc, float beta) {
    __shared__ float As[16][64 + 4];
    __shared__ float Bs[16][64 + 4];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += 16) {
        for (int e = threadIdx.x; e < 16 * 64; e += 256) {
            const int kk = e / 64, mm = e % 64;
            const int m = m0 + mm, k = k0 + kk;
            float a = 0.0f;
            if (m < M && k < K) a = TA ? A[(size_t)k * lda + m] : A[(size_t)m * lda + k];
            As[kk][mm] = a;
            const int n = n0 + mm;
            float b = 0.0f;
            if (n < N && k < K) b = TB ? B[(size_t)n * ldb + k] : B[(size_t)k * ldb + n];
            Bs[kk][mm] = b;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; kk++) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int m = m0 + ty * 4 + i, n = n0 + tx * 4 + j;
            if (m < M && n < N) {
                float *c = C + (size_t)m * ldc + n;
                *c = beta != 0.0f ? acc[i][j] + beta * *c : acc[i][j];
            }
        }
}

__device__ __forceinline__ float sigm(float z) { return 1.0f / (1.0f + expf(-z)); }

// Z += b (row-broadcast); A = silu(Z) when act, else A = Z
__global__ void mlp_bias_act_kernel(float *Z, const float *__restrict__ b, float *A, int M, int N, int act) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < (long long)M * N;
         e += (long long)gridDim.x * blockDim.x) {
        const float z = Z[e] + b[e % N];
        Z[e] = z;
        A[e] = act ? z * sigm(z) : z;
    }
}

// dZ = dA * silu'(Z)
__global__ void mlp_act_bwd_kernel(const float *__restrict__ Z, const float *__restrict__ dA, float *dZ, long long n) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const float s = sigm(Z[e]);
        dZ[e] = dA[e] * (s + Z[e] * s * (1.0f - s));
    }
}

// db[n] = sum_m dZ[m, n]
__global__ void mlp_colsum_kernel(const float *__restrict__ dZ, int M, int N, float *db) {
    const int n = blockIdx.x;
    float s = 0.0f;
    for (int m = threadIdx.x; m < M; m += blockDim.x) s += dZ[(size_t)m * N + n];
    __shared__ float red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) db[n] = red[0];
}

// log(sinh k) and 1/k - coth k, stable for small and large k
__device__ __forceinline__ void vmf_terms(float k, float &logsinh, float &f) {
    logsinh = k + log1pf(-expf(-2.0f * k)) - 0.69314718f;
    f = (k < 1e-3f) ? -k / 3.0f : 1.0f / k - 1.0f / tanhf(k);
}

// mixture negative log-likelihood of the unit target x per sample, its
// gradient w.r.t. the 40 outputs (scaled by gscale), loss per sample
__global__ void mlp_vmf_nll_kernel(const float *__restrict__ Y, const float *__restrict__ X, int B, float gscale,
                                   float *loss, float *dY) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B) return;
    const float *y = Y + (size_t)i * kMlpOut;
    const float x0 = X[3 * i], x1 = X[3 * i + 1], x2 = X[3 * i + 2];
    float s[kMlpComp], kap[kMlpComp], dot[kMlpComp], nrm[kMlpComp], mu[kMlpComp][3], fk[kMlpComp];
    float lmax = -INFINITY;
    for (int k = 0; k < kMlpComp; k++) lmax = fmaxf(lmax, y[5 * k + 4]);
    float lse_l = 0.0f;
    for (int k = 0; k < kMlpComp; k++) lse_l += expf(y[5 * k + 4] - lmax);
    lse_l = lmax + logf(lse_l);
    float smax = -INFINITY;
    for (int k = 0; k < kMlpComp; k++) {
        const float m0 = y[5 * k], m1 = y[5 * k + 1], m2 = y[5 * k + 2];
        nrm[k] = sqrtf(m0 * m0 + m1 * m1 + m2 * m2) + 1e-12f;
        mu[k][0] = m0 / nrm[k];
        mu[k][1] = m1 / nrm[k];
        mu[k][2] = m2 / nrm[k];
        const float kr = y[5 * k + 3];
        kap[k] = (kr > 20.0f ? kr : log1pf(expf(kr))) + 1e-3f;
        dot[k] = mu[k][0] * x0 + mu[k][1] * x1 + mu[k][2] * x2;
        float logsinh;
        vmf_terms(kap[k], logsinh, fk[k]);
        const float logc = logf(kap[k]) - 2.5310242f - logsinh;  // log(4 pi) = 2.5310242
        s[k] = (y[5 * k + 4] - lse_l) + logc + kap[k] * dot[k];
        smax = fmaxf(smax, s[k]);
    }
    float tot = 0.0f;
    for (int k = 0; k < kMlpComp; k++) tot += expf(s[k] - smax);
    const float lse = smax + logf(tot);
    loss[i] = -lse;
    float *g = dY + (size_t)i * kMlpOut;
    for (int k = 0; k < kMlpComp; k++) {
        const float r = expf(s[k] - lse);
        const float pi = expf(y[5 * k + 4] - lse_l);
        g[5 * k + 4] = gscale * (pi - r);
        const float kr = y[5 * k + 3];
        g[5 * k + 3] = gscale * (-r * (fk[k] + dot[k]) * sigm(kr));
        const float c = -r * kap[k] / nrm[k];
        g[5 * k + 0] = gscale * c * (x0 - dot[k] * mu[k][0]);
        g[5 * k + 1] = gscale * c * (x1 - dot[k] * mu[k][1]);
        g[5 * k + 2] = gscale * c * (x2 - dot[k] * mu[k][2]);
    }
}

__global__ void mlp_adam_kernel(float *p, const float *__restrict__ g, float *m, float *v, long long n, float lr,
                                float b1, float b2, float eps, float c1, float c2) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const float gg = g[e];
        const float mm = b1 * m[e] + (1.0f - b1) * gg;
        const float vv = b2 * v[e] + (1.0f - b2) * gg * gg;
        m[e] = mm;
        v[e] = vv;
        p[e] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    }
}

// ---- fused inference: weights in shared memory, one warp per sample
// params layout (floats): W1[128x48] b1[128] W2[128x128] b2 W3[128x128] b3 W4[40x128] b4[40]
constexpr int kMlpW1 = kMlpHid * kMlpIn, kMlpW2 = kMlpHid * kMlpHid, kMlpW4 = kMlpOut * kMlpHid;
constexpr int kMlpParams = kMlpW1 + kMlpHid + 2 * (kMlpW2 + kMlpHid) + kMlpW4 + kMlpOut;

__global__ void __launch_bounds__(256, 1)
    mlp_infer_kernel(const float *__restrict__ params, const float *__restrict__ X, int B, float *__restrict__ Y) {
    extern __shared__ float sm[];
    // transposed weights: Wt[l][i][o]
    float *w1 = sm, *w2 = w1 + kMlpW1, *w3 = w2 + kMlpW2, *w4 = w3 + kMlpW2;
    float *bias = w4 + kMlpW4;  // b1 b2 b3 b4
    float *act = bias + 3 * kMlpHid + kMlpOut;  // per warp 2 x 128
    const float *P1 = params, *B1 = P1 + kMlpW1, *P2 = B1 + kMlpHid, *B2 = P2 + kMlpW2, *P3 = B2 + kMlpHid;
    const float *B3 = P3 + kMlpW2, *P4 = B3 + kMlpHid, *B4 = P4 + kMlpW4;
    for (int e = threadIdx.x; e < kMlpW1; e += blockDim.x) w1[(e % kMlpIn) * kMlpHid + e / kMlpIn] = P1[e];
    for (int e = threadIdx.x; e < kMlpW2; e += blockDim.x) {
        w2[(e % kMlpHid) * kMlpHid + e / kMlpHid] = P2[e];
        w3[(e % kMlpHid) * kMlpHid + e / kMlpHid] = P3[e];
    }
    for (int e = threadIdx.x; e < kMlpW4; e += blockDim.x) w4[(e % kMlpHid) * kMlpOut + e / kMlpHid] = P4[e];
    for (int e = threadIdx.x; e < kMlpHid; e += blockDim.x) {
        bias[e] = B1[e];
        bias[kMlpHid + e] = B2[e];
        bias[2 * kMlpHid + e] = B3[e];
    }
    for (int e = threadIdx.x; e < kMlpOut; e += blockDim.x) bias[3 * kMlpHid + e] = B4[e];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    float *a0 = act + warp * 2 * kMlpHid, *a1 = a0 + kMlpHid;
    for (int i = blockIdx.x * nw + warp; i < B; i += gridDim.x * nw) {
        for (int q = lane; q < kMlpIn; q += 32) a0[q] = X[(size_t)i * kMlpIn + q];
        __syncwarp();
        const float *wl[3] = {w1, w2, w3};
        const int nin[3] = {kMlpIn, kMlpHid, kMlpHid};
        float *src = a0, *dst = a1;
        for (int l = 0; l < 3; l++) {
            float o[4];
#pragma unroll
            for (int j = 0; j < 4; j++) o[j] = bias[l * kMlpHid + lane + 32 * j];
            for (int q = 0; q < nin[l]; q++) {
                const float x = src[q];
#pragma unroll
                for (int j = 0; j < 4; j++) o[j] = fmaf(x, wl[l][q * kMlpHid + lane + 32 * j], o[j]);
            }
            __syncwarp();
#pragma unroll
            for (int j = 0; j < 4; j++) dst[lane + 32 * j] = o[j] * sigm(o[j]);
            __syncwarp();
            float *tmp = src;
            src = dst;
            dst = tmp;
        }
        for (int j = 0; j < 2; j++) {
            const int oo = lane + 32 * j;
            if (oo < kMlpOut) {
                float o = bias[3 * kMlpHid + oo];
                for (int q = 0; q < kMlpHid; q++) o = fmaf(src[q], w4[q * kMlpOut + oo], o);
                Y[(size_t)i * kMlpOut + oo] = o;
            }
        }
        __syncwarp();
    }
}

}  // namespace csl

using namespace csl;

// ---- C ABI (declared in include/gpustreamlines_b200.h); all pointers device memory
extern "C" int csl_mlp_gemm(int ta, int tb, int M, int N, int K, const float *A, int lda, const float *B, int ldb,
                            float *C, int ldc, float beta, void *stream) {
    if (M < 0 || N < 0 || K < 0 || !A || !B || !C) return -1;
    if (M == 0 || N == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    const dim3 grid((N + 63) / 64, (M + 63) / 64);
    if (ta && tb) mlp_gemm_kernel<true, true><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, beta);
    else if (ta) mlp_gemm_kernel<true, false><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, beta);
    else if (tb) mlp_gemm_kernel<false, true><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, beta);
    else mlp_gemm_kernel<false, false><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, beta);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

extern "C" int csl_mlp_bias_act(float *Z, const float *b, float *A, int M, int N, int act, void *stream) {
    if (!Z || !b || !A || M < 0 || N <= 0) return -1;
    if (M == 0) return 0;
    mlp_bias_act_kernel<<<1024, 256, 0, (cudaStream_t)stream>>>(Z, b, A, M, N, act);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

extern "C" int csl_mlp_act_bwd(const float *Z, const float *dA, float *dZ, long long n, void *stream) {
    if (!Z || !dA || !dZ || n < 0) return -1;
    if (n == 0) return 0;
    mlp_act_bwd_kernel<<<1024, 256, 0, (cudaStream_t)stream>>>(Z, dA, dZ, n);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

extern "C" int csl_mlp_colsum(const float *dZ, int M, int N, float *db, void *stream) {
    if (!dZ || !db || M < 0 || N <= 0) return -1;
    mlp_colsum_kernel<<<N, 256, 0, (cudaStream_t)stream>>>(dZ, M, N, db);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

extern "C" int csl_mlp_vmf_nll(const float *Y, const float *X, int B, float gscale, float *loss, float *dY,
                               void *stream) {
    if (!Y || !X || !loss || !dY || B < 0) return -1;
    if (B == 0) return 0;
    mlp_vmf_nll_kernel<<<(B + 127) / 128, 128, 0, (cudaStream_t)stream>>>(Y, X, B, gscale, loss, dY);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

extern "C" int csl_mlp_adam(float *p, const float *g, float *m, float *v, long long n, float lr, float b1, float b2,
                            float eps, int step, void *stream) {
    if (!p || !g || !m || !v || n < 0 || step < 1) return -1;
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    mlp_adam_kernel<<<1024, 256, 0, (cudaStream_t)stream>>>(p, g, m, v, n, lr, b1, b2, eps, c1, c2);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

extern "C" int csl_mlp_param_count(void) { return kMlpParams; }

extern "C" int csl_mlp_infer(const float *params, const float *X, int B, float *Y, float *ms_out, void *stream) {
    if (!params || !X || !Y || B < 0) return -1;
    if (B == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    const int smem = (kMlpW1 + 2 * kMlpW2 + kMlpW4 + 3 * kMlpHid + kMlpOut + 8 * 2 * kMlpHid) * 4;
    if (cudaFuncSetAttribute(mlp_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
        return -2;
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ms_out) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, st);
    }
    mlp_infer_kernel<<<nsm, 256, smem, st>>>(params, X, B, Y);
    cudaError_t e = cudaGetLastError();
    if (ms_out) {
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(ms_out, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    return e == cudaSuccess ? 0 : -2;
}
