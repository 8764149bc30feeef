// Streamline linearisation on the device (the step generic_tracker.py:139-144
// runs on the host through DIPY's compress_streamlines after to_world()).
//
//   world_kernel     voxel -> world coordinates, float64 affine, rounded to
//                    float32 (Tractogram.to_world)
//   mask_kernel      one warp per streamline: Presseau et al. 2015 greedy
//                    linearisation; the segment from the last kept point to
//                    point i is accepted while it is no longer than
//                    max_segment_length and every point between lies within
//                    tol_error of it; the lanes test the points between in
//                    parallel.  float32 arithmetic without contraction
//                    (__f*_rn), so the decisions equal the host restatement
//                    (gpustreamlines_b200/io.py: _compress_one) bit for bit
//   gather_kernel    kept points in order, compacted by a scan of the counts
// Streamlines outside [minlen, maxlen] points get no output (the chunk
// filter of SeedBatchPropagator).
#include <cuda_runtime.h>

#include "kernels.h"

namespace csl {

struct Affine34 {
    double m[12];  // rows of the upper 3x4 block
};

__global__ void world_kernel(const float *__restrict__ pts, long long npts, Affine34 A, float *__restrict__ out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npts;
         i += (long long)gridDim.x * blockDim.x) {
        const double x = pts[3 * i], y = pts[3 * i + 1], z = pts[3 * i + 2];
#pragma unroll
        for (int r = 0; r < 3; r++) {
            const double v = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, A.m[4 * r]), __dmul_rn(y, A.m[4 * r + 1])),
                                                 __dmul_rn(z, A.m[4 * r + 2])),
                                       A.m[4 * r + 3]);
            out[3 * i + r] = __double2float_rn(v);
        }
    }
}

__device__ __forceinline__ float3 ld3(const float *__restrict__ p, long long i) {
    return make_float3(__ldg(p + 3 * i), __ldg(p + 3 * i + 1), __ldg(p + 3 * i + 2));
}

__global__ void compress_mask_kernel(const float *__restrict__ w, const long long *__restrict__ off,
                                     const int *__restrict__ len, int nsl, int minlen, int maxlen, double tol2,
                                     double maxseg, unsigned char *__restrict__ keep, int *__restrict__ cnt) {
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x / 32;
    for (int sl = blockIdx.x * wpb + threadIdx.x / 32; sl < nsl; sl += gridDim.x * wpb) {
        const long long o = off[sl];
        const int n = len[sl];
        if (n < minlen || n > maxlen) {
            if (lane == 0) cnt[sl] = 0;
            continue;
        }
        if (n <= 2) {
            if (lane < n) keep[o + lane] = 1;
            if (lane == 0) cnt[sl] = n;
            continue;
        }
        int start = 0, c = 1;
        if (lane == 0) keep[o] = 1;
        for (int i = 2; i < n; i++) {
            const float3 a = ld3(w, o + start), b = ld3(w, o + i);
            const float3 ab = make_float3(__fsub_rn(b.x, a.x), __fsub_rn(b.y, a.y), __fsub_rn(b.z, a.z));
            const float L = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(ab.x, ab.x), __fmul_rn(ab.y, ab.y)),
                                                 __fmul_rn(ab.z, ab.z)));
            bool ok = (double)L <= maxseg;
            if (ok && i - start > 1) {
                float3 u = ab;
                if (L > 0.0f) u = make_float3(__fdiv_rn(ab.x, L), __fdiv_rn(ab.y, L), __fdiv_rn(ab.z, L));
                bool bad = false;
                for (int j = start + 1 + lane; j < i; j += 32) {
                    const float3 p = ld3(w, o + j);
                    const float3 m = make_float3(__fsub_rn(p.x, a.x), __fsub_rn(p.y, a.y), __fsub_rn(p.z, a.z));
                    float d2;
                    if (L > 0.0f) {
                        const float cx = __fsub_rn(__fmul_rn(m.y, u.z), __fmul_rn(m.z, u.y));
                        const float cy = __fsub_rn(__fmul_rn(m.z, u.x), __fmul_rn(m.x, u.z));
                        const float cz = __fsub_rn(__fmul_rn(m.x, u.y), __fmul_rn(m.y, u.x));
                        d2 = __fadd_rn(__fadd_rn(__fmul_rn(cx, cx), __fmul_rn(cy, cy)), __fmul_rn(cz, cz));
                    } else {
                        d2 = __fadd_rn(__fadd_rn(__fmul_rn(m.x, m.x), __fmul_rn(m.y, m.y)), __fmul_rn(m.z, m.z));
                    }
                    bad |= !((double)d2 <= tol2);
                }
                ok = __ballot_sync(0xffffffffu, bad) == 0u;
            }
            if (!ok) {
                if (lane == 0) keep[o + i - 1] = 1;
                c++;
                start = i - 1;
            }
        }
        if (lane == 0) {
            keep[o + n - 1] = 1;
            cnt[sl] = c + 1;
        }
    }
}

__global__ void compress_gather_kernel(const float *__restrict__ w, const long long *__restrict__ off,
                                       const int *__restrict__ len, const unsigned char *__restrict__ keep,
                                       const long long *__restrict__ coff, int nsl, float *__restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x / 32;
    const unsigned lmask = (1u << lane) - 1u;
    for (int sl = blockIdx.x * wpb + threadIdx.x / 32; sl < nsl; sl += gridDim.x * wpb) {
        const long long o = off[sl];
        const int n = len[sl];
        long long dst = coff[sl];
        if (coff[sl + 1] == dst) continue;
        for (int j0 = 0; j0 < n; j0 += 32) {
            const int j = j0 + lane;
            const bool k = j < n && keep[o + j];
            const unsigned m = __ballot_sync(0xffffffffu, k);
            if (k) {
                const long long d = dst + __popc(m & lmask);
                out[3 * d] = w[3 * (o + j)];
                out[3 * d + 1] = w[3 * (o + j) + 1];
                out[3 * d + 2] = w[3 * (o + j) + 2];
            }
            dst += __popc(m);
        }
    }
}

cudaError_t launch_compress(const float *pts, long long npts, const double *affine16, const long long *off,
                            const int *len, int nsl, int minlen, int maxlen, double tol, double maxseg, float *world,
                            unsigned char *keep, int *cnt, cudaStream_t st) {
    Affine34 A{};
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 4; c++) A.m[4 * r + c] = affine16 ? affine16[4 * r + c] : (r == c ? 1.0 : 0.0);
    if (npts > 0) {
        world_kernel<<<1024, 256, 0, st>>>(pts, npts, A, world);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        e = cudaMemsetAsync(keep, 0, (size_t)npts, st);
        if (e != cudaSuccess) return e;
    }
    if (nsl > 0) {
        compress_mask_kernel<<<2048, 256, 0, st>>>(world, off, len, nsl, minlen, maxlen, tol * tol, maxseg, keep,
                                                    cnt);
    }
    return cudaGetLastError();
}

cudaError_t launch_compress_gather(const float *world, const long long *off, const int *len,
                                   const unsigned char *keep, const long long *coff, int nsl, float *out,
                                   cudaStream_t st) {
    if (nsl > 0) compress_gather_kernel<<<2048, 256, 0, st>>>(world, off, len, keep, coff, nsl, out);
    return cudaGetLastError();
}

}  // namespace csl
