// Tracking kernels and their launchers.
//
// Pass 1 (seed peaks, one warp per seed) and pass 2 (tracking) follow the
// reference's two-pass structure (cu_propagate_seeds.py:206-233), with the
// host-side Python scan replaced by device scans and the padded
// nSlines x 1002 x float3 output replaced by a point pool plus a final
// compaction, so only valid points are ever copied off the device.
//
// Pass 2 is a persistent kernel: one block per SM slot, each warp takes the
// next seed from an atomic queue, tracks every peak of that seed (backward,
// then forward, the RNG stream continuing across them as in
// genStreamlinesMerge*_k), reserves space in the pool with one atomicAdd
// and copies the streamline there.  Uneven streamline lengths therefore
// never idle a warp while work remains.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>

#include "boot.cuh"
#include "common.cuh"
#include "kernels.h"
#include "prob.cuh"
#include "ptt.cuh"
#include "track.cuh"

namespace csl {

__host__ int smem_bytes(const DevParams &P, int warps, bool track) {
    return (kMaxSortLayers * kWarp) * 4 + warps * warp_smem_floats(P, track) * 4;
}

// ---------------------------------------------------------------------------
// pass 1: initial directions per seed

template <int MODEL>
__global__ void __launch_bounds__(256) seed_peaks_kernel(DevParams P, const float *__restrict__ seeds,
                                                         int n, long long rng_base, const int *partner,
                                                         int *npeaks, short *peaks, int max_store) {
    extern __shared__ float smem[];
    int *partner_sh = reinterpret_cast<int *>(smem);
    load_partner(partner, partner_sh);
    __syncthreads();
    const int warp = threadIdx.x / kWarp, lane = threadIdx.x & 31;
    const WarpBufs W = carve(P, smem + kMaxSortLayers * kWarp, warp, false, nullptr);
    const int wpb = blockDim.x / kWarp;
    for (int s = blockIdx.x * wpb + warp; s < n; s += gridDim.x * wpb) {
        const float3 seed = make_float3(seeds[3 * s], seeds[3 * s + 1], seeds[3 * s + 2]);
        const unsigned long long gid = 32ull * (unsigned long long)(s + rng_base) + lane;
        const int np = seed_peaks_dispatch<MODEL>(P, seed, W, partner_sh, lane, gid);
        if (lane == 0) npeaks[s] = np;
        if (peaks)
            for (int k = lane; k < max_store; k += kWarp)
                peaks[(size_t)s * max_store + k] = (short)(k < np ? W.ind[k] : -1);
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// pass 2: tracking

// 30-bit Morton code of each seed's voxel (10 bits per axis)
__device__ __forceinline__ uint32_t spread3(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__global__ void morton_kernel(const float *__restrict__ seeds, int n, uint32_t *keys, int *vals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t c[3];
    for (int a = 0; a < 3; a++) {
        const float f = floorf(seeds[3 * i + a] + 0.5f);
        c[a] = (f != f || f < 0.0f) ? 0u : (f > 1023.0f ? 1023u : (uint32_t)f);
    }
    keys[i] = spread3(c[0]) | (spread3(c[1]) << 1) | (spread3(c[2]) << 2);
    vals[i] = i;
}

__global__ void block_ranges_kernel(int n, int nblocks, int *next, int *end) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblocks) return;
    next[b] = (int)((long long)n * b / nblocks);
    end[b] = (int)((long long)n * (b + 1) / nblocks);
}

// ---------------------------------------------------------------------------
// post-processing: gather pool -> compacted, ordered points

__global__ void gather_kernel(const float *__restrict__ pool, const long long *__restrict__ src,
                              const int *__restrict__ len, const long long *__restrict__ pt_off,
                              int nsl, float *__restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x / kWarp;
    for (int sl = blockIdx.x * wpb + threadIdx.x / kWarp; sl < nsl; sl += gridDim.x * wpb) {
        const long long s = src[sl];
        const int n3 = 3 * len[sl];
        const float *a = pool + 3 * s;
        float *b = out + 3 * pt_off[sl];
        for (int j = lane; j < n3; j += kWarp) b[j] = a[j];
    }
}

// ---------------------------------------------------------------------------
// tables and constants

// keep-bit table of the probabilistic cone filter: bit (32c + l) of row
// (sign, k) is set when vertex 32c+l survives `dot < cos(max_angle)` for the
// incoming direction (-1)^sign * vertex k (generate_streamlines_cuda.cu:141-152)
__global__ void cone_mask_kernel(DevParams P, uint32_t *mask) {
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x * (blockDim.x / kWarp) + threadIdx.x / kWarp;
    if (row >= 2 * P.nvert) return;
    const int neg = row / P.nvert, k = row % P.nvert;
    float3 d = vert3(P.verts, k);
    if (neg) d = make_float3(-d.x, -d.y, -d.z);
    const float cos_similarity = P.cos_max_angle;
    for (int ch = 0; ch < P.nch; ch++) {
        const int t = ch * kWarp + lane;
        bool keep = false;
        if (t < P.samplm_nr) {
            const float3 sv = vert3(P.verts, t);
            float dot = d.x * sv.x + d.y * sv.y + d.z * sv.z;
            if (P.sphere_symm) dot = fabsf(dot);
            keep = !(dot < cos_similarity);
        }
        const unsigned b = __ballot_sync(FULL, keep);
        if (lane == 0) mask[(size_t)row * P.nch + ch] = b;
    }
}

// the same keep bits transposed per lane: word (row, l) bit ch = vertex 32*ch+l
__global__ void cone_mask_t_kernel(DevParams P, const uint32_t *mask, uint32_t *mask_t) {
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x * (blockDim.x / kWarp) + threadIdx.x / kWarp;
    if (row >= 2 * P.nvert) return;
    uint32_t bits = 0u;
    for (int ch = 0; ch < P.nch; ch++)
        bits |= ((mask[(size_t)row * P.nch + ch] >> lane) & 1u) << ch;
    mask_t[(size_t)row * kWarp + lane] = bits;
}

__global__ void device_cos_kernel(float a, float b, float *out) {
    out[0] = __cosf(a);
    out[1] = __cosf(b);
}

__global__ void philox_stream_kernel(unsigned long long seed, unsigned long long subseq,
                                     unsigned long long offset, long long n, unsigned *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Philox g;
    g.init(seed, subseq, offset);
    for (long long i = 0; i < n; i++) out[i] = g.next();
}

// One direction-getter call per query (test entry point).  Query q runs on
// warp q; lane l uses Philox subsequence subseq[q] + l at offset offs[q]
// (the reference's per-lane streams), lane 0's draws are counted.
template <int MODEL>
__global__ void get_direction_kernel(DevParams P, const int *partner, const float *pts,
                                     const float *dirs, const unsigned long long *subseq,
                                     const unsigned long long *offs, int n, float *frames,
                                     float *out_dirs, int *out_ok, int *out_draws) {
    extern __shared__ float smem[];
    int *partner_sh = reinterpret_cast<int *>(smem);
    load_partner(partner, partner_sh);
    __syncthreads();
    const int warp = threadIdx.x / kWarp, lane = threadIdx.x & 31;
    const WarpBufs W = carve(P, smem + kMaxSortLayers * kWarp, warp, false, nullptr);
    const int q = blockIdx.x * (blockDim.x / kWarp) + warp;
    if (q >= n) return;
    const float3 pt = make_float3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
    DirState d{make_float3(dirs[3 * q], dirs[3 * q + 1], dirs[3 * q + 2]), -1, 0};
    typename RngOf<MODEL>::T rng;
    if constexpr (MODEL == PROB) rng.st = W.rng;
    rng.init(P.rng_seed, subseq[q] + lane, offs[q]);
    DirState nd;
    nd.d = d.d;
    nd.vtx = -1;
    nd.neg = 0;
    int ok = 0, draws = 0;
    if constexpr (MODEL == PROB) {
        ok = prob_get_direction(P, pt, d, W.odf, rng, lane, &nd, &draws);
    } else if constexpr (MODEL == PTT) {
        if (lane < 9) W.frame[lane] = frames[9 * q + lane];
        __syncwarp();
        ok = ptt_step_direction<false>(P, rng, d.d, W.frame, pt, W.face, lane, &nd.d);
        __syncwarp();
        if (lane < 9) frames[9 * q + lane] = W.frame[lane];
    } else {
        BootSmem S{W.vox, W.msk, W.r, W.h, W.ind};
        ok = boot_get_direction<5, MODEL>(P, rng, d.d, pt, S, partner_sh, lane, &nd.d, &draws);
    }
    if (lane == 0) {
        out_dirs[3 * q] = nd.d.x;
        out_dirs[3 * q + 1] = nd.d.y;
        out_dirs[3 * q + 2] = nd.d.z;
        out_ok[q] = ok;
        if (out_draws) out_draws[q] = draws;
    }
}

// ODF of one bootstrap fit at given points with given resample indices, in
// the per-warp FP32 arithmetic of the tracking path (boot_get_direction up
// to the sphere sampling; boot.cu:393-560): the plain-fit side of the
// accuracy measurement.  One warp per point; rows of length vstride.
template <int MODEL>
__global__ void boot_odf_plain_kernel(DevParams P, const float *pts, const int *idx, int n, float *odf,
                                      int vstride) {
    extern __shared__ float smem[];
    const int warp = threadIdx.x / kWarp, lane = threadIdx.x & 31;
    const WarpBufs W = carve(P, smem + kMaxSortLayers * kWarp, warp, false, nullptr);
    const int q = blockIdx.x * (blockDim.x / kWarp) + warp;
    if (q >= n) return;
    const int T = P.dimt, hr = P.hr_side, nr = P.samplm_nr;
    const float3 point = make_float3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
    Corners c;
    const bool inb = trilinear_setup(P, point, c);
    float *out = odf + (size_t)q * vstride;
    if (!inb) {
        for (int j = lane; j < nr; j += kWarp) out[j] = 0.0f;
        return;
    }
    for (int t = lane; t < T; t += kWarp) W.vox[t] = trilinear_elem(P.dataf, c, t);
    __syncwarp();
    mask_get(T, P.b0s_mask, W.vox, W.msk, lane);
    __syncwarp();
    ndotp_rows<0>(hr, hr, W.msk, P.R, W.r, lane);
    ndotp_rows<0>(hr, hr, W.msk, P.H, W.h, lane);
    __syncwarp();
    for (int j = lane; j < hr; j += kWarp) W.h[j] += W.r[idx[(size_t)q * hr + j]];
    __syncwarp();
    mask_put(T, P.b0s_mask, W.h, W.vox, lane);
    __syncwarp();
    for (int j = lane; j < T; j += kWarp) {
        const float x = W.vox[j];
        W.vox[j] = (P.min_signal > x) ? P.min_signal : x;
    }
    __syncwarp();
    const float denom = avg_mask(T, P.b0s_mask, W.vox, lane);
    for (int j = lane; j < T; j += kWarp) W.vox[j] /= denom;
    __syncwarp();
    mask_get(T, P.b0s_mask, W.vox, W.msk, lane);
    __syncwarp();
    if (MODEL == OPDT) {
        ndotp_rows<1>(P.delta_nr, hr, W.msk, P.delta_q, W.r, lane);
        ndotp_rows<0>(P.delta_nr, hr, W.msk, P.delta_b, W.h, lane);
        __syncwarp();
        for (int j = lane; j < P.delta_nr; j += kWarp) W.r[j] -= W.h[j];
        __syncwarp();
    } else {
        ndotp_rows<2>(P.delta_nr, hr, W.msk, P.delta_q, W.r, lane);
        __syncwarp();
        if (lane == 0) W.r[0] = kN0Const;
        __syncwarp();
    }
    ndotp_rows<0>(nr, P.delta_nr, W.r, P.sampling, W.h, lane);
    __syncwarp();
    for (int j = lane; j < nr; j += kWarp) out[j] = W.h[j];
}

// ---------------------------------------------------------------------------
// launchers

#define CSL_DISPATCH_MODEL(model, ...)                      \
    switch (model) {                                         \
        case OPDT: { constexpr int M = OPDT; __VA_ARGS__; } break;  \
        case CSA: { constexpr int M = CSA; __VA_ARGS__; } break;    \
        case PROB: { constexpr int M = PROB; __VA_ARGS__; } break;  \
        default: { constexpr int M = PTT; __VA_ARGS__; } break;     \
    }

template <typename K>
static cudaError_t set_smem(K kernel, int bytes) {
    return raise_smem_limit(kernel, bytes);
}

cudaError_t launch_seed_peaks(const DevParams &P, const float *seeds, int n, long long rng_base,
                              const int *partner, int *npeaks, short *peaks, int max_store,
                              int grid, int block, cudaStream_t st) {
    const int smem = smem_bytes(P, block / kWarp, false);
    cudaError_t e = cudaSuccess;
    CSL_DISPATCH_MODEL(P.model, {
        e = set_smem(seed_peaks_kernel<M>, smem);
        if (e != cudaSuccess) return e;
        seed_peaks_kernel<M><<<grid, block, smem, st>>>(P, seeds, n, rng_base, partner, npeaks,
                                                        peaks, max_store);
    });
    return cudaGetLastError();
}

cudaError_t track_occupancy(const DevParams &P, int block, int *blocks_per_sm) {
    if (P.env) return track_occupancy_env(P, block, blocks_per_sm);
    const int smem = smem_bytes(P, block / kWarp, true);
    cudaError_t e = cudaSuccess;
    CSL_DISPATCH_MODEL(P.model, {
        e = set_smem(track_kernel<M>, smem);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, track_kernel<M>, block,
                                                          smem);
    });
    return e;
}

cudaError_t launch_track(const DevParams &P, const BatchArgs &B, const int *partner,
                         const int *npeaks, const short *peaks, int max_store, const int *sl_off,
                         int *out_len, int *out_seed, long long *out_src, int grid, int block,
                         cudaStream_t st) {
    if (P.env)
        return launch_track_env(P, B, partner, npeaks, peaks, max_store, sl_off, out_len, out_seed, out_src,
                                grid, block, st);
    const int smem = smem_bytes(P, block / kWarp, true);
    cudaError_t e = cudaSuccess;
    CSL_DISPATCH_MODEL(P.model, {
        e = set_smem(track_kernel<M>, smem);
        if (e != cudaSuccess) return e;
        track_kernel<M><<<grid, block, smem, st>>>(P, B, partner, npeaks, peaks, max_store, sl_off,
                                                   out_len, out_seed, out_src);
    });
    return cudaGetLastError();
}

cudaError_t launch_get_direction(const DevParams &P, const int *partner, const float *pts,
                                 const float *dirs, const unsigned long long *subseq,
                                 const unsigned long long *offs, int n, float *frames,
                                 float *out_dirs, int *out_ok, int *out_draws, cudaStream_t st) {
    const int block = 128;
    const int smem = smem_bytes(P, block / kWarp, false);
    const int grid = (n + 3) / 4;
    cudaError_t e = cudaSuccess;
    CSL_DISPATCH_MODEL(P.model, {
        e = set_smem(get_direction_kernel<M>, smem);
        if (e != cudaSuccess) return e;
        get_direction_kernel<M><<<grid, block, smem, st>>>(P, partner, pts, dirs, subseq, offs, n,
                                                           frames, out_dirs, out_ok, out_draws);
    });
    return cudaGetLastError();
}

cudaError_t launch_gather(const float *pool, const long long *src, const int *len,
                          const long long *pt_off, int nsl, float *out, int grid, cudaStream_t st) {
    if (nsl <= 0) return cudaSuccess;
    gather_kernel<<<grid, 256, 0, st>>>(pool, src, len, pt_off, nsl, out);
    return cudaGetLastError();
}

cudaError_t launch_cone_mask(const DevParams &P, uint32_t *mask, uint32_t *mask_t, cudaStream_t st) {
    const int rows = 2 * P.nvert;
    cone_mask_kernel<<<(rows + 7) / 8, 256, 0, st>>>(P, mask);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    cone_mask_t_kernel<<<(rows + 7) / 8, 256, 0, st>>>(P, mask, mask_t);
    return cudaGetLastError();
}

cudaError_t launch_device_cos(float a, float b, float *out, cudaStream_t st) {
    device_cos_kernel<<<1, 1, 0, st>>>(a, b, out);
    return cudaGetLastError();
}

cudaError_t launch_philox_stream(unsigned long long seed, unsigned long long subseq,
                                 unsigned long long offset, long long n, unsigned *out,
                                 cudaStream_t st) {
    philox_stream_kernel<<<1, 32, 0, st>>>(seed, subseq, offset, n, out);
    return cudaGetLastError();
}

// temporary storage for an n-element exclusive scan (either output type)
cudaError_t spatial_order(const float *seeds, int n, int nblocks, uint32_t *keys, uint32_t *keys_sorted,
                          int *vals, int *perm, int *blk_next, int *blk_end, void *tmp,
                          size_t *tmp_bytes, cudaStream_t st) {
    if (!tmp) {
        return cub::DeviceRadixSort::SortPairs(nullptr, *tmp_bytes, keys, keys_sorted, vals, perm, n, 0,
                                               30, st);
    }
    morton_kernel<<<(n + 255) / 256, 256, 0, st>>>(seeds, n, keys, vals);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = cub::DeviceRadixSort::SortPairs(tmp, *tmp_bytes, keys, keys_sorted, vals, perm, n, 0, 30, st);
    if (e != cudaSuccess) return e;
    block_ranges_kernel<<<(nblocks + 255) / 256, 256, 0, st>>>(n, nblocks, blk_next, blk_end);
    return cudaGetLastError();
}

cudaError_t scan_temp_bytes(int n, size_t *bytes) {
    size_t a = 0, b = 0;
    cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, a, (const int *)nullptr, (int *)nullptr, n);
    if (e != cudaSuccess) return e;
    e = cub::DeviceScan::ExclusiveSum(nullptr, b, (const int *)nullptr, (long long *)nullptr, n);
    *bytes = a > b ? a : b;
    return e;
}

cudaError_t exclusive_scan_i32(void *tmp, size_t tmp_bytes, const int *in, int *out, int n,
                               cudaStream_t st) {
    cudaError_t e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, in, out, n, st);
    return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t exclusive_scan_i64(void *tmp, size_t tmp_bytes, const int *in, long long *out, int n,
                               cudaStream_t st) {
    cudaError_t e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, in, out, n, st);
    return e != cudaSuccess ? e : cudaGetLastError();
}

}  // namespace csl

namespace csl {
cudaError_t launch_boot_odf_plain(const DevParams &P, const float *pts, const int *idx, int n, float *odf,
                                  int vstride, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int block = 128;
    const int smem = smem_bytes(P, block / kWarp, false);
    const int grid = (n + 3) / 4;
    cudaError_t e;
    if (P.model == OPDT) {
        e = set_smem(boot_odf_plain_kernel<OPDT>, smem);
        if (e != cudaSuccess) return e;
        boot_odf_plain_kernel<OPDT><<<grid, block, smem, st>>>(P, pts, idx, n, odf, vstride);
    } else {
        e = set_smem(boot_odf_plain_kernel<CSA>, smem);
        if (e != cudaSuccess) return e;
        boot_odf_plain_kernel<CSA><<<grid, block, smem, st>>>(P, pts, idx, n, odf, vstride);
    }
    return cudaGetLastError();
}
}  // namespace csl
