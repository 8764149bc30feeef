// Allocation-free tracking entry point (csl_track_noalloc).
//
// Some callers cannot call cudaMalloc while they track: code running inside a
// host framework that owns all device memory through its own pool (and
// forbids other allocators), real-time pipelines that must not allocate after
// start-up, and callers whose allocation would synchronise the device in the
// middle of their own stream work.  For them this file provides a variant of
// the pass-2 tracking kernel that needs no allocation at all: the caller
// passes the seeds and the output buffers, and the per-warp scratch the
// tracking kernel needs (backward / forward point buffers, the peak list)
// lives in one file-scope static __device__ array of fixed size.
//
// The variant fuses the seed-peak search into the tracking kernel and writes
// seed-major fixed slots (seed s, peak k -> slot s * max_peaks + k) instead of
// the compacted, scanned output of csl_propagate, so it needs no scan buffer
// and no point pool.  Its streamlines are the same as csl_propagate's.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/gpustreamlines_b200.h"
#include "track.cuh"

namespace csl {

// Fixed capacity of the static scratch: 592 resident warps (148 SMs x 4),
// each with two 501-point buffers and a 1024-entry peak list -> 9.5 MiB,
// held by every GPU that loads the library until the process exits.
constexpr int kNoallocWarps = 592;
constexpr int kNoallocWarpsPerBlock = 4;
constexpr int kNoallocMaxLen = 501;
constexpr int kNoallocMaxVerts = 1024;
constexpr int kNoallocMaxPeaks = 32;
constexpr size_t kNoallocWarpFloats = (size_t)2 * kNoallocMaxLen * 3 + kNoallocMaxVerts;
constexpr size_t kNoallocCounterFloats = 64;
constexpr size_t kNoallocFloats = kNoallocWarps * kNoallocWarpFloats + kNoallocCounterFloats;

// internal accessors of the tracker handle (capi.cu)
int tracker_view(csl_tracker *t, DevParams *P, const int **partner, int *device);
int tracker_fail(csl_tracker *t, int code, const char *msg);

}  // namespace csl

static __device__ __align__(256) float g_noalloc_scratch[csl::kNoallocFloats];

namespace csl {

template <int MODEL>
__global__ void __launch_bounds__(kNoallocWarpsPerBlock * 32)
    track_noalloc_kernel(DevParams P, const float *__restrict__ seeds, int n, long long rng_base,
                         const int *partner, int max_peaks, float *scratch, int *counts_out,
                         int *lens_out, float *points_out) {
    extern __shared__ float smem[];
    int *partner_sh = reinterpret_cast<int *>(smem);
    load_partner(partner, partner_sh);
    __syncthreads();
    const int warp = threadIdx.x / kWarp, lane = threadIdx.x & 31;
    const size_t gwarp = (size_t)blockIdx.x * (blockDim.x / kWarp) + warp;
    float *scrB = scratch + gwarp * kNoallocWarpFloats;
    float *scrF = scrB + (size_t)kNoallocMaxLen * 3;
    int *plist = reinterpret_cast<int *>(scrF + (size_t)kNoallocMaxLen * 3);
    int *queue = reinterpret_cast<int *>(scratch + kNoallocWarps * kNoallocWarpFloats);
    const WarpBufs W = carve(P, smem + kMaxSortLayers * kWarp, warp, true, plist);
    const size_t slot_floats = (size_t)2 * P.max_sline_len * 3;
    EnvCount cnt = {0, 0, 0, 0};  // used only by the envelope sampler, which this kernel does not run
    EnvStream es{0ull, 0ull};

    for (;;) {
        int s = 0;
        if (lane == 0) s = atomicAdd(queue, 1);
        s = __shfl_sync(FULL, s, 0);
        if (s >= n) break;
        const float3 seed = make_float3(seeds[3 * s], seeds[3 * s + 1], seeds[3 * s + 2]);
        const unsigned long long gid = 32ull * (unsigned long long)(s + rng_base) + lane;
        const int np = seed_peaks_dispatch<MODEL>(P, seed, W, partner_sh, lane, gid);
        if (W.ind != plist)
            for (int k = lane; k < np; k += kWarp) plist[k] = W.ind[k];
        if (lane == 0) counts_out[s] = np;
        __syncwarp();
        typename RngOf<MODEL>::T rng;
        if constexpr (MODEL == PROB) rng.st = W.rng;
        rng.init(P.rng_seed, gid + 1, 0);
        const int ntrack = np < max_peaks ? np : max_peaks;
        for (int k = 0; k < ntrack; k++) {
            const int pv = plist[k];
            const float3 fs = vert3(P.verts, pv);
            int nB = 1, nF = 1, len = 1;
            bool single = false;
            if constexpr (MODEL == PTT) {
                if (!ptt_start_frames(P, rng, fs, seed, W.frame, W.face, lane)) single = true;
            }
            if (single) {
                if (lane == 0) store_pt(scrB, 0, seed);
            } else {
                DirState db{make_float3(-fs.x, -fs.y, -fs.z), pv, 1};
                DirState df{fs, pv, 0};
                nB = track_one<MODEL>(P, rng, seed, db, W.frame, scrB, W, partner_sh, lane, cnt, es);
                nF = track_one<MODEL>(P, rng, seed, df, W.frame + 9, scrF, W, partner_sh, lane, cnt, es);
                len = nB - 1 + nF;
            }
            __syncwarp();
            float *dst = points_out + ((size_t)s * max_peaks + k) * slot_floats;
            for (int j = lane; j < len; j += kWarp) {
                const float *p = (j < nB) ? scrB + 3 * (nB - 1 - j) : scrF + 3 * (j - nB + 1);
                dst[3 * j] = p[0];
                dst[3 * j + 1] = p[1];
                dst[3 * j + 2] = p[2];
            }
            if (lane == 0) lens_out[(size_t)s * max_peaks + k] = len;
            __syncwarp();
        }
    }
}

// per-device device address of the static scratch, looked up once
static std::mutex g_noalloc_mu;
static float *g_noalloc_ptr[64] = {nullptr};

static cudaError_t noalloc_scratch(int device, float **ptr) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
    if (!g_noalloc_ptr[device]) {
        cudaError_t e = cudaSetDevice(device);
        if (e != cudaSuccess) return e;
        float *p = nullptr;
        e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[device] = p;
    }
    *ptr = g_noalloc_ptr[device];
    return cudaSuccess;
}

}  // namespace csl

using namespace csl;

extern "C" int csl_track_noalloc(csl_tracker *t, const float *seeds_dev, long long n,
                                 long long rng_index_base, int max_peaks, int *counts_dev,
                                 int *lens_dev, float *points_dev, void *stream) {
    if (!t) return CSL_E_INVALID;
    DevParams P;
    const int *partner = nullptr;
    int device = 0;
    int rc = tracker_view(t, &P, &partner, &device);
    if (rc) return rc;
    if (n < 0 || n > (1ll << 30))
        return tracker_fail(t, CSL_E_INVALID, "csl_track_noalloc: n must be in [0, 2^30]");
    if (max_peaks < 1 || max_peaks > kNoallocMaxPeaks)
        return tracker_fail(t, CSL_E_INVALID, "csl_track_noalloc: max_peaks must be in [1, 32]");
    if (P.max_sline_len > kNoallocMaxLen)
        return tracker_fail(t, CSL_E_INVALID,
                            "csl_track_noalloc: max_sline_len above the static scratch limit (501)");
    if (P.samplm_nr > kNoallocMaxVerts)
        return tracker_fail(t, CSL_E_INVALID,
                            "csl_track_noalloc: more than 1024 sphere samples (static scratch limit)");
    if (n == 0) return CSL_OK;
    if (!seeds_dev || !counts_dev || !lens_dev || !points_dev)
        return tracker_fail(t, CSL_E_INVALID, "csl_track_noalloc: NULL buffer");
    float *scratch = nullptr;
    cudaError_t e = noalloc_scratch(device, &scratch);
    if (e == cudaSuccess) e = cudaSetDevice(device);
    if (e != cudaSuccess) return tracker_fail(t, CSL_E_CUDA, cudaGetErrorName(e));
    cudaStream_t st = (cudaStream_t)stream;
    // the queue counter starts at zero; everything else is written before it is read
    e = cudaMemsetAsync(scratch + kNoallocWarps * kNoallocWarpFloats, 0, sizeof(int), st);
    const int smem = smem_bytes(P, kNoallocWarpsPerBlock, true);
    const int grid = kNoallocWarps / kNoallocWarpsPerBlock;
    const int block = kNoallocWarpsPerBlock * 32;
#define CSL_NOALLOC_LAUNCH(M)                                                                    \
    do {                                                                                         \
        if (e == cudaSuccess)                                                                    \
            e = cudaFuncSetAttribute(track_noalloc_kernel<M>,                                    \
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, smem);         \
        if (e == cudaSuccess)                                                                    \
            track_noalloc_kernel<M><<<grid, block, smem, st>>>(P, seeds_dev, (int)n,             \
                                                               rng_index_base, partner,          \
                                                               max_peaks, scratch, counts_dev,   \
                                                               lens_dev, points_dev);            \
    } while (0)
    switch (P.model) {
        case OPDT: CSL_NOALLOC_LAUNCH(OPDT); break;
        case CSA: CSL_NOALLOC_LAUNCH(CSA); break;
        case PROB: CSL_NOALLOC_LAUNCH(PROB); break;
        default: CSL_NOALLOC_LAUNCH(PTT); break;
    }
#undef CSL_NOALLOC_LAUNCH
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return tracker_fail(t, CSL_E_CUDA, cudaGetErrorName(e));
    return CSL_OK;
}
