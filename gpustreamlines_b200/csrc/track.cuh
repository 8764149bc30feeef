// Device building blocks of the tracking kernels, shared by the kernels that
// use global scratch (kernels.cu) and the allocation-free variant (noalloc.cu):
// per-warp shared-memory layout, pass-1 dispatch, and the per-direction
// tracking loop (tracker_d / tracker_boot_d of the reference).
#pragma once
#include "boot.cuh"
#include "common.cuh"
#include "envelope.cuh"
#include "kernels.h"
#include "prob.cuh"
#include "ptt.cuh"

// resident 256-thread blocks per SM the probabilistic tracker is compiled for
#ifndef CSL_BOOT_MIN_BLOCKS
#define CSL_BOOT_MIN_BLOCKS 2
#endif
#ifndef CSL_PROB_MIN_BLOCKS
#define CSL_PROB_MIN_BLOCKS 4
#endif
#ifndef CSL_ENV_MIN_BLOCKS
#define CSL_ENV_MIN_BLOCKS 4
#endif
#ifndef CSL_PTT_MIN_BLOCKS
#define CSL_PTT_MIN_BLOCKS 2
#endif


namespace csl {

// ---------------------------------------------------------------------------
// shared-memory layout

struct WarpBufs {
    float *odf;     // [n32] ODF / PMF / CDF
    int *ind;       // [max(n32, samplm_nr)] peak flags / indices
    float *vox;     // BOOT [n32t]
    float *msk;     // BOOT [n32t]
    float *r;       // BOOT [rh]
    float *h;       // BOOT [rh]
    Philox *rng;    // PROB: lane 0's generator state
    float *frame;   // PTT [18]
    float *face;    // PTT [32]
    float *vpdf;    // PTT [32]
};

__host__ __device__ inline int round32(int x) { return (x + 31) / 32 * 32; }

// `track`: pass-2 layout, where PROB and PTT keep the (rarely used) peak
// index buffer in global scratch so more warps fit on an SM
__host__ __device__ inline int warp_smem_floats(const DevParams &P, bool track) {
    const int nr = round32(P.samplm_nr);
    if (P.model == OPDT || P.model == CSA) {
        const int n32t = round32(P.dimt);
        const int rh = n32t > nr ? n32t : nr;
        return 2 * n32t + 2 * rh + nr;
    }
    int f = track ? nr : 2 * nr;
    if (P.model == PTT) f += 18 + 32 + 32;
    if (P.model == PROB) f += 16;
    return f;
}

__device__ inline WarpBufs carve(const DevParams &P, float *base, int warp, bool track,
                                 int *global_ind) {
    WarpBufs b = {};
    float *p = base + (size_t)warp * warp_smem_floats(P, track);
    const int nr = round32(P.samplm_nr);
    if (P.model == OPDT || P.model == CSA) {
        const int n32t = round32(P.dimt);
        const int rh = n32t > nr ? n32t : nr;
        b.vox = p;
        b.msk = p + n32t;
        b.r = p + 2 * n32t;
        b.h = p + 2 * n32t + rh;
        b.ind = reinterpret_cast<int *>(p + 2 * n32t + 2 * rh);
        b.odf = b.h;
    } else {
        b.odf = p;
        const int f = track ? nr : 2 * nr;
        b.ind = track ? global_ind : reinterpret_cast<int *>(p + nr);
        if (P.model == PROB) b.rng = reinterpret_cast<Philox *>(p + f);
        if (P.model == PTT) {
            b.frame = p + f;
            b.face = b.frame + 18;
            b.vpdf = b.face + 32;
        }
    }
    return b;
}

__device__ inline void load_partner(const int *__restrict__ g, int *sh) {
    for (int i = threadIdx.x; i < kMaxSortLayers * kWarp; i += blockDim.x) sh[i] = g[i];
}

// ---------------------------------------------------------------------------
// pass 1: initial directions per seed

template <int MODEL>
__device__ __forceinline__ int seed_peaks_dispatch(const DevParams &P, float3 seed, const WarpBufs &W,
                                   const int *partner_sh, int lane, unsigned long long subseq) {
    if (MODEL == PROB) return prob_seed_peaks(P, seed, W.odf, W.ind, partner_sh, lane);
    if (MODEL == PTT) return ptt_seed_odf_peaks(P, seed, W.odf, W.ind, partner_sh, lane);
    // bootstrap: one attempt with the pass-1 stream (boot.cu:649)
    Philox rng;
    rng.init(P.rng_seed, subseq, 0);
    BootSmem S{W.vox, W.msk, W.r, W.h, W.ind};
    float3 unused;
    return boot_get_direction<1, MODEL>(P, rng, make_float3(0, 0, 0), seed, S, partner_sh, lane,
                                        &unused, nullptr);
}

// ---------------------------------------------------------------------------
// pass 2: tracking

// Template tag of the probabilistic tracker with the bounded-envelope sampler
// (P.model stays PROB; envelope.cuh).
constexpr int PROB_ENV = 4;
__host__ __device__ constexpr int base_model(int m) { return m == PROB_ENV ? PROB : m; }

template <int MODEL>
struct RngOf {
    using T = Philox;
};
template <>
struct RngOf<PROB_ENV> {
    using T = PhiloxShared;
};
template <>
struct RngOf<PROB> {
    using T = PhiloxShared;
};
template <>
struct RngOf<PTT> {
    using T = PhiloxN;
};

__device__ __forceinline__ void store_pt(float *out, int i, float3 p) {
    out[3 * i] = p.x;
    out[3 * i + 1] = p.y;
    out[3 * i + 2] = p.z;
}

// tracker_d / tracker_boot_d (generate_streamlines_cuda.cu:283-421, boot.cu:725-824)
template <int MODEL>
__device__ __forceinline__ int track_one(const DevParams &P, typename RngOf<MODEL>::T &rng, float3 seed,
                         DirState dir, float *frame, float *out, const WarpBufs &W,
                         const int *partner_sh, int lane, EnvCount &cnt, EnvStream &es) {
    if constexpr (MODEL == PROB) return prob_track(P, rng, seed, dir, out, W.odf, lane);
    if constexpr (MODEL == PROB_ENV) return prob_env_track(P, rng, es, seed, dir, out, W.odf, lane, cnt);
    const int step_frac = (MODEL == PTT) ? P.step_frac : 1;
    const double ss = P.step_size / step_frac;
    float3 pt = seed;
    if (lane == 0) store_pt(out, 0, pt);
    __syncwarp();
    int i;
    const int imax = P.max_sline_len * step_frac;
    for (i = 1; i < imax; i++) {
        DirState nd;
        nd.vtx = -1;
        nd.neg = 0;
        int ndir = 0;
        if constexpr (MODEL == PROB) {
            ndir = prob_get_direction(P, pt, dir, W.odf, rng, lane, &nd, nullptr);
        } else if constexpr (MODEL == PTT) {
            ndir = ptt_step_direction<false>(P, rng, dir.d, frame, pt, W.face, lane, &nd.d);
        } else if constexpr (MODEL == OPDT || MODEL == CSA) {
            BootSmem S{W.vox, W.msk, W.r, W.h, W.ind};
            ndir = boot_get_direction<5, MODEL>(P, rng, dir.d, pt, S, partner_sh, lane, &nd.d,
                                                nullptr);
        }
        __syncwarp();
        if (ndir == 0) break;
        dir = nd;
        pt.x = (float)fma((double)dir.d.x, ss, (double)pt.x);
        pt.y = (float)fma((double)dir.d.y, ss, (double)pt.y);
        pt.z = (float)fma((double)dir.d.z, ss, (double)pt.z);
        if (lane == 0 && (i % step_frac) == 0) store_pt(out, i / step_frac, pt);
        __syncwarp();
        if (check_point(P, pt) != TRACKPOINT) break;
    }
    int nsteps = i / step_frac;
    if (((i % step_frac) != 0) && i < step_frac * (P.max_sline_len - 1)) nsteps++;
    return nsteps;
}


// ---------------------------------------------------------------------------
// pass 2: the persistent tracking kernel

// Next seed for the calling warp (lane 0).  Input order: one global counter.
// Spatial order: the seeds are sorted by the Morton code of their voxel and
// each block owns a contiguous range of that order, so the warps of a block
// track neighbouring seeds at the same time and share voxel rows in L1; a
// block whose range is exhausted takes positions from the following blocks'
// ranges.  Every position is claimed exactly once; results do not depend on
// the order.
__device__ __forceinline__ int next_seed(const BatchArgs &B) {
    if (!B.perm) return atomicAdd(B.queue, 1);
    const int nb = gridDim.x;
    for (int k = 0; k < nb; k++) {
        const int b = (blockIdx.x + k) % nb;
        const int p = atomicAdd(B.blk_next + b, 1);
        if (p < B.blk_end[b]) return B.perm[p];
    }
    return B.nseeds;
}

template <int MODEL>
__global__ void __launch_bounds__(256, MODEL == PROB_ENV ? CSL_ENV_MIN_BLOCKS : MODEL == PROB ? CSL_PROB_MIN_BLOCKS
                                         : (MODEL == PTT ? CSL_PTT_MIN_BLOCKS : CSL_BOOT_MIN_BLOCKS)) track_kernel(DevParams P, BatchArgs B, const int *partner,
                                                    const int *__restrict__ npeaks,
                                                    const short *__restrict__ peaks, int max_store,
                                                    const int *__restrict__ sl_off, int *out_len,
                                                    int *out_seed, long long *out_src) {
    extern __shared__ float smem[];
    int *partner_sh = reinterpret_cast<int *>(smem);
    load_partner(partner, partner_sh);
    __syncthreads();
    const int warp = threadIdx.x / kWarp, lane = threadIdx.x & 31;
    const size_t gwarp = (size_t)blockIdx.x * (blockDim.x / kWarp) + warp;
    float *scrB = B.scratch + gwarp * (size_t)scratch_floats_per_warp(P);
    float *scrF = scrB + (size_t)P.max_sline_len * 3;
    int *plist = reinterpret_cast<int *>(scrF + (size_t)P.max_sline_len * 3);
    const WarpBufs W = carve(P, smem + kMaxSortLayers * kWarp, warp, true, plist);
    EnvCount cnt = {0, 0, 0, 0};

    for (;;) {
        int s = 0;
        if (lane == 0) s = next_seed(B);
        s = __shfl_sync(FULL, s, 0);
        if (s >= B.nseeds) {
            if constexpr (MODEL == PROB_ENV) env_flush(P, cnt, lane);
            break;
        }
        const int np = npeaks[s];
        if (np == 0) continue;
        const int base = sl_off[s];
        if (base + np > B.sl_cap) {
            if (lane == 0) atomicOr(B.status, ST_SLOT_OVERFLOW);
            continue;
        }
        const float3 seed = make_float3(B.seeds[3 * s], B.seeds[3 * s + 1], B.seeds[3 * s + 2]);
        const unsigned long long gid = 32ull * (unsigned long long)(s + B.rng_index_base) + lane;
        // peak list: stored by pass 1, or recomputed into this warp's scratch
        const short *stored = peaks + (size_t)s * max_store;
        if (np > max_store) {
            seed_peaks_dispatch<base_model(MODEL)>(P, seed, W, partner_sh, lane, gid);
            if (W.ind != plist)
                for (int k = lane; k < np; k += kWarp) plist[k] = W.ind[k];
        }
        __syncwarp();
        typename RngOf<MODEL>::T rng;
        if constexpr (base_model(MODEL) == PROB) rng.st = W.rng;
        rng.init(P.rng_seed, gid + 1, 0);
        EnvStream es{kEnvSubseqBase + (unsigned long long)(s + B.rng_index_base), 0ull};
        {
            for (int k = 0; k < np; k++) {
                const int pv = (np > max_store) ? plist[k] : (int)stored[k];
                const float3 fs = vert3(P.verts, pv);
                int len;
                int nB = 0, nF = 0;
                bool single = false;
                if constexpr (MODEL == PTT) {
                    if (!ptt_start_frames(P, rng, fs, seed, W.frame, W.face, lane)) single = true;
                }
                if (single) {
                    if (lane == 0) store_pt(scrB, 0, seed);
                    __syncwarp();
                    nB = 1;
                    nF = 1;
                    len = 1;
                } else {
                    DirState db{make_float3(-fs.x, -fs.y, -fs.z), pv, 1};
                    DirState df{fs, pv, 0};
                    nB = track_one<MODEL>(P, rng, seed, db, W.frame, scrB, W, partner_sh, lane, cnt, es);
                    nF = track_one<MODEL>(P, rng, seed, df, W.frame + 9, scrF, W, partner_sh, lane, cnt, es);
                    len = nB - 1 + nF;
                }
                __syncwarp();
                unsigned long long off = 0;
                if (lane == 0) off = atomicAdd(B.pool_count, (unsigned long long)len);
                off = __shfl_sync(FULL, off, 0);
                long long src = -1;
                if (off + (unsigned long long)len <= B.pool_cap) {
                    src = (long long)off;
                    float *dst = B.pool + off * 3;
                    for (int j = lane; j < len; j += kWarp) {
                        const float *p = (j < nB) ? scrB + 3 * (nB - 1 - j) : scrF + 3 * (j - nB + 1);
                        dst[3 * j] = p[0];
                        dst[3 * j + 1] = p[1];
                        dst[3 * j + 2] = p[2];
                    }
                } else if (lane == 0) {
                    atomicOr(B.status, ST_POOL_OVERFLOW);
                }
                if (lane == 0) {
                    out_len[base + k] = len;
                    out_seed[base + k] = s;
                    out_src[base + k] = src;
                }
                __syncwarp();
            }
        }
    }
}

}  // namespace csl
