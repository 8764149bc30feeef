// Device building blocks of the tracking kernels, shared by the kernels that
// use global scratch (kernels.cu) and the allocation-free variant (noalloc.cu):
// per-warp shared-memory layout, pass-1 dispatch, and the per-direction
// tracking loop (tracker_d / tracker_boot_d of the reference).
#pragma once
#include "boot.cuh"
#include "common.cuh"
#include "kernels.h"
#include "prob.cuh"
#include "ptt.cuh"

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
    if (MODEL == PTT) return ptt_seed_peaks(P, seed, W.odf, W.ind, partner_sh, lane);
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

template <int MODEL>
struct RngOf {
    using T = Philox;
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
                         const int *partner_sh, int lane) {
    if constexpr (MODEL == PROB) return prob_track(P, rng, seed, dir, out, W.odf, lane);
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
        int ndir;
        if constexpr (MODEL == PROB) {
            ndir = prob_get_direction(P, pt, dir, W.odf, rng, lane, &nd, nullptr);
        } else if constexpr (MODEL == PTT) {
            PttSmem S{W.face, W.vpdf};
            ndir = ptt_get_direction<false>(P, rng, dir.d, frame, pt, S, lane, &nd.d);
        } else {
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


}  // namespace csl
