// Exact rejection sampler of the probabilistic getter's target distribution
// with a proposal bounded by per-voxel vertex-cluster maxima.
//
// Target (get_direction_prob_d, generate_streamlines_cuda.cu:54-275): vertex v
// with probability proportional to
//     p(v) = P(v) * [P(v) >= thr] * [v in the cone of the incoming direction],
// P the trilinearly interpolated PMF and thr = PMF_THRESHOLD_P * max_u P(u).
// The reference builds the inverse CDF over all V vertices, which needs the 8
// corner rows of the PMF (8 x 724 x 4 B = 23 KB per step at V = 724).
//
// This sampler reads a per-voxel table instead.  The sphere's vertices are
// partitioned into K = 64 compact clusters C_k (at most 32 vertices each);
// the table holds, per voxel x and cluster k, M_x(k) = max over v in C_k of
// pmf_x(v), rounded up to bfloat16 (64 clusters = one 128-byte line per
// voxel, an 84 MB table at 81x106x76 voxels that stays in L2).  With the
// corner weights w_q >= 0 and the same fused multiply-add chain as P(v),
//     U(k) = fma(M_x7(k), w_7, ... fma(M_x0(k), w_0, 0))  >=  P(v)  for v in C_k,
// because round-to-nearest is monotone.  Let n(k) = |C_k within the cone|.
//   1. propose cluster k with probability U(k) n(k) / Z, Z = sum_k U(k) n(k),
//      then v uniformly among the n(k) cone members of C_k: q(v) = U(k) / Z;
//   2. evaluate P(v) exactly (8 scattered loads) and accept with probability
//      p(v) / U(k) = p(v) / (Z q(v)) <= 1.
// Accepted draws are distributed as p, exactly (von Neumann's rejection
// method).  The threshold needs the maximum of P over ALL vertices, which the
// sampler brackets: max_k U(k) >= max P >= every P(v) evaluated so far.  When
// a proposal can be accepted and the bracket does not decide whether
// P(v) >= thr, the corner rows are gathered after all and the maximum is made
// exact (a lazily evaluated acceptance test of the same draw, so still exact).
// After kEnvMaxTrials rejected proposals -- or when Z is not a positive finite
// number -- the step finishes with the reference's inverse-CDF sampler on the
// gathered rows; the sampler's output does not depend on how many proposals
// were rejected before it, so this switch leaves the distribution unchanged.
// Per step the sampler reads 1 KB of table, a 256 B cone-bit row and 8 PMF
// values per proposal (about 1.8 proposals per accepted step on the 81x106x76
// phantom) instead of 23 KB.  Four proposals are evaluated at once, one per
// group of 8 lanes, and taken in draw order.
//
// Random numbers: the proposals read a Philox stream of their own per seed
// (three uniforms per proposal); the inverse-CDF fallback draws from lane 0's
// stream, as the plain sampler does.  Streamlines are therefore not identical
// to the plain path's, only identically distributed.
#pragma once
#include "common.cuh"
#include "kernels.h"
#include "prob.cuh"

namespace csl {

constexpr int kEnvMaxTrials = 16;

__device__ __forceinline__ float fma_ftz(float a, float b, float c) {
    float d;
    asm("fma.rn.ftz.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float bf16_low(uint32_t x) { return __uint_as_float(x << 16); }
__device__ __forceinline__ float bf16_high(uint32_t x) { return __uint_as_float(x & 0xffff0000u); }

// Per-warp counters, kept by lane 0 and flushed once per warp.
struct EnvCount {
    unsigned long long steps, proposals, resolves, fallbacks;
};

// Loads of one step: lane l holds the table words of clusters 2l and 2l+1 for
// the 8 corners and the cone bits of the same two clusters.
struct EnvLoads {
    uint32_t m[8];
    uint2 cone;
};

__device__ __forceinline__ void env_issue(const DevParams &P, const int (&vox)[8], const DirState &dir, int lane,
                                          EnvLoads &L) {
#pragma unroll
    for (int q = 0; q < 8; q++) L.m[q] = __ldg(P.env_cmax + (size_t)vox[q] * kWarp + lane);
    L.cone = __ldg(reinterpret_cast<const uint2 *>(P.env_cone) +
                   ((size_t)(dir.neg * P.nvert + dir.vtx) * kWarp + lane));
}

// PMF value of vertex v at the interpolation point, bit-identical to the
// element the plain gather computes (same corner order, fma.rn.ftz chain).
__device__ __forceinline__ float env_pmf_at(const DevParams &P, const int (&vox)[8], const float (&w)[8], int v,
                                            int lane) {
    int myvox = vox[0];
#pragma unroll
    for (int q = 1; q < 8; q++)
        if (lane == q) myvox = vox[q];
    float d = 0.0f;
    if (lane < 8) d = __ldg(P.dataf + (size_t)myvox * P.dimt + v);
    float acc = 0.0f;
#pragma unroll
    for (int q = 0; q < 8; q++) acc = fma_ftz(__shfl_sync(FULL, d, q), w[q], acc);
    return acc;
}

// The plain path's full gather at the same point: interpolated rows into
// cdf_sh, returns the exact maximum.
__device__ __forceinline__ float env_gather(const DevParams &P, const int (&vox)[8], const float (&w)[8],
                                            float *cdf_sh, int lane) {
    Corners c;
#pragma unroll
    for (int q = 0; q < 8; q++) {
        c.base[q] = (long long)vox[q] * P.dimt;
        c.w[q] = w[q];
    }
    return warp_max_ref(prob_gather(P, c, cdf_sh, lane));
}

__device__ __forceinline__ void env_out(const DevParams &P, int v, const DirState &dir, DirState *out) {
    const float3 sv = vert3(P.verts, v);
    if ((dir.d.x * sv.x + dir.d.y * sv.y + dir.d.z * sv.z) > 0) {
        out->d = sv;
        out->neg = 0;
    } else {
        out->d = make_float3(-sv.x, -sv.y, -sv.z);
        out->neg = 1;
    }
    out->vtx = v;
}

// Proposal random numbers: a Philox stream of its own per seed (key
// rng_seed, subsequence kEnvSubseqBase + global seed index), read block by
// block: each round of kEnvGroups draws takes kEnvGroups blocks, block g
// giving draw g its three uniforms (cluster, member, acceptance).
constexpr unsigned long long kEnvSubseqBase = 1ull << 61;
constexpr int kEnvGroups = 4;  // draws evaluated together, 8 lanes each

struct EnvStream {
    unsigned long long sub;   // Philox subsequence (high 64 counter bits)
    unsigned long long nblk;  // blocks consumed (low 64 counter bits)
};

__device__ __forceinline__ uint4 env_block(const DevParams &P, const EnvStream &es, unsigned long long i) {
    const unsigned long long lo = es.nblk + i;
    const uint4 ctr = make_uint4((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)es.sub, (uint32_t)(es.sub >> 32));
    return philox4x32_10(ctr, make_uint2((uint32_t)P.rng_seed, (uint32_t)(P.rng_seed >> 32)));
}

// One direction.  `dir.vtx` must be a sphere vertex (always true along a
// streamline: initial directions are pass-1 peaks, later ones sampled
// vertices).  Draws are made kEnvGroups at a time (lane group g = lane / 8
// evaluates draw g) and taken in draw order, so the result is that of the
// sequential rejection sampler.
__device__ __forceinline__ int env_sample(const DevParams &P, const int (&vox)[8], const float (&w)[8],
                                          const EnvLoads &L, DirState dir, float *cdf_sh, PhiloxShared &rng,
                                          EnvStream &es, int lane, DirState *out, EnvCount &cnt) {
    // cluster bounds U(2l), U(2l+1)
    float u0 = 0.0f, u1 = 0.0f;
#pragma unroll
    for (int q = 0; q < 8; q++) {
        u0 = fma_ftz(bf16_low(L.m[q]), w[q], u0);
        u1 = fma_ftz(bf16_high(L.m[q]), w[q], u1);
    }
    const float mx_hi = warp_max_ref(fmax_ref(u0, u1));
    const float w0 = u0 * (float)__popc(L.cone.x);
    const float w1 = u1 * (float)__popc(L.cone.y);
    // cumulative proposal weights over clusters 0..63 (lane l: 2l, 2l+1)
    float s = w0 + w1;
#pragma unroll
    for (int i = 1; i < kWarp; i <<= 1) {
        const float y = __shfl_up_sync(FULL, s, i);
        if (lane >= i) s += y;
    }
    float ex = __shfl_up_sync(FULL, s, 1);
    if (lane == 0) ex = 0.0f;
    const float c1 = s;
    const float c0 = fminf(ex + w0, s);
    const float Z = __shfl_sync(FULL, s, 31);
    if (lane == 0) cnt.steps++;

    const float thr_hi = (float)(P.pmf_threshold * (double)mx_hi);
    const int grp = lane >> 3, q = lane & 7;
    int myvox = vox[0];
#pragma unroll
    for (int k = 1; k < 8; k++)
        if (q == k) myvox = vox[k];
    // proposals only when Z is a positive finite number
    int round = (Z > 0.0f && Z < FLT_MAX && mx_hi > 0.0f) ? 0 : kEnvMaxTrials / kEnvGroups;
    float lo = 0.0f;         // largest P(v) evaluated: max P >= lo
    bool gathered = false;   // corner rows gathered, exact maximum known
    float m_exact = 0.0f, thr_x = 0.0f;
    for (; round < kEnvMaxTrials / kEnvGroups; round++) {
        // draw g's uniforms from block g of this round (computed by lane 8g)
        uint4 blk = make_uint4(0u, 0u, 0u, 0u);
        if (q == 0) blk = env_block(P, es, (unsigned long long)grp);
        es.nblk += kEnvGroups;
        const float a = Philox::uint_to_uniform(__shfl_sync(FULL, blk.x, 0, 8));
        const float b = Philox::uint_to_uniform(__shfl_sync(FULL, blk.y, 0, 8));
        const float g = Philox::uint_to_uniform(__shfl_sync(FULL, blk.z, 0, 8));
        if (lane == 0) cnt.proposals += kEnvGroups;
        // cluster of each draw: first k whose cumulative weight reaches a * Z
        int src = 0;
        bool first = false;
#pragma unroll
        for (int d = 0; d < kEnvGroups; d++) {
            const float x = __shfl_sync(FULL, a, 8 * d) * Z;
            const unsigned bA = __ballot_sync(FULL, c0 >= x);
            const unsigned bB = __ballot_sync(FULL, c1 >= x);
            const int sd = bB ? __ffs(bB) - 1 : kWarp - 1;
            if (grp == d) {
                src = sd;
                first = (bA >> sd) & 1u;
            }
        }
        const float uA = __shfl_sync(FULL, u0, src), uB = __shfl_sync(FULL, u1, src);
        const unsigned mA = __shfl_sync(FULL, L.cone.x, src), mB = __shfl_sync(FULL, L.cone.y, src);
        const float uk = first ? uA : uB;
        const unsigned mk = first ? mA : mB;
        const int k = 2 * src + (first ? 0 : 1);
        // member: uniform among the cluster's cone members
        const int nk = __popc(mk);
        int r = (int)(b * (float)nk);
        if (r >= nk) r = nk - 1;
        const int pos = (nk > 0) ? (int)__fns(mk, 0u, r + 1) : 0;  // r-th set bit of mk (0-based r)
        const int v = (nk > 0) ? (int)__ldg(P.env_member + k * kEnvMaxMembers + pos) : -1;
        // P(v): lane 8g+q reads corner q, the group combines in corner order
        float dv = 0.0f;
        if (v >= 0) dv = __ldg(P.dataf + (size_t)myvox * P.dimt + v);
        float pv = 0.0f;
#pragma unroll
        for (int c = 0; c < 8; c++) pv = fma_ftz(__shfl_sync(FULL, dv, c, 8), w[c], pv);
        lo = fmax_ref(lo, warp_max_ref(v >= 0 ? pv : 0.0f));
        const bool take = v >= 0 && g * uk < pv;  // accepted if p(v) = P(v)
        const bool decided = gathered || !(pv < thr_hi) || pv < (float)(P.pmf_threshold * (double)lo);
        const bool keep = gathered ? !(pv < thr_x) : !(pv < thr_hi);
        const unsigned acc = __ballot_sync(FULL, q == 0 && decided && keep && take);
        const unsigned amb = __ballot_sync(FULL, q == 0 && !decided && take);
        const unsigned ev = acc | amb;
        if (ev == 0u) continue;
        int win = (__ffs(ev) - 1) >> 3;
        if ((amb >> (8 * win)) & 1u) {
            // the first event needs the exact threshold: gather the corner rows
            // and decide it and the draws after it in order
            m_exact = env_gather(P, vox, w, cdf_sh, lane);
            thr_x = (float)(P.pmf_threshold * (double)m_exact);
            gathered = true;
            if (lane == 0) cnt.resolves++;
            const unsigned acc2 = __ballot_sync(FULL, q == 0 && grp >= win && take && !(pv < thr_x));
            if (acc2 == 0u) continue;
            win = (__ffs(acc2) - 1) >> 3;
        }
        const int vw = __shfl_sync(FULL, v, 8 * win);
        env_out(P, vw, dir, out);
        return 1;
    }
    // inverse-CDF fallback on the gathered rows
    if (lane == 0) cnt.fallbacks++;
    if (!gathered) m_exact = env_gather(P, vox, w, cdf_sh, lane);
    return prob_finish(P, m_exact, dir, cdf_sh, rng, lane, out, nullptr);
}

// tracker_d for the probabilistic getter with the envelope sampler: the loop
// of prob_track (stop-map check of step i overlapped with the loads of step
// i + 1), same stopping rules and point layout.
__device__ __forceinline__ int prob_env_track(const DevParams &P, PhiloxShared &rng, EnvStream &es, float3 seed,
                                              DirState dir, float *out, float *cdf_sh, int lane, EnvCount &cnt) {
    float3 pt = seed;
    if (lane == 0) {
        out[0] = pt.x;
        out[1] = pt.y;
        out[2] = pt.z;
    }
    __syncwarp();
    const int imax = P.max_sline_len;
    float sval = 0.0f;
    bool pending = false;
    int i = 1;
    for (;;) {
        if (i >= imax) {
            if (pending && !((double)sval > P.tc_threshold)) i = i - 1;
            break;
        }
        int vox[8];
        float w[8];
        const bool inb = trilinear_vox(P, pt, vox, w);
        EnvLoads L;
        if (inb) env_issue(P, vox, dir, lane, L);
        if (pending) {
            pending = false;
            if (!((double)sval > P.tc_threshold)) {
                i = i - 1;
                break;
            }
        }
        if (!inb) break;
        DirState nd;
        if (!env_sample(P, vox, w, L, dir, cdf_sh, rng, es, lane, &nd, cnt)) break;
        dir = nd;
        pt.x = (float)fma((double)dir.d.x, P.step_size, (double)pt.x);
        pt.y = (float)fma((double)dir.d.y, P.step_size, (double)pt.y);
        pt.z = (float)fma((double)dir.d.z, P.step_size, (double)pt.z);
        if (lane == 0) {
            out[3 * i] = pt.x;
            out[3 * i + 1] = pt.y;
            out[3 * i + 2] = pt.z;
        }
        sval = tex3D<float>(P.stop_tex, pt.z, pt.y, pt.x);
        pending = true;
        i++;
    }
    __syncwarp();
    return i;
}

__device__ __forceinline__ void env_flush(const DevParams &P, const EnvCount &cnt, int lane) {
    if (lane == 0 && P.env_stats && cnt.steps) {
        atomicAdd(P.env_stats + 0, cnt.steps);
        atomicAdd(P.env_stats + 1, cnt.proposals);
        atomicAdd(P.env_stats + 2, cnt.resolves);
        atomicAdd(P.env_stats + 3, cnt.fallbacks);
    }
}

}  // namespace csl
