// Probabilistic direction getter (generate_streamlines_cuda.cu:54-275).
//
// Per step: trilinear PMF gather (lane l owns vertices l, l+32, ...), absolute threshold at PMF_THRESHOLD_P * max, cone filter,
// reference-order inclusive scan, one Philox uniform drawn by lane 0, the
// reference's bisection + ballot search, and the hemisphere flip.
//
// The cone filter reads a precomputed keep-bit table (one 32-bit word per
// lane and step, bit c for vertex 32c + lane) instead of evaluating
// 3 * V multiply-adds per step: along a streamline the incoming direction is
// always +/- a sphere vertex (pass-1 peaks and every sampled step are
// vertices), and the table bits are produced on the device with the same dot
// product expression, so the filter is bit-identical.
#pragma once
#include <cstring>

#include "common.cuh"

namespace csl {

// Direction state along a streamline: the float3 plus, when it is exactly
// +/- a sphere vertex, that vertex and the sign (vtx < 0: arbitrary vector).
struct DirState {
    float3 d;
    int vtx;
    int neg;
};

// Two fused multiply-adds with flush-to-zero, one instruction (Blackwell
// packed FP32).  Each half rounds exactly as a scalar fma.rn.ftz.f32, the
// form the reference's fast-math build uses for `acc += w * d`.
__device__ __forceinline__ float2 ffma2_ftz(float2 a, float2 b, float2 c) {
    unsigned long long ra, rb, rc, rd;
    memcpy(&ra, &a, 8);
    memcpy(&rb, &b, 8);
    memcpy(&rc, &c, 8);
    asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(rd) : "l"(ra), "l"(rb), "l"(rc));
    float2 d;
    memcpy(&d, &rd, 8);
    return d;
}

// Gather the trilinearly interpolated PMF into cdf_sh, return the lane's max.
// Vector path: 128-bit loads (lane l owns float4 slots l, l+32, ...; every
// voxel row is 16-byte aligned when V % 4 == 0) and packed FMAs; the per-
// element order (corners in (i,j,k) order, acc = fma(w, d, acc)) is the
// reference's.  Slot offsets are compile-time, so each load is one
// instruction with an immediate offset.
__device__ __forceinline__ float prob_gather(const DevParams &P, const Corners &c, float *cdf_sh,
                                             int lane) {
    const int len = P.samplm_nr;
    float m = -FLT_MAX;
    if (P.vec4) {
        constexpr int kNJ = 8;  // up to 1024 vertices
        const int f4 = len >> 2;
        const float4 *rows[8];
#pragma unroll
        for (int q = 0; q < 8; q++) rows[q] = reinterpret_cast<const float4 *>(P.dataf + c.base[q]) + lane;
#pragma unroll
        for (int j = 0; j < kNJ; j++) {
            if (lane + 32 * j < f4) {
                float4 d[8];
#pragma unroll
                for (int q = 0; q < 8; q++) d[q] = __ldg(rows[q] + 32 * j);
                float2 lo = make_float2(0.0f, 0.0f), hi = make_float2(0.0f, 0.0f);
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    const float2 ww = make_float2(c.w[q], c.w[q]);
                    lo = ffma2_ftz(make_float2(d[q].x, d[q].y), ww, lo);
                    hi = ffma2_ftz(make_float2(d[q].z, d[q].w), ww, hi);
                }
                reinterpret_cast<float4 *>(cdf_sh)[lane + 32 * j] = make_float4(lo.x, lo.y, hi.x, hi.y);
                m = fmax_ref(fmax_ref(fmax_ref(fmax_ref(m, lo.x), lo.y), hi.x), hi.y);
            }
        }
    } else {
        const float *rows[8];
#pragma unroll
        for (int q = 0; q < 8; q++) rows[q] = P.dataf + c.base[q];
        for (int t = lane; t < len; t += kWarp) {
            float acc = 0.0f;
#pragma unroll
            for (int q = 0; q < 8; q++) acc += c.w[q] * __ldg(rows[q] + t);
            cdf_sh[t] = acc;
            m = fmax_ref(m, acc);
        }
    }
    return m;
}

__device__ __forceinline__ int prob_finish(const DevParams &P, float m, DirState dir,
                                           float *cdf_sh, PhiloxShared &rng, int lane,
                                           DirState *out, int *ndraws) {
    const int len = P.samplm_nr;
    const int nch = P.nch;
    m = warp_max_ref(m);
    const float thr = (float)(P.pmf_threshold * (double)m);
    __syncwarp();

    // threshold + cone filter + reference-order scan, chunk by chunk.  A chunk
    // whose 32 values are all zero scans to the carry in every position (each
    // addition adds an exact zero), so it is written without the shuffle tree.
    const uint32_t *row = (dir.vtx >= 0)
                              ? P.cone_mask + ((size_t)dir.neg * P.nvert + dir.vtx) * nch
                              : nullptr;
    // keep bits of this lane, one coalesced word: bit ch <=> vertex 32*ch + lane
    const uint32_t kbits_t = (dir.vtx >= 0)
        ? __ldg(P.cone_mask_t + ((size_t)dir.neg * P.nvert + dir.vtx) * kWarp + lane) : 0u;
    const float cos_similarity = P.cos_max_angle;
    float carry = 0.0f;
    for (int ch = 0; ch < nch; ch++) {
        const int t = ch * kWarp + lane;
        const bool valid = t < len;
        bool keep;
        if (row) {
            keep = (kbits_t >> ch) & 1u;
        } else {
            keep = true;
            if (valid) {
                const float3 sv = vert3(P.verts, t);
                float dot = dir.d.x * sv.x + dir.d.y * sv.y + dir.d.z * sv.z;
                if (P.sphere_symm) dot = fabsf(dot);
                keep = !(dot < cos_similarity);
            }
        }
        float x = 0.0f;
        if (keep && valid) {
            x = cdf_sh[t];
            if (x < thr) x = 0.0f;
        }
        if (__ballot_sync(FULL, x != 0.0f) == 0u) {
            if (valid) cdf_sh[t] = carry;
            continue;
        }
        if (lane == 0 && ch != 0) x = x + carry;
#pragma unroll
        for (int i = 1; i < kWarp; i <<= 1) {
            const float y = __shfl_up_sync(FULL, x, i);
            if (lane >= i && valid) x += y;
        }
        if (valid) cdf_sh[t] = x;
        carry = __shfl_sync(FULL, x, 31);
    }
    __syncwarp();
    const float last_cdf = cdf_sh[len - 1];
    if (last_cdf == 0) return 0;

    float sel = 0.0f;
    if (lane == 0) sel = rng.uniform() * last_cdf;
    sel = __shfl_sync(FULL, sel, 0);
    if (ndraws) *ndraws += 1;

    int low = 0, high = len - 1;
    while ((high - low) >= kWarp) {
        const int mid = (low + high) / 2;
        if (cdf_sh[mid] < sel)
            low = mid;
        else
            high = mid;
    }
    const bool b = (low + lane <= high) ? (sel < cdf_sh[low + lane]) : false;
    const unsigned msk = __ballot_sync(FULL, b);
    int ind = low + __ffs(msk) - 1;
    // The reference reads vertex[-1] in this (measure-zero) case; stay in bounds.
    if (ind < 0) ind = 0;
    __syncwarp();

    const float3 sv = vert3(P.verts, ind);
    if ((dir.d.x * sv.x + dir.d.y * sv.y + dir.d.z * sv.z) > 0) {
        out->d = sv;
        out->neg = 0;
    } else {
        out->d = make_float3(-sv.x, -sv.y, -sv.z);
        out->neg = 1;
    }
    out->vtx = ind;
    return 1;
}

__device__ __forceinline__ int prob_get_direction(const DevParams &P, float3 pt, DirState dir,
                                                  float *cdf_sh, PhiloxShared &rng, int lane,
                                                  DirState *out, int *ndraws) {
    Corners c;
    if (!trilinear_setup(P, pt, c)) return 0;
    const float m = prob_gather(P, c, cdf_sh, lane);
    return prob_finish(P, m, dir, cdf_sh, rng, lane, out, ndraws);
}

// One tracking direction of the probabilistic getter (tracker_d,
// generate_streamlines_cuda.cu:283-421) with the stop-map check of step i
// overlapped with the PMF gather of step i + 1: the texture fetch is issued,
// the next gather's loads go out, and only then is the check evaluated.  A
// stop discards the gathered values (no random number has been drawn yet),
// so points, counts and RNG consumption are exactly the sequential ones.
__device__ __forceinline__ int prob_track(const DevParams &P, PhiloxShared &rng, float3 seed, DirState dir,
                                          float *out, float *cdf_sh, int lane) {
    float3 pt = seed;
    if (lane == 0) { out[0] = pt.x; out[1] = pt.y; out[2] = pt.z; }
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
        Corners c;
        const bool inb = trilinear_setup(P, pt, c);
        float m = -FLT_MAX;
        if (inb) m = prob_gather(P, c, cdf_sh, lane);
        if (pending) {
            pending = false;
            // check_point_d: -1 (outside) and values <= the threshold both stop
            if (!((double)sval > P.tc_threshold)) { i = i - 1; break; }
        }
        if (!inb) break;
        DirState nd;
        if (!prob_finish(P, m, dir, cdf_sh, rng, lane, &nd, nullptr)) break;
        dir = nd;
        pt.x = (float)fma((double)dir.d.x, P.step_size, (double)pt.x);
        pt.y = (float)fma((double)dir.d.y, P.step_size, (double)pt.y);
        pt.z = (float)fma((double)dir.d.z, P.step_size, (double)pt.z);
        if (lane == 0) { out[3 * i] = pt.x; out[3 * i + 1] = pt.y; out[3 * i + 2] = pt.z; }
        sval = tex3D<float>(P.stop_tex, pt.z, pt.y, pt.x);
        pending = true;
        i++;
    }
    __syncwarp();
    return i;
}

// Pass-1 peaks at a seed (getNumStreamlinesProb_k, generate_streamlines_cuda.cu:427-462).
__device__ __forceinline__ int prob_seed_peaks(const DevParams &P, float3 seed, float *odf_sh,
                                               int *ind_sh, const int *partner_sh, int lane) {
    Corners c;
    if (!trilinear_setup(P, seed, c)) return 0;
    const int len = P.samplm_nr;
    float m = -FLT_MAX;
    for (int t = lane; t < len; t += kWarp) {
        const float x = trilinear_elem(P.dataf, c, t);
        odf_sh[t] = x;
        m = fmax_ref(m, x);
    }
    m = warp_max_ref(m);
    const float thr = (float)(P.pmf_threshold * (double)m);
    for (int t = lane; t < len; t += kWarp)
        if (odf_sh[t] < thr) odf_sh[t] = 0.0f;
    __syncwarp();
    return peak_directions(P, odf_sh, ind_sh, len, partner_sh, lane);
}

}  // namespace csl
