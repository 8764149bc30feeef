// Residual-bootstrap direction getter (boot.cu:20-608), plain FP32 warp path.
//
// Per attempt: trilinear DWI gather -> non-b0 compaction -> r = R s and
// h = H s -> h += r[perm] with a per-lane Philox draw (curand() % hr) ->
// scatter back, clamp at min_signal, divide by the b0 mean -> OPDT or CSA
// SH fit -> ODF = sampling_matrix . coef -> 5%-of-max threshold -> peaks ->
// closest peak within max_angle.  Every reduction keeps the reference's
// order (lane-strided fused multiply-add partials, then a shfl_down tree), so
// the FP32 results match the reference kernel bit for bit.  Independent rows
// of each mat-vec are interleaved four at a time for instruction-level
// parallelism; interleaving does not change any row's arithmetic.
//
// Deliberate difference: the reference's tracking step passes a one-element
// shared slot as the peak buffer and peak_directions_d writes every peak
// into it, overrunning into the neighbouring warp's slot whenever a step
// has more than one peak.  Here each warp has a peak buffer of its own.
#pragma once
#include "common.cuh"

namespace csl {

struct BootSmem {
    float *vox;  // [n32t]
    float *msk;  // [n32t]
    float *r;    // [max(n32t, samplm_nr)]
    float *h;    // [max(n32t, samplm_nr)]
    int *ind;    // [samplm_nr]
};

constexpr float kN0Const = 0.28209479177387814f;  // .5 / sqrt(pi)

// dst[i] = sum_j v[j] * M[i*m + j]   (ndotp_d, boot.cu:195-230).
// NPER = compile-time bound on the elements per lane (m <= 32 * NPER), so the
// unrolled loops carry no dead iterations; the arithmetic of each row does
// not depend on NPER.
template <int KIND, int NPER>  // KIND: 0 plain, 1 OPDT transform, 2 CSA transform
__device__ __forceinline__ void ndotp_rows_n(int nrows, int m, const float *v_sh,
                                             const float *__restrict__ M, float *dst, int lane) {
    // transformed source values of this lane (the transform is per element)
    constexpr int kMaxPer = NPER;
    float sv[kMaxPer];
    const int nper = (m + kWarp - 1) / kWarp;
#pragma unroll
    for (int q = 0; q < kMaxPer; q++) {
        sv[q] = 0.0f;
        const int j = q * kWarp + lane;
        if (q < nper && j < m) {
            const float x = v_sh[j];
            if (KIND == 0) {
                sv[q] = x;
            } else if (KIND == 1) {
                const float ONEP5 = 1.5f;
                sv[q] = -__logf(x) * (ONEP5 + __logf(x)) * x;
            } else {
                const float lo = 0.001f, hi = 0.999f;
                float c = (x > lo) ? x : lo;
                c = (c < hi) ? c : hi;
                sv[q] = __logf(-__logf(c));
            }
        }
    }
    // 32 rows at a time: lane l accumulates its lane-strided partial of every
    // row, then a transposing xor butterfly (16, 8, 4, 2, 1) leaves the sum of
    // row r0 + l in lane l.  At each level a lane adds its own partial to its
    // partner's for the half of the rows it keeps: the same pairs, in the same
    // association, as the reference's shfl_down tree, which only lane 0 reads.
    const int npr = nper;
    for (int r0 = 0; r0 < nrows; r0 += kWarp) {
        float v[kWarp];
#pragma unroll
        for (int r = 0; r < kWarp; r++) {
            float t = 0.0f;
            if (r0 + r < nrows) {
                const float *row = M + (size_t)(r0 + r) * m;
#pragma unroll
                for (int q = 0; q < kMaxPer; q++) {
                    const int j = q * kWarp + lane;
                    if (q < npr && j < m) t += sv[q] * __ldg(row + j);
                }
            }
            v[r] = t;
        }
#pragma unroll
        for (int o = kWarp / 2; o; o >>= 1) {
            const bool up = (lane & o) != 0;
#pragma unroll
            for (int i = 0; i < o; i++) {
                const float send = up ? v[i] : v[i + o];
                const float keep = up ? v[i + o] : v[i];
                v[i] = keep + __shfl_xor_sync(FULL, send, o);
            }
        }
        if (r0 + lane < nrows) dst[r0 + lane] = v[0];
    }
}

template <int KIND>
__device__ __forceinline__ void ndotp_rows(int nrows, int m, const float *v_sh,
                                           const float *__restrict__ M, float *dst, int lane) {
    if (m <= 2 * kWarp)
        ndotp_rows_n<KIND, 2>(nrows, m, v_sh, M, dst, lane);
    else if (m <= 5 * kWarp)
        ndotp_rows_n<KIND, 5>(nrows, m, v_sh, M, dst, lane);
    else
        ndotp_rows_n<KIND, 16>(nrows, m, v_sh, M, dst, lane);
}

// maskGet (boot.cu:52-83): compact entries with mask == 0
__device__ __forceinline__ int mask_get(int n, const int *__restrict__ mask, const float *plain,
                                        float *masked, int lane) {
    const unsigned lmask = (1u << lane) - 1u;
    int woff = 0;
    for (int j = 0; j < n; j += kWarp) {
        const int act = (j + lane < n) ? !__ldg(mask + j + lane) : 0;
        const unsigned msk = __ballot_sync(FULL, act);
        if (act) masked[woff + __popc(msk & lmask)] = plain[j + lane];
        woff += __popc(msk);
    }
    return woff;
}

// maskPut (boot.cu:85-113): scatter back to the mask == 0 entries
__device__ __forceinline__ void mask_put(int n, const int *__restrict__ mask, const float *masked,
                                         float *plain, int lane) {
    const unsigned lmask = (1u << lane) - 1u;
    int woff = 0;
    for (int j = 0; j < n; j += kWarp) {
        const int act = (j + lane < n) ? !__ldg(mask + j + lane) : 0;
        const unsigned msk = __ballot_sync(FULL, act);
        if (act) plain[j + lane] = masked[woff + __popc(msk & lmask)];
        woff += __popc(msk);
    }
}

// avgMask (boot.cu:20-50): mean of the mask != 0 entries
__device__ __forceinline__ float avg_mask(int n, const int *__restrict__ mask, const float *data,
                                          int lane) {
    int cnt = 0;
    float sum = 0.0f;
    for (int i = lane; i < n; i += kWarp) {
        if (__ldg(mask + i)) {
            cnt++;
            sum += data[i];
        }
    }
#pragma unroll
    for (int i = 16; i; i >>= 1) {
        sum += __shfl_xor_sync(FULL, sum, i);
        cnt += __shfl_xor_sync(FULL, cnt, i);
    }
    return sum / cnt;
}

// closest_peak_d (boot.cu:115-193); peaks are vertices ind[0..npeaks)
__device__ __forceinline__ int closest_peak(const DevParams &P, const float *verts, float3 direction, int npeaks,
                                            const int *ind, int lane, float3 *peak) {
    const float cos_similarity = P.cos_max_angle;
    float cpeak_dot = 0;
    int cpeak_idx = -1;
    for (int j = 0; j < npeaks; j += kWarp) {
        if (j + lane < npeaks) {
            const float3 p = vert3_any(verts, ind[j + lane]);
            const float dot = direction.x * p.x + direction.y * p.y + direction.z * p.z;
            if (fabsf(dot) > fabsf(cpeak_dot)) {
                cpeak_dot = dot;
                cpeak_idx = j + lane;
            }
        }
    }
#pragma unroll
    for (int j = 16; j; j >>= 1) {
        const float dot = __shfl_xor_sync(FULL, cpeak_dot, j);
        const int idx = __shfl_xor_sync(FULL, cpeak_idx, j);
        if (fabsf(dot) > fabsf(cpeak_dot)) {
            cpeak_dot = dot;
            cpeak_idx = idx;
        }
    }
    // lane 0's choice is the one the reference stores
    cpeak_dot = __shfl_sync(FULL, cpeak_dot, 0);
    cpeak_idx = __shfl_sync(FULL, cpeak_idx, 0);
    if (cpeak_idx >= 0) {
        const float3 p = vert3_any(verts, ind[cpeak_idx]);
        if (cpeak_dot >= cos_similarity) {
            *peak = p;
            return 1;
        }
        if (cpeak_dot <= -cos_similarity) {
            *peak = make_float3(-p.x, -p.y, -p.z);
            return 1;
        }
    }
    return 0;
}

// get_direction_boot_d (boot.cu:393-608).  NATTEMPTS == 1: seed peaks
// (returns their count, vertices in S.ind); otherwise one tracking step
// (returns 1 and the new direction in *newdir, or 0).
template <int NATTEMPTS, int MODEL>
__device__ int boot_get_direction(const DevParams &P, Philox &rng, float3 dir, float3 point,
                                  const BootSmem &S, const int *partner_sh, int lane,
                                  float3 *newdir, int *ndraws) {
    const int T = P.dimt;
    const int hr = P.hr_side;
    const int nr = P.samplm_nr;
    for (int att = 0; att < NATTEMPTS; att++) {
        Corners c;
        const bool inb = trilinear_setup(P, point, c);
        if (inb)
            for (int t = lane; t < T; t += kWarp) S.vox[t] = trilinear_elem(P.dataf, c, t);
        __syncwarp();
        mask_get(T, P.b0s_mask, S.vox, S.msk, lane);
        __syncwarp();
        if (inb) {
            ndotp_rows<0>(hr, hr, S.msk, P.R, S.r, lane);
            ndotp_rows<0>(hr, hr, S.msk, P.H, S.h, lane);
            __syncwarp();
            for (int j = 0; j < hr; j += kWarp) {
                if (j + lane < hr) {
                    const int src = (int)(rng.next() % (unsigned)hr);
                    S.h[j + lane] += S.r[src];
                    if (ndraws) ndraws[0] += 1;
                }
            }
            __syncwarp();
            mask_put(T, P.b0s_mask, S.h, S.vox, lane);
            __syncwarp();
            for (int j = lane; j < T; j += kWarp) {
                const float x = S.vox[j];
                S.vox[j] = (P.min_signal > x) ? P.min_signal : x;
            }
            __syncwarp();
            const float denom = avg_mask(T, P.b0s_mask, S.vox, lane);
            for (int j = lane; j < T; j += kWarp) S.vox[j] /= denom;
            __syncwarp();
            mask_get(T, P.b0s_mask, S.vox, S.msk, lane);
            __syncwarp();
            if (MODEL == OPDT) {
                ndotp_rows<1>(P.delta_nr, hr, S.msk, P.delta_q, S.r, lane);
                ndotp_rows<0>(P.delta_nr, hr, S.msk, P.delta_b, S.h, lane);
                __syncwarp();
                for (int j = lane; j < P.delta_nr; j += kWarp) S.r[j] -= S.h[j];
                __syncwarp();
            } else {
                ndotp_rows<2>(P.delta_nr, hr, S.msk, P.delta_q, S.r, lane);
                __syncwarp();
                if (lane == 0) S.r[0] = kN0Const;
                __syncwarp();
            }
            ndotp_rows<0>(nr, P.delta_nr, S.r, P.sampling, S.h, lane);
        } else {
            for (int j = lane; j < nr; j += kWarp) S.h[j] = 0;
        }
        __syncwarp();

        float m = -FLT_MAX;
        for (int i = lane; i < nr; i += kWarp) m = fmax_ref(m, S.h[i]);
        m = warp_max_ref(m);
        const float thr = (float)(P.pmf_threshold * (double)m);
        __syncwarp();
        for (int j = lane; j < nr; j += kWarp)
            if (S.h[j] < thr) S.h[j] = 0;
        __syncwarp();

        const int ndir = peak_directions(P, S.h, S.ind, nr, partner_sh, lane);
        if (NATTEMPTS == 1) return ndir;
        if (ndir > 0) {
            float3 peak;
            const int found = closest_peak(P, P.verts, dir, ndir, S.ind, lane, &peak);
            __syncwarp();
            if (found) {
                *newdir = peak;
                return 1;
            }
        }
    }
    return 0;
}

}  // namespace csl
