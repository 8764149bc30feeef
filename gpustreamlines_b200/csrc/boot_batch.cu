// Batched residual-bootstrap tracking on the tensor cores (CSA and OPDT models).
//
// The plain bootstrap getter (boot.cuh, boot.cu:393-608 in the reference)
// runs one streamline per warp and streams the fit matrices H, R (150 x 150),
// the SH fit Delta (C x 150) and the sphere basis (724 x C) from L2 on every
// bootstrap attempt: ~310 KB of matrix reads for ~85 k multiply-adds.  Here a
// CTA owns 128 streamline halves ("slots") and advances all of them by one
// bootstrap attempt per iteration, so the three contractions become GEMMs
// with M = 128 slots that read each matrix once per 128 attempts:
//
//   gather    128 DWI signals (trilinear, non-b0 volumes)       -> A1 [128 x K1]
//   MMA 1     A1 x [R ; H]^T                                     -> D1 [128 x 2 K1]  (TMEM)
//   epilogue  h + r[random index], clamp, / b0 mean, CSA
//             transform log(-log(x)) or OPDT -log x (1.5+log x) x -> A2 [128 x K1]
//   MMA 2     A2 x Delta_q^T (OPDT: then += x (-Delta_b)^T)      -> D2 [128 x C]     (TMEM)
//   epilogue  coefficients (c0 = 1 / (2 sqrt(pi)))               -> A3 [128 x C]
//   MMA 3     A3 x B^T in 256-vertex chunks                      -> ODF rows         (TMEM -> L2)
//   peaks     5 % threshold, local maxima, sort, separation,
//             closest peak: the plain getter's own warp code, one warp per slot
//
// Each product runs in BF16 with the three-term split a*b ~ ah*bh + ah*bl +
// al*bh (x = xh + xl, xh = bf16(x), xl = bf16(x - xh)), accumulated in FP32
// in tensor memory: about 2^-17 relative error per product, against 2^-24
// for FP32.  The peak search, the thresholds, the stopping rule and the point
// update are the plain getter's, in FP32/FP64 as the reference has them.
//
// What differs from the plain path: bootstrap draws come from one Philox
// stream per streamline half (not the reference's per-lane streams), and the
// ODF carries the BF16x3 rounding, so streamlines are statistically, not
// bitwise, equal to the plain path's.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "boot.cuh"
#include "common.cuh"
#include "kernels.h"
#include "tc.cuh"
#include "track.cuh"

namespace csl {

constexpr int kSlots = 128;         // slots per CTA = MMA M = TMEM lanes
constexpr int kBWarps = 16;
constexpr int kBThreads = kBWarps * kWarp;
constexpr int kBootAttempts = 5;    // bootstrap draws per step (boot.cu tracking)
constexpr int kOdfChunk = 256;      // vertices per MMA-3 chunk (TMEM columns)
constexpr int kTmemCols = 512;
constexpr unsigned long long kBatchSubseqBase = 1ull << 62;  // disjoint from pass-1 streams

__host__ __device__ inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

BootBatchGeom boot_batch_geom(const DevParams &P, int hr, int nb0) {
    BootBatchGeom g{};
    g.hr = hr;
    g.nb0 = nb0;
    g.HP = round_up(hr, 32);
    g.N1 = 2 * g.HP;
    g.C = P.delta_nr;
    g.N2 = round_up(P.delta_nr, 16);
    g.V = P.samplm_nr;
    g.nchunk1 = g.HP / 32;
    g.nchunk3 = (P.samplm_nr + kOdfChunk - 1) / kOdfChunk;
    g.vstride = round_up(P.samplm_nr, 4);
    g.TP = round_up(P.dimt, 4);
    g.b1_chunk = 128 * g.N1;          // 2 terms x N1 rows x 32 k x 2 B
    g.b2_bytes = 4 * g.N2 * g.HP;     // 2 terms x N2 rows x HP k x 2 B
    g.b3_chunk = 1024 * g.N2;         // 2 terms x 256 rows x N2 k x 2 B
    const int a1 = 512 * g.HP, rbuf = 512 * (hr + 1), a3 = 512 * g.N2;
    const int pk = kBWarps * 3 * g.vstride * 4;  // per-warp 2 ODF rows + flags, spans R0 and R1
    g.r0 = round_up(std::max(std::max(a1, rbuf), a3), 1024);
    g.r1 = round_up(std::max(std::max(std::max(2 * g.b1_chunk, 512 * g.HP), g.b3_chunk), pk - g.r0), 1024);
    g.r2 = round_up(g.b2_bytes, 1024);
    g.nbr_shorts = round_up(g.V * kMaxDegree, 8);
    g.smem = 1024 + g.r0 + g.r1 + g.r2 + 3 * kSlots * 16 + 2 * kSlots * 4 + g.nbr_shorts * 2 +
             kMaxSortLayers * kWarp * 4 + 128;
    // the sphere vertices join shared memory when they fit in the per-CTA limit
    g.verts_floats = round_up(3 * g.V, 4);
    if (g.smem + g.verts_floats * 4 <= 227 * 1024)
        g.smem += g.verts_floats * 4;
    else
        g.verts_floats = 0;
    return g;
}

// ---------------------------------------------------------------------------
// set-up: the three matrices in the operand layout of tc.cuh, BF16 hi / lo

__global__ void boot_batch_pack_kernel(DevParams P, BootBatchGeom g, __nv_bfloat16 *B1g,
                                       __nv_bfloat16 *B2g, __nv_bfloat16 *B3g) {
    const long long n1 = (long long)g.N1 * g.HP, n2 = (long long)g.N2 * g.HP * (P.model == OPDT ? 2 : 1);
    const long long n3 = (long long)g.nchunk3 * kOdfChunk * g.N2;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n1 + n2 + n3;
         e += (long long)gridDim.x * blockDim.x) {
        float x;
        char *hi, *lo;
        uint32_t off;
        if (e < n1) {
            // rows [0, HP): R, rows [HP, 2 HP): H; k = non-b0 volume index
            const int n = (int)(e / g.HP), k = (int)(e % g.HP);
            const int row = n < g.HP ? n : n - g.HP;
            const float *M = n < g.HP ? P.R : P.H;
            x = (row < g.hr && k < g.hr) ? M[(size_t)row * g.hr + k] : 0.0f;
            hi = reinterpret_cast<char *>(B1g) + (size_t)(k / 32) * g.b1_chunk;
            lo = hi + g.b1_chunk / 2;
            off = kmajor_off(n, k % 32, g.N1);
        } else if (e < n1 + n2) {
            // delta_q, then (OPDT) -delta_b as a second packed operand
            const long long f = e - n1;
            const int part = (int)(f / ((long long)g.N2 * g.HP));
            const long long f2 = f % ((long long)g.N2 * g.HP);
            const int n = (int)(f2 / g.HP), k = (int)(f2 % g.HP);
            const float *M = part == 0 ? P.delta_q : P.delta_b;
            x = (n < g.C && k < g.hr) ? M[(size_t)n * g.hr + k] : 0.0f;
            if (part == 1) x = -x;
            hi = reinterpret_cast<char *>(B2g) + (size_t)part * g.b2_bytes;
            lo = hi + g.b2_bytes / 2;
            off = kmajor_off(n, k, g.N2);
        } else {
            const long long f = e - n1 - n2;
            const int ch = (int)(f / ((long long)kOdfChunk * g.N2));
            const int r = (int)((f / g.N2) % kOdfChunk), k = (int)(f % g.N2);
            const int v = ch * kOdfChunk + r;
            x = (v < g.V && k < g.C) ? P.sampling[(size_t)v * g.C + k] : 0.0f;
            hi = reinterpret_cast<char *>(B3g) + (size_t)ch * g.b3_chunk;
            lo = hi + g.b3_chunk / 2;
            off = kmajor_off(r, k, kOdfChunk);
        }
        const __nv_bfloat16 h = __float2bfloat16_rn(x);
        const __nv_bfloat16 l = __float2bfloat16_rn(x - __bfloat162float(h));
        *reinterpret_cast<__nv_bfloat16 *>(hi + off) = h;
        *reinterpret_cast<__nv_bfloat16 *>(lo + off) = l;
    }
}

// DWI copy for the batched gather: T axis reordered by volidx (non-b0 volumes
// first, then the b0s) and padded to TP so every voxel row is 16-byte aligned
__global__ void boot_batch_dwi_kernel(const float *__restrict__ src, const int *__restrict__ volidx,
                                      long long nvox, int T, int TP, float *__restrict__ dst) {
    const long long n = nvox * TP;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        const long long vox = e / TP;
        const int k = (int)(e - vox * TP);
        dst[e] = k < T ? src[vox * T + volidx[k]] : 0.0f;
    }
}

// streamline -> (seed, initial vertex) from the pass-1 outputs; streamlines
// at or past cap (the slot capacity of a graph-captured batch) are not
// written and flag ST_SLOT_OVERFLOW
__global__ void boot_batch_prep_kernel(const int *__restrict__ npeaks, const int *__restrict__ sl_off,
                                       const short *__restrict__ peaks, int max_store, int n, int cap,
                                       int *sl_seed, short *sl_vert, int *status) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const int np = npeaks[s], base = sl_off[s];
        if (np > max_store) atomicOr(status, ST_PEAKS_OVERFLOW);
        const int m = np < max_store ? np : max_store;
        for (int k = 0; k < m; k++) {
            if (base + k >= cap) {
                atomicOr(status, ST_SLOT_OVERFLOW);
                break;
            }
            sl_seed[base + k] = s;
            sl_vert[base + k] = peaks[(size_t)s * max_store + k];
        }
    }
}

// the streamline count of a batch: nsl, or min(*count, nsl) when the count is
// in device memory (graph-captured batches, nsl = their slot capacity)
__device__ __forceinline__ int batch_count(const int *count, int nsl) {
    if (!count) return nsl;
    const int c = *count;
    return c < 0 ? 0 : (c < nsl ? c : nsl);
}

// streamline length = backward half + forward half - the shared seed point
__global__ void boot_batch_join_kernel(const int *__restrict__ half_len, const int *__restrict__ sl_seed,
                                       int nsl, const int *__restrict__ count, int *out_len, int *out_seed) {
    nsl = batch_count(count, nsl);
    for (int sl = blockIdx.x * blockDim.x + threadIdx.x; sl < nsl; sl += gridDim.x * blockDim.x) {
        out_len[sl] = half_len[2 * sl] - 1 + half_len[2 * sl + 1];
        out_seed[sl] = sl_seed[sl];
    }
}

// reversed backward half, then the forward half without its seed point;
// nothing when the batch's status shows an overflow (it is re-run)
__global__ void gather_halves_kernel(const float *__restrict__ pool, const long long *__restrict__ half_off,
                                     const int *__restrict__ half_len, const long long *__restrict__ pt_off,
                                     int nsl, const int *__restrict__ count, const int *__restrict__ status,
                                     float *__restrict__ out) {
    if (status && (*status & (ST_POOL_OVERFLOW | ST_SLOT_OVERFLOW | ST_PEAKS_OVERFLOW))) return;
    nsl = batch_count(count, nsl);
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x / kWarp;
    for (int sl = blockIdx.x * wpb + threadIdx.x / kWarp; sl < nsl; sl += gridDim.x * wpb) {
        const int nB = half_len[2 * sl], nF = half_len[2 * sl + 1];
        const long long oB = half_off[2 * sl], oF = half_off[2 * sl + 1];
        const int n3 = 3 * (nB - 1 + nF);
        float *dst = out + 3 * pt_off[sl];
        for (int j = lane; j < n3; j += kWarp) {
            const int p = j / 3, c = j - 3 * p;
            dst[j] = (p < nB) ? pool[3 * (oB + nB - 1 - p) + c] : pool[3 * (oF + p - nB + 1) + c];
        }
    }
}

// ---------------------------------------------------------------------------
// the tracking kernel

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t *>(&v);
}

// split 8 floats into BF16 hi and lo words (element k in the low half of word k/2)
__device__ __forceinline__ void split8(const float (&x)[8], uint4 &hi, uint4 &lo) {
    uint32_t h[4], l[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const __nv_bfloat162 hv = __floats2bfloat162_rn(x[2 * q], x[2 * q + 1]);
        const float2 hf = __bfloat1622float2(hv);
        h[q] = *reinterpret_cast<const uint32_t *>(&hv);
        l[q] = pack_bf16x2(x[2 * q] - hf.x, x[2 * q + 1] - hf.y);
    }
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    lo = make_uint4(l[0], l[1], l[2], l[3]);
}

// Tail of the peak search: kept maxima ind[0..n) in ascending vertex order ->
// descending sort by value (the reference's network), minimum-separation filter.
__device__ __forceinline__ int peaks_finish(const DevParams &P, const float *vs, const float *odf, int *ind, int n,
                                            const int *partner_sh, int lane) {
    const unsigned lmask = (1u << lane) - 1u;
    if (n == 0) return 0;
    if (n < kWarp) {
        float k = -FLT_MAX;
        int v = 0;
        if (lane < n) {
            v = ind[lane];
            k = odf[v];
        }
        warp_sort_desc(partner_sh, lane, k, v);
        // greedy minimum-separation filter: candidate i is kept unless a
        // kept peak before it lies within the separation angle
        const float3 pv = vert3_any(vs, lane < n ? v : 0);
        unsigned kept = 1u;
        for (int i = 1; i < n; i++) {
            const float3 abc = make_float3(__shfl_sync(FULL, pv.x, i), __shfl_sync(FULL, pv.y, i),
                                           __shfl_sync(FULL, pv.z, i));
            float cs = abc.x * pv.x + abc.y * pv.y + abc.z * pv.z;
            if (P.sphere_symm) cs = fabsf(cs);
            const bool hit = ((kept >> lane) & 1u) && cs > P.cos_min_sep;
            if (__ballot_sync(FULL, hit) == 0u) kept |= 1u << i;
        }
        __syncwarp();
        if ((kept >> lane) & 1u) ind[__popc(kept & lmask)] = v;
        __syncwarp();
        return __popc(kept);
    }
    // 32 or more peaks: the reference skips the sort; serial filter on lane 0
    if (lane == 0) {
        int k = 1;
        for (int i = 1; i < n; i++) {
            const int vi = ind[i];
            const float3 abc = vert3_any(vs, vi);
            int j = 0;
            for (; j < k; j++) {
                const float3 d = vert3_any(vs, ind[j]);
                float cs = abc.x * d.x + abc.y * d.y + abc.z * d.z;
                if (P.sphere_symm) cs = fabsf(cs);
                if (cs > P.cos_min_sep) break;
            }
            if (j == k) ind[k++] = vi;
        }
        n = k;
    }
    n = __shfl_sync(FULL, n, 0);
    __syncwarp();
    return n;
}

// Peak search of one thresholded ODF row, warp-cooperative, with the
// semantics of peak_directions_d (tracking_helpers.cu:75-245) and fewer
// instructions:
//  * only vertices that can be maxima are tested: after the 5 % threshold all
//    values are >= 0 when the row maximum is positive, so a zero vertex has no
//    smaller neighbour and is never a maximum;
//  * a vertex is a maximum when no neighbour is larger and some neighbour is
//    smaller -- the flag the edge loop with atomics leaves (its -1 wins over
//    |= 1); neighbours come from a per-vertex table (unused entries hold the
//    vertex itself, which is neither larger nor smaller);
//  * maxima are kept in ascending vertex order, so the relative threshold,
//    the descending sort network and its tie order are those of the reference;
//  * the minimum-separation filter runs the reference's greedy loop with the
//    inner scan over the kept peaks done by all lanes at once.
// cand[] and ind[] may alias.  Returns the number of kept peaks, in ind[].
__device__ __forceinline__ int peaks_sparse(const DevParams &P, const float *vs, float *odf, int *ind, int nr, float m,
                                            const short *__restrict__ nbr, const int *partner_sh, int lane) {
    const unsigned lmask = (1u << lane) - 1u;
    const float thr = (float)(P.pmf_threshold * (double)m);
    const bool all_cand = !(m > 0.0f);
    // threshold in place, row minimum, candidate list (ascending)
    float mn = FLT_MAX;
    int nc = 0;
    for (int j = 0; j < nr; j += kWarp) {
        const int v = j + lane;
        bool c = false;
        if (v < nr) {
            float x = odf[v];
            if (x < thr) {
                x = 0;
                odf[v] = 0;
            }
            mn = fmin_ref(mn, x);
            c = all_cand || x > 0.0f;
        }
        const unsigned msk = __ballot_sync(FULL, c);
        if (c) ind[nc + __popc(msk & lmask)] = v;
        nc += __popc(msk);
    }
    float odf_min = warp_min_ref(mn);
    odf_min = (0 > odf_min) ? 0 : odf_min;
    __syncwarp();
    // local maxima among the candidates, compacted in place (ascending)
    int nm = 0;
    for (int c0 = 0; c0 < nc; c0 += kWarp) {
        bool mx = false;
        int v = 0;
        if (c0 + lane < nc) {
            v = ind[c0 + lane];
            const float x = odf[v];
            const uint4 nb = *reinterpret_cast<const uint4 *>(nbr + v * kMaxDegree);
            const uint32_t w4[4] = {nb.x, nb.y, nb.z, nb.w};
            bool larger = false, smaller = false;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const float y0 = odf[w4[q] & 0xffffu], y1 = odf[w4[q] >> 16];
                larger |= (x < y0) | (x < y1);
                smaller |= (y0 < x) | (y1 < x);
            }
            mx = !larger && smaller;
        }
        const unsigned msk = __ballot_sync(FULL, mx);
        if (mx) ind[nm + __popc(msk & lmask)] = v;
        nm += __popc(msk);
    }
    __syncwarp();
    // RELATIVE_PEAK_THRESH * max over maxima of (odf + (-odf_min)), then filter
    float mm = -FLT_MAX;
    const float neg_min = -odf_min;
    for (int c = lane; c < nm; c += kWarp) mm = fmax_ref(mm, odf[ind[c]] + neg_min);
    mm = warp_max_ref(mm);
    const float comp_thres = (float)(P.relative_peak_thresh * (double)mm);
    int n = 0;
    for (int c0 = 0; c0 < nm; c0 += kWarp) {
        int v = 0;
        bool keep = false;
        if (c0 + lane < nm) {
            v = ind[c0 + lane];
            keep = (odf[v] - odf_min) >= comp_thres;
        }
        const unsigned msk = __ballot_sync(FULL, keep);
        __syncwarp();
        if (keep) ind[n + __popc(msk & lmask)] = v;
        n += __popc(msk);
    }
    __syncwarp();
    return peaks_finish(P, vs, odf, ind, n, partner_sh, lane);
}

// Faster exact path of the same search.  A peak is kept only if
// (value - min) >= RELATIVE_PEAK_THRESH * (max over maxima of value - min);
// when the arg-max vertex is a strict local maximum that bound is known from
// one pass, so the local-maximum test runs only on vertices that could be
// kept (often a minority of the 724), thresholded values computed on the fly.
// Returns -1 (warp-uniform) when the arg-max is not a strict maximum or the
// row maximum is not positive; the caller then runs peaks_sparse.
__device__ __forceinline__ int peaks_fast(const DevParams &P, const float *vs, const float *odf, int *ind, int nr,
                                          const short *__restrict__ nbr, const int *partner_sh, int lane) {
    const unsigned lmask = (1u << lane) - 1u;
    float m = -FLT_MAX, mn = FLT_MAX;
    int am = 0x7fffffff;
    for (int v = lane; v < nr; v += kWarp) {
        const float x = odf[v];
        if (x > m) {
            m = x;
            am = v;
        }
        mn = fmin_ref(mn, x);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const float om = __shfl_xor_sync(FULL, m, o);
        const int oa = __shfl_xor_sync(FULL, am, o);
        if (om > m || (om == m && oa < am)) {
            m = om;
            am = oa;
        }
        mn = fmin_ref(mn, __shfl_xor_sync(FULL, mn, o));
    }
    if (!(m > 0.0f)) return -1;
    const float thr = (float)(P.pmf_threshold * (double)m);
    float odf_min = (mn < thr) ? 0.0f : mn;
    odf_min = (0 > odf_min) ? 0 : odf_min;
    {
        float y = m;
        if (lane < kMaxDegree) {
            y = odf[nbr[am * kMaxDegree + lane]];
            y = (y < thr) ? 0.0f : y;
        }
        const unsigned larger = __ballot_sync(FULL, m < y), smaller = __ballot_sync(FULL, y < m);
        if (larger != 0u || smaller == 0u) return -1;
    }
    const float mm = m + (-odf_min);
    const float comp_thres = (float)(P.relative_peak_thresh * (double)mm);
    // vertices that could be kept (thresholded value - min >= comp_thres),
    // compacted in ascending order into ind; then the local-maximum test on
    // the compacted list with every lane busy, kept ones compacted in place
    int nc = 0;
    for (int j = 0; j < nr; j += kWarp) {
        const int v = j + lane;
        bool c = false;
        if (v < nr) {
            float x = odf[v];
            x = (x < thr) ? 0.0f : x;
            c = (x - odf_min) >= comp_thres;
        }
        const unsigned msk = __ballot_sync(FULL, c);
        if (c) ind[nc + __popc(msk & lmask)] = v;
        nc += __popc(msk);
    }
    __syncwarp();
    int n = 0;
    for (int c0 = 0; c0 < nc; c0 += kWarp) {
        bool keep = false;
        int v = 0;
        if (c0 + lane < nc) {
            v = ind[c0 + lane];
            float x = odf[v];
            x = (x < thr) ? 0.0f : x;
            const uint4 nb = *reinterpret_cast<const uint4 *>(nbr + v * kMaxDegree);
            const uint32_t w4[4] = {nb.x, nb.y, nb.z, nb.w};
            bool larger = false, smaller = false;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                float y0 = odf[w4[q] & 0xffffu], y1 = odf[w4[q] >> 16];
                y0 = (y0 < thr) ? 0.0f : y0;
                y1 = (y1 < thr) ? 0.0f : y1;
                larger |= (x < y0) | (x < y1);
                smaller |= (y0 < x) | (y1 < x);
            }
            keep = !larger && smaller;
        }
        const unsigned msk = __ballot_sync(FULL, keep);
        __syncwarp();  // every lane has read its entry before any is overwritten
        if (keep) ind[n + __popc(msk & lmask)] = v;
        n += __popc(msk);
    }
    __syncwarp();
    return peaks_finish(P, vs, odf, ind, n, partner_sh, lane);
}

// ---------------------------------------------------------------------------
// near-tie re-evaluation in float64

// True when a decision of the peak search that shapes the kept peaks lies
// within tol x (row maximum) of flipping: the local-maximum test of a vertex
// that could be kept, its relative-threshold test, or its order against a
// kept peak closer than the separation angle (the descending sort decides
// which of the two the separation filter keeps).  The BF16x3 row differs from
// the float64 one by ~3e-5 of its maximum at most, so a row without such a
// decision selects the float64 row's peaks.
__device__ __forceinline__ bool near_tie(const DevParams &P, const float *vs, const float *odf, const int *ind, int n,
                                         int nr,
                                         const short *__restrict__ nbr, float tol, int lane) {
    float m = -FLT_MAX;
    for (int v = lane; v < nr; v += kWarp) m = fmax_ref(m, odf[v]);
    m = warp_max_ref(m);
    if (!(m > 0.0f)) return false;
    const float thr = (float)(P.pmf_threshold * (double)m);
    const float tm = tol * m;
    float mn = FLT_MAX;
    for (int v = lane; v < nr; v += kWarp) {
        const float x = odf[v];
        mn = fmin_ref(mn, x < thr ? 0.0f : x);
    }
    float odf_min = warp_min_ref(mn);
    odf_min = (0 > odf_min) ? 0 : odf_min;
    const float comp = (float)(P.relative_peak_thresh * (double)(m - odf_min));
    bool hit = false;
    for (int v = lane; v < nr; v += kWarp) {
        float x = odf[v];
        x = x < thr ? 0.0f : x;
        if (x - odf_min < comp - tm) continue;  // cannot be kept
        bool bigger = false, close = false;
#pragma unroll
        for (int q = 0; q < kMaxDegree; q++) {
            const int u = nbr[v * kMaxDegree + q];
            if (u == v) continue;
            float y = odf[u];
            y = y < thr ? 0.0f : y;
            bigger |= y > x + tm;
            close |= fabsf(y - x) <= tm;
        }
        if (bigger) continue;  // not a maximum, by more than the margin
        if (close || fabsf((x - odf_min) - comp) <= tm) {
            hit = true;
            continue;
        }
        const float3 pv = vert3_any(vs, v);
        for (int k = 0; k < n; k++) {
            const int p = ind[k];
            if (p == v) continue;
            float y = odf[p];
            y = y < thr ? 0.0f : y;
            if (fabsf(y - x) > tm) continue;
            const float3 pp = vert3_any(vs, p);
            float cs = pv.x * pp.x + pv.y * pp.y + pv.z * pp.z;
            if (P.sphere_symm) cs = fabsf(cs);
            if (cs > P.cos_min_sep) {
                hit = true;
                break;
            }
        }
    }
    return __any_sync(FULL, hit);
}

// One bootstrap attempt fitted again in float64 for a flagged row, with the
// resample the batched fit used (the probe item's indices, or the Philox
// words regenerated from the counters saved when they were drawn): trilinear
// DWI in double, residual and hat products over the non-b0 volumes,
// h + r[idx], clamp at min_signal, division by the mean clamped b0 signal, the
// CSA transform (coefficient 0 fixed) or the OPDT form, and the sphere
// sampling; the row is rounded to float into odf.  Arithmetic of the float64
// accuracy reference (oracle/fp64.py); the float32 matrix entries are exact in
// double.
//
// Layout for speed (one warp, the tables in L2): vectors over the hr non-b0
// volumes live in registers, element j in lane j % 32, slot j / 32
// (hr <= 160), broadcast with shuffles; the tables of refit_tab_layout are
// transposed so that the warp's 32 lanes read 32 consecutive entries, and the
// loops are unrolled so that several rows of loads are in flight.  idx: hr
// ints of this warp's scratch.
constexpr int kRefitJ = 5;  // register slots per lane for an hr-vector (hr <= 160)

__device__ __forceinline__ double shfl_d(double x, int src) { return __shfl_sync(FULL, x, src); }

// slot k of a register-distributed hr-vector (k warp-uniform)
__device__ __forceinline__ double slot_of(const double (&x)[kRefitJ], int k) {
    double r = 0.0;
#pragma unroll
    for (int q = 0; q < kRefitJ; q++)
        if (q == k) r = x[q];
    return r;
}

__device__ __noinline__ void boot_refit_fp64(const DevParams &P, int hr, int nblk1, const int *__restrict__ volidx,
                                             float4 pt4, const int *pidx, const uint32_t *saved,
                                             const float *__restrict__ tab, int *idx, float *odf, int lane) {
    const int T = P.dimt, C = P.delta_nr, V = P.samplm_nr;
    const RefitTab L = refit_tab_layout(hr, C, V);
    const float2 *rh = reinterpret_cast<const float2 *>(tab + L.rh);
    const float *dq = tab + L.dq, *db = tab + L.db, *smp = tab + L.smp;
    const double px = pt4.x, py = pt4.y, pz = pt4.z;
    const bool inb = (px >= -0.5) && (px + 0.5 < P.dimx) && (py >= -0.5) && (py + 0.5 < P.dimy) &&
                     (pz >= -0.5) && (pz + 0.5 < P.dimz);
    if (!inb) {
        for (int v = lane; v < V; v += kWarp) odf[v] = 0.0f;
        __syncwarp();
        return;
    }
    // resample indices: given, or the batched fit's draws (part p drew columns
    // 16b .. 16b+15 for b = p, p + 4, ... in order)
    if (pidx) {
        for (int j = lane; j < hr; j += kWarp) idx[j] = pidx[j];
    } else if (lane < 4) {
        Philox g;
        g.key = make_uint2((uint32_t)P.rng_seed, (uint32_t)(P.rng_seed >> 32));
        g.ctr = make_uint4(saved[5 * lane], saved[5 * lane + 1], saved[5 * lane + 2], saved[5 * lane + 3]);
        g.out = philox4x32_10(g.ctr, g.key);
        g.idx = (int)saved[5 * lane + 4];
        for (int b = lane; b < nblk1; b += 4)
            for (int e = 0; e < 16; e++)
                if (16 * b + e < hr) idx[16 * b + e] = (int)(g.next() % (unsigned)hr);
    }
    // trilinear interpolation in double (corners in (i, j, k) order) of volume t
    const double fx = floor(px), fy = floor(py), fz = floor(pz);
    const double wx = px - fx, wy = py - fy, wz = pz - fz;
    const int lx = fx < 0 ? 0 : (int)fx, ly = fy < 0 ? 0 : (int)fy, lz = fz < 0 ? 0 : (int)fz;
    const int hx = min(lx + 1, P.dimx - 1), hy = min(ly + 1, P.dimy - 1), hz = min(lz + 1, P.dimz - 1);
    auto interp = [&](int t) {
        double acc = 0.0;
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int i = q >> 2, j = (q >> 1) & 1, k = q & 1;
            const double w = __dmul_rn(__dmul_rn(i ? wx : 1.0 - wx, j ? wy : 1.0 - wy), k ? wz : 1.0 - wz);
            const long long vx = ((long long)(i ? hx : lx) * P.dimy + (j ? hy : ly)) * P.dimz + (k ? hz : lz);
            acc = __dadd_rn(acc, __dmul_rn(w, (double)__ldg(P.dataf + vx * T + t)));
        }
        return acc;
    };
    const double ms = (double)P.min_signal;
    double sv[kRefitJ];
#pragma unroll
    for (int k = 0; k < kRefitJ; k++) {
        const int j = lane + 32 * k;
        sv[k] = j < hr ? interp(__ldg(volidx + j)) : 0.0;
    }
    // b0 mean of the clamped signal (the b0 volumes are not resampled)
    double bs = 0.0;
    for (int j = hr + lane; j < T; j += kWarp) {
        const double x = interp(__ldg(volidx + j));
        bs += x > ms ? x : ms;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) bs += shfl_d(bs, lane ^ o);
    const double denom = bs / (T - hr);
    // r = R s and h = H s: lane j accumulates rows j + 32k over i in order
    double rr[kRefitJ], hh[kRefitJ];
#pragma unroll
    for (int k = 0; k < kRefitJ; k++) rr[k] = hh[k] = 0.0;
    for (int i0 = 0; i0 < hr; i0 += 32) {
        const double sc = slot_of(sv, i0 >> 5);
        const int nb = min(32, hr - i0);
#pragma unroll 4
        for (int ii = 0; ii < nb; ii++) {
            const double si = shfl_d(sc, ii);
            const float2 *row = rh + (size_t)(i0 + ii) * hr;
#pragma unroll
            for (int k = 0; k < kRefitJ; k++) {
                const int j = lane + 32 * k;
                if (j < hr) {
                    const float2 m = __ldg(row + j);
                    rr[k] = fma((double)m.x, si, rr[k]);
                    hh[k] = fma((double)m.y, si, hh[k]);
                }
            }
        }
    }
    __syncwarp();  // idx written
    // bootstrap, clamp, normalise, transform: y = x / denom; CSA: log(-log c),
    // OPDT: -log y (1.5 + log y) y (y kept for the second product)
    const bool opdt = P.model == OPDT;
    double yv[kRefitJ], tv[kRefitJ];
#pragma unroll
    for (int k = 0; k < kRefitJ; k++) {
        const int j = lane + 32 * k;
        const int src = j < hr ? idx[j] : 0;
        double rs = 0.0;
#pragma unroll
        for (int q = 0; q < kRefitJ; q++) {
            const double v = shfl_d(rr[q], src & 31);
            if ((src >> 5) == q) rs = v;
        }
        double x = hh[k] + rs;
        x = x > ms ? x : ms;
        const double y = x / denom;
        yv[k] = y;
        if (opdt) {
            tv[k] = -log(y) * (1.5 + log(y)) * y;
        } else {
            const double c = y < 0.001 ? 0.001 : (y > 0.999 ? 0.999 : y);
            tv[k] = log(-log(c));
        }
        if (j >= hr) yv[k] = tv[k] = 0.0;
    }
    // SH coefficients: lane c accumulates c and c + 32 over j in order (the
    // tables are zero past C)
    double cf0 = 0.0, cf1 = 0.0, cb0 = 0.0, cb1 = 0.0;
    for (int j0 = 0; j0 < hr; j0 += 32) {
        const double tc = slot_of(tv, j0 >> 5), yc = slot_of(yv, j0 >> 5);
        const int nb = min(32, hr - j0);
#pragma unroll 8
        for (int jj = 0; jj < nb; jj++) {
            const double tj = shfl_d(tc, jj);
            const float *dr = dq + (size_t)(j0 + jj) * kRefitCP;
            cf0 = fma((double)__ldg(dr + lane), tj, cf0);
            cf1 = fma((double)__ldg(dr + 32 + lane), tj, cf1);
            if (opdt) {
                const double yj = shfl_d(yc, jj);
                const float *br = db + (size_t)(j0 + jj) * kRefitCP;
                cb0 = fma((double)__ldg(br + lane), yj, cb0);
                cb1 = fma((double)__ldg(br + 32 + lane), yj, cb1);
            }
        }
    }
    if (opdt) {
        cf0 -= cb0;
        cf1 -= cb1;
    } else if (lane == 0) {
        cf0 = 0.28209479177387814;  // 1 / (2 sqrt(pi))
    }
    // sphere sampling: lane v accumulates vertices v + 32q over c in order, 8 at a time
    for (int v0 = 0; v0 < V; v0 += 8 * kWarp) {
        double o[8];
#pragma unroll
        for (int q = 0; q < 8; q++) o[q] = 0.0;
#pragma unroll 3
        for (int c = 0; c < C; c++) {
            const double cc = shfl_d(c < 32 ? cf0 : cf1, c & 31);
            const float *sr = smp + (size_t)c * L.vp + v0 + lane;
#pragma unroll
            for (int q = 0; q < 8; q++)
                if (v0 + lane + 32 * q < L.vp) o[q] = fma((double)__ldg(sr + 32 * q), cc, o[q]);
        }
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int v = v0 + lane + 32 * q;
            if (v < V) odf[v] = (float)o[q];
        }
    }
    __syncwarp();
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// One CTA = 128 slots, 16 warps.  Warp w owns TMEM lane quadrant w % 4 for
// the epilogues (the four warps of a quadrant split the columns) and slots
// 8w .. 8w+7 for the warp-cooperative gather and peak search; threads
// 0..127 own slot t's tracking state.
__global__ void __launch_bounds__(kBThreads, 1)
    boot_batch_kernel(DevParams P, BootBatchGeom g, BootBatchArgs A, const int *partner) {
    extern __shared__ unsigned char smraw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smraw) + 1023) & ~(uintptr_t)1023);
    unsigned char *R0 = sm;
    unsigned char *R1 = R0 + g.r0;
    unsigned char *R2 = R1 + g.r1;
    float4 *s_pt = reinterpret_cast<float4 *>(R2 + g.r2);   // [128] position, .w = b0 mean
    float4 *s_dir = s_pt + kSlots;                           // [128] incoming direction
    float4 *s_new = s_dir + kSlots;                          // [128] new direction, .w = found
    int *s_h = reinterpret_cast<int *>(s_new + kSlots);      // [128] half id, -1 = empty
    int *s_live = s_h + kSlots;                              // [128] attempt this iteration
    short *nbr_sh = reinterpret_cast<short *>(s_live + kSlots);  // [V][kMaxDegree]
    int *partner_sh = reinterpret_cast<int *>(nbr_sh + g.nbr_shorts);
    uint64_t *bars = reinterpret_cast<uint64_t *>(partner_sh + kMaxSortLayers * kWarp);
    // bars: 0, 1 = B1 stage loaded; 2, 3 = B1 stage consumed; 4 = MMA batch done; 5 = B2/B3 loaded
    uint32_t *tmem_sh = reinterpret_cast<uint32_t *>(bars + 6);
    float *verts_smem = reinterpret_cast<float *>(tmem_sh + 4);  // [3 V] sphere vertices, when they fit
    const float *verts_sh = g.verts_floats ? verts_smem : P.verts;

    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    const int qd = w & 3, part = w >> 2;        // epilogue: lane quadrant, column share
    const int eslot = qd * 32 + lane;           // epilogue slot of this thread
    for (int i = t; i < kMaxSortLayers * kWarp; i += kBThreads) partner_sh[i] = partner[i];
    for (int i = t; i < g.V * kMaxDegree; i += kBThreads) nbr_sh[i] = A.nbr[i];
    if (g.verts_floats)
        for (int i = t; i < 3 * g.V; i += kBThreads) verts_smem[i] = P.verts[i];
    if (t < kSlots) s_h[t] = -1;
    if (t == 0) {
        for (int b = 0; b < 6; b++) mbar_init(&bars[b], 1);
        mbar_fence_init();
    }
    if (w == 0) tmem_alloc(tmem_sh, kTmemCols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *tmem_sh;
    const uint32_t trow = tbase + ((uint32_t)(qd * 32) << 16);

    uint32_t ph_load[2] = {0, 0}, ph_free[2] = {0, 0}, ph_mma = 0, ph_aux = 0;
    bool ok = true;
    if (t == 0) {
        mbar_arrive_expect_tx(&bars[5], (uint32_t)g.b2_bytes);
        bulk_g2s(R2, A.B2g, (uint32_t)g.b2_bytes, &bars[5]);
        ok = mbar_wait(&bars[5], ph_aux);
        ph_aux ^= 1;
    }

    const uint32_t idesc1 = umma_idesc_bf16(128, g.HP);
    const uint32_t idesc2 = umma_idesc_bf16(128, g.N2);
    const uint32_t idesc3 = umma_idesc_bf16(128, kOdfChunk);
    const uint32_t a1_term = 256 * g.HP, a3_term = 256 * g.N2;
    const uint32_t b1_term = g.b1_chunk / 2, b2_term = g.b2_bytes / 2, b3_term = g.b3_chunk / 2;
    const int imax = P.max_sline_len;

    // tracking state of slot t (threads 0..127)
    int my_h = -1, my_i = 0, my_att = 0;
    float3 my_pt = make_float3(0, 0, 0), my_dir = make_float3(0, 0, 0);
    bool queue_empty = false;
    // bootstrap stream of (epilogue slot, column share)
    Philox rng;
    rng.init(0, 0, 0);
    int rng_h = -1;
    unsigned long long rows_searched = 0, rows_refit = 0;  // lane-uniform per warp
    const int nsl = batch_count(A.nsl_dev, A.nsl);

    for (;;) {
        // ---- refill empty slots from the queue of streamline halves
        if (t < kSlots) {
            if (my_h < 0 && !queue_empty && A.nprobe > 0) {
                const int h = atomicAdd(A.hq, 1);
                if (h >= A.nprobe) {
                    queue_empty = true;
                } else {
                    my_h = h;
                    my_pt = make_float3(A.probe_pts[3 * h], A.probe_pts[3 * h + 1], A.probe_pts[3 * h + 2]);
                    if (A.probe_dirs)
                        my_dir = make_float3(A.probe_dirs[3 * h], A.probe_dirs[3 * h + 1], A.probe_dirs[3 * h + 2]);
                    my_i = 1;
                }
            } else if (my_h < 0 && !queue_empty) {
                const int h = atomicAdd(A.hq, 1);
                if (h >= 2 * nsl) {
                    queue_empty = true;
                } else {
                    my_h = h;
                    const int sl = h >> 1, half = h & 1;
                    const int s = A.sl_seed[sl];
                    const float3 v = vert3(P.verts, (int)A.sl_vert[sl]);
                    my_pt = make_float3(A.seeds[3 * s], A.seeds[3 * s + 1], A.seeds[3 * s + 2]);
                    my_dir = half ? v : make_float3(-v.x, -v.y, -v.z);
                    my_i = 1;
                    my_att = 0;
                    store_pt(A.pts + ((size_t)blockIdx.x * kSlots + t) * (size_t)imax * 3, 0, my_pt);
                }
            }
            s_h[t] = my_h;
            s_live[t] = (my_h >= 0) && (my_i < imax);
            s_pt[t] = make_float4(my_pt.x, my_pt.y, my_pt.z, 1.0f);
            s_dir[t] = make_float4(my_dir.x, my_dir.y, my_dir.z, 0.0f);
        }
        if (__syncthreads_or(!ok)) {
            if (t == 0) atomicOr(A.status, ST_WAIT_TIMEOUT);
            break;
        }
        if (!__syncthreads_or(t < kSlots && my_h >= 0)) break;

        // ---- B1 stages 0 and 1 (R1 is free: the last iteration's MMAs are done)
        if (t == 0) {
            for (int c = 0; c < 2 && c < g.nchunk1; c++) {
                mbar_arrive_expect_tx(&bars[c], (uint32_t)g.b1_chunk);
                bulk_g2s(R1 + c * g.b1_chunk, A.B1g + (size_t)c * g.b1_chunk, (uint32_t)g.b1_chunk, &bars[c]);
            }
        }

        // ---- gather: warp w interpolates slots 8w..8w+7 into A1 rows from the
        //      volume copy whose T axis holds the hr non-b0 volumes first and
        //      the b0s after them (padded to TP = 4k): lane l owns float4 l and
        //      l + 32 of the row; values past hr add up as clamped b0s
        {
            DevParams Pg = P;
            Pg.dimt = g.TP;
            const int nq = g.TP / 4, nw = nq > g.HP / 4 ? nq : g.HP / 4;
            for (int i = 0; i < kSlots / kBWarps; i++) {
                const int slot = w * (kSlots / kBWarps) + i;
                const float4 p4 = s_pt[slot];
                Corners c;
                bool inb = false;
                if (s_live[slot]) inb = trilinear_setup(Pg, make_float3(p4.x, p4.y, p4.z), c);
                float bsum = 0.0f;
#pragma unroll
                for (int r = 0; r < 2; r++) {
                    const int f = lane + 32 * r;
                    if (f >= nw) continue;
                    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (inb && f < nq) {
#pragma unroll
                        for (int q = 0; q < 8; q++) {
                            const float4 d = __ldg(reinterpret_cast<const float4 *>(A.dwi + c.base[q]) + f);
                            acc.x += c.w[q] * d.x;
                            acc.y += c.w[q] * d.y;
                            acc.z += c.w[q] * d.z;
                            acc.w += c.w[q] * d.w;
                        }
                    }
                    float x[4] = {acc.x, acc.y, acc.z, acc.w};
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const int k = 4 * f + e;
                        if (k >= g.hr) {
                            if (inb && k < g.hr + g.nb0) bsum += (P.min_signal > x[e]) ? P.min_signal : x[e];
                            x[e] = 0.0f;
                        }
                    }
                    if (4 * f < g.HP) {
                        const __nv_bfloat162 h01 = __floats2bfloat162_rn(x[0], x[1]);
                        const __nv_bfloat162 h23 = __floats2bfloat162_rn(x[2], x[3]);
                        const float2 f01 = __bfloat1622float2(h01), f23 = __bfloat1622float2(h23);
                        const uint2 hi = make_uint2(*reinterpret_cast<const uint32_t *>(&h01),
                                                    *reinterpret_cast<const uint32_t *>(&h23));
                        const uint2 lo = make_uint2(pack_bf16x2(x[0] - f01.x, x[1] - f01.y),
                                                    pack_bf16x2(x[2] - f23.x, x[3] - f23.y));
                        const uint32_t off = kmajor_off(slot, 4 * f, kSlots);
                        *reinterpret_cast<uint2 *>(R0 + off) = hi;
                        *reinterpret_cast<uint2 *>(R0 + a1_term + off) = lo;
                    }
                }
#pragma unroll
                for (int o = 16; o; o >>= 1) bsum += __shfl_xor_sync(FULL, bsum, o);
                if (lane == 0) {
                    s_pt[slot].w = bsum / (float)g.nb0;
                    s_live[slot] = inb ? 1 : 0;  // outside the data: every attempt would fail
                }
            }
        }
        fence_async_smem();
        __syncthreads();

        // ---- MMA 1: D1[:, 0:HP) = A1 R^T, D1[:, HP:2HP) = A1 H^T
        if (t == 0 && ok) {
            tc_fence_after();
            for (int c = 0; c < g.nchunk1 && ok; c++) {
                const int st = c & 1;
                ok = mbar_wait(&bars[st], ph_load[st]);
                ph_load[st] ^= 1;
                if (!ok) break;
                const uint32_t bst = smem_u32(R1 + st * g.b1_chunk);
#pragma unroll
                for (int kk = 0; kk < 2; kk++) {
                    const int k16 = 2 * c + kk;
#pragma unroll
                    for (int term = 0; term < 3; term++) {
                        const uint32_t aoff = (term == 2 ? a1_term : 0) + (uint32_t)(k16 * 2) * (kSlots * 16);
                        const uint32_t boff = (term == 1 ? b1_term : 0) + (uint32_t)(kk * 2) * (g.N1 * 16);
                        const uint64_t ad = umma_sdesc(smem_u32(R0) + aoff, kSlots * 16, 128);
#pragma unroll
                        for (int nb = 0; nb < 2; nb++) {
                            const uint64_t bd =
                                umma_sdesc(bst + boff + (uint32_t)(nb * g.HP / 8) * 128, g.N1 * 16, 128);
                            umma_bf16(tbase + nb * g.HP, ad, bd, idesc1, (k16 > 0 || term > 0) ? 1u : 0u);
                        }
                    }
                }
                if (c + 2 < g.nchunk1) {
                    umma_commit(&bars[2 + st]);
                    ok = mbar_wait(&bars[2 + st], ph_free[st]);
                    ph_free[st] ^= 1;
                    if (!ok) break;
                    mbar_arrive_expect_tx(&bars[st], (uint32_t)g.b1_chunk);
                    bulk_g2s(R1 + st * g.b1_chunk, A.B1g + (size_t)(c + 2) * g.b1_chunk, (uint32_t)g.b1_chunk,
                             &bars[st]);
                }
            }
            umma_commit(&bars[4]);
        }
        if (!mbar_wait(&bars[4], ph_mma)) ok = false;
        ph_mma ^= 1;
        tc_fence_after();

        // ---- epilogue 1: residuals to shared memory (this thread's column
        //      blocks), then bootstrap, clamp, normalise, transform -> A2
        //      (CSA: log(-log x); OPDT: -log x (1.5 + log x) x, with x itself
        //      kept in the freed TMEM columns [0, HP) for the second product)
        float *rb = reinterpret_cast<float *>(R0) + (size_t)eslot * (g.hr + 1);
        const int nblk1 = g.HP / 16;
        for (int b = part; b < nblk1; b += 4) {
            float v[16];
            tmem_ld16(trow + 16 * b, v);
#pragma unroll
            for (int q = 0; q < 16; q++)
                if (16 * b + q < g.hr) rb[16 * b + q] = v[q];
        }
        __syncthreads();
        {
            const int h = s_h[eslot];
            const bool live = s_live[eslot] != 0;
            const float denom = s_pt[eslot].w;
            const int *pidx = A.nprobe > 0 ? A.probe_idx + (size_t)(h >= 0 ? h : 0) * g.hr : nullptr;
            if (live && !pidx && h != rng_h) {
                const int sl = h >> 1, half = h & 1;
                rng.init(P.rng_seed,
                         kBatchSubseqBase + 8ull * (unsigned long long)(sl + A.rng_base) + 4 * half + part, 0);
                rng_h = h;
            }
            if (live && !pidx && A.refit) {
                uint32_t *sv = A.rng_save + (((size_t)blockIdx.x * kSlots + eslot) * 4 + part) * 5;
                sv[0] = rng.ctr.x;
                sv[1] = rng.ctr.y;
                sv[2] = rng.ctr.z;
                sv[3] = rng.ctr.w;
                sv[4] = (uint32_t)rng.idx;
            }
            const bool opdt = P.model == OPDT;
            for (int b = part; b < nblk1; b += 4) {
                float hv[16], xs[16];
                tmem_ld16(trow + g.HP + 16 * b, hv);
#pragma unroll
                for (int gq = 0; gq < 2; gq++) {
                    float y[8];
#pragma unroll
                    for (int e = 0; e < 8; e++) {
                        const int j = 16 * b + gq * 8 + e;
                        y[e] = 0.0f;
                        xs[gq * 8 + e] = 0.0f;
                        if (live && j < g.hr) {
                            const int src = pidx ? pidx[j] : (int)(rng.next() % (unsigned)g.hr);
                            float x = hv[gq * 8 + e] + rb[src];
                            x = (P.min_signal > x) ? P.min_signal : x;
                            x = x / denom;
                            if (opdt) {
                                const float ONEP5 = 1.5f;
                                y[e] = -__logf(x) * (ONEP5 + __logf(x)) * x;
                                xs[gq * 8 + e] = x;
                            } else {
                                const float lo_c = 0.001f, hi_c = 0.999f;
                                float cc = (x > lo_c) ? x : lo_c;
                                cc = (cc < hi_c) ? cc : hi_c;
                                y[e] = __logf(-__logf(cc));
                            }
                        }
                    }
                    uint4 hi, lo;
                    split8(y, hi, lo);
                    const uint32_t off = kmajor_off(eslot, 16 * b + gq * 8, kSlots);
                    *reinterpret_cast<uint4 *>(R1 + off) = hi;
                    *reinterpret_cast<uint4 *>(R1 + a1_term + off) = lo;
                }
                if (opdt) tmem_st16(trow + 16 * b, xs);
            }
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();

        // ---- MMA 2: D2 = A2 Delta^T  (TMEM columns [N1, N1 + N2))
        if (t == 0 && ok) {
            tc_fence_after();
            for (int k16 = 0; k16 < g.HP / 16; k16++) {
#pragma unroll
                for (int term = 0; term < 3; term++) {
                    const uint32_t aoff = (term == 2 ? a1_term : 0) + (uint32_t)(k16 * 2) * (kSlots * 16);
                    const uint32_t boff = (term == 1 ? b2_term : 0) + (uint32_t)(k16 * 2) * (g.N2 * 16);
                    umma_bf16(tbase + g.N1, umma_sdesc(smem_u32(R1) + aoff, kSlots * 16, 128),
                              umma_sdesc(smem_u32(R2) + boff, g.N2 * 16, 128), idesc2,
                              (k16 > 0 || term > 0) ? 1u : 0u);
                }
            }
            umma_commit(&bars[4]);
        }
        if (!mbar_wait(&bars[4], ph_mma)) ok = false;
        ph_mma ^= 1;
        tc_fence_after();

        // ---- OPDT: D2 += x (-Delta_b)^T, x back from TMEM into A2 (R1), the
        //      packed -Delta_b streamed into R0 (the residual buffer is dead)
        if (P.model == OPDT) {
            if (t == 0 && ok) {
                mbar_arrive_expect_tx(&bars[5], (uint32_t)g.b2_bytes);
                bulk_g2s(R0, A.B2g + g.b2_bytes, (uint32_t)g.b2_bytes, &bars[5]);
            }
            for (int b = part; b < g.HP / 16; b += 4) {
                float xv[16];
                tmem_ld16(trow + 16 * b, xv);
#pragma unroll
                for (int gq = 0; gq < 2; gq++) {
                    float x[8];
#pragma unroll
                    for (int e = 0; e < 8; e++) x[e] = xv[gq * 8 + e];
                    uint4 hi, lo;
                    split8(x, hi, lo);
                    const uint32_t off = kmajor_off(eslot, 16 * b + gq * 8, kSlots);
                    *reinterpret_cast<uint4 *>(R1 + off) = hi;
                    *reinterpret_cast<uint4 *>(R1 + a1_term + off) = lo;
                }
            }
            fence_async_smem();
            tc_fence_before();
            __syncthreads();
            if (t == 0 && ok) {
                ok = mbar_wait(&bars[5], ph_aux);
                ph_aux ^= 1;
                if (ok) {
                    tc_fence_after();
                    for (int k16 = 0; k16 < g.HP / 16; k16++) {
#pragma unroll
                        for (int term = 0; term < 3; term++) {
                            const uint32_t aoff = (term == 2 ? a1_term : 0) + (uint32_t)(k16 * 2) * (kSlots * 16);
                            const uint32_t boff = (term == 1 ? b2_term : 0) + (uint32_t)(k16 * 2) * (g.N2 * 16);
                            umma_bf16(tbase + g.N1, umma_sdesc(smem_u32(R1) + aoff, kSlots * 16, 128),
                                      umma_sdesc(smem_u32(R0) + boff, g.N2 * 16, 128), idesc2, 1u);
                        }
                    }
                }
                umma_commit(&bars[4]);
            }
            if (!mbar_wait(&bars[4], ph_mma)) ok = false;
            ph_mma ^= 1;
            tc_fence_after();
        }

        // ---- the first B3 chunk streams into R1 (free: the second product has
        //      completed) while epilogue 2 runs
        if (t == 0 && ok) {
            mbar_arrive_expect_tx(&bars[5], (uint32_t)g.b3_chunk);
            bulk_g2s(R1, A.B3g, (uint32_t)g.b3_chunk, &bars[5]);
        }

        // ---- epilogue 2: SH coefficients -> A3 (coefficient 0 fixed, boot.cu CSA branch)
        for (int b = part; b < g.N2 / 16; b += 4) {
            float v[16];
            tmem_ld16(trow + g.N1 + 16 * b, v);
#pragma unroll
            for (int gq = 0; gq < 2; gq++) {
                float x[8];
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const int k = 16 * b + gq * 8 + e;
                    x[e] = (k == 0 && P.model == CSA) ? kN0Const : (k < g.C ? v[gq * 8 + e] : 0.0f);
                }
                uint4 hi, lo;
                split8(x, hi, lo);
                const uint32_t off = kmajor_off(eslot, 16 * b + gq * 8, kSlots);
                *reinterpret_cast<uint4 *>(R0 + off) = hi;
                *reinterpret_cast<uint4 *>(R0 + a3_term + off) = lo;
            }
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();

        // ---- MMA 3 in 256-vertex chunks: ODF rows -> L2 scratch
        float *e_odf = A.odf + ((size_t)blockIdx.x * kSlots + eslot) * g.vstride;
        if (A.nprobe > 0 && s_live[eslot]) e_odf = A.probe_odf + (size_t)s_h[eslot] * A.probe_stride;
        for (int ch = 0; ch < g.nchunk3; ch++) {
            if (t == 0 && ok) {
                ok = mbar_wait(&bars[5], ph_aux);  // chunk ch (issued before epilogue 2 or the last epilogue)
                ph_aux ^= 1;
                if (ok) {
                    tc_fence_after();
                    for (int k16 = 0; k16 < g.N2 / 16; k16++) {
#pragma unroll
                        for (int term = 0; term < 3; term++) {
                            const uint32_t aoff =
                                (term == 2 ? a3_term : 0) + (uint32_t)(k16 * 2) * (kSlots * 16);
                            const uint32_t boff =
                                (term == 1 ? b3_term : 0) + (uint32_t)(k16 * 2) * (kOdfChunk * 16);
                            umma_bf16(tbase, umma_sdesc(smem_u32(R0) + aoff, kSlots * 16, 128),
                                      umma_sdesc(smem_u32(R1) + boff, kOdfChunk * 16, 128), idesc3,
                                      (k16 > 0 || term > 0) ? 1u : 0u);
                        }
                    }
                }
                umma_commit(&bars[4]);
            }
            if (!mbar_wait(&bars[4], ph_mma)) ok = false;
            ph_mma ^= 1;
            tc_fence_after();
            // the next chunk streams into R1 (this chunk's product has read it) during this epilogue
            if (t == 0 && ok && ch + 1 < g.nchunk3) {
                mbar_arrive_expect_tx(&bars[5], (uint32_t)g.b3_chunk);
                bulk_g2s(R1, A.B3g + (size_t)(ch + 1) * g.b3_chunk, (uint32_t)g.b3_chunk, &bars[5]);
            }
            for (int b = part; b < kOdfChunk / 16; b += 4) {
                float v[16];
                tmem_ld16(trow + 16 * b, v);
                const int vb = ch * kOdfChunk + 16 * b;
                if (vb + 16 <= g.V) {
#pragma unroll
                    for (int q = 0; q < 16; q += 4)
                        __stcg(reinterpret_cast<float4 *>(e_odf + vb + q),
                               make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]));
                } else {
#pragma unroll
                    for (int q = 0; q < 16; q++)
                        if (vb + q < g.V) e_odf[vb + q] = v[q];
                }
            }
            tc_fence_before();
            __syncthreads();
        }

        if (A.nprobe > 0 && !A.probe_dirs) {  // probe mode: the ODF rows are the output
            if (t < kSlots) my_h = -1;
            continue;
        }

        // ---- peaks and closest peak: warp w searches slots 8w..8w+7; the
        //      next live slot's ODF row is copied in while this one is searched
        {
            float *obuf = reinterpret_cast<float *>(R0) + (size_t)w * 3 * g.vstride;
            int *ind_sh = reinterpret_cast<int *>(obuf + 2 * g.vstride);
            const int base = w * (kSlots / kBWarps);
            unsigned live = 0;
            for (int i = 0; i < kSlots / kBWarps; i++) live |= (s_live[base + i] ? 1u : 0u) << i;
            const int nch = g.vstride / 4;
            auto fetch = [&](int slot, float *dst) {
                const float *src = A.nprobe > 0 ? A.probe_odf + (size_t)s_h[slot] * A.probe_stride
                                                : A.odf + ((size_t)blockIdx.x * kSlots + slot) * g.vstride;
                for (int c = lane; c < nch; c += kWarp) cp_async16(dst + 4 * c, src + 4 * c);
            };
            int cur = live ? __ffs(live) - 1 : -1;
            if (cur >= 0) fetch(base + cur, obuf);
            cp_async_commit();
            int buf = 0;
            while (cur >= 0) {
                const unsigned rest = live & ~((2u << cur) - 1u);
                const int nxt = rest ? __ffs(rest) - 1 : -1;
                if (nxt >= 0) fetch(base + nxt, obuf + (buf ^ 1) * g.vstride);
                cp_async_commit();
                cp_async_wait1();
                __syncwarp();
                float *odf_sh = obuf + buf * g.vstride;
                const int slot = base + cur;
                int ndir = -1;
                bool refitted = false;
                for (int pass = 0; pass < 2; pass++) {
                    ndir = peaks_fast(P, verts_sh, odf_sh, ind_sh, g.V, nbr_sh, partner_sh, lane);
                    if (ndir < 0) {
                        float m = -FLT_MAX;
                        for (int v = lane; v < g.V; v += kWarp) m = fmax_ref(m, odf_sh[v]);
                        m = warp_max_ref(m);
                        ndir = peaks_sparse(P, verts_sh, odf_sh, ind_sh, g.V, m, nbr_sh, partner_sh, lane);
                    }
                    if (pass == 1 || !A.refit) break;
                    rows_searched++;
                    if (!near_tie(P, verts_sh, odf_sh, ind_sh, ndir, g.V, nbr_sh, A.refit_tol, lane)) break;
                    // the decision is within the BF16x3 error: fit this row again in float64
                    const int h = s_h[slot];
                    boot_refit_fp64(P, g.hr, g.HP / 16, A.volidx, s_pt[slot],
                                    A.nprobe > 0 ? A.probe_idx + (size_t)h * g.hr : nullptr,
                                    A.rng_save + ((size_t)blockIdx.x * kSlots + slot) * 20, A.refit_tab,
                                    A.refit_idx + ((size_t)blockIdx.x * kBWarps + w) * kRefitIdx, odf_sh, lane);
                    refitted = true;
                    rows_refit++;
                }
                int found = 0;
                float3 pk = make_float3(0, 0, 0);
                if (ndir > 0) {
                    const float4 d4 = s_dir[slot];
                    found = closest_peak(P, verts_sh, make_float3(d4.x, d4.y, d4.z), ndir, ind_sh, lane, &pk);
                }
                __syncwarp();
                if (lane == 0) {
                    s_new[slot] = make_float4(pk.x, pk.y, pk.z, found ? 1.0f : 0.0f);
                    if (A.nprobe > 0)
                        reinterpret_cast<float4 *>(A.probe_step)[s_h[slot]] =
                            make_float4(pk.x, pk.y, pk.z, (found ? 1.0f : 0.0f) + (refitted ? 2.0f : 0.0f));
                }
                cur = nxt;
                buf ^= 1;
            }
            asm volatile("cp.async.wait_all;" ::: "memory");
        }
        __syncthreads();
        if (A.nprobe > 0) {  // probe mode with directions: one search per item
            if (t < kSlots) my_h = -1;
            continue;
        }

        // ---- step (tracker_boot_d, boot.cu:725-824): one attempt per iteration
        if (w < kSlots / kWarp) {
            bool done = false;
            int nsteps = 0;
            if (my_h >= 0) {
                const float4 nw = s_new[t];
                if (!s_live[t]) {
                    done = true;  // no step left, or outside the data: every attempt would fail
                    nsteps = my_i;
                } else if (nw.w != 0.0f) {
                    my_dir = make_float3(nw.x, nw.y, nw.z);
                    const double ss = P.step_size;
                    my_pt.x = (float)fma((double)my_dir.x, ss, (double)my_pt.x);
                    my_pt.y = (float)fma((double)my_dir.y, ss, (double)my_pt.y);
                    my_pt.z = (float)fma((double)my_dir.z, ss, (double)my_pt.z);
                    store_pt(A.pts + ((size_t)blockIdx.x * kSlots + t) * (size_t)imax * 3, my_i, my_pt);
                    my_att = 0;
                    if (check_point(P, my_pt) != TRACKPOINT) {
                        done = true;
                        nsteps = my_i;
                    } else if (++my_i >= imax) {
                        done = true;
                        nsteps = my_i;
                    }
                } else if (++my_att >= kBootAttempts) {
                    done = true;
                    nsteps = my_i;
                }
            }

            // finished halves: append their points to the pool
            __syncwarp();
            unsigned dm = __ballot_sync(FULL, done);
            while (dm) {
                const int i = __ffs(dm) - 1;
                dm &= dm - 1;
                const int n = __shfl_sync(FULL, nsteps, i);
                const int h = __shfl_sync(FULL, my_h, i);
                const float *src = A.pts + ((size_t)blockIdx.x * kSlots + w * 32 + i) * (size_t)imax * 3;
                unsigned long long off = 0;
                if (lane == 0) off = atomicAdd(A.pool_count, (unsigned long long)n);
                off = __shfl_sync(FULL, off, 0);
                long long o = -1;
                if (off + (unsigned long long)n <= A.pool_cap) {
                    o = (long long)off;
                    for (int j = lane; j < 3 * n; j += kWarp) A.pool[3 * off + j] = __ldcg(src + j);
                } else if (lane == 0) {
                    atomicOr(A.status, ST_POOL_OVERFLOW);
                }
                if (lane == 0) {
                    A.half_len[h] = n;
                    A.half_off[h] = o;
                }
            }
            if (done) my_h = -1;
        }
    }

    if (A.refit && A.refit_count && lane == 0 && rows_searched) {
        atomicAdd(A.refit_count, rows_searched);
        atomicAdd(A.refit_count + 1, rows_refit);
    }
    // ---- teardown: every MMA has completed (each batch was waited for)
    tc_fence_before();
    __syncthreads();
    if (w == 0) {
        tc_fence_after();
        tmem_dealloc(tbase, kTmemCols);
    }
}

// ---------------------------------------------------------------------------
// launchers

cudaError_t launch_boot_batch_pack(const DevParams &P, const BootBatchGeom &g, void *B1g, void *B2g,
                                   void *B3g, cudaStream_t st) {
    boot_batch_pack_kernel<<<256, 256, 0, st>>>(P, g, reinterpret_cast<__nv_bfloat16 *>(B1g),
                                                 reinterpret_cast<__nv_bfloat16 *>(B2g),
                                                 reinterpret_cast<__nv_bfloat16 *>(B3g));
    return cudaGetLastError();
}

cudaError_t launch_boot_batch_dwi(const float *src, const int *volidx, long long nvox, int T, int TP,
                                  float *dst, cudaStream_t st) {
    boot_batch_dwi_kernel<<<1024, 256, 0, st>>>(src, volidx, nvox, T, TP, dst);
    return cudaGetLastError();
}

cudaError_t launch_boot_batch_prep(const int *npeaks, const int *sl_off, const short *peaks, int max_store,
                                   int n, int cap, int *sl_seed, short *sl_vert, int *status, cudaStream_t st) {
    const int grid = std::max(1, std::min((n + 255) / 256, 4096));
    boot_batch_prep_kernel<<<grid, 256, 0, st>>>(npeaks, sl_off, peaks, max_store, n, cap, sl_seed, sl_vert,
                                                 status);
    return cudaGetLastError();
}

cudaError_t launch_boot_batch_join(const int *half_len, const int *sl_seed, int nsl, const int *count,
                                   int *out_len, int *out_seed, cudaStream_t st) {
    const int grid = std::max(1, std::min((nsl + 255) / 256, 4096));
    boot_batch_join_kernel<<<grid, 256, 0, st>>>(half_len, sl_seed, nsl, count, out_len, out_seed);
    return cudaGetLastError();
}

cudaError_t launch_gather_halves(const float *pool, const long long *half_off, const int *half_len,
                                 const long long *pt_off, int nsl, const int *count, const int *status,
                                 float *out, int grid, cudaStream_t st) {
    gather_halves_kernel<<<grid, 256, 0, st>>>(pool, half_off, half_len, pt_off, nsl, count, status, out);
    return cudaGetLastError();
}

cudaError_t boot_batch_set_smem(const BootBatchGeom &g) {
    return raise_smem_limit(boot_batch_kernel, g.smem);
}

cudaError_t launch_boot_batch(const DevParams &P, const BootBatchGeom &g, const BootBatchArgs &A,
                              const int *partner, int grid, cudaStream_t st) {
    const cudaError_t e = raise_smem_limit(boot_batch_kernel, g.smem);
    if (e != cudaSuccess) return e;
    boot_batch_kernel<<<grid, kBThreads, g.smem, st>>>(P, g, A, partner);
    return cudaGetLastError();
}

}  // namespace csl
