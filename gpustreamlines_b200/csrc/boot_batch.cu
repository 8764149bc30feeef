// Batched residual-bootstrap tracking on the tensor cores (CSA model).
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
//             transform log(-log(x))                             -> A2 [128 x K1]
//   MMA 2     A2 x Delta^T                                       -> D2 [128 x C]     (TMEM)
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
constexpr int kBThreads = 128;      // one thread per slot, 4 warps
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
    g.b1_chunk = 128 * g.N1;          // 2 terms x N1 rows x 32 k x 2 B
    g.b2_bytes = 4 * g.N2 * g.HP;     // 2 terms x N2 rows x HP k x 2 B
    g.b3_chunk = 1024 * g.N2;         // 2 terms x 256 rows x N2 k x 2 B
    const int a1 = 512 * g.HP, rbuf = 512 * (hr + 1), a3 = 512 * g.N2, pk = 32 * g.vstride;
    g.r0 = round_up(std::max(std::max(a1, rbuf), std::max(a3, pk)), 1024);
    g.r1 = round_up(std::max(std::max(2 * g.b1_chunk, 512 * g.HP), g.b3_chunk), 1024);
    g.r2 = round_up(g.b2_bytes, 1024);
    g.smem = 1024 + g.r0 + g.r1 + g.r2 + 4 * g.HP * 4 + kMaxSortLayers * kWarp * 4 + 128;
    return g;
}

// ---------------------------------------------------------------------------
// set-up: the three matrices in the operand layout of tc.cuh, BF16 hi / lo

__global__ void boot_batch_pack_kernel(DevParams P, BootBatchGeom g, __nv_bfloat16 *B1g,
                                       __nv_bfloat16 *B2g, __nv_bfloat16 *B3g) {
    const long long n1 = (long long)g.N1 * g.HP, n2 = (long long)g.N2 * g.HP;
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
            const long long f = e - n1;
            const int n = (int)(f / g.HP), k = (int)(f % g.HP);
            x = (n < g.C && k < g.hr) ? P.delta_q[(size_t)n * g.hr + k] : 0.0f;
            hi = reinterpret_cast<char *>(B2g);
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

// streamline -> (seed, initial vertex) from the pass-1 outputs
__global__ void boot_batch_prep_kernel(const int *__restrict__ npeaks, const int *__restrict__ sl_off,
                                       const short *__restrict__ peaks, int max_store, int n,
                                       int *sl_seed, short *sl_vert, int *status) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const int np = npeaks[s], base = sl_off[s];
        if (np > max_store) atomicOr(status, ST_PEAKS_OVERFLOW);
        const int m = np < max_store ? np : max_store;
        for (int k = 0; k < m; k++) {
            sl_seed[base + k] = s;
            sl_vert[base + k] = peaks[(size_t)s * max_store + k];
        }
    }
}

// streamline length = backward half + forward half - the shared seed point
__global__ void boot_batch_join_kernel(const int *__restrict__ half_len, const int *__restrict__ sl_seed,
                                       int nsl, int *out_len, int *out_seed) {
    for (int sl = blockIdx.x * blockDim.x + threadIdx.x; sl < nsl; sl += gridDim.x * blockDim.x) {
        out_len[sl] = half_len[2 * sl] - 1 + half_len[2 * sl + 1];
        out_seed[sl] = sl_seed[sl];
    }
}

// reversed backward half, then the forward half without its seed point
__global__ void gather_halves_kernel(const float *__restrict__ pool, const long long *__restrict__ half_off,
                                     const int *__restrict__ half_len, const long long *__restrict__ pt_off,
                                     int nsl, float *__restrict__ out) {
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

__global__ void __launch_bounds__(kBThreads, 1)
    boot_batch_kernel(DevParams P, BootBatchGeom g, BootBatchArgs A, const int *partner) {
    extern __shared__ unsigned char smraw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smraw) + 1023) & ~(uintptr_t)1023);
    unsigned char *R0 = sm;
    unsigned char *R1 = R0 + g.r0;
    unsigned char *R2 = R1 + g.r1;
    float *sig = reinterpret_cast<float *>(R2 + g.r2);
    int *partner_sh = reinterpret_cast<int *>(sig + 4 * g.HP);
    uint64_t *bars = reinterpret_cast<uint64_t *>(partner_sh + kMaxSortLayers * kWarp);
    // bars: 0, 1 = B1 stage loaded; 2, 3 = B1 stage consumed; 4 = MMA batch done; 5 = B2/B3 loaded
    uint32_t *tmem_sh = reinterpret_cast<uint32_t *>(bars + 6);

    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    for (int i = t; i < kMaxSortLayers * kWarp; i += kBThreads) partner_sh[i] = partner[i];
    if (t == 0) {
        for (int b = 0; b < 6; b++) mbar_init(&bars[b], 1);
        mbar_fence_init();
    }
    if (w == 0) tmem_alloc(tmem_sh, kTmemCols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *tmem_sh;
    const uint32_t trow = tbase + ((uint32_t)(w * 32) << 16);

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
    const int T = P.dimt;
    const int slot_g = blockIdx.x * kSlots + t;
    float *my_pts = A.pts + (size_t)slot_g * (size_t)imax * 3;
    float *my_odf = A.odf + (size_t)slot_g * g.vstride;

    int my_h = -1, my_i = 0, my_att = 0;
    float3 my_pt = make_float3(0, 0, 0), my_dir = make_float3(0, 0, 0);
    bool my_valid = false, queue_empty = false;
    float my_denom = 1.0f;
    Philox rng;
    rng.init(0, 0, 0);

    for (;;) {
        // ---- refill empty slots from the queue of streamline halves
        if (my_h < 0 && !queue_empty) {
            const int h = atomicAdd(A.hq, 1);
            if (h >= 2 * A.nsl) {
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
                rng.init(P.rng_seed, kBatchSubseqBase + 2ull * (unsigned long long)(sl + A.rng_base) + half,
                         0);
                store_pt(my_pts, 0, my_pt);
            }
        }
        if (__syncthreads_or(!ok)) {
            if (t == 0) atomicOr(A.status, ST_WAIT_TIMEOUT);
            break;
        }
        if (!__syncthreads_or(my_h >= 0)) break;
        const bool attempt = (my_h >= 0) && (my_i < imax);

        // ---- B1 stages 0 and 1 (R1 is free: the last iteration's MMAs are done)
        if (t == 0) {
            for (int c = 0; c < 2 && c < g.nchunk1; c++) {
                mbar_arrive_expect_tx(&bars[c], (uint32_t)g.b1_chunk);
                bulk_g2s(R1 + c * g.b1_chunk, A.B1g + (size_t)c * g.b1_chunk, (uint32_t)g.b1_chunk, &bars[c]);
            }
        }

        // ---- gather: the warp interpolates its 32 slots' signals into A1 rows
        {
            float *sg = sig + w * g.HP;
            const unsigned am = __ballot_sync(FULL, attempt);
            bool vmine = false;
            float dmine = 1.0f;
            for (int i = 0; i < kWarp; i++) {
                const int slot = w * 32 + i;
                const float3 p = make_float3(__shfl_sync(FULL, my_pt.x, i), __shfl_sync(FULL, my_pt.y, i),
                                             __shfl_sync(FULL, my_pt.z, i));
                Corners c;
                bool inb = false;
                if ((am >> i) & 1u) inb = trilinear_setup(P, p, c);
                float bsum = 0.0f;
                if (inb) {
                    for (int tt = lane; tt < T; tt += kWarp) {
                        const float v = trilinear_elem(P.dataf, c, tt);
                        const int k = __ldg(A.nbpos + tt);
                        if (k >= 0)
                            sg[k] = v;
                        else
                            bsum += (P.min_signal > v) ? P.min_signal : v;
                    }
                }
#pragma unroll
                for (int o = 16; o; o >>= 1) bsum += __shfl_xor_sync(FULL, bsum, o);
                __syncwarp();
                for (int gq = lane; gq < g.HP / 8; gq += kWarp) {
                    float x[8];
#pragma unroll
                    for (int e = 0; e < 8; e++) {
                        const int k = gq * 8 + e;
                        x[e] = (inb && k < g.hr) ? sg[k] : 0.0f;
                    }
                    uint4 hi, lo;
                    split8(x, hi, lo);
                    const uint32_t off = kmajor_off(slot, gq * 8, kSlots);
                    *reinterpret_cast<uint4 *>(R0 + off) = hi;
                    *reinterpret_cast<uint4 *>(R0 + a1_term + off) = lo;
                }
                __syncwarp();
                if (lane == i) {
                    vmine = inb;
                    dmine = bsum / (float)g.nb0;
                }
            }
            my_valid = vmine;
            my_denom = dmine;
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

        // ---- epilogue 1: residuals to shared memory, bootstrap, CSA transform -> A2
        {
            float *rb = reinterpret_cast<float *>(R0) + (size_t)t * (g.hr + 1);
            for (int c0 = 0; c0 < g.HP; c0 += 16) {
                float v[16];
                tmem_ld16(trow + c0, v);
#pragma unroll
                for (int q = 0; q < 16; q++)
                    if (c0 + q < g.hr) rb[c0 + q] = v[q];
            }
            const bool live = attempt && my_valid;
            for (int c0 = 0; c0 < g.HP; c0 += 16) {
                float hv[16];
                tmem_ld16(trow + g.HP + c0, hv);
#pragma unroll
                for (int gq = 0; gq < 2; gq++) {
                    float y[8];
#pragma unroll
                    for (int e = 0; e < 8; e++) {
                        const int j = c0 + gq * 8 + e;
                        y[e] = 0.0f;
                        if (live && j < g.hr) {
                            const int src = (int)(rng.next() % (unsigned)g.hr);
                            float x = hv[gq * 8 + e] + rb[src];
                            x = (P.min_signal > x) ? P.min_signal : x;
                            x = x / my_denom;
                            const float lo_c = 0.001f, hi_c = 0.999f;
                            float cc = (x > lo_c) ? x : lo_c;
                            cc = (cc < hi_c) ? cc : hi_c;
                            y[e] = __logf(-__logf(cc));
                        }
                    }
                    uint4 hi, lo;
                    split8(y, hi, lo);
                    const uint32_t off = kmajor_off(t, c0 + gq * 8, kSlots);
                    *reinterpret_cast<uint4 *>(R1 + off) = hi;
                    *reinterpret_cast<uint4 *>(R1 + a1_term + off) = lo;
                }
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

        // ---- epilogue 2: SH coefficients -> A3 (coefficient 0 fixed, boot.cu CSA branch)
        for (int c0 = 0; c0 < g.N2; c0 += 16) {
            float v[16];
            tmem_ld16(trow + g.N1 + c0, v);
#pragma unroll
            for (int gq = 0; gq < 2; gq++) {
                float x[8];
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const int k = c0 + gq * 8 + e;
                    x[e] = (k == 0) ? kN0Const : (k < g.C ? v[gq * 8 + e] : 0.0f);
                }
                uint4 hi, lo;
                split8(x, hi, lo);
                const uint32_t off = kmajor_off(t, c0 + gq * 8, kSlots);
                *reinterpret_cast<uint4 *>(R0 + off) = hi;
                *reinterpret_cast<uint4 *>(R0 + a3_term + off) = lo;
            }
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();

        // ---- MMA 3 in 256-vertex chunks: ODF rows -> L2 scratch
        for (int ch = 0; ch < g.nchunk3; ch++) {
            if (t == 0 && ok) {
                mbar_arrive_expect_tx(&bars[5], (uint32_t)g.b3_chunk);
                bulk_g2s(R1, A.B3g + (size_t)ch * g.b3_chunk, (uint32_t)g.b3_chunk, &bars[5]);
                ok = mbar_wait(&bars[5], ph_aux);
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
            for (int c0 = 0; c0 < kOdfChunk; c0 += 16) {
                float v[16];
                tmem_ld16(trow + c0, v);
                const int vb = ch * kOdfChunk + c0;
                if (vb + 16 <= g.V) {
#pragma unroll
                    for (int q = 0; q < 16; q += 4)
                        __stcg(reinterpret_cast<float4 *>(my_odf + vb + q),
                               make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]));
                } else {
#pragma unroll
                    for (int q = 0; q < 16; q++)
                        if (vb + q < g.V) my_odf[vb + q] = v[q];
                }
            }
            tc_fence_before();
            __syncthreads();
        }

        // ---- peaks and closest peak: one warp per slot, the plain getter's code
        bool my_found = false;
        float3 my_new = make_float3(0, 0, 0);
        {
            float *odf_sh = reinterpret_cast<float *>(R0) + (size_t)w * 2 * g.vstride;
            int *ind_sh = reinterpret_cast<int *>(odf_sh + g.vstride);
            const unsigned am = __ballot_sync(FULL, attempt && my_valid);
            for (int i = 0; i < kWarp; i++) {
                if (!((am >> i) & 1u)) continue;
                const float *src = A.odf + ((size_t)blockIdx.x * kSlots + w * 32 + i) * g.vstride;
                for (int v = lane; v < g.V; v += kWarp) odf_sh[v] = __ldcg(src + v);
                __syncwarp();
                const float3 di = make_float3(__shfl_sync(FULL, my_dir.x, i), __shfl_sync(FULL, my_dir.y, i),
                                              __shfl_sync(FULL, my_dir.z, i));
                float m = -FLT_MAX;
                for (int v = lane; v < g.V; v += kWarp) m = fmax_ref(m, odf_sh[v]);
                m = warp_max_ref(m);
                const float thr = (float)(P.pmf_threshold * (double)m);
                __syncwarp();
                for (int v = lane; v < g.V; v += kWarp)
                    if (odf_sh[v] < thr) odf_sh[v] = 0;
                __syncwarp();
                const int ndir = peak_directions(P, odf_sh, ind_sh, g.V, partner_sh, lane);
                int found = 0;
                float3 pk = make_float3(0, 0, 0);
                if (ndir > 0) found = closest_peak(P, di, ndir, ind_sh, lane, &pk);
                __syncwarp();
                if (lane == i) {
                    my_found = found != 0;
                    my_new = pk;
                }
            }
        }

        // ---- step (tracker_boot_d, boot.cu:725-824): one attempt per iteration
        bool done = false;
        int nsteps = 0;
        if (my_h >= 0) {
            if (!attempt || !my_valid) {
                done = true;  // no step left, or outside the data: every attempt would fail
                nsteps = my_i;
            } else if (my_found) {
                my_dir = my_new;
                const double ss = P.step_size;
                my_pt.x = (float)fma((double)my_dir.x, ss, (double)my_pt.x);
                my_pt.y = (float)fma((double)my_dir.y, ss, (double)my_pt.y);
                my_pt.z = (float)fma((double)my_dir.z, ss, (double)my_pt.z);
                store_pt(my_pts, my_i, my_pt);
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

        // ---- finished halves: append their points to the pool
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

cudaError_t launch_boot_batch_prep(const int *npeaks, const int *sl_off, const short *peaks, int max_store,
                                   int n, int *sl_seed, short *sl_vert, int *status, cudaStream_t st) {
    const int grid = std::max(1, std::min((n + 255) / 256, 4096));
    boot_batch_prep_kernel<<<grid, 256, 0, st>>>(npeaks, sl_off, peaks, max_store, n, sl_seed, sl_vert,
                                                 status);
    return cudaGetLastError();
}

cudaError_t launch_boot_batch_join(const int *half_len, const int *sl_seed, int nsl, int *out_len,
                                   int *out_seed, cudaStream_t st) {
    const int grid = std::max(1, std::min((nsl + 255) / 256, 4096));
    boot_batch_join_kernel<<<grid, 256, 0, st>>>(half_len, sl_seed, nsl, out_len, out_seed);
    return cudaGetLastError();
}

cudaError_t launch_gather_halves(const float *pool, const long long *half_off, const int *half_len,
                                 const long long *pt_off, int nsl, float *out, int grid, cudaStream_t st) {
    gather_halves_kernel<<<grid, 256, 0, st>>>(pool, half_off, half_len, pt_off, nsl, out);
    return cudaGetLastError();
}

cudaError_t boot_batch_set_smem(const BootBatchGeom &g) {
    return cudaFuncSetAttribute(boot_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, g.smem);
}

cudaError_t launch_boot_batch(const DevParams &P, const BootBatchGeom &g, const BootBatchArgs &A,
                              const int *partner, int grid, cudaStream_t st) {
    boot_batch_kernel<<<grid, kBThreads, g.smem, st>>>(P, g, A, partner);
    return cudaGetLastError();
}

}  // namespace csl
