// ODF / PMF volume from spherical-harmonic coefficients on the tensor cores:
//     out[x, v] = max(0, sum_c coef[x, c] * basis[v, c])     (clip optional)
// the step before tracking that the reference runs on the host
// (run_gpu_streamlines.py:357-380: fit.odf(sphere), clipped to >= 0 for the
// probabilistic getter).  M = voxels in tiles of 128 (TMEM lanes), N = sphere
// vertices in chunks of 256 (TMEM columns, double-buffered), K = coefficients
// padded to 16.  Products in BF16x3 (x = xh + xl, three BF16 MMAs, FP32
// accumulation), so the result carries ~1e-5 relative error of the row scale.
// The kernel is bound by the HBM write of the output (4 B per voxel-vertex).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "kernels.h"
#include "tc.cuh"

namespace csl {

constexpr int kOgRows = 128;       // voxels per tile (MMA M)
constexpr int kOgChunk = 256;      // vertices per MMA (TMEM columns)
constexpr int kOgThreads = 256;    // 8 warps: two per TMEM lane quadrant
constexpr int kOgMaxK = 64;

struct OdfGemmGeom {
    int C, KP;          // coefficients, padded to 16
    int V, nchunk;      // vertices, 256-vertex chunks
    int b_chunk;        // bytes of one packed basis chunk (hi + lo)
    int a_bytes;        // bytes of the packed A tile (hi + lo)
    int smem;
};

OdfGemmGeom odf_gemm_geom(int C, int V) {
    OdfGemmGeom g{};
    g.C = C;
    g.KP = (C + 15) / 16 * 16;
    g.V = V;
    g.nchunk = (V + kOgChunk - 1) / kOgChunk;
    g.b_chunk = 2 * kOgChunk * g.KP * 2;
    g.a_bytes = 2 * kOgRows * g.KP * 2;
    g.smem = 1024 + g.nchunk * g.b_chunk + g.a_bytes + kOgRows * 256 + 64;
    return g;
}

__global__ void odf_basis_pack_kernel(const float *__restrict__ basis, OdfGemmGeom g, __nv_bfloat16 *out) {
    const int n = g.nchunk * kOgChunk * g.KP;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int ch = e / (kOgChunk * g.KP), r = (e / g.KP) % kOgChunk, k = e % g.KP;
        const int v = ch * kOgChunk + r;
        const float x = (v < g.V && k < g.C) ? basis[(size_t)v * g.C + k] : 0.0f;
        char *hi = reinterpret_cast<char *>(out) + (size_t)ch * g.b_chunk;
        const uint32_t off = kmajor_off(r, k, kOgChunk);
        const __nv_bfloat16 h = __float2bfloat16_rn(x);
        *reinterpret_cast<__nv_bfloat16 *>(hi + off) = h;
        *reinterpret_cast<__nv_bfloat16 *>(hi + g.b_chunk / 2 + off) = __float2bfloat16_rn(x - __bfloat162float(h));
    }
}

__global__ void __launch_bounds__(kOgThreads, 1)
    odf_gemm_kernel(const float *__restrict__ coef, long long nvox, OdfGemmGeom g,
                    const unsigned char *__restrict__ Bpk, int clip, float *__restrict__ out, int *status) {
    extern __shared__ unsigned char smraw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smraw) + 1023) & ~(uintptr_t)1023);
    unsigned char *Bs = sm;                                   // all basis chunks, resident
    unsigned char *As = Bs + (size_t)g.nchunk * g.b_chunk;    // A tile hi | lo
    unsigned char *Ss = As + g.a_bytes;                       // output staging, 128 rows x 256 B
    uint64_t *bars = reinterpret_cast<uint64_t *>(Ss + kOgRows * 256);  // 0: basis loaded, 1: MMA done
    uint32_t *tmem_sh = reinterpret_cast<uint32_t *>(bars + 2);

    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    const int qd = w & 3, half = w >> 2;
    const int row = qd * 32 + lane;  // TMEM lane = voxel row of the tile
    if (t == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_fence_init();
    }
    if (w == 0) tmem_alloc(tmem_sh, 512);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *tmem_sh;
    const uint32_t trow = tbase + ((uint32_t)(qd * 32) << 16);
    bool ok = true;
    uint32_t ph_mma = 0;
    if (t == 0) {
        const uint32_t bytes = (uint32_t)(g.nchunk * g.b_chunk);
        mbar_arrive_expect_tx(&bars[0], bytes);
        // the packed basis is contiguous: copy it in pieces of <= 64 KB
        for (uint32_t o = 0; o < bytes; o += 65536u)
            bulk_g2s(Bs + o, Bpk + o, bytes - o < 65536u ? bytes - o : 65536u, &bars[0]);
        ok = mbar_wait(&bars[0], 0);
    }
    const uint32_t a_term = (uint32_t)(g.a_bytes / 2), b_term = (uint32_t)(g.b_chunk / 2);
    const long long ntile = (nvox + kOgRows - 1) / kOgRows;
    const bool vec4 = (g.V % 4) == 0;  // 16-byte aligned output rows

    for (long long tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
        if (__syncthreads_or(!ok)) break;
        // A tile: row r = voxel tile*128 + r, k groups of 8, split hi / lo
        const long long v0 = tile * kOgRows;
        for (int e = t; e < kOgRows * (g.KP / 8); e += kOgThreads) {
            const int r = e / (g.KP / 8), gq = e % (g.KP / 8);
            const long long vox = v0 + r;
            float x[8];
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const int k = gq * 8 + q;
                x[q] = (vox < nvox && k < g.C) ? __ldg(coef + vox * g.C + k) : 0.0f;
            }
            uint32_t hw[4], lw[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const __nv_bfloat162 hv = __floats2bfloat162_rn(x[2 * q], x[2 * q + 1]);
                const float2 hf = __bfloat1622float2(hv);
                const __nv_bfloat162 lv = __floats2bfloat162_rn(x[2 * q] - hf.x, x[2 * q + 1] - hf.y);
                hw[q] = *reinterpret_cast<const uint32_t *>(&hv);
                lw[q] = *reinterpret_cast<const uint32_t *>(&lv);
            }
            const uint32_t off = kmajor_off(r, gq * 8, kOgRows);
            *reinterpret_cast<uint4 *>(As + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
            *reinterpret_cast<uint4 *>(As + a_term + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        // chunks in pairs: columns [0,256) and [256,512) of TMEM
        for (int c0 = 0; c0 < g.nchunk; c0 += 2) {
            if (t == 0 && ok) {
                tc_fence_after();
                for (int cc = 0; cc < 2 && c0 + cc < g.nchunk; cc++) {
                    const uint32_t bbase = smem_u32(Bs + (size_t)(c0 + cc) * g.b_chunk);
                    for (int k16 = 0; k16 < g.KP / 16; k16++) {
#pragma unroll
                        for (int term = 0; term < 3; term++) {
                            const uint32_t aoff = (term == 2 ? a_term : 0) + (uint32_t)(k16 * 2) * (kOgRows * 16);
                            const uint32_t boff = (term == 1 ? b_term : 0) + (uint32_t)(k16 * 2) * (kOgChunk * 16);
                            umma_bf16(tbase + cc * kOgChunk, umma_sdesc(smem_u32(As) + aoff, kOgRows * 16, 128),
                                      umma_sdesc(bbase + boff, kOgChunk * 16, 128),
                                      umma_idesc_bf16(kOgRows, kOgChunk), (k16 > 0 || term > 0) ? 1u : 0u);
                        }
                    }
                }
                umma_commit(&bars[1]);
            }
            if (!mbar_wait(&bars[1], ph_mma)) ok = false;
            ph_mma ^= 1;
            tc_fence_after();
            // epilogue, 64 columns at a time: TMEM rows -> swizzled shared staging
            // (16-byte chunk c of row r at slot c ^ (r & 7): conflict-free both
            // ways) -> coalesced stores, two 256-byte row segments per warp store
            for (int cc = 0; cc < 2 && c0 + cc < g.nchunk; cc++) {
                for (int grp = 0; grp < kOgChunk / 64; grp++) {
                    const int cbase = (c0 + cc) * kOgChunk + grp * 64;
                    if (cbase >= g.V) break;  // uniform over the CTA
#pragma unroll
                    for (int bb = 0; bb < 2; bb++) {
                        const int b = half * 2 + bb;  // 16-column block within the group
                        float v[16];
                        tmem_ld16(trow + cc * kOgChunk + grp * 64 + 16 * b, v);
                        if (clip) {
#pragma unroll
                            for (int q = 0; q < 16; q++) v[q] = v[q] > 0.0f ? v[q] : 0.0f;
                        }
#pragma unroll
                        for (int q = 0; q < 4; q++) {
                            const int c = 4 * b + q;
                            *reinterpret_cast<float4 *>(Ss + row * 256 + ((c ^ (row & 7)) << 4)) =
                                make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                        }
                    }
                    __syncthreads();
#pragma unroll
                    for (int k = 0; k < (kOgRows * 16) / kOgThreads; k++) {
                        const int idx = t + k * kOgThreads;
                        const int r = idx >> 4, c = idx & 15;
                        const long long vox = v0 + r;
                        const int col = cbase + 4 * c;
                        if (vox < nvox && col < g.V) {
                            const float4 x = *reinterpret_cast<const float4 *>(Ss + r * 256 + ((c ^ (r & 7)) << 4));
                            float *dst = out + vox * g.V + col;
                            if (vec4 && col + 4 <= g.V) {
                                __stcs(reinterpret_cast<float4 *>(dst), x);
                            } else {
                                const float xs[4] = {x.x, x.y, x.z, x.w};
                                for (int q = 0; q < 4 && col + q < g.V; q++) dst[q] = xs[q];
                            }
                        }
                    }
                    __syncthreads();
                }
            }
            tc_fence_before();
            __syncthreads();
        }
    }
    if (!ok && t == 0) atomicOr(status, ST_WAIT_TIMEOUT);
    tc_fence_before();
    __syncthreads();
    if (w == 0) {
        tc_fence_after();
        tmem_dealloc(tbase, 512);
    }
}

}  // namespace csl

using namespace csl;

// C ABI (declared in include/gpustreamlines_b200.h)
extern "C" int csl_odf_volume(const float *coef_dev, long long nvox, int ncoef, const float *basis_dev, int nvert,
                              int clip, float *out_dev, void *workspace_dev, long long workspace_bytes,
                              float *ms_out, void *stream) {
    if (!coef_dev || !basis_dev || !out_dev || nvox < 0 || ncoef <= 0 || ncoef > kOgMaxK || nvert <= 0 ||
        nvert > 1024)
        return -1;  // CSL_E_INVALID
    const OdfGemmGeom g = odf_gemm_geom(ncoef, nvert);
    if (!workspace_dev || workspace_bytes < (long long)g.nchunk * g.b_chunk + 16) return -1;
    if (g.smem > 227 * 1024) return -1;
    if (nvox == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0, nsm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    unsigned char *Bpk = reinterpret_cast<unsigned char *>(workspace_dev);
    int *status = reinterpret_cast<int *>(Bpk + (size_t)g.nchunk * g.b_chunk);
    if (e == cudaSuccess) e = cudaMemsetAsync(status, 0, sizeof(int), st);
    if (e == cudaSuccess) {
        odf_basis_pack_kernel<<<64, 256, 0, st>>>(basis_dev, g, reinterpret_cast<__nv_bfloat16 *>(Bpk));
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaFuncSetAttribute(odf_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, g.smem);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ms_out && e == cudaSuccess) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, st);
    }
    if (e == cudaSuccess) {
        const long long ntile = (nvox + kOgRows - 1) / kOgRows;
        const int grid = (int)std::min<long long>(ntile, nsm);
        odf_gemm_kernel<<<grid, kOgThreads, g.smem, st>>>(coef_dev, nvox, g, Bpk, clip, out_dev, status);
        e = cudaGetLastError();
    }
    int hstatus = 0;
    if (e == cudaSuccess && ms_out) {
        cudaEventRecord(e1, st);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hstatus, status, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess && ms_out) cudaEventElapsedTime(ms_out, e0, e1);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (e != cudaSuccess) return -2;  // CSL_E_CUDA
    if (hstatus & ST_WAIT_TIMEOUT) return -5;  // CSL_E_KERNEL
    return 0;
}
