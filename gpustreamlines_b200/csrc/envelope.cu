// Set-up and launchers of the probabilistic tracker with the bounded-envelope
// sampler (envelope.cuh): the vertex clustering, the per-voxel cluster-maxima
// table, the per-direction cone bits of each cluster, the persistent tracking
// kernel instantiated for the sampler, and a one-step test kernel.
#include <cmath>
#include <vector>

#include "envelope.cuh"
#include "kernels.h"
#include "track.cuh"

namespace csl {

// ---------------------------------------------------------------------------
// host: vertex clusters

// Spherical k-means (Lloyd) with farthest-point initial centres, deterministic.
// member[k * 32 + j] = j-th vertex of cluster k (ascending ids), -1 padded.
// Returns false when some cluster would hold more than 32 vertices.
bool env_clusters(const float *verts, int V, std::vector<short> &member) {
    const int K = kEnvClusters;
    std::vector<double> c((size_t)K * 3), acc((size_t)K * 3);
    std::vector<int> lab(V, 0);
    auto dot = [&](int v, int k) {
        return (double)verts[3 * v] * c[3 * k] + (double)verts[3 * v + 1] * c[3 * k + 1] +
               (double)verts[3 * v + 2] * c[3 * k + 2];
    };
    // farthest-point seeding from vertex 0
    std::vector<double> best(V, -2.0);
    int pick = 0;
    for (int k = 0; k < K; k++) {
        for (int a = 0; a < 3; a++) c[3 * k + a] = verts[3 * pick + a];
        int next = 0;
        double low = 2.0;
        for (int v = 0; v < V; v++) {
            const double d = dot(v, k);
            if (d > best[v]) best[v] = d;
            if (best[v] < low) {
                low = best[v];
                next = v;
            }
        }
        pick = next;
    }
    for (int it = 0; it < 50; it++) {
        bool changed = false;
        for (int v = 0; v < V; v++) {
            int arg = 0;
            double bd = -3.0;
            for (int k = 0; k < K; k++) {
                const double d = dot(v, k);
                if (d > bd) {
                    bd = d;
                    arg = k;
                }
            }
            changed |= (lab[v] != arg) || it == 0;
            lab[v] = arg;
        }
        if (!changed) break;
        std::fill(acc.begin(), acc.end(), 0.0);
        for (int v = 0; v < V; v++)
            for (int a = 0; a < 3; a++) acc[3 * lab[v] + a] += verts[3 * v + a];
        for (int k = 0; k < K; k++) {
            const double n = std::sqrt(acc[3 * k] * acc[3 * k] + acc[3 * k + 1] * acc[3 * k + 1] +
                                       acc[3 * k + 2] * acc[3 * k + 2]);
            if (n > 0)
                for (int a = 0; a < 3; a++) c[3 * k + a] = acc[3 * k + a] / n;
        }
    }
    member.assign((size_t)K * kEnvMaxMembers, (short)-1);
    std::vector<int> cnt(K, 0);
    for (int v = 0; v < V; v++) {
        const int k = lab[v];
        if (cnt[k] == kEnvMaxMembers) return false;
        member[(size_t)k * kEnvMaxMembers + cnt[k]++] = (short)v;
    }
    return true;
}

// ---------------------------------------------------------------------------
// device: tables

// bf16 bit pattern of the smallest bfloat16 >= x (x finite or +-inf)
__device__ __forceinline__ uint32_t bf16_round_up(float x) {
    uint32_t b = __float_as_uint(x);
    if (x != x) return 0x7fc0u;
    if (x > 0.0f && (b & 0xffffu)) b = (b & 0xffff0000u) + 0x10000u;  // toward +inf (may reach +inf)
    return b >> 16;                                                    // exact, or a negative truncated
}

// One warp per voxel: lane l writes the maxima of clusters 2l and 2l+1.
__global__ void env_cmax_kernel(const float *__restrict__ pmf, long long nvox, int T,
                                const short *__restrict__ member, uint32_t *__restrict__ out) {
    const int lane = threadIdx.x & 31;
    const long long wpb = blockDim.x / kWarp;
    for (long long x = blockIdx.x * wpb + threadIdx.x / kWarp; x < nvox; x += (long long)gridDim.x * wpb) {
        const float *row = pmf + x * T;
        float m[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const short *mem = member + (2 * lane + h) * kEnvMaxMembers;
            float v = 0.0f;
            bool any = false;
            for (int j = 0; j < kEnvMaxMembers; j++) {
                const int t = mem[j];
                if (t < 0) break;
                const float d = __ldg(row + t);
                v = any ? fmaxf(v, d) : d;
                any = true;
            }
            m[h] = v;
        }
        out[x * kWarp + lane] = bf16_round_up(m[0]) | (bf16_round_up(m[1]) << 16);
    }
}

// Cone bits of each cluster's members for every incoming direction row
// (sign, vertex), taken from the plain sampler's keep-bit table, so the cone is
// the reference's (generate_streamlines_cuda.cu:141-152).
__global__ void env_cone_kernel(DevParams P, const short *__restrict__ member, uint32_t *__restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long rows = 2LL * P.nvert;
    if (i >= rows * kEnvClusters) return;
    const long long row = i / kEnvClusters;
    const int k = (int)(i % kEnvClusters);
    uint32_t bits = 0u;
    for (int j = 0; j < kEnvMaxMembers; j++) {
        const int t = member[k * kEnvMaxMembers + j];
        if (t < 0) break;
        const uint32_t word = P.cone_mask[row * P.nch + (t >> 5)];
        bits |= ((word >> (t & 31)) & 1u) << j;
    }
    out[i] = bits;
}

cudaError_t launch_env_tables(const DevParams &P, const short *member, uint32_t *cmax, uint32_t *cone,
                              int nsm, cudaStream_t st) {
    const long long nvox = (long long)P.dimx * P.dimy * P.dimz;
    env_cmax_kernel<<<nsm * 8, 256, 0, st>>>(P.dataf, nvox, P.dimt, member, cmax);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const long long n = 2LL * P.nvert * kEnvClusters;
    env_cone_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(P, member, cone);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// tracking with the envelope sampler

template <typename K>
static cudaError_t set_smem_env(K kernel, int bytes) {
    return raise_smem_limit(kernel, bytes);
}

cudaError_t track_occupancy_env(const DevParams &P, int block, int *blocks_per_sm) {
    const int smem = smem_bytes(P, block / kWarp, true);
    cudaError_t e = set_smem_env(track_kernel<PROB_ENV>, smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, track_kernel<PROB_ENV>, block, smem);
}

cudaError_t launch_track_env(const DevParams &P, const BatchArgs &B, const int *partner, const int *npeaks,
                             const short *peaks, int max_store, const int *sl_off, int *out_len, int *out_seed,
                             long long *out_src, int grid, int block, cudaStream_t st) {
    const int smem = smem_bytes(P, block / kWarp, true);
    cudaError_t e = set_smem_env(track_kernel<PROB_ENV>, smem);
    if (e != cudaSuccess) return e;
    track_kernel<PROB_ENV><<<grid, block, smem, st>>>(P, B, partner, npeaks, peaks, max_store, sl_off, out_len,
                                                      out_seed, out_src);
    return cudaGetLastError();
}

// One envelope-sampler step per query (test entry point): query q at point
// pts[q], incoming direction (-1)^dir_neg[q] * vertex dir_vtx[q]; proposals
// from the envelope stream of subsequence 2^61 + subseq[q], the inverse-CDF
// fallback from lane 0's stream at (subseq[q], offset 0).  Outputs the sampled vertex (-1 when
// the getter stops) and the sign of the returned direction.
__global__ void env_step_kernel(DevParams P, const float *pts, const int *dir_vtx, const int *dir_neg,
                                const unsigned long long *subseq, int n, int *out_vtx, int *out_neg) {
    extern __shared__ float smem[];
    const int warp = threadIdx.x / kWarp, lane = threadIdx.x & 31;
    const WarpBufs W = carve(P, smem + kMaxSortLayers * kWarp, warp, true, nullptr);
    const int q = blockIdx.x * (blockDim.x / kWarp) + warp;
    if (q >= n) return;
    PhiloxShared rng;
    rng.st = W.rng;
    rng.init(P.rng_seed, subseq[q], 0);
    const int u = dir_vtx[q], sg = dir_neg[q];
    float3 d = vert3(P.verts, u);
    if (sg) d = make_float3(-d.x, -d.y, -d.z);
    const DirState dir{d, u, sg};
    const float3 pt = make_float3(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
    int vox[8];
    float w[8];
    int ok = 0;
    DirState nd{d, -1, 0};
    EnvCount cnt = {0, 0, 0, 0};
    if (trilinear_vox(P, pt, vox, w)) {
        EnvLoads L;
        env_issue(P, vox, dir, lane, L);
        EnvStream es{kEnvSubseqBase + subseq[q], 0ull};
        ok = env_sample(P, vox, w, L, dir, W.odf, rng, es, lane, &nd, cnt);
    }
    if (lane == 0) {
        out_vtx[q] = ok ? nd.vtx : -1;
        out_neg[q] = ok ? nd.neg : 0;
    }
    env_flush(P, cnt, lane);
}

cudaError_t launch_env_step(const DevParams &P, const float *pts, const int *dir_vtx, const int *dir_neg,
                            const unsigned long long *subseq, int n, int *out_vtx, int *out_neg,
                            cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int block = 128;
    const int smem = smem_bytes(P, block / kWarp, true);
    cudaError_t e = set_smem_env(env_step_kernel, smem);
    if (e != cudaSuccess) return e;
    env_step_kernel<<<(n + 3) / 4, block, smem, st>>>(P, pts, dir_vtx, dir_neg, subseq, n, out_vtx, out_neg);
    return cudaGetLastError();
}

}  // namespace csl
