// Device-side building blocks shared by the three direction getters.
//
// Numerics follow the reference kernels operation by operation (same
// summation order, same float/double promotions, same comparison
// directions), so that the integer outputs (peak counts, offsets, vertex
// choices) come out identical on the same inputs.  Each helper cites the
// reference routine it restates.  Work is warp-cooperative: one warp owns
// one seed, lane `l` owns elements l, l+32, l+64, ... of every length-T
// vector, the same lane-to-element map the reference uses.
#pragma once
#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

#include "philox.cuh"

namespace csl {

constexpr unsigned FULL = 0xffffffffu;
constexpr int kWarp = 32;
constexpr int kMaxSortLayers = 15;

enum TissueClass { OUTSIDEIMAGE = 0, INVALIDPOINT = 1, TRACKPOINT = 2, ENDPOINT = 3 };
enum Model { OPDT = 0, CSA = 1, PROB = 2, PTT = 3 };

// Everything a kernel needs, passed by value as a kernel parameter (one
// library instance serves trackers with different shapes at the same time).
struct DevParams {
    int model;
    int dimx, dimy, dimz, dimt;
    int nvert, nedges, samplm_nr;
    int sphere_symm;
    int max_sline_len;
    int nch;            // ceil(samplm_nr / 32) for PROB, 1 otherwise
    int vec4;           // PROB: samplm_nr % 4 == 0 (16-byte aligned voxel rows)
    int step_frac;
    double step_size, max_angle, tc_threshold, relative_peak_thresh;
    double min_separation_angle, pmf_threshold;
    unsigned long long rng_seed;
    float cos_max_angle;    // cos(MAX_ANGLE) as the reference evaluates it
    float cos_min_sep;      // cos(MIN_SEPARATION_ANGLE)
    const float *__restrict__ dataf;     // [X,Y,Z,T]
    const float *__restrict__ verts;     // [V,3]
    const int2 *__restrict__ edges;      // [E]
    cudaTextureObject_t stop_tex;        // stop map, border -1, linear filter
    const uint32_t *__restrict__ cone_mask;    // PROB: [2][V][nch] keep bits
    const uint32_t *__restrict__ cone_mask_t;  // PROB: [2][V][32] the same bits, per lane
    // PROB with the bounded-envelope sampler (env != 0; envelope.cuh)
    int env;
    const uint32_t *__restrict__ env_cmax;    // [X*Y*Z][32]: cluster maxima rounded up to bf16, 2 per word
    const uint32_t *__restrict__ env_cone;    // [2][V][64]: cone bits of each cluster's members
    const short *__restrict__ env_member;     // [64][32]: vertex ids of each cluster (-1 padded)
    unsigned long long *env_stats;            // [4] counters: steps, proposals, exact resolutions, fallbacks
    // bootstrap
    float min_signal;
    int delta_nr, hr_side;
    const float *__restrict__ H;
    const float *__restrict__ R;
    const float *__restrict__ delta_b;
    const float *__restrict__ delta_q;
    const float *__restrict__ sampling;
    const int *__restrict__ b0s_mask;
    // PTT
    cudaTextureObject_t odf_tex;         // tiled ODF texture, linear filter
    cudaTextureObject_t lut_tex;         // nearest-vertex LUT, point filter, normalised
    int log2_x, log2_y, width_mask, height_mask;
    float probe_step_size, probe_quality;
    double max_curvature;  // MAX_CURVATURE is a double literal in the reference
};

// Per-batch work arrays (device pointers).
struct BatchArgs {
    const float *__restrict__ seeds;    // [n,3]
    int nseeds;
    long long rng_index_base;
    int *queue;                         // atomic seed counter (input order)
    const int *__restrict__ perm;       // spatial order: position -> seed (or nullptr)
    int *blk_next;                      // per-block next position in `perm`
    const int *__restrict__ blk_end;    // per-block end position
    unsigned long long *pool_count;     // atomic, in points
    float *pool;                        // [pool_cap,3]
    unsigned long long pool_cap;
    float *scratch;                     // per-warp point buffers + peak list
    int *status;                        // error/overflow flags
    int sl_cap;                         // streamline slots in out_len / out_seed / out_src: a seed
                                        // whose slots would pass it is skipped and flagged
};

enum StatusBits {
    ST_POOL_OVERFLOW = 1,   // point pool too small: the batch is re-run with an exact size
    ST_PEAKS_OVERFLOW = 2,  // a seed has more initial directions than pass 1 stores
    ST_WAIT_TIMEOUT = 4,    // a bounded wait on an mbarrier gave up (never expected)
    ST_SLOT_OVERFLOW = 8,   // more streamlines than the fixed slot capacity of a graph-captured batch
};

// ---------------------------------------------------------------------------
// warp reductions (utils.cu:1-80): lane-strided partial, then xor butterfly

__device__ __forceinline__ float fmax_ref(float a, float b) { return (a > b) ? a : b; }
__device__ __forceinline__ float fmin_ref(float a, float b) { return (a < b) ? a : b; }

__device__ __forceinline__ float warp_max_ref(float m) {
#pragma unroll
    for (int i = 16; i; i >>= 1) m = fmax_ref(m, __shfl_xor_sync(FULL, m, i));
    return m;
}
__device__ __forceinline__ float warp_min_ref(float m) {
#pragma unroll
    for (int i = 16; i; i >>= 1) m = fmin_ref(m, __shfl_xor_sync(FULL, m, i));
    return m;
}

// ---------------------------------------------------------------------------
// trilinear interpolation (tracking_helpers.cu:4-61)

struct Corners {
    long long base[8];  // element offsets of the 8 corner rows
    float w[8];         // ((wx*wy)*wz) in (i,j,k) lexicographic order
};

// Corner voxels (flat index (x*Y + y)*Z + z) and weights of the trilinear
// interpolation at p; false outside the volume.
__device__ __forceinline__ bool trilinear_vox(const DevParams &P, float3 p, int (&vox)[8], float (&w)[8]) {
    const float HALF = 0.5f;
    if (!(p.x == p.x) || !(p.y == p.y) || !(p.z == p.z)) return false;
    if (p.x < -HALF || p.x + HALF >= (float)P.dimx || p.y < -HALF || p.y + HALF >= (float)P.dimy ||
        p.z < -HALF || p.z + HALF >= (float)P.dimz)
        return false;
    const float flx = floorf(p.x), fly = floorf(p.y), flz = floorf(p.z);
    float wgh[3][2];
    int coo[3][2];
    wgh[0][1] = p.x - flx;
    wgh[0][0] = 1.0f - wgh[0][1];
    coo[0][0] = (int)((0 > flx) ? 0 : flx);
    coo[0][1] = ((P.dimx - 1) < coo[0][0] + 1) ? (P.dimx - 1) : coo[0][0] + 1;
    wgh[1][1] = p.y - fly;
    wgh[1][0] = 1.0f - wgh[1][1];
    coo[1][0] = (int)((0 > fly) ? 0 : fly);
    coo[1][1] = ((P.dimy - 1) < coo[1][0] + 1) ? (P.dimy - 1) : coo[1][0] + 1;
    wgh[2][1] = p.z - flz;
    wgh[2][0] = 1.0f - wgh[2][1];
    coo[2][0] = (int)((0 > flz) ? 0 : flz);
    coo[2][1] = ((P.dimz - 1) < coo[2][0] + 1) ? (P.dimz - 1) : coo[2][0] + 1;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 2; j++)
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const int q = (i << 2) | (j << 1) | k;
                vox[q] = (coo[0][i] * P.dimy + coo[1][j]) * P.dimz + coo[2][k];
                w[q] = wgh[0][i] * wgh[1][j] * wgh[2][k];
            }
    return true;
}

__device__ __forceinline__ bool trilinear_setup(const DevParams &P, float3 p, Corners &c) {
    int vox[8];
    if (!trilinear_vox(P, p, vox, c.w)) return false;
#pragma unroll
    for (int q = 0; q < 8; q++) c.base[q] = (long long)vox[q] * P.dimt;
    return true;
}

// value of element t: sum over corners in reference order, fused multiply-adds
__device__ __forceinline__ float trilinear_elem(const float *__restrict__ data, const Corners &c,
                                                long long t) {
    float acc = 0.0f;
#pragma unroll
    for (int q = 0; q < 8; q++) acc += c.w[q] * __ldg(data + c.base[q] + t);
    return acc;
}

// ---------------------------------------------------------------------------
// stop check (tracking_helpers.cu:63-73): hardware filtered fetch of the stop
// map (border colour -1, unnormalised coordinates, texel centres at +0.5)

__device__ __forceinline__ int check_point(const DevParams &P, float3 p) {
    const float val = tex3D<float>(P.stop_tex, p.z, p.y, p.x);
    if (val == -1.0f) return OUTSIDEIMAGE;
    return ((double)val > P.tc_threshold) ? TRACKPOINT : ENDPOINT;
}

// ---------------------------------------------------------------------------
// inclusive scan in reference order (utils.cu:82-120): 32-element chunks,
// lane 0 adds the previous chunk's last value, then a Hillis-Steele scan.

// Same scan over a shared-memory array (used by the smaller PTT face CDF).
__device__ __forceinline__ void scan_smem_ref(float *num, int len, int lane) {
    for (int j = 0; j < len; j += kWarp) {
        if (lane == 0 && j != 0) num[j] += num[j - 1];
        __syncwarp();
        float x = 0.0f;
        if (j + lane < len) x = num[j + lane];
        for (int i = 1; i < kWarp; i <<= 1) {
            const float y = __shfl_up_sync(FULL, x, i);
            if (lane >= i && j + lane < len) x += y;
        }
        if (j + lane < len) num[j + lane] = x;
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// key/value sort of <= 32 entries, descending (cuwsort.cuh:133-168).  The
// comparator network is Batcher's merge exchange (Knuth, TAOCP 3, 5.2.2 M)
// with ASAP layering; the host builds the partner table.  Ties never swap, so
// the order of equal keys follows the network, as in the reference.

__device__ __forceinline__ void warp_sort_desc(const int *__restrict__ partner_sh, int lane,
                                               float &k, int &v) {
#pragma unroll
    for (int l = 0; l < kMaxSortLayers; l++) {
        const int src = partner_sh[l * kWarp + lane];
        const float a = __shfl_sync(FULL, k, src);
        const int b = __shfl_sync(FULL, v, src);
        if (lane >= src) {  // (lane < src) == DEC(0): keep the smaller key
            if (a < k) { k = a; v = b; }
        } else {
            if (a > k) { k = a; v = b; }
        }
    }
}

__device__ __forceinline__ float3 vert3(const float *__restrict__ verts, int i) {
    return make_float3(__ldg(verts + 3 * i), __ldg(verts + 3 * i + 1), __ldg(verts + 3 * i + 2));
}
// the same from global or shared memory (generic loads; __ldg is global-only)
__device__ __forceinline__ float3 vert3_any(const float *verts, int i) {
    return make_float3(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]);
}

// ---------------------------------------------------------------------------
// peak extraction (tracking_helpers.cu:75-245): local maxima over sphere
// edges, relative threshold, sort, min-separation de-duplication.
// `odf` and `ind` are per-warp shared arrays of length >= nr.  On return
// ind[0..n) hold the kept peak vertex indices in reference order.

__device__ __forceinline__ int peak_select(const DevParams &P, const float *odf, int *ind, int nr,
                                           float odf_min, const int *__restrict__ partner_sh, int lane);

__device__ __forceinline__ int peak_directions(const DevParams &P, const float *odf, int *ind, int nr,
                               const int *__restrict__ partner_sh, int lane) {
    for (int j = lane; j < nr; j += kWarp) ind[j] = 0;

    float mn = FLT_MAX;
    for (int i = lane; i < nr; i += kWarp) mn = fmin_ref(mn, odf[i]);
    float odf_min = warp_min_ref(mn);
    odf_min = (0 > odf_min) ? 0 : odf_min;
    __syncwarp();

    for (int j = 0; j < P.nedges; j += kWarp) {
        if (j + lane < P.nedges) {
            const int2 e = __ldg(P.edges + j + lane);
            const float uv = odf[e.x], vv = odf[e.y];
            if (uv < vv) {
                atomicExch(ind + e.x, -1);
                atomicOr(ind + e.y, 1);
            } else if (vv < uv) {
                atomicExch(ind + e.y, -1);
                atomicOr(ind + e.x, 1);
            }
        }
    }
    __syncwarp();

    return peak_select(P, odf, ind, nr, odf_min, partner_sh, lane);
}

// The part of peak_directions_d after the local-maximum flags are in ind[]
// (1 = local maximum, tracking_helpers.cu:163-244): relative threshold over the
// maxima, compaction, descending sort, minimum-separation filter.
__device__ __forceinline__ int peak_select(const DevParams &P, const float *odf, int *ind, int nr,
                                           float odf_min, const int *__restrict__ partner_sh, int lane) {
    const unsigned lmask = (1u << lane) - 1u;
    // RELATIVE_PEAK_THRESH * max over maxima of (odf + (-odf_min))
    float mm = -FLT_MAX;
    const float neg_min = -odf_min;
    for (int i = lane; i < nr; i += kWarp)
        if (ind[i] > 0) mm = fmax_ref(mm, odf[i] + neg_min);
    mm = warp_max_ref(mm);
    const float comp_thres = (float)(P.relative_peak_thresh * (double)mm);

    int n = 0;
    for (int j = 0; j < nr; j += kWarp) {
        const int vflag = (j + lane < nr) ? ind[j + lane] : -1;
        const int keep = (vflag > 0) && ((odf[j + lane] - odf_min) >= comp_thres);
        const unsigned msk = __ballot_sync(FULL, keep);
        if (keep) ind[n + __popc(msk & lmask)] = j + lane;
        n += __popc(msk);
    }
    __syncwarp();

    if (n < kWarp) {
        float k = -FLT_MAX;
        int v = 0;
        if (lane < n) {
            v = ind[lane];
            k = odf[v];
        }
        warp_sort_desc(partner_sh, lane, k, v);
        __syncwarp();
        if (lane < n) ind[lane] = v;
    }
    __syncwarp();

    if (n != 0) {
        if (lane == 0) {
            const float cos_similarity = P.cos_min_sep;
            int k = 1;
            for (int i = 1; i < n; i++) {
                const int vi = ind[i];
                const float3 abc = vert3(P.verts, vi);
                int j = 0;
                for (; j < k; j++) {
                    const float3 d = vert3(P.verts, ind[j]);
                    float cs = abc.x * d.x + abc.y * d.y + abc.z * d.z;
                    if (P.sphere_symm) cs = fabsf(cs);
                    if (cs > cos_similarity) break;
                }
                if (j == k) ind[k++] = vi;
            }
            n = k;
        }
        n = __shfl_sync(FULL, n, 0);
        __syncwarp();
    }
    return n;
}

}  // namespace csl
