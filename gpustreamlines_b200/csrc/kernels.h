// Launchers of the tracking kernels (implemented in kernels.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "common.cuh"

namespace csl {

constexpr int kMaxStoredPeaksPerSeed = 32;

// floats of global scratch per resident warp: backward and forward point
// buffers plus a peak list for seeds with more peaks than pass 1 stores
__host__ __device__ inline size_t scratch_floats_per_warp(const DevParams &P) {
    return (size_t)2 * P.max_sline_len * 3 + (size_t)P.samplm_nr;
}

int smem_bytes(const DevParams &P, int warps, bool track);

// Raise (never lower) a kernel's dynamic shared-memory limit.  Several
// trackers launch the same kernel with their own sizes, and a captured graph
// holds launches of several of them, so the limit only ever grows.
template <typename K>
inline cudaError_t raise_smem_limit(K kernel, int bytes) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, reinterpret_cast<const void *>(kernel));
    if (e != cudaSuccess) return e;
    if (fa.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
    return cudaFuncSetAttribute(reinterpret_cast<const void *>(kernel), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                bytes);
}

cudaError_t launch_seed_peaks(const DevParams &P, const float *seeds, int n, long long rng_base,
                              const int *partner, int *npeaks, short *peaks, int max_store,
                              int grid, int block, cudaStream_t st);
cudaError_t track_occupancy(const DevParams &P, int block, int *blocks_per_sm);
cudaError_t launch_track(const DevParams &P, const BatchArgs &B, const int *partner,
                         const int *npeaks, const short *peaks, int max_store, const int *sl_off,
                         int *out_len, int *out_seed, long long *out_src, int grid, int block,
                         cudaStream_t st);
// ---- probabilistic tracking with the bounded-envelope sampler (envelope.cu)
constexpr int kEnvClusters = 64;    // vertex clusters: two per lane
constexpr int kEnvMaxMembers = 32;  // vertices per cluster (one 32-bit cone word)
bool env_clusters(const float *verts, int V, std::vector<short> &member);
cudaError_t launch_env_tables(const DevParams &P, const short *member, uint32_t *cmax, uint32_t *cone,
                              int nsm, cudaStream_t st);
cudaError_t track_occupancy_env(const DevParams &P, int block, int *blocks_per_sm);
cudaError_t launch_track_env(const DevParams &P, const BatchArgs &B, const int *partner, const int *npeaks,
                             const short *peaks, int max_store, const int *sl_off, int *out_len, int *out_seed,
                             long long *out_src, int grid, int block, cudaStream_t st);
cudaError_t launch_env_step(const DevParams &P, const float *pts, const int *dir_vtx, const int *dir_neg,
                            const unsigned long long *subseq, int n, int *out_vtx, int *out_neg,
                            cudaStream_t st);
cudaError_t launch_get_direction(const DevParams &P, const int *partner, const float *pts,
                                 const float *dirs, const unsigned long long *subseq,
                                 const unsigned long long *offs, int n, float *frames,
                                 float *out_dirs, int *out_ok, int *out_draws, cudaStream_t st);
cudaError_t launch_gather(const float *pool, const long long *src, const int *len,
                          const long long *pt_off, int nsl, float *out, int grid, cudaStream_t st);
cudaError_t launch_cone_mask(const DevParams &P, uint32_t *mask, uint32_t *mask_t, cudaStream_t st);
cudaError_t launch_device_cos(float a, float b, float *out, cudaStream_t st);
cudaError_t launch_philox_stream(unsigned long long seed, unsigned long long subseq,
                                 unsigned long long offset, long long n, unsigned *out,
                                 cudaStream_t st);
// ---- batched bootstrap fit on the tensor cores (boot_batch.cu)
constexpr int kMaxDegree = 8;  // neighbour-table width of the batched peak search

struct BootBatchGeom {
    int hr, nb0;        // non-b0 / b0 volumes
    int HP, N1;         // hr padded to 32; rows of [R ; H] = 2 HP
    int C, N2;          // SH coefficients, padded to 16
    int V, nchunk1, nchunk3, vstride;
    int TP;             // DWI volumes per voxel in the reordered copy (padded to 4)
    int b1_chunk, b2_bytes, b3_chunk;  // bytes of one packed operand chunk (hi + lo)
    int r0, r1, r2, smem;              // shared-memory regions and total
    int nbr_shorts;                    // V * kMaxDegree, padded to 16 bytes
    int verts_floats;                  // 3 V sphere-vertex coordinates in shared memory, padded to 4
};

struct BootBatchArgs {
    const unsigned char *B1g;  // [HP/32][2][2HP x 32] packed [R ; H]
    const unsigned char *B2g;  // [2][N2 x HP] packed delta_q
    const unsigned char *B3g;  // [nchunk3][2][256 x N2] packed sampling matrix
    const int *volidx;         // [T] volume indices: the hr non-b0 volumes, then the b0s
    const short *nbr;          // [V][kMaxDegree] sphere neighbours, padded with the vertex itself
    const float *dwi;          // [X,Y,Z,TP] DWI with the T axis in volidx order
    const float *seeds;
    const int *sl_seed;        // streamline -> seed (batch-local)
    const short *sl_vert;      // streamline -> initial vertex
    int nsl;                   // streamlines (graph-captured batches: the slot capacity)
    const int *nsl_dev;        // NULL, or the streamline count in device memory (clamped to nsl)
    long long rng_base;
    int *hq;                   // atomic queue of streamline halves
    float *odf;                // [grid * 128][vstride] ODF rows
    float *pts;                // [grid * 128][max_sline_len * 3] points of the running halves
    unsigned long long *pool_count;
    float *pool;
    unsigned long long pool_cap;
    // probe mode (nprobe > 0): work items are points, not streamline halves;
    // each gets one fit with the given resample indices and its ODF row is
    // written to probe_odf[item * probe_stride]; no tracking
    int nprobe;
    const float *probe_pts;    // [nprobe,3]
    const int *probe_idx;      // [nprobe][hr] bootstrap source index of each non-b0 volume
    float *probe_odf;          // [nprobe][probe_stride]
    int probe_stride;
    int *half_len;             // [2 nsl] points per half (seed included)
    long long *half_off;       // [2 nsl] pool offset of each half (-1 when the pool overflowed)
    int *status;
    // near-tie re-evaluation (refit != 0): a row whose peak decisions lie within
    // refit_tol x (row maximum) of flipping is fitted again in float64 and searched
    // again before the closest peak is chosen
    int refit;
    float refit_tol;
    uint32_t *rng_save;                 // [grid * 128 * 4][5]: Philox counter and index at each attempt's draws
    const float *refit_tab;             // transposed fit matrices, refit_tab_layout
    int *refit_idx;                     // [grid * 16 warps][kRefitIdx] resample indices of a re-fit
    unsigned long long *refit_count;    // [2]: rows searched, rows fitted again
    // probe mode with directions: the chosen step of each probe item
    const float *probe_dirs;            // [nprobe, 3] incoming directions (NULL: ODF rows only)
    float *probe_step;                  // [nprobe, 4]: direction, found + 2 * (row fitted again)
};
constexpr int kRefitIdx = 160;          // ints of re-fit scratch per warp (hr <= 160)

// tables of the near-tie re-fit (float32 entries, exact in double; offsets in
// floats): rh = (R[j][i], H[j][i]) pairs at [i][j], dq / db = Delta_q /
// Delta_b transposed [hr][64], smp = the sampling matrix transposed [C][vp],
// vp = V rounded up to 32; zero past C and V
constexpr int kRefitCP = 64;
struct RefitTab {
    size_t rh, dq, db, smp, total;
    int vp;
};
__host__ __device__ inline RefitTab refit_tab_layout(int hr, int C, int V) {
    RefitTab L;
    L.vp = (V + 31) / 32 * 32;
    L.rh = 0;
    L.dq = L.rh + 2 * (size_t)hr * hr;
    L.db = L.dq + (size_t)hr * kRefitCP;
    L.smp = L.db + (size_t)hr * kRefitCP;
    L.total = L.smp + (size_t)C * L.vp;
    return L;
}

BootBatchGeom boot_batch_geom(const DevParams &P, int hr, int nb0);
cudaError_t launch_boot_batch_pack(const DevParams &P, const BootBatchGeom &g, void *B1g, void *B2g,
                                   void *B3g, cudaStream_t st);
cudaError_t launch_boot_batch_dwi(const float *src, const int *volidx, long long nvox, int T, int TP,
                                  float *dst, cudaStream_t st);
// count (may be NULL): the streamline count in device memory, clamped to nsl
// (graph-captured batches); status (may be NULL): gather nothing on overflow
cudaError_t launch_boot_batch_prep(const int *npeaks, const int *sl_off, const short *peaks, int max_store,
                                   int n, int cap, int *sl_seed, short *sl_vert, int *status, cudaStream_t st);
cudaError_t launch_boot_batch_join(const int *half_len, const int *sl_seed, int nsl, const int *count,
                                   int *out_len, int *out_seed, cudaStream_t st);
cudaError_t launch_gather_halves(const float *pool, const long long *half_off, const int *half_len,
                                 const long long *pt_off, int nsl, const int *count, const int *status,
                                 float *out, int grid, cudaStream_t st);
cudaError_t boot_batch_set_smem(const BootBatchGeom &g);
cudaError_t launch_boot_odf_plain(const DevParams &P, const float *pts, const int *idx, int n, float *odf,
                                  int vstride, cudaStream_t st);
cudaError_t launch_boot_batch(const DevParams &P, const BootBatchGeom &g, const BootBatchArgs &A,
                              const int *partner, int grid, cudaStream_t st);

cudaError_t launch_compress(const float *pts, long long npts, const double *affine16, const long long *off,
                            const int *len, int nsl, int minlen, int maxlen, double tol, double maxseg, float *world,
                            unsigned char *keep, int *cnt, cudaStream_t st);
cudaError_t launch_compress_gather(const float *world, const long long *off, const int *len,
                                   const unsigned char *keep, const long long *coff, int nsl, float *out,
                                   cudaStream_t st);

// ---- device-counted compaction for graph-captured batches (multi.cu)
constexpr int kCountedScanBlocks = 1024;  // CTAs of the counted scan = length of its partial-sum buffer
cudaError_t launch_counted_scan(const int *len, const int *count, int cap, long long *bsum, long long *pt_off,
                                cudaStream_t st);
cudaError_t launch_gather_counted(const float *pool, const long long *src, const int *len, const long long *pt_off,
                                  const int *count, int cap, const int *status, long long pts_cap, float *out,
                                  int grid, cudaStream_t st);
cudaError_t launch_batch_summary(const int *count, int cap, const long long *pt_off, const int *status,
                                 const unsigned long long *pool_count, long long *out4, cudaStream_t st);

cudaError_t scan_temp_bytes(int n, size_t *bytes);
// Morton-sort the seeds (perm = position -> seed) and split the order into
// per-block ranges; with tmp == nullptr only reports the sort's temp size.
cudaError_t spatial_order(const float *seeds, int n, int nblocks, uint32_t *keys, uint32_t *keys_sorted,
                          int *vals, int *perm, int *blk_next, int *blk_end, void *tmp,
                          size_t *tmp_bytes, cudaStream_t st);
cudaError_t exclusive_scan_i32(void *tmp, size_t tmp_bytes, const int *in, int *out, int n,
                               cudaStream_t st);
cudaError_t exclusive_scan_i64(void *tmp, size_t tmp_bytes, const int *in, long long *out, int n,
                               cudaStream_t st);

}  // namespace csl
