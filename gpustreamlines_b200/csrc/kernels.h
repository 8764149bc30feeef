// Launchers of the tracking kernels (implemented in kernels.cu).
#pragma once
#include <cstddef>
#include <cstdint>
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

cudaError_t launch_seed_peaks(const DevParams &P, const float *seeds, int n, long long rng_base,
                              const int *partner, int *npeaks, short *peaks, int max_store,
                              int grid, int block, cudaStream_t st);
cudaError_t track_occupancy(const DevParams &P, int block, int *blocks_per_sm);
cudaError_t launch_track(const DevParams &P, const BatchArgs &B, const int *partner,
                         const int *npeaks, const short *peaks, int max_store, const int *sl_off,
                         int *out_len, int *out_seed, long long *out_src, int grid, int block,
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
