// Device-side compaction for graph-captured batches (the multi-subject run).
//
// The plain batch path reads the streamline count back to the host after
// pass 1 and sizes its buffers and its scan from it.  A batch that is one
// branch of a captured CUDA graph cannot: its launch shapes are fixed when the
// graph is captured.  These kernels take the streamline count from device
// memory instead (sl_off[nseeds], written by the pass-1 scan) and clamp it to
// the capacity the buffers were sized for:
//   * counted_scan: exclusive scan of the streamline lengths over
//     [0, min(count, cap)) into pt_off, total in pt_off[n] -- three phases
//     (per-CTA sums over contiguous chunks, one-CTA scan of the sums,
//     per-CTA rescan with the chunk's offset), one pass over the lengths each;
//   * gather_counted: copies each streamline's points from the pool into the
//     compacted output, nothing when the batch overflowed its pool or slots
//     (the host then re-runs that batch on the plain path);
//   * batch_summary: count, points, status and pool use of the batch, for one
//     device-to-host copy of all subjects at the end of the graph.
#include <cub/block/block_reduce.cuh>
#include <cub/block/block_scan.cuh>

#include "kernels.h"

namespace csl {

namespace {

constexpr int kScanThreads = 256;

__device__ __forceinline__ int clamped_count(const int *count, int cap) {
    const int n = *count;
    return n < 0 ? 0 : (n > cap ? cap : n);
}

__global__ void __launch_bounds__(kScanThreads)
    counted_scan_sums(const int *__restrict__ len, const int *__restrict__ count, int cap,
                      long long *__restrict__ bsum) {
    using Reduce = cub::BlockReduce<long long, kScanThreads>;
    __shared__ typename Reduce::TempStorage tmp;
    const long long n = clamped_count(count, cap);
    const long long chunk = (n + gridDim.x - 1) / gridDim.x;
    const long long lo = (long long)blockIdx.x * chunk;
    const long long hi = lo + chunk < n ? lo + chunk : n;
    long long acc = 0;
    for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) acc += len[i];
    const long long s = Reduce(tmp).Sum(acc);
    if (threadIdx.x == 0) bsum[blockIdx.x] = s;
}

// one CTA of kCountedScanBlocks threads: exclusive scan of the per-CTA sums in
// place, total into pt_off[n]
__global__ void __launch_bounds__(kCountedScanBlocks)
    counted_scan_top(long long *__restrict__ bsum, const int *__restrict__ count, int cap,
                     long long *__restrict__ pt_off) {
    using Scan = cub::BlockScan<long long, kCountedScanBlocks>;
    __shared__ typename Scan::TempStorage tmp;
    long long v = bsum[threadIdx.x], x, total;
    Scan(tmp).ExclusiveSum(v, x, total);
    bsum[threadIdx.x] = x;
    if (threadIdx.x == 0) pt_off[clamped_count(count, cap)] = total;
}

__global__ void __launch_bounds__(kScanThreads)
    counted_scan_apply(const int *__restrict__ len, const int *__restrict__ count, int cap,
                       const long long *__restrict__ bsum, long long *__restrict__ pt_off) {
    using Scan = cub::BlockScan<long long, kScanThreads>;
    __shared__ typename Scan::TempStorage tmp;
    const long long n = clamped_count(count, cap);
    const long long chunk = (n + gridDim.x - 1) / gridDim.x;
    const long long lo = (long long)blockIdx.x * chunk;
    const long long hi = lo + chunk < n ? lo + chunk : n;
    long long run = bsum[blockIdx.x];
    for (long long base = lo; base < hi; base += blockDim.x) {
        const long long i = base + threadIdx.x;
        const long long v = i < hi ? len[i] : 0;
        long long x, tile;
        Scan(tmp).ExclusiveSum(v, x, tile);
        if (i < hi) pt_off[i] = run + x;
        run += tile;
        __syncthreads();  // TempStorage reuse
    }
}

__global__ void gather_counted_kernel(const float *__restrict__ pool, const long long *__restrict__ src,
                                      const int *__restrict__ len, const long long *__restrict__ pt_off,
                                      const int *__restrict__ count, int cap, const int *__restrict__ status,
                                      long long pts_cap, float *__restrict__ out) {
    if (*status & (ST_POOL_OVERFLOW | ST_SLOT_OVERFLOW)) return;
    const int n = clamped_count(count, cap);
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x / kWarp;
    for (int sl = blockIdx.x * wpb + threadIdx.x / kWarp; sl < n; sl += gridDim.x * wpb) {
        const long long s = src[sl];
        const int l = len[sl];
        const long long o = pt_off[sl];
        if (s < 0 || l < 0 || o < 0 || o + l > pts_cap) continue;
        const float *a = pool + 3 * s;
        float *b = out + 3 * o;
        for (int j = lane; j < 3 * l; j += kWarp) b[j] = a[j];
    }
}

__global__ void batch_summary_kernel(const int *count, int cap, const long long *pt_off, const int *status,
                                     const unsigned long long *pool_count, long long *out4) {
    out4[0] = *count;
    out4[1] = pt_off[clamped_count(count, cap)];
    out4[2] = *status;
    out4[3] = (long long)*pool_count;
}

}  // namespace

cudaError_t launch_counted_scan(const int *len, const int *count, int cap, long long *bsum, long long *pt_off,
                                cudaStream_t st) {
    counted_scan_sums<<<kCountedScanBlocks, kScanThreads, 0, st>>>(len, count, cap, bsum);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    counted_scan_top<<<1, kCountedScanBlocks, 0, st>>>(bsum, count, cap, pt_off);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    counted_scan_apply<<<kCountedScanBlocks, kScanThreads, 0, st>>>(len, count, cap, bsum, pt_off);
    return cudaGetLastError();
}

cudaError_t launch_gather_counted(const float *pool, const long long *src, const int *len, const long long *pt_off,
                                  const int *count, int cap, const int *status, long long pts_cap, float *out,
                                  int grid, cudaStream_t st) {
    gather_counted_kernel<<<grid, 256, 0, st>>>(pool, src, len, pt_off, count, cap, status, pts_cap, out);
    return cudaGetLastError();
}

cudaError_t launch_batch_summary(const int *count, int cap, const long long *pt_off, const int *status,
                                 const unsigned long long *pool_count, long long *out4, cudaStream_t st) {
    batch_summary_kernel<<<1, 1, 0, st>>>(count, cap, pt_off, status, pool_count, out4);
    return cudaGetLastError();
}

}  // namespace csl
