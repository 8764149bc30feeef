// PTT data preparation on the device: the host step of the reference's
// PttDirectionGetter.prepare_data (cuslines/cuda_python/cu_direction_getters.py:531-625)
// -- clip the ODF at 0, zero it where the stop map is below the threshold,
// normalise each voxel to a maximum of 1, lay the vertex axis out over
// power-of-two (tx, ty, tz) tiles of the texture, and map a res^3 grid on
// [-1, 1]^3 to the nearest sphere vertex (the reference builds a KD-tree on the
// host and queries ~2 M points).
//
// Both outputs equal the host restatement (direction_getters.py,
// prepare_data_host) bit for bit: the division is the correctly rounded one,
// the grid coordinates are numpy.linspace's (i * step + start, endpoint exact),
// and the nearest vertex minimises the float64 squared distance (first index
// on exact ties; a KD-tree may break those differently).
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/gpustreamlines_b200.h"
#include "common.cuh"

struct csl_tracker;

namespace csl {

int tracker_fail(csl_tracker *t, int code, const char *msg);  // capi.cu: sets the library's last error

struct PttTiles {
    int nx, ny, nz, log2x, log2y;
};

static PttTiles ptt_tiles(int T) {
    PttTiles t{1, 1, 1, 0, 0};
    while (t.nx * t.ny * t.nz < T) {
        if (t.nx <= t.ny && t.nx <= t.nz)
            t.nx *= 2;
        else if (t.ny <= t.nx && t.ny <= t.nz)
            t.ny *= 2;
        else
            t.nz *= 2;
    }
    while ((1 << t.log2x) < t.nx) t.log2x++;
    while ((1 << t.log2y) < t.ny) t.log2y++;
    return t;
}

// One warp per voxel: lane-strided over the vertex slots of the tiled layout.
__global__ void ptt_tile_kernel(const float *__restrict__ odf, const float *__restrict__ stop, int X, int Y, int Z,
                                int T, double thr, PttTiles tl, float *__restrict__ tiled) {
    const int lane = threadIdx.x & 31;
    const long long nvox = (long long)X * Y * Z;
    const long long wpb = blockDim.x / kWarp;
    const long long W = (long long)tl.nx * X, H = (long long)tl.ny * Y;
    const int slots = tl.nx * tl.ny * tl.nz;
    for (long long vx = blockIdx.x * wpb + threadIdx.x / kWarp; vx < nvox; vx += (long long)gridDim.x * wpb) {
        const int z = (int)(vx % Z), y = (int)((vx / Z) % Y), x = (int)(vx / ((long long)Y * Z));
        const float *row = odf + vx * T;
        const bool masked = (double)stop[vx] < thr;
        float m = 0.0f;
        for (int t = lane; t < T; t += kWarp) {
            const float v = masked ? 0.0f : fmaxf(__ldg(row + t), 0.0f);
            m = fmaxf(m, v);
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
        for (int t = lane; t < slots; t += kWarp) {
            float v = 0.0f;
            if (t < T && !masked) {
                v = fmaxf(__ldg(row + t), 0.0f);
                if (m > 0.0f) v = __fdiv_rn(v, m);
            }
            const int tx = t & (tl.nx - 1), ty = (t >> tl.log2x) & (tl.ny - 1), tz = t >> (tl.log2x + tl.log2y);
            tiled[((long long)(tz * Z + z) * H + (ty * Y + y)) * W + (tx * X + x)] = v;
        }
    }
}

// One thread per grid point: nearest vertex (or antipode, when symmetric).
__global__ void ptt_lut_kernel(const float *__restrict__ verts, int V, int symm, int res, float *__restrict__ lut) {
    extern __shared__ double sv[];
    for (int i = threadIdx.x; i < 3 * V; i += blockDim.x) sv[i] = (double)verts[i];
    __syncthreads();
    const long long n = (long long)res * res * res;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const double step = 2.0 / (double)(res - 1);
    auto coord = [&](int i) { return i == res - 1 ? 1.0 : __dadd_rn(__dmul_rn((double)i, step), -1.0); };
    const double gx = coord((int)(p / ((long long)res * res)));
    const double gy = coord((int)((p / res) % res));
    const double gz = coord((int)(p % res));
    double best = 1e300;
    int arg = 0;
    for (int s = 0; s <= symm; s++) {
        const double sg = s ? -1.0 : 1.0;
        for (int v = 0; v < V; v++) {
            const double dx = __dadd_rn(gx, -sg * sv[3 * v]);
            const double dy = __dadd_rn(gy, -sg * sv[3 * v + 1]);
            const double dz = __dadd_rn(gz, -sg * sv[3 * v + 2]);
            const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
            if (d2 < best) {
                best = d2;
                arg = v;
            }
        }
    }
    lut[p] = (float)arg;
}

}  // namespace csl

using namespace csl;

extern "C" {

int csl_ptt_layout(int T, int *nx, int *ny, int *nz, int *log2_x, int *log2_y) {
    if (T <= 0 || !nx || !ny || !nz || !log2_x || !log2_y)
        return tracker_fail(nullptr, CSL_E_INVALID, "csl_ptt_layout: T must be positive, outputs non-NULL");
    const PttTiles t = ptt_tiles(T);
    *nx = t.nx;
    *ny = t.ny;
    *nz = t.nz;
    *log2_x = t.log2x;
    *log2_y = t.log2y;
    return CSL_OK;
}

int csl_ptt_prepare(const float *odf_dev, const float *stop_dev, int X, int Y, int Z, int T, double stop_threshold,
                    const float *verts_dev, int V, int sphere_symm, int lut_res, float *tiled_dev, float *lut_dev,
                    void *stream) {
    if (!odf_dev || !stop_dev || !verts_dev || !tiled_dev || !lut_dev || X <= 0 || Y <= 0 || Z <= 0 || T <= 0 ||
        V <= 0 || V > 4096 || lut_res < 2 || lut_res > 1024)
        return tracker_fail(nullptr, CSL_E_INVALID,
                            "csl_ptt_prepare: null buffer or size out of range (V <= 4096, 2 <= lut_res <= 1024)");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const PttTiles tl = ptt_tiles(T);
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev))
        return tracker_fail(nullptr, CSL_E_CUDA, "csl_ptt_prepare: no current CUDA device");
    ptt_tile_kernel<<<nsm * 8, 256, 0, st>>>(odf_dev, stop_dev, X, Y, Z, T, stop_threshold, tl, tiled_dev);
    if (cudaGetLastError() != cudaSuccess) return tracker_fail(nullptr, CSL_E_CUDA, "csl_ptt_prepare: tile launch");
    const long long n = (long long)lut_res * lut_res * lut_res;
    const int smem = 3 * V * (int)sizeof(double);
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(ptt_lut_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
        return tracker_fail(nullptr, CSL_E_CUDA, "csl_ptt_prepare: LUT shared memory");
    ptt_lut_kernel<<<(unsigned)((n + 255) / 256), 256, smem, st>>>(verts_dev, V, sphere_symm ? 1 : 0, lut_res,
                                                                     lut_dev);
    if (cudaGetLastError() != cudaSuccess) return tracker_fail(nullptr, CSL_E_CUDA, "csl_ptt_prepare: LUT launch");
    return CSL_OK;
}

}  // extern "C"
