// GPU probes used only by the test suite to pin the CPU oracle:
//  - the CUDA toolkit generator (curand_init / curand / curand_uniform /
//    curand_normal) as the reference kernels call it, for the black-box
//    Philox stream-layout check;
//  - the float arithmetic of the reference's source expressions compiled
//    with the reference's flags (--use_fast_math), e.g. 3-term dot products;
//  - hardware linear filtering of a 3D float texture with border colour -1
//    (the reference's stop-map check).
// One thread per query; every index is guarded by `q < n`.
#include <cuda_runtime.h>
#include <curand_kernel.h>

__global__ void k_curand(unsigned long long seed, const unsigned long long *subseq,
                         const unsigned long long *offs, int n, int ndraw, unsigned *u32,
                         float *uni, float *nrm) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    curandStatePhilox4_32_10_t st;
    curand_init(seed, subseq[q], offs[q], &st);
    for (int i = 0; i < ndraw; i++) u32[(size_t)q * ndraw + i] = curand(&st);
    curand_init(seed, subseq[q], offs[q], &st);
    for (int i = 0; i < ndraw; i++) uni[(size_t)q * ndraw + i] = curand_uniform(&st);
    curand_init(seed, subseq[q], offs[q], &st);
    for (int i = 0; i < ndraw; i++) nrm[(size_t)q * ndraw + i] = curand_normal(&st);
}

struct f3 { float x, y, z; };

__global__ void k_dot(const f3 *a, const f3 *b, int n, float *out) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const f3 u = a[q], v = b[q];
    out[q] = u.x * v.x + u.y * v.y + u.z * v.z;
}

__global__ void k_tex(cudaTextureObject_t tex, const float *pts, int n, float *out) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    out[q] = tex3D<float>(tex, pts[3 * q + 2], pts[3 * q + 1], pts[3 * q]);
}

__global__ void k_fast(const float *x, int n, float *c, float *l) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    c[q] = __cosf(x[q]);
    l[q] = __logf(x[q]);
}

template <typename T>
static T *dup(const T *h, size_t n) {
    T *d = nullptr;
    if (cudaMalloc(&d, n * sizeof(T) + 16) != cudaSuccess) return nullptr;
    if (h) cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice);
    return d;
}

extern "C" int probe_curand(unsigned long long seed, const unsigned long long *subseq,
                            const unsigned long long *offs, int n, int ndraw, unsigned *u32,
                            float *uni, float *nrm) {
    auto *ds = dup(subseq, n);
    auto *dof = dup(offs, n);
    auto *du = dup<unsigned>(nullptr, (size_t)n * ndraw);
    auto *dn = dup<float>(nullptr, (size_t)n * ndraw);
    auto *dm = dup<float>(nullptr, (size_t)n * ndraw);
    if (!ds || !dof || !du || !dn || !dm) return -1;
    k_curand<<<(n + 63) / 64, 64>>>(seed, ds, dof, n, ndraw, du, dn, dm);
    cudaMemcpy(u32, du, (size_t)n * ndraw * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(uni, dn, (size_t)n * ndraw * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(nrm, dm, (size_t)n * ndraw * 4, cudaMemcpyDeviceToHost);
    const cudaError_t e = cudaDeviceSynchronize();
    cudaFree(ds); cudaFree(dof); cudaFree(du); cudaFree(dn); cudaFree(dm);
    return e == cudaSuccess ? 0 : (int)e;
}

extern "C" int probe_dot(const float *a, const float *b, int n, float *out) {
    auto *da = dup(reinterpret_cast<const f3 *>(a), n);
    auto *db = dup(reinterpret_cast<const f3 *>(b), n);
    auto *dout = dup<float>(nullptr, n);
    if (!da || !db || !dout) return -1;
    k_dot<<<(n + 127) / 128, 128>>>(da, db, n, dout);
    cudaMemcpy(out, dout, (size_t)n * 4, cudaMemcpyDeviceToHost);
    const cudaError_t e = cudaDeviceSynchronize();
    cudaFree(da); cudaFree(db); cudaFree(dout);
    return e == cudaSuccess ? 0 : (int)e;
}

extern "C" int probe_fast(const float *x, int n, float *c, float *l) {
    auto *dx = dup(x, n);
    auto *dc = dup<float>(nullptr, n);
    auto *dl = dup<float>(nullptr, n);
    if (!dx || !dc || !dl) return -1;
    k_fast<<<(n + 127) / 128, 128>>>(dx, n, dc, dl);
    cudaMemcpy(c, dc, (size_t)n * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(l, dl, (size_t)n * 4, cudaMemcpyDeviceToHost);
    const cudaError_t e = cudaDeviceSynchronize();
    cudaFree(dx); cudaFree(dc); cudaFree(dl);
    return e == cudaSuccess ? 0 : (int)e;
}

// vol is C-order [X,Y,Z]; sampled at (z, y, x) like the reference's stop check
extern "C" int probe_tex3d(const float *vol, int X, int Y, int Z, const float *pts, int n, float *out) {
    cudaChannelFormatDesc cd = cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat);
    cudaExtent ext = make_cudaExtent(Z, Y, X);
    cudaArray_t arr = nullptr;
    if (cudaMalloc3DArray(&arr, &cd, ext, 0) != cudaSuccess) return -1;
    cudaMemcpy3DParms cp = {};
    cp.srcPtr = make_cudaPitchedPtr((void *)vol, (size_t)Z * 4, Z, Y);
    cp.dstArray = arr;
    cp.extent = ext;
    cp.kind = cudaMemcpyHostToDevice;
    cudaMemcpy3D(&cp);
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td = {};
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
    td.borderColor[0] = td.borderColor[1] = td.borderColor[2] = td.borderColor[3] = -1.0f;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    cudaTextureObject_t tex = 0;
    if (cudaCreateTextureObject(&tex, &rd, &td, nullptr) != cudaSuccess) return -2;
    auto *dp = dup(pts, (size_t)n * 3);
    auto *dout = dup<float>(nullptr, n);
    k_tex<<<(n + 127) / 128, 128>>>(tex, dp, n, dout);
    cudaMemcpy(out, dout, (size_t)n * 4, cudaMemcpyDeviceToHost);
    const cudaError_t e = cudaDeviceSynchronize();
    cudaDestroyTextureObject(tex);
    cudaFreeArray(arr);
    cudaFree(dp); cudaFree(dout);
    return e == cudaSuccess ? 0 : (int)e;
}
