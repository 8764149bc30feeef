// Launcher for the REFERENCE's own CUDA kernels, compiled from the reference
// sources where they lie (see oracle/build_ref.py) -- TEST INFRASTRUCTURE ONLY.
//
// The reference launches its kernels from Python through cuda.core with a
// macro set baked in at NVRTC time (cu_direction_getters.py:53-144) and the
// host loop of cu_propagate_seeds.py:206-233.  cuda.core is not installed,
// so this file re-creates that host loop in C++: upload, pass 1
// (getNumStreamlines*_k), host exclusive scan, pass 2
// (genStreamlinesMerge*_k), and a copy of the padded output buffers.  It is
// compiled once per volume shape / parameter set, because the reference
// takes those as macros.  Texture handles are passed through device memory
// (the reference passes the address of a host-side handle).
#include <cstdio>
#include <vector>

#include "generate_streamlines_cuda.cu"

#ifndef REF_MODEL
#error "REF_MODEL must be 0 (OPDT), 1 (CSA), 2 (PROB) or 3 (PTT)"
#endif

#define REF_CK(x)                                                              \
    do {                                                                       \
        cudaError_t _e = (x);                                                  \
        if (_e != cudaSuccess) {                                               \
            fprintf(stderr, "ref_launcher: %s at %d\n", cudaGetErrorString(_e), \
                    __LINE__);                                                 \
            return -(int)_e;                                                   \
        }                                                                      \
    } while (0)

static int make_tex(const float *host, int w, int h, int d, bool border, bool linear, bool norm,
                    cudaArray_t *arr, cudaTextureObject_t *tex) {
    cudaChannelFormatDesc cd = cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat);
    cudaExtent ext = make_cudaExtent(w, h, d);
    REF_CK(cudaMalloc3DArray(arr, &cd, ext, 0));
    cudaMemcpy3DParms cp = {};
    cp.srcPtr = make_cudaPitchedPtr((void *)host, (size_t)w * 4, w, h);
    cp.dstArray = *arr;
    cp.extent = ext;
    cp.kind = cudaMemcpyHostToDevice;
    REF_CK(cudaMemcpy3D(&cp));
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = *arr;
    cudaTextureDesc td = {};
    const cudaTextureAddressMode am = border ? cudaAddressModeBorder : cudaAddressModeClamp;
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = am;
    if (border) td.borderColor[0] = td.borderColor[1] = td.borderColor[2] = -1.0f;
    td.filterMode = linear ? cudaFilterModeLinear : cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = norm ? 1 : 0;
    REF_CK(cudaCreateTextureObject(tex, &rd, &td, nullptr));
    return 0;
}

template <typename T>
static T *dev_copy(const T *h, size_t n) {
    T *d = nullptr;
    if (cudaMalloc(&d, (n ? n : 1) * sizeof(T)) != cudaSuccess) return nullptr;
    if (h && n) cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice);
    return d;
}

extern "C" const char *ref_config(void) {
    static char buf[256];
    snprintf(buf, sizeof(buf), "model=%d dims=%d,%d,%d,%d samplm=%d edges=%d", (int)REF_MODEL, DIMX,
             DIMY, DIMZ, DIMT, SAMPLM_NR, NUM_EDGES);
    return buf;
}

// One batch through the reference kernels.  Outputs (host):
//   counts[n]                       pass-1 peak counts (slineOutOff before the scan)
//   dirs[n * SAMPLM_NR * 3]         pass-1 directions (may be NULL)
//   sl_seed[cap], sl_len[cap]       slineSeed / slineLen
//   slines[cap * 2*MAX_SLINE_LEN*3] padded streamline buffer (may be NULL: not copied)
//   ms_out[2]                       pass-1 / pass-2 kernel times, CUDA events (may be NULL)
// Returns the number of streamlines (or a negative error); when it exceeds
// `cap` only counts/dirs are filled.
extern "C" long long ref_track(const float *seeds, int n, const float *dataf, const float *stop_map,
                               const float *verts, const int *edges, const float *H, const float *R,
                               const float *delta_b, const float *delta_q, const float *sampling,
                               const int *b0s, float min_signal, int delta_nr,
                               const float *ptt_tiled, int tw, int th, int td, const float *ptt_lut,
                               int lut_res, int *counts, float *dirs, int cap, int *sl_seed,
                               int *sl_len, float *slines, float *ms_out) {
    if (n <= 0) return 0;
    cudaEvent_t ev[4];
    for (auto &e : ev) cudaEventCreate(&e);
    const int block_y = THR_X_BL / THR_X_SL;
    dim3 block(THR_X_SL, block_y, 1);
    dim3 grid((n + block_y - 1) / block_y, 1, 1);
    const size_t nvox = (size_t)DIMX * DIMY * DIMZ;

    float3 *seeds_d = (float3 *)dev_copy(seeds, (size_t)n * 3);
    float *verts_d = dev_copy(verts, (size_t)SAMPLM_NR * 3);
    if (REF_MODEL == 2 || REF_MODEL == 3) {
        cudaFree(verts_d);
        verts_d = dev_copy(verts, (size_t)DIMT * 3);
    }
    int2 *edges_d = (int2 *)dev_copy(edges, (size_t)NUM_EDGES * 2);
    int *offs_d = dev_copy<int>(nullptr, n + 1);
    float3 *shdir_d = (float3 *)dev_copy<float>(nullptr, (size_t)SAMPLM_NR * 3 * grid.x * block_y);
    cudaArray_t stop_arr = nullptr, odf_arr = nullptr, lut_arr = nullptr;
    cudaTextureObject_t stop_tex = 0, odf_tex = 0, lut_tex = 0;
    if (make_tex(stop_map, DIMZ, DIMY, DIMX, true, true, false, &stop_arr, &stop_tex)) return -1000;
    cudaTextureObject_t *stop_tex_d = dev_copy(&stop_tex, 1);
    float *dataf_d = nullptr;
    float *H_d = nullptr, *R_d = nullptr, *db_d = nullptr, *dq_d = nullptr, *smp_d = nullptr;
    int *b0_d = nullptr;
    cudaTextureObject_t *odf_tex_d = nullptr, *lut_tex_d = nullptr;
    size_t dyn = 0;
    if (REF_MODEL != 3) dataf_d = dev_copy(dataf, nvox * DIMT);
#if REF_MODEL == 0 || REF_MODEL == 1
    int hr = 0;
    for (int i = 0; i < DIMT; i++) hr += b0s[i] ? 0 : 1;
    H_d = dev_copy(H, (size_t)hr * hr);
    R_d = dev_copy(R, (size_t)hr * hr);
    db_d = dev_copy(delta_b, (size_t)delta_nr * hr);
    dq_d = dev_copy(delta_q, (size_t)delta_nr * hr);
    smp_d = dev_copy(sampling, (size_t)SAMPLM_NR * delta_nr);
    b0_d = dev_copy(b0s, (size_t)DIMT);
    dyn = sizeof(float) * block_y * 2 * (N32DIMT + (N32DIMT > SAMPLM_NR ? N32DIMT : SAMPLM_NR)) +
          sizeof(int) * block_y * SAMPLM_NR;
#endif
#if REF_MODEL == 3
    if (make_tex(ptt_tiled, tw, th, td, false, true, false, &odf_arr, &odf_tex)) return -1001;
    if (make_tex(ptt_lut, lut_res, lut_res, lut_res, false, false, true, &lut_arr, &lut_tex))
        return -1002;
    odf_tex_d = dev_copy(&odf_tex, 1);
    lut_tex_d = dev_copy(&lut_tex, 1);
#endif

    // pass 1
    cudaEventRecord(ev[0]);
#if REF_MODEL == 2
    getNumStreamlinesProb_k<THR_X_SL, THR_X_BL / THR_X_SL, float, float3>
        <<<grid, block>>>(n, seeds_d, dataf_d, (float3 *)verts_d, edges_d, shdir_d, offs_d);
#elif REF_MODEL == 3
    getNumStreamlinesPtt_k<THR_X_SL, THR_X_BL / THR_X_SL, float, float3>
        <<<grid, block>>>(n, seeds_d, odf_tex_d, (float3 *)verts_d, edges_d, shdir_d, offs_d);
#else
    REF_CK(cudaFuncSetAttribute(getNumStreamlinesBoot_k<THR_X_SL, THR_X_BL / THR_X_SL, float, float3>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
    getNumStreamlinesBoot_k<THR_X_SL, THR_X_BL / THR_X_SL, float, float3><<<grid, block, dyn>>>(
        (ModelType)REF_MODEL, min_signal, n, seeds_d, dataf_d, H_d, R_d, delta_nr, db_d, dq_d, b0_d,
        smp_d, (float3 *)verts_d, edges_d, shdir_d, offs_d);
#endif
    REF_CK(cudaGetLastError());
    cudaEventRecord(ev[1]);
    REF_CK(cudaDeviceSynchronize());
    if (ms_out) cudaEventElapsedTime(&ms_out[0], ev[0], ev[1]);
    std::vector<int> off(n + 1);
    REF_CK(cudaMemcpy(off.data(), offs_d, sizeof(int) * n, cudaMemcpyDeviceToHost));
    for (int s = 0; s < n; s++) counts[s] = off[s];
    if (dirs) {
        std::vector<float> hd((size_t)n * SAMPLM_NR * 3);
        REF_CK(cudaMemcpy(hd.data(), shdir_d, hd.size() * 4, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < hd.size(); i++) dirs[i] = hd[i];
    }
    // exclusive scan on the host, as _cumsum_offsets (cu_propagate_seeds.py:95-129)
    long long nsl = 0;
    for (int s = 0; s < n; s++) {
        const int c = off[s];
        off[s] = (int)nsl;
        nsl += c;
    }
    off[n] = (int)nsl;
#if REF_MODEL == 0 || REF_MODEL == 1
    // The reference's bootstrap pass 2 (genStreamlinesMergeBoot_k) is not
    // launched: it faulted with an illegal memory access on this pool.  By
    // reading: its tracking step hands peak_directions_d a one-element shared
    // slot (__sh_new_dir + tidy, boot.cu:773) and every peak after the first
    // is written past it (tracking_helpers.cu:220-226), over shared arrays that
    // hold vertex indices.  Only pass 1 (getNumStreamlinesBoot_k) runs here.
    goto done;
#endif
    if (nsl > cap || nsl == 0) goto done;
    {
        REF_CK(cudaMemcpy(offs_d, off.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
        int *seed_d = dev_copy<int>(nullptr, nsl);
        int *len_d = dev_copy<int>(nullptr, nsl);
        float3 *sl_d = (float3 *)dev_copy<float>(nullptr, (size_t)nsl * 2 * MAX_SLINE_LEN * 3);
        REF_CK(cudaMemset(seed_d, 0xff, sizeof(int) * nsl));
        cudaEventRecord(ev[2]);
#if REF_MODEL == 2
        genStreamlinesMergeProb_k<THR_X_SL, THR_X_BL / THR_X_SL, PROB, const float *__restrict__, float,
                                  float3><<<grid, block>>>(0, n, seeds_d, dataf_d, stop_tex_d, verts_d,
                                                           edges_d, offs_d, shdir_d, seed_d, len_d,
                                                           sl_d);
#elif REF_MODEL == 3
        genStreamlinesMergeProb_k<THR_X_SL, THR_X_BL / THR_X_SL, PTT,
                                  const cudaTextureObject_t *__restrict__, float, float3>
            <<<grid, block>>>(0, n, seeds_d, odf_tex_d, stop_tex_d, lut_tex_d, edges_d, offs_d, shdir_d,
                              seed_d, len_d, sl_d);
#endif
        REF_CK(cudaGetLastError());
        cudaEventRecord(ev[3]);
        REF_CK(cudaDeviceSynchronize());
        if (ms_out) cudaEventElapsedTime(&ms_out[1], ev[2], ev[3]);
        REF_CK(cudaMemcpy(sl_seed, seed_d, sizeof(int) * nsl, cudaMemcpyDeviceToHost));
        REF_CK(cudaMemcpy(sl_len, len_d, sizeof(int) * nsl, cudaMemcpyDeviceToHost));
        if (slines)
            REF_CK(cudaMemcpy(slines, sl_d, (size_t)nsl * 2 * MAX_SLINE_LEN * 12, cudaMemcpyDeviceToHost));
        cudaFree(seed_d);
        cudaFree(len_d);
        cudaFree(sl_d);
    }
done:
    for (auto &e : ev) cudaEventDestroy(e);
    cudaFree(seeds_d); cudaFree(verts_d); cudaFree(edges_d); cudaFree(offs_d); cudaFree(shdir_d);
    cudaFree(stop_tex_d); cudaDestroyTextureObject(stop_tex); cudaFreeArray(stop_arr);
    if (dataf_d) cudaFree(dataf_d);
    if (H_d) { cudaFree(H_d); cudaFree(R_d); cudaFree(db_d); cudaFree(dq_d); cudaFree(smp_d); cudaFree(b0_d); }
    if (odf_tex_d) { cudaFree(odf_tex_d); cudaDestroyTextureObject(odf_tex); cudaFreeArray(odf_arr); }
    if (lut_tex_d) { cudaFree(lut_tex_d); cudaDestroyTextureObject(lut_tex); cudaFreeArray(lut_arr); }
    return nsl;
}
