// C ABI of the tracker (declared in include/gpustreamlines_b200.h).
//
// Host orchestration per batch (replaces SeedBatchPropagator.propagate,
// cu_propagate_seeds.py:206-233):
//   H2D seeds -> pass 1 (seed peaks) -> device exclusive scan of the peak
//   counts -> pass 2 (persistent tracker into a point pool) -> device scan
//   of the streamline lengths -> gather into compacted, ordered points.
// Two 8-byte reads cross PCIe inside a batch (streamline and point totals,
// needed to size the outputs); the pool is grown and pass 2 re-run if the
// first guess of its size was too small (results are deterministic, so a
// re-run produces the same output).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gpustreamlines_b200.h"
#include "kernels.h"

using namespace csl;

namespace {

thread_local std::string g_lib_error;

template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t cap = 0;  // elements
    cudaError_t ensure(size_t n) {
        if (n <= cap && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        const size_t m = std::max<size_t>(n, 1);
        cudaError_t e = cudaMalloc(&p, m * sizeof(T));
        if (e == cudaSuccess) cap = m;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

}  // namespace

struct csl_tracker {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    csl_params hp{};
    DevParams P{};
    std::string err;
    int nsm = 0;
    int block = 256;
    int blocks_per_sm = 1;
    // inputs
    DevBuf<float> dataf, verts, H, R, delta_b, delta_q, sampling;
    DevBuf<int> edges, b0s, partner;
    DevBuf<uint32_t> cone, cone_t;
    // bounded-envelope sampler (prob_sampler == 1)
    DevBuf<uint32_t> env_cmax, env_cone;
    DevBuf<short> env_member;
    DevBuf<unsigned long long> env_stats;
    cudaArray_t stop_arr = nullptr, odf_arr = nullptr, lut_arr = nullptr;
    cudaTextureObject_t stop_tex = 0, odf_tex = 0, lut_tex = 0;
    DevBuf<float> consts;
    // batch
    DevBuf<float> seeds;
    DevBuf<int> npeaks, sl_off, out_len, out_seed, queue, status;
    DevBuf<short> peaks;
    DevBuf<long long> out_src, pt_off;
    DevBuf<unsigned long long> pool_count;
    DevBuf<float> pool, scratch, points;
    DevBuf<unsigned char> scan_tmp, sort_tmp;
    DevBuf<uint32_t> mkeys, mkeys_sorted;
    DevBuf<int> mvals, perm, blk_next, blk_end;
    // batched bootstrap fit (boot_fit 1 or 2)
    BootBatchGeom bgeom{};
    DevBuf<unsigned char> bb_B1, bb_B2, bb_B3;
    DevBuf<int> bb_volidx, bb_sl_seed, bb_half_len, bb_hq;
    DevBuf<short> bb_nbr;
    DevBuf<short> bb_sl_vert;
    DevBuf<long long> bb_half_off;
    DevBuf<float> bb_odf, bb_pts, bb_dwi;
    DevBuf<uint32_t> bb_rng_save;                 // near-tie re-evaluation: saved Philox counters
    DevBuf<float> bb_refit_tab;                   // transposed fit matrices for the re-fit (refit_tab_layout)
    DevBuf<int> bb_refit_idx;                     // resample indices of a re-fit, per warp
    DevBuf<unsigned long long> bb_refit_count;    // rows searched, rows fitted again
    // compression of the last batch (csl_compress)
    DevBuf<float> cmp_world, cmp_pts;
    DevBuf<unsigned char> cmp_keep;
    DevBuf<int> cmp_cnt;
    DevBuf<long long> cmp_off;
    long long cmp_npts = -1;
    long long *host_stage = nullptr;  // pinned 16-byte staging for the two totals
    long long last_n = -1, nsl = 0, npts = 0;
    int ok_batch = 0;
    cudaStream_t last_stream = nullptr;
    // timing events of the last batch: start, pass 1 + scan, pass 2, compaction
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    float ms[4] = {0, 0, 0, 0};
    int pass2_runs = 0;
};

namespace csl {
// internal accessors for the allocation-free entry point (noalloc.cu)
int tracker_view(csl_tracker *t, DevParams *P, const int **partner, int *device) {
    if (!t) return CSL_E_INVALID;
    *P = t->P;
    *partner = t->partner.p;
    *device = t->device;
    return CSL_OK;
}
int tracker_fail(csl_tracker *t, int code, const char *msg) {
    (void)cudaGetLastError();
    if (t)
        t->err = msg;
    else
        g_lib_error = msg;
    return code;
}
}  // namespace csl

static int fail(csl_tracker *t, int code, const char *fmt, ...) {
    (void)cudaGetLastError();  // a failed call's error must not surface in a later launch check
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (t)
        t->err = buf;
    else
        g_lib_error = buf;
    return code;
}

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t _e = (call);                                                          \
        if (_e != cudaSuccess)                                                            \
            return fail(t, _e == cudaErrorMemoryAllocation ? CSL_E_NOMEM : CSL_E_CUDA,    \
                        "CUDA error code=%d(%s) at %s:%d", (int)_e, cudaGetErrorName(_e), \
                        __FILE__, __LINE__);                                              \
    } while (0)

// Batcher's merge-exchange network (Knuth, TAOCP vol. 3, 5.2.2 Algorithm M)
// for 32 keys, comparators placed in the earliest layer their inputs allow.
// partner[l][i] = lane compared with lane i in layer l (i itself if idle).
static std::vector<int> merge_exchange_partners() {
    const int N = 32, t = 5;
    std::vector<std::vector<std::pair<int, int>>> rounds;
    for (int p = 1 << (t - 1); p > 0; p >>= 1) {
        int q = 1 << (t - 1), r = 0, d = p;
        for (;;) {
            std::vector<std::pair<int, int>> rnd;
            for (int i = 0; i < N - d; i++)
                if ((i & p) == r) rnd.emplace_back(i, i + d);
            rounds.push_back(rnd);
            if (q != p) {
                d = q - p;
                q >>= 1;
                r = p;
            } else {
                break;
            }
        }
    }
    std::vector<int> last(N, -1);
    std::vector<std::vector<int>> layers;
    for (auto &rnd : rounds)
        for (auto &c : rnd) {
            const int l = std::max(last[c.first], last[c.second]) + 1;
            while ((int)layers.size() <= l) {
                std::vector<int> id(N);
                for (int i = 0; i < N; i++) id[i] = i;
                layers.push_back(id);
            }
            layers[l][c.first] = c.second;
            layers[l][c.second] = c.first;
            last[c.first] = last[c.second] = l;
        }
    std::vector<int> flat(kMaxSortLayers * N);
    for (int l = 0; l < kMaxSortLayers; l++)
        for (int i = 0; i < N; i++)
            flat[l * N + i] = l < (int)layers.size() ? layers[l][i] : i;
    return flat;
}

static int make_texture3d(csl_tracker *t, const float *src, int w, int h, int d, bool border,
                          bool linear, bool normalized, cudaArray_t *arr, cudaTextureObject_t *tex) {
    cudaChannelFormatDesc cd = cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat);
    cudaExtent ext = make_cudaExtent(w, h, d);
    CK(cudaMalloc3DArray(arr, &cd, ext, 0));
    cudaMemcpy3DParms cp = {};
    cp.srcPtr = make_cudaPitchedPtr((void *)src, (size_t)w * 4, w, h);
    cp.dstArray = *arr;
    cp.extent = ext;
    cp.kind = cudaMemcpyDefault;  // host or device source (unified addressing)
    CK(cudaMemcpy3D(&cp));
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = *arr;
    cudaTextureDesc td = {};
    const cudaTextureAddressMode am = border ? cudaAddressModeBorder : cudaAddressModeClamp;
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = am;
    if (border) td.borderColor[0] = td.borderColor[1] = td.borderColor[2] = td.borderColor[3] = -1.0f;
    td.filterMode = linear ? cudaFilterModeLinear : cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = normalized ? 1 : 0;
    CK(cudaCreateTextureObject(tex, &rd, &td, nullptr));
    return CSL_OK;
}

template <typename T>
static int upload(csl_tracker *t, DevBuf<T> &b, const T *host, size_t n) {
    CK(b.ensure(n));
    CK(cudaMemcpy(b.p, host, n * sizeof(T), cudaMemcpyHostToDevice));
    return CSL_OK;
}

static void release_all(csl_tracker *t) {
    if (t->stop_tex) cudaDestroyTextureObject(t->stop_tex);
    if (t->odf_tex) cudaDestroyTextureObject(t->odf_tex);
    if (t->lut_tex) cudaDestroyTextureObject(t->lut_tex);
    if (t->stop_arr) cudaFreeArray(t->stop_arr);
    if (t->odf_arr) cudaFreeArray(t->odf_arr);
    if (t->lut_arr) cudaFreeArray(t->lut_arr);
    t->stop_tex = t->odf_tex = t->lut_tex = 0;
    t->stop_arr = t->odf_arr = t->lut_arr = nullptr;
    DevBuf<float> *fb[] = {&t->dataf, &t->verts, &t->H, &t->R, &t->delta_b, &t->delta_q,
                           &t->sampling, &t->consts, &t->seeds, &t->pool, &t->scratch, &t->points};
    for (auto *b : fb) b->release();
    DevBuf<int> *ib[] = {&t->edges, &t->b0s, &t->partner, &t->npeaks, &t->sl_off,
                         &t->out_len, &t->out_seed, &t->queue, &t->status};
    for (auto *b : ib) b->release();
    t->cone.release();
    t->cone_t.release();
    t->env_cmax.release();
    t->env_cone.release();
    t->env_member.release();
    t->env_stats.release();
    t->peaks.release();
    t->out_src.release();
    t->pt_off.release();
    t->pool_count.release();
    t->scan_tmp.release();
    t->sort_tmp.release();
    t->mkeys.release();
    t->mkeys_sorted.release();
    DevBuf<int> *ib2[] = {&t->mvals, &t->perm, &t->blk_next, &t->blk_end, &t->bb_volidx,
                          &t->bb_sl_seed, &t->bb_half_len, &t->bb_hq};
    for (auto *b : ib2) b->release();
    t->bb_B1.release();
    t->bb_B2.release();
    t->bb_B3.release();
    t->bb_sl_vert.release();
    t->bb_nbr.release();
    t->bb_half_off.release();
    t->bb_odf.release();
    t->bb_pts.release();
    t->bb_dwi.release();
    t->bb_rng_save.release();
    t->bb_refit_tab.release();
    t->bb_refit_idx.release();
    t->bb_refit_count.release();
    t->cmp_world.release();
    t->cmp_pts.release();
    t->cmp_keep.release();
    t->cmp_cnt.release();
    t->cmp_off.release();
    for (auto &e : t->ev)
        if (e) cudaEventDestroy(e);
    if (t->host_stage) cudaFreeHost(t->host_stage);
    t->host_stage = nullptr;
    if (t->own_stream) cudaStreamDestroy(t->own_stream);
    t->own_stream = nullptr;
}

static int validate(const csl_params *p, const csl_inputs *in, csl_tracker *t) {
    if (!p || !in) return fail(t, CSL_E_INVALID, "params and inputs must not be NULL");
    if (p->model < CSL_MODEL_OPDT || p->model > CSL_MODEL_PTT)
        return fail(t, CSL_E_INVALID, "Invalid model type %d", p->model);
    if (p->dimx <= 0 || p->dimy <= 0 || p->dimz <= 0 || p->dimt <= 0)
        return fail(t, CSL_E_INVALID, "volume dimensions must be positive");
    if ((long long)p->dimx * p->dimy * p->dimz >= (1LL << 31))
        return fail(t, CSL_E_INVALID, "at most 2^31 - 1 voxels");
    if (p->nvertices <= 0 || p->nedges <= 0) return fail(t, CSL_E_INVALID, "empty sphere");
    if (p->prob_sampler != 0 && p->prob_sampler != 1)
        return fail(t, CSL_E_INVALID, "prob_sampler must be 0 or 1");
    if (p->prob_sampler == 1 && p->model != CSL_MODEL_PROB)
        return fail(t, CSL_E_INVALID, "prob_sampler=1 applies to the probabilistic getter only");
    if (p->prob_sampler == 1 && p->dimt > 16 * 64)
        return fail(t, CSL_E_INVALID, "prob_sampler=1 supports at most 1024 sphere vertices");
    if (p->nvertices > 32767) return fail(t, CSL_E_INVALID, "at most 32767 sphere vertices");
    if (p->max_sline_len < 2) return fail(t, CSL_E_INVALID, "max_sline_len must be >= 2");
    if (p->seed_order != 0 && p->seed_order != 1) return fail(t, CSL_E_INVALID, "seed_order must be 0 or 1");
    if (!in->stop_map || !in->vertices || !in->edges)
        return fail(t, CSL_E_INVALID, "stop_map, vertices and edges are required");
    const bool boot = p->model == CSL_MODEL_OPDT || p->model == CSL_MODEL_CSA;
    if (boot) {
        if (!in->dataf || !in->H || !in->R || !in->delta_b || !in->delta_q || !in->sampling_matrix ||
            !in->b0s_mask)
            return fail(t, CSL_E_INVALID, "bootstrap getter needs dataf, H, R, delta_b, delta_q, "
                                          "sampling_matrix and b0s_mask");
        if (p->delta_nr <= 0 || p->samplm_nr <= 0)
            return fail(t, CSL_E_INVALID, "delta_nr and samplm_nr must be positive");
        if (p->samplm_nr != p->nvertices)
            return fail(t, CSL_E_INVALID, "sampling_matrix rows (%d) must equal sphere vertices (%d)",
                        p->samplm_nr, p->nvertices);
        if (p->boot_fit < 0 || p->boot_fit > 2) return fail(t, CSL_E_INVALID, "boot_fit must be 0, 1 or 2");
        if (p->boot_fit >= 1) {
            if (p->dimt > 512) return fail(t, CSL_E_INVALID, "the batched fit supports at most 512 volumes");
            if (p->delta_nr > 64) return fail(t, CSL_E_INVALID, "the batched fit supports at most 64 SH coefficients");
            if (p->samplm_nr > 768) return fail(t, CSL_E_INVALID, "the batched fit supports at most 768 sphere samples");
        }
    } else {
        if (p->nvertices != p->dimt)
            return fail(t, CSL_E_INVALID,
                        "Number of sphere vertices (%d) must match last dimension of dataf (%d), "
                        "because dataf should be an ODF when using prob or ptt tracking",
                        p->nvertices, p->dimt);
        if (p->model == CSL_MODEL_PROB && !in->dataf)
            return fail(t, CSL_E_INVALID, "prob getter needs dataf");
        if (p->model == CSL_MODEL_PROB && p->dimt > 1024)
            return fail(t, CSL_E_INVALID, "prob getter supports at most 1024 sphere vertices");
        if (p->model == CSL_MODEL_PTT) {
            if (!in->ptt_odf_tiled || !in->ptt_lut)
                return fail(t, CSL_E_INVALID, "PTT getter needs ptt_odf_tiled and ptt_lut");
            if (p->step_frac <= 0 || p->odf_lut_res <= 0 || p->tile_nx <= 0 || p->tile_ny <= 0 ||
                p->tile_nz <= 0)
                return fail(t, CSL_E_INVALID, "bad PTT parameters");
        }
    }
    return CSL_OK;
}

extern "C" {

const char *csl_version(void) { return "gpustreamlines_b200 0.1.0 (sm_100a)"; }

int csl_last_error(const csl_tracker *t, char *buf, int buflen) {
    const std::string &s = t ? t->err : g_lib_error;
    if (buf && buflen > 0) {
        std::strncpy(buf, s.c_str(), buflen - 1);
        buf[buflen - 1] = 0;
    }
    return (int)s.size();
}

int csl_create(const csl_params *params, const csl_inputs *inputs, int device, csl_tracker **out) {
    csl_tracker *t = nullptr;
    if (!out) return fail(nullptr, CSL_E_INVALID, "out must not be NULL");
    *out = nullptr;
    int rc = validate(params, inputs, nullptr);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(nullptr, CSL_E_CUDA, "no CUDA device available");
    if (device < 0 || device >= ndev)
        return fail(nullptr, CSL_E_INVALID, "Requested device %d but only %d available", device, ndev);
    t = new csl_tracker();
    t->device = device;
    t->hp = *params;
    rc = [&]() -> int {
        CK(cudaSetDevice(device));
        CK(cudaStreamCreateWithFlags(&t->own_stream, cudaStreamNonBlocking));
        CK(cudaDeviceGetAttribute(&t->nsm, cudaDevAttrMultiProcessorCount, device));
        const csl_params &p = *params;
        DevParams &P = t->P;
        P.model = p.model;
        P.dimx = p.dimx;
        P.dimy = p.dimy;
        P.dimz = p.dimz;
        P.dimt = p.dimt;
        P.nvert = p.nvertices;
        P.nedges = p.nedges;
        const bool boot = p.model == OPDT || p.model == CSA;
        P.samplm_nr = boot ? p.samplm_nr : p.dimt;
        P.sphere_symm = p.sphere_symm ? 1 : 0;
        P.max_sline_len = p.max_sline_len;
        P.nch = (p.model == PROB) ? (P.samplm_nr + 31) / 32 : 1;
        P.vec4 = (p.model == PROB) && (P.samplm_nr % 4 == 0);
        P.step_frac = (p.model == PTT) ? p.step_frac : 1;
        P.step_size = p.step_size;
        P.max_angle = p.max_angle;
        P.tc_threshold = p.tc_threshold;
        P.relative_peak_thresh = p.relative_peak_thresh;
        P.min_separation_angle = p.min_separation_angle;
        P.pmf_threshold = p.pmf_threshold;
        P.rng_seed = p.rng_seed;
        const size_t nvox = (size_t)p.dimx * p.dimy * p.dimz;
        if (p.model != PTT) {
            int r = upload(t, t->dataf, inputs->dataf, nvox * p.dimt);
            if (r) return r;
            P.dataf = t->dataf.p;
        }
        int r = upload(t, t->verts, inputs->vertices, (size_t)p.nvertices * 3);
        if (r) return r;
        r = upload(t, t->edges, inputs->edges, (size_t)p.nedges * 2);
        if (r) return r;
        P.verts = t->verts.p;
        P.edges = reinterpret_cast<const int2 *>(t->edges.p);
        const std::vector<int> part = merge_exchange_partners();
        r = upload(t, t->partner, part.data(), part.size());
        if (r) return r;
        r = make_texture3d(t, inputs->stop_map, p.dimz, p.dimy, p.dimx, true, true, false,
                           &t->stop_arr, &t->stop_tex);
        if (r) return r;
        P.stop_tex = t->stop_tex;
        // cos() of the angles, evaluated on the device with the fast cosine
        CK(t->consts.ensure(2));
        CK(launch_device_cos((float)p.max_angle, (float)p.min_separation_angle, t->consts.p,
                             t->own_stream));
        float cs[2];
        CK(cudaMemcpyAsync(cs, t->consts.p, sizeof(cs), cudaMemcpyDeviceToHost, t->own_stream));
        CK(cudaStreamSynchronize(t->own_stream));
        P.cos_max_angle = cs[0];
        P.cos_min_sep = cs[1];
        if (boot) {
            int hr = 0;
            for (int i = 0; i < p.dimt; i++) hr += inputs->b0s_mask[i] ? 0 : 1;
            if (hr <= 0 || hr > 512)
                return fail(t, CSL_E_INVALID, "bootstrap needs 1..512 non-b0 volumes, got %d", hr);
            if (p.delta_nr > 512) return fail(t, CSL_E_INVALID, "delta_nr must be <= 512");
            P.hr_side = hr;
            P.delta_nr = p.delta_nr;
            P.min_signal = (float)p.min_signal;
            if ((r = upload(t, t->H, inputs->H, (size_t)hr * hr))) return r;
            if ((r = upload(t, t->R, inputs->R, (size_t)hr * hr))) return r;
            if ((r = upload(t, t->delta_b, inputs->delta_b, (size_t)p.delta_nr * hr))) return r;
            if ((r = upload(t, t->delta_q, inputs->delta_q, (size_t)p.delta_nr * hr))) return r;
            if ((r = upload(t, t->sampling, inputs->sampling_matrix, (size_t)p.samplm_nr * p.delta_nr)))
                return r;
            if ((r = upload(t, t->b0s, inputs->b0s_mask, (size_t)p.dimt))) return r;
            P.H = t->H.p;
            P.R = t->R.p;
            P.delta_b = t->delta_b.p;
            P.delta_q = t->delta_q.p;
            P.sampling = t->sampling.p;
            P.b0s_mask = t->b0s.p;
            if (p.boot_fit >= 1) {
                if (hr > 160)
                    return fail(t, CSL_E_INVALID, "the batched fit supports at most 160 non-b0 volumes, got %d", hr);
                // volume order of the batched gather: non-b0 volumes, then b0s
                std::vector<int> volidx;
                for (int i = 0; i < p.dimt; i++)
                    if (!inputs->b0s_mask[i]) volidx.push_back(i);
                for (int i = 0; i < p.dimt; i++)
                    if (inputs->b0s_mask[i]) volidx.push_back(i);
                // sphere neighbour table for the batched peak search
                std::vector<short> nbr((size_t)p.nvertices * kMaxDegree);
                std::vector<int> deg(p.nvertices, 0);
                for (int v = 0; v < p.nvertices; v++)
                    for (int d = 0; d < kMaxDegree; d++) nbr[(size_t)v * kMaxDegree + d] = (short)v;
                for (int e = 0; e < p.nedges; e++) {
                    const int a = inputs->edges[2 * e], b = inputs->edges[2 * e + 1];
                    if (a < 0 || b < 0 || a >= p.nvertices || b >= p.nvertices)
                        return fail(t, CSL_E_INVALID, "edge %d references a missing vertex", e);
                    const int ab[2][2] = {{a, b}, {b, a}};
                    for (const auto &q : ab) {
                        bool seen = false;
                        for (int d = 0; d < deg[q[0]]; d++) seen |= nbr[(size_t)q[0] * kMaxDegree + d] == q[1];
                        if (seen) continue;
                        if (deg[q[0]] == kMaxDegree)
                            return fail(t, CSL_E_INVALID, "the batched fit supports spheres of vertex degree <= %d",
                                        kMaxDegree);
                        nbr[(size_t)q[0] * kMaxDegree + deg[q[0]]++] = (short)q[1];
                    }
                }
                const BootBatchGeom g = boot_batch_geom(P, hr, p.dimt - hr);
                t->bgeom = g;
                if (g.smem > 227 * 1024)
                    return fail(t, CSL_E_INVALID, "the batched fit needs %d B of shared memory per block", g.smem);
                if ((r = upload(t, t->bb_volidx, volidx.data(), volidx.size()))) return r;
                CK(t->bb_dwi.ensure(nvox * (size_t)g.TP));
                CK(launch_boot_batch_dwi(t->dataf.p, t->bb_volidx.p, (long long)nvox, p.dimt, g.TP,
                                         t->bb_dwi.p, t->own_stream));
                nbr.resize((size_t)g.nbr_shorts, 0);
                if ((r = upload(t, t->bb_nbr, nbr.data(), nbr.size()))) return r;
                CK(t->bb_B1.ensure((size_t)g.nchunk1 * g.b1_chunk));
                CK(t->bb_B2.ensure((size_t)g.b2_bytes * (p.model == OPDT ? 2 : 1)));
                CK(t->bb_B3.ensure((size_t)g.nchunk3 * g.b3_chunk));
                CK(t->bb_hq.ensure(1));
                CK(launch_boot_batch_pack(P, g, t->bb_B1.p, t->bb_B2.p, t->bb_B3.p, t->own_stream));
                CK(boot_batch_set_smem(g));
                const size_t slots = (size_t)t->nsm * 128;
                CK(t->bb_odf.ensure(slots * g.vstride));
                CK(t->bb_pts.ensure(slots * (size_t)p.max_sline_len * 3));
                if (p.boot_fit == 2) {
                    // the near-tie re-fit: saved Philox counters, per-warp index
                    // scratch, and the fit matrices transposed for coalesced reads
                    CK(t->bb_rng_save.ensure(slots * 4 * 5));
                    CK(t->bb_refit_idx.ensure((size_t)t->nsm * 16 * kRefitIdx));
                    const int C = p.delta_nr, V = p.samplm_nr;
                    const RefitTab L = refit_tab_layout(hr, C, V);
                    std::vector<float> tab(L.total, 0.0f);
                    for (int i = 0; i < hr; i++)
                        for (int j = 0; j < hr; j++) {
                            tab[L.rh + 2 * ((size_t)i * hr + j)] = inputs->R[(size_t)j * hr + i];
                            tab[L.rh + 2 * ((size_t)i * hr + j) + 1] = inputs->H[(size_t)j * hr + i];
                        }
                    for (int j = 0; j < hr; j++)
                        for (int c = 0; c < C; c++) {
                            tab[L.dq + (size_t)j * kRefitCP + c] = inputs->delta_q[(size_t)c * hr + j];
                            tab[L.db + (size_t)j * kRefitCP + c] = inputs->delta_b[(size_t)c * hr + j];
                        }
                    for (int c = 0; c < C; c++)
                        for (int v = 0; v < V; v++)
                            tab[L.smp + (size_t)c * L.vp + v] = inputs->sampling_matrix[(size_t)v * C + c];
                    if ((r = upload(t, t->bb_refit_tab, tab.data(), tab.size()))) return r;
                }
                CK(t->bb_refit_count.ensure(2));
                CK(cudaMemsetAsync(t->bb_refit_count.p, 0, 2 * sizeof(unsigned long long), t->own_stream));
            }
        }
        if (p.model == PROB) {
            CK(t->cone.ensure((size_t)2 * P.nvert * P.nch));
            CK(t->cone_t.ensure((size_t)2 * P.nvert * kWarp));
            P.cone_mask = t->cone.p;
            P.cone_mask_t = t->cone_t.p;
            CK(launch_cone_mask(P, t->cone.p, t->cone_t.p, t->own_stream));
            if (p.prob_sampler == 1) {
                std::vector<short> member;
                if (!env_clusters(inputs->vertices, p.nvertices, member))
                    return fail(t, CSL_E_INVALID, "prob_sampler=1: a vertex cluster exceeds %d vertices",
                                kEnvMaxMembers);
                if ((r = upload(t, t->env_member, member.data(), member.size()))) return r;
                CK(t->env_cmax.ensure(nvox * kWarp));
                CK(t->env_cone.ensure((size_t)2 * P.nvert * kEnvClusters));
                CK(t->env_stats.ensure(4));
                CK(cudaMemsetAsync(t->env_stats.p, 0, 4 * sizeof(unsigned long long), t->own_stream));
                CK(launch_env_tables(P, t->env_member.p, t->env_cmax.p, t->env_cone.p, t->nsm, t->own_stream));
                P.env = 1;
                P.env_cmax = t->env_cmax.p;
                P.env_cone = t->env_cone.p;
                P.env_member = t->env_member.p;
                P.env_stats = t->env_stats.p;
            }
        }
        if (p.model == PTT) {
            r = make_texture3d(t, inputs->ptt_odf_tiled, p.tile_nx * p.dimx, p.tile_ny * p.dimy,
                               p.tile_nz * p.dimz, false, true, false, &t->odf_arr, &t->odf_tex);
            if (r) return r;
            r = make_texture3d(t, inputs->ptt_lut, p.odf_lut_res, p.odf_lut_res, p.odf_lut_res, false,
                               false, true, &t->lut_arr, &t->lut_tex);
            if (r) return r;
            P.odf_tex = t->odf_tex;
            P.lut_tex = t->lut_tex;
            P.log2_x = p.tile_log2_x;
            P.log2_y = p.tile_log2_y;
            P.width_mask = p.tile_nx - 1;
            P.height_mask = p.tile_ny - 1;
            P.probe_step_size = (float)p.probe_step_size;
            P.probe_quality = (float)p.probe_quality;
            P.max_curvature = p.max_curvature;
            // PTT: 128-thread CTAs track 1.33x faster than 256-thread ones on B200
            // (csl_autotune on 100k seeds of the 81x106x76 phantom: 43.3 s vs 57.7 s)
            t->block = 128;
        }
        const int smem = smem_bytes(P, t->block / kWarp, true);
        if (smem > 227 * 1024) {
            t->block = 128;
        }
        CK(track_occupancy(P, t->block, &t->blocks_per_sm));
        if (t->blocks_per_sm < 1) {
            t->block = 64;
            CK(track_occupancy(P, t->block, &t->blocks_per_sm));
            if (t->blocks_per_sm < 1)
                return fail(t, CSL_E_INVALID, "kernel does not fit on the device (shared memory %d B)",
                            smem_bytes(P, t->block / kWarp, true));
        }
        for (auto &e : t->ev) CK(cudaEventCreate(&e));
        CK(cudaMallocHost(&t->host_stage, 2 * sizeof(long long)));
        CK(t->queue.ensure(1));
        CK(t->status.ensure(1));
        CK(t->pool_count.ensure(1));
        CK(cudaStreamSynchronize(t->own_stream));
        return CSL_OK;
    }();
    if (rc) {
        g_lib_error = t->err;
        release_all(t);
        delete t;
        return rc;
    }
    *out = t;
    return CSL_OK;
}

int csl_destroy(csl_tracker *t) {
    if (!t) return CSL_OK;
    cudaSetDevice(t->device);
    cudaDeviceSynchronize();
    release_all(t);
    delete t;
    return CSL_OK;
}

// Pass 2 with the batched tensor-core fit (boot_fit 1 or 2): streamline halves
// are tracked independently, 128 per CTA, and joined afterwards.  Returns
// kUsePerWarpPath when a seed has more initial directions than pass 1 stores
// (the per-warp path recomputes them).
static constexpr int kUsePerWarpPath = 1;

// pass 2 of this tracker runs the batched tensor-core fit (whenever pass 1
// stored every seed's initial directions)
static bool uses_batched_fit(const csl_tracker *t) {
    return t->hp.boot_fit >= 1 && (t->P.model == CSA || t->P.model == OPDT);
}

// Near-tie re-evaluation of the batched fit: on for boot_fit = 2, off for 1.
// The flag margin is 8e-5 of the row maximum: a decision compares two ODF
// values, each off by at most 2.9e-5 of the row maximum in BF16x3 (the
// largest error measured against float64), so only a gap below 5.8e-5 can
// flip.
static void set_refit(csl_tracker *t, BootBatchArgs &A) {
    A.refit = t->hp.boot_fit == 2 ? 1 : 0;
    A.refit_tol = 8e-5f;
    A.rng_save = t->bb_rng_save.p;
    A.refit_tab = t->bb_refit_tab.p;
    A.refit_idx = t->bb_refit_idx.p;
    A.refit_count = t->bb_refit_count.p;
}

// the batched pass 2 of a batch of nsl streamlines (nsl: the slot capacity
// when the count is read on the device), pool_cap points of pool
static void boot_args(csl_tracker *t, BootBatchArgs &A, const float *seeds_dev, int nsl, long long rng_base,
                      unsigned long long pool_cap) {
    A.B1g = t->bb_B1.p;
    A.B2g = t->bb_B2.p;
    A.B3g = t->bb_B3.p;
    A.volidx = t->bb_volidx.p;
    A.nbr = t->bb_nbr.p;
    A.dwi = t->bb_dwi.p;
    A.seeds = seeds_dev;
    A.sl_seed = t->bb_sl_seed.p;
    A.sl_vert = t->bb_sl_vert.p;
    A.nsl = nsl;
    A.rng_base = rng_base;
    A.hq = t->bb_hq.p;
    A.odf = t->bb_odf.p;
    A.pts = t->bb_pts.p;
    A.pool_count = t->pool_count.p;
    A.pool = t->pool.p;
    A.pool_cap = pool_cap;
    A.half_len = t->bb_half_len.p;
    A.half_off = t->bb_half_off.p;
    A.status = t->status.p;
    set_refit(t, A);
}

static int run_boot_batch(csl_tracker *t, const float *seeds_dev, int ni, int nsl, long long rng_base,
                          cudaStream_t st) {
    const DevParams &P = t->P;
    const BootBatchGeom &g = t->bgeom;
    CK(t->bb_sl_seed.ensure((size_t)nsl + 1));
    CK(t->bb_sl_vert.ensure((size_t)nsl + 1));
    CK(t->bb_half_len.ensure((size_t)2 * nsl + 2));
    CK(t->bb_half_off.ensure((size_t)2 * nsl + 2));
    CK(cudaMemsetAsync(t->status.p, 0, sizeof(int), st));
    CK(launch_boot_batch_prep(t->npeaks.p, t->sl_off.p, t->peaks.p, kMaxStoredPeaksPerSeed, ni, nsl,
                              t->bb_sl_seed.p, t->bb_sl_vert.p, t->status.p, st));
    CK(cudaMemcpyAsync(t->host_stage, t->status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if ((int)(t->host_stage[0] & 0xffffffff) & ST_PEAKS_OVERFLOW) return kUsePerWarpPath;

    unsigned long long want = std::max<unsigned long long>(t->pool.cap / 3, (unsigned long long)nsl * 96ull);
    for (int attempt = 0; attempt < 2; attempt++) {
        CK(t->pool.ensure(want * 3));
        BootBatchArgs A{};
        boot_args(t, A, seeds_dev, nsl, rng_base, t->pool.cap / 3);
        CK(cudaMemsetAsync(t->bb_hq.p, 0, sizeof(int), st));
        CK(cudaMemsetAsync(t->status.p, 0, sizeof(int), st));
        CK(cudaMemsetAsync(t->pool_count.p, 0, sizeof(unsigned long long), st));
        CK(cudaEventRecord(t->ev[2], st));
        if (nsl > 0) CK(launch_boot_batch(P, g, A, t->partner.p, t->nsm, st));
        CK(cudaEventRecord(t->ev[3], st));
        t->pass2_runs++;
        CK(cudaMemcpyAsync(t->host_stage, t->status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(t->host_stage + 1, t->pool_count.p, sizeof(unsigned long long),
                           cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        const int status = (int)(t->host_stage[0] & 0xffffffff);
        const unsigned long long used = (unsigned long long)t->host_stage[1];
        if (status & ST_WAIT_TIMEOUT) return fail(t, CSL_E_KERNEL, "tensor-core pipeline wait timed out");
        if (!(status & ST_POOL_OVERFLOW)) break;
        if (attempt == 1) return fail(t, CSL_E_KERNEL, "point pool overflow after resize");
        want = used + used / 8 + 1024;
    }

    // join the halves, scan the lengths, gather
    CK(launch_boot_batch_join(t->bb_half_len.p, t->bb_sl_seed.p, nsl, nullptr, t->out_len.p, t->out_seed.p, st));
    CK(cudaMemsetAsync(t->out_len.p + nsl, 0, sizeof(int), st));
    size_t tmpb = 0;
    CK(scan_temp_bytes(nsl + 1, &tmpb));
    if (tmpb > t->scan_tmp.cap) {
        CK(cudaStreamSynchronize(st));
        CK(t->scan_tmp.ensure(tmpb));
    }
    CK(exclusive_scan_i64(t->scan_tmp.p, t->scan_tmp.cap, t->out_len.p, t->pt_off.p, nsl + 1, st));
    CK(cudaMemcpyAsync(t->host_stage, t->pt_off.p + nsl, sizeof(long long), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const long long npts = t->host_stage[0];
    t->npts = npts;
    CK(t->points.ensure((size_t)npts * 3 + 3));
    if (nsl > 0)
        CK(launch_gather_halves(t->pool.p, t->bb_half_off.p, t->bb_half_len.p, t->pt_off.p, nsl, nullptr,
                                nullptr, t->points.p, t->nsm * 8, st));
    CK(cudaEventRecord(t->ev[4], st));
    CK(cudaStreamSynchronize(st));
    CK(cudaEventElapsedTime(&t->ms[0], t->ev[0], t->ev[1]));
    CK(cudaEventElapsedTime(&t->ms[1], t->ev[1], t->ev[2]));
    CK(cudaEventElapsedTime(&t->ms[2], t->ev[2], t->ev[3]));
    CK(cudaEventElapsedTime(&t->ms[3], t->ev[3], t->ev[4]));
    t->ok_batch = 1;
    return CSL_OK;
}

static int run_batch(csl_tracker *t, const float *seeds_dev, long long n, long long rng_base, cudaStream_t st) {
    const DevParams &P = t->P;
    t->ok_batch = 0;
    t->cmp_npts = -1;
    t->nsl = t->npts = 0;
    t->last_n = n;
    t->last_stream = st;
    for (float &m : t->ms) m = 0;
    t->pass2_runs = 0;
    if (n == 0) {
        t->ok_batch = 1;
        return CSL_OK;
    }
    if (n > (1ll << 30)) return fail(t, CSL_E_INVALID, "batch too large (%lld seeds)", n);
    const int ni = (int)n;
    CK(t->npeaks.ensure(ni + 1));
    CK(t->sl_off.ensure(ni + 1));
    CK(t->peaks.ensure((size_t)ni * kMaxStoredPeaksPerSeed));
    size_t tmpb = 0;
    CK(scan_temp_bytes(ni + 1, &tmpb));
    CK(t->scan_tmp.ensure(tmpb));

    // pass 1
    CK(cudaEventRecord(t->ev[0], st));
    const int wpb = t->block / kWarp;
    const int grid1 = std::min<long long>((n + wpb - 1) / wpb, (long long)t->nsm * 16);
    CK(cudaMemsetAsync(t->npeaks.p + ni, 0, sizeof(int), st));
    CK(launch_seed_peaks(P, seeds_dev, ni, rng_base, t->partner.p, t->npeaks.p, t->peaks.p,
                         kMaxStoredPeaksPerSeed, grid1, t->block, st));
    CK(exclusive_scan_i32(t->scan_tmp.p, t->scan_tmp.cap, t->npeaks.p, t->sl_off.p, ni + 1, st));
    CK(cudaEventRecord(t->ev[1], st));
    int *nsl_h = reinterpret_cast<int *>(t->host_stage);
    CK(cudaMemcpyAsync(nsl_h, t->sl_off.p + ni, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const int nsl = *nsl_h;
    t->nsl = nsl;
    CK(t->out_len.ensure((size_t)nsl + 1));
    CK(t->out_seed.ensure((size_t)nsl + 1));
    CK(t->out_src.ensure((size_t)nsl + 1));
    CK(t->pt_off.ensure((size_t)nsl + 1));

    if (uses_batched_fit(t)) {
        const int r = run_boot_batch(t, seeds_dev, ni, nsl, rng_base, st);
        if (r != kUsePerWarpPath) return r;
    }

    // pass 2 (re-run once with an exact pool size if the guess was short)
    const long long warps_needed = n;
    const int grid2 = (int)std::max<long long>(
        1, std::min<long long>((long long)t->nsm * t->blocks_per_sm, (warps_needed + wpb - 1) / wpb));
    CK(t->scratch.ensure((size_t)grid2 * wpb * scratch_floats_per_warp(P)));
    if (t->hp.seed_order == 1) {
        size_t sb = 0;
        CK(spatial_order(nullptr, ni, grid2, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                         nullptr, &sb, st));
        CK(t->sort_tmp.ensure(sb));
        CK(t->mkeys.ensure(ni));
        CK(t->mkeys_sorted.ensure(ni));
        CK(t->mvals.ensure(ni));
        CK(t->perm.ensure(ni));
        CK(t->blk_next.ensure(grid2));
        CK(t->blk_end.ensure(grid2));
    }
    unsigned long long want = std::max<unsigned long long>(t->pool.cap / 3, (unsigned long long)nsl * 96ull);
    for (int attempt = 0; attempt < 2; attempt++) {
        CK(t->pool.ensure(want * 3));
        BatchArgs B{};
        B.seeds = seeds_dev;
        B.nseeds = ni;
        B.rng_index_base = rng_base;
        B.queue = t->queue.p;
        B.pool_count = t->pool_count.p;
        B.pool = t->pool.p;
        B.pool_cap = t->pool.cap / 3;
        B.scratch = t->scratch.p;
        B.status = t->status.p;
        B.sl_cap = nsl;
        if (t->hp.seed_order == 1) {
            size_t sb = t->sort_tmp.cap;
            CK(spatial_order(seeds_dev, ni, grid2, t->mkeys.p, t->mkeys_sorted.p, t->mvals.p, t->perm.p,
                             t->blk_next.p, t->blk_end.p, t->sort_tmp.p, &sb, st));
            B.perm = t->perm.p;
            B.blk_next = t->blk_next.p;
            B.blk_end = t->blk_end.p;
        }
        CK(cudaMemsetAsync(t->queue.p, 0, sizeof(int), st));
        CK(cudaMemsetAsync(t->status.p, 0, sizeof(int), st));
        CK(cudaMemsetAsync(t->pool_count.p, 0, sizeof(unsigned long long), st));
        CK(cudaEventRecord(t->ev[2], st));
        CK(launch_track(P, B, t->partner.p, t->npeaks.p, t->peaks.p, kMaxStoredPeaksPerSeed,
                        t->sl_off.p, t->out_len.p, t->out_seed.p, t->out_src.p, grid2, t->block, st));
        CK(cudaEventRecord(t->ev[3], st));
        t->pass2_runs++;
        CK(cudaMemcpyAsync(t->host_stage, t->status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(t->host_stage + 1, t->pool_count.p, sizeof(unsigned long long),
                           cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        const int status = (int)(t->host_stage[0] & 0xffffffff);
        const unsigned long long used = (unsigned long long)t->host_stage[1];
        if (!(status & ST_POOL_OVERFLOW)) break;
        if (attempt == 1) return fail(t, CSL_E_KERNEL, "point pool overflow after resize");
        want = used + used / 8 + 1024;
    }

    // compaction
    CK(cudaMemsetAsync(t->out_len.p + nsl, 0, sizeof(int), st));
    CK(scan_temp_bytes(nsl + 1, &tmpb));
    if (tmpb > t->scan_tmp.cap) {
        CK(cudaStreamSynchronize(st));
        CK(t->scan_tmp.ensure(tmpb));
    }
    CK(exclusive_scan_i64(t->scan_tmp.p, t->scan_tmp.cap, t->out_len.p, t->pt_off.p, nsl + 1, st));
    CK(cudaMemcpyAsync(t->host_stage, t->pt_off.p + nsl, sizeof(long long), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const long long npts = t->host_stage[0];
    t->npts = npts;
    CK(t->points.ensure((size_t)npts * 3 + 3));
    CK(launch_gather(t->pool.p, t->out_src.p, t->out_len.p, t->pt_off.p, nsl, t->points.p,
                     t->nsm * 8, st));
    CK(cudaEventRecord(t->ev[4], st));
    CK(cudaStreamSynchronize(st));
    CK(cudaEventElapsedTime(&t->ms[0], t->ev[0], t->ev[1]));
    CK(cudaEventElapsedTime(&t->ms[1], t->ev[1], t->ev[2]));
    CK(cudaEventElapsedTime(&t->ms[2], t->ev[2], t->ev[3]));
    CK(cudaEventElapsedTime(&t->ms[3], t->ev[3], t->ev[4]));
    t->ok_batch = 1;
    return CSL_OK;
}

static int boot_probe(csl_tracker *t, const float *points_dev, const int *resample_dev, long long n, int fit,
                      float *odf_dev, int odf_stride, const float *dirs_dev, float *step_dev, void *stream) {
    if (!t) return fail(nullptr, CSL_E_INVALID, "NULL tracker");
    const DevParams &P = t->P;
    if (P.model != CSA && P.model != OPDT) return fail(t, CSL_E_STATE, "csl_boot_odf needs a bootstrap tracker");
    if (n < 0 || n > (1ll << 30)) return fail(t, CSL_E_INVALID, "bad point count");
    if (fit != 0 && fit != 1) return fail(t, CSL_E_INVALID, "fit must be 0 or 1");
    if (fit == 1 && t->hp.boot_fit < 1)
        return fail(t, CSL_E_STATE, "fit=1 needs a tracker created with boot_fit 1 or 2");
    if (odf_stride < P.samplm_nr || odf_stride % 4 != 0)
        return fail(t, CSL_E_INVALID, "odf_stride must be >= samplm_nr and a multiple of 4");
    if (n == 0) return CSL_OK;
    if (!points_dev || !resample_dev || !odf_dev) return fail(t, CSL_E_INVALID, "NULL buffer");
    CK(cudaSetDevice(t->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : t->own_stream;
    CK(cudaMemsetAsync(odf_dev, 0, (size_t)n * odf_stride * sizeof(float), st));
    if (fit == 0) {
        CK(launch_boot_odf_plain(P, points_dev, resample_dev, (int)n, odf_dev, odf_stride, st));
    } else {
        const BootBatchGeom &g = t->bgeom;
        BootBatchArgs A{};
        A.B1g = t->bb_B1.p;
        A.B2g = t->bb_B2.p;
        A.B3g = t->bb_B3.p;
        A.volidx = t->bb_volidx.p;
        A.nbr = t->bb_nbr.p;
        A.dwi = t->bb_dwi.p;
        A.hq = t->bb_hq.p;
        A.odf = t->bb_odf.p;
        A.pts = t->bb_pts.p;
        A.status = t->status.p;
        A.nprobe = (int)n;
        A.probe_pts = points_dev;
        A.probe_idx = resample_dev;
        A.probe_odf = odf_dev;
        A.probe_stride = odf_stride;
        set_refit(t, A);
        A.probe_dirs = dirs_dev;
        A.probe_step = step_dev;
        CK(cudaMemsetAsync(t->bb_hq.p, 0, sizeof(int), st));
        CK(cudaMemsetAsync(t->status.p, 0, sizeof(int), st));
        CK(launch_boot_batch(P, g, A, t->partner.p, t->nsm, st));
        CK(cudaMemcpyAsync(t->host_stage, t->status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    if (fit == 1 && ((int)(t->host_stage[0] & 0xffffffff) & ST_WAIT_TIMEOUT))
        return fail(t, CSL_E_KERNEL, "tensor-core pipeline wait timed out");
    return CSL_OK;
}

int csl_boot_odf(csl_tracker *t, const float *points_dev, const int *resample_dev, long long n, int fit,
                 float *odf_dev, int odf_stride, void *stream) {
    return boot_probe(t, points_dev, resample_dev, n, fit, odf_dev, odf_stride, nullptr, nullptr, stream);
}

int csl_boot_step(csl_tracker *t, const float *points_dev, const int *resample_dev, const float *dirs_dev,
                  long long n, float *odf_dev, int odf_stride, float *step_dev, void *stream) {
    if (!t) return fail(nullptr, CSL_E_INVALID, "NULL tracker");
    if (t->hp.boot_fit < 1) return fail(t, CSL_E_STATE, "csl_boot_step needs a tracker created with boot_fit >= 1");
    if (n > 0 && (!dirs_dev || !step_dev)) return fail(t, CSL_E_INVALID, "NULL buffer");
    return boot_probe(t, points_dev, resample_dev, n, 1, odf_dev, odf_stride, dirs_dev, step_dev, stream);
}

int csl_boot_refit_stats(csl_tracker *t, unsigned long long *out2, int reset) {
    if (!t) return fail(nullptr, CSL_E_INVALID, "NULL tracker");
    if (t->hp.boot_fit < 1) return fail(t, CSL_E_STATE, "no batched fit on this tracker");
    CK(cudaSetDevice(t->device));
    if (out2)
        CK(cudaMemcpyAsync(out2, t->bb_refit_count.p, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                           t->own_stream));
    if (reset) CK(cudaMemsetAsync(t->bb_refit_count.p, 0, 2 * sizeof(unsigned long long), t->own_stream));
    CK(cudaStreamSynchronize(t->own_stream));
    return CSL_OK;
}

int csl_compress(csl_tracker *t, const double *affine16, double tol_error, double max_segment_length,
                 int minlen, int maxlen, long long *npts_out) {
    if (!t) return fail(nullptr, CSL_E_INVALID, "NULL tracker");
    if (!t->ok_batch) return fail(t, CSL_E_STATE, "no completed batch to compress");
    if (!(tol_error >= 0.0) || !(max_segment_length > 0.0))
        return fail(t, CSL_E_INVALID, "tol_error must be >= 0 and max_segment_length > 0");
    CK(cudaSetDevice(t->device));
    cudaStream_t st = t->last_stream ? t->last_stream : t->own_stream;
    const int nsl = (int)t->nsl;
    const long long npts = t->npts;
    CK(t->cmp_world.ensure((size_t)std::max<long long>(npts, 1) * 3));
    CK(t->cmp_pts.ensure((size_t)std::max<long long>(npts, 1) * 3));
    CK(t->cmp_keep.ensure((size_t)std::max<long long>(npts, 1)));
    CK(t->cmp_cnt.ensure((size_t)nsl + 1));
    CK(t->cmp_off.ensure((size_t)nsl + 1));
    CK(launch_compress(t->points.p, npts, affine16, t->pt_off.p, t->out_len.p, nsl, minlen, maxlen, tol_error,
                       max_segment_length, t->cmp_world.p, t->cmp_keep.p, t->cmp_cnt.p, st));
    CK(cudaMemsetAsync(t->cmp_cnt.p + nsl, 0, sizeof(int), st));
    size_t tmpb = 0;
    CK(scan_temp_bytes(nsl + 1, &tmpb));
    if (tmpb > t->scan_tmp.cap) {
        CK(cudaStreamSynchronize(st));
        CK(t->scan_tmp.ensure(tmpb));
    }
    CK(exclusive_scan_i64(t->scan_tmp.p, t->scan_tmp.cap, t->cmp_cnt.p, t->cmp_off.p, nsl + 1, st));
    CK(launch_compress_gather(t->cmp_world.p, t->pt_off.p, t->out_len.p, t->cmp_keep.p, t->cmp_off.p, nsl,
                              t->cmp_pts.p, st));
    CK(cudaMemcpyAsync(t->host_stage, t->cmp_off.p + nsl, sizeof(long long), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    t->cmp_npts = t->host_stage[0];
    if (npts_out) *npts_out = t->cmp_npts;
    return CSL_OK;
}

int csl_fetch_compressed(csl_tracker *t, int *counts_host, float *points_host) {
    if (!t) return fail(nullptr, CSL_E_INVALID, "NULL tracker");
    if (!t->ok_batch || t->cmp_npts < 0) return fail(t, CSL_E_STATE, "call csl_compress first");
    CK(cudaSetDevice(t->device));
    cudaStream_t st = t->last_stream ? t->last_stream : t->own_stream;
    if (counts_host && t->nsl > 0)
        CK(cudaMemcpyAsync(counts_host, t->cmp_cnt.p, (size_t)t->nsl * sizeof(int), cudaMemcpyDeviceToHost, st));
    if (points_host && t->cmp_npts > 0)
        CK(cudaMemcpyAsync(points_host, t->cmp_pts.p, (size_t)t->cmp_npts * 3 * sizeof(float),
                           cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return CSL_OK;
}

int csl_propagate_device(csl_tracker *t, const float *seeds_dev, long long n, long long rng_index_base,
                         void *stream) {
    if (!t) return fail(nullptr, CSL_E_INVALID, "NULL tracker");
    if (n < 0 || (n > 0 && !seeds_dev)) return fail(t, CSL_E_INVALID, "bad seeds");
    CK(cudaSetDevice(t->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : t->own_stream;
    return run_batch(t, seeds_dev, n, rng_index_base, st);
}

int csl_propagate(csl_tracker *t, const float *seeds_host, long long n, long long rng_index_base,
                  void *stream) {
    if (!t) return fail(nullptr, CSL_E_INVALID, "NULL tracker");
    if (n < 0 || (n > 0 && !seeds_host)) return fail(t, CSL_E_INVALID, "bad seeds");
    CK(cudaSetDevice(t->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : t->own_stream;
    CK(t->seeds.ensure((size_t)std::max<long long>(n, 1) * 3));
    if (n > 0)
        CK(cudaMemcpyAsync(t->seeds.p, seeds_host, (size_t)n * 3 * sizeof(float),
                           cudaMemcpyHostToDevice, st));
    return run_batch(t, t->seeds.p, n, rng_index_base, st);
}

int csl_counts(csl_tracker *t, long long *n_streamlines, long long *n_points) {
    if (!t) return fail(nullptr, CSL_E_INVALID, "NULL tracker");
    if (!t->ok_batch) return fail(t, CSL_E_STATE, "no completed batch");
    if (n_streamlines) *n_streamlines = t->nsl;
    if (n_points) *n_points = t->npts;
    return CSL_OK;
}

int csl_fetch(csl_tracker *t, int *lengths, int *seed_index, float *points) {
    if (!t) return fail(nullptr, CSL_E_INVALID, "NULL tracker");
    if (!t->ok_batch) return fail(t, CSL_E_STATE, "no completed batch");
    CK(cudaSetDevice(t->device));
    cudaStream_t st = t->last_stream ? t->last_stream : t->own_stream;
    if (t->nsl > 0) {
        if (lengths)
            CK(cudaMemcpyAsync(lengths, t->out_len.p, (size_t)t->nsl * sizeof(int),
                               cudaMemcpyDeviceToHost, st));
        if (seed_index)
            CK(cudaMemcpyAsync(seed_index, t->out_seed.p, (size_t)t->nsl * sizeof(int),
                               cudaMemcpyDeviceToHost, st));
    }
    if (points && t->npts > 0)
        CK(cudaMemcpyAsync(points, t->points.p, (size_t)t->npts * 3 * sizeof(float),
                           cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return CSL_OK;
}

int csl_device_results(csl_tracker *t, const int **lengths, const int **seed_index,
                       const long long **point_offsets, const float **points) {
    if (!t) return fail(nullptr, CSL_E_INVALID, "NULL tracker");
    if (!t->ok_batch) return fail(t, CSL_E_STATE, "no completed batch");
    if (lengths) *lengths = t->out_len.p;
    if (seed_index) *seed_index = t->out_seed.p;
    if (point_offsets) *point_offsets = t->pt_off.p;
    if (points) *points = t->points.p;
    return CSL_OK;
}

int csl_seed_peaks(csl_tracker *t, const float *seeds_host, long long n, int max_peaks, int *counts,
                   int *peak_vertex, float *peak_dirs) {
    if (!t) return fail(nullptr, CSL_E_INVALID, "NULL tracker");
    if (n < 0 || (n > 0 && (!seeds_host || !counts)) || max_peaks < 0 || max_peaks > 32767)
        return fail(t, CSL_E_INVALID, "bad arguments");
    if (n == 0) return CSL_OK;
    CK(cudaSetDevice(t->device));
    cudaStream_t st = t->own_stream;
    const int ni = (int)n;
    const int mp = std::max(max_peaks, 1);
    DevBuf<float> sd;
    DevBuf<int> cnt;
    DevBuf<short> pk;
    auto cleanup = [&]() { sd.release(); cnt.release(); pk.release(); };
    cudaError_t e = sd.ensure((size_t)ni * 3);
    if (e == cudaSuccess) e = cnt.ensure(ni);
    if (e == cudaSuccess) e = pk.ensure((size_t)ni * mp);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(sd.p, seeds_host, (size_t)ni * 3 * sizeof(float), cudaMemcpyHostToDevice, st);
    const int wpb = t->block / kWarp;
    if (e == cudaSuccess)
        e = launch_seed_peaks(t->P, sd.p, ni, 0, t->partner.p, cnt.p, pk.p, mp,
                              std::min((ni + wpb - 1) / wpb, t->nsm * 16), t->block, st);
    std::vector<short> hpk((size_t)ni * mp);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(counts, cnt.p, (size_t)ni * sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(hpk.data(), pk.p, hpk.size() * sizeof(short), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cleanup();
    CK(e);
    std::vector<float> hv((size_t)t->P.nvert * 3);
    if (peak_dirs) CK(cudaMemcpy(hv.data(), t->verts.p, hv.size() * 4, cudaMemcpyDeviceToHost));
    for (int s = 0; s < ni; s++)
        for (int k = 0; k < max_peaks; k++) {
            const int v = (k < counts[s]) ? hpk[(size_t)s * mp + k] : -1;
            if (peak_vertex) peak_vertex[(size_t)s * max_peaks + k] = v;
            if (peak_dirs)
                for (int c = 0; c < 3; c++)
                    peak_dirs[((size_t)s * max_peaks + k) * 3 + c] = v >= 0 ? hv[3 * v + c] : 0.0f;
        }
    return CSL_OK;
}

int csl_get_direction(csl_tracker *t, const float *points, const float *dirs,
                      const unsigned long long *subsequence, const unsigned long long *offset,
                      long long n, float *frames, float *new_dirs, int *ok, int *draws) {
    if (!t) return fail(nullptr, CSL_E_INVALID, "NULL tracker");
    if (n < 0 || (n > 0 && (!points || !dirs || !subsequence || !offset || !new_dirs || !ok)))
        return fail(t, CSL_E_INVALID, "bad arguments");
    if (t->P.model == PTT && n > 0 && !frames) return fail(t, CSL_E_INVALID, "PTT needs frames");
    if (n == 0) return CSL_OK;
    CK(cudaSetDevice(t->device));
    cudaStream_t st = t->own_stream;
    const int ni = (int)n;
    DevBuf<float> pd, dd, fr, od;
    DevBuf<unsigned long long> sq, of;
    DevBuf<int> okd, drd;
    cudaError_t e = cudaSuccess;
    auto step = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
    step(pd.ensure((size_t)ni * 3));
    step(dd.ensure((size_t)ni * 3));
    step(fr.ensure((size_t)ni * 9));
    step(od.ensure((size_t)ni * 3));
    step(sq.ensure(ni));
    step(of.ensure(ni));
    step(okd.ensure(ni));
    step(drd.ensure(ni));
    step(cudaMemcpyAsync(pd.p, points, (size_t)ni * 12, cudaMemcpyHostToDevice, st));
    step(cudaMemcpyAsync(dd.p, dirs, (size_t)ni * 12, cudaMemcpyHostToDevice, st));
    step(cudaMemcpyAsync(sq.p, subsequence, (size_t)ni * 8, cudaMemcpyHostToDevice, st));
    step(cudaMemcpyAsync(of.p, offset, (size_t)ni * 8, cudaMemcpyHostToDevice, st));
    if (frames) step(cudaMemcpyAsync(fr.p, frames, (size_t)ni * 36, cudaMemcpyHostToDevice, st));
    step(launch_get_direction(t->P, t->partner.p, pd.p, dd.p, sq.p, of.p, ni, fr.p, od.p, okd.p,
                              drd.p, st));
    step(cudaMemcpyAsync(new_dirs, od.p, (size_t)ni * 12, cudaMemcpyDeviceToHost, st));
    step(cudaMemcpyAsync(ok, okd.p, (size_t)ni * 4, cudaMemcpyDeviceToHost, st));
    if (draws) step(cudaMemcpyAsync(draws, drd.p, (size_t)ni * 4, cudaMemcpyDeviceToHost, st));
    if (frames) step(cudaMemcpyAsync(frames, fr.p, (size_t)ni * 36, cudaMemcpyDeviceToHost, st));
    step(cudaStreamSynchronize(st));
    pd.release(); dd.release(); fr.release(); od.release();
    sq.release(); of.release(); okd.release(); drd.release();
    CK(e);
    return CSL_OK;
}

int csl_batch_timings(csl_tracker *t, float *ms4, int *pass2_runs) {
    if (!t) return fail(nullptr, CSL_E_INVALID, "NULL tracker");
    if (!t->ok_batch) return fail(t, CSL_E_STATE, "no completed batch");
    if (ms4)
        for (int i = 0; i < 4; i++) ms4[i] = t->ms[i];
    if (pass2_runs) *pass2_runs = t->pass2_runs;
    return CSL_OK;
}

int csl_device_count(int *n) {
    if (!n) return fail(nullptr, CSL_E_INVALID, "n must not be NULL");
    *n = 0;
    const cudaError_t e = cudaGetDeviceCount(n);
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) {
        *n = 0;
        cudaGetLastError();
        return CSL_OK;
    }
    if (e != cudaSuccess) return fail(nullptr, CSL_E_CUDA, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
    return CSL_OK;
}

int csl_dev_alloc(int device, unsigned long long bytes, void **ptr) {
    if (!ptr) return fail(nullptr, CSL_E_INVALID, "ptr must not be NULL");
    *ptr = nullptr;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(nullptr, CSL_E_CUDA, "cudaSetDevice(%d): %s", device, cudaGetErrorString(e));
    e = cudaMalloc(ptr, bytes ? bytes : 1);
    if (e != cudaSuccess) {
        *ptr = nullptr;
        return fail(nullptr, CSL_E_NOMEM, "cudaMalloc(%llu B): %s", bytes, cudaGetErrorString(e));
    }
    return CSL_OK;
}

int csl_dev_free(int device, void *ptr) {
    if (!ptr) return CSL_OK;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaFree(ptr);
    if (e != cudaSuccess) return fail(nullptr, CSL_E_CUDA, "cudaFree: %s", cudaGetErrorString(e));
    return CSL_OK;
}

int csl_dev_copy(int device, void *dst, const void *src, unsigned long long bytes, int kind) {
    if (bytes == 0) return CSL_OK;
    if (!dst || !src || kind < 1 || kind > 3) return fail(nullptr, CSL_E_INVALID, "bad copy arguments");
    const cudaMemcpyKind k = kind == 1 ? cudaMemcpyHostToDevice
                                       : (kind == 2 ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice);
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaMemcpy(dst, src, bytes, k);
    if (e != cudaSuccess) return fail(nullptr, CSL_E_CUDA, "cudaMemcpy: %s", cudaGetErrorString(e));
    return CSL_OK;
}

int csl_dev_sync(int device) {
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return fail(nullptr, CSL_E_CUDA, "cudaDeviceSynchronize: %s", cudaGetErrorString(e));
    return CSL_OK;
}

int csl_sampler_stats(csl_tracker *t, unsigned long long *out4, int reset) {
    if (!t) return fail(nullptr, CSL_E_INVALID, "NULL tracker");
    if (!t->P.env) return fail(t, CSL_E_STATE, "the tracker does not use the envelope sampler (prob_sampler=1)");
    CK(cudaSetDevice(t->device));
    if (out4) {
        CK(cudaMemcpyAsync(out4, t->env_stats.p, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                           t->own_stream));
    }
    if (reset) CK(cudaMemsetAsync(t->env_stats.p, 0, 4 * sizeof(unsigned long long), t->own_stream));
    CK(cudaStreamSynchronize(t->own_stream));
    return CSL_OK;
}

int csl_env_step(csl_tracker *t, const float *points, const int *dir_vertex, const int *dir_neg,
                 const unsigned long long *subsequence, long long n, int *out_vertex, int *out_neg) {
    if (!t) return fail(nullptr, CSL_E_INVALID, "NULL tracker");
    if (!t->P.env) return fail(t, CSL_E_STATE, "the tracker does not use the envelope sampler (prob_sampler=1)");
    if (n < 0 || n > (1LL << 30) ||
        (n > 0 && (!points || !dir_vertex || !dir_neg || !subsequence || !out_vertex || !out_neg)))
        return fail(t, CSL_E_INVALID, "bad arguments");
    for (long long i = 0; i < n; i++)
        if (dir_vertex[i] < 0 || dir_vertex[i] >= t->P.nvert || (dir_neg[i] != 0 && dir_neg[i] != 1))
            return fail(t, CSL_E_INVALID, "query %lld: direction must be +/- a sphere vertex", i);
    if (n == 0) return CSL_OK;
    CK(cudaSetDevice(t->device));
    cudaStream_t st = t->own_stream;
    const int ni = (int)n;
    DevBuf<float> pd;
    DevBuf<int> dv, dn, ov, on;
    DevBuf<unsigned long long> sq;
    cudaError_t e = cudaSuccess;
    auto step = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
    step(pd.ensure((size_t)ni * 3));
    step(dv.ensure(ni));
    step(dn.ensure(ni));
    step(ov.ensure(ni));
    step(on.ensure(ni));
    step(sq.ensure(ni));
    step(cudaMemcpyAsync(pd.p, points, (size_t)ni * 12, cudaMemcpyHostToDevice, st));
    step(cudaMemcpyAsync(dv.p, dir_vertex, (size_t)ni * 4, cudaMemcpyHostToDevice, st));
    step(cudaMemcpyAsync(dn.p, dir_neg, (size_t)ni * 4, cudaMemcpyHostToDevice, st));
    step(cudaMemcpyAsync(sq.p, subsequence, (size_t)ni * 8, cudaMemcpyHostToDevice, st));
    step(launch_env_step(t->P, pd.p, dv.p, dn.p, sq.p, ni, ov.p, on.p, st));
    step(cudaMemcpyAsync(out_vertex, ov.p, (size_t)ni * 4, cudaMemcpyDeviceToHost, st));
    step(cudaMemcpyAsync(out_neg, on.p, (size_t)ni * 4, cudaMemcpyDeviceToHost, st));
    step(cudaStreamSynchronize(st));
    pd.release(); dv.release(); dn.release(); ov.release(); on.release(); sq.release();
    CK(e);
    return CSL_OK;
}

int csl_device_constants(csl_tracker *t, float *cos_max_angle, float *cos_min_separation) {
    if (!t) return fail(nullptr, CSL_E_INVALID, "NULL tracker");
    if (cos_max_angle) *cos_max_angle = t->P.cos_max_angle;
    if (cos_min_separation) *cos_min_separation = t->P.cos_min_sep;
    return CSL_OK;
}

int csl_philox_stream(unsigned long long seed, unsigned long long subsequence,
                      unsigned long long offset, long long n, unsigned int *out) {
    csl_tracker *t = nullptr;
    if (n < 0 || (n > 0 && !out)) return fail(nullptr, CSL_E_INVALID, "bad arguments");
    if (n == 0) return CSL_OK;
    DevBuf<unsigned> d;
    CK(d.ensure(n));
    cudaError_t e = launch_philox_stream(seed, subsequence, offset, n, d.p, 0);
    if (e == cudaSuccess) e = cudaMemcpy(out, d.p, (size_t)n * 4, cudaMemcpyDeviceToHost);
    d.release();
    CK(e);
    return CSL_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Multi-subject run: the batches of many trackers (subjects) as independent
// branches of ONE captured CUDA graph, launched with one cudaGraphLaunch.
//
// Each branch is the plain batch path without its host round trips: pass 1
// (seed peaks) and its scan, pass 2 (the persistent tracking kernel) into a
// point pool and streamline slots of fixed capacity, then the device-counted
// scan and gather of multi.cu, and a four-value summary.  Branches share no
// buffer, so the GPU runs their CTAs side by side: the tail of one subject's
// persistent kernel is filled by the next subject's CTAs.  Capacities come
// from a pass-1 count at plan creation (slots) and a points-per-streamline
// estimate (pool); a subject that overflows either is re-run on the plain
// path by csl_multi_wait (exact sizes, same streamlines) and its capacities
// grow for the next capture.  Before every launch the plan compares the
// device buffers and launch shape each branch was captured with against the
// trackers' current ones and re-captures when any changed.

struct csl_multi {
    int device = 0;
    int nsub = 0;
    std::vector<csl_tracker *> sub;
    std::vector<const float *> seeds;
    std::vector<long long> n, rng_base;
    std::vector<int> sl_cap;
    std::vector<unsigned long long> pool_cap;  // points
    std::vector<std::vector<const void *>> captured;
    std::vector<DevBuf<unsigned char>> scan_tmp;
    std::vector<DevBuf<long long>> bsum;
    DevBuf<long long> summary;  // [nsub][4]: streamlines, points, status, pool points used
    long long *summary_h = nullptr;
    cudaStream_t st = nullptr, launch_st = nullptr;
    std::vector<cudaStream_t> br;
    std::vector<cudaEvent_t> join;
    cudaEvent_t fork = nullptr, ev0 = nullptr, ev1 = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaEvent_t> tracked;  // end of each branch's tracking kernel (concurrency limit)
    std::vector<int> order;            // branch order: grouped by getter, larger batches first
    int max_concurrent = 2;            // tracking kernels in flight at once (0: no limit)
    bool dirty = true, in_flight = false;
    int captures = 0;
    float ms = 0;
};

static std::vector<const void *> branch_fingerprint(const csl_tracker *u) {
    return {u->npeaks.p, u->sl_off.p, u->peaks.p, u->out_len.p, u->out_seed.p, u->out_src.p, u->pt_off.p,
            u->pool.p, u->points.p, u->scratch.p, u->queue.p, u->status.p, u->pool_count.p, u->sort_tmp.p,
            u->mkeys.p, u->mkeys_sorted.p, u->mvals.p, u->perm.p, u->blk_next.p, u->blk_end.p,
            u->bb_sl_seed.p, u->bb_sl_vert.p, u->bb_half_len.p, u->bb_half_off.p,
            (const void *)(intptr_t)u->block, (const void *)(intptr_t)u->blocks_per_sm,
            (const void *)(intptr_t)u->hp.seed_order};
}

static int branch_grid(const csl_tracker *u, long long ni) {
    const int wpb = u->block / kWarp;
    return (int)std::max<long long>(1, std::min<long long>((long long)u->nsm * u->blocks_per_sm, (ni + wpb - 1) / wpb));
}

// grow subject i's buffers to the plan's capacities (no-op when they fit)
static int multi_size(csl_multi *m, int i) {
    csl_tracker *t = nullptr;  // errors go to the library-wide message
    csl_tracker *u = m->sub[i];
    const long long ni = m->n[i];
    const int cap = m->sl_cap[i];
    const unsigned long long pc = m->pool_cap[i];
    CK(u->npeaks.ensure(ni + 1));
    CK(u->sl_off.ensure(ni + 1));
    CK(u->peaks.ensure((size_t)ni * kMaxStoredPeaksPerSeed));
    size_t tb = 0;
    CK(scan_temp_bytes((int)ni + 1, &tb));
    CK(m->scan_tmp[i].ensure(tb));
    CK(m->bsum[i].ensure(kCountedScanBlocks));
    CK(u->out_len.ensure((size_t)cap + 1));
    CK(u->out_seed.ensure((size_t)cap + 1));
    CK(u->out_src.ensure((size_t)cap + 1));
    CK(u->pt_off.ensure((size_t)cap + 1));
    CK(u->pool.ensure((size_t)pc * 3));
    CK(u->points.ensure((size_t)pc * 3 + 3));
    if (uses_batched_fit(u)) {
        CK(u->bb_sl_seed.ensure((size_t)cap + 1));
        CK(u->bb_sl_vert.ensure((size_t)cap + 1));
        CK(u->bb_half_len.ensure((size_t)2 * cap + 2));
        CK(u->bb_half_off.ensure((size_t)2 * cap + 2));
        return CSL_OK;
    }
    const int grid2 = branch_grid(u, ni);
    CK(u->scratch.ensure((size_t)grid2 * (u->block / kWarp) * scratch_floats_per_warp(u->P)));
    if (u->hp.seed_order == 1) {
        size_t sb = 0;
        CK(spatial_order(nullptr, (int)ni, grid2, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                         &sb, 0));
        CK(u->sort_tmp.ensure(sb));
        CK(u->mkeys.ensure(ni));
        CK(u->mkeys_sorted.ensure(ni));
        CK(u->mvals.ensure(ni));
        CK(u->perm.ensure(ni));
        CK(u->blk_next.ensure(grid2));
        CK(u->blk_end.ensure(grid2));
    }
    return CSL_OK;
}

// record subject i's batch on stream s (inside the capture); its tracking
// kernel starts after the event wait_for (another branch's tracking kernel)
static int multi_record(csl_multi *m, int i, cudaStream_t s, cudaEvent_t wait_for) {
    csl_tracker *t = nullptr;
    csl_tracker *u = m->sub[i];
    const DevParams &P = u->P;
    const int ni = (int)m->n[i];
    const int cap = m->sl_cap[i];
    const int wpb = u->block / kWarp;
    const int grid1 = (int)std::min<long long>(((long long)ni + wpb - 1) / wpb, (long long)u->nsm * 16);
    const int grid2 = branch_grid(u, ni);
    CK(cudaMemsetAsync(u->npeaks.p + ni, 0, sizeof(int), s));
    CK(launch_seed_peaks(P, m->seeds[i], ni, m->rng_base[i], u->partner.p, u->npeaks.p, u->peaks.p,
                         kMaxStoredPeaksPerSeed, grid1, u->block, s));
    CK(exclusive_scan_i32(m->scan_tmp[i].p, m->scan_tmp[i].cap, u->npeaks.p, u->sl_off.p, ni + 1, s));
    const int *count = u->sl_off.p + ni;
    if (uses_batched_fit(u)) {
        // the batched tensor-core fit, its streamline count read on the device
        CK(cudaMemsetAsync(u->status.p, 0, sizeof(int), s));
        CK(launch_boot_batch_prep(u->npeaks.p, u->sl_off.p, u->peaks.p, kMaxStoredPeaksPerSeed, ni, cap,
                                  u->bb_sl_seed.p, u->bb_sl_vert.p, u->status.p, s));
        BootBatchArgs A{};
        boot_args(u, A, m->seeds[i], cap, m->rng_base[i], m->pool_cap[i]);
        A.nsl_dev = count;
        CK(cudaMemsetAsync(u->bb_hq.p, 0, sizeof(int), s));
        CK(cudaMemsetAsync(u->pool_count.p, 0, sizeof(unsigned long long), s));
        if (wait_for) CK(cudaStreamWaitEvent(s, wait_for, 0));
        CK(launch_boot_batch(P, u->bgeom, A, u->partner.p, u->nsm, s));
        CK(cudaEventRecord(m->tracked[i], s));
        CK(launch_boot_batch_join(u->bb_half_len.p, u->bb_sl_seed.p, cap, count, u->out_len.p, u->out_seed.p, s));
        CK(launch_counted_scan(u->out_len.p, count, cap, m->bsum[i].p, u->pt_off.p, s));
        CK(launch_gather_halves(u->pool.p, u->bb_half_off.p, u->bb_half_len.p, u->pt_off.p, cap, count,
                                u->status.p, u->points.p, u->nsm * 8, s));
        CK(launch_batch_summary(count, cap, u->pt_off.p, u->status.p, u->pool_count.p, m->summary.p + 4 * i, s));
        return CSL_OK;
    }
    BatchArgs B{};
    B.seeds = m->seeds[i];
    B.nseeds = ni;
    B.rng_index_base = m->rng_base[i];
    B.queue = u->queue.p;
    B.pool_count = u->pool_count.p;
    B.pool = u->pool.p;
    B.pool_cap = m->pool_cap[i];
    B.scratch = u->scratch.p;
    B.status = u->status.p;
    B.sl_cap = cap;
    if (u->hp.seed_order == 1) {
        size_t sb = u->sort_tmp.cap;
        CK(spatial_order(m->seeds[i], ni, grid2, u->mkeys.p, u->mkeys_sorted.p, u->mvals.p, u->perm.p,
                         u->blk_next.p, u->blk_end.p, u->sort_tmp.p, &sb, s));
        B.perm = u->perm.p;
        B.blk_next = u->blk_next.p;
        B.blk_end = u->blk_end.p;
    }
    CK(cudaMemsetAsync(u->queue.p, 0, sizeof(int), s));
    CK(cudaMemsetAsync(u->status.p, 0, sizeof(int), s));
    CK(cudaMemsetAsync(u->pool_count.p, 0, sizeof(unsigned long long), s));
    if (wait_for) CK(cudaStreamWaitEvent(s, wait_for, 0));
    CK(launch_track(P, B, u->partner.p, u->npeaks.p, u->peaks.p, kMaxStoredPeaksPerSeed, u->sl_off.p,
                    u->out_len.p, u->out_seed.p, u->out_src.p, grid2, u->block, s));
    CK(cudaEventRecord(m->tracked[i], s));
    CK(launch_counted_scan(u->out_len.p, count, cap, m->bsum[i].p, u->pt_off.p, s));
    CK(launch_gather_counted(u->pool.p, u->out_src.p, u->out_len.p, u->pt_off.p, count, cap, u->status.p,
                             (long long)m->pool_cap[i], u->points.p, u->nsm * 8, s));
    CK(launch_batch_summary(count, cap, u->pt_off.p, u->status.p, u->pool_count.p, m->summary.p + 4 * i, s));
    return CSL_OK;
}

static int multi_capture(csl_multi *m) {
    csl_tracker *t = nullptr;
    if (m->exec) cudaGraphExecDestroy(m->exec);
    if (m->graph) cudaGraphDestroy(m->graph);
    m->exec = nullptr;
    m->graph = nullptr;
    CK(cudaStreamBeginCapture(m->st, cudaStreamCaptureModeRelaxed));
    int rc = CSL_OK;
    cudaError_t e = cudaEventRecord(m->fork, m->st);
    std::vector<int> live;  // branches in order
    for (int i : m->order)
        if (m->n[i] > 0) live.push_back(i);
    for (size_t j = 0; j < live.size() && rc == CSL_OK && e == cudaSuccess; j++) {
        const int i = live[j];
        const int k = m->max_concurrent;
        cudaEvent_t wait_for = (k > 0 && (int)j >= k) ? m->tracked[live[j - k]] : nullptr;
        e = cudaStreamWaitEvent(m->br[i], m->fork, 0);
        if (e == cudaSuccess) rc = multi_record(m, i, m->br[i], wait_for);
        if (rc == CSL_OK && e == cudaSuccess) e = cudaEventRecord(m->join[i], m->br[i]);
        if (rc == CSL_OK && e == cudaSuccess) e = cudaStreamWaitEvent(m->st, m->join[i], 0);
    }
    if (rc == CSL_OK && e == cudaSuccess)
        e = cudaMemcpyAsync(m->summary_h, m->summary.p, (size_t)m->nsub * 4 * sizeof(long long),
                            cudaMemcpyDeviceToHost, m->st);
    cudaGraph_t g = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(m->st, &g);
    if (rc != CSL_OK || e != cudaSuccess || e2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        if (rc != CSL_OK) return rc;
        CK(e != cudaSuccess ? e : e2);
    }
    m->graph = g;
    CK(cudaGraphInstantiate(&m->exec, g, 0));
    m->captures++;
    for (int i = 0; i < m->nsub; i++) m->captured[i] = branch_fingerprint(m->sub[i]);
    m->dirty = false;
    return CSL_OK;
}

static void multi_release(csl_multi *m) {
    if (m->exec) cudaGraphExecDestroy(m->exec);
    if (m->graph) cudaGraphDestroy(m->graph);
    for (auto &b : m->scan_tmp) b.release();
    for (auto &b : m->bsum) b.release();
    m->summary.release();
    if (m->summary_h) cudaFreeHost(m->summary_h);
    for (auto s : m->br)
        if (s) cudaStreamDestroy(s);
    for (auto ev : m->join)
        if (ev) cudaEventDestroy(ev);
    for (auto ev : m->tracked)
        if (ev) cudaEventDestroy(ev);
    cudaEvent_t evs[] = {m->fork, m->ev0, m->ev1};
    for (auto ev : evs)
        if (ev) cudaEventDestroy(ev);
    if (m->st) cudaStreamDestroy(m->st);
}

extern "C" {

int csl_multi_create(csl_tracker *const *subjects, const float *const *seeds_dev, const long long *n_seeds,
                     const long long *rng_index_base, int n_subjects, int points_per_streamline,
                     csl_multi **out) {
    csl_tracker *t = nullptr;
    if (!out) return fail(nullptr, CSL_E_INVALID, "NULL output");
    *out = nullptr;
    if (n_subjects < 1 || !subjects || !seeds_dev || !n_seeds)
        return fail(nullptr, CSL_E_INVALID, "csl_multi_create: need at least one subject");
    if (points_per_streamline < 0) return fail(nullptr, CSL_E_INVALID, "points_per_streamline must be >= 0");
    for (int i = 0; i < n_subjects; i++) {
        if (!subjects[i]) return fail(nullptr, CSL_E_INVALID, "subject %d is NULL", i);
        if (subjects[i]->device != subjects[0]->device)
            return fail(nullptr, CSL_E_INVALID, "all subjects must be on one device");
        if (n_seeds[i] < 0 || n_seeds[i] > (1ll << 30) || (n_seeds[i] > 0 && !seeds_dev[i]))
            return fail(nullptr, CSL_E_INVALID, "subject %d: bad seeds", i);
        for (int j = 0; j < i; j++)
            if (subjects[j] == subjects[i]) return fail(nullptr, CSL_E_INVALID, "subject %d repeats subject %d", i, j);
    }
    csl_multi *m = new csl_multi();
    m->nsub = n_subjects;
    m->device = subjects[0]->device;
    m->sub.assign(subjects, subjects + n_subjects);
    m->seeds.assign(seeds_dev, seeds_dev + n_subjects);
    m->n.assign(n_seeds, n_seeds + n_subjects);
    m->rng_base.assign(n_subjects, 0);
    if (rng_index_base)
        for (int i = 0; i < n_subjects; i++) m->rng_base[i] = rng_index_base[i];
    m->sl_cap.assign(n_subjects, 0);
    m->pool_cap.assign(n_subjects, 0);
    m->captured.resize(n_subjects);
    m->scan_tmp.resize(n_subjects);
    m->bsum.resize(n_subjects);
    m->br.assign(n_subjects, nullptr);
    m->join.assign(n_subjects, nullptr);
    m->tracked.assign(n_subjects, nullptr);
    m->max_concurrent = 2;
    m->order.resize(n_subjects);
    for (int i = 0; i < n_subjects; i++) m->order[i] = i;
    std::stable_sort(m->order.begin(), m->order.end(), [&](int a, int b) {
        if (subjects[a]->P.model != subjects[b]->P.model) return subjects[a]->P.model < subjects[b]->P.model;
        return n_seeds[a] > n_seeds[b];
    });
    auto bail = [&](int rc) {
        multi_release(m);
        delete m;
        return rc;
    };
#define MK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t _e = (call);                                                                   \
        if (_e != cudaSuccess)                                                                     \
            return bail(fail(nullptr, _e == cudaErrorMemoryAllocation ? CSL_E_NOMEM : CSL_E_CUDA, \
                             "CUDA error code=%d(%s) at %s:%d", (int)_e, cudaGetErrorName(_e),     \
                             __FILE__, __LINE__));                                                 \
    } while (0)
    MK(cudaSetDevice(m->device));
    MK(cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking));
    for (int i = 0; i < n_subjects; i++) {
        MK(cudaStreamCreateWithFlags(&m->br[i], cudaStreamNonBlocking));
        MK(cudaEventCreateWithFlags(&m->join[i], cudaEventDisableTiming));
        MK(cudaEventCreateWithFlags(&m->tracked[i], cudaEventDisableTiming));
    }
    MK(cudaEventCreateWithFlags(&m->fork, cudaEventDisableTiming));
    MK(cudaEventCreate(&m->ev0));
    MK(cudaEventCreate(&m->ev1));
    MK(m->summary.ensure((size_t)n_subjects * 4));
    MK(cudaMemset(m->summary.p, 0, (size_t)n_subjects * 4 * sizeof(long long)));
    MK(cudaMallocHost(&m->summary_h, (size_t)n_subjects * 4 * sizeof(long long)));
    // slot capacity from a pass-1 count of each subject's seeds (plus margin
    // for seeds rewritten in place before a later launch)
    const long long ppsl = points_per_streamline > 0 ? points_per_streamline : 128;
    for (int i = 0; i < n_subjects; i++) {
        csl_tracker *u = m->sub[i];
        const long long ni = m->n[i];
        long long nsl = 0;
        if (ni > 0) {
            MK(u->npeaks.ensure(ni + 1));
            MK(u->sl_off.ensure(ni + 1));
            MK(u->peaks.ensure((size_t)ni * kMaxStoredPeaksPerSeed));
            size_t tb = 0;
            MK(scan_temp_bytes((int)ni + 1, &tb));
            MK(u->scan_tmp.ensure(tb));
            const int wpb = u->block / kWarp;
            const int grid1 = (int)std::min<long long>((ni + wpb - 1) / wpb, (long long)u->nsm * 16);
            MK(cudaMemsetAsync(u->npeaks.p + ni, 0, sizeof(int), m->st));
            MK(launch_seed_peaks(u->P, m->seeds[i], (int)ni, m->rng_base[i], u->partner.p, u->npeaks.p,
                                 u->peaks.p, kMaxStoredPeaksPerSeed, grid1, u->block, m->st));
            MK(exclusive_scan_i32(u->scan_tmp.p, u->scan_tmp.cap, u->npeaks.p, u->sl_off.p, (int)ni + 1, m->st));
            int c = 0;
            MK(cudaMemcpyAsync(&c, u->sl_off.p + ni, sizeof(int), cudaMemcpyDeviceToHost, m->st));
            MK(cudaStreamSynchronize(m->st));
            nsl = c;
        }
        const long long cap = std::min<long long>(nsl + nsl / 16 + 256, (long long)INT32_MAX - 1);
        m->sl_cap[i] = (int)cap;
        m->pool_cap[i] = (unsigned long long)(cap * ppsl);
    }
#undef MK
    *out = m;
    return CSL_OK;
}

int csl_multi_launch(csl_multi *m, void *stream) {
    csl_tracker *t = nullptr;
    if (!m) return fail(nullptr, CSL_E_INVALID, "NULL plan");
    if (m->in_flight) return fail(nullptr, CSL_E_STATE, "csl_multi_launch: wait for the previous launch first");
    CK(cudaSetDevice(m->device));
    for (int i = 0; i < m->nsub; i++) {
        if (m->n[i] == 0) continue;
        const int rc = multi_size(m, i);
        if (rc != CSL_OK) return rc;
        if (m->captured[i] != branch_fingerprint(m->sub[i])) m->dirty = true;
    }
    if (m->dirty) {
        const int rc = multi_capture(m);
        if (rc != CSL_OK) return rc;
    }
    m->launch_st = stream ? (cudaStream_t)stream : m->st;
    CK(cudaEventRecord(m->ev0, m->launch_st));
    CK(cudaGraphLaunch(m->exec, m->launch_st));
    CK(cudaEventRecord(m->ev1, m->launch_st));
    m->in_flight = true;
    return CSL_OK;
}

int csl_multi_wait(csl_multi *m, long long *n_streamlines, long long *n_points, int *replayed, float *ms) {
    csl_tracker *t = nullptr;
    if (!m) return fail(nullptr, CSL_E_INVALID, "NULL plan");
    if (!m->in_flight) return fail(nullptr, CSL_E_STATE, "csl_multi_wait: nothing launched");
    CK(cudaSetDevice(m->device));
    CK(cudaStreamSynchronize(m->launch_st));
    m->in_flight = false;
    CK(cudaEventElapsedTime(&m->ms, m->ev0, m->ev1));
    if (ms) *ms = m->ms;
    for (int i = 0; i < m->nsub; i++) {
        csl_tracker *u = m->sub[i];
        const long long *S = m->summary_h + 4 * i;
        int again = 0;
        // overflowed capacities, or (batched fit) a seed with more initial
        // directions than pass 1 stores: re-run on the plain path, which sizes
        // exactly and takes the per-warp fit for such a batch as csl_propagate does
        const int rerun = ST_POOL_OVERFLOW | ST_SLOT_OVERFLOW | (uses_batched_fit(u) ? ST_PEAKS_OVERFLOW : 0);
        if (m->n[i] > 0 && (S[2] & rerun)) {
            const int rc = run_batch(u, m->seeds[i], m->n[i], m->rng_base[i], u->own_stream);
            if (rc != CSL_OK) return fail(nullptr, rc, "subject %d: %s", i, u->err.c_str());
            m->sl_cap[i] = (int)std::min<long long>(
                std::max<long long>(m->sl_cap[i], u->nsl + u->nsl / 8 + 256), (long long)INT32_MAX - 1);
            m->pool_cap[i] = std::max<unsigned long long>(m->pool_cap[i],
                                                          (unsigned long long)(u->npts + u->npts / 8 + 4096));
            m->dirty = true;
            again = 1;
        } else if (m->n[i] > 0 && S[2] != 0) {
            return fail(nullptr, CSL_E_KERNEL, "subject %d: kernel status %lld", i, S[2]);
        } else {
            u->ok_batch = 1;
            u->cmp_npts = -1;
            u->last_n = m->n[i];
            u->last_stream = m->launch_st;
            u->nsl = m->n[i] > 0 ? S[0] : 0;
            u->npts = m->n[i] > 0 ? S[1] : 0;
            u->pass2_runs = 1;
            for (float &x : u->ms) x = 0;
        }
        if (n_streamlines) n_streamlines[i] = u->nsl;
        if (n_points) n_points[i] = u->npts;
        if (replayed) replayed[i] = again;
    }
    return CSL_OK;
}

int csl_multi_set_concurrency(csl_multi *m, int max_concurrent) {
    if (!m) return fail(nullptr, CSL_E_INVALID, "NULL plan");
    if (max_concurrent < 0) return fail(nullptr, CSL_E_INVALID, "max_concurrent must be >= 0");
    if (m->in_flight) return fail(nullptr, CSL_E_STATE, "csl_multi_set_concurrency: a launch is in flight");
    if (max_concurrent != m->max_concurrent) m->dirty = true;
    m->max_concurrent = max_concurrent;
    return CSL_OK;
}

int csl_multi_info(csl_multi *m, int *captures, int *slot_caps, long long *pool_caps) {
    if (!m) return fail(nullptr, CSL_E_INVALID, "NULL plan");
    if (captures) *captures = m->captures;
    for (int i = 0; i < m->nsub; i++) {
        if (slot_caps) slot_caps[i] = m->sl_cap[i];
        if (pool_caps) pool_caps[i] = (long long)m->pool_cap[i];
    }
    return CSL_OK;
}

int csl_multi_destroy(csl_multi *m) {
    if (!m) return CSL_OK;
    cudaSetDevice(m->device);
    if (m->in_flight) cudaStreamSynchronize(m->launch_st);
    multi_release(m);
    delete m;
    return CSL_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Launch-shape tuning of the per-warp tracking path: threads per CTA of the
// pass-1 and pass-2 kernels (64, 128 or 256; CTAs per SM follow from the
// occupancy calculator) and the seed schedule (input or Morton order).
// Neither changes a streamline -- the RNG stream of a seed depends only on
// the seed's index -- so the tuner only times them.

// the tracking kernel's shared memory at this CTA size stays within the
// per-CTA limit (asked of the occupancy calculator only then)
static bool launch_fits(const csl_tracker *t, int block) {
    return smem_bytes(t->P, block / kWarp, true) <= 227 * 1024;
}

static int set_launch(csl_tracker *t, int block, int seed_order) {
    if (block != 64 && block != 128 && block != 256)
        return fail(t, CSL_E_INVALID, "threads per CTA must be 64, 128 or 256");
    if (seed_order != 0 && seed_order != 1) return fail(t, CSL_E_INVALID, "seed_order must be 0 or 1");
    if (!launch_fits(t, block))
        return fail(t, CSL_E_INVALID, "%d threads per CTA do not fit on the device", block);
    int bps = 0;
    CK(track_occupancy(t->P, block, &bps));
    if (bps < 1) return fail(t, CSL_E_INVALID, "%d threads per CTA do not fit on the device", block);
    t->block = block;
    t->blocks_per_sm = bps;
    t->hp.seed_order = seed_order;
    return CSL_OK;
}

extern "C" {

int csl_set_launch(csl_tracker *t, int threads_per_block, int seed_order) {
    if (!t) return fail(nullptr, CSL_E_INVALID, "NULL tracker");
    CK(cudaSetDevice(t->device));
    return set_launch(t, threads_per_block, seed_order);
}

int csl_get_launch(csl_tracker *t, int *threads_per_block, int *seed_order, int *blocks_per_sm) {
    if (!t) return fail(nullptr, CSL_E_INVALID, "NULL tracker");
    if (threads_per_block) *threads_per_block = t->block;
    if (seed_order) *seed_order = t->hp.seed_order;
    if (blocks_per_sm) *blocks_per_sm = t->blocks_per_sm;
    return CSL_OK;
}

int csl_autotune(csl_tracker *t, const float *seeds_dev, long long n, long long rng_index_base, int repeats,
                 float *ms_out) {
    if (!t) return fail(nullptr, CSL_E_INVALID, "NULL tracker");
    if (n < 1 || !seeds_dev) return fail(t, CSL_E_INVALID, "csl_autotune: need a seed sample");
    if (repeats < 1) return fail(t, CSL_E_INVALID, "csl_autotune: repeats must be >= 1");
    CK(cudaSetDevice(t->device));
    static const int kBlocks[3] = {256, 128, 64};
    const int block0 = t->block, order0 = t->hp.seed_order;
    float best = -1.0f;
    int best_b = block0, best_o = order0;
    for (int c = 0; c < 6; c++) {
        const int b = kBlocks[c / 2], o = c % 2;
        float total = -1.0f;
        int bps = 0;
        if (launch_fits(t, b)) CK(track_occupancy(t->P, b, &bps));
        if (bps >= 1) {
            t->block = b;
            t->blocks_per_sm = bps;
            t->hp.seed_order = o;
            int rc = run_batch(t, seeds_dev, n, rng_index_base, t->own_stream);  // warm-up, sizes buffers
            for (int r = 0; r < repeats && rc == CSL_OK; r++) {
                rc = run_batch(t, seeds_dev, n, rng_index_base, t->own_stream);
                const float ms = t->ms[0] + t->ms[1] + t->ms[2] + t->ms[3];
                if (total < 0 || ms < total) total = ms;
            }
            if (rc != CSL_OK) {
                set_launch(t, block0, order0);
                return rc;
            }
            if (best < 0 || total < best) {
                best = total;
                best_b = b;
                best_o = o;
            }
        }
        if (ms_out) ms_out[c] = total;
    }
    return set_launch(t, best_b, best_o);
}

}  // extern "C"
