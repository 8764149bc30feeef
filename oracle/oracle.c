/*
 * CPU oracle for the streamline-tracking path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference tracker (dipy/GPUStreamlines,
 * cuslines/cuda_c/*.cu), used by tests/ as the checker and by bench.py as the
 * timed CPU baseline.  The product never links, imports or calls this file.
 *
 * It follows the reference's float32 arithmetic step by step: the same
 * summation orders (fused multiply-adds where the CUDA compiler contracts),
 * the same float/double promotions of the macro constants, the same
 * comparison directions.  Values the reference computes with GPU-only fast
 * intrinsics (cos of the angle thresholds, __logf) are either passed in from
 * the device (cos) or computed with libm (log), so the bootstrap path agrees
 * to float tolerance rather than bitwise.  The hardware texture filter of the
 * stop map is emulated with 8-bit fractional weights.
 *
 * Reference routines restated (file:line within cuslines/cuda_c):
 *   Philox4x32-10 / curand_init layout    generate_streamlines_cuda.cu:445,500
 *   trilinear_interp_d                    tracking_helpers.cu:4-61
 *   check_point_d                         tracking_helpers.cu:63-73
 *   peak_directions_d                     tracking_helpers.cu:75-245
 *   warp_sort                             cuwsort.cuh:133-168
 *   max_d / min_d / prefix_sum_sh_d       utils.cu:1-120
 *   get_direction_prob_d                  generate_streamlines_cuda.cu:54-275
 *   tracker_d / genStreamlinesMergeProb_k generate_streamlines_cuda.cu:283-622
 *   get_direction_boot_d and helpers      boot.cu:20-608
 *   tracker_boot_d / genStreamlinesMergeBoot_k boot.cu:725-980
 *   get_direction_ptt_d, init_frame_ptt_d, PTT helpers  ptt.cu:1-474
 *   getNumStreamlinesPtt_k                ptt_init.cu:5-63
 * The PTT restatement emulates the tiled ODF texture (linear filter, clamp,
 * 8-bit fractional weights) and the nearest-vertex LUT (point filter,
 * normalised coordinates), and evaluates sin/cos/rsqrt in libm, so its
 * streamlines agree with the device's statistically, not bitwise.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#if defined(__x86_64__)
#include <xmmintrin.h>
#include <pmmintrin.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#define OPDT 0
#define CSA 1
#define PROB 2
#define PTT 3

typedef struct {
    int model;
    int dimx, dimy, dimz, dimt;
    int nvert, nedges, samplm_nr;
    int sphere_symm, max_sline_len;
    double step_size, max_angle, tc_threshold, relative_peak_thresh, min_separation_angle,
        pmf_threshold;
    uint64_t rng_seed;
    float cos_max_angle, cos_min_sep;
    float min_signal;
    int delta_nr;
    const float *dataf;     /* [X,Y,Z,T] */
    const float *stop_map;  /* [X,Y,Z] */
    const float *verts;     /* [V,3] */
    const int *edges;       /* [E,2] */
    const float *H, *R, *delta_b, *delta_q, *sampling;
    const int *b0s_mask;
    /* PTT */
    const float *ptt_odf;  /* tiled texture data [nz*Z][ny*Y][nx*X] */
    const float *ptt_lut;  /* nearest-vertex index [res][res][res], as float */
    int lut_res, log2_x, log2_y, tile_nx, tile_ny, tile_nz, step_frac, ptt_pad;
    float probe_step_size, probe_quality;
    double max_curvature;
    long long rng_base;     /* Philox index of seed 0 (csl_propagate's rng_index_base) */
} orc_params;

static void set_ftz(void) {
#if defined(__x86_64__)
    _MM_SET_FLUSH_ZERO_MODE(_MM_FLUSH_ZERO_ON);
    _MM_SET_DENORMALS_ZERO_MODE(_MM_DENORMALS_ZERO_ON);
#endif
}

/* ------------------------------------------------------------------ Philox */

typedef struct {
    uint32_t ctr[4], key[2], out[4];
    int idx;
} philox_t;

static void philox10(const uint32_t c_in[4], const uint32_t k_in[2], uint32_t o[4]) {
    uint32_t c0 = c_in[0], c1 = c_in[1], c2 = c_in[2], c3 = c_in[3];
    uint32_t k0 = k_in[0], k1 = k_in[1];
    for (int r = 0; r < 10; r++) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        const uint32_t n1 = (uint32_t)p1;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        const uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    o[0] = c0; o[1] = c1; o[2] = c2; o[3] = c3;
}

static void ctr_add(philox_t *g, uint64_t v) {
    const uint64_t lo = ((uint64_t)g->ctr[1] << 32) | g->ctr[0];
    const uint64_t nlo = lo + v;
    g->ctr[0] = (uint32_t)nlo;
    g->ctr[1] = (uint32_t)(nlo >> 32);
    if (nlo < lo) {
        if (++g->ctr[2] == 0) ++g->ctr[3];
    }
}

static void philox_init(philox_t *g, uint64_t seed, uint64_t subseq, uint64_t offset) {
    g->key[0] = (uint32_t)seed;
    g->key[1] = (uint32_t)(seed >> 32);
    g->ctr[0] = 0;
    g->ctr[1] = 0;
    g->ctr[2] = (uint32_t)subseq;
    g->ctr[3] = (uint32_t)(subseq >> 32);
    ctr_add(g, offset >> 2);
    philox10(g->ctr, g->key, g->out);
    g->idx = (int)(offset & 3);
}

static uint32_t philox_next(philox_t *g) {
    if (g->idx == 4) {
        ctr_add(g, 1);
        philox10(g->ctr, g->key, g->out);
        g->idx = 0;
    }
    return g->out[g->idx++];
}

static float philox_uniform(philox_t *g) {
    const float x = (float)philox_next(g);
    return fmaf(x, 2.3283064365386963e-10f, 2.3283064365386963e-10f / 2.0f);
}

void orc_philox_stream(uint64_t seed, uint64_t subseq, uint64_t offset, long long n, uint32_t *out) {
    philox_t g;
    philox_init(&g, seed, subseq, offset);
    for (long long i = 0; i < n; i++) out[i] = philox_next(&g);
}

void orc_philox_uniform(uint64_t seed, uint64_t subseq, uint64_t offset, long long n, float *out) {
    philox_t g;
    philox_init(&g, seed, subseq, offset);
    for (long long i = 0; i < n; i++) out[i] = philox_uniform(&g);
}

/* ------------------------------------------------------------ sort network */

static int g_partner[15][32];
static int g_partner_ready = 0;

/* Batcher's merge exchange (Knuth TAOCP 5.2.2 M), comparators in the
 * earliest free layer. */
static void build_partner(void) {
    if (g_partner_ready) return;
    int last[32];
    for (int i = 0; i < 32; i++) last[i] = -1;
    for (int l = 0; l < 15; l++)
        for (int i = 0; i < 32; i++) g_partner[l][i] = i;
    const int N = 32, t = 5;
    for (int p = 1 << (t - 1); p > 0; p >>= 1) {
        int q = 1 << (t - 1), r = 0, d = p;
        for (;;) {
            for (int i = 0; i < N - d; i++) {
                if ((i & p) != r) continue;
                const int a = i, b = i + d;
                int l = (last[a] > last[b] ? last[a] : last[b]) + 1;
                g_partner[l][a] = b;
                g_partner[l][b] = a;
                last[a] = last[b] = l;
            }
            if (q != p) {
                d = q - p;
                q >>= 1;
                r = p;
            } else {
                break;
            }
        }
    }
    g_partner_ready = 1;
}

void orc_sort_partners(int *out) {
    build_partner();
    memcpy(out, g_partner, sizeof(g_partner));
}

/* descending key/value sort of 32 slots, simulating the lane exchange */
static void net_sort_desc(float k[32], int v[32]) {
    build_partner();
    for (int l = 0; l < 15; l++) {
        float nk[32];
        int nv[32];
        for (int i = 0; i < 32; i++) {
            const int s = g_partner[l][i];
            const float a = k[s];
            const int b = v[s];
            nk[i] = k[i];
            nv[i] = v[i];
            if (i >= s) {
                if (a < k[i]) { nk[i] = a; nv[i] = b; }
            } else {
                if (a > k[i]) { nk[i] = a; nv[i] = b; }
            }
        }
        memcpy(k, nk, sizeof(nk));
        memcpy(v, nv, sizeof(nv));
    }
}

/* --------------------------------------------------------------- helpers */

static float fmax_ref(float a, float b) { return (a > b) ? a : b; }
static float fmin_ref(float a, float b) { return (a < b) ? a : b; }

/* warp max/min: lane-strided partials then xor butterfly (exact for max/min) */
static float arr_max(const float *x, int n) {
    float m = -FLT_MAX;
    for (int i = 0; i < n; i++) m = fmax_ref(m, x[i]);
    return m;
}

typedef struct {
    long long base[8];
    float w[8];
} corners_t;

static int trilinear_setup(const orc_params *P, const float p[3], corners_t *c) {
    const float HALF = 0.5f;
    if (p[0] != p[0] || p[1] != p[1] || p[2] != p[2]) return 0;
    if (p[0] < -HALF || p[0] + HALF >= (float)P->dimx || p[1] < -HALF ||
        p[1] + HALF >= (float)P->dimy || p[2] < -HALF || p[2] + HALF >= (float)P->dimz)
        return 0;
    const int dims[3] = {P->dimx, P->dimy, P->dimz};
    float wgh[3][2];
    long long coo[3][2];
    for (int a = 0; a < 3; a++) {
        const float fl = floorf(p[a]);
        wgh[a][1] = p[a] - fl;
        wgh[a][0] = 1.0f - wgh[a][1];
        coo[a][0] = (long long)((0 > fl) ? 0 : fl);
        coo[a][1] = ((dims[a] - 1) < coo[a][0] + 1) ? (dims[a] - 1) : coo[a][0] + 1;
    }
    const long long T = P->dimt, ZT = (long long)P->dimz * T, YZT = (long long)P->dimy * ZT;
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            for (int k = 0; k < 2; k++) {
                const int q = (i << 2) | (j << 1) | k;
                c->base[q] = coo[0][i] * YZT + coo[1][j] * ZT + coo[2][k] * T;
                c->w[q] = (wgh[0][i] * wgh[1][j]) * wgh[2][k];
            }
    return 1;
}

static void trilinear_vec(const float *data, const corners_t *c, int len, float *out) {
    for (int t = 0; t < len; t++) {
        float acc = 0.0f;
        for (int q = 0; q < 8; q++) acc = fmaf(c->w[q], data[c->base[q] + t], acc);
        out[t] = acc;
    }
}

/* Hardware linear filter of a [X,Y,Z] float volume fetched at texture
 * coordinates (u=z, v=y, w=x), unnormalised, border colour -1: sample at
 * coord - 0.5, weights quantised to 8 fractional bits. */
static float tex_stop(const orc_params *P, const float p[3]) {
    const float cz = p[2] - 0.5f, cy = p[1] - 0.5f, cx = p[0] - 0.5f;
    const float fz = floorf(cz), fy = floorf(cy), fx = floorf(cx);
    const float az = rintf((cz - fz) * 256.0f) / 256.0f;
    const float ay = rintf((cy - fy) * 256.0f) / 256.0f;
    const float ax = rintf((cx - fx) * 256.0f) / 256.0f;
    const long long iz = (long long)fz, iy = (long long)fy, ix = (long long)fx;
    float acc = 0.0f;
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            for (int k = 0; k < 2; k++) {
                const long long x = ix + i, y = iy + j, z = iz + k;
                float v = -1.0f;
                if (x >= 0 && x < P->dimx && y >= 0 && y < P->dimy && z >= 0 && z < P->dimz)
                    v = P->stop_map[(x * P->dimy + y) * P->dimz + z];
                const float w = (i ? ax : 1.0f - ax) * (j ? ay : 1.0f - ay) * (k ? az : 1.0f - az);
                acc += w * v;
            }
    return acc;
}

void orc_sample_stop(const orc_params *P, const float *pts, long long n, float *out) {
    for (long long i = 0; i < n; i++) out[i] = tex_stop(P, pts + 3 * i);
}

#define TRACKPOINT 2

static int check_point(const orc_params *P, const float p[3]) {
    const float val = tex_stop(P, p);
    if (val == -1.0f) return 0;
    return ((double)val > P->tc_threshold) ? TRACKPOINT : 3;
}

static float dot3(const float a[3], const float *b) {
    /* a.x*b.x + a.y*b.y + a.z*b.z as the CUDA compiler contracts it
     * (pinned on the GPU: tests/test_gpu_parity.py::test_dot_contraction_matches_oracle) */
    return fmaf(a[2], b[2], fmaf(a[0], b[0], a[1] * b[1]));
}

/* peak_directions_d: odf [nr] -> kept peak vertex indices in ind[0..n) */
static int peak_directions(const orc_params *P, const float *odf, int nr, int *ind) {
    for (int j = 0; j < nr; j++) ind[j] = 0;
    float mn = FLT_MAX;
    for (int i = 0; i < nr; i++) mn = fmin_ref(mn, odf[i]);
    float odf_min = (0 > mn) ? 0 : mn;
    for (int e = 0; e < P->nedges; e++) {
        const int u = P->edges[2 * e], v = P->edges[2 * e + 1];
        const float uv = odf[u], vv = odf[v];
        if (uv < vv) {
            ind[u] = -1;
            ind[v] |= 1;
        } else if (vv < uv) {
            ind[v] = -1;
            ind[u] |= 1;
        }
    }
    float mm = -FLT_MAX;
    const float neg_min = -odf_min;
    for (int i = 0; i < nr; i++)
        if (ind[i] > 0) mm = fmax_ref(mm, odf[i] + neg_min);
    const float comp_thres = (float)(P->relative_peak_thresh * (double)mm);
    int n = 0;
    for (int j = 0; j < nr; j++)
        if (ind[j] > 0 && (odf[j] - odf_min) >= comp_thres) ind[n++] = j;
    if (n < 32) {
        float k[32];
        int v[32];
        for (int l = 0; l < 32; l++) {
            k[l] = -FLT_MAX;
            v[l] = 0;
            if (l < n) {
                v[l] = ind[l];
                k[l] = odf[v[l]];
            }
        }
        net_sort_desc(k, v);
        for (int l = 0; l < n; l++) ind[l] = v[l];
    }
    if (n != 0) {
        const float cos_similarity = P->cos_min_sep;
        int k = 1;
        for (int i = 1; i < n; i++) {
            const int vi = ind[i];
            const float *abc = P->verts + 3 * vi;
            int j = 0;
            for (; j < k; j++) {
                const float *d = P->verts + 3 * ind[j];
                float cs = dot3(abc, d);
                if (P->sphere_symm) cs = fabsf(cs);
                if (cs > cos_similarity) break;
            }
            if (j == k) ind[k++] = vi;
        }
        n = k;
    }
    return n;
}

/* ------------------------------------------------------------------ prob */

static int prob_seed_peaks(const orc_params *P, const float seed[3], float *odf, int *ind) {
    corners_t c;
    if (!trilinear_setup(P, seed, &c)) return 0;
    const int len = P->samplm_nr;
    trilinear_vec(P->dataf, &c, len, odf);
    const float m = arr_max(odf, len);
    const float thr = (float)(P->pmf_threshold * (double)m);
    for (int t = 0; t < len; t++)
        if (odf[t] < thr) odf[t] = 0.0f;
    return peak_directions(P, odf, len, ind);
}

/* reference chunked scan: per 32-chunk, element 0 += previous last, then
 * Hillis-Steele with shfl_up offsets 1,2,4,8,16 */
static void scan_ref(float *x, int len) {
    for (int j = 0; j < len; j += 32) {
        if (j != 0) x[j] = x[j] + x[j - 1];
        const int n = (len - j) < 32 ? (len - j) : 32;
        float cur[32], nxt[32];
        for (int l = 0; l < 32; l++) cur[l] = l < n ? x[j + l] : 0.0f;
        for (int o = 1; o < 32; o <<= 1) {
            for (int l = 0; l < 32; l++) {
                nxt[l] = cur[l];
                if (l >= o && l < n) nxt[l] = cur[l] + cur[l - o];
            }
            memcpy(cur, nxt, sizeof(cur));
        }
        for (int l = 0; l < n; l++) x[j + l] = cur[l];
    }
}

static int prob_get_direction(const orc_params *P, const float pt[3], const float dir[3],
                              float *cdf, philox_t *g, float newdir[3], int *ndraws) {
    corners_t c;
    if (!trilinear_setup(P, pt, &c)) return 0;
    const int len = P->samplm_nr;
    trilinear_vec(P->dataf, &c, len, cdf);
    const float m = arr_max(cdf, len);
    const float thr = (float)(P->pmf_threshold * (double)m);
    const float cs = P->cos_max_angle;
    for (int i = 0; i < len; i++) {
        if (cdf[i] < thr) cdf[i] = 0.0f;
        float d = dot3(dir, P->verts + 3 * i);
        if (P->sphere_symm) d = fabsf(d);
        if (d < cs) cdf[i] = 0.0f;
    }
    scan_ref(cdf, len);
    const float last = cdf[len - 1];
    if (last == 0) return 0;
    const float sel = philox_uniform(g) * last;
    if (ndraws) (*ndraws)++;
    int low = 0, high = len - 1;
    while ((high - low) >= 32) {
        const int mid = (low + high) / 2;
        if (cdf[mid] < sel)
            low = mid;
        else
            high = mid;
    }
    int ind = -1;
    for (int l = 0; l < 32; l++)
        if (low + l <= high && sel < cdf[low + l]) {
            ind = low + l;
            break;
        }
    if (ind < 0) ind = low - 1;
    if (ind < 0) ind = 0;
    const float *sv = P->verts + 3 * ind;
    if (dot3(dir, sv) > 0) {
        newdir[0] = sv[0]; newdir[1] = sv[1]; newdir[2] = sv[2];
    } else {
        newdir[0] = -sv[0]; newdir[1] = -sv[1]; newdir[2] = -sv[2];
    }
    return 1;
}

/* ------------------------------------------------------------------ boot */

typedef struct {
    float *vox, *msk, *r, *h;
    int *ind;
} boot_ws;

/* warp-order dot product: lane-strided fma partials, then shfl_down tree */
static float warp_dot(const float *v, const float *row, int m) {
    float part[32];
    for (int l = 0; l < 32; l++) {
        float t = 0.0f;
        for (int j = l; j < m; j += 32) t = fmaf(v[j], row[j], t);
        part[l] = t;
    }
    for (int o = 16; o; o >>= 1)
        for (int l = 0; l < 32 - o; l++) part[l] = part[l] + part[l + o];
    return part[0];
}

static float warp_sum_xor(const float *x, int n, const int *mask, int *cnt_out) {
    float part[32];
    int cnt[32];
    for (int l = 0; l < 32; l++) {
        part[l] = 0.0f;
        cnt[l] = 0;
        for (int i = l; i < n; i += 32)
            if (mask[i]) {
                cnt[l]++;
                part[l] += x[i];
            }
    }
    for (int o = 16; o; o >>= 1) {
        float np[32];
        int nc[32];
        for (int l = 0; l < 32; l++) {
            np[l] = part[l] + part[l ^ o];
            nc[l] = cnt[l] + cnt[l ^ o];
        }
        memcpy(part, np, sizeof(np));
        memcpy(cnt, nc, sizeof(nc));
    }
    *cnt_out = cnt[0];
    return part[0];
}

static int boot_get_direction(const orc_params *P, philox_t *lanes, int nattempts,
                              const float dir[3], const float pt[3], boot_ws *W, float newdir[3]) {
    const int T = P->dimt, nr = P->samplm_nr;
    int hr = 0;
    for (int i = 0; i < T; i++) hr += P->b0s_mask[i] ? 0 : 1;
    for (int att = 0; att < nattempts; att++) {
        corners_t c;
        const int inb = trilinear_setup(P, pt, &c);
        if (inb) {
            trilinear_vec(P->dataf, &c, T, W->vox);
            int k = 0;
            for (int i = 0; i < T; i++)
                if (!P->b0s_mask[i]) W->msk[k++] = W->vox[i];
            for (int i = 0; i < hr; i++) W->r[i] = warp_dot(W->msk, P->R + (size_t)i * hr, hr);
            for (int i = 0; i < hr; i++) W->h[i] = warp_dot(W->msk, P->H + (size_t)i * hr, hr);
            /* lane l draws for entries l, l+32, ... in order */
            for (int j = 0; j < hr; j += 32)
                for (int l = 0; l < 32 && j + l < hr; l++) {
                    const int src = (int)(philox_next(&lanes[l]) % (uint32_t)hr);
                    W->h[j + l] = W->h[j + l] + W->r[src];
                }
            k = 0;
            for (int i = 0; i < T; i++)
                if (!P->b0s_mask[i]) W->vox[i] = W->h[k++];
            for (int i = 0; i < T; i++) W->vox[i] = (P->min_signal > W->vox[i]) ? P->min_signal : W->vox[i];
            int cnt = 0;
            const float sum = warp_sum_xor(W->vox, T, P->b0s_mask, &cnt);
            const float denom = sum / (float)cnt;
            for (int i = 0; i < T; i++) W->vox[i] = W->vox[i] / denom;
            k = 0;
            for (int i = 0; i < T; i++)
                if (!P->b0s_mask[i]) W->msk[k++] = W->vox[i];
            float tr[512];
            if (P->model == OPDT) {
                for (int j = 0; j < hr; j++) {
                    const float x = W->msk[j];
                    const float L = logf(x);
                    tr[j] = ((-L) * (1.5f + L)) * x;
                }
                for (int i = 0; i < P->delta_nr; i++)
                    W->r[i] = warp_dot(tr, P->delta_q + (size_t)i * hr, hr);
                for (int i = 0; i < P->delta_nr; i++)
                    W->h[i] = warp_dot(W->msk, P->delta_b + (size_t)i * hr, hr);
                for (int i = 0; i < P->delta_nr; i++) W->r[i] = W->r[i] - W->h[i];
            } else {
                for (int j = 0; j < hr; j++) {
                    float x = W->msk[j];
                    x = (x > 0.001f) ? x : 0.001f;
                    x = (x < 0.999f) ? x : 0.999f;
                    tr[j] = logf(-logf(x));
                }
                for (int i = 0; i < P->delta_nr; i++)
                    W->r[i] = warp_dot(tr, P->delta_q + (size_t)i * hr, hr);
                W->r[0] = 0.28209479177387814f;
            }
            for (int i = 0; i < nr; i++)
                W->h[i] = warp_dot(W->r, P->sampling + (size_t)i * P->delta_nr, P->delta_nr);
        } else {
            for (int i = 0; i < nr; i++) W->h[i] = 0;
        }
        const float m = arr_max(W->h, nr);
        const float thr = (float)(P->pmf_threshold * (double)m);
        for (int i = 0; i < nr; i++)
            if (W->h[i] < thr) W->h[i] = 0;
        const int ndir = peak_directions(P, W->h, nr, W->ind);
        if (nattempts == 1) return ndir;
        if (ndir > 0) {
            /* closest_peak_d: lane-strided |dot| max, xor butterfly, lane 0 */
            float cd[32];
            int ci[32];
            for (int l = 0; l < 32; l++) {
                cd[l] = 0;
                ci[l] = -1;
                for (int j = l; j < ndir; j += 32) {
                    const float d = dot3(dir, P->verts + 3 * W->ind[j]);
                    if (fabsf(d) > fabsf(cd[l])) {
                        cd[l] = d;
                        ci[l] = j;
                    }
                }
            }
            for (int o = 16; o; o >>= 1) {
                float nd[32];
                int ni[32];
                for (int l = 0; l < 32; l++) {
                    nd[l] = cd[l];
                    ni[l] = ci[l];
                    if (fabsf(cd[l ^ o]) > fabsf(cd[l])) {
                        nd[l] = cd[l ^ o];
                        ni[l] = ci[l ^ o];
                    }
                }
                memcpy(cd, nd, sizeof(nd));
                memcpy(ci, ni, sizeof(ni));
            }
            if (ci[0] >= 0) {
                const float *p = P->verts + 3 * W->ind[ci[0]];
                if (cd[0] >= P->cos_max_angle) {
                    newdir[0] = p[0]; newdir[1] = p[1]; newdir[2] = p[2];
                    return 1;
                }
                if (cd[0] <= -P->cos_max_angle) {
                    newdir[0] = -p[0]; newdir[1] = -p[1]; newdir[2] = -p[2];
                    return 1;
                }
            }
        }
    }
    return 0;
}

/* ------------------------------------------------------------------- PTT */

#define DISC_V 24
#define DISC_F 31
/* disc triangulation at sampling quality 2 (data from nibrary, BSD-3) */
static const float disc_vert[DISC_V * 2] = {
    -0.99680788f, -0.07983759f, -0.94276539f, 0.33345677f, -0.87928469f, -0.47629658f,
    -0.72856617f, 0.68497542f,  -0.60006556f, -0.79995082f, -0.54129995f, -0.02761342f,
    -0.39271207f, 0.37117272f,  -0.39217391f, 0.91989110f,  -0.36362884f, -0.40757367f,
    -0.22391316f, -0.97460910f, -0.00130022f, 0.53966106f,  0.00000000f,  0.00000000f,
    0.00973999f,  0.99995257f,  0.01606516f,  -0.54289908f, 0.21342395f,  -0.97695968f,
    0.38192071f,  -0.38666136f, 0.38897094f,  0.37442837f,  0.40696681f,  0.91344295f,
    0.54387161f,  -0.01477123f, 0.59119367f,  -0.80652963f, 0.73955688f,  0.67309406f,
    0.87601150f,  -0.48229022f, 0.94617928f,  0.32364298f,  0.99585368f,  -0.09096944f};
static const int disc_face[DISC_F * 3] = {
    9,  8,  4,  11, 16, 10, 5,  8,  11, 5,  1,  0,  18, 16, 11, 11, 15, 18, 13, 8,  9,
    11, 8,  13, 13, 15, 11, 22, 18, 23, 22, 20, 16, 16, 18, 22, 16, 20, 17, 12, 10, 17,
    17, 10, 16, 15, 19, 21, 23, 18, 21, 21, 18, 15, 2,  4,  8,  2,  5,  0,  8,  5,  2,
    7,  10, 12, 6,  7,  3,  10, 7,  6,  3,  1,  6,  1,  5,  6,  11, 10, 6,  6,  5,  11,
    14, 19, 15, 15, 13, 14, 14, 13, 9};
#define PTT_TRIES 1024
#define K_SMALL 0.0001f

typedef struct {
    philox_t g;
    float cached;
    int has_cached;
} pttrng_t;

static void pttrng_init(pttrng_t *r, uint64_t seed, uint64_t subseq) {
    philox_init(&r->g, seed, subseq, 0);
    r->has_cached = 0;
    r->cached = 0.0f;
}

/* Box-Muller, the sine value first and the cosine value cached */
static float pttrng_normal(pttrng_t *r) {
    if (r->has_cached) {
        r->has_cached = 0;
        return r->cached;
    }
    const float u1 = fmaf((float)philox_next(&r->g), 2.3283064365386963e-10f, 2.3283064365386963e-10f / 2.0f);
    const float u2 = fmaf((float)philox_next(&r->g), 2.3283064365386963e-10f, 2.3283064365386963e-10f / 2.0f);
    const float rr = sqrtf(-2.0f * logf(u1));
    const double a = 2.0 * M_PI * (double)u2;
    r->cached = rr * (float)cos(a);
    r->has_cached = 1;
    return rr * (float)sin(a);
}

static float ptt_texel(const orc_params *P, long long ix, long long iy, long long iz) {
    const long long W = (long long)P->tile_nx * P->dimx, H = (long long)P->tile_ny * P->dimy,
                    D = (long long)P->tile_nz * P->dimz;
    ix = ix < 0 ? 0 : (ix >= W ? W - 1 : ix);
    iy = iy < 0 ? 0 : (iy >= H ? H - 1 : iy);
    iz = iz < 0 ? 0 : (iz >= D ? D - 1 : iz);
    return P->ptt_odf[(iz * H + iy) * W + ix];
}

/* tiled ODF texture: unnormalised, clamp, linear with 8-bit fractional weights */
static float tex_odf(const orc_params *P, float x, float y, float z) {
    const float cx = x - 0.5f, cy = y - 0.5f, cz = z - 0.5f;
    const float fx = floorf(cx), fy = floorf(cy), fz = floorf(cz);
    const float ax = rintf((cx - fx) * 256.0f) / 256.0f;
    const float ay = rintf((cy - fy) * 256.0f) / 256.0f;
    const float az = rintf((cz - fz) * 256.0f) / 256.0f;
    const long long ix = (long long)fx, iy = (long long)fy, iz = (long long)fz;
    float acc = 0.0f;
    for (int k = 0; k < 2; k++)
        for (int j = 0; j < 2; j++)
            for (int i = 0; i < 2; i++) {
                const float w = (i ? ax : 1.0f - ax) * (j ? ay : 1.0f - ay) * (k ? az : 1.0f - az);
                acc += w * ptt_texel(P, ix + i, iy + j, iz + k);
            }
    return acc;
}

/* nearest-vertex LUT: normalised coordinates (u fastest), point filter, clamp */
static float tex_lut(const orc_params *P, float u, float v, float w) {
    const int n = P->lut_res;
    long long iu = (long long)floorf(u * n), iv = (long long)floorf(v * n), iw = (long long)floorf(w * n);
    iu = iu < 0 ? 0 : (iu >= n ? n - 1 : iu);
    iv = iv < 0 ? 0 : (iv >= n ? n - 1 : iv);
    iw = iw < 0 ? 0 : (iw >= n ? n - 1 : iw);
    return P->ptt_lut[(iw * n + iv) * n + iu];
}

static float interp4(const orc_params *P, const float pos[3], const float *frame) {
    const float u = fmaf(frame[0], 0.5f, 0.5f), v = fmaf(frame[1], 0.5f, 0.5f), w = fmaf(frame[2], 0.5f, 0.5f);
    const int idx = (int)tex_lut(P, w, v, u);
    const int tx = idx & (P->tile_nx - 1);
    const int ty = (idx >> P->log2_x) & (P->tile_ny - 1);
    const int tz = idx >> (P->log2_x + P->log2_y);
    return tex_odf(P, (float)(tx * P->dimx) + pos[0], (float)(ty * P->dimy) + pos[1],
                   (float)(tz * P->dimz) + pos[2]);
}

static void norm3(float *x, int fail) {
    const double n2 = (double)x[0] * x[0] + (double)x[1] * x[1] + (double)x[2] * x[2];
    const float inv = (float)(1.0 / sqrt(n2));
    if (isfinite(inv) && inv > 0.0f && inv < 1e8f) {
        x[0] *= inv; x[1] *= inv; x[2] *= inv;
    } else {
        x[0] = x[1] = x[2] = 0;
        x[fail] = 1.0f;
    }
}

static void crossnorm3(float *d, const float *a, const float *b, int fail) {
    d[0] = a[1] * b[2] - a[2] * b[1];
    d[1] = a[2] * b[0] - a[0] * b[2];
    d[2] = a[0] * b[1] - a[1] * b[0];
    norm3(d, fail);
}

static void prepare_propagator(float k1, float k2, float arclength, float *pr) {
    if (fabsf(k1) < K_SMALL && fabsf(k2) < K_SMALL) {
        pr[0] = arclength; pr[1] = 0; pr[2] = 0; pr[3] = 1; pr[4] = 0; pr[5] = 0; pr[6] = 0; pr[7] = 0; pr[8] = 1;
        return;
    }
    if (fabsf(k1) < K_SMALL) k1 = K_SMALL;
    if (fabsf(k2) < K_SMALL) k2 = K_SMALL;
    const float k = sqrtf(k1 * k1 + k2 * k2);
    const float sinkt = sinf(k * arclength), coskt = cosf(k * arclength);
    const float kk = 1 / (k * k);
    pr[0] = sinkt / k;
    pr[1] = k1 * (1 - coskt) * kk;
    pr[2] = k2 * (1 - coskt) * kk;
    pr[3] = coskt;
    pr[4] = k1 * sinkt / k;
    pr[5] = k2 * sinkt / k;
    pr[6] = -pr[5];
    pr[7] = k1 * k2 * (coskt - 1) * kk;
    pr[8] = (k1 * k1 + k2 * k2 * coskt) * kk;
}

static void random_normal(pttrng_t *r, float *pf) {
    pf[3] = pttrng_normal(r);
    pf[4] = pttrng_normal(r);
    pf[5] = pttrng_normal(r);
    const float dot = pf[3] * pf[0] + pf[4] * pf[1] + pf[5] * pf[2];
    pf[3] -= dot * pf[0];
    pf[4] -= dot * pf[1];
    pf[5] -= dot * pf[2];
    const float n2 = pf[3] * pf[3] + pf[4] * pf[4] + pf[5] * pf[5];
    if (n2 < 1e-8f) {
        const float ax = fabsf(pf[0]), ay = fabsf(pf[1]), az = fabsf(pf[2]);
        if (ax <= ay && ax <= az) { pf[3] = 0.0f; pf[4] = pf[2]; pf[5] = -pf[1]; }
        else if (ay <= az) { pf[3] = -pf[2]; pf[4] = 0.0f; pf[5] = pf[0]; }
        else { pf[3] = pf[1]; pf[4] = -pf[0]; pf[5] = 0.0f; }
    }
}

static void probing_frame(int init, const float *frame, pttrng_t *r, float *pf) {
    if (init) {
        for (int i = 0; i < 3; i++) pf[i] = frame[i];
        norm3(pf, 0);
        random_normal(r, pf);
        norm3(pf + 3, 1);
        crossnorm3(pf + 6, pf, pf + 3, 2);
    } else {
        for (int i = 0; i < 9; i++) pf[i] = frame[i];
    }
}

static void propagate_frame(const float *pr, float *frame, float *direc) {
    float tmp[3];
    for (int i = 0; i < 3; i++) {
        direc[i] = pr[0] * frame[i] + pr[1] * frame[3 + i] + pr[2] * frame[6 + i];
        tmp[i] = pr[3] * frame[i] + pr[4] * frame[3 + i] + pr[5] * frame[6 + i];
        frame[6 + i] = pr[6] * frame[i] + pr[7] * frame[3 + i] + pr[8] * frame[6 + i];
    }
    norm3(tmp, 0);
    crossnorm3(frame + 3, frame + 6, tmp, 1);
    crossnorm3(frame + 6, tmp, frame + 3, 2);
    for (int i = 0; i < 3; i++) frame[i] = tmp[i];
}

static float data_support(const orc_params *P, float support, const float pos[3], float k1, float k2, float *pf) {
    float pr[9], direc[3];
    float pp[3] = {pos[0], pos[1], pos[2]};
    prepare_propagator(k1, k2, P->probe_step_size, pr);
    for (int i = 0; i < (int)P->probe_quality; i++) {
        propagate_frame(pr, pf, direc);
        pp[0] += direc[0]; pp[1] += direc[1]; pp[2] += direc[2];
        support += interp4(P, pp, pf);
    }
    return support;
}

/* get_direction_ptt_d for one warp: lanes[32] generators, frame[9] shared */
static int ptt_get_direction(const orc_params *P, pttrng_t *lanes, int init, const float dir[3], float *frame,
                             const float pos[3], float newdir[3]) {
    if (init) { frame[0] = dir[0]; frame[1] = dir[1]; frame[2] = dir[2]; }
    const float first_val = interp4(P, pos, frame);
    const double thr = (double)P->probe_quality * P->pmf_threshold;
    float vert_pdf[DISC_V], face_cdf[32];
    int found = 0;
    for (int ii = 0; ii < DISC_V; ii++) {
        float pf[9];
        const float k1 = (float)(disc_vert[2 * ii] * P->max_curvature);
        const float k2 = (float)(disc_vert[2 * ii + 1] * P->max_curvature);
        probing_frame(init, frame, &lanes[ii], pf);
        const float sup = data_support(P, first_val, pos, k1, k2, pf);
        if ((double)sup < thr) vert_pdf[ii] = 0;
        else { vert_pdf[ii] = sup; found = 1; }
    }
    if (!found) return 0;
    for (int ii = 0; ii < DISC_F; ii++) {
        face_cdf[ii] = 0;
        for (int jj = 0; jj < 3; jj++) {
            const float v = vert_pdf[disc_face[3 * ii + jj]];
            if (v == 0) { face_cdf[ii] = 0; break; }
            face_cdf[ii] += v;
        }
    }
    scan_ref(face_cdf, DISC_F);
    const float last = face_cdf[DISC_F - 1];
    if (last == 0) return 0;
    for (int it = 0; it < PTT_TRIES / 32; it++) {
        float sup[32], k1s[32], k2s[32], pfs[32][9];
        for (int l = 0; l < 32; l++) {
            float r1 = fmaf((float)philox_next(&lanes[l].g), 2.3283064365386963e-10f, 2.3283064365386963e-10f / 2.0f);
            float r2 = fmaf((float)philox_next(&lanes[l].g), 2.3283064365386963e-10f, 2.3283064365386963e-10f / 2.0f);
            if (r1 + r2 > 1) { r1 = 1 - r1; r2 = 1 - r2; }
            const float tmp = fmaf((float)philox_next(&lanes[l].g), 2.3283064365386963e-10f,
                                   2.3283064365386963e-10f / 2.0f) * last;
            int jj;
            for (jj = 0; jj < DISC_F - 1; jj++)
                if (face_cdf[jj] >= tmp) break;
            const double mc = P->max_curvature;
            const float vx0 = (float)(mc * disc_vert[disc_face[jj * 3] * 2]);
            const float vx1 = (float)(mc * disc_vert[disc_face[jj * 3 + 1] * 2]);
            const float vx2 = (float)(mc * disc_vert[disc_face[jj * 3 + 2] * 2]);
            const float vy0 = (float)(mc * disc_vert[disc_face[jj * 3] * 2 + 1]);
            const float vy1 = (float)(mc * disc_vert[disc_face[jj * 3 + 1] * 2 + 1]);
            const float vy2 = (float)(mc * disc_vert[disc_face[jj * 3 + 2] * 2 + 1]);
            k1s[l] = vx0 + r1 * (vx1 - vx0) + r2 * (vx2 - vx0);
            k2s[l] = vy0 + r1 * (vy1 - vy0) + r2 * (vy2 - vy0);
            probing_frame(init, frame, &lanes[l], pfs[l]);
            sup[l] = data_support(P, first_val, pos, k1s[l], k2s[l], pfs[l]);
        }
        int win = -1;
        if (init) {
            float mx = sup[0];
            for (int l = 1; l < 32; l++) mx = fmaxf(mx, sup[l]);
            if ((double)mx >= thr)
                for (int l = 0; l < 32; l++)
                    if (sup[l] == mx) { win = l; break; }
        } else {
            for (int l = 0; l < 32; l++)
                if ((double)sup[l] >= thr) { win = l; break; }
        }
        if (win >= 0) {
            newdir[0] = dir[0]; newdir[1] = dir[1]; newdir[2] = dir[2];
            float *pf = pfs[win];
            if (!init) {
                float pr[9], d3[3];
                prepare_propagator(k1s[win], k2s[win], (float)(P->step_size / P->step_frac), pr);
                probing_frame(0, frame, &lanes[win], pf);
                propagate_frame(pr, pf, d3);
                norm3(d3, 0);
                newdir[0] = d3[0]; newdir[1] = d3[1]; newdir[2] = d3[2];
            }
            for (int q = 0; q < 9; q++) frame[q] = pf[q];
            return 1;
        }
    }
    return 0;
}

/* init_frame_ptt_d: frame[0..8] backward, frame[9..17] forward (forward
 * binormal = backward binormal, as the device library sets it) */
static int ptt_init_frame(const orc_params *P, pttrng_t *lanes, const float fs[3], const float seed[3],
                          float *frame) {
    float tmp[3];
    int ok = ptt_get_direction(P, lanes, 1, fs, frame, seed, tmp);
    if (!ok) {
        const float nfs[3] = {-fs[0], -fs[1], -fs[2]};
        ok = ptt_get_direction(P, lanes, 1, nfs, frame, seed, tmp);
        if (!ok) return 0;
    } else {
        for (int i = 0; i < 6; i++) frame[i] = -frame[i];
    }
    for (int i = 0; i < 6; i++) frame[9 + i] = -frame[i];
    for (int i = 6; i < 9; i++) frame[9 + i] = frame[i];
    return 1;
}

/* getNumStreamlinesPtt_k: ODF at the seed from the tiled texture */
static int ptt_seed_peaks(const orc_params *P, const float seed[3], float *odf, int *ind) {
    const int T = P->dimt;
    for (int i = 0; i < T; i++) {
        const int tx = i & (P->tile_nx - 1);
        const int ty = (i >> P->log2_x) & (P->tile_ny - 1);
        const int tz = i >> (P->log2_x + P->log2_y);
        float v = tex_odf(P, (float)(tx * P->dimx) + seed[0], (float)(ty * P->dimy) + seed[1],
                          (float)(tz * P->dimz) + seed[2]);
        if ((double)v < P->pmf_threshold) v = 0.0f;
        odf[i] = v;
    }
    return peak_directions(P, odf, T, ind);
}

/* PTT tracking of one direction with step_frac sub-steps per stored point */
static int ptt_track_one(const orc_params *P, pttrng_t *lanes, const float seed[3], const float d0[3],
                         float *frame, float *out) {
    const int sf = P->step_frac;
    const double ss = P->step_size / sf;
    float pt[3] = {seed[0], seed[1], seed[2]};
    float dir[3] = {d0[0], d0[1], d0[2]};
    out[0] = pt[0]; out[1] = pt[1]; out[2] = pt[2];
    const int imax = P->max_sline_len * sf;
    int i;
    for (i = 1; i < imax; i++) {
        float nd[3];
        if (!ptt_get_direction(P, lanes, 0, dir, frame, pt, nd)) break;
        dir[0] = nd[0]; dir[1] = nd[1]; dir[2] = nd[2];
        for (int a = 0; a < 3; a++) pt[a] = (float)fma((double)dir[a], ss, (double)pt[a]);
        if (i % sf == 0) { out[3 * (i / sf)] = pt[0]; out[3 * (i / sf) + 1] = pt[1]; out[3 * (i / sf) + 2] = pt[2]; }
        if (check_point(P, pt) != TRACKPOINT) break;
    }
    int n = i / sf;
    if ((i % sf) != 0 && i < sf * (P->max_sline_len - 1)) n++;
    return n;
}

/* --------------------------------------------------------------- tracker */

typedef struct {
    float *odf;
    int *ind;
    boot_ws bw;
    philox_t lanes[32];
} ws_t;

static void ws_alloc(ws_t *w, const orc_params *P) {
    const int n = (P->samplm_nr > P->dimt ? P->samplm_nr : P->dimt) + 64;
    w->odf = (float *)malloc(sizeof(float) * n);
    w->ind = (int *)malloc(sizeof(int) * n);
    w->bw.vox = (float *)malloc(sizeof(float) * n);
    w->bw.msk = (float *)malloc(sizeof(float) * n);
    w->bw.r = (float *)malloc(sizeof(float) * n);
    w->bw.h = (float *)malloc(sizeof(float) * n);
    w->bw.ind = w->ind;
}

static void ws_free(ws_t *w) {
    free(w->odf); free(w->ind); free(w->bw.vox); free(w->bw.msk); free(w->bw.r); free(w->bw.h);
}

static int seed_peaks(const orc_params *P, const float seed[3], long long slid, ws_t *w) {
    if (P->model == PROB) return prob_seed_peaks(P, seed, w->odf, w->ind);
    if (P->model == PTT) return ptt_seed_peaks(P, seed, w->odf, w->ind);
    for (int l = 0; l < 32; l++) philox_init(&w->lanes[l], P->rng_seed, 32ull * (slid + P->rng_base) + l, 0);
    float unused[3];
    const float zero[3] = {0, 0, 0};
    return boot_get_direction(P, w->lanes, 1, zero, seed, &w->bw, unused);
}

/* tracker_d / tracker_boot_d: points written to out[0..], returns nsteps */
static int track_one(const orc_params *P, ws_t *w, const float seed[3], const float d0[3],
                     float *out) {
    float pt[3] = {seed[0], seed[1], seed[2]};
    float dir[3] = {d0[0], d0[1], d0[2]};
    out[0] = pt[0]; out[1] = pt[1]; out[2] = pt[2];
    int i;
    for (i = 1; i < P->max_sline_len; i++) {
        float nd[3];
        int ndir;
        if (P->model == PROB)
            ndir = prob_get_direction(P, pt, dir, w->odf, &w->lanes[0], nd, NULL);
        else
            ndir = boot_get_direction(P, w->lanes, 5, dir, pt, &w->bw, nd);
        if (ndir == 0) break;
        dir[0] = nd[0]; dir[1] = nd[1]; dir[2] = nd[2];
        for (int a = 0; a < 3; a++) pt[a] = (float)fma((double)dir[a], P->step_size, (double)pt[a]);
        out[3 * i] = pt[0]; out[3 * i + 1] = pt[1]; out[3 * i + 2] = pt[2];
        if (check_point(P, pt) != TRACKPOINT) break;
    }
    return i;
}

/* Pass 1: counts[n] and up to maxp peak vertex indices per seed. */
int orc_seed_peaks(const orc_params *P, const float *seeds, long long n, int *counts, int *peaks,
                   int maxp, int nthreads) {
    set_ftz();
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
#endif
    {
        set_ftz();
        ws_t w;
        ws_alloc(&w, P);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
        for (long long s = 0; s < n; s++) {
            const int np = seed_peaks(P, seeds + 3 * s, s, &w);
            counts[s] = np;
            if (peaks)
                for (int k = 0; k < maxp; k++) peaks[s * maxp + k] = k < np ? w.ind[k] : -1;
        }
        ws_free(&w);
    }
    return 0;
}

/*
 * Pass 2 for seeds with `counts` / `peaks` from pass 1 (counts[s] <= maxp).
 * Streamline j (in seed order) gets lens[j] points at pts[j*2*max_len*3 ..]
 * (padded slots, the reference's layout).  Returns the number of streamlines.
 */
long long orc_track(const orc_params *P, const float *seeds, long long n, const int *counts,
                    const int *peaks, int maxp, int *lens, int *seed_idx, float *pts, int nthreads) {
    set_ftz();
    long long *off = (long long *)malloc(sizeof(long long) * (n + 1));
    off[0] = 0;
    for (long long s = 0; s < n; s++) off[s + 1] = off[s] + counts[s];
    const size_t slot = (size_t)2 * P->max_sline_len * 3;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
#endif
    {
        set_ftz();
        ws_t w;
        ws_alloc(&w, P);
        float *bufB = (float *)malloc(sizeof(float) * 3 * P->max_sline_len);
        float *bufF = (float *)malloc(sizeof(float) * 3 * P->max_sline_len);
        pttrng_t plane[32];
        float frame[18];
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 4)
#endif
        for (long long s = 0; s < n; s++) {
            const float *seed = seeds + 3 * s;
            for (int l = 0; l < 32; l++) philox_init(&w.lanes[l], P->rng_seed, 32ull * (s + P->rng_base) + l + 1, 0);
            if (P->model == PTT)
                for (int l = 0; l < 32; l++) pttrng_init(&plane[l], P->rng_seed, 32ull * (s + P->rng_base) + l + 1);
            for (int k = 0; k < counts[s]; k++) {
                const int pv = peaks[s * maxp + k];
                const float *fs = P->verts + 3 * pv;
                const float back[3] = {-fs[0], -fs[1], -fs[2]};
                int nB, nF;
                if (P->model == PTT) {
                    if (!ptt_init_frame(P, plane, fs, seed, frame)) {
                        bufB[0] = seed[0]; bufB[1] = seed[1]; bufB[2] = seed[2];
                        nB = 1;
                        nF = 1;
                    } else {
                        nB = ptt_track_one(P, plane, seed, back, frame, bufB);
                        nF = ptt_track_one(P, plane, seed, fs, frame + 9, bufF);
                    }
                } else {
                    nB = track_one(P, &w, seed, back, bufB);
                    nF = track_one(P, &w, seed, fs, bufF);
                }
                const long long j = off[s] + k;
                const int len = nB - 1 + nF;
                lens[j] = len;
                if (seed_idx) seed_idx[j] = (int)s;
                float *dst = pts + (size_t)j * slot;
                for (int q = 0; q < len; q++) {
                    const float *p = q < nB ? bufB + 3 * (nB - 1 - q) : bufF + 3 * (q - nB + 1);
                    dst[3 * q] = p[0]; dst[3 * q + 1] = p[1]; dst[3 * q + 2] = p[2];
                }
            }
        }
        free(bufB);
        free(bufF);
        ws_free(&w);
    }
    const long long total = off[n];
    free(off);
    return total;
}

/* One direction-getter call per query (fixed position, direction, Philox
 * subsequence/offset per lane as in the device entry point). */
int orc_get_direction(const orc_params *P, const float *pts, const float *dirs, const uint64_t *subseq,
                      const uint64_t *offs, long long n, float *new_dirs, int *ok, int *draws, float *frames) {
    set_ftz();
    ws_t w;
    ws_alloc(&w, P);
    for (long long q = 0; q < n; q++) {
        for (int l = 0; l < 32; l++) philox_init(&w.lanes[l], P->rng_seed, subseq[q] + l, offs[q]);
        int nd = 0;
        float out[3] = {dirs[3 * q], dirs[3 * q + 1], dirs[3 * q + 2]};
        int r;
        if (P->model == PTT) {
            /* PTT generators at offset 0 of each lane's subsequence; frames[9q..9q+8] in/out */
            pttrng_t pl[32];
            for (int l = 0; l < 32; l++) pttrng_init(&pl[l], P->rng_seed, subseq[q] + l);
            r = ptt_get_direction(P, pl, 0, dirs + 3 * q, frames + 9 * q, pts + 3 * q, out);
        } else if (P->model == PROB)
            r = prob_get_direction(P, pts + 3 * q, dirs + 3 * q, w.odf, &w.lanes[0], out, &nd);
        else
            r = boot_get_direction(P, w.lanes, 5, dirs + 3 * q, pts + 3 * q, &w.bw, out);
        ok[q] = r;
        if (draws) draws[q] = nd;
        new_dirs[3 * q] = out[0]; new_dirs[3 * q + 1] = out[1]; new_dirs[3 * q + 2] = out[2];
    }
    ws_free(&w);
    return 0;
}

/* Candidate contraction orders of a*b (3-term dot), for pinning dot3()
 * against the GPU: out[3q+0] = fma(az,bz, fma(ay,by, ax*bx)),
 * out[3q+1] = fma(az,bz, fma(ax,bx, ay*by)), out[3q+2] = plain float ops. */
void orc_dot3_forms(const float *a, const float *b, long long n, float *out) {
    for (long long q = 0; q < n; q++) {
        const float *u = a + 3 * q, *v = b + 3 * q;
        out[3 * q] = fmaf(u[2], v[2], fmaf(u[1], v[1], u[0] * v[0]));
        out[3 * q + 1] = fmaf(u[2], v[2], fmaf(u[0], v[0], u[1] * v[1]));
        volatile float p0 = u[0] * v[0], p1 = u[1] * v[1], p2 = u[2] * v[2];
        volatile float s = p0 + p1;
        out[3 * q + 2] = s + p2;
    }
}

/* One Philox4x32-10 block: out = philox(ctr, key) (known-answer tests). */
void orc_philox_block(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    philox10(ctr, key, out);
}
