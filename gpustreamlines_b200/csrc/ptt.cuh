// Parallel-transport tractography (PTT) direction getter.
//
// Method: D. B. Aydogan and Y. Shi, "Parallel Transport Tractography", IEEE
// TMI 40(2):635-647, 2021.  A streamline carries an orthonormal frame
// (tangent T, normal N, binormal B).  A candidate continuation is an arc of
// constant curvature kappa = |(k1, k2)| bending in the normal-plane direction
// u = (k1 N + k2 B) / kappa; its data support is the ODF amplitude at the
// current point along T plus the amplitudes at Q probe points along the arc
// (each read along the arc's local tangent).  The sampling scheme is the one
// the reference's get_direction_ptt_d applies (cuslines/cuda_c/ptt.cu:194-412,
// ptt_init.cu:5-63), kept so that the output distribution is the reference's:
//   1. supports of the 24 curvature-disc vertices (k = disc vertex * max
//      curvature), zeroed below Q * PMF_THRESHOLD_P;
//   2. face weights (sum of the three vertex supports, zero if any is zero)
//      and their cumulative distribution over the 31 disc faces;
//   3. rounds of 32 candidates drawn uniformly inside faces picked from that
//      distribution; the first candidate (in lane order) whose support clears
//      the threshold wins and the frame moves one step along its arc.  The
//      initial-frame search draws a random normal per candidate and keeps the
//      largest support.
//
// Design for the B200:
//   * the frame is read from shared memory into each candidate's registers
//     (probe frames are private to a lane); only the winner writes it back;
//   * an arc is applied as a rotation of the frame in the (T, u) plane by
//     theta = kappa * s:  T' = cos T + sin u,  N' = N - (k1/kappa) e,
//     B' = B - (k2/kappa) e  with e = sin T + (1 - cos) u, and the chord
//     d = (sin/kappa) T + ((1 - cos)/kappa) u; probe frames are not
//     re-orthonormalised (8 rotations drift by ~1e-7), the kept frame is;
//   * a candidate's Q probe points and tangents are computed first, then its Q
//     nearest-vertex lookups are issued together, then its Q ODF fetches:
//     two texture latencies per candidate instead of 2 Q dependent ones;
//   * the face CDF is built with warp shuffles (vertex supports gathered by
//     face, Hillis-Steele scan in registers) and searched by bisection.
//
// Textures (the reference's layout, cu_direction_getters.py:531-625): the ODF
// is hardware-filtered from a 3D texture whose vertex axis is tiled over
// (tx, ty, tz) power-of-two tiles -- vertex t of voxel (x, y, z) sits at texel
// (tx X + x, ty Y + y, tz Z + z) -- and directions map to vertices through a
// point-sampled 128^3 nearest-vertex LUT addressed by (T + 1) / 2.
//
// Normal variates: Box-Muller (Box & Muller 1958) on two Philox words, the
// sine value first and the cosine value cached for the next draw (the order
// the toolkit generator's normals show, pinned by the GPU tests).
//
// Deliberate difference: after the initial-frame search the forward frame
// gets the kept binormal too; the reference copies only T and N there
// (ptt.cu:464-468) and leaves the forward binormal at a stale value.
#pragma once
#include "common.cuh"

namespace csl {

// Disc triangulation at sampling quality 2: 24 vertices, 31 faces.  The
// numbers must equal the reference's table for the face CDF and the curvature
// samples to agree.  Data from nibrary (src/math/disc.h), BSD 3-Clause,
// Copyright (c) 2024, Dogu Baran Aydogan.
constexpr int kDiscVertCnt = 24;
constexpr int kDiscFaceCnt = 31;
__constant__ float c_disc_vert[kDiscVertCnt * 2] = {
    -0.99680788f, -0.07983759f, -0.94276539f, 0.33345677f, -0.87928469f, -0.47629658f,
    -0.72856617f, 0.68497542f,  -0.60006556f, -0.79995082f, -0.54129995f, -0.02761342f,
    -0.39271207f, 0.37117272f,  -0.39217391f, 0.91989110f,  -0.36362884f, -0.40757367f,
    -0.22391316f, -0.97460910f, -0.00130022f, 0.53966106f,  0.00000000f,  0.00000000f,
    0.00973999f,  0.99995257f,  0.01606516f,  -0.54289908f, 0.21342395f,  -0.97695968f,
    0.38192071f,  -0.38666136f, 0.38897094f,  0.37442837f,  0.40696681f,  0.91344295f,
    0.54387161f,  -0.01477123f, 0.59119367f,  -0.80652963f, 0.73955688f,  0.67309406f,
    0.87601150f,  -0.48229022f, 0.94617928f,  0.32364298f,  0.99585368f,  -0.09096944f};
__constant__ int c_disc_face[kDiscFaceCnt * 3] = {
    9,  8,  4,  11, 16, 10, 5,  8,  11, 5,  1,  0,  18, 16, 11, 11, 15, 18, 13, 8,  9,
    11, 8,  13, 13, 15, 11, 22, 18, 23, 22, 20, 16, 16, 18, 22, 16, 20, 17, 12, 10, 17,
    17, 10, 16, 15, 19, 21, 23, 18, 21, 21, 18, 15, 2,  4,  8,  2,  5,  0,  8,  5,  2,
    7,  10, 12, 6,  7,  3,  10, 7,  6,  3,  1,  6,  1,  5,  6,  11, 10, 6,  6,  5,  11,
    14, 19, 15, 15, 13, 14, 14, 13, 9};

constexpr int kPttRounds = 1024 / kWarp;  // 1024 candidates at most per direction
#ifndef CSL_PTT_WAVE
#define CSL_PTT_WAVE 2
#endif
constexpr int kProbeWave = CSL_PTT_WAVE;  // probe points whose fetches are issued together
constexpr int kPttFirst = 1;              // candidates probed before the rest of a round
constexpr float kCurvMin = 1e-4f;         // |k1|, |k2| below this count as straight / are raised to it
constexpr float kTinyNorm2 = 1e-8f;

// Philox with a cached second Box-Muller value (per lane).
struct PhiloxN {
    Philox g;
    float cached;
    int has_cached;
    __device__ __forceinline__ void init(uint64_t seed, uint64_t subseq, uint64_t offset) {
        g.init(seed, subseq, offset);
        has_cached = 0;
        cached = 0.0f;
    }
    __device__ __forceinline__ float uniform() { return g.uniform(); }
    __device__ __forceinline__ float normal() {
        if (has_cached) {
            has_cached = 0;
            return cached;
        }
        const float u1 = Philox::uint_to_uniform(g.next());
        const float u2 = Philox::uint_to_uniform(g.next());
        const float r = sqrtf(-2.0f * logf(u1));
        float sn, cs;
        sincospif(2.0f * u2, &sn, &cs);
        cached = r * cs;
        has_cached = 1;
        return r * sn;
    }
};

struct Frame3 {
    float3 t, n, b;
};

__device__ __forceinline__ float3 f3_axpy(float a, float3 x, float3 y) {
    return make_float3(fmaf(a, x.x, y.x), fmaf(a, x.y, y.y), fmaf(a, x.z, y.z));
}
// Products and sums are spelled out as fused or separately rounded operations
// so that every kernel that inlines this getter rounds identically (implicit
// contraction may differ with the surrounding code, and a PTT streamline
// amplifies a last-bit difference into another path).
__device__ __forceinline__ float f3_dot(float3 a, float3 b) {
    return fmaf(a.z, b.z, fmaf(a.y, b.y, __fmul_rn(a.x, b.x)));
}
__device__ __forceinline__ float f3_cross_c(float p, float q, float r, float s) {
    return fmaf(p, q, -__fmul_rn(r, s));  // p q - r s
}
__device__ __forceinline__ float3 f3_cross(float3 a, float3 b) {
    return make_float3(f3_cross_c(a.y, b.z, a.z, b.y), f3_cross_c(a.z, b.x, a.x, b.z), f3_cross_c(a.x, b.y, a.y, b.x));
}
__device__ __forceinline__ float3 f3_scale(float a, float3 x) { return make_float3(a * x.x, a * x.y, a * x.z); }

// Unit vector along v; a degenerate v (zero, huge or not finite) becomes the
// unit axis `axis` (a measure-zero event along a streamline).
__device__ __forceinline__ float3 unit_or_axis(float3 v, int axis) {
    const float r = rnorm3df(v.x, v.y, v.z);
    if (isfinite(r) && r > 0.0f && r < 1e8f) return f3_scale(r, v);
    return make_float3(axis == 0 ? 1.0f : 0.0f, axis == 1 ? 1.0f : 0.0f, axis == 2 ? 1.0f : 0.0f);
}

// Re-orthonormalise a transported frame (tangent first, then the binormal,
// the normal closes the right-handed triad T x N = B).
__device__ __forceinline__ void frame_fix(Frame3 &F) {
    F.t = unit_or_axis(F.t, 0);
    F.b = unit_or_axis(f3_axpy(-f3_dot(F.b, F.t), F.t, F.b), 2);
    F.n = unit_or_axis(f3_cross(F.b, F.t), 1);
}

// A circular arc of curvature (k1, k2) and length s, as a frame rotation.
struct Arc {
    bool straight;
    float c, s;     // cos, sin of kappa * len
    float kn, kb;   // k1 / kappa, k2 / kappa
    float dt, du;   // chord = dt T + du u
};

__device__ __forceinline__ Arc make_arc(float k1, float k2, float len) {
    Arc a;
    a.straight = fabsf(k1) < kCurvMin && fabsf(k2) < kCurvMin;
    if (a.straight) {
        a.c = 1.0f;
        a.s = a.kn = a.kb = a.du = 0.0f;
        a.dt = len;
        return a;
    }
    if (fabsf(k1) < kCurvMin) k1 = kCurvMin;
    if (fabsf(k2) < kCurvMin) k2 = kCurvMin;
    const float kap = sqrtf(fmaf(k1, k1, __fmul_rn(k2, k2)));
    const float inv = 1.0f / kap;
    __sincosf(kap * len, &a.s, &a.c);
    a.kn = k1 * inv;
    a.kb = k2 * inv;
    a.dt = a.s * inv;
    a.du = (1.0f - a.c) * inv;
    return a;
}

// Move frame F along the arc; returns the chord (displacement).
__device__ __forceinline__ float3 arc_move(const Arc &a, Frame3 &F) {
    if (a.straight) return f3_scale(a.dt, F.t);
    const float3 u = f3_axpy(a.kn, F.n, f3_scale(a.kb, F.b));
    const float3 d = f3_axpy(a.dt, F.t, f3_scale(a.du, u));
    const float3 e = f3_axpy(a.s, F.t, f3_scale(1.0f - a.c, u));
    F.t = f3_axpy(a.c, F.t, f3_scale(a.s, u));
    F.n = f3_axpy(-a.kn, e, F.n);
    F.b = f3_axpy(-a.kb, e, F.b);
    return d;
}

// LUT texel of a tangent, and the tiled ODF texel of a vertex at a position
__device__ __forceinline__ float lut_vertex(const DevParams &P, float3 t) {
    return tex3D<float>(P.lut_tex, fmaf(t.z, 0.5f, 0.5f), fmaf(t.y, 0.5f, 0.5f), fmaf(t.x, 0.5f, 0.5f));
}
__device__ __forceinline__ float odf_at(const DevParams &P, int v, float3 p) {
    const int tx = v & P.width_mask;
    const int ty = (v >> P.log2_x) & P.height_mask;
    const int tz = v >> (P.log2_x + P.log2_y);
    return tex3D<float>(P.odf_tex, (float)(tx * P.dimx) + p.x, (float)(ty * P.dimy) + p.y,
                        (float)(tz * P.dimz) + p.z);
}

// Support of one candidate: `base` (the amplitude at the current point) plus
// the amplitudes at the probe points of the arc.  F ends as the frame at the
// last probe point.
__device__ __forceinline__ float arc_support(const DevParams &P, float3 pos, Frame3 &F, const Arc &a, float base,
                                             int nprobe) {
    float sup = base;
    for (int w0 = 0; w0 < nprobe; w0 += kProbeWave) {
        float3 pt[kProbeWave];
        float val[kProbeWave];
#pragma unroll
        for (int i = 0; i < kProbeWave; i++) {
            if (w0 + i < nprobe) {
                const float3 d = arc_move(a, F);
                pos = make_float3(pos.x + d.x, pos.y + d.y, pos.z + d.z);
                pt[i] = pos;
                val[i] = lut_vertex(P, F.t);
            }
        }
#pragma unroll
        for (int i = 0; i < kProbeWave; i++)
            if (w0 + i < nprobe) val[i] = odf_at(P, (int)val[i], pt[i]);
#pragma unroll
        for (int i = 0; i < kProbeWave; i++)
            if (w0 + i < nprobe) sup += val[i];
    }
    return sup;
}

// Random frame around tangent t for the initial search: a normal drawn from
// three Gaussian variates with the tangent component removed.
__device__ __forceinline__ Frame3 random_frame(float3 t, PhiloxN &rng) {
    Frame3 F;
    F.t = unit_or_axis(t, 0);
    float3 g;
    g.x = rng.normal();
    g.y = rng.normal();
    g.z = rng.normal();
    g = f3_axpy(-f3_dot(g, F.t), F.t, g);
    if (f3_dot(g, g) < kTinyNorm2) {
        // any vector orthogonal to t: drop t's smallest component
        const float ax = fabsf(F.t.x), ay = fabsf(F.t.y), az = fabsf(F.t.z);
        if (ax <= ay && ax <= az)
            g = make_float3(0.0f, F.t.z, -F.t.y);
        else if (ay <= az)
            g = make_float3(-F.t.z, 0.0f, F.t.x);
        else
            g = make_float3(F.t.y, -F.t.x, 0.0f);
    }
    F.n = unit_or_axis(g, 1);
    F.b = unit_or_axis(f3_cross(F.t, F.n), 2);
    return F;
}

__device__ __forceinline__ Frame3 load_frame(const float *f) {
    Frame3 F;
    F.t = make_float3(f[0], f[1], f[2]);
    F.n = make_float3(f[3], f[4], f[5]);
    F.b = make_float3(f[6], f[7], f[8]);
    return F;
}
__device__ __forceinline__ void store_frame(float *f, const Frame3 &F) {
    f[0] = F.t.x; f[1] = F.t.y; f[2] = F.t.z;
    f[3] = F.n.x; f[4] = F.n.y; f[5] = F.n.z;
    f[6] = F.b.x; f[7] = F.b.y; f[8] = F.b.z;
}

// Curvature of disc vertex i (the reference scales the float table by the
// double MAX_CURVATURE and rounds to float)
__device__ __forceinline__ float2 disc_curv(const DevParams &P, int i) {
    return make_float2((float)(P.max_curvature * (double)c_disc_vert[2 * i]),
                       (float)(P.max_curvature * (double)c_disc_vert[2 * i + 1]));
}

// One PTT direction.  `frame_sh` (9 floats, shared) is the streamline's frame;
// for INIT it receives the kept candidate's frame.  `cdf_sh` is 32 floats of
// per-warp scratch.  Returns 0 when no candidate has enough support.
template <bool INIT>
__device__ int ptt_step_direction(const DevParams &P, PhiloxN &rng, float3 dir, float *frame_sh, float3 pos,
                                  float *cdf_sh, int lane, float3 *newdir) {
    // The frame stays in shared memory and is re-read where needed, which
    // keeps the candidate loop's registers to one frame and one probe wave.
    __syncwarp();
    if (INIT) {
        if (lane == 0) {
            frame_sh[0] = dir.x;
            frame_sh[1] = dir.y;
            frame_sh[2] = dir.z;
        }
        __syncwarp();
    }
    const int nprobe = (int)P.probe_quality;
    const double thr = (double)P.probe_quality * P.pmf_threshold;
    const float3 t0 = make_float3(frame_sh[0], frame_sh[1], frame_sh[2]);
    const float base = odf_at(P, (int)lut_vertex(P, t0), pos);

    // 1. supports of the disc vertices, one per lane
    float wv = 0.0f;
    if (lane < kDiscVertCnt) {
        const float2 k = disc_curv(P, lane);
        Frame3 G = INIT ? random_frame(t0, rng) : load_frame(frame_sh);
        const float s = arc_support(P, pos, G, make_arc(k.x, k.y, P.probe_step_size), base, nprobe);
        wv = ((double)s < thr) ? 0.0f : s;
    }
    if (__ballot_sync(FULL, wv != 0.0f) == 0u) return 0;

    // 2. face weights and their cumulative distribution, lane f = face f
    const int fi = lane < kDiscFaceCnt ? lane : 0;
    const float a = __shfl_sync(FULL, wv, c_disc_face[3 * fi]);
    const float b = __shfl_sync(FULL, wv, c_disc_face[3 * fi + 1]);
    const float c = __shfl_sync(FULL, wv, c_disc_face[3 * fi + 2]);
    float cdf = (lane < kDiscFaceCnt && a != 0.0f && b != 0.0f && c != 0.0f) ? (a + b) + c : 0.0f;
#pragma unroll
    for (int i = 1; i < kWarp; i <<= 1) {
        const float y = __shfl_up_sync(FULL, cdf, i);
        if (lane >= i) cdf += y;
    }
    const float total = __shfl_sync(FULL, cdf, kDiscFaceCnt - 1);
    if (total == 0.0f) return 0;
    cdf_sh[lane] = cdf;
    __syncwarp();

    // 3. rounds of 32 candidates
    for (int round = 0; round < kPttRounds; round++) {
        float r1 = rng.uniform();
        float r2 = rng.uniform();
        if (r1 + r2 > 1.0f) {
            r1 = 1.0f - r1;
            r2 = 1.0f - r2;
        }
        const float x = rng.uniform() * total;
        // first face whose cumulative weight reaches x (the last face if none)
        int lo = 0, hi = kDiscFaceCnt - 1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (cdf_sh[mid] >= x)
                hi = mid;
            else
                lo = mid + 1;
        }
        const float2 k0 = disc_curv(P, c_disc_face[3 * lo]);
        const float2 k1 = disc_curv(P, c_disc_face[3 * lo + 1]);
        const float2 k2 = disc_curv(P, c_disc_face[3 * lo + 2]);
        const float kx = fmaf(r2, k2.x - k0.x, fmaf(r1, k1.x - k0.x, k0.x));
        const float ky = fmaf(r2, k2.y - k0.y, fmaf(r1, k1.y - k0.y, k0.y));
        Frame3 G = INIT ? random_frame(t0, rng) : load_frame(frame_sh);
        const Arc arc = make_arc(kx, ky, P.probe_step_size);
        unsigned won;
        if (INIT) {
            const float s = arc_support(P, pos, G, arc, base, nprobe);
            const float best = warp_max_ref(s);
            won = __ballot_sync(FULL, s == best && (double)best >= thr);
        } else {
            // the lowest lane whose candidate has enough support wins: candidates
            // 0..kPttFirst-1 are probed first, the others only when none of those
            // passes (every lane has drawn its numbers, so the result and the
            // streams are those of probing all 32 at once)
            won = 0u;
            for (int pass = 0; pass < 2 && won == 0u; pass++) {
                const bool mine = (lane < kPttFirst) == (pass == 0);
                float s = 0.0f;
                if (mine) s = arc_support(P, pos, G, arc, base, nprobe);
                won = __ballot_sync(FULL, mine && (double)s >= thr);
            }
        }
        if (won == 0u) continue;
        const int src = __ffs(won) - 1;
        float3 nd = dir;
        __syncwarp();
        if (lane == src) {
            if (INIT) {
                frame_fix(G);
                store_frame(frame_sh, G);  // the candidate's frame at its last probe point
            } else {
                Frame3 H = load_frame(frame_sh);
                const float3 d = arc_move(make_arc(kx, ky, (float)(P.step_size / P.step_frac)), H);
                frame_fix(H);
                store_frame(frame_sh, H);
                nd = unit_or_axis(d, 0);
            }
        }
        nd.x = __shfl_sync(FULL, nd.x, src);
        nd.y = __shfl_sync(FULL, nd.y, src);
        nd.z = __shfl_sync(FULL, nd.z, src);
        __syncwarp();
        *newdir = nd;
        return 1;
    }
    return 0;
}

// Initial frames of one streamline (ptt_init.cu / init_frame_ptt_d semantics):
// search with the pass-1 direction, else with its opposite; frame[0..8] is the
// backward frame, frame[9..17] the forward one (T and N reversed).
__device__ __forceinline__ bool ptt_start_frames(const DevParams &P, PhiloxN &rng, float3 first, float3 seed,
                                                 float *frame, float *cdf_sh, int lane) {
    float3 unused;
    const bool fwd_ok = ptt_step_direction<true>(P, rng, first, frame, seed, cdf_sh, lane, &unused);
    __syncwarp();
    if (!fwd_ok) {
        const float3 back = make_float3(-first.x, -first.y, -first.z);
        if (!ptt_step_direction<true>(P, rng, back, frame, seed, cdf_sh, lane, &unused)) return false;
        __syncwarp();
    }
    if (lane < 9) {
        // found along `first`: the backward frame is the reversed one
        const float v = frame[lane];
        const float bw = (fwd_ok && lane < 6) ? -v : v;
        frame[lane] = bw;
        frame[9 + lane] = (lane < 6) ? -bw : bw;
    }
    __syncwarp();
    return true;
}

// Pass 1 at a seed: ODF amplitude of every vertex from the texture,
// thresholded, then the peak search.
__device__ __forceinline__ int ptt_seed_odf_peaks(const DevParams &P, float3 seed, float *odf_sh, int *ind_sh,
                                                  const int *partner_sh, int lane) {
    for (int v = lane; v < P.dimt; v += kWarp) {
        const float x = odf_at(P, v, seed);
        odf_sh[v] = ((double)x < P.pmf_threshold) ? 0.0f : x;
    }
    __syncwarp();
    return peak_directions(P, odf_sh, ind_sh, P.dimt, partner_sh, lane);
}

}  // namespace csl
