// Parallel-transport tractography getter (ptt.cu:1-474, ptt_init.cu:5-63).
//
// Method: Aydogan & Shi, "Parallel Transport Tractography", IEEE TMI 40(2),
// 2021.  Each lane probes one candidate curvature (k1, k2) on a triangulated
// disc: the frame is propagated PROBE_QUALITY times along the candidate arc
// and the ODF amplitude is summed (the data support).  Candidates are drawn
// from the disc-face CDF and accepted by a first-lane-above-threshold ballot.
//
// The ODF is read through a hardware-filtered 3D texture in the reference's
// tiled layout (vertex t of voxel (x,y,z) at texel (tx*X+x, ty*Y+y, tz*Z+z))
// and a point-sampled nearest-vertex LUT texture, so the filtered values are
// the reference's own.  Normal variates use the Box-Muller transform (Box &
// Muller 1958) on two Philox words, the second value cached for the next
// call; the GPU tests compare them with the toolkit generator's normals
// within a stated tolerance.
//
// Deliberate difference: after the initial frame search the reference copies
// only the tangent and normal into the forward half of the frame
// (ptt.cu:464-468), leaving the forward binormal at whatever the shared slot
// held before.  Here the forward binormal is the backward binormal, which is
// the parallel-transported binormal the comment there describes.
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

constexpr int kTriesPerRejection = 1024;
constexpr float kKSmall = 0.0001f;
constexpr float kNormEps = 1e-8f;
constexpr float kInvNormEps = 1e8f;

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
        // Box-Muller pair r sin(2 pi U2), r cos(2 pi U2) with r = sqrt(-2 ln U1); the
        // sine value is returned first (the order the toolkit generator's
        // streams show, pinned by the GPU tests)
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

template <int FAIL_IND>
__device__ __forceinline__ void norm3(float *num) {
    const float inv_scale = rnorm3df(num[0], num[1], num[2]);
    if (isfinite(inv_scale) && inv_scale > 0.0f && inv_scale < kInvNormEps) {
        num[0] *= inv_scale;
        num[1] *= inv_scale;
        num[2] *= inv_scale;
    } else {
        num[0] = num[1] = num[2] = 0;
        num[FAIL_IND] = 1.0;
    }
}

template <int FAIL_IND>
__device__ __forceinline__ void crossnorm3(float *dest, const float *src1, const float *src2) {
    dest[0] = src1[1] * src2[2] - src1[2] * src2[1];
    dest[1] = src1[2] * src2[0] - src1[0] * src2[2];
    dest[2] = src1[0] * src2[1] - src1[1] * src2[0];
    norm3<FAIL_IND>(dest);
}

__device__ __forceinline__ float interp4(const DevParams &P, const float3 pos, const float *frame) {
    const float3 uvw = {fmaf(frame[0], 0.5f, 0.5f), fmaf(frame[1], 0.5f, 0.5f),
                        fmaf(frame[2], 0.5f, 0.5f)};
    const int odf_idx = static_cast<int>(tex3D<float>(P.lut_tex, uvw.z, uvw.y, uvw.x));
    const int tx = odf_idx & P.width_mask;
    const int ty = (odf_idx >> P.log2_x) & P.height_mask;
    const int tz = (odf_idx >> (P.log2_x + P.log2_y));
    const float x_query = (float)(tx * P.dimx) + pos.x;
    const float y_query = (float)(ty * P.dimy) + pos.y;
    const float z_query = (float)(tz * P.dimz) + pos.z;
    return tex3D<float>(P.odf_tex, x_query, y_query, z_query);
}

__device__ __forceinline__ void prepare_propagator(float k1, float k2, float arclength,
                                                   float *propagator) {
    if ((fabsf(k1) < kKSmall) && (fabsf(k2) < kKSmall)) {
        propagator[0] = arclength;
        propagator[1] = 0;
        propagator[2] = 0;
        propagator[3] = 1;
        propagator[4] = 0;
        propagator[5] = 0;
        propagator[6] = 0;
        propagator[7] = 0;
        propagator[8] = 1;
    } else {
        if (fabsf(k1) < kKSmall) k1 = kKSmall;
        if (fabsf(k2) < kKSmall) k2 = kKSmall;
        const float k = sqrtf(k1 * k1 + k2 * k2);
        const float sinkt = __sinf(k * arclength);
        const float coskt = __cosf(k * arclength);
        const float kk = 1 / (k * k);
        propagator[0] = sinkt / k;
        propagator[1] = k1 * (1 - coskt) * kk;
        propagator[2] = k2 * (1 - coskt) * kk;
        propagator[3] = coskt;
        propagator[4] = k1 * sinkt / k;
        propagator[5] = k2 * sinkt / k;
        propagator[6] = -propagator[5];
        propagator[7] = k1 * k2 * (coskt - 1) * kk;
        propagator[8] = (k1 * k1 + k2 * k2 * coskt) * kk;
    }
}

__device__ __forceinline__ void random_normal(PhiloxN &st, float *probing_frame) {
    probing_frame[3] = st.normal();
    probing_frame[4] = st.normal();
    probing_frame[5] = st.normal();
    float dot = probing_frame[3] * probing_frame[0] + probing_frame[4] * probing_frame[1] +
                probing_frame[5] * probing_frame[2];
    probing_frame[3] -= dot * probing_frame[0];
    probing_frame[4] -= dot * probing_frame[1];
    probing_frame[5] -= dot * probing_frame[2];
    float n2 = probing_frame[3] * probing_frame[3] + probing_frame[4] * probing_frame[4] +
               probing_frame[5] * probing_frame[5];
    if (n2 < kNormEps) {
        float abs_x = fabsf(probing_frame[0]);
        float abs_y = fabsf(probing_frame[1]);
        float abs_z = fabsf(probing_frame[2]);
        if (abs_x <= abs_y && abs_x <= abs_z) {
            probing_frame[3] = 0.0;
            probing_frame[4] = probing_frame[2];
            probing_frame[5] = -probing_frame[1];
        } else if (abs_y <= abs_z) {
            probing_frame[3] = -probing_frame[2];
            probing_frame[4] = 0.0;
            probing_frame[5] = probing_frame[0];
        } else {
            probing_frame[3] = probing_frame[1];
            probing_frame[4] = -probing_frame[0];
            probing_frame[5] = 0.0;
        }
    }
}

template <bool IS_INIT>
__device__ __forceinline__ void get_probing_frame(const float *frame, PhiloxN &st,
                                                  float *probing_frame) {
    if (IS_INIT) {
        for (int ii = 0; ii < 3; ii++) probing_frame[ii] = frame[ii];
        norm3<0>(probing_frame);
        random_normal(st, probing_frame);
        norm3<1>(probing_frame + 3);
        crossnorm3<2>(probing_frame + 2 * 3, probing_frame, probing_frame + 3);
    } else {
        for (int ii = 0; ii < 9; ii++) probing_frame[ii] = frame[ii];
    }
}

__device__ __forceinline__ void propagate_frame(const float *propagator, float *frame,
                                                float *direc) {
    float tmp[3];
    for (int ii = 0; ii < 3; ii++) {
        direc[ii] = propagator[0] * frame[ii] + propagator[1] * frame[3 + ii] +
                    propagator[2] * frame[6 + ii];
        tmp[ii] = propagator[3] * frame[ii] + propagator[4] * frame[3 + ii] +
                  propagator[5] * frame[6 + ii];
        frame[2 * 3 + ii] = propagator[6] * frame[ii] + propagator[7] * frame[3 + ii] +
                            propagator[8] * frame[6 + ii];
    }
    norm3<0>(tmp);
    crossnorm3<1>(frame + 3, frame + 2 * 3, tmp);
    crossnorm3<2>(frame + 2 * 3, tmp, frame + 3);
    for (int ii = 0; ii < 3; ii++) frame[ii] = tmp[ii];
}

__device__ __forceinline__ float calculate_data_support(const DevParams &P, float support,
                                                        const float3 pos, float k1, float k2,
                                                        float *probing_frame) {
    float probing_prop[9];
    float direc[3];
    float3 probing_pos;
    prepare_propagator(k1, k2, P.probe_step_size, probing_prop);
    probing_pos = pos;
    for (int ii = 0; ii < P.probe_quality; ii++) {
        propagate_frame(probing_prop, probing_frame, direc);
        probing_pos.x += direc[0];
        probing_pos.y += direc[1];
        probing_pos.z += direc[2];
        const float fod_amp = interp4(P, probing_pos, probing_frame);
        support += fod_amp;
    }
    return support;
}

struct PttSmem {
    float *face_cdf;  // [kDiscFaceCnt]
    float *vert_pdf;  // [kDiscVertCnt]
};

// get_direction_ptt_d (ptt.cu:194-412).  `frame_sh` (9 floats, shared) is the
// warp's frame; the winning lane rewrites it.
template <bool IS_INIT>
__device__ int ptt_get_direction(const DevParams &P, PhiloxN &st, float3 dir, float *frame_sh,
                                 float3 pos, const PttSmem &S, int lane, float3 *newdir) {
    __syncwarp();
    if (IS_INIT) {
        if (lane == 0) {
            frame_sh[0] = dir.x;
            frame_sh[1] = dir.y;
            frame_sh[2] = dir.z;
        }
    }
    __syncwarp();
    const float first_val = interp4(P, pos, frame_sh);
    __syncwarp();

    float probing_frame[9];
    float k1_probe = 0.f, k2_probe = 0.f;
    bool support_found = 0;
    for (int ii = lane; ii < kDiscVertCnt; ii += kWarp) {
        k1_probe = (float)(c_disc_vert[ii * 2] * P.max_curvature);
        k2_probe = (float)(c_disc_vert[ii * 2 + 1] * P.max_curvature);
        get_probing_frame<IS_INIT>(frame_sh, st, probing_frame);
        const float this_support =
            calculate_data_support(P, first_val, pos, k1_probe, k2_probe, probing_frame);
        if ((double)this_support < P.probe_quality * P.pmf_threshold) {
            S.vert_pdf[ii] = 0;
        } else {
            S.vert_pdf[ii] = this_support;
            support_found = 1;
        }
    }
    if (__ballot_sync(FULL, support_found) == 0) return 0;

    for (int ii = lane; ii < kDiscFaceCnt; ii += kWarp) S.face_cdf[ii] = 0;
    __syncwarp();
    for (int ii = lane; ii < kDiscFaceCnt; ii += kWarp) {
        for (int jj = 0; jj < 3; jj++) {
            const float vert_val = S.vert_pdf[c_disc_face[ii * 3 + jj]];
            if (vert_val == 0) {
                S.face_cdf[ii] = 0;
                break;
            }
            S.face_cdf[ii] += vert_val;
        }
    }
    __syncwarp();
    scan_smem_ref(S.face_cdf, kDiscFaceCnt, lane);
    const float last_cdf = S.face_cdf[kDiscFaceCnt - 1];
    if (last_cdf == 0) return 0;

    for (int ii = 0; ii < kTriesPerRejection / kWarp; ii++) {
        float r1 = st.uniform();
        float r2 = st.uniform();
        if (r1 + r2 > 1) {
            r1 = 1 - r1;
            r2 = 1 - r2;
        }
        const float tmp = st.uniform() * last_cdf;
        int jj;
        for (jj = 0; jj < kDiscFaceCnt - 1; jj++)
            if (S.face_cdf[jj] >= tmp) break;
        const double mc = P.max_curvature;
        const float vx0 = (float)(mc * c_disc_vert[c_disc_face[jj * 3] * 2]);
        const float vx1 = (float)(mc * c_disc_vert[c_disc_face[jj * 3 + 1] * 2]);
        const float vx2 = (float)(mc * c_disc_vert[c_disc_face[jj * 3 + 2] * 2]);
        const float vy0 = (float)(mc * c_disc_vert[c_disc_face[jj * 3] * 2 + 1]);
        const float vy1 = (float)(mc * c_disc_vert[c_disc_face[jj * 3 + 1] * 2 + 1]);
        const float vy2 = (float)(mc * c_disc_vert[c_disc_face[jj * 3 + 2] * 2 + 1]);
        k1_probe = vx0 + r1 * (vx1 - vx0) + r2 * (vx2 - vx0);
        k2_probe = vy0 + r1 * (vy1 - vy0) + r2 * (vy2 - vy0);
        get_probing_frame<IS_INIT>(frame_sh, st, probing_frame);
        const float this_support =
            calculate_data_support(P, first_val, pos, k1_probe, k2_probe, probing_frame);
        __syncwarp();
        int winning_lane = -1;
        if (IS_INIT) {
            float tmp_support = this_support;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
                tmp_support = fmaxf(tmp_support, __shfl_down_sync(FULL, tmp_support, o));
            const float max_support = __shfl_sync(FULL, tmp_support, 0);
            const unsigned msk = __ballot_sync(
                FULL, (this_support == max_support) &&
                          ((double)max_support >= P.probe_quality * P.pmf_threshold));
            if (msk != 0) winning_lane = __ffs(msk) - 1;
        } else {
            const unsigned msk = __ballot_sync(
                FULL, (double)this_support >= P.probe_quality * P.pmf_threshold);
            if (msk != 0) winning_lane = __ffs(msk) - 1;
        }
        if (winning_lane != -1) {
            float3 nd = dir;
            if (lane == winning_lane) {
                if (!IS_INIT) {
                    float prop[9];
                    float d3[3];
                    prepare_propagator(k1_probe, k2_probe, (float)(P.step_size / P.step_frac), prop);
                    get_probing_frame<false>(frame_sh, st, probing_frame);
                    propagate_frame(prop, probing_frame, d3);
                    norm3<0>(d3);
                    nd = make_float3(d3[0], d3[1], d3[2]);
                }
                for (int q = 0; q < 9; q++) frame_sh[q] = probing_frame[q];
            }
            nd.x = __shfl_sync(FULL, nd.x, winning_lane);
            nd.y = __shfl_sync(FULL, nd.y, winning_lane);
            nd.z = __shfl_sync(FULL, nd.z, winning_lane);
            __syncwarp();
            *newdir = nd;
            return 1;
        }
    }
    return 0;
}

// init_frame_ptt_d (ptt.cu:415-474): frame[0..8] backward, frame[9..17] forward
__device__ __forceinline__ bool ptt_init_frame(const DevParams &P, PhiloxN &st, float3 first_step, float3 seed,
                               float *frame, const PttSmem &S, int lane) {
    float3 tmp;
    bool ok = ptt_get_direction<true>(P, st, first_step, frame, seed, S, lane, &tmp);
    __syncwarp();
    if (!ok) {
        ok = ptt_get_direction<true>(P, st,
                                     make_float3(-first_step.x, -first_step.y, -first_step.z),
                                     frame, seed, S, lane, &tmp);
        __syncwarp();
        if (!ok) return false;
    } else {
        if (lane == 0)
            for (int ii = 0; ii < 6; ii++) frame[ii] = -frame[ii];
        __syncwarp();
    }
    if (lane == 0) {
        for (int ii = 0; ii < 6; ii++) frame[9 + ii] = -frame[ii];
        for (int ii = 6; ii < 9; ii++) frame[9 + ii] = frame[ii];
    }
    __syncwarp();
    return true;
}

// Pass-1 peaks at a seed (getNumStreamlinesPtt_k, ptt_init.cu:5-63)
__device__ __forceinline__ int ptt_seed_peaks(const DevParams &P, float3 point, float *odf_sh,
                                              int *ind_sh, const int *partner_sh, int lane) {
    const int T = P.dimt;
    for (int i = lane; i < T; i += kWarp) {
        const int tx = i & P.width_mask;
        const int ty = (i >> P.log2_x) & P.height_mask;
        const int tz = (i >> (P.log2_x + P.log2_y));
        const float xq = (float)(tx * P.dimx) + point.x;
        const float yq = (float)(ty * P.dimy) + point.y;
        const float zq = (float)(tz * P.dimz) + point.z;
        float v = tex3D<float>(P.odf_tex, xq, yq, zq);
        if ((double)v < P.pmf_threshold) v = 0.0f;
        odf_sh[i] = v;
    }
    __syncwarp();
    return peak_directions(P, odf_sh, ind_sh, T, partner_sh, lane);
}

}  // namespace csl
