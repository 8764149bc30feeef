/*
 * gpustreamlines_b200 -- C ABI of the B200 streamline tracker.
 *
 * The reference (dipy/GPUStreamlines, package `cuslines`) has no C ABI: its
 * Python host code JIT-compiles the kernels with NVRTC and launches them with
 * raw device pointers in a fixed argument order
 * (cuslines/cuda_python/cu_direction_getters.py:313-364, 381-414, 632-648).
 * Each entry point below names the reference interface it replaces.
 *
 * Conventions
 *  - Every function returns an int status: 0 (CSL_OK) on success, a negative
 *    CSL_E* code otherwise.  Nothing in the library calls exit().
 *  - The caller owns every host buffer; the library owns every device buffer
 *    it allocates.  One tracker handle is bound to one CUDA device.
 *  - A handle is not thread safe (the reference drives all GPUs from one host
 *    thread, cu_propagate_seeds.py:45-54).
 *  - Arrays are C-order float32 unless stated otherwise.  Seeds and points are
 *    voxel coordinates [n,3].
 */
#ifndef GPUSTREAMLINES_B200_H
#define GPUSTREAMLINES_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define CSL_OK 0
#define CSL_E_INVALID (-1)   /* bad argument or shape (ValueError in the reference) */
#define CSL_E_CUDA (-2)      /* a CUDA runtime call failed (RuntimeError in the reference) */
#define CSL_E_NOMEM (-3)     /* device allocation failed */
#define CSL_E_STATE (-4)     /* call out of order (e.g. fetch before propagate) */
#define CSL_E_KERNEL (-5)    /* a kernel reported an error status */

/* Model / direction-getter kinds (cuslines/cuda_c/globals.h:82-87). */
#define CSL_MODEL_OPDT 0
#define CSL_MODEL_CSA 1
#define CSL_MODEL_PROB 2
#define CSL_MODEL_PTT 3

typedef struct csl_tracker csl_tracker;

/*
 * Tracking parameters.  Replaces the compile-time macro set the reference
 * builds per tracker (cu_direction_getters.py:70-107, 456-468); here they are
 * runtime values, so one loaded library serves any volume.
 * Floating-point parameters are doubles holding the float32-rounded value the
 * reference passes (it stores REAL_DTYPE(x), cu_tractography.py:149-153).
 */
typedef struct csl_params {
    int model;                    /* CSL_MODEL_* */
    int dimx, dimy, dimz, dimt;   /* data volume [X,Y,Z,T] */
    int nvertices;                /* sphere vertices V (== dimt for PROB/PTT) */
    int nedges;                   /* sphere edges E */
    int samplm_nr;                /* ODF samples: rows of sampling_matrix (BOOT) or dimt */
    int sphere_symm;              /* SPHERE_SYMM */
    int max_sline_len;            /* MAX_SLINE_LEN, 501 in the reference (_globals.py:3) */
    int seed_order;               /* 0: seeds scheduled in input order; 1: scheduled in spatial
                                     (Morton) order with per-block ranges -- same results */
    double step_size;             /* STEP_SIZE, voxels */
    double max_angle;             /* MAX_ANGLE, radians */
    double tc_threshold;          /* TC_THRESHOLD */
    double relative_peak_thresh;  /* RELATIVE_PEAK_THRESH */
    double min_separation_angle;  /* MIN_SEPARATION_ANGLE, radians */
    double pmf_threshold;         /* PMF_THRESHOLD_P, 0.05 (_globals.py:4) */
    unsigned long long rng_seed;  /* RNG_SEED */
    /* bootstrap getter (BootDirectionGetter, cu_direction_getters.py:147-175) */
    double min_signal;
    int delta_nr;                 /* rows of delta_b / delta_q (SH coefficients) */
    int boot_fit;                 /* bootstrap fit: 0 = one warp per streamline in FP32 with the
                                     reference's arithmetic (results identical to it); 1 = batched
                                     fit on the tensor cores in BF16x3 with FP32 accumulation, 128
                                     streamline halves per CTA (CSA or OPDT; no counterpart in the
                                     reference, whose getter is the per-warp one, boot.cu:393-608);
                                     2 = as 1, and rows whose peak decisions lie within 8e-5 of the
                                     row maximum of flipping are fitted again in float64 before the
                                     closest peak is chosen */
    /* PTT getter (PttDirectionGetter, cu_direction_getters.py:417-468) */
    int odf_lut_res;              /* nearest-vertex LUT resolution (128) */
    int step_frac;                /* STEP_FRAC = round(step / target_short_step) */
    double probe_step_size;       /* PROBE_STEP_SIZE (probe_length) */
    double probe_quality;         /* PROBE_QUALITY */
    double max_curvature;         /* MAX_CURVATURE = 8 sin(max_angle / 2) */
    int tile_log2_x, tile_log2_y; /* PTT ODF texture tiling (LOG2_X, LOG2_Y) */
    int tile_nx, tile_ny, tile_nz;/* tiles per axis (nx, ny, nz) */
    int prob_sampler;             /* probabilistic getter's sampler: 0 = inverse CDF over the whole
                                     PMF, the reference's (get_direction_prob_d,
                                     generate_streamlines_cuda.cu:54-275; results identical to it);
                                     1 = exact rejection sampler of the same distribution with a
                                     proposal bounded by per-voxel vertex-cluster maxima (no
                                     counterpart in the reference; same distribution, different
                                     random draws, so streamlines differ individually) */
} csl_params;

/*
 * Host input arrays, uploaded once by csl_create (replaces GPUTracker._allocate
 * and the getters' allocate_on_gpu, cu_tractography.py:189-258,
 * cu_direction_getters.py:217-280, 470-517).
 */
typedef struct csl_inputs {
    const float *dataf;           /* [X,Y,Z,T]: DWI (BOOT) or PMF/ODF (PROB); NULL for PTT */
    const float *stop_map;        /* [X,Y,Z] stopping metric (e.g. FA) */
    const float *vertices;        /* [V,3] sphere vertices */
    const int *edges;             /* [E,2] sphere edges */
    /* BOOT only (NULL otherwise) */
    const float *H;               /* [hr,hr] hat matrix over the non-b0 volumes */
    const float *R;               /* [hr,hr] leveraged centred residual matrix */
    const float *delta_b;         /* [delta_nr,hr] */
    const float *delta_q;         /* [delta_nr,hr] */
    const float *sampling_matrix; /* [samplm_nr,delta_nr] */
    const int *b0s_mask;          /* [T] 1 where the volume is a b0 */
    /* PTT only (NULL otherwise) */
    const float *ptt_odf_tiled;   /* [nz*Z, ny*Y, nx*X] tiled, normalised ODF texture data (host or
                                     device memory, e.g. from csl_ptt_prepare) */
    const float *ptt_lut;         /* [res,res,res] nearest-vertex index, stored as float (host or
                                     device memory) */
} csl_inputs;

/* Create a tracker on `device`: validate, upload inputs, build textures and
 * tables.  Replaces GPUTracker.__init__/_allocate + compile_program
 * (cu_tractography.py:37-258, cu_direction_getters.py:53-144). */
int csl_create(const csl_params *params, const csl_inputs *inputs, int device,
               csl_tracker **out);

/* Release every device resource of the tracker.  Replaces GPUTracker.__exit__
 * (cu_tractography.py:260-300). */
int csl_destroy(csl_tracker *t);

/*
 * Track one batch of seeds held in HOST memory [n,3]: upload, then the fused
 * seed-peak + tracking kernel, then the device-side exclusive scans and
 * compaction.  Returns when the results are complete.  Replaces
 * SeedBatchPropagator.propagate (cu_propagate_seeds.py:206-233), i.e. pass 1
 * (getNumStreamlines*_k), the host scan (_cumsum_offsets, :95-129) and pass 2
 * (genStreamlinesMerge*_k).
 * `rng_index_base` is added to the batch-local seed index before it selects
 * the Philox subsequence; 0 reproduces the reference, whose kernels index
 * streams by the chunk-local seed id (generate_streamlines_cuda.cu:498-500).
 * `stream` is a cudaStream_t (NULL = the tracker's own stream).
 */
int csl_propagate(csl_tracker *t, const float *seeds_host, long long n,
                  long long rng_index_base, void *stream);

/* As csl_propagate, with the seeds already in device memory of the tracker's
 * device ([n,3] float32).  Results stay on the device until csl_fetch. */
int csl_propagate_device(csl_tracker *t, const float *seeds_dev, long long n,
                         long long rng_index_base, void *stream);

/* Number of streamlines and of points of the last batch.  Replaces reading
 * SeedBatchPropagator.nSlines / sline_lens (cu_propagate_seeds.py:120,235-243). */
int csl_counts(csl_tracker *t, long long *n_streamlines, long long *n_points);

/*
 * Copy the last batch's compacted results to host buffers (any may be NULL):
 *   lengths    int32 [n_streamlines]   points per streamline (slineLen)
 *   seed_index int32 [n_streamlines]   batch-local seed id (slineSeed)
 *   points     float32 [n_points,3]    streamlines back to back, in order
 * Replaces _cleanup's D2H copy of the padded nSlines x 1002 x float3 buffer
 * (cu_propagate_seeds.py:171-204); only the valid points cross PCIe.
 */
int csl_fetch(csl_tracker *t, int *lengths, int *seed_index, float *points);

/* Device pointers of the last batch's compacted results (valid until the next
 * propagate or destroy); any output may be NULL. */
int csl_device_results(csl_tracker *t, const int **lengths, const int **seed_index,
                       const long long **point_offsets, const float **points);

/*
 * Pass 1 only: number of initial directions per seed and their sphere-vertex
 * indices, as getNumStreamlines*_k computes them (boot.cu:614-718,
 * generate_streamlines_cuda.cu:427-462, ptt_init.cu:5-63).  Host buffers:
 * counts int32 [n]; peak_vertex int32 [n, max_peaks] (-1 padded, may be NULL);
 * peak_dirs float32 [n, max_peaks, 3] (may be NULL).
 */
int csl_seed_peaks(csl_tracker *t, const float *seeds_host, long long n, int max_peaks,
                   int *counts, int *peak_vertex, float *peak_dirs);

/*
 * One direction-getter call per query at a fixed position, incoming direction
 * and Philox state (subsequence, offset), as the tracking step loop makes it
 * (get_direction_prob_d / get_direction_boot_d / get_direction_ptt_d).
 * For PTT the 9-float frame per query is read from/written to `frames`.
 * Outputs: new_dirs float32 [n,3], ok int32 [n] (the getter's return value),
 * draws int32 [n] (Philox draws consumed by lane 0, may be NULL).
 */
int csl_get_direction(csl_tracker *t, const float *points, const float *dirs,
                      const unsigned long long *subsequence, const unsigned long long *offset,
                      long long n, float *frames, float *new_dirs, int *ok, int *draws);

/* Device-side durations (ms, CUDA events on the batch's stream) of the last
 * batch: [0] pass 1 + peak-count scan, [1] host sizing gap, [2] pass 2 (the
 * tracking kernel, last run), [3] length scan + compaction; pass2_runs is 1,
 * or 2 when the point pool had to grow.  The reference has no equivalent. */
int csl_batch_timings(csl_tracker *t, float *ms4, int *pass2_runs);

/* Values the kernels derive on the device: cos(max_angle) and
 * cos(min_separation_angle) as the tracker uses them. */
int csl_device_constants(csl_tracker *t, float *cos_max_angle, float *cos_min_separation);

/* Raw Philox4x32-10 stream of this library (curand_init(seed, subsequence,
 * offset) semantics): out uint32 [n]. */
int csl_philox_stream(unsigned long long seed, unsigned long long subsequence,
                      unsigned long long offset, long long n, unsigned int *out);

/*
 * Allocation-free tracking, for callers that cannot call cudaMalloc while they
 * track (device memory owned by a host framework's pool, no allocation after
 * start-up).  No counterpart in the reference.  Runs a variant of the
 * tracking kernel whose per-warp scratch is one static __device__ array of
 * 9.5 MiB in the library (held by every GPU that loads it until exit); the
 * call allocates nothing and only launches work on `stream`: results are
 * ready when the stream reaches that point.  Inputs and outputs are DEVICE
 * buffers owned by the caller:
 *   seeds_dev  float32 [n,3]
 *   counts_dev int32 [n]                      peaks per seed (all of them)
 *   lens_dev   int32 [n*max_peaks]            length of slot s*max_peaks+k
 *   points_dev float32 [n*max_peaks][2*max_sline_len][3]  slot s*max_peaks+k
 * Only the first min(counts[s], max_peaks) slots of a seed are written.  The
 * kernel always runs the per-warp paths: the FP32 bootstrap fit and the
 * inverse-CDF probabilistic sampler, so its streamlines equal csl_propagate's
 * for trackers created with boot_fit = 0 and prob_sampler = 0 (for the other
 * trackers they equal those of the same tracker created with 0 there).
 * Limits (CSL_E_INVALID beyond them):
 * 1 <= max_peaks <= 32, max_sline_len <= 501, at most 1024 sphere samples.
 * The first call on a device looks up the scratch's device address (and
 * loads the module): make it before any stream capture.  All calls share
 * the scratch, so calls that overlap on the GPU race; serialise them.
 */
int csl_track_noalloc(csl_tracker *t, const float *seeds_dev, long long n, long long rng_index_base,
                      int max_peaks, int *counts_dev, int *lens_dev, float *points_dev, void *stream);

/* Last error message of the handle (or of the library when t is NULL). */
int csl_last_error(const csl_tracker *t, char *buf, int buflen);

/* Library version string. */
/*
 * Measurement entry point (no counterpart in the reference): the ODF of one
 * bootstrap fit at each of n device points, with the bootstrap source index
 * of every non-b0 volume given (resample[n][hr], 0 <= index < hr) instead of
 * drawn, so that fits can be compared at a fixed state.  fit = 0: the
 * per-warp FP32 arithmetic of the tracking path; fit = 1: the batched
 * tensor-core BF16x3 fit (needs a tracker created with boot_fit 1 or 2).  Row i
 * of odf (stride odf_stride >= samplm_nr, a multiple of 4) receives the
 * samplm_nr ODF values; points outside the data give a zero row.
 */
int csl_boot_odf(csl_tracker *tracker, const float *points_dev, const int *resample_dev, long long n, int fit,
                 float *odf_dev, int odf_stride, void *stream);

/*
 * The batched fit's step at fixed state (measurement entry point, no
 * counterpart in the reference): as csl_boot_odf with fit = 1, plus the peak
 * search and closest-peak choice for the incoming direction dirs_dev[i]
 * (float32 [n,3]), the near-tie float64 re-evaluation included when the
 * tracker has boot_fit = 2.  step_dev[i] (float32 [n,4]) = the new direction,
 * and in .w: 1 if a peak was found, + 2 if the row was fitted again in float64.
 * csl_boot_refit_stats reads {rows searched, rows fitted again} of the batched
 * fit since creation or the last reset (reset != 0 zeroes them).
 */
int csl_boot_step(csl_tracker *tracker, const float *points_dev, const int *resample_dev, const float *dirs_dev,
                  long long n, float *odf_dev, int odf_stride, float *step_dev, void *stream);
int csl_boot_refit_stats(csl_tracker *tracker, unsigned long long *out2, int reset);

/*
 * ODF / PMF volume from SH coefficients on the tensor cores (the host step
 * before tracking in run_gpu_streamlines.py:357-380, fit.odf(sphere) clipped
 * to >= 0 for the probabilistic getter):
 *     out[x, v] = sum_c coef[x, c] * basis[v, c], clipped at 0 when clip != 0
 * coef [nvox, ncoef] f32 (ncoef <= 64), basis [nvert, ncoef] f32 (nvert <=
 * 1024), out [nvox, nvert] f32, all device memory; products in BF16x3 with
 * FP32 accumulation (~1e-5 of the row scale).  workspace: caller-owned device
 * memory of at least ceil(nvert / 256) * 256 * ceil16(ncoef) * 4 + 16 bytes.
 * *ms_out (optional) receives the kernel time.  Returns CSL_OK or CSL_E_*.
 */
int csl_odf_volume(const float *coef_dev, long long nvox, int ncoef, const float *basis_dev, int nvert, int clip,
                   float *out_dev, void *workspace_dev, long long workspace_bytes, float *ms_out, void *stream);

/*
 * Linearise the last batch's streamlines on the device (replaces the host
 * Tractogram.to_world() + DIPY compress_streamlines of generic_tracker.py:
 * 133-144): points are mapped to world coordinates with the 4x4 affine
 * (row-major doubles; NULL = identity), then compressed with tolerance
 * tol_error and segments of at most max_segment_length (world units);
 * streamlines with fewer than minlen or more than maxlen points are dropped
 * (count 0).  *npts_out receives the number of kept points.
 */
int csl_compress(csl_tracker *tracker, const double *affine16, double tol_error, double max_segment_length,
                 int minlen, int maxlen, long long *npts_out);
/* Compressed results of csl_compress: counts[n_streamlines] (0 = dropped) and
 * the kept world points [npts_out, 3], streamlines in order. */
int csl_fetch_compressed(csl_tracker *tracker, int *counts_host, float *points_host);

/*
 * Learned direction proposal (no counterpart in the reference): kernels of
 * the 48 -> 128 -> 128 -> 128 -> 40 SiLU MLP that parameterises an 8-component
 * von Mises-Fisher mixture.  All pointers are device memory, row-major FP32.
 *   csl_mlp_gemm       C[M,N] = op(A) op(B) (+ beta C), op = transpose when ta / tb
 *   csl_mlp_bias_act   Z += b per row; A = silu(Z) (act != 0) or Z
 *   csl_mlp_act_bwd    dZ = dA * silu'(Z)
 *   csl_mlp_colsum     db[n] = sum over rows of dZ[:, n]
 *   csl_mlp_vmf_nll    per-sample mixture negative log-likelihood of unit
 *                      targets X[B,3] and its gradient w.r.t. Y[B,40] (x gscale)
 *   csl_mlp_adam       Adam step (step >= 1) on n parameters
 *   csl_mlp_infer      fused inference, weights in shared memory; params in the
 *                      layout W1 b1 W2 b2 W3 b3 W4 b4 (csl_mlp_param_count floats)
 */
int csl_mlp_gemm(int ta, int tb, int M, int N, int K, const float *A, int lda, const float *B, int ldb, float *C,
                 int ldc, float beta, void *stream);
int csl_mlp_bias_act(float *Z, const float *b, float *A, int M, int N, int act, void *stream);
int csl_mlp_act_bwd(const float *Z, const float *dA, float *dZ, long long n, void *stream);
int csl_mlp_colsum(const float *dZ, int M, int N, float *db, void *stream);
int csl_mlp_vmf_nll(const float *Y, const float *X, int B, float gscale, float *loss, float *dY, void *stream);
int csl_mlp_adam(float *p, const float *g, float *m, float *v, long long n, float lr, float b1, float b2, float eps,
                 int step, void *stream);
int csl_mlp_param_count(void);
int csl_mlp_infer(const float *params, const float *X, int B, float *Y, float *ms_out, void *stream);

/*
 * The steps before tracking that run_gpu_streamlines.py:289-314 performs on
 * the host through DIPY, on the device (device pointers; bvals/bvecs host):
 *   csl_dti_fa           FA from a WLS tensor fit of dwi [nvox, T] (7 <= T <= 512),
 *                        log signals clamped at min_signal; voxels with
 *                        mask <= 0 (mask may be NULL) get 0
 *   csl_seeds_from_mask  n seeds [n, 3] uniform over the voxels of mask
 *                        [X, Y, Z] above threshold, plus U[-0.5, 0.5)^3 jitter,
 *                        from Philox streams keyed by seed; *nvox_out = voxels
 *                        in the mask.  Returns CSL_E_INVALID for an empty mask.
 */
int csl_dti_fa(const float *dwi_dev, long long nvox, int T, const double *bvals, const double *bvecs,
               const float *mask_dev, double min_signal, float *fa_dev, void *stream);
int csl_seeds_from_mask(const float *mask_dev, int X, int Y, int Z, float threshold, long long n,
                        unsigned long long seed, float *seeds_dev, long long *nvox_out, void *stream);

/*
 * Multi-subject run (no counterpart in the reference, which tracks one
 * subject per GPUTracker and per call; replaces a host loop of
 * GPUTracker.generate_streamlines / _propagate calls, cu_tractography.py:264-300).
 * A plan binds n_subjects trackers (one device, each tracker at most once)
 * to their seed batches (device float32 [n_seeds[i], 3]; pointers and counts
 * fixed for the plan's life, contents may be rewritten between launches) and
 * runs every batch as one branch of ONE captured CUDA graph: per subject,
 * pass 1, pass 2 (the tracker's own pass 2: the per-warp path, or the
 * batched tensor-core fit for a CSA / OPDT tracker with boot_fit >= 1, its
 * streamline count read on the device) and compaction into the tracker's own
 * result buffers, with no host round trip.  Streamlines are identical to
 * csl_propagate_device's for every tracker.  Slot capacity comes from a
 * pass-1 count at creation, pool capacity from points_per_streamline (0:
 * 128); a subject that overflows either (or, batched fit, has a seed with
 * more initial directions than pass 1 stores, which csl_propagate tracks on
 * the per-warp path) is re-run on the plain path inside csl_multi_wait (replayed[i] = 1)
 * and its capacities grow for the next launch, which re-captures the graph
 * (it also re-captures when a tracker's buffers or launch shape changed).
 *   csl_multi_launch  one cudaGraphLaunch on stream (NULL: the plan's own)
 *   csl_multi_wait    waits, finishes overflowed subjects; per subject
 *                     n_streamlines / n_points (arrays of n_subjects, may be
 *                     NULL); *ms = device time of the graph launch.  Results
 *                     are then read per tracker: csl_counts, csl_fetch,
 *                     csl_device_results, csl_compress.
 *   csl_multi_info    graph captures so far, slot / pool capacities
 * Destroy the plan before its trackers.  Errors: csl_last_error(NULL, ...).
 */
typedef struct csl_multi csl_multi;
int csl_multi_create(csl_tracker *const *subjects, const float *const *seeds_dev, const long long *n_seeds,
                     const long long *rng_index_base, int n_subjects, int points_per_streamline,
                     csl_multi **out);
int csl_multi_launch(csl_multi *plan, void *stream);
int csl_multi_wait(csl_multi *plan, long long *n_streamlines, long long *n_points, int *replayed, float *ms);
int csl_multi_info(csl_multi *plan, int *captures, int *slot_caps, long long *pool_caps);
/* At most max_concurrent tracking kernels in flight (0: no limit; default 2):
 * branches run grouped by getter, larger batches first, and each branch's
 * tracking kernel waits for the one max_concurrent places earlier; pass 1,
 * scans and compaction of the other branches still overlap.  Takes effect at
 * the next launch (re-capture). */
int csl_multi_set_concurrency(csl_multi *plan, int max_concurrent);
int csl_multi_destroy(csl_multi *plan);

/*
 * Launch shape of the per-warp tracking path (no counterpart in the
 * reference, which fixes 128 threads per block and one CTA grid per call,
 * cu_tractography.py:275-300).  threads_per_block 64, 128 or 256 (CTAs per SM
 * from the occupancy calculator), seed_order 0 (input order) or 1 (Morton
 * order).  Streamlines do not depend on either.
 *   csl_autotune  times the 6 shapes on a device seed sample (one warm-up
 *                 plus `repeats` batches each, best of the repeats: pass 1,
 *                 pass 2 and compaction), keeps the fastest; ms_out[6]
 *                 (optional) = the times in the order (256,0) (256,1)
 *                 (128,0) (128,1) (64,0) (64,1), -1 for a shape that does
 *                 not fit.  The tracker's last batch is then the sample's.
 */
int csl_set_launch(csl_tracker *t, int threads_per_block, int seed_order);
int csl_get_launch(csl_tracker *t, int *threads_per_block, int *seed_order, int *blocks_per_sm);
int csl_autotune(csl_tracker *t, const float *seeds_dev, long long n, long long rng_index_base, int repeats,
                 float *ms_out);

/*
 * PTT data preparation on the device (replaces the host step of
 * PttDirectionGetter.prepare_data, cu_direction_getters.py:531-625).
 *   csl_ptt_layout   power-of-two tiles (nx, ny, nz) of the texture's vertex
 *                    axis for T vertices, and log2 of nx, ny
 *   csl_ptt_prepare  DEVICE buffers: odf [X,Y,Z,T], stop map [X,Y,Z], sphere
 *                    vertices [V,3] in; out the tiled, normalised texture data
 *                    [nz*Z][ny*Y][nx*X] (ODF clipped at 0, zeroed where
 *                    stop < stop_threshold, each voxel divided by its
 *                    maximum) and the nearest-vertex LUT [res][res][res]
 *                    (index as float; grid numpy.linspace(-1, 1, res) per
 *                    axis; with sphere_symm the nearer of +-v).  Both equal
 *                    the host computation bit for bit except that exact
 *                    distance ties take the lower vertex index.  Enqueued on
 *                    `stream`.  csl_create accepts these device buffers as
 *                    csl_inputs.ptt_odf_tiled / ptt_lut directly.
 */
int csl_ptt_layout(int T, int *nx, int *ny, int *nz, int *log2_x, int *log2_y);
int csl_ptt_prepare(const float *odf_dev, const float *stop_dev, int X, int Y, int Z, int T, double stop_threshold,
                    const float *verts_dev, int V, int sphere_symm, int lut_res, float *tiled_dev, float *lut_dev,
                    void *stream);

/*
 * Device plumbing for hosts without a CUDA runtime binding of their own (the
 * reference's Python host uses cuda-python for these, cu_tractography.py:
 * 189-258 and cu_propagate_seeds.py:171-204).  Synchronous.
 *   csl_device_count  CUDA devices visible (0 without a driver or device)
 *   csl_dev_alloc     `bytes` of device memory on `device` (*ptr = NULL on error)
 *   csl_dev_free      release memory from csl_dev_alloc (NULL is a no-op)
 *   csl_dev_copy      kind 1 host -> device, 2 device -> host, 3 device -> device
 *   csl_dev_sync      wait for all work on `device`
 */
int csl_device_count(int *n);
int csl_dev_alloc(int device, unsigned long long bytes, void **ptr);
int csl_dev_free(int device, void *ptr);
int csl_dev_copy(int device, void *dst, const void *src, unsigned long long bytes, int kind);
int csl_dev_sync(int device);

/*
 * Bounded-envelope sampler of the probabilistic getter (prob_sampler = 1; no
 * counterpart in the reference, whose sampler is the inverse CDF of
 * get_direction_prob_d, generate_streamlines_cuda.cu:54-275).
 *   csl_sampler_stats  out4 = {steps sampled, proposals evaluated (4 per round),
 *                      rounds whose threshold test needed the exact maximum
 *                      (corner rows gathered), steps finished by the
 *                      inverse-CDF fallback}
 *                      accumulated over batches since creation or the last
 *                      reset (reset != 0 zeroes them after reading).
 *   csl_env_step       one direction per query with the sampler (test entry
 *                      point, like csl_get_direction): query i at points[i],
 *                      incoming direction (-1)^dir_neg[i] * vertex
 *                      dir_vertex[i]; proposals from the Philox stream
 *                      (rng_seed, 2^61 + subsequence[i]), the inverse-CDF
 *                      fallback from (rng_seed, subsequence[i], offset 0).  out_vertex[i] =
 *                      the sampled vertex or -1 when the getter stops;
 *                      out_neg[i] = 1 when the returned direction is its
 *                      negation.  Host arrays.
 */
int csl_sampler_stats(csl_tracker *t, unsigned long long *out4, int reset);
int csl_env_step(csl_tracker *t, const float *points, const int *dir_vertex, const int *dir_neg,
                 const unsigned long long *subsequence, long long n, int *out_vertex, int *out_neg);

const char *csl_version(void);

#ifdef __cplusplus
}
#endif
#endif /* GPUSTREAMLINES_B200_H */
