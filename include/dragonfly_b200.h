/* dragonfly_b200: one EMC iteration (expand -> maximize -> compress) of
 * duaneloh/Dragonfly on an NVIDIA B200 (sm_100a), behind a plain C ABI.
 *
 * A context owns one GPU's copies of the detector, the sparse photon frames,
 * the orientation list, the model and the per-frame parameters, plus all work
 * buffers. Arguments are plain host pointers and sizes in the reference's own
 * layouts; nothing in this header needs CUDA or torch types.
 *
 * Every function returns DFG_OK (0) or an error code; dfg_last_error() gives a
 * readable message. A context is not re-entrant: calls on one context must not
 * overlap (the reference's maximize() has the same rule, recon.pyx:99).
 *
 * Library: dragonfly_b200/libdfgpu.so. Python binding: dragonfly_b200/_lib.py.
 */
#ifndef DRAGONFLY_B200_H
#define DRAGONFLY_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define DFG_API __attribute__((visibility("default")))
#else
#define DFG_API
#endif

#define DFG_OK 0
#define DFG_ERR_ARG 1      /* invalid argument (message says which) */
#define DFG_ERR_CUDA 2     /* a CUDA call failed */
#define DFG_ERR_STATE 3    /* required input not set yet */
#define DFG_ERR_NOMEM 4    /* device allocation failed */

typedef struct dfg_ctx dfg_ctx;

/* Per-call parameters of one iteration. Mirrors the struct params fields that
 * maximize() and EMCRecon.update_beta read (dragonfly/src/params.h:6-34). */
typedef struct dfg_iter_params {
	int iteration;     /* params.iteration, 1-based */
	int need_scaling;  /* per-frame scale factors phi_d in the likelihood */
	int update_scale;  /* update phi_d = fcounts_d / psum_d after the M-step */
	int known_scale;   /* use phi_d in the likelihood from iteration 1 */
	double beta_jump;  /* beta schedule: beta_d = min(1, beta_start_d * */
	int beta_period;   /*   beta_jump^((iteration-1)/beta_period) * beta_factor) */
	double beta_factor;
} dfg_iter_params;

/* ---- lifetime -------------------------------------------------------------
 * Replaces EMCRecon.__init__ / free (dragonfly/recon.pyx:37-46, 176-180). */
DFG_API int dfg_create(int device, dfg_ctx **out);
DFG_API void dfg_destroy(dfg_ctx *ctx);
DFG_API const char *dfg_last_error(const dfg_ctx *ctx);
/* Version string of the library. */
DFG_API const char *dfg_version(void);

/* ---- inputs ---------------------------------------------------------------
 * Detector: qvals [num_pix][3] (voxel units), corr [num_pix], raw_mask
 * [num_pix] (0 good, 1 merge only, 2 bad). Replaces CDetector.parse / setters
 * (dragonfly/detector.pyx:31-74, 161-206) and struct detector
 * (dragonfly/src/detector.h:6-16). */
DFG_API int dfg_set_detector(dfg_ctx *ctx, int num_pix, const double *qvals, const double *corr,
                     const uint8_t *raw_mask);

/* Sparse photon frames in the .emc layout: ones[num_data], multi[num_data],
 * place_ones[sum ones], place_multi[sum multi], count_multi[sum multi]
 * (dragonfly/src/emcfile.h:12-32, parse_binarydataset emcfile.c:3-57). Also
 * computes fcounts, sum_fact and mean_count (calc_frame_counts and
 * calc_sum_fact, dragonfly/src/iterate.c:3-117; ln c! as lgamma(c + 1)),
 * resets the blacklist to all-good and phi_d to 1. Replaces Iterate.set_data
 * (dragonfly/iterate.pyx:241-266). */
DFG_API int dfg_set_frames(dfg_ctx *ctx, int num_data, const int *ones, const int *multi,
                   const int *place_ones, const int *place_multi, const int *count_multi);

/* Orientations quats [num_rot][5] = (q0, q1, q2, q3, weight). Replaces
 * Iterate.set_quat (dragonfly/iterate.pyx:268-274), struct quaternion
 * (dragonfly/src/quaternion.h:11-15). */
DFG_API int dfg_set_quaternions(dfg_ctx *ctx, int num_rot, const double *quats);

/* Model model1 [num_modes][size][size][size] (C order), centre size / 2;
 * [num_modes][size][size] for 2-D and RZ models (dfg_set_model_type).
 * Replaces Iterate.set_model / Model.allocate (dragonfly/iterate.pyx:184-190,
 * dragonfly/model.pyx:43-103). */
DFG_API int dfg_set_model(dfg_ctx *ctx, long size, int num_modes, const double *model1);

/* Model type, as struct model's mtype (model.h:13-17) and params.rtype:
 * 0 = 3-D volume (quaternion orientations; the default), 1 = stack of 2-D
 * images (orientation = the in-plane angle quats[r][0]; slice_gen2d /
 * slice_merge2d, model.c:65-99, 254-290), 2 = RZ image (orientation =
 * (phi, beta); slice_genrz / slice_mergerz, model.c:106-150, 299-340; the one-
 * slice operations only, as the reference's run_iteration selects no RZ slice
 * functions, recon.pyx:86-91). friedel_sym: update_model applies the 2-D
 * Friedel average (symmetrize_friedel2d, model.c:495-515) to 2-D models
 * (params.friedel_sym, recon.pyx:118-119); RZ models always get it. Changing
 * the type clears the model: call dfg_set_model afterwards. */
DFG_API int dfg_set_model_type(dfg_ctx *ctx, int model_type, int friedel_sym);

/* Detector distance in pixels (struct detector's detd, detector.h:15), used by
 * the RZ geometry. */
DFG_API int dfg_set_detector_distance(dfg_ctx *ctx, double detd);

/* Per-frame arrays (num_data entries). Replace the Iterate.scale setter,
 * parse_blacklist and calc_beta (dragonfly/iterate.pyx:284-402;
 * dragonfly/src/iterate.c:66-83). dfg_calc_beta: start > 0 sets every
 * beta_start_d = start; start <= 0 selects the reference's empirical rule. */
DFG_API int dfg_set_scale(dfg_ctx *ctx, const double *scale);
DFG_API int dfg_set_blacklist(dfg_ctx *ctx, const uint8_t *blacklist);
DFG_API int dfg_set_beta_start(dfg_ctx *ctx, const double *beta_start);
DFG_API int dfg_calc_beta(dfg_ctx *ctx, double start, int need_scaling);

/* Per-pixel background [num_pix] of the detector (CDetector.parse_background,
 * detector.pyx:100-104; NULL removes it) and per-frame background scales
 * [num_data] (Iterate.parse_scale(bg=True), iterate.pyx:146-171, 311-312; NULL
 * means ones). With a background and need_scaling, dfg_maximize takes the
 * background-aware E-step (max_prob.c:134-156), tomogram update by bracketed
 * root finding (update_tomogram_bg, max_update.c:232-543) and scale update
 * (update_scale_bg, max_scale.c:21-288); the powder sum it needs is formed
 * from the frames (calc_powder, iterate.c:119-177). That path needs all frames
 * in one chunk (DFG_ERR_NOMEM otherwise; see option pair_budget_mb). */
DFG_API int dfg_set_background(dfg_ctx *ctx, const double *background);
DFG_API int dfg_set_bgscale(dfg_ctx *ctx, const double *bgscale);

/* ---- the iteration --------------------------------------------------------
 * update_beta (recon.pyx:151-174) then maximize (dragonfly/src/maximize.c:8-56):
 * rescale, E-step with the reference's pruning rule, normalisation, M-step,
 * merge into model2 / inter_weight and, when need_scaling && update_scale, the
 * phi update (dragonfly/src/max_scale.c:3-19). Writes the average
 * log-likelihood to *avg_likelihood. Replaces `maximize(struct max_data*)`
 * (dragonfly/src/maximize.h:45, called at recon.pyx:99). */
DFG_API int dfg_maximize(dfg_ctx *ctx, const dfg_iter_params *par, double *avg_likelihood);

/* EMCRecon.update_model for 3-D reconstructions with Friedel symmetry
 * (recon.pyx:112-149 with model.c:470-490): symmetrise the merged sums,
 * divide by inter_weight, rms change against model1, model1 <- model2
 * (alpha = 0) or alpha * model1 + (1 - alpha) * model2. */
DFG_API int dfg_update_model(dfg_ctx *ctx, double alpha, double *rms_change);

/* Model symmetries applied by dfg_update_model, as EMCRecon.update_model
 * (recon.pyx:120-134): point_group 1 (S4, Quaternion point_group 'S4') or 2
 * (A5, 'A5') replaces the Friedel average by symmetrize_octahedral /
 * symmetrize_icosahedral (model.c:636-757); axial_order > 1 then applies
 * symmetrize_axial (params.axial_sym, model.c:527-571). 0 and 0 restore the
 * default (Friedel only). The orientation list is reduced to the group's
 * asymmetric unit on the host (Quaternion.reduce_octahedral /
 * reduce_icosahedral, quaternion.pyx:177-255). */
DFG_API int dfg_set_symmetry(dfg_ctx *ctx, int point_group, int axial_order);

/* Coarse-to-fine orientation refinement (params.refine with iterate.quat_mapping,
 * rel_quat and num_rel_quat; maximize consults them at max_prob.c:110-120,
 * max_update.c:73-83 / :170-180 and max_scale.c:69-79; the legacy engine fills
 * them at src/iterate.c:103-130 and parse_rel_quat, src/iterate.c:364-527):
 * frame d evaluates orientation r only when quat_mapping[r] (its nearest
 * coarse orientation, [num_rot]) is one of rel_quat[rel_off[d] .. rel_off[d+1]).
 * quat_mapping == NULL switches refinement off. Needs frames and quaternions;
 * setting either again switches it off. One model mode only. */
DFG_API int dfg_set_refinement(dfg_ctx *ctx, int num_coarse, const int *quat_mapping,
                               const long long *rel_off, const int *rel_quat);
/* The same from a top-K array: frame d's relevant coarse orientations are
 * top[d * K .. d * K + K) (entries -1 are unused slots), except for the n_all
 * frames in all_frames, which evaluate every orientation (learned proposals
 * with held-out frames). */
DFG_API int dfg_set_refinement_topk(dfg_ctx *ctx, int num_coarse, const int *quat_mapping, int K, const int *top,
                                    int n_all, const int *all_frames);

/* Watched frames of a refined (proposal-restricted) search: frames[n]
 * (ascending) and, per frame, a list of coarse cells cells[cell_off[i] ..
 * cell_off[i+1]). After each dfg_maximize / dfg_run_iteration,
 * dfg_get_watch_mass gives for every watched frame the share of its
 * probability (sum of P) on orientations whose coarse cell is in its list:
 * with the frame searched in full and the list its proposal, the probability
 * mass the proposal would have captured. n = 0 clears. */
DFG_API int dfg_set_watch(dfg_ctx *ctx, int n, const int *frames, const long long *cell_off, const int *cells);
DFG_API int dfg_get_watch_mass(dfg_ctx *ctx, double *mass);

/* voronoi_subset (quaternion.c:844-862, Quaternion.voronoi_subset
 * quaternion.pyx:257-281): nearest[i] = the coarse orientation with the
 * smallest 1 - (q_i . c_j)^2, first on ties. Quaternions are rows of five
 * (q0..q3, weight). Runs on the context's device. */
DFG_API int dfg_voronoi_subset(dfg_ctx *ctx, int num_coarse, const double *coarse, int num_fine,
                               const double *fine, int *nearest);

/* Iterate.normalize_scale (dragonfly/iterate.pyx:361-384): mean phi over
 * good frames, mode-0 model1 *= mean, phi /= mean. Writes the mean. */
DFG_API int dfg_normalize_scale(dfg_ctx *ctx, double *mean_scale);

/* ---- results (host copies; NULL pointers are skipped) ---------------------
 * The read-only properties of EMCRecon / Iterate / Model
 * (dragonfly/recon.pyx:306-415, iterate.pyx:470-592, model.pyx:295-313). */
DFG_API int dfg_get_frame_results(dfg_ctx *ctx, int *rmax, double *info, double *likelihood,
                          double *max_exp, double *p_norm, double *psum_d);
DFG_API int dfg_get_quat_norm(dfg_ctx *ctx, double *quat_norm);             /* [num_data][num_modes] */
DFG_API int dfg_get_orientation_results(dfg_ctx *ctx, double *u, double *psum_r); /* [modes*num_rot] */
DFG_API int dfg_get_model(dfg_ctx *ctx, double *model1, double *model2, double *inter_weight);
DFG_API int dfg_get_frame_params(dfg_ctx *ctx, double *scale, double *beta, double *beta_start,
                         int *fcounts, double *sum_fact, uint8_t *blacklist);
/* out[0..4] = rescale, mutual_info, average log-likelihood, mean_count, rms_change */
DFG_API int dfg_get_scalars(dfg_ctx *ctx, double *out);
DFG_API int dfg_get_num_prob(dfg_ctx *ctx, int *num_prob);  /* kept pairs per frame */

/* Sparse probabilities of the last dfg_maximize, present when the option
 * "keep_prob" was set before it (replaces EMCRecon.prob / place_prob,
 * recon.pyx:409-415, which the reference fills when save_prob is set:
 * combine_information_omp, max_prob.c:294-325). For every frame, the pairs
 * with P > 1e-6 in ascending orientation order; frame d's entries are
 * [offsets[d], offsets[d + 1]) of place_prob (orientation index) and prob
 * (P, FP64). offsets has num_data + 1 entries; DFG_ERR_STATE without them. */
DFG_API int dfg_get_sparse_prob_offsets(dfg_ctx *ctx, long long *offsets);
DFG_API int dfg_get_sparse_prob(dfg_ctx *ctx, int *place_prob, double *prob);

/* Photon tomograms of orientations r0 .. r0 + n - 1 of the last dfg_maximize,
 * each divided by its psum_r where that is positive, as out[n][num_pix] FP64
 * (the views update_tomogram_nobg forms per orientation, max_update.c:142-230,
 * exposed by the reference only as the per-thread EMCRecon.all_views,
 * recon.pyx:342-351). */
DFG_API int dfg_get_tomograms(dfg_ctx *ctx, int r0, int n, double *out);

/* ---- one-slice operations -------------------------------------------------
 * Model.slice_gen (dragonfly/model.pyx:105-132 -> model.c:11-59, 65-150):
 * slice of model1 at one orientation, out[num_pix]; quat is a quaternion (5
 * values), an angle (2-D) or (phi, beta) (RZ) by the model type. */
DFG_API int dfg_slice_gen(dfg_ctx *ctx, const double *quat, int mode, double *out);
/* Model.slice_merge (dragonfly/model.pyx:134-151 -> model.c:171-340): merges
 * view[num_pix] into the host arrays model2 / inter_weight [modes][size^3]
 * ([modes][size^2] for 2-D and RZ models). */
DFG_API int dfg_slice_merge(dfg_ctx *ctx, const double *quat, int mode, const double *view,
                    double *model2, double *inter_weight);

/* Model.rotate_model (dragonfly/model.pyx:226-254 -> rotate_model,
 * model.c:381-425) on host arrays: for every voxel v of the cube
 * [-max_r, max_r)^3 around the centre, rotmodel[v + c] += the trilinear
 * interpolation of model at rot v + c (rot row-major 3x3; max_r 0 means
 * size / 2; voxels whose rotated position leaves the model get nothing).
 * model and rotmodel are [size][size][size]; rotmodel is read and updated. */
DFG_API int dfg_model_rotate(dfg_ctx *ctx, const double *rot, int size, int max_r, const double *model,
                             double *rotmodel);
/* Model.symmetrize_octahedral / symmetrize_icosahedral / symmetrize_axial
 * (dragonfly/model.pyx:175-210 -> model.c:527-757) on host arrays, in place:
 * weights <- sum over the group of the rotated weights, model <- (sum of the
 * rotated model x weights) / that sum where it is positive, else 0. group 1 =
 * S4 (48 rotations), 2 = A5 (60), 3 = the order-fold axial group about z. */
DFG_API int dfg_model_symmetrize(dfg_ctx *ctx, int group, int order, int size, double *model, double *weights);

/* dfg_slice_gen without any device allocation. No counterpart in the
 * reference: it is for callers that cannot allocate device memory while they
 * run -- an application whose own pool allocator owns the device memory
 * budget, or a real-time loop where a cudaMalloc / cudaFree would synchronise
 * the device. The scratch (quaternion and output slice) is a fixed file-scope
 * device array of DFG_NOALLOC_MAX_PIXELS doubles (2 MiB plus 64 bytes) that
 * each GPU loading the library holds until exit; detectors with more pixels
 * are rejected with DFG_ERR_ARG. The first call on a device looks the array's
 * address up (make it before any stream capture) and keeps it for the life of
 * the process: do not use this entry point across a cudaDeviceReset (or any
 * other teardown of the device's primary context) in the host process, since
 * the kept address would then point into freed memory. All calls share the
 * array: calls that overlap on the GPU race and must be serialised by the
 * caller. */
#define DFG_NOALLOC_MAX_PIXELS 262144
DFG_API int dfg_slice_gen_noalloc(dfg_ctx *ctx, const double *quat, int mode, double *out);

/* ---- one whole iteration --------------------------------------------------
 * EMCRecon.run_iteration's compute (recon.pyx:93-104) on the resident inputs:
 * dfg_maximize, dfg_update_model(alpha) and, when need_scaling and the model
 * is a volume, dfg_normalize_scale, with one host synchronisation at the end.
 * out[5] (may be NULL) = average log-likelihood, rms change (after the scale
 * normalisation), mutual information, rescale, mean scale (1 without
 * normalisation). Unless option keep_prob, timing or the background-aware
 * scale search needs the host between kernels, the iteration's kernels are
 * captured into a CUDA graph and launched as one (option graph, default 1);
 * later iterations update that graph in place. */
DFG_API int dfg_run_iteration(dfg_ctx *ctx, const dfg_iter_params *par, double alpha, double *out);

/* Autotuner: on the context's current inputs, times the slice kernel with
 * 128, 64, 32 and 16 orientations per block, and the E-step photon term and
 * the M-step each in their sparse (gathers) and dense (tensor-core) forms on
 * the first frame chunk, and keeps the fastest of each for later iterations
 * when option autotune is 1 (with option autotune, dfg_maximize /
 * dfg_run_iteration tune by themselves whenever the inputs changed).
 * When the sparse forms win it also times the sparse E-step at 2, 3 and 4
 * resident blocks per SM and the sparse M-step at 3, 4 and 5 (launch bounds:
 * registers per thread traded against warps in flight) and keeps the fastest.
 * report[DFG_TUNE_REPORT] (may be NULL): [0-3] slice ms per block size (-1:
 * not tried), [4-5] sparse and dense E-step ms (-1: form refused), [6] the
 * chosen block, [7] the chosen forms (E-step + 2 x M-step, 1 = dense), [8-9]
 * sparse and dense M-step ms, [10-12] sparse E-step ms at 2, 3, 4 blocks per
 * SM, [13-15] sparse M-step ms at 3, 4, 5 blocks per SM (-1: not timed),
 * [16] and [17] the chosen E-step and M-step blocks per SM. */
#define DFG_TUNE_REPORT 18
DFG_API int dfg_autotune(dfg_ctx *ctx, const dfg_iter_params *par, double *report);
/* The last autotuner report (DFG_TUNE_REPORT values) for the current inputs
 * (DFG_ERR_STATE if none). */
DFG_API int dfg_get_autotune_report(dfg_ctx *ctx, double *report);

/* ---- several detectors in one reconstruction -----------------------------
 * Replaces the reference's num_det loops (Iterate with in_detector_list,
 * dragonfly/iterate.pyx:432-456; calculate_rescale and calculate_prob,
 * dragonfly/src/max_prob.c:31-60, 96-106; calc_psum_r, update_tomogram_nobg
 * and merge_tomogram, dragonfly/src/max_update.c:18-40, 55-128, 153-229).
 * Member k is a context holding detector k and the frames seen by it, with
 * the same orientations, model (shape, type, values), parameters and
 * refinement setting as the others; member 0 also holds the model update's
 * symmetries. The per-detector quantities (u, rescale, psum_r, tomograms)
 * stay in the members; every member's merged sums are added into member 0's
 * (one model2 / inter_weight, as in the reference), member 0 updates the
 * model and the others receive a copy. Averages (log-likelihood, mutual
 * information) and normalize_scale's mean scale are taken over the frames of
 * all detectors. Background-aware updates with several detectors return
 * DFG_ERR_ARG. Per-frame results: dfg_get_frame_results on each member (its
 * frames in its own order); the model: dfg_get_model on member 0. */
typedef struct dfg_group dfg_group;
DFG_API int dfg_group_create(dfg_ctx *const *members, int n, dfg_group **out);
DFG_API void dfg_group_destroy(dfg_group *group);
DFG_API const char *dfg_group_last_error(const dfg_group *group);
/* maximize() over all detectors (maximize.c:8-56 with num_det > 1). */
DFG_API int dfg_group_maximize(dfg_group *group, const dfg_iter_params *par, double *avg_likelihood);
/* EMCRecon.update_model (recon.pyx:112-149) on the shared model. */
DFG_API int dfg_group_update_model(dfg_group *group, double alpha, double *rms_change);
/* Iterate.normalize_scale (iterate.pyx:361-384) over all detectors' frames. */
DFG_API int dfg_group_normalize_scale(dfg_group *group, double *mean_scale);
/* One iteration as dfg_run_iteration; out[5]: average log-likelihood, rms
 * change, mutual information, detector 0's rescale factor, mean scale. */
DFG_API int dfg_group_run_iteration(dfg_group *group, const dfg_iter_params *par, double alpha, double *out);

/* ---- batches of independent reconstructions -------------------------------
 * Several contexts on one GPU (different detectors, frames, orientation sets,
 * models and modes) iterated together: dfg_batch_run runs dfg_run_iteration
 * on every context with pars[i] and alphas[i] (NULL: 0), captured as one CUDA
 * graph in which each reconstruction runs on its own stream, forked from and
 * joined back into the batch's stream (see dfg_batch_set_lanes), with no host
 * synchronisation between reconstructions. out
 * (may be NULL) receives n x 5 values as dfg_run_iteration's. When a context
 * needs the host between kernels (keep_prob, the background-aware scale
 * search) the batch queues them without a graph. No counterpart in the
 * reference (one reconstruction per process). */
typedef struct dfg_batch dfg_batch;
DFG_API int dfg_batch_create(dfg_ctx *const *ctxs, int n, dfg_batch **out);
DFG_API int dfg_batch_run(dfg_batch *batch, const dfg_iter_params *pars, const double *alphas, double *out);
DFG_API const char *dfg_batch_last_error(const dfg_batch *batch);
/* Concurrent branches of the batch graph (default 1: the reconstructions run
 * one after another inside one launch). With more lanes, reconstructions are
 * dealt out by decreasing frame x orientation count to the least-loaded lane
 * and the lanes run side by side (useful when single reconstructions leave
 * SMs idle; concurrent reconstructions compete for L2). */
DFG_API int dfg_batch_set_lanes(dfg_batch *batch, int lanes);
/* out[0] = graph launches, out[1] = instantiations, out[2] = in-place updates. */
DFG_API int dfg_batch_stats(dfg_batch *batch, long *out);
DFG_API void dfg_batch_destroy(dfg_batch *batch);

/* ---- learned orientation proposals ----------------------------------------
 * A small convolutional network (csrc/proposal.cu) mapping a frame's photon
 * image (log(1 + photons) binned on a 32 x 32 grid: pixel_bin[p] in
 * [0, 1024) or -1) to logits over num_classes coarse orientations: conv 3x3
 * 1->32, 32->32 (stride 2), 32->64, 64->64 (stride 2), fully connected
 * 4096->256->num_classes, ReLU between; BF16 weights in the products, FP32
 * accumulation and Adam state. Training and inference run on the GPU by this
 * library's own kernels. The top-K classes of a frame restrict its E-step
 * (dfg_set_refinement with the coarse map of dfg_voronoi_subset). No
 * counterpart in the reference. Parameters are flat FP32: per layer the
 * weights [cout][fan_in] (convolution rows ordered ky, kx, c), then the
 * biases. */
typedef struct dfg_pnet dfg_pnet;
DFG_API int dfg_pnet_create(int device, int num_classes, int batch, unsigned long long seed, dfg_pnet **out);
DFG_API void dfg_pnet_destroy(dfg_pnet *net);
DFG_API const char *dfg_pnet_last_error(const dfg_pnet *net);
DFG_API long long dfg_pnet_num_params(const dfg_pnet *net);
DFG_API int dfg_pnet_get_params(dfg_pnet *net, float *out);
DFG_API int dfg_pnet_set_params(dfg_pnet *net, const float *in);
DFG_API int dfg_pnet_set_bins(dfg_pnet *net, int num_pix, const int *pixel_bin);
/* Images of the context's frames (its mask-0 photons), kept on the device. */
DFG_API int dfg_pnet_load_frames(dfg_pnet *net, dfg_ctx *ctx);
/* Images [n][1024] from the host (tests), and the loaded images back. */
DFG_API int dfg_pnet_set_images(dfg_pnet *net, long long n, const float *images);
DFG_API int dfg_pnet_get_images(dfg_pnet *net, float *out);
/* epochs of Adam over the loaded images (shuffled by seed) against labels
 * [n] in [0, num_classes); *mean_loss = the last epoch's mean loss. */
DFG_API int dfg_pnet_train(dfg_pnet *net, const int *labels, int epochs, double lr, unsigned long long seed,
                           double *mean_loss);
/* Soft targets of the loaded images (until images are loaded again): image
 * i's classes t_cls[t_off[i] .. t_off[i + 1]) with weights t_w (distinct
 * classes, weights >= 0 summing to 1). dfg_pnet_train and dfg_pnet_gradients
 * called with labels == NULL minimise the cross-entropy against them. */
DFG_API int dfg_pnet_set_targets(dfg_pnet *net, const long long *t_off, const int *t_cls, const float *t_w);
/* Inference products (dfg_pnet_topk, dfg_pnet_logits) of layers 1-5 on the
 * tcgen05 tensor cores with BF16 activations (on = 1, the default) or on the
 * FP32 path (on = 0). */
DFG_API int dfg_pnet_set_tensor_cores(dfg_pnet *net, int on);
/* Network options by name (no counterpart in the reference): "tensor_cores"
 * (as dfg_pnet_set_tensor_cores); "tensor_core_training" (1, the default:
 * dfg_pnet_train and dfg_pnet_gradients compute the products of layers 1-5,
 * forward, weight and input gradients, on the tcgen05 tensor cores with BF16
 * operands and FP32 accumulation; 0: on the FP32 path, FP32 activations and
 * gradients against BF16 weights); and two failure-detection test hooks of
 * the tensor-core products, "wait_cycles" (clock cycles after which a
 * pipeline wait gives up, default 2e9) and "withhold_stage" (a stage whose
 * copies are never issued, so its waits run out and the call returns
 * DFG_ERR_CUDA; -1, the default, issues every stage). */
DFG_API int dfg_pnet_set_option(dfg_pnet *net, const char *key, double value);

/* out[n][K]: the K largest logits' classes of every loaded image, largest first. */
DFG_API int dfg_pnet_topk(dfg_pnet *net, int K, int *out);
/* Mass-covering proposals (no counterpart in the reference): out[n][K_max],
 * per image the classes in decreasing order of their logits, K_min of them
 * and then more until their softmax probabilities sum to `mass`, at most
 * K_max; unused slots are -1. */
DFG_API int dfg_pnet_topk_mass(dfg_pnet *net, int K_min, int K_max, double mass, int *out);
DFG_API int dfg_pnet_logits(dfg_pnet *net, float *out);
/* Mean loss and gradients (flat, as the parameters) on the first
 * min(n, batch) loaded images with labels; the parameters are not changed. */
DFG_API int dfg_pnet_gradients(dfg_pnet *net, const int *labels, float *grads, double *mean_loss);

/* Graph use of dfg_run_iteration: out[0] = graph launches, out[1] =
 * instantiations, out[2] = in-place updates. */
DFG_API int dfg_get_graph_stats(dfg_ctx *ctx, long *out);

/* ---- end to end from host buffers ----------------------------------------
 * EMCRecon.run_iteration's compute (recon.pyx:93-104): model1_inout (host,
 * [modes][size^3]) is uploaded, dfg_run_iteration runs, and the new model1,
 * rmax[num_data] and likelihood[num_data] come back to host memory. */
DFG_API int dfg_run_iteration_host(dfg_ctx *ctx, const dfg_iter_params *par, double alpha,
                           double *model1_inout, int *rmax, double *likelihood,
                           double *avg_likelihood, double *rms_change);

/* ---- synthetic data -------------------------------------------------------
 * GPU counterpart of the reference simulator's gen_and_save_dataset
 * (dragonfly/utils/src/make_data.c:115-326): for each frame d, the slice of
 * intens [size^3] (centre size / 2) at quats4[d] (q0..q3) on the context's
 * detector, times phi[d], Poisson-sampled on pixels with mask <= 1. The frames
 * become the context's frames (as dfg_set_frames). totals[0..2] = ones total,
 * multi total, photons. dfg_get_frames copies the context's frames out
 * (arrays sized from dfg_set_frames / the totals). */
DFG_API int dfg_simulate_frames(dfg_ctx *ctx, long size, const double *intens, int num_data,
                                const double *quats4, const double *phi, unsigned long long seed,
                                long long *totals);
DFG_API int dfg_get_frames(dfg_ctx *ctx, int *ones, int *multi, int *place_ones, int *place_multi,
                           int *count_multi);

/* Binary .emc files (1024-byte header of int32 num_data, num_pix, type): load
 * one or more (type 0 sparse, or type 1 dense integer, turned sparse) into the
 * context as dfg_set_frames would; save the context's frames as one sparse
 * file. Replace CDataset / EMCReader parsing (parse_binarydataset,
 * emcfile.c:3-57; emcfile.pyx:200-330) and EMCWriter (emcfile.pyx:420-532). */
DFG_API int dfg_load_emc(dfg_ctx *ctx, int num_files, const char *const *paths);
DFG_API int dfg_save_emc(dfg_ctx *ctx, const char *path);

/* ---- tuning and instrumentation ------------------------------------------
 * Options: "pair_budget_mb" (device memory for the per-pair buffers, which
 * sets the frame chunk), "timing" (1: record per-phase CUDA-event times),
 * "keep_prob" (1: keep the sparse probability lists), "graph" (1: capture
 * iterations as CUDA graphs), "autotune" (1: time the kernel forms on the
 * inputs and keep the fastest), "estep_form" / "mstep_form" (0 sparse, 1
 * tensor-core products), "slice_block" (orientations per slice block, 0
 * automatic), "tile_skip" (skip dead (tile, frame) pairs without
 * refinement), "pair_lists" (1: restricted searches store only their live
 * (tile, frame) pairs, orientations in blocks), "block_budget_mb" (device
 * memory for one block of log-slices (and tomograms); without refinement a
 * value > 0 runs the full search in orientation blocks, which it also does
 * when the resident log-slices and tomograms would exceed half the memory),
 * "estep_blocks_per_sm" / "mstep_blocks_per_sm" (resident blocks per SM of
 * the sparse E-step, 2-4, and M-step, 3-5; 0, the default, takes the
 * autotuner's choice or the build's default), and two failure-detection test
 * hooks of the tensor-core kernels:
 * "dense_wait_cycles" (clock cycles after which a pipeline wait gives up,
 * default 2e9, about a second) and "dense_withhold_stage" (a stage index
 * whose copies are never issued, so the waits on it run out and the call
 * returns DFG_ERR_CUDA; -1, the default, issues every stage). */
DFG_API int dfg_set_option(dfg_ctx *ctx, const char *key, double value);
/* Phase times in ms summed since the last reset, and launch counts:
 * names[i] = "slice", "estep", "norm", "psum", "mstep", "merge", "update".
 * n = number of slots provided. Returns the number of phases. */
DFG_API int dfg_get_phase_times(dfg_ctx *ctx, double *ms, long *launches, int n);
DFG_API const char *dfg_phase_name(int i);
/* Device timing on the context's stream: dfg_event_record puts a CUDA event
 * (slot 0..7) on the stream; dfg_event_elapsed waits for slot b and writes the
 * milliseconds from slot a to slot b. */
DFG_API int dfg_event_record(dfg_ctx *ctx, int slot);
DFG_API int dfg_event_elapsed(dfg_ctx *ctx, int a, int b, double *ms);
DFG_API int dfg_reset_phase_times(dfg_ctx *ctx);
/* Sizes of the last iteration: out[0] = R (modes * num_rot), out[1] = frames,
 * out[2] = photon entries in the E-step lists, out[3] = M-step entries,
 * out[4] = frame chunks, out[5] = frames per chunk, out[6] = kernels launched
 * by this context so far, out[7] = mask < 2 pixel columns of the dense forms
 * (padded to 64; 0 before it is used), out[8] = forms of the last
 * iteration: 1 = dense E-step, 2 = dense M-step (bits), out[9] = live
 * (tile, frame) pairs of the pair lists (0 without them), out[10] =
 * orientation tiles per block of the pair lists. out must hold 11 values. */
DFG_API int dfg_get_workload(dfg_ctx *ctx, long long *out);

/* Ceiling of the gather kernels' access pattern on the context's device. No
 * counterpart in the reference (a measurement helper): reads uniformly random
 * 512-byte rows (one 16-byte load per lane, eight rows in flight per lane, all
 * SMs at full occupancy) of a device table of `rows` rows, the shape of the
 * E-step's log-slice tile [P + 1][128] FP32 or the M-step's probability tile;
 * writes the best of `reps` timed launches (after one warm-up launch) in GB/s
 * of row bytes. Allocates the table for the call and frees it. */
DFG_API int dfg_measure_gather_rate(dfg_ctx *ctx, long long rows, int reps, double *gbs);

#ifdef __cplusplus
}
#endif
#endif
