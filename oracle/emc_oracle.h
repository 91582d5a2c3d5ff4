/* CPU oracle for one EMC iteration (expand -> maximize -> compress) on sparse
 * photon data. TEST INFRASTRUCTURE ONLY: the product never links it; tests/,
 * the smoke check and bench.py's CPU-baseline leg use it as the checker.
 *
 * An FP64 restatement of duaneloh/Dragonfly's packaged engine
 * (dragonfly/src/maximize.c, max_prob.c, max_update.c, max_scale.c, model.c,
 * iterate.c) and of the model update in dragonfly/recon.pyx:112-149. Floating
 * point operations are written in the reference's order so that, built without
 * FMA contraction, results are bit-identical to the reference engine run with
 * one OpenMP thread, at any thread count of the oracle itself (it parallelises
 * only where every sum keeps its order). Pinned against the compiled reference
 * (oracle/_ref) and against committed golden vectors by tests/test_oracle.py.
 */
#ifndef DFG_EMC_ORACLE_H
#define DFG_EMC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Rotation matrix of a unit quaternion (model.c:759-786). */
void orc_make_rot_quat(const double *q, double rot[3][3]);

/* W_t = corr_t * trilinear(model[mode], R q_t + center); out-of-bounds -> DBL_MIN
 * (model.c:11-59). */
void orc_slice_gen3d(const double *quat, int mode, double *slice, int num_pix, const double *qvals,
                     const double *corr, long size, long center, const double *model1);

/* model2 += f * slice/corr, weight += f over the 8 corners, pixels with mask < 2
 * (model.c:171-244). */
void orc_slice_merge3d(const double *quat, int mode, const double *slice, double *model2, double *weight,
                       long size, int num_pix, const double *qvals, const double *corr, const uint8_t *mask);

/* Friedel average of un-normalised sums (model.c:470-490). */
void orc_symmetrize_friedel(double *array, const double *weights, int size);

/* fcounts, sum_fact (ln c! as lgamma(c+1)) and mean_count (iterate.c:3-117). */
void orc_frame_stats(int num_data, const int *ones, const int *multi, const int *place_ones,
                     const int *place_multi, const int *count_multi, const uint8_t *mask,
                     int *fcounts, double *sum_fact, double *mean_count);

/* beta_start per frame (iterate.c:66-83). start < 0 selects the empirical rule. */
void orc_calc_beta(int num_data, double start, int need_scaling, double mean_count, const int *fcounts,
                   double *beta_start);

/* One call of maximize() (maximize.c:8-56) for one detector and one dataset.
 * Outputs (caller-allocated):
 *   model2, weight      [M*V]  un-normalised merge sums (zeroed first)
 *   u                   [M*R]  sum of W over mask==0 pixels per orientation
 *   psum_r              [M*R]
 *   rmax, info, likelihood, max_exp, p_norm, psum_d   [N]
 *   quat_norm           [N*M]  (only written when M > 1)
 *   scale               [N]    in/out: updated in place when need_scaling && update_scale
 *   scalars_out         [3]    rescale, mutual_info, avg_likelihood
 *   num_prob            [N]    kept-list length per frame (may be NULL)
 * Returns the average log-likelihood. */
double orc_maximize(int num_pix, const double *qvals, const double *corr, const uint8_t *mask,
                    int num_data, const int *ones, const int *multi, const int *place_ones,
                    const int *place_multi, const int *count_multi,
                    int num_rot, int num_modes, const double *quats,
                    long size, const double *model1,
                    double *scale, const double *beta, const double *sum_fact, const int *fcounts,
                    const uint8_t *blacklist, double mean_count,
                    int need_scaling, int update_scale, int known_scale, int iteration,
                    double *model2, double *weight, double *u, double *psum_r,
                    int *rmax, double *info, double *likelihood, double *max_exp, double *p_norm,
                    double *psum_d, double *quat_norm, int *num_prob, double *scalars_out);

/* orc_maximize for several detectors (Iterate with in_detector_list,
 * iterate.pyx:432-456): detector k has num_pix[k] pixels with qvals[k]
 * [num_pix][3], corr[k] and mask[k]; frame d is seen by detector det_of[d];
 * mean_count [K] per detector. Per-detector outputs: u and psum_r [K*M*R]
 * (detector-major), rescale [K]; scalars_out [2]: mutual_info,
 * avg_likelihood. The merge adds, per orientation, the detectors in
 * ascending order (max_update.c:34-36). */
double orc_maximize_dets(int num_det, const int *num_pix, const double *const *qvals,
                         const double *const *corr, const uint8_t *const *mask, const int *det_of,
                         int num_data, const int *ones, const int *multi, const int *place_ones,
                         const int *place_multi, const int *count_multi,
                         int num_rot, int num_modes, const double *quats,
                         long size, const double *model1,
                         double *scale, const double *beta, const double *sum_fact, const int *fcounts,
                         const uint8_t *blacklist, const double *mean_count,
                         int need_scaling, int update_scale, int known_scale, int iteration,
                         double *model2, double *weight, double *u, double *psum_r,
                         int *rmax, double *info, double *likelihood, double *max_exp, double *p_norm,
                         double *psum_d, double *quat_norm, int *num_prob, double *rescale,
                         double *scalars_out);

/* With on != 0, orc_maximize keeps its per-frame probability lists (kept
 * orientations in ascending order and their normalised probabilities P) until
 * the next call; orc_kept_prob(d, pos, val) copies frame d's list into pos /
 * val (either may be NULL) and returns its length, -1 when none is kept. */
void orc_set_keep_prob(int on);
int orc_kept_prob(int d, int *pos, double *val);

/* EMCRecon.update_model for RECON3D with Friedel symmetry only (recon.pyx:112-149).
 * model2 is normalised in place and model1 is replaced (alpha = 0) or mixed.
 * Returns rms_change. */
double orc_update_model(long size, int num_modes, double *model1, double *model2, double *weight,
                        double alpha);

#ifdef __cplusplus
}
#endif
#endif
