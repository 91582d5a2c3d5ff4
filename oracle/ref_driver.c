/* Driver for the reference's own packaged C engine, built from its unmodified
 * sources (dragonfly/src/{maximize,max_prob,max_update,max_scale,model,iterate,
 * quaternion}.c) into oracle/_ref/. TEST INFRASTRUCTURE ONLY: tests/, the smoke
 * check and bench.py's CPU-baseline leg use it as the checker and as the timed
 * reference arm; the product never links it.
 *
 * The reference's Python layer (dragonfly/recon.pyx, iterate.pyx) cannot be
 * built here (no mpi4py/h5py), so this file takes its place around the C engine:
 *   - it fills the reference structs the way Iterate.set_data / set_quat /
 *     set_model / calc_beta do (dragonfly/iterate.pyx:241-266, 386-402),
 *   - ref_maximize() runs EMCRecon.run_iteration's compute steps
 *     (dragonfly/recon.pyx:86-99): select slice_gen3d/slice_merge3d, update_beta
 *     (recon.pyx:151-174), then the reference's maximize() (maximize.c:8-56),
 *   - ref_update_model() restates EMCRecon.update_model (recon.pyx:112-149) for
 *     the 3-D Friedel case, calling the reference's symmetrize_friedel.
 * Iterate.normalize_scale (iterate.pyx:361-384) is numpy code in the reference
 * and is restated in numpy by oracle/oracle.py.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "max_internal.h"

typedef struct ref_engine {
	struct detector det;
	struct dataset dset;
	struct quaternion quat;
	struct model mod;
	struct params par;
	struct iterate iter;
	struct max_data *mdata;
	int det_mapping[1];
	double avg_likelihood;
	double beta_start;          /* calc_beta's argument, for ref_add_detector */
	int num_threads;            /* OpenMP threads of this engine's calls (<= 0: the default) */
	/* more detectors (ref_add_detector): all detectors contiguous (detector 0
	 * a copy of det), their datasets linked after dset, one per detector */
	struct detector *dets;
	struct dataset **extra;
	int *det_map;
	int n_extra;
} ref_engine;

static void *dup_mem(const void *src, size_t bytes) {
	void *dst = malloc(bytes > 0 ? bytes : 1);
	if (src != NULL && bytes > 0)
		memcpy(dst, src, bytes);
	return dst;
}

/* Frees the per-call arrays that maximize() allocates on the common struct
 * (maximize.c:58-97). The reference itself leaks them on every call. */
static void free_common(struct max_data *c, int num_data, int num_det) {
	int d;
	if (c->rmax == NULL)
		return;
	free(c->rmax); free(c->info); free(c->likelihood); free(c->max_exp_p);
	free(c->quat_norm); free(c->num_prob); free(c->psum_d);
	if (c->prob != NULL) {
		for (d = 0; d < num_data; ++d) {
			free(c->prob[d]);
			free(c->place_prob[d]);
		}
	}
	free(c->prob); free(c->place_prob);
	if (c->u != NULL) {
		for (d = 0; d < num_det; ++d)
			free(c->u[d]);
		free(c->u);
	}
	free(c->max_exp); free(c->p_norm); free(c->offset_prob);
	memset(c, 0, sizeof(*c));
}

ref_engine *ref_create(int num_pix, const double *qvals, const double *corr, const uint8_t *mask,
                       int num_data, const int *ones, const int *multi, const int *place_ones,
                       const int *place_multi, const int *count_multi,
                       int num_rot, const double *quats,
                       long size, int num_modes, int mtype, const double *model1,
                       int need_scaling, int update_scale, int known_scale, double alpha,
                       double beta_start, double beta_jump, int beta_period, double beta_factor,
                       const double *scale, const uint8_t *blacklist, int num_threads) {
	long d, ones_total = 0, multi_total = 0;
	ref_engine *e = calloc(1, sizeof(ref_engine));
	/* the thread count applies to this engine's calls only (ref_maximize,
	 * ref_update_model): setting it for the process would also slow every
	 * later OpenMP region of the caller (the oracle's among them) */
	e->num_threads = num_threads;

	/* Detector (detector.pyx:61-74) */
	e->det.num_pix = num_pix;
	e->det.qvals = dup_mem(qvals, (size_t)num_pix * 3 * sizeof(double));
	e->det.corr = dup_mem(corr, (size_t)num_pix * sizeof(double));
	e->det.raw_mask = dup_mem(mask, (size_t)num_pix);
	e->det.with_bg = 0;

	/* Sparse dataset, as parse_binarydataset lays it out (emcfile.c:15-37) */
	e->dset.ftype = SPARSE;
	e->dset.num_data = num_data;
	e->dset.num_pix = num_pix;
	e->dset.det = &e->det;
	e->dset.next = NULL;
	e->dset.num_offset = 0;
	e->dset.ones = dup_mem(ones, (size_t)num_data * sizeof(int));
	e->dset.multi = dup_mem(multi, (size_t)num_data * sizeof(int));
	e->dset.ones_accum = malloc((size_t)(num_data > 0 ? num_data : 1) * sizeof(long));
	e->dset.multi_accum = malloc((size_t)(num_data > 0 ? num_data : 1) * sizeof(long));
	for (d = 0; d < num_data; ++d) {
		e->dset.ones_accum[d] = ones_total;
		e->dset.multi_accum[d] = multi_total;
		ones_total += ones[d];
		multi_total += multi[d];
	}
	e->dset.ones_total = ones_total;
	e->dset.multi_total = multi_total;
	e->dset.place_ones = dup_mem(place_ones, (size_t)ones_total * sizeof(int));
	e->dset.place_multi = dup_mem(place_multi, (size_t)multi_total * sizeof(int));
	e->dset.count_multi = dup_mem(count_multi, (size_t)multi_total * sizeof(int));

	/* Parameters (params.pyx:13-46 defaults, then the values we are given) */
	e->par.rank = 0;
	e->par.num_proc = 1;
	e->par.rtype = mtype == MODEL_2D ? RECON2D : (mtype == MODEL_RZ ? RECONRZ : RECON3D);
	e->par.verbosity = 0;
	e->par.need_scaling = need_scaling;
	e->par.update_scale = update_scale;
	e->par.known_scale = known_scale;
	e->par.alpha = alpha;
	e->par.beta_jump = beta_jump;
	e->par.beta_period = beta_period;
	e->par.beta_factor = beta_factor;
	e->par.num_modes = num_modes;
	e->par.nonrot_modes = 0;
	e->par.axial_sym = 1;
	e->par.iteration = 1;

	/* Orientations; Quaternion.divide for one rank (quaternion.pyx:156-175) */
	e->quat.num_rot = num_rot;
	e->quat.quats = dup_mem(quats, (size_t)num_rot * 5 * sizeof(double));
	e->quat.num_rot_p = num_modes * num_rot;

	/* Model (model.pyx:24-63, 280-284): a volume, or a stack of 2-D images
	 * (MODEL_2D, MODEL_RZ) */
	e->mod.mtype = mtype;
	e->mod.size = size;
	e->mod.center = size / 2;
	e->mod.vol = mtype == MODEL_3D ? size * size * size : size * size;
	e->mod.num_modes = num_modes;
	e->mod.model1 = dup_mem(model1, (size_t)num_modes * e->mod.vol * sizeof(double));
	e->mod.model2 = calloc((size_t)num_modes * e->mod.vol, sizeof(double));
	e->mod.inter_weight = calloc((size_t)num_modes * e->mod.vol, sizeof(double));

	/* Iterate.set_data (iterate.pyx:241-266) with one detector and one file */
	e->iter.det = &e->det;
	e->iter.mod = &e->mod;
	e->iter.dset = &e->dset;
	e->iter.quat = &e->quat;
	e->iter.par = &e->par;
	e->iter.tot_num_data = num_data;
	e->iter.num_det = 1;
	e->iter.num_dfiles = 1;
	e->det_mapping[0] = 0;
	e->iter.det_mapping = e->det_mapping;
	calc_frame_counts(&e->iter);
	/* Iterate.parse_blacklist copies the flags but never sets num_blacklist
	 * (iterate.pyx:317-359), so it stays 0 as calloc left it. */
	e->iter.blacklist = calloc((size_t)(num_data > 0 ? num_data : 1), 1);
	if (blacklist != NULL)
		memcpy(e->iter.blacklist, blacklist, (size_t)num_data);
	calc_sum_fact(&e->iter);
	if (need_scaling) {
		e->iter.scale = malloc((size_t)(num_data > 0 ? num_data : 1) * sizeof(double));
		for (d = 0; d < num_data; ++d)
			e->iter.scale[d] = scale != NULL ? scale[d] : 1.;
	}
	e->beta_start = beta_start;
	calc_beta(beta_start, &e->iter);

	e->mdata = calloc(1, sizeof(struct max_data));
	e->mdata->iter = &e->iter;
	return e;
}

/* recon.pyx:151-174 (update_beta) followed by recon.pyx:86-99 (maximize). */
double ref_maximize(ref_engine *e, int iteration) {
	int d;
	struct iterate *it = &e->iter;
	double factor;

	e->par.iteration = iteration;
	factor = pow(e->par.beta_jump, (double)((iteration - 1) / e->par.beta_period));
	factor *= e->par.beta_factor;
	for (d = 0; d < it->tot_num_data; ++d) {
		if (it->blacklist[d] == 1)
			continue;
		it->beta[d] = it->beta_start[d] * factor;
		if (it->beta[d] > 1.)
			it->beta[d] = 1.;
	}

	/* recon.pyx:86-91: 3-D or 2-D slice functions (none for RECONRZ there) */
	if (e->par.rtype == RECON2D) {
		slice_gen = &slice_gen2d;
		slice_merge = &slice_merge2d;
	}
	else {
		slice_gen = &slice_gen3d;
		slice_merge = &slice_merge3d;
	}
	free_common(e->mdata, it->tot_num_data, it->num_det);
	e->mdata->iter = it;
	e->mdata->within_openmp = 0;
	{
		const int prev = omp_get_max_threads();
		if (e->num_threads > 0)
			omp_set_num_threads(e->num_threads);
		e->avg_likelihood = maximize(e->mdata);
		omp_set_num_threads(prev);
	}
	return e->avg_likelihood;
}

/* recon.pyx:112-149: for RECONRZ, or RECON2D with params.friedel_sym, the
 * 2-D Friedel average of every layer; for RECON3D the icosahedral or
 * octahedral point group (Quaternion.icosahedral_flag / octahedral_flag) in
 * place of the Friedel average, then the axial symmetry (params.axial_sym,
 * volumes only); then the division. */
double ref_update_model(ref_engine *e) {
	long x;
	double diff, change = 0.;
	struct model *mod = &e->mod;

	if (e->par.rtype == RECONRZ || (e->par.rtype == RECON2D && e->par.friedel_sym))
		symmetrize_friedel2d(mod->model2, mod->inter_weight, mod->num_modes, (int)mod->size);
	for (x = 0; x < mod->num_modes && e->par.rtype == RECON3D; ++x) {
		double *m2 = &mod->model2[x * mod->vol], *w = &mod->inter_weight[x * mod->vol];
		if (e->quat.icosahedral_flag)
			symmetrize_icosahedral(m2, w, (int)mod->size);
		else if (e->quat.octahedral_flag)
			symmetrize_octahedral(m2, w, (int)mod->size);
		else
			symmetrize_friedel(m2, w, (int)mod->size);
	}
	if (e->par.axial_sym > 1 && e->par.rtype == RECON3D)
		for (x = 0; x < mod->num_modes; ++x)
			symmetrize_axial(&mod->model2[x * mod->vol], &mod->inter_weight[x * mod->vol], (int)mod->size,
			                 e->par.axial_sym);
	for (x = 0; x < mod->num_modes * mod->vol; ++x)
		if (mod->inter_weight[x] > 0.)
			mod->model2[x] /= mod->inter_weight[x];
	for (x = 0; x < mod->num_modes * mod->vol; ++x) {
		diff = mod->model2[x] - mod->model1[x];
		change += diff * diff;
		if (e->par.alpha > 0.)
			mod->model1[x] = e->par.alpha * mod->model1[x] + (1 - e->par.alpha) * mod->model2[x];
		else
			mod->model1[x] = mod->model2[x];
	}
	e->iter.rms_change = sqrt(change / mod->num_modes / mod->vol);
	return e->iter.rms_change;
}

void ref_set_refinement(ref_engine *e, const int *quat_mapping, const long long *rel_off, const int *rel_quat);

static void copy_or_zero(void *dst, const void *src, size_t bytes);

/* One more detector with one dataset of frames seen by it, appended after the
 * frames so far (Iterate.set_data with a dataset list whose files name
 * several detectors, iterate.pyx:241-266 and _gen_detlist :432-456; the new
 * detector gets the next index). The per-frame arrays are formed again as
 * set_data / parse_scale / parse_blacklist / calc_beta form them; scale and
 * blacklist give the new frames' values (NULL: 1 and 0). */
void ref_add_detector(ref_engine *e, int num_pix, const double *qvals, const double *corr, const uint8_t *mask,
                      int num_data, const int *ones, const int *multi, const int *place_ones,
                      const int *place_multi, const int *count_multi, const double *scale,
                      const uint8_t *blacklist) {
	struct iterate *it = &e->iter;
	const int K = it->num_det + 1, old_n = it->tot_num_data, n = old_n + num_data;
	struct detector *dets = calloc((size_t)K, sizeof(struct detector));
	struct dataset *ds = calloc(1, sizeof(struct dataset)), *curr;
	long d, ones_total = 0, multi_total = 0;
	int k;

	memcpy(dets, it->det, (size_t)(K - 1) * sizeof(struct detector));
	dets[K - 1].num_pix = num_pix;
	dets[K - 1].qvals = dup_mem(qvals, (size_t)num_pix * 3 * sizeof(double));
	dets[K - 1].corr = dup_mem(corr, (size_t)num_pix * sizeof(double));
	dets[K - 1].raw_mask = dup_mem(mask, (size_t)num_pix);
	dets[K - 1].detd = e->det.detd;
	free(e->dets);
	e->dets = dets;
	it->det = dets;

	ds->ftype = SPARSE;
	ds->num_data = num_data;
	ds->num_pix = num_pix;
	ds->num_offset = old_n;
	ds->ones = dup_mem(ones, (size_t)num_data * sizeof(int));
	ds->multi = dup_mem(multi, (size_t)num_data * sizeof(int));
	ds->ones_accum = malloc((size_t)(num_data > 0 ? num_data : 1) * sizeof(long));
	ds->multi_accum = malloc((size_t)(num_data > 0 ? num_data : 1) * sizeof(long));
	for (d = 0; d < num_data; ++d) {
		ds->ones_accum[d] = ones_total;
		ds->multi_accum[d] = multi_total;
		ones_total += ones[d];
		multi_total += multi[d];
	}
	ds->ones_total = ones_total;
	ds->multi_total = multi_total;
	ds->place_ones = dup_mem(place_ones, (size_t)ones_total * sizeof(int));
	ds->place_multi = dup_mem(place_multi, (size_t)multi_total * sizeof(int));
	ds->count_multi = dup_mem(count_multi, (size_t)multi_total * sizeof(int));
	e->extra = realloc(e->extra, (size_t)(e->n_extra + 1) * sizeof(struct dataset *));
	e->extra[e->n_extra++] = ds;
	for (curr = &e->dset; curr->next != NULL; curr = curr->next)
		;
	curr->next = ds;
	/* every dataset's detector in the new array (calc_frame_counts reads it) */
	e->dset.det = &dets[0];
	for (k = 0; k < e->n_extra; ++k)
		e->extra[k]->det = &dets[k + 1];

	free(e->det_map);
	e->det_map = malloc((size_t)K * sizeof(int));
	for (k = 0; k < K; ++k)
		e->det_map[k] = k;
	it->det_mapping = e->det_map;
	it->num_det = K;
	it->num_dfiles = K;
	it->tot_num_data = n;

	free(it->fcounts); it->fcounts = NULL;
	free(it->mean_count); it->mean_count = NULL;
	free(it->rescale); it->rescale = NULL;
	calc_frame_counts(it);
	it->blacklist = realloc(it->blacklist, (size_t)(n > 0 ? n : 1));
	for (d = 0; d < num_data; ++d)
		it->blacklist[old_n + d] = blacklist != NULL ? blacklist[d] : 0;
	free(it->sum_fact); it->sum_fact = NULL;
	calc_sum_fact(it);
	if (e->par.need_scaling) {
		it->scale = realloc(it->scale, (size_t)(n > 0 ? n : 1) * sizeof(double));
		for (d = 0; d < num_data; ++d)
			it->scale[old_n + d] = scale != NULL ? scale[d] : 1.;
	}
	free(it->beta); it->beta = NULL;
	free(it->beta_start); it->beta_start = NULL;
	calc_beta(e->beta_start, it);
}

/* Per-detector results of the last maximize: u [num_rot_p] of detector k,
 * and rescale / mean_count of every detector. */
void ref_get_u_det(ref_engine *e, int k, double *o) {
	copy_or_zero(o, e->mdata->u != NULL ? e->mdata->u[k] : NULL, (size_t)e->quat.num_rot_p * sizeof(double));
}

void ref_get_det_scalars(ref_engine *e, double *rescale, double *mean_count) {
	memcpy(rescale, e->iter.rescale, (size_t)e->iter.num_det * sizeof(double));
	memcpy(mean_count, e->iter.mean_count, (size_t)e->iter.num_det * sizeof(double));
}

void ref_destroy(ref_engine *e) {
	if (e == NULL)
		return;
	free_common(e->mdata, e->iter.tot_num_data, e->iter.num_det);
	free(e->mdata);
	free(e->det.qvals); free(e->det.corr); free(e->det.raw_mask);
	free(e->dset.ones); free(e->dset.multi); free(e->dset.ones_accum); free(e->dset.multi_accum);
	free(e->dset.place_ones); free(e->dset.place_multi); free(e->dset.count_multi);
	free(e->quat.quats);
	free(e->mod.model1); free(e->mod.model2); free(e->mod.inter_weight);
	free(e->iter.fcounts); free(e->iter.mean_count); free(e->iter.rescale);
	free(e->iter.blacklist); free(e->iter.sum_fact); free(e->iter.scale);
	free(e->iter.beta); free(e->iter.beta_start);
	free(e->det.background); free(e->det.powder); free(e->iter.bgscale);
	ref_set_refinement(e, NULL, NULL, NULL);
	for (int k = 0; k < e->n_extra; ++k) {
		struct dataset *ds = e->extra[k];
		struct detector *dt = &e->dets[k + 1];
		free(ds->ones); free(ds->multi); free(ds->ones_accum); free(ds->multi_accum);
		free(ds->place_ones); free(ds->place_multi); free(ds->count_multi);
		free(ds);
		free(dt->qvals); free(dt->corr); free(dt->raw_mask);
	}
	free(e->extra);
	free(e->dets);
	free(e->det_map);
	free(e);
}

/* Background-aware model: per-pixel background (detector.pyx:100-104), per-frame
 * background scale (iterate.pyx:146-171, 311-312) and the powder sum that the
 * reference derives from the frames (calc_powder, iterate.c:119-177). With
 * need_scaling, maximize then takes the background-aware E-step, tomogram and
 * scale updates (max_prob.c:134-156, max_update.c:232-543, max_scale.c:21-288). */
void ref_set_background(ref_engine *e, const double *background, const double *bgscale) {
	free(e->det.background);
	free(e->iter.bgscale);
	e->det.background = dup_mem(background, (size_t)e->det.num_pix * sizeof(double));
	e->iter.bgscale = dup_mem(bgscale, (size_t)e->iter.tot_num_data * sizeof(double));
	e->det.with_bg = 1;
	calc_powder(&e->iter);
}

/* ---- accessors (copies; arrays that a call did not produce are zero-filled) ---- */

static void copy_or_zero(void *dst, const void *src, size_t bytes) {
	if (src != NULL)
		memcpy(dst, src, bytes);
	else
		memset(dst, 0, bytes);
}

long ref_model_len(ref_engine *e) { return e->mod.num_modes * e->mod.vol; }
void ref_get_powder(ref_engine *e, double *o) {
	copy_or_zero(o, e->det.powder, (size_t)e->det.num_pix * sizeof(double));
}
void ref_get_model1(ref_engine *e, double *o) { memcpy(o, e->mod.model1, ref_model_len(e) * sizeof(double)); }
void ref_set_model1(ref_engine *e, const double *i) { memcpy(e->mod.model1, i, ref_model_len(e) * sizeof(double)); }
void ref_get_model2(ref_engine *e, double *o) { memcpy(o, e->mod.model2, ref_model_len(e) * sizeof(double)); }
void ref_get_weight(ref_engine *e, double *o) { memcpy(o, e->mod.inter_weight, ref_model_len(e) * sizeof(double)); }

void ref_get_frame_arrays(ref_engine *e, int *rmax, double *info, double *likelihood, double *max_exp,
                          double *p_norm, double *psum_d) {
	size_t n = (size_t)e->iter.tot_num_data;
	struct max_data *c = e->mdata;
	copy_or_zero(rmax, c->rmax, n * sizeof(int));
	copy_or_zero(info, c->info, n * sizeof(double));
	copy_or_zero(likelihood, c->likelihood, n * sizeof(double));
	copy_or_zero(max_exp, c->max_exp, n * sizeof(double));
	copy_or_zero(p_norm, c->p_norm, n * sizeof(double));
	copy_or_zero(psum_d, c->psum_d, n * sizeof(double));
}

/* Model symmetries of update_model: point_group 1 = S4 (octahedral_flag),
 * 2 = A5 (icosahedral_flag), 0 = none; axial_order = params.axial_sym. */
void ref_set_symmetry(ref_engine *e, int point_group, int axial_order) {
	e->quat.octahedral_flag = point_group == 1;
	e->quat.icosahedral_flag = point_group == 2;
	e->par.axial_sym = axial_order > 1 ? axial_order : 1;
}

/* Asks the reference to form the combined per-frame probability lists (the
 * save_prob path of combine_information_omp, max_prob.c:294-325). */
void ref_set_save_prob(ref_engine *e, int on) { e->par.save_prob = on; }

/* Frame d's combined list after ref_maximize with save_prob: copies
 * num_prob[d] entries (orientation index, P) when the pointers are non-NULL
 * and returns the count (0 without lists). */
int ref_get_frame_prob(ref_engine *e, int d, int *place, double *prob) {
	struct max_data *c = e->mdata;
	if (c == NULL || c->num_prob == NULL || c->prob == NULL || c->prob[d] == NULL)
		return 0;
	int n = c->num_prob[d];
	if (place != NULL)
		memcpy(place, c->place_prob[d], (size_t)n * sizeof(int));
	if (prob != NULL)
		memcpy(prob, c->prob[d], (size_t)n * sizeof(double));
	return n;
}

void ref_get_quat_norm(ref_engine *e, double *o) {
	size_t n = (size_t)e->iter.tot_num_data * e->mod.num_modes;
	copy_or_zero(o, e->mod.num_modes > 1 ? e->mdata->quat_norm : NULL, n * sizeof(double));
}

void ref_get_u(ref_engine *e, double *o) {
	copy_or_zero(o, e->mdata->u != NULL ? e->mdata->u[0] : NULL, (size_t)e->quat.num_rot_p * sizeof(double));
}

void ref_get_iter_arrays(ref_engine *e, int *fcounts, double *sum_fact, double *scale, double *beta,
                         double *beta_start) {
	size_t n = (size_t)e->iter.tot_num_data;
	copy_or_zero(fcounts, e->iter.fcounts, n * sizeof(int));
	copy_or_zero(sum_fact, e->iter.sum_fact, n * sizeof(double));
	copy_or_zero(scale, e->iter.scale, n * sizeof(double));
	copy_or_zero(beta, e->iter.beta, n * sizeof(double));
	copy_or_zero(beta_start, e->iter.beta_start, n * sizeof(double));
}

void ref_set_scale(ref_engine *e, const double *scale) {
	if (e->iter.scale != NULL)
		memcpy(e->iter.scale, scale, (size_t)e->iter.tot_num_data * sizeof(double));
}

void ref_get_scalars(ref_engine *e, double *out) {
	out[0] = e->iter.rescale[0];
	out[1] = e->iter.mean_count[0];
	out[2] = e->iter.mutual_info;
	out[3] = e->avg_likelihood;
	out[4] = e->iter.rms_change;
}

void ref_set_rms(ref_engine *e, double rms) { e->iter.rms_change = rms; }

/* Model.slice_gen / slice_merge (model.pyx:105-151) on this engine's detector,
 * by model type: quat is a quaternion (3-D), an angle (2-D) or (phi, beta) (RZ). */
void ref_slice_gen(ref_engine *e, const double *quat, int mode, double *out) {
	if (e->mod.mtype == MODEL_2D)
		slice_gen2d((double *)quat, mode, out, &e->det, &e->mod);
	else if (e->mod.mtype == MODEL_RZ)
		slice_genrz((double *)quat, mode, out, &e->det, &e->mod);
	else
		slice_gen3d((double *)quat, mode, out, &e->det, &e->mod);
}

void ref_slice_merge(ref_engine *e, const double *quat, int mode, const double *view, double *model2,
                     double *weight) {
	if (e->mod.mtype == MODEL_2D)
		slice_merge2d((double *)quat, mode, (double *)view, model2, weight, e->mod.size, &e->det);
	else if (e->mod.mtype == MODEL_RZ)
		slice_mergerz((double *)quat, mode, (double *)view, model2, weight, e->mod.size, &e->det);
	else
		slice_merge3d((double *)quat, mode, (double *)view, model2, weight, e->mod.size, &e->det);
}

/* params.friedel_sym (2-D Friedel average in update_model) and the detector
 * distance detd that the RZ geometry uses (detector.pyx:50). */
void ref_set_friedel_detd(ref_engine *e, int friedel_sym, double detd) {
	e->par.friedel_sym = friedel_sym;
	e->det.detd = detd;
}

/* Quaternion.generate_3d (quaternion.pyx:94-102): count, and the list if out != NULL. */
int ref_quat_gen(int num_div, double *out) {
	struct quaternion q;
	int n;
	memset(&q, 0, sizeof(q));
	n = quat_gen(num_div, &q);
	if (out != NULL)
		memcpy(out, q.quats, (size_t)n * 5 * sizeof(double));
	free(q.quats);
	return n;
}

/* Coarse-to-fine refinement: params.refine with iterate.quat_mapping, rel_quat
 * and num_rel_quat filled as the legacy engine's setup does (src/iterate.c:
 * 103-130: quat_mapping from voronoi_subset, rel_quat per frame from the
 * coarse probabilities). The packaged engine consults them in max_prob.c:
 * 110-120, max_update.c:73-83 / 170-180 and max_scale.c:69-79; its Python
 * layer never fills them. quat_mapping == NULL switches refinement off. */
void ref_set_refinement(ref_engine *e, const int *quat_mapping, const long long *rel_off, const int *rel_quat) {
	int d, n = e->iter.tot_num_data;
	if (e->iter.rel_quat != NULL) {
		for (d = 0; d < n; ++d)
			free(e->iter.rel_quat[d]);
		free(e->iter.rel_quat);
	}
	free(e->iter.num_rel_quat);
	free(e->iter.quat_mapping);
	e->iter.rel_quat = NULL;
	e->iter.num_rel_quat = NULL;
	e->iter.quat_mapping = NULL;
	e->par.refine = 0;
	if (quat_mapping == NULL)
		return;
	e->iter.quat_mapping = dup_mem(quat_mapping, (size_t)e->quat.num_rot * sizeof(int));
	e->iter.num_rel_quat = malloc((size_t)(n > 0 ? n : 1) * sizeof(int));
	e->iter.rel_quat = malloc((size_t)(n > 0 ? n : 1) * sizeof(int *));
	for (d = 0; d < n; ++d) {
		e->iter.num_rel_quat[d] = (int)(rel_off[d + 1] - rel_off[d]);
		e->iter.rel_quat[d] = dup_mem(rel_quat + rel_off[d], (size_t)e->iter.num_rel_quat[d] * sizeof(int));
	}
	e->par.refine = 1;
}

/* Quaternion.voronoi_subset (quaternion.pyx:257-281): the nearest of the
 * num_div = coarse_div orientations for each of the fine ones. */
void ref_voronoi_subset(int coarse_div, int num_fine, const double *fine, int *nearest) {
	struct quaternion qc, qf;
	memset(&qc, 0, sizeof(qc));
	memset(&qf, 0, sizeof(qf));
	quat_gen(coarse_div, &qc);
	qf.num_rot = num_fine;
	qf.quats = (double *)fine;
	voronoi_subset(&qc, &qf, nearest);
	free(qc.quats);
}
