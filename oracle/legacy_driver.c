/* Driver of the reference's legacy EMC engine (src/max_emc.c with
 * src/interp.c, the `emc` binary's maximize()). TEST INFRASTRUCTURE ONLY: it
 * is compiled with the unmodified legacy sources into
 * _ref/libdragonfly_legacy_fast.so and timed as a CPU baseline beside the
 * packaged engine (dragonfly/src). Nothing in the product links it.
 *
 * The legacy engine keeps its state in globals (det, quat, frames, iter,
 * param: src/emc.h:15-19); leg_create fills them the way the legacy setup does
 * for one sparse dataset and one detector (src/setup_emc.c, src/iterate.c:
 * calc_mean_counts / calc_scale, src/dataset.c: parse_dataset's mean count
 * and calc_sum_fact with ln c! = lgamma(c + 1)), and leg_run_iteration runs
 * one iteration of src/recon_emc.c:102-131 (update_beta, maximize,
 * update_model with the Friedel average, normalize_scale). Only one engine
 * exists at a time (the globals). The output writers of src/output_emc.c
 * (metrics and probability files) are replaced by no-ops: the baseline
 * writes no files.
 */
#define EXTERN
#include "emc.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

void save_metrics(struct max_data *data) { (void)data; }
void save_prob(struct max_data *data) { (void)data; }

static struct detector g_det;
static struct rotation g_quat;
static struct dataset g_frames;
static struct iterate g_iter;
static struct params g_param;
static int g_live = 0;

static void *dup_bytes(const void *p, size_t n) {
	void *q = malloc(n > 0 ? n : 1);
	if (n > 0)
		memcpy(q, p, n);
	return q;
}

int leg_create(int num_pix, const double *qvals, const double *corr, const uint8_t *mask, int num_data,
               const int *ones, const int *multi, const int *place_ones, const int *place_multi,
               const int *count_multi, int num_rot, const double *quats, long size, const double *model1,
               int need_scaling, int update_scale, double beta, double beta_jump, int beta_period) {
	long t, d, ot = 0, mt = 0;
	if (g_live)
		return -1;
	memset(&g_det, 0, sizeof(g_det));
	memset(&g_quat, 0, sizeof(g_quat));
	memset(&g_frames, 0, sizeof(g_frames));
	memset(&g_iter, 0, sizeof(g_iter));
	memset(&g_param, 0, sizeof(g_param));

	/* detector: pixels as (qx, qy, qz, corr) (src/detector.c parse_detector) */
	g_det.num_pix = num_pix;
	g_det.pixels = malloc((size_t)num_pix * 4 * sizeof(double));
	g_det.mask = dup_bytes(mask, (size_t)num_pix);
	for (t = 0; t < num_pix; ++t) {
		g_det.pixels[4 * t] = qvals[3 * t];
		g_det.pixels[4 * t + 1] = qvals[3 * t + 1];
		g_det.pixels[4 * t + 2] = qvals[3 * t + 2];
		g_det.pixels[4 * t + 3] = corr[t];
		if (mask[t] < 1)
			g_det.rel_num_pix++;
	}
	g_det.num_det = 1;
	g_det.num_dfiles = 1;
	g_det.mapping[0] = 0;

	/* orientations: one rank, one mode (src/quat.c divide_quat) */
	g_quat.num_rot = num_rot;
	g_quat.num_rot_p = num_rot;
	g_quat.quat = dup_bytes(quats, (size_t)num_rot * 5 * sizeof(double));

	/* one sparse dataset */
	g_frames.type = 0;
	g_frames.num_data = num_data;
	g_frames.num_pix = num_pix;
	g_frames.num_data_prev = 0;
	g_frames.ones = dup_bytes(ones, (size_t)num_data * sizeof(int));
	g_frames.multi = dup_bytes(multi, (size_t)num_data * sizeof(int));
	g_frames.ones_accum = malloc((size_t)num_data * sizeof(long));
	g_frames.multi_accum = malloc((size_t)num_data * sizeof(long));
	for (d = 0; d < num_data; ++d) {
		g_frames.ones_accum[d] = ot;
		g_frames.multi_accum[d] = mt;
		ot += ones[d];
		mt += multi[d];
	}
	g_frames.ones_total = ot;
	g_frames.multi_total = mt;
	g_frames.place_ones = dup_bytes(place_ones, (size_t)ot * sizeof(int));
	g_frames.place_multi = dup_bytes(place_multi, (size_t)mt * sizeof(int));
	g_frames.count_multi = dup_bytes(count_multi, (size_t)mt * sizeof(int));
	g_frames.next = NULL;
	g_frames.tot_num_data = num_data;
	g_frames.num_blacklist = 0;
	g_frames.blacklist = calloc((size_t)num_data, 1);
	g_frames.count = calloc((size_t)num_data, sizeof(int));
	g_frames.sum_fact = calloc((size_t)num_data, sizeof(double));
	g_frames.mean_count = 0.;
	for (d = 0; d < num_data; ++d) {
		long a = g_frames.ones_accum[d], b = g_frames.multi_accum[d];
		for (t = 0; t < ones[d]; ++t)
			if (mask[place_ones[a + t]] < 1)
				g_frames.count[d]++;
		for (t = 0; t < multi[d]; ++t)
			if (mask[place_multi[b + t]] < 1) {
				g_frames.count[d] += count_multi[b + t];
				g_frames.sum_fact[d] += lgamma((double)count_multi[b + t] + 1.);
			}
		g_frames.mean_count += g_frames.count[d];
	}
	g_frames.mean_count /= num_data;
	g_frames.tot_mean_count = g_frames.mean_count;

	/* iterate */
	g_iter.size = size;
	g_iter.center = size / 2;
	g_iter.vol = size * size * size;
	g_iter.modes = 1;
	g_iter.tot_num_data = num_data;
	g_iter.model1 = dup_bytes(model1, (size_t)g_iter.vol * sizeof(double));
	g_iter.model2 = calloc((size_t)g_iter.vol, sizeof(double));
	g_iter.inter_weight = calloc((size_t)g_iter.vol, sizeof(double));
	g_iter.scale = malloc((size_t)num_data * sizeof(double));
	g_iter.bgscale = malloc((size_t)num_data * sizeof(double));
	for (d = 0; d < num_data; ++d)
		g_iter.scale[d] = g_iter.bgscale[d] = 1.;
	g_iter.rescale = calloc(1, sizeof(double));
	g_iter.mean_count = calloc(1, sizeof(double));
	g_iter.mean_count[0] = g_frames.mean_count;

	/* parameters */
	g_param.rank = 0;
	g_param.num_proc = 1;
	g_param.recon_type = RECON3D;
	g_param.need_scaling = need_scaling;
	g_param.update_scale = update_scale;
	g_param.known_scale = 0;
	g_param.beta_jump = beta_jump;
	g_param.beta_period = beta_period;
	g_param.beta_factor = 1.;
	g_param.modes = 1;
	g_param.nonrot_modes = 0;
	g_param.beta = malloc((size_t)num_data * sizeof(double));
	g_param.beta_start = malloc((size_t)num_data * sizeof(double));
	for (d = 0; d < num_data; ++d)
		g_param.beta_start[d] = beta;

	det = &g_det;
	quat = &g_quat;
	frames = &g_frames;
	iter = &g_iter;
	param = &g_param;
	slice_gen = slice_gen3d;
	slice_merge = slice_merge3d;
	g_live = 1;
	return 0;
}

/* One iteration as src/recon_emc.c:102-131 runs it: update_beta (:159-176),
 * maximize, update_model (:133-157, Friedel average, alpha = 0),
 * normalize_scale (src/iterate.c) when need_scaling. Returns the average
 * log-likelihood. */
double leg_run_iteration(int iteration) {
	long d, x;
	double factor, ll, change = 0.;
	if (!g_live)
		return 0.;
	param->iteration = iteration;
	factor = pow(param->beta_jump, (iteration - 1) / param->beta_period) * param->beta_factor;
	for (d = 0; d < frames->tot_num_data; ++d) {
		param->beta[d] = param->beta_start[d] * factor;
		if (param->beta[d] > 1.)
			param->beta[d] = 1.;
	}
	ll = maximize();
	for (x = 0; x < iter->vol; ++x)
		if (iter->inter_weight[x] > 0.)
			iter->model2[x] *= 1. / iter->inter_weight[x];
	symmetrize_friedel(iter->model2, iter->inter_weight, (int)iter->size);
	for (x = 0; x < iter->vol; ++x) {
		double diff = iter->model2[x] - iter->model1[x];
		change += diff * diff;
		iter->model1[x] = iter->model2[x];
	}
	iter->rms_change = sqrt(change / iter->vol);
	if (param->need_scaling) {
		double mean_scale = 0.;
		for (d = 0; d < iter->tot_num_data; ++d)
			mean_scale += iter->scale[d];
		mean_scale /= iter->tot_num_data;
		for (x = 0; x < iter->vol; ++x)
			iter->model1[x] *= mean_scale;
		for (d = 0; d < iter->tot_num_data; ++d)
			iter->scale[d] /= mean_scale;
		iter->rms_change *= mean_scale;
	}
	return ll;
}

void leg_get_model1(double *out) {
	if (g_live)
		memcpy(out, iter->model1, (size_t)iter->vol * sizeof(double));
}

void leg_set_scale(const double *scale) {
	if (g_live)
		memcpy(iter->scale, scale, (size_t)iter->tot_num_data * sizeof(double));
}

void leg_destroy(void) {
	if (!g_live)
		return;
	free(g_det.pixels);
	free(g_det.mask);
	free(g_quat.quat);
	free(g_frames.ones);
	free(g_frames.multi);
	free(g_frames.ones_accum);
	free(g_frames.multi_accum);
	free(g_frames.place_ones);
	free(g_frames.place_multi);
	free(g_frames.count_multi);
	free(g_frames.blacklist);
	free(g_frames.count);
	free(g_frames.sum_fact);
	free(g_iter.model1);
	free(g_iter.model2);
	free(g_iter.inter_weight);
	free(g_iter.scale);
	free(g_iter.bgscale);
	free(g_iter.rescale);
	free(g_iter.mean_count);
	free(g_param.beta);
	free(g_param.beta_start);
	g_live = 0;
}
