/* CPU oracle for one EMC iteration. TEST INFRASTRUCTURE ONLY (see emc_oracle.h).
 *
 * Written from the algorithm of duaneloh/Dragonfly's packaged engine; each
 * function names the reference lines it restates. The data structures are our
 * own (flat arrays instead of the reference's linked dataset list and per-thread
 * max_data), but arithmetic follows the reference's operation order so that a
 * build without FMA contraction is bit-identical to the one-thread reference.
 */
#include "emc_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PROB_MIN 1.e-6         /* max_internal.h:6 */
#define ORC_PDIFF_THRESH 14.       /* max_internal.h:7 */
#define ORC_MAX_EXP_START -1.e100  /* max_internal.h:8 */

void orc_make_rot_quat(const double *q, double rot[3][3]) {
	/* model.c:759-786 */
	double q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3];
	double q01 = q0 * q1, q02 = q0 * q2, q03 = q0 * q3;
	double q11 = q1 * q1, q12 = q1 * q2, q13 = q1 * q3;
	double q22 = q2 * q2, q23 = q2 * q3, q33 = q3 * q3;
	rot[0][0] = (1. - 2. * (q22 + q33));
	rot[0][1] = 2. * (q12 + q03);
	rot[0][2] = 2. * (q13 - q02);
	rot[1][0] = 2. * (q12 - q03);
	rot[1][1] = (1. - 2. * (q11 + q33));
	rot[1][2] = 2. * (q01 + q23);
	rot[2][0] = 2. * (q02 + q13);
	rot[2][1] = 2. * (q23 - q01);
	rot[2][2] = (1. - 2. * (q11 + q22));
}

/* Rotated voxel position of pixel t: sum_j rot[i][j] q_j, then + center,
 * accumulated from 0 in j order (model.c:19-25). */
static void rotate_pixel(double rot[3][3], const double *qv, double center, double pos[3]) {
	int i, j;
	for (i = 0; i < 3; ++i) {
		double acc = 0.;
		for (j = 0; j < 3; ++j)
			acc += rot[i][j] * qv[j];
		acc += center;
		pos[i] = acc;
	}
}

void orc_slice_gen3d(const double *quat, int mode, double *slice, int num_pix, const double *qvals,
                     const double *corr, long size, long center, const double *model1) {
	/* model.c:11-59 */
	long t, x, y, z, vol = size * size * size;
	double rot[3][3], pos[3], fx, fy, fz, cx, cy, cz;
	const double *m = &model1[(long)mode * vol];
	orc_make_rot_quat(quat, rot);
	for (t = 0; t < num_pix; ++t) {
		rotate_pixel(rot, &qvals[t * 3], (double)center, pos);
		x = (long)pos[0];  /* truncation toward zero, as the reference's assignment */
		y = (long)pos[1];
		z = (long)pos[2];
		if (x < 0 || x > size - 2 || y < 0 || y > size - 2 || z < 0 || z > size - 2) {
			slice[t] = DBL_MIN;
			continue;
		}
		fx = pos[0] - x; fy = pos[1] - y; fz = pos[2] - z;
		cx = 1. - fx; cy = 1. - fy; cz = 1. - fz;
		{
			long x1 = (x + 1) % size, y1 = (y + 1) % size, z1 = (z + 1) % size;
			long s2 = size * size;
			double v = cx * cy * cz * m[x * s2 + y * size + z] +
			           cx * cy * fz * m[x * s2 + y * size + z1] +
			           cx * fy * cz * m[x * s2 + y1 * size + z] +
			           cx * fy * fz * m[x * s2 + y1 * size + z1] +
			           fx * cy * cz * m[x1 * s2 + y * size + z] +
			           fx * cy * fz * m[x1 * s2 + y * size + z1] +
			           fx * fy * cz * m[x1 * s2 + y1 * size + z] +
			           fx * fy * fz * m[x1 * s2 + y1 * size + z1];
			slice[t] = v * corr[t];
		}
	}
}

void orc_slice_merge3d(const double *quat, int mode, const double *slice, double *model2, double *weight,
                       long size, int num_pix, const double *qvals, const double *corr, const uint8_t *mask) {
	/* model.c:171-244 */
	long t, x, y, z, vol = size * size * size, s2 = size * size;
	double rot[3][3], pos[3], fx, fy, fz, cx, cy, cz, w, f;
	double *m = &model2[(long)mode * vol], *wt = &weight[(long)mode * vol];
	orc_make_rot_quat(quat, rot);
	for (t = 0; t < num_pix; ++t) {
		if (mask[t] > 1)
			continue;
		rotate_pixel(rot, &qvals[t * 3], (double)(size / 2), pos);
		x = (long)pos[0];
		y = (long)pos[1];
		z = (long)pos[2];
		if (x < 0 || x > size - 2 || y < 0 || y > size - 2 || z < 0 || z > size - 2)
			continue;
		fx = pos[0] - x; fy = pos[1] - y; fz = pos[2] - z;
		cx = 1. - fx; cy = 1. - fy; cz = 1. - fz;
		w = slice[t] / corr[t];
		{
			long x1 = (x + 1) % size, y1 = (y + 1) % size, z1 = (z + 1) % size;
			long idx[8] = {x * s2 + y * size + z, x * s2 + y * size + z1, x * s2 + y1 * size + z,
			               x * s2 + y1 * size + z1, x1 * s2 + y * size + z, x1 * s2 + y * size + z1,
			               x1 * s2 + y1 * size + z, x1 * s2 + y1 * size + z1};
			double fw[8] = {cx * cy * cz, cx * cy * fz, cx * fy * cz, cx * fy * fz,
			                fx * cy * cz, fx * cy * fz, fx * fy * cz, fx * fy * fz};
			int k;
			for (k = 0; k < 8; ++k) {
				f = fw[k];
				wt[idx[k]] += f;
				m[idx[k]] += f * w;
			}
		}
	}
}

void orc_symmetrize_friedel(double *array, const double *weights, int size) {
	/* model.c:470-490: visits z <= center, so pairs inside the z == center plane
	 * are averaged twice, the second time from the other member of the pair. */
	int x, y, z, v1, v2, lo = (size % 2 == 0) ? 1 : 0, c = size / 2;
	double a, wsum;
	for (x = lo; x < size; ++x)
		for (y = lo; y < size; ++y)
			for (z = lo; z <= c; ++z) {
				v1 = x * size * size + y * size + z;
				v2 = (2 * c - x) * size * size + (2 * c - y) * size + (2 * c - z);
				a = 0.5 * (array[v1] * weights[v1] + array[v2] * weights[v2]);
				wsum = 0.5 * (weights[v1] + weights[v2]);
				a = (wsum > 0) ? a / wsum : 0.;
				array[v1] = a;
				array[v2] = a;
			}
}

void orc_frame_stats(int num_data, const int *ones, const int *multi, const int *place_ones,
                     const int *place_multi, const int *count_multi, const uint8_t *mask,
                     int *fcounts, double *sum_fact, double *mean_count) {
	/* iterate.c:3-64 (calc_frame_counts) and 85-117 (calc_sum_fact) */
	long d, t, o = 0, mo = 0;
	double mc = 0.;
	for (d = 0; d < num_data; ++d) {
		int fc = 0;
		double sf = 0.;
		for (t = 0; t < ones[d]; ++t)
			if (mask[place_ones[o + t]] < 1)
				fc++;
		for (t = 0; t < multi[d]; ++t)
			if (mask[place_multi[mo + t]] < 1) {
				fc += count_multi[mo + t];
				sf += lgamma((double)count_multi[mo + t] + 1.0);
			}
		fcounts[d] = fc;
		sum_fact[d] = sf;
		mc += fc;
		o += ones[d];
		mo += multi[d];
	}
	*mean_count = mc / num_data;
}

void orc_calc_beta(int num_data, double start, int need_scaling, double mean_count, const int *fcounts,
                   double *beta_start) {
	/* iterate.c:66-83 */
	int d;
	if (!need_scaling && start < 0)
		start = exp(-6.5 * pow(mean_count * 1.e-5, 0.15));
	for (d = 0; d < num_data; ++d)
		beta_start[d] = start > 0 ? start : exp(-6.5 * pow(fcounts[d] * 1.e-5, 0.15));
}

/* Per-frame list of kept (orientation, log-probability) pairs, in the order
 * the orientations were visited (max_prob.c:184-203, resparsify 429-448).
 * Orientations are visited in ascending order, so each list stays sorted by
 * orientation and can be searched by bisection. */
typedef struct {
	int n, cap;
	int *pos;
	double *val;
} kept_list;

static void list_push(kept_list *l, int r, double v) {
	if (l->n == l->cap) {
		l->cap = l->cap ? 2 * l->cap : 8;
		l->pos = realloc(l->pos, (size_t)l->cap * sizeof(int));
		l->val = realloc(l->val, (size_t)l->cap * sizeof(double));
	}
	l->pos[l->n] = r;
	l->val[l->n] = v;
	l->n++;
}

/* Drops entries <= thresh, keeping order (max_prob.c:429-448). */
static void list_prune(kept_list *l, double thresh) {
	int i, k = 0;
	for (i = 0; i < l->n; ++i)
		if (!(l->val[i] <= thresh)) {
			l->pos[k] = l->pos[i];
			l->val[k] = l->val[i];
			k++;
		}
	l->n = k;
}

/* Index of orientation r in the sorted list, or -1 (the lookup that
 * max_update.c:86-93 does by linear search). */
static int list_find(const kept_list *l, int r) {
	int lo = 0, hi = l->n - 1;
	while (lo <= hi) {
		int mid = (lo + hi) / 2;
		if (l->pos[mid] == r)
			return mid;
		if (l->pos[mid] < r)
			lo = mid + 1;
		else
			hi = mid - 1;
	}
	return -1;
}

/* Probability lists of the last orc_maximize call, kept when g_keep_prob is
 * set (the save_prob path of max_prob.c:294-325 needs the same lists). */
static int g_keep_prob = 0;
static kept_list *g_kept = NULL;
static int g_kept_n = 0;

static void orc_free_kept(void) {
	int d;
	for (d = 0; d < g_kept_n; ++d) {
		free(g_kept[d].pos);
		free(g_kept[d].val);
	}
	free(g_kept);
	g_kept = NULL;
	g_kept_n = 0;
}

void orc_set_keep_prob(int on) {
	g_keep_prob = on != 0;
	if (!g_keep_prob)
		orc_free_kept();
}

int orc_kept_prob(int d, int *pos, double *val) {
	const kept_list *l;
	if (g_kept == NULL || d < 0 || d >= g_kept_n)
		return -1;
	l = &g_kept[d];
	if (pos != NULL)
		memcpy(pos, l->pos, (size_t)l->n * sizeof(int));
	if (val != NULL)
		memcpy(val, l->val, (size_t)l->n * sizeof(double));
	return l->n;
}

/* Orientations are processed in blocks whose slices fit in this many doubles. */
#define ORC_BLOCK_DOUBLES (1L << 27)

/* Geometry of one (orientation, pixel) term of the merge: base voxel index
 * (mode * vol + x * size^2 + y * size + z; -1 when the pixel is skipped),
 * fractional offsets and the merged value slice / corr. */
typedef struct {
	long base;
	double fx, fy, fz, w;
} merge_rec;

/* Orientations per sub-block of the parallel merge. */
#define ORC_MERGE_SUB 64

/* Scratch of merge_block: per (orientation, detector, pixel) geometry, and
 * per (orientation, detector, grid plane) the pixels with corners on that
 * plane. */
typedef struct {
	merge_rec *rec;     /* [ORC_MERGE_SUB][num_det][max_pix] */
	int *idx;           /* [ORC_MERGE_SUB][num_det][2 * max_pix] */
	long *off;          /* [ORC_MERGE_SUB][num_det][planes + 1] */
	double *acc;        /* [M * V][2]: weight, model2 */
	long planes;        /* M * size */
	int num_det, max_pix;
} merge_scratch;

/* One detector of a maximize call: its geometry and, per block of
 * orientations, its slices. */
typedef struct {
	int num_pix;
	const double *qvals, *corr;
	const uint8_t *mask;
	double *views;      /* [blk][num_pix] */
} det_view;

/* slice_merge3d (model.c:171-244) for orientations r0 .. r1-1 in ascending
 * order and, per orientation, the detectors in ascending order, as the
 * sequential loop of merge_tomogram (max_update.c:18-40) does. The additions
 * to every voxel happen in the order of that loop (orientation, detector,
 * pixel, corner), so the sums are bit-identical to it at any thread count:
 * the geometry of each (orientation, detector, pixel) is computed in parallel
 * over orientations and listed under the two grid planes (mode * size + x and
 * x + 1) its corners lie on; then the planes are shared out among the threads
 * and each walks its planes' lists in orientation, detector and pixel order.
 * A detector merges an orientation only where its psum_r is positive
 * (max_update.c:34-36). The sums go to acc, (weight, model2) interleaved per
 * voxel so that one cache line holds both. */
static void merge_block(int r0, int r1, int M, int R, const double *quats, const double *psum_r,
                        const det_view *dv, double *acc, long size, merge_scratch *ms) {
	const long vol = size * size * size, s2 = size * size;
	const long planes = ms->planes;
	const int K = ms->num_det, P = ms->max_pix;
	int s0;
	for (s0 = r0; s0 < r1; s0 += ORC_MERGE_SUB) {
		const int s1 = s0 + ORC_MERGE_SUB < r1 ? s0 + ORC_MERGE_SUB : r1;
		int r;
		long j;
		#pragma omp parallel for schedule(dynamic, 1)
		for (r = s0; r < s1; ++r) {
			int k;
			double rot[3][3];
			orc_make_rot_quat(&quats[(r / M) * 5], rot);
			for (k = 0; k < K; ++k) {
				const long set = (long)(r - s0) * K + k;
				merge_rec *out = &ms->rec[set * P];
				int *idx = &ms->idx[set * 2 * P];
				long *off = &ms->off[set * (planes + 1)];
				const det_view *v = &dv[k];
				const double *slice = &v->views[(long)(r - r0) * v->num_pix];
				double pos[3];
				long t, x, y, z, p;
				for (p = 0; p <= planes; ++p)
					off[p] = 0;
				if (!(psum_r[(long)k * R + r] > 0.))
					continue;
				for (t = 0; t < v->num_pix; ++t) {
					long pl;
					out[t].base = -1;
					if (v->mask[t] > 1)
						continue;
					rotate_pixel(rot, &v->qvals[t * 3], (double)(size / 2), pos);
					x = (long)pos[0];
					y = (long)pos[1];
					z = (long)pos[2];
					if (x < 0 || x > size - 2 || y < 0 || y > size - 2 || z < 0 || z > size - 2)
						continue;
					out[t].base = (long)(r % M) * vol + x * s2 + y * size + z;
					out[t].fx = pos[0] - x;
					out[t].fy = pos[1] - y;
					out[t].fz = pos[2] - z;
					out[t].w = slice[t] / v->corr[t];
					/* corners 0-3 lie on plane pl, 4-7 on pl + 1 (x + 1 <= size - 1) */
					pl = (long)(r % M) * size + x;
					off[pl + 1]++;
					off[pl + 2]++;
				}
				for (p = 0; p < planes; ++p)
					off[p + 1] += off[p];
				for (t = 0; t < v->num_pix; ++t) {
					long pl;
					if (out[t].base < 0)
						continue;
					pl = out[t].base / s2;
					idx[off[pl]++] = (int)t;
					idx[off[pl + 1]++] = (int)t;
				}
				/* the fill advanced each start to the next plane's: shift back */
				for (p = planes; p > 0; --p)
					off[p] = off[p - 1];
				off[0] = 0;
			}
		}
		#pragma omp parallel for schedule(dynamic, 1)
		for (j = 0; j < planes; ++j) {
			int rr, k;
			for (rr = s0; rr < s1; ++rr)
				for (k = 0; k < K; ++k) {
					const long set = (long)(rr - s0) * K + k;
					const merge_rec *rec = &ms->rec[set * P];
					const int *idx = &ms->idx[set * 2 * P];
					const long *off = &ms->off[set * (planes + 1)];
					long i;
					int c;
					for (i = off[j]; i < off[j + 1]; ++i) {
						const merge_rec *e = &rec[idx[i]];
						const long b = e->base;
						const int upper = b / s2 != j;     /* j is the plane of corners 4-7 */
						const double fx = e->fx, fy = e->fy, fz = e->fz, w = e->w;
						const double cx = 1. - fx, cy = 1. - fy, cz = 1. - fz;
						const long id[8] = {b, b + 1, b + size, b + size + 1,
						                    b + s2, b + s2 + 1, b + s2 + size, b + s2 + size + 1};
						const double fw[8] = {cx * cy * cz, cx * cy * fz, cx * fy * cz, cx * fy * fz,
						                      fx * cy * cz, fx * cy * fz, fx * fy * cz, fx * fy * fz};
						for (c = upper ? 4 : 0; c < (upper ? 8 : 4); ++c) {
							acc[2 * id[c]] += fw[c];
							acc[2 * id[c] + 1] += fw[c] * w;
						}
					}
				}
		}
	}
}

/* The reference visits orientations in an outer loop and frames in an inner
 * loop. Every quantity it accumulates is either per frame (summed over
 * orientations in ascending order) or per orientation (summed over frames in
 * ascending order); this restatement keeps each of those orders and
 * parallelises only across independent frames or orientations, so its results
 * do not depend on the thread count. The merge into model2 adds to every voxel
 * in orientation order, as with one reference thread (merge_block).
 *
 * Several detectors (Iterate with in_detector_list, iterate.pyx:432-456):
 * frame d is seen by detector det_of[d]; u, the rescale factor, psum_r and
 * the tomograms are per detector (max_prob.c:31-42, 56-60; max_update.c:
 * 55-128, 153-229) and every frame's likelihood uses its own detector's
 * slice, u and rescale (max_prob.c:96-106, 122-127). */
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
                         double *scalars_out) {
	const int M = num_modes, R = num_modes * num_rot, K = num_det;
	const long vol = size * size * size, center = size / 2;
	long *ones_off = malloc((size_t)(num_data + 1) * sizeof(long));
	long *multi_off = malloc((size_t)(num_data + 1) * sizeof(long));
	long blk, tot_pix = 0;
	det_view *dv = calloc((size_t)K, sizeof(det_view));
	merge_scratch ms;
	kept_list *lists = calloc((size_t)num_data, sizeof(kept_list));
	double avg_ll = 0., mutual_info = 0.;
	const int use_scale = need_scaling && (iteration > 1 || known_scale);
	int d, r, r0, k;

	ms.max_pix = 1;
	for (k = 0; k < K; ++k) {
		dv[k].num_pix = num_pix[k];
		dv[k].qvals = qvals[k];
		dv[k].corr = corr[k];
		dv[k].mask = mask[k];
		tot_pix += num_pix[k];
		if (num_pix[k] > ms.max_pix)
			ms.max_pix = num_pix[k];
	}
	blk = ORC_BLOCK_DOUBLES / (tot_pix > 0 ? tot_pix : 1);
	if (blk < 1)
		blk = 1;
	if (blk > R)
		blk = R;
	for (k = 0; k < K; ++k)
		dv[k].views = malloc((size_t)blk * (num_pix[k] > 0 ? num_pix[k] : 1) * sizeof(double));
	ms.num_det = K;
	ms.planes = (long)M * size;
	ms.rec = malloc((size_t)ORC_MERGE_SUB * K * ms.max_pix * sizeof(merge_rec));
	ms.idx = malloc((size_t)ORC_MERGE_SUB * K * 2 * ms.max_pix * sizeof(int));
	ms.off = malloc((size_t)ORC_MERGE_SUB * K * (ms.planes + 1) * sizeof(long));
	ms.acc = calloc((size_t)2 * M * vol, sizeof(double));
	ones_off[0] = multi_off[0] = 0;
	for (d = 0; d < num_data; ++d) {
		ones_off[d + 1] = ones_off[d] + ones[d];
		multi_off[d + 1] = multi_off[d] + multi[d];
	}
	memset(model2, 0, (size_t)M * vol * sizeof(double));
	memset(weight, 0, (size_t)M * vol * sizeof(double));
	for (d = 0; d < num_data; ++d) {
		rmax[d] = 0;
		info[d] = likelihood[d] = p_norm[d] = psum_d[d] = 0.;
		max_exp[d] = ORC_MAX_EXP_START;
	}
	if (M > 1)
		memset(quat_norm, 0, (size_t)num_data * M * sizeof(double));

	/* Orientation index r -> (rotation, mode) (max_prob.c:80-85 for one rank) */
#define ROTIND(r) ((r) / M)
#define MODE(r) ((r) % M)

	/* calculate_rescale (max_prob.c:3-64): u_r = sum of W over mask==0 pixels,
	 * per detector */
	#pragma omp parallel for schedule(dynamic, 4)
	for (r = 0; r < R; ++r) {
		int t, kk;
		for (kk = 0; kk < K; ++kk) {
			double *view = malloc((size_t)(num_pix[kk] > 0 ? num_pix[kk] : 1) * sizeof(double)), acc = 0.;
			orc_slice_gen3d(&quats[ROTIND(r) * 5], MODE(r), view, num_pix[kk], qvals[kk], corr[kk], size, center,
			                model1);
			for (t = 0; t < num_pix[kk]; ++t)
				if (mask[kk][t] < 1)
					acc += view[t];
			u[(long)kk * R + r] = acc;
			free(view);
		}
	}
	for (k = 0; k < K; ++k) {
		double total = 0.;
		for (r = 0; r < R; ++r)
			total += quats[ROTIND(r) * 5 + 4] * u[(long)k * R + r];
		rescale[k] = mean_count[k] / total * M;
	}

	/* calculate_prob (max_prob.c:66-213): per frame, orientations in order */
	for (r0 = 0; r0 < R; r0 += (int)blk) {
		int r1 = r0 + (int)blk < R ? r0 + (int)blk : R;
		#pragma omp parallel for schedule(dynamic, 1)
		for (r = r0; r < r1; ++r) {
			int t, kk;
			for (kk = 0; kk < K; ++kk) {
				double *view = &dv[kk].views[(long)(r - r0) * num_pix[kk]];
				orc_slice_gen3d(&quats[ROTIND(r) * 5], MODE(r), view, num_pix[kk], qvals[kk], corr[kk], size,
				                center, model1);
				for (t = 0; t < num_pix[kk]; ++t)
					view[t] = log(view[t]);
			}
		}
		#pragma omp parallel for schedule(dynamic, 16)
		for (d = 0; d < num_data; ++d) {
			int rr;
			long i;
			const int kd = det_of[d];
			const uint8_t *mk = mask[kd];
			if (blacklist[d])
				continue;
			for (rr = r0; rr < r1; ++rr) {
				const double *view = &dv[kd].views[(long)(rr - r0) * num_pix[kd]];
				const double w = quats[ROTIND(rr) * 5 + 4];
				double pval, thr;
				if (use_scale)
					pval = log(w) - u[(long)kd * R + rr] * scale[d];
				else
					pval = log(w) - u[(long)kd * R + rr] * rescale[kd];
				for (i = ones_off[d]; i < ones_off[d + 1]; ++i)
					if (mk[place_ones[i]] < 1)
						pval += view[place_ones[i]];
				for (i = multi_off[d]; i < multi_off[d + 1]; ++i)
					if (mk[place_multi[i]] < 1)
						pval += count_multi[i] * view[place_multi[i]];
				thr = ORC_PDIFF_THRESH / beta[d];
				if (pval + thr > max_exp[d])
					list_push(&lists[d], rr, pval);
				if (pval > max_exp[d]) {
					max_exp[d] = pval;
					rmax[d] = rr;
					list_prune(&lists[d], pval - thr);
				}
			}
		}
	}

	/* normalize_prob (max_prob.c:215-265) and the per-frame half of calc_psum_r
	 * (max_update.c:95-130): P, likelihood, psum_d, quat_norm, info, each summed
	 * over the frame's kept orientations in ascending order. */
	#pragma omp parallel for schedule(dynamic, 16)
	for (d = 0; d < num_data; ++d) {
		int kk;
		double s = 0.;
		kept_list *l = &lists[d];
		const int kd = det_of[d];
		if (max_exp[d] == ORC_MAX_EXP_START)
			rmax[d] = -1;
		for (kk = 0; kk < l->n; ++kk)
			s += exp(beta[d] * (l->val[kk] - max_exp[d]));
		p_norm[d] = s;
		if (blacklist[d])
			continue;
		for (kk = 0; kk < l->n; ++kk) {
			const int rr = l->pos[kk];
			const double w = quats[ROTIND(rr) * 5 + 4];
			double temp = l->val[kk];
			double P = exp(beta[d] * (temp - max_exp[d])) / p_norm[d];
			l->val[kk] = P;
			likelihood[d] += P * (temp - sum_fact[d]);
			if (need_scaling && update_scale)
				psum_d[d] += P * u[(long)kd * R + rr] * rescale[kd];
			if (P < ORC_PROB_MIN)
				continue;
			if (M > 1)
				quat_norm[d * M + MODE(rr)] += P;
			info[d] += P * log(P / w * M);
		}
	}

	/* Per-orientation half of calc_psum_r (max_update.c:108-116), then
	 * update_tomogram_nobg (max_update.c:142-230) and merge_tomogram
	 * (max_update.c:18-40), block by block; merges run in orientation order. */
	for (r0 = 0; r0 < R; r0 += (int)blk) {
		int r1 = r0 + (int)blk < R ? r0 + (int)blk : R;
		#pragma omp parallel for schedule(dynamic, 1)
		for (r = r0; r < r1; ++r) {
			int dd, t, kk;
			long i;
			for (kk = 0; kk < K; ++kk)
				psum_r[(long)kk * R + r] = 0.;
			for (dd = 0; dd < num_data; ++dd) {
				int ind;
				if (blacklist[dd])
					continue;
				ind = list_find(&lists[dd], r);
				if (ind < 0)
					continue;
				psum_r[(long)det_of[dd] * R + r] += need_scaling ? lists[dd].val[ind] * scale[dd]
				                                                 : lists[dd].val[ind];
			}
			for (kk = 0; kk < K; ++kk)
				memset(&dv[kk].views[(long)(r - r0) * num_pix[kk]], 0, (size_t)num_pix[kk] * sizeof(double));
			for (dd = 0; dd < num_data; ++dd) {
				int ind;
				double P;
				const int kd = det_of[dd];
				const uint8_t *mk = mask[kd];
				double *view = &dv[kd].views[(long)(r - r0) * num_pix[kd]];
				if (blacklist[dd])
					continue;
				ind = list_find(&lists[dd], r);
				if (ind < 0)
					continue;
				P = lists[dd].val[ind];
				if (!(P > ORC_PROB_MIN))
					continue;
				for (i = ones_off[dd]; i < ones_off[dd + 1]; ++i)
					if (mk[place_ones[i]] < 2)
						view[place_ones[i]] += P;
				for (i = multi_off[dd]; i < multi_off[dd + 1]; ++i)
					if (mk[place_multi[i]] < 2)
						view[place_multi[i]] += count_multi[i] * P;
			}
			for (kk = 0; kk < K; ++kk) {
				const double pr = psum_r[(long)kk * R + r];
				double *view = &dv[kk].views[(long)(r - r0) * num_pix[kk]];
				if (pr > 0.)
					for (t = 0; t < num_pix[kk]; ++t)
						view[t] /= pr;
			}
		}
		merge_block(r0, r1, M, R, quats, psum_r, dv, ms.acc, size, &ms);
	}

	for (r0 = 0; r0 < M; ++r0) {
		long x;
		for (x = r0 * vol; x < (r0 + 1) * vol; ++x) {
			weight[x] = ms.acc[2 * x];
			model2[x] = ms.acc[2 * x + 1];
		}
	}

	/* combine_information_mpi (max_prob.c:344-427). The packaged Iterate never
	 * sets num_blacklist (iterate.pyx:35, 317-359), so averages divide by N. */
	for (d = 0; d < num_data; ++d)
		if (!blacklist[d]) {
			mutual_info += info[d];
			avg_ll += likelihood[d];
		}
	mutual_info /= num_data;
	avg_ll /= num_data;

	/* update_scale (max_scale.c:3-19) */
	if (need_scaling && update_scale)
		for (d = 0; d < num_data; ++d)
			if (!blacklist[d])
				scale[d] = fcounts[d] / psum_d[d];

	if (num_prob != NULL)
		for (d = 0; d < num_data; ++d)
			num_prob[d] = lists[d].n;
	scalars_out[0] = mutual_info;
	scalars_out[1] = avg_ll;

	if (g_keep_prob) {      /* retained for orc_kept_prob until the next call */
		orc_free_kept();
		g_kept = lists;
		g_kept_n = num_data;
	}
	else {
		for (d = 0; d < num_data; ++d) {
			free(lists[d].pos);
			free(lists[d].val);
		}
		free(lists);
	}
	for (k = 0; k < K; ++k)
		free(dv[k].views);
	free(dv);
	free(ms.rec);
	free(ms.idx);
	free(ms.off);
	free(ms.acc);
	free(ones_off);
	free(multi_off);
#undef ROTIND
#undef MODE
	return avg_ll;
}

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
                    double *psum_d, double *quat_norm, int *num_prob, double *scalars_out) {
	/* one detector: every frame is detector 0's */
	int *det_of = calloc((size_t)(num_data > 0 ? num_data : 1), sizeof(int));
	double sc[2], avg;
	avg = orc_maximize_dets(1, &num_pix, &qvals, &corr, &mask, det_of, num_data, ones, multi, place_ones,
	                        place_multi, count_multi, num_rot, num_modes, quats, size, model1, scale, beta,
	                        sum_fact, fcounts, blacklist, &mean_count, need_scaling, update_scale, known_scale,
	                        iteration, model2, weight, u, psum_r, rmax, info, likelihood, max_exp, p_norm,
	                        psum_d, quat_norm, num_prob, &scalars_out[0], sc);
	scalars_out[1] = sc[0];
	scalars_out[2] = sc[1];
	free(det_of);
	return avg;
}

double orc_update_model(long size, int num_modes, double *model1, double *model2, double *weight,
                        double alpha) {
	/* recon.pyx:112-149, RECON3D branch with Friedel symmetry (recon.pyx:128-130) */
	long x, vol = size * size * size, n = vol * num_modes;
	double diff, change = 0.;
	for (x = 0; x < num_modes; ++x)
		orc_symmetrize_friedel(&model2[x * vol], &weight[x * vol], (int)size);
	for (x = 0; x < n; ++x)
		if (weight[x] > 0.)
			model2[x] /= weight[x];
	for (x = 0; x < n; ++x) {
		diff = model2[x] - model1[x];
		change += diff * diff;
		if (alpha > 0.)
			model1[x] = alpha * model1[x] + (1 - alpha) * model2[x];
		else
			model1[x] = model2[x];
	}
	return sqrt(change / num_modes / vol);
}
