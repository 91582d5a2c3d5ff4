// Pair lists for restricted searches (refinement, learned proposals).
//
// A restricted search evaluates, per frame, only the orientation tiles that
// hold an orientation of one of the frame's relevant coarse cells. The pair
// layout stores just those (tile, frame) pairs, tile-major: pair q has tile
// pair_tile[q] and frame pair_frame[q], the pairs of tile t are
// [tile_off[t], tile_off[t + 1]) in ascending frame order, and frame d lists
// its pairs in ascending tile order in frame_pair[frame_off[d] ..]. Per pair:
// the FP64 photon sums of the tile's 128 orientations (raw, 1 KB) and their
// FP32 probabilities (Pq, sign = PROB_MIN gate as Pst), which the
// normalisation writes over the first half of the same row once it has read
// it (so a pair costs 1 KB, not 1.5). With the orientations split
// into blocks of whole tiles, one block-sized buffer holds the block's
// log-slices during the E-step and its tomograms during the M-step, so the
// full log-slice and tomogram arrays (4 B x R x P each) are never resident.
//
// Results equal the dense restricted path (estep_kernel<true> +
// norm_kernel<., true>): the log-likelihood of a pair is the same FP64
// expression, formed in the normalisation instead of the E-step (so the
// E-step needs neither u_r nor the rescale factor, which need every block's
// slices), and each lane adds its kept pairs in the same order. The tomograms
// are scattered with FP32 atomics (order-dependent rounding, about 1e-7
// relative) instead of the dense path's compensated gathers.
#pragma once

#include "emc_device.cuh"

namespace dfg {

// floats from one pair's probabilities to the next: they live in the first
// half of the pair's FP64 row of raw
constexpr int PQ_STRIDE = 2 * TILE;

// Photon sums of the 4 (LW) orientations of one lane over one frame's E-step
// lists (the loop of estep_kernel): compensated FP32, formed in FP64.
__device__ __forceinline__ void pair_photon_sums(const float *__restrict__ L, const uint32_t *__restrict__ ph,
                                                 long long beg, long long mid, long long end, int P,
                                                 double (&out)[LW]) {
	const uint4 *w4 = reinterpret_cast<const uint4 *>(ph);
	float s[ECH][LW], c[ECH][LW];
#pragma unroll
	for (int h = 0; h < ECH; ++h)
#pragma unroll
		for (int k = 0; k < LW; ++k)
			s[h][k] = c[h][k] = 0.f;
	uint4 a = make_uint4(P, P, P, P), b = a;
	if (beg < mid) {
		a = __ldg(w4 + (beg >> 2));
		b = __ldg(w4 + (beg >> 2) + 1);
	}
	for (long long j = beg; j < mid; j += 8) {
		float v[8][LW];
		ld_row(L + a.x * TILE, v[0]);
		ld_row(L + a.y * TILE, v[1]);
		ld_row(L + a.z * TILE, v[2]);
		ld_row(L + a.w * TILE, v[3]);
		ld_row(L + b.x * TILE, v[4]);
		ld_row(L + b.y * TILE, v[5]);
		ld_row(L + b.z * TILE, v[6]);
		ld_row(L + b.w * TILE, v[7]);
		if (j + 8 < mid) {
			a = __ldg(w4 + ((j + 8) >> 2));
			b = __ldg(w4 + ((j + 8) >> 2) + 1);
		}
#pragma unroll
		for (int q = 0; q < 8; ++q)
#pragma unroll
			for (int k = 0; k < LW; ++k)
				kahan_add(s[q % ECH][k], c[q % ECH][k], v[q][k]);
	}
	for (long long j = mid; j < end; j += 8) {
		const uint4 a2 = __ldg(w4 + (j >> 2)), b2 = __ldg(w4 + (j >> 2) + 1);
		const uint32_t e[8] = {a2.x, a2.y, a2.z, a2.w, b2.x, b2.y, b2.z, b2.w};
		float v[8][LW];
#pragma unroll
		for (int q = 0; q < 8; ++q)
			ld_row(L + (e[q] & IDX_MASK) * TILE, v[q]);
#pragma unroll
		for (int q = 0; q < 8; ++q)
#pragma unroll
			for (int k = 0; k < LW; ++k)
				kahan_add_count(s[q % ECH][k], c[q % ECH][k], e[q] >> IDX_BITS, v[q][k]);
	}
#pragma unroll
	for (int k = 0; k < LW; ++k) {
		double v = kahan_value(s[0][k], c[0][k]);
		if (ECH == 2)
			v = dadd(v, kahan_value(s[ECH - 1][k], c[ECH - 1][k]));
		out[k] = v;
	}
}

// E-step of the pairs [q0, q0 + nq) (all in the orientation block whose first
// tile is t0; logW holds the block's tiles): raw[q][j] = photon sum of
// orientation tile * 128 + j, -inf where that orientation's cell is not
// relevant for the frame (or past R). One warp per pair.
__global__ void __launch_bounds__(256, ESTEP_MINB) estep_pairs_kernel(
    const float *__restrict__ logW, int t0, long long q0, long long nq, const int *__restrict__ pair_tile,
    const int *__restrict__ pair_frame, const uint32_t *__restrict__ ph, const long long *__restrict__ ph_off,
    const long long *__restrict__ ph_mid, const uint8_t *__restrict__ blacklist, int R, int P, RefineMask rm,
    double *__restrict__ raw) {
	const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (w >= nq)
		return;
	const long long q = q0 + w;
	const int rt = pair_tile[q], d = pair_frame[q];
	if (blacklist[d])
		return;  // the normalisation reads no pair of a blacklisted frame
	const int r0 = rt * TILE + lane * LW;
	const unsigned live = refine_live(rm, d, r0);
	double acc[LW];
	if (__any_sync(FULL, live)) {
		const float *L = logW + (size_t)(rt - t0) * (P + 1) * TILE + lane * LW;
		pair_photon_sums(L, ph, ph_off[d], ph_mid[d], ph_off[d + 1], P, acc);
	}
#pragma unroll
	for (int k = 0; k < LW; ++k)
		if (!(live >> k & 1u) || r0 + k >= R)
			acc[k] = -INFINITY;
	st_row(raw + (size_t)q * TILE + lane * LW, acc);
}

// Normalisation over pair lists (norm_kernel's arithmetic, one mode): one
// warp per frame, three passes over the frame's pairs (maximum and its lowest
// orientation, kept sum, probabilities and frame sums). The log-likelihood is
// x = log w_r - u_r s_d + raw, as the E-step forms it in the dense layout.
// Pq aliases raw (PQ_STRIDE): a pair's row belongs to one frame, and the last
// pass stores its probabilities only after every lane of the warp has read
// the row.
__global__ void __launch_bounds__(256) norm_pairs_kernel(
    const double *raw, const long long *__restrict__ frame_off, const int *__restrict__ frame_pair,
    const int *__restrict__ pair_tile, int N, int R, const double *__restrict__ logw, const double *__restrict__ u,
    const double *__restrict__ scale, int use_scale, const double *__restrict__ beta,
    const double *__restrict__ sum_fact, const uint8_t *__restrict__ blacklist, int psum_d_on,
    const double *__restrict__ scalars, float *Pq, int *__restrict__ rmax,
    double *__restrict__ max_exp, double *__restrict__ p_norm, double *__restrict__ info,
    double *__restrict__ likelihood, double *__restrict__ psum_d, int *__restrict__ num_prob) {
	const int d = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
	if (d >= N)
		return;
	const long long k0 = frame_off[d], k1 = frame_off[d + 1];
	const double rescale = scalars[0];
	const double sd = use_scale ? scale[d] : rescale;
	auto loglik = [&](long long k, double (&x)[LW], int &r0) {
		const int q = frame_pair[k];
		r0 = pair_tile[q] * TILE + lane * LW;
		ld_row(raw + (size_t)q * TILE + lane * LW, x);
#pragma unroll
		for (int e = 0; e < LW; ++e)
			if (r0 + e < R)
				x[e] = dadd(dsub(logw[r0 + e], dmul(u[r0 + e], sd)), x[e]);
	};
	double m = MAX_EXP_START;
	int am = -1;
	const bool bl = blacklist[d] != 0;
	if (!bl) {
		for (long long k = k0; k < k1; ++k) {
			double x[LW];
			int r0;
			loglik(k, x, r0);
#pragma unroll
			for (int e = 0; e < LW; ++e)
				if (r0 + e < R && x[e] > m) {
					m = x[e];
					am = r0 + e;
				}
		}
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		double om = __shfl_xor_sync(FULL, m, o);
		int oa = __shfl_xor_sync(FULL, am, o);
		if (om > m || (om == m && oa >= 0 && (am < 0 || oa < am))) {
			m = om;
			am = oa;
		}
	}
	if (bl || m == MAX_EXP_START) {
		float zero[LW];
#pragma unroll
		for (int e = 0; e < LW; ++e)
			zero[e] = 0.f;
		for (long long k = k0; k < k1; ++k)
			st_row(Pq + (size_t)frame_pair[k] * PQ_STRIDE + lane * LW, zero);
		if (lane == 0) {
			rmax[d] = -1;
			max_exp[d] = MAX_EXP_START;
			p_norm[d] = 0.;
			info[d] = 0.;
			likelihood[d] = 0.;
			psum_d[d] = 0.;
			num_prob[d] = 0;
		}
		return;
	}
	const double b = beta[d];
	const double thr = PDIFF_THRESH / b;
	const double lo = dsub(m, thr);
	const int rstar = am;
	double s = 0.;
	int cnt = 0;
	for (long long k = k0; k < k1; ++k) {
		double x[LW];
		int r0;
		loglik(k, x, r0);
#pragma unroll
		for (int e = 0; e < LW; ++e) {
			const int r = r0 + e;
			if (r < R) {
				const bool kept = (r <= rstar) ? (x[e] > lo) : (dadd(x[e], thr) > m);
				if (kept) {
					s += exp(dmul(b, dsub(x[e], m)));
					cnt++;
				}
			}
		}
	}
	s = warp_sum(s);
	for (int o = 16; o > 0; o >>= 1)
		cnt += __shfl_xor_sync(FULL, cnt, o);
	const double sf = sum_fact[d];
	const double inv_s = 1. / s, cinf = -log(s);  // log(M) = 0 with one mode
	double ll = 0., pd = 0., inf = 0.;
	for (long long k = k0; k < k1; ++k) {
		double x[LW];
		int r0;
		loglik(k, x, r0);
		float out[LW];
#pragma unroll
		for (int e = 0; e < LW; ++e) {
			const int r = r0 + e;
			out[e] = 0.f;
			if (r < R) {
				const bool kept = (r <= rstar) ? (x[e] > lo) : (dadd(x[e], thr) > m);
				if (kept) {
					const double y = dmul(b, dsub(x[e], m));
					const double P = exp(y) * inv_s;
					ll += P * (x[e] - sf);
					if (psum_d_on)
						pd += P * u[r] * rescale;
					if (!(P < PROB_MIN))
						inf += P * (y + cinf - logw[r]);
					out[e] = (P > PROB_MIN) ? (float)P : -(float)P;
				}
			}
		}
		__syncwarp();  // every lane has read the row that the stores overwrite
		st_row(Pq + (size_t)frame_pair[k] * PQ_STRIDE + lane * LW, out);
	}
	ll = warp_sum(ll);
	pd = warp_sum(pd);
	inf = warp_sum(inf);
	if (lane == 0) {
		rmax[d] = rstar;
		max_exp[d] = m;
		p_norm[d] = s;
		likelihood[d] = ll;
		info[d] = inf;
		psum_d[d] = pd;
		num_prob[d] = cnt;
	}
}

// psum_r over pair lists: one block per tile, its 8 warps striding over the
// tile's pairs, sum of |P| (times phi_d with need_scaling) per orientation;
// the warps' partial sums are added in warp order.
__global__ void __launch_bounds__(256) psum_pairs_kernel(const float *__restrict__ Pq,
                                                          const long long *__restrict__ tile_off,
                                                          const int *__restrict__ pair_frame,
                                                          const double *__restrict__ scale, int need_scaling,
                                                          int R, double *__restrict__ psum_r) {
	__shared__ double s[8][TILE];
	const int rt = blockIdx.x, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
	double acc[LW];
#pragma unroll
	for (int k = 0; k < LW; ++k)
		acc[k] = 0.;
	for (long long q = tile_off[rt] + w; q < tile_off[rt + 1]; q += 8) {
		float v[LW];
		ld_row(Pq + (size_t)q * PQ_STRIDE + lane * LW, v);
		const double f = need_scaling ? scale[pair_frame[q]] : 1.;
#pragma unroll
		for (int k = 0; k < LW; ++k)
			acc[k] += need_scaling ? fabs((double)v[k]) * f : fabs((double)v[k]);
	}
#pragma unroll
	for (int k = 0; k < LW; ++k)
		s[w][lane * LW + k] = acc[k];
	__syncthreads();
	for (int j = threadIdx.x; j < TILE; j += blockDim.x) {
		double t = 0.;
#pragma unroll
		for (int k = 0; k < 8; ++k)
			t += s[k][j];
		const int r = rt * TILE + j;
		if (r < R)
			psum_r[r] = t;
	}
}

// Tomograms of one orientation block from its pairs [q0, q0 + nq): one warp
// per pair holds the pair's probabilities above PROB_MIN (4 per lane) and adds
// count x P to T[tile - t0][p][.] for every photon of the frame on a mask < 2
// pixel (mw: pixel | count << IDX_BITS per word, frame d's words at
// [mw_off[d], mw_off[d + 1])), one 16-byte atomic add per lane and photon. A
// pair without a probability above PROB_MIN adds nothing and returns.
__global__ void __launch_bounds__(256) mstep_pairs_kernel(const float *__restrict__ Pq, int t0, long long q0,
                                                           long long nq, const int *__restrict__ pair_tile,
                                                           const int *__restrict__ pair_frame,
                                                           const uint32_t *__restrict__ mw,
                                                           const long long *__restrict__ mw_off, int P,
                                                           float *__restrict__ T) {
	const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (w >= nq)
		return;
	const long long q = q0 + w;
	float v[LW];
	ld_row(Pq + (size_t)q * PQ_STRIDE + lane * LW, v);
	bool any = false;
#pragma unroll
	for (int k = 0; k < LW; ++k) {
		v[k] = fmaxf(v[k], 0.f);
		any |= v[k] > 0.f;
	}
	if (!__any_sync(FULL, any))
		return;
	const int rt = pair_tile[q], d = pair_frame[q];
	float *Tt = T + (size_t)(rt - t0) * P * TILE + lane * LW;
	const long long beg = mw_off[d], end = mw_off[d + 1];
	for (long long j0 = beg; j0 < end; j0 += 32) {
		const int n = (int)min(32LL, end - j0);
		const uint32_t mine = lane < n ? __ldg(mw + j0 + lane) : 0u;
		for (int i = 0; i < n; ++i) {
			const uint32_t word = __shfl_sync(FULL, mine, i);
			const float c = (float)(word >> IDX_BITS);
			float *dst = Tt + (size_t)(word & IDX_MASK) * TILE;
			if constexpr (LW == 4) {
				atomicAdd(reinterpret_cast<float4 *>(dst), make_float4(c * v[0], c * v[1], c * v[2], c * v[3]));
			} else {
#pragma unroll
				for (int k = 0; k < LW; ++k)
					atomicAdd(dst + k, c * v[k]);
			}
		}
	}
}

// Orientation-blocked full search, second pass: the probabilities of the
// tiles [t0, t0 + nt) for one frame chunk from their log-likelihoods (pval,
// the chunk's dense layout) and the per-frame results of the first pass
// (max_exp = maximum, rmax = its first orientation, p_norm = kept sum): the
// kept rule and P exactly as the one-exp normalisation forms them (E =
// exp(beta (x - max)) rounded to FP32, times 1 / p_norm in FP32), sign =
// PROB_MIN gate. One warp per (tile, frame); warp index Nc of a tile writes
// the chunk's zero row.
__global__ void __launch_bounds__(256) prob_block_kernel(const double *__restrict__ pval, int t0, int nt, int Nc,
                                                         int d0, int R, const double *__restrict__ beta,
                                                         const double *__restrict__ max_exp,
                                                         const int *__restrict__ rmax,
                                                         const double *__restrict__ p_norm,
                                                         const uint8_t *__restrict__ blacklist,
                                                         float *__restrict__ Pst) {
	const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (w >= (long long)nt * (Nc + 1))
		return;
	const int rl = (int)(w / (Nc + 1)), dl = (int)(w - (long long)rl * (Nc + 1)), rt = t0 + rl;
	float out[LW];
#pragma unroll
	for (int e = 0; e < LW; ++e)
		out[e] = 0.f;
	float *dst = Pst + ((size_t)rt * (Nc + 1) + dl) * TILE + lane * LW;
	if (dl == Nc) {
		st_row(dst, out);
		return;
	}
	const int d = d0 + dl;
	const double m = max_exp[d], s = p_norm[d];
	if (!blacklist[d] && m != MAX_EXP_START && s > 0.) {
		double x[LW];
		ld_row(pval + ((size_t)rt * Nc + dl) * TILE + lane * LW, x);
		const double b = beta[d];
		const double thr = PDIFF_THRESH / b;
		const double lo = dsub(m, thr);
		const int rstar = rmax[d];
		const float inv_sf = (float)(1. / s);
#pragma unroll
		for (int e = 0; e < LW; ++e) {
			const int r = rt * TILE + lane * LW + e;
			if (r < R) {
				const bool kept = (r <= rstar) ? (x[e] > lo) : (dadd(x[e], thr) > m);
				if (kept) {
					const float P = (float)exp(dmul(b, dsub(x[e], m))) * inv_sf;
					out[e] = (P > (float)PROB_MIN) ? P : -P;
				}
			}
		}
	}
	st_row(dst, out);
}

// Captured probability mass of watched frames over pair lists (as
// captured_mass_kernel): for watched frame wf[w] the sum of |P| over the
// orientations whose cell is among its proposed cells, over the sum of all.
__global__ void __launch_bounds__(256) captured_mass_pairs_kernel(
    const float *__restrict__ Pq, const long long *__restrict__ frame_off, const int *__restrict__ frame_pair,
    const int *__restrict__ pair_tile, const int *__restrict__ qmap, const int *__restrict__ wf, int nw,
    const uint32_t *__restrict__ bits, int rwords, double *__restrict__ mass) {
	const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
	if (w >= nw)
		return;
	const int d = wf[w];
	const uint32_t *b = bits + (size_t)w * rwords;
	double in = 0., all = 0.;
	for (long long k = frame_off[d]; k < frame_off[d + 1]; ++k) {
		const int q = frame_pair[k];
		const int r0 = pair_tile[q] * TILE + lane * LW;
		float v[LW];
		ld_row(Pq + (size_t)q * PQ_STRIDE + lane * LW, v);
#pragma unroll
		for (int e = 0; e < LW; ++e) {
			const double p = fabs((double)v[e]);
			const int c = qmap[r0 + e];
			all += p;
			if (c >= 0 && (b[c >> 5] >> (c & 31) & 1u))
				in += p;
		}
	}
	in = warp_sum(in);
	all = warp_sum(all);
	if (lane == 0)
		mass[w] = all > 0. ? in / all : 0.;
}

}  // namespace dfg
