// Background-aware iteration for sm_100a (detector with a per-pixel background
// and need_scaling): E-step with the background in the predicted counts,
// tomograms and scale factors by bracketed root finding. Layouts as in
// emc_common.cuh, except that the slices are W itself in FP64 (not log W in
// FP32): the tomogram roots may be negative, so the model and slices may be,
// and W phi + b bg can cancel, which FP32 would not resolve. All frames form
// one chunk. Included by emc_api.cu only.
#pragma once

#include "emc_common.cuh"

namespace dfg {

constexpr float LOG_DBL_MIN_F = -708.39642f;  // log(DBL_MIN): the reference's value for a negative prediction
constexpr double BG_GRAD_TOL = 1.e-4;         // max_update.c:348
constexpr double BG_SCALE_TOL = 1.e-3;        // max_scale.c:229, 264

// ---------------------------------------------------------------------------
// E-step (max_prob.c:94, 134-156): the photon term is
// sum_k c_k log(W_r[p_k] phi_d + b_d bg[p_k]) on the un-logged slice, with
// log(DBL_MIN) where the prediction is negative. The prediction is formed in
// FP64 in the reference's operation order; its logarithm is taken in FP32
// (relative error 6e-8, as the plain path's log-slices) and summed with
// compensation; padding words (pixel P) are skipped.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256, 3) estep_bg_kernel(
    const double *__restrict__ Wsl, const double *__restrict__ u, const double *__restrict__ logw, int R,
    const uint32_t *__restrict__ ph, const long long *__restrict__ ph_off, const long long *__restrict__ ph_mid,
    const double *__restrict__ scale, const double *__restrict__ bgscale, const double *__restrict__ bg,
    const uint8_t *__restrict__ blacklist, int d0, int Nc, int use_scale, const double *__restrict__ scalars,
    int P, int RT, double *__restrict__ pval, double *__restrict__ tmax, int *__restrict__ targ, RefineMask rm) {
	const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (warp >= (long long)RT * Nc)
		return;
	const int rt = (int)(warp / Nc), dl = (int)(warp - (long long)rt * Nc), d = d0 + dl;
	if (blacklist[d])
		return;
	const int r0 = rt * TILE + lane * LW;
	const unsigned live = refine_live(rm, d, r0);
	if (rm.qmap != nullptr && !__any_sync(FULL, live)) {
		refine_skip_tile(tmax, targ, rt, Nc, dl, lane);
		return;
	}
	const double *L = Wsl + (size_t)rt * (P + 1) * TILE + lane * LW;
	const long long beg = ph_off[d], mid = ph_mid[d], end = ph_off[d + 1];
	const uint4 *w4 = reinterpret_cast<const uint4 *>(ph);
	const double sd = scale[d], bs = bgscale[d];
	float s[LW], c[LW];
#pragma unroll
	for (int k = 0; k < LW; ++k)
		s[k] = c[k] = 0.f;
	for (long long j = beg; j < end; j += 8) {
		const uint4 a = __ldg(w4 + (j >> 2)), b = __ldg(w4 + (j >> 2) + 1);
		const uint32_t e[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
		const bool multi = j >= mid;
#pragma unroll
		for (int q = 0; q < 8; ++q) {
			const uint32_t idx = multi ? (e[q] & IDX_MASK) : e[q];
			if (idx == (uint32_t)P)  // padding (identical in every lane)
				continue;
			double v[LW];
			ld_row(L + idx * TILE, v);
			const double bb = dmul(bs, __ldg(bg + idx));
#pragma unroll
			for (int k = 0; k < LW; ++k) {
				const double ip = dadd(dmul(v[k], sd), bb);
				const float lg = ip < 0. ? LOG_DBL_MIN_F : (ip < 1.e-30 ? (float)log(ip) : logf((float)ip));
				if (multi)
					kahan_add_count(s[k], c[k], e[q] >> IDX_BITS, lg);
				else
					kahan_add(s[k], c[k], lg);
			}
		}
	}
	const double su = use_scale ? scale[d] : scalars[0];
	double acc[LW];
	double m = MAX_EXP_START;
	int am = -1;
#pragma unroll
	for (int k = 0; k < LW; ++k) {
		const int r = r0 + k;
		acc[k] = 0.;
		if (r < R) {
			acc[k] = dadd(dsub(logw[r], dmul(u[r], su)), kahan_value(s[k], c[k]));
			if (!(live >> k & 1u))
				acc[k] = -INFINITY;
			else if (acc[k] > m) {
				m = acc[k];
				am = r;
			}
		}
	}
	st_row(pval + ((size_t)rt * Nc + dl) * TILE + lane * LW, acc);
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		double om = __shfl_xor_sync(FULL, m, o);
		int oa = __shfl_xor_sync(FULL, am, o);
		if (om > m || (om == m && oa >= 0 && (am < 0 || oa < am))) {
			m = om;
			am = oa;
		}
	}
	if (lane == 0) {
		tmax[(size_t)rt * Nc + dl] = m;
		targ[(size_t)rt * Nc + dl] = am;
	}
}

// scalemax per orientation: the largest phi_d over frames with P >= PROB_MIN
// (calc_psum_r's return value, max_update.c:132-133), as partial maxima per
// frame split; grid (RT, splits) like psum_r_kernel.
__global__ void __launch_bounds__(256) scalemax_kernel(const double *__restrict__ Pd, int Nc, int d0,
                                                       int frames_per_split, const double *__restrict__ scale,
                                                       double *__restrict__ part, int R_pad) {
	__shared__ double s[8][TILE];
	const int rt = blockIdx.x, split = blockIdx.y, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int beg = split * frames_per_split, end = min(Nc, beg + frames_per_split);
	double mx[LW];
#pragma unroll
	for (int k = 0; k < LW; ++k)
		mx[k] = -DBL_MAX;
	const double *p = Pd + (size_t)rt * (Nc + 1) * TILE + lane * LW;
	for (int dl = beg + w; dl < end; dl += 8) {
		double v[LW];
		ld_row(p + (size_t)dl * TILE, v);
		const double f = scale[d0 + dl];
#pragma unroll
		for (int k = 0; k < LW; ++k)
			if (v[k] > 0. && f > mx[k])
				mx[k] = f;
	}
#pragma unroll
	for (int k = 0; k < LW; ++k)
		s[w][lane * LW + k] = mx[k];
	__syncthreads();
	for (int j = threadIdx.x; j < TILE; j += blockDim.x) {
		double t = -DBL_MAX;
#pragma unroll
		for (int k = 0; k < 8; ++k)
			t = fmax(t, s[k][j]);
		part[(size_t)split * R_pad + rt * TILE + j] = t;
	}
}

__global__ void scalemax_reduce_kernel(const double *__restrict__ part, int nsplit, int R, int R_pad,
                                       double *__restrict__ scalemax) {
	const int r = blockIdx.x * blockDim.x + threadIdx.x;
	if (r >= R)
		return;
	double t = -DBL_MAX;
	for (int k = 0; k < nsplit; ++k)
		t = fmax(t, part[(size_t)k * R_pad + r]);
	scalemax[r] = t;
}

// ---------------------------------------------------------------------------
// Tomograms (update_tomogram_bg, max_update.c:343-543, with gradient_rt
// :232-341): for every (orientation r, pixel p) the view W solving
//   G(W) = -psum_r + sum_d P_dr c_dp phi_d / (W phi_d + b_d bg_p) = 0
// over the frames with P_dr > PROB_MIN and photons at p, bracketed and refined
// by Ridder's method with the reference's state rules:
//     0 still searching, 1 no photons (view 0), 128 negligible background
//   (standard update sum P c / psum_r), 160 bracket below the smallest
//   background-only prediction, 192 bracket found, 255 done.
// Every (r, p) evolves from its own state only, so per-warp loops with the
// reference's round limits (10 bracketing rounds, 50 Ridder rounds) give its
// results. One warp per (orientation tile, pixel) of the pixel-major index;
// each lane keeps the search of its LW orientations in registers and every
// gradient evaluation walks the pixel's frame list again (L1/L2-resident).
// Everything is FP64, in the reference's operation order per term (the search
// brackets reach 1e-8 above the pole W = -b bg / phi, where W phi + b bg
// cancels), with P in FP64. The final views go to T.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) mstep_bg_kernel(
    const double *__restrict__ Pd, int Nc, int d0, const uint32_t *__restrict__ cs,
    const long long *__restrict__ cs_off, const long long *__restrict__ cs_mid, const int *__restrict__ pix,
    int npix, int P, int RT, int R, const double *__restrict__ psum_r, const double *__restrict__ scalemax,
    const double *__restrict__ scale, const double *__restrict__ bgscale, const double *__restrict__ background,
    const double *__restrict__ powder, double mean_per_pixel, float *__restrict__ T) {
	const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (warp >= (long long)RT * npix)
		return;
	const int rt = (int)(warp / npix), kp = (int)(warp - (long long)rt * npix);
	const int p = pix[kp];
	const double *Pr = Pd + (size_t)rt * (Nc + 1) * TILE + lane * LW;
	const long long beg = cs_off[p], mid = cs_mid[p], end = cs_off[p + 1];
	const uint4 *w4 = reinterpret_cast<const uint4 *>(cs);
	const double bgp = background[p], pw = powder[p];

	int st[LW];
	double psr[LW], Wold[LW], Wnew[LW], Wmid[LW], Wlat[LW], Gold[LW], Gnew[LW], Gmid[LW], Glat[LW], view[LW];
#pragma unroll
	for (int k = 0; k < LW; ++k) {
		const int r = rt * TILE + lane * LW + k;
		Wold[k] = Wnew[k] = Wmid[k] = Wlat[k] = 0.;
		Gold[k] = Gnew[k] = Gmid[k] = Glat[k] = 0.;
		view[k] = 0.;
		psr[k] = 0.;
		st[k] = 255;
		if (r < R) {
			psr[k] = psum_r[r];
			const double smax = scalemax[r];
			if (bgp / smax < 1.e-2 * pw) {
				st[k] = 128;
			} else {
				st[k] = 0;
				Wnew[k] = 1.e-8 - bgp / smax;
			}
		}
	}

	// gradient_rt at the points Wx; updates the 0/1 states as the reference does
	auto grad = [&](const double (&Wx)[LW], double (&G)[LW]) {
		double acc[LW], mx[LW];
		bool hit[LW];
#pragma unroll
		for (int k = 0; k < LW; ++k) {
			acc[k] = 0.;
			mx[k] = -1.e100;
			hit[k] = false;
		}
		for (long long j = beg; j < end; j += 8) {
			const uint4 a = __ldg(w4 + (j >> 2)), b = __ldg(w4 + (j >> 2) + 1);
			const uint32_t e[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
			const bool multi = j >= mid;
#pragma unroll 2
			for (int q = 0; q < 8; ++q) {
				const uint32_t dl = multi ? (e[q] & IDX_MASK) : e[q];
				if (dl == (uint32_t)Nc)  // padding
					continue;
				const double cnt = multi ? (double)(e[q] >> IDX_BITS) : 1.;
				double pv[LW];
				ld_row(Pr + (size_t)dl * TILE, pv);
				const double sd = scale[d0 + dl], bd = bgscale[d0 + dl];
				const double bb = dmul(bd, bgp);
#pragma unroll
				for (int k = 0; k < LW; ++k) {
					if (!(pv[k] > 0.))
						continue;
					const double pk = dmul(pv[k], cnt);
					if (st[k] < 128) {
						const double val = dadd(dmul(Wx[k], sd), bb);
						acc[k] = dadd(acc[k], dmul(pk, sd) / val);
						hit[k] = true;
					} else if (st[k] == 128) {
						acc[k] = dadd(acc[k], pk);
					} else if (st[k] == 160) {
						mx[k] = fmax(mx[k], sd / bd);
					}
				}
			}
		}
#pragma unroll
		for (int k = 0; k < LW; ++k) {
			if (st[k] < 128) {
				G[k] = dadd(-psr[k], acc[k]);
				st[k] = hit[k] ? 0 : 1;
			} else if (st[k] == 128) {
				G[k] = acc[k];
			} else if (st[k] == 160) {
				G[k] = mx[k];
			} else {
				G[k] = 0.;
			}
		}
	};
	auto any_state = [&](int s0, int s1) {
		bool a = false;
#pragma unroll
		for (int k = 0; k < LW; ++k)
			a |= (st[k] == s0 || st[k] == s1);
		return __any_sync(FULL, a);
	};

	// search bounds: G(0) and the far end (max_update.c:380-433)
	grad(Wold, Gold);
#pragma unroll
	for (int k = 0; k < LW; ++k) {
		if (st[k] == 255)
			continue;
		if (fabs(Gold[k]) < BG_GRAD_TOL) {
			view[k] = 0.;
			st[k] = 255;
		} else if (Gold[k] > 0.) {
			Wnew[k] = 2. * (pw > mean_per_pixel ? pw : mean_per_pixel);
		}
	}
	for (int i = 0; i < 10 && any_state(0, 160); ++i) {
		grad(Wnew, Gnew);
#pragma unroll
		for (int k = 0; k < LW; ++k) {
			if (st[k] == 0) {
				if (Gold[k] < 0. && Gnew[k] < 0.)
					st[k] = 160;
				else if (Gold[k] > 0. && Gnew[k] > 0.)
					Wnew[k] *= 2.;
				else
					st[k] = 192;
			} else if (st[k] == 160) {
				Wnew[k] = 1.e-8 - bgp / Gnew[k];
				st[k] = 0;
			}
		}
	}
	// Ridder's method (max_update.c:435-543)
	for (int i = 0; i < 50; ++i) {
#pragma unroll
		for (int k = 0; k < LW; ++k) {
			if (st[k] == 1) {
				st[k] = 255;
				view[k] = 0.;
			} else if (st[k] == 128) {
				view[k] = Gold[k] / psr[k];
				st[k] = 255;
			} else if (st[k] == 192 || st[k] == 0) {
				st[k] = 0;
				Wmid[k] = 0.5 * (Wold[k] + Wnew[k]);
			}
		}
		if (!any_state(0, 0))
			break;
		grad(Wmid, Gmid);
#pragma unroll
		for (int k = 0; k < LW; ++k) {
			if (st[k] == 1) {
				st[k] = 255;
				view[k] = 0.;
			} else if (st[k] == 0) {
				if (fabs(Gmid[k]) < BG_GRAD_TOL) {
					view[k] = Wmid[k];
					st[k] = 255;
				} else {
					const double s = sqrt(Gmid[k] * Gmid[k] - Gold[k] * Gnew[k]);
					if (s < 1.e-15) {
						Wlat[k] = Wmid[k];
					} else {
						Wlat[k] = Wmid[k] + (Wmid[k] - Wold[k]) * copysign(1.0, Gold[k]) * Gmid[k] / s;
						const double lo = fmin(Wold[k], Wnew[k]), hi = fmax(Wold[k], Wnew[k]);
						if (Wlat[k] <= lo || Wlat[k] >= hi)
							Wlat[k] = Wmid[k];
					}
				}
			}
		}
		if (!any_state(0, 0))
			break;
		grad(Wlat, Glat);
#pragma unroll
		for (int k = 0; k < LW; ++k) {
			if (st[k] == 1) {
				st[k] = 255;
				view[k] = 0.;
			} else if (st[k] == 0) {
				if (fabs(Glat[k]) < BG_GRAD_TOL) {
					view[k] = Wlat[k];
					st[k] = 255;
				} else if (Gmid[k] * Glat[k] < 0.) {
					Wold[k] = Wmid[k];
					Gold[k] = Gmid[k];
					Wnew[k] = Wlat[k];
					Gnew[k] = Glat[k];
				} else if (Gold[k] * Glat[k] < 0.) {
					Wnew[k] = Wlat[k];
					Gnew[k] = Glat[k];
				} else {
					Wold[k] = Wlat[k];
					Gold[k] = Glat[k];
				}
			}
		}
	}
	// states 1 and 128 that the Ridder loop did not visit (it breaks as soon as
	// no search is left) settle as in its first phase
#pragma unroll
	for (int k = 0; k < LW; ++k) {
		if (st[k] == 128)
			view[k] = Gold[k] / psr[k];
		else if (st[k] != 255)
			view[k] = st[k] == 1 ? 0. : view[k];
	}
	float o[LW];
#pragma unroll
	for (int k = 0; k < LW; ++k)
		o[k] = (float)view[k];
	st_row(T + ((size_t)rt * P + p) * TILE + lane * LW, o);
}

// ---------------------------------------------------------------------------
// Scale factors (update_scale_bg, max_scale.c:129-288): per frame the phi
// solving G_d(phi) = sum_r P_dr sum_k c_k v_r[p_k] / (v_r[p_k] phi + b_d bg_k)
// - psum_d = 0 (gradient_d, max_scale.c:21-127), v_r = W_r * rescale, over the
// pairs with P > PROB_MIN and the frame's mask-0 photons. The bracketing and
// Ridder steps run on the host per frame; this kernel evaluates the sums for
// the frames still searching (active), one warp per (orientation tile, frame),
// in FP64 (slices may be negative, so v phi + b bg may cancel), and writes
// per-tile partials for a fixed-order reduction.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256, 3) grad_d_kernel(
    const double *__restrict__ Wsl, const double *__restrict__ Pd, int Nc, int d0, int RT, int P,
    const uint32_t *__restrict__ ph, const long long *__restrict__ ph_off, const long long *__restrict__ ph_mid,
    const double *__restrict__ scalars, const double *__restrict__ s_eval, const double *__restrict__ bgscale,
    const double *__restrict__ bg, const uint8_t *__restrict__ active, double *__restrict__ part) {
	const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (warp >= (long long)RT * Nc)
		return;
	const int rt = (int)(warp / Nc), dl = (int)(warp - (long long)rt * Nc), d = d0 + dl;
	if (!active[d])
		return;
	double pv[LW];
	ld_row(Pd + ((size_t)rt * (Nc + 1) + dl) * TILE + lane * LW, pv);
	bool any = false;
#pragma unroll
	for (int k = 0; k < LW; ++k)
		any |= pv[k] > 0.;
	if (!__any_sync(FULL, any)) {
		if (lane == 0)
			part[(size_t)rt * Nc + dl] = 0.;
		return;
	}
	const double *L = Wsl + (size_t)rt * (P + 1) * TILE + lane * LW;
	const long long beg = ph_off[d], mid = ph_mid[d], end = ph_off[d + 1];
	const uint4 *w4 = reinterpret_cast<const uint4 *>(ph);
	const double resc = scalars[0], sd = s_eval[d], bs = bgscale[d];
	double s[LW];
#pragma unroll
	for (int k = 0; k < LW; ++k)
		s[k] = 0.;
	for (long long j = beg; j < end; j += 8) {
		const uint4 a = __ldg(w4 + (j >> 2)), b = __ldg(w4 + (j >> 2) + 1);
		const uint32_t e[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
		const bool multi = j >= mid;
#pragma unroll
		for (int q = 0; q < 8; ++q) {
			const uint32_t idx = multi ? (e[q] & IDX_MASK) : e[q];
			if (idx == (uint32_t)P)
				continue;
			double v[LW];
			ld_row(L + idx * TILE, v);
			const double bb = dmul(bs, __ldg(bg + idx));
			const double cnt = multi ? (double)(e[q] >> IDX_BITS) : 1.;
#pragma unroll
			for (int k = 0; k < LW; ++k) {
				const double vr = dmul(v[k], resc);
				s[k] = dadd(s[k], dmul(cnt, vr) / dadd(dmul(vr, sd), bb));
			}
		}
	}
	double acc = 0.;
#pragma unroll
	for (int k = 0; k < LW; ++k)
		if (pv[k] > 0.)
			acc += pv[k] * s[k];
	acc = warp_sum(acc);
	if (lane == 0)
		part[(size_t)rt * Nc + dl] = acc;
}

// G_d = sum over tiles (fixed order) - psum_d, for the active frames
__global__ void grad_d_reduce_kernel(const double *__restrict__ part, int RT, int Nc, int d0,
                                     const double *__restrict__ psum_d, const uint8_t *__restrict__ active,
                                     double *__restrict__ G) {
	const int dl = blockIdx.x * blockDim.x + threadIdx.x;
	if (dl >= Nc || !active[d0 + dl])
		return;
	double t = 0.;
	for (int rt = 0; rt < RT; ++rt)
		t += part[(size_t)rt * Nc + dl];
	G[d0 + dl] = t - psum_d[d0 + dl];
}

}  // namespace dfg
