// Kernels of one EMC iteration for sm_100a (B200); layouts in emc_common.cuh.
// Included by emc_api.cu only (one definition of each kernel).
#pragma once

#include "emc_common.cuh"

namespace dfg {

// ---------------------------------------------------------------------------
// (a) slice generation: logW[tile][p][j] = log(W_r[p]) and u_r, r = tile * TILE + j
// ---------------------------------------------------------------------------
// Block = one orientation tile; it walks every pixel in chunks of SB pixels,
// in pixel order. Per chunk the 256 threads compute W for SB pixels x TILE
// orientations into shared memory (thread (i = t % SB, g = t / SB) takes
// pixel i of orientations g, g + 256/SB, ..., so a warp walks 32 neighbouring
// pixels of one orientation); then thread j < TILE adds the chunk's mask-0
// values of orientation j to u_j in pixel order, which keeps u_r
// bit-identical to the reference's sequential sum (max_prob.c:32-38), while
// the warps store log W as coalesced rows (max_prob.c:94-97); with Wd given
// (background-aware path, max_prob.c:94) they store W itself in FP64 there.
constexpr int SB = 32;

template <typename MT, int GEO>
__global__ void __launch_bounds__(256) slice_u_tile_kernel(
    const double *__restrict__ quats, int M, int R, const double *__restrict__ qvals,
    const double *__restrict__ corr, const uint8_t *__restrict__ mask, int P, const MT *__restrict__ model,
    long long S, long long V, float *__restrict__ logW, double *__restrict__ u, double *__restrict__ Wd) {
	__shared__ double s_rot[TILE][9];
	__shared__ int s_mode[TILE];
	__shared__ double s_w[SB][TILE + 1];
	__shared__ double s_q[SB][4];
	__shared__ int s_m[SB];
	const int t = threadIdx.x, rt = blockIdx.x;
	for (int j = t; j < TILE; j += blockDim.x) {
		int r = rt * TILE + j;
		int rr = r < R ? r : 0;
		geo_setup<GEO>(quats, rr / M, s_rot[j]);
		s_mode[j] = rr % M;
	}
	const double center = (double)(S / 2);
	const int i = t % SB, g = t / SB, w = t >> 5, lane = t & 31;
	double acc = 0.;
	for (int p0 = 0; p0 < P; p0 += SB) {
		if (t < SB) {
			const int p = p0 + t;
			if (p < P) {
				s_q[t][0] = qvals[3 * (size_t)p];
				s_q[t][1] = qvals[3 * (size_t)p + 1];
				s_q[t][2] = qvals[3 * (size_t)p + 2];
				s_q[t][3] = corr[p];
				s_m[t] = mask[p];
			} else {
				s_m[t] = -1;
			}
		}
		__syncthreads();
		if (s_m[i] >= 0) {
			const double qx = s_q[i][0], qy = s_q[i][1], qz = s_q[i][2], cr = s_q[i][3];
#pragma unroll 2
			for (int j = g; j < TILE; j += 256 / SB) {
				if constexpr (GEO == MT_3D) {
					Cell c = locate(s_rot[j], qx, qy, qz, center, S);
					s_w[i][j] = interp(c, model + (size_t)s_mode[j] * V, S, cr);
				} else {
					s_w[i][j] = geo_sample<GEO>(s_rot[j], qx, qy, qz, center, S, model + (size_t)s_mode[j] * V, cr);
				}
			}
		}
		__syncthreads();
		if (t < TILE) {
#pragma unroll 8
			for (int k = 0; k < SB; ++k)
				if (s_m[k] == 0)
					acc = dadd(acc, s_w[k][t]);
		}
		for (int row = w; row < SB; row += 8) {
			const int pp = p0 + row;
			if (pp < P) {
				if (Wd != nullptr) {
					double v[LW];
#pragma unroll
					for (int k = 0; k < LW; ++k)
						v[k] = s_w[row][lane * LW + k];
					st_row(Wd + ((size_t)rt * (P + 1) + pp) * TILE + lane * LW, v);
				} else {
					float v[LW];
#pragma unroll
					for (int k = 0; k < LW; ++k)
						v[k] = (float)log(s_w[row][lane * LW + k]);
					st_row(logW + ((size_t)rt * (P + 1) + pp) * TILE + lane * LW, v);
				}
			}
		}
		__syncthreads();
	}
	if (t < TILE && rt * TILE + t < R)
		u[rt * TILE + t] = acc;
}

// Block = OB consecutive orientations (OB divides TILE); it walks every pixel
// in chunks of 4096 / OB pixels, in pixel order. Per chunk the 256 threads
// compute W for the chunk's pixels x OB orientations into shared memory
// (consecutive threads take consecutive pixels of one orientation, so a warp
// reads neighbouring model voxels); then thread j < OB adds the chunk's
// mask-0 values of its orientation to u in pixel order, which keeps u_r
// bit-identical to the reference's sequential sum (max_prob.c:32-38), while
// all threads store log W as coalesced row segments (max_prob.c:94-97). The
// host uses it when whole tiles would give the SMs too few blocks.
template <typename MT, int OB, int GEO>
__global__ void __launch_bounds__(256) slice_u_kernel(
    const double *__restrict__ quats, int M, int R, const double *__restrict__ qvals,
    const double *__restrict__ corr, const uint8_t *__restrict__ mask, int P, const MT *__restrict__ model,
    long long S, long long V, float *__restrict__ logW, double *__restrict__ u, double *__restrict__ Wd) {
	static_assert(TILE % OB == 0 && OB % LW == 0, "orientation block must divide the tile");
	constexpr int CB = 4096 / OB;  // pixels per chunk
	static_assert(256 % CB == 0, "a thread keeps one pixel of the chunk");
	constexpr int SEG = OB / LW;   // vector stores per row segment
	__shared__ double s_rot[OB][9];
	__shared__ int s_mode[OB];
	__shared__ double s_w[CB][OB + 1];
	__shared__ double s_q[CB][4];
	__shared__ int s_m[CB];
	const int t = threadIdx.x, r0 = blockIdx.x * OB, rt = r0 / TILE, jj0 = r0 % TILE;
	for (int j = t; j < OB; j += blockDim.x) {
		const int r = r0 + j;
		const int rr = r < R ? r : 0;
		geo_setup<GEO>(quats, rr / M, s_rot[j]);
		s_mode[j] = rr % M;
	}
	const double center = (double)(S / 2);
	double acc = 0.;
	for (int p0 = 0; p0 < P; p0 += CB) {
		for (int k = t; k < CB; k += blockDim.x) {
			const int p = p0 + k;
			if (p < P) {
				s_q[k][0] = qvals[3 * (size_t)p];
				s_q[k][1] = qvals[3 * (size_t)p + 1];
				s_q[k][2] = qvals[3 * (size_t)p + 2];
				s_q[k][3] = corr[p];
				s_m[k] = mask[p];
			} else {
				s_m[k] = -1;
			}
		}
		__syncthreads();
		{
			// 256 is a multiple of CB: thread t keeps pixel t % CB in registers
			// and takes orientations t / CB, t / CB + 256 / CB, ...
			const int i = t % CB;
			if (s_m[i] >= 0) {
				const double qx = s_q[i][0], qy = s_q[i][1], qz = s_q[i][2], cr = s_q[i][3];
#pragma unroll 2
				for (int j = t / CB; j < OB; j += 256 / CB) {
					if constexpr (GEO == MT_3D) {
						Cell c = locate(s_rot[j], qx, qy, qz, center, S);
						s_w[i][j] = interp(c, model + (size_t)s_mode[j] * V, S, cr);
					} else {
						s_w[i][j] =
						    geo_sample<GEO>(s_rot[j], qx, qy, qz, center, S, model + (size_t)s_mode[j] * V, cr);
					}
				}
			}
		}
		__syncthreads();
		if (t < OB) {
#pragma unroll 8
			for (int k = 0; k < CB; ++k)
				if (s_m[k] == 0)
					acc = dadd(acc, s_w[k][t]);
		}
		for (int idx = t; idx < CB * SEG; idx += blockDim.x) {
			const int row = idx / SEG, seg = idx % SEG, pp = p0 + row;
			if (pp < P) {
				if (Wd != nullptr) {
					double v[LW];
#pragma unroll
					for (int k = 0; k < LW; ++k)
						v[k] = s_w[row][seg * LW + k];
					st_row(Wd + ((size_t)rt * (P + 1) + pp) * TILE + jj0 + seg * LW, v);
				} else {
					float v[LW];
#pragma unroll
					for (int k = 0; k < LW; ++k)
						v[k] = (float)log(s_w[row][seg * LW + k]);
					st_row(logW + ((size_t)rt * (P + 1) + pp) * TILE + jj0 + seg * LW, v);
				}
			}
		}
		__syncthreads();
	}
	if (t < OB && r0 + t < R)
		u[r0 + t] = acc;
}

// log w_r per orientation, so that no pair evaluates a logarithm of its
// orientation weight (max_prob.c:122).
__global__ void logw_kernel(const double *__restrict__ quats, int M, int R, double *__restrict__ logw) {
	const int r = blockIdx.x * blockDim.x + threadIdx.x;
	if (r < R)
		logw[r] = log(quats[(r / M) * 5 + 4]);
}

// rescale = mean_count / sum_r w_r u_r * M, summed in orientation order
// (max_prob.c:40, 55-60): the block stages 256 products at a time in shared
// memory and one thread adds them in order.
__global__ void __launch_bounds__(256) rescale_kernel(const double *__restrict__ u, const double *__restrict__ quats,
                                                      int M, int R, double mean_count, double *__restrict__ scalars) {
	__shared__ double s_p[256];
	double total = 0.;
	for (int r0 = 0; r0 < R; r0 += 256) {
		const int r = r0 + threadIdx.x;
		s_p[threadIdx.x] = r < R ? dmul(quats[(r / M) * 5 + 4], u[r]) : 0.;
		__syncthreads();
		if (threadIdx.x == 0) {
			const int n = min(256, R - r0);
#pragma unroll 8
			for (int k = 0; k < n; ++k)
				total = dadd(total, s_p[k]);
		}
		__syncthreads();
	}
	if (threadIdx.x == 0)
		scalars[0] = mean_count / total * M;
}

// ---------------------------------------------------------------------------
// (b) E-step: pval[tile][d][j] = log w_r - u_r * s_d + sum_k c_k logW_r[p_k]
// ---------------------------------------------------------------------------
// One warp per (orientation tile, frame), tiles outermost so that resident
// warps share one tile's log-slices in L2. Each photon costs one coalesced
// row read (one LW-wide vector load per lane) and a compensated FP32
// addition per orientation (no conversion instructions in the loop; with one
// orientation per lane two interleaved accumulators halve the dependency
// chain); padded segments need no per-photon bounds test. The photon sum is
// formed in FP64 once per pair. s_d = phi_d when need_scaling &&
// (iteration > 1 || known_scale), else the rescale factor (max_prob.c:122-128).
constexpr int ECH = LW == 1 ? 2 : 1;  // accumulator chains per orientation
constexpr int ESTEP_MINB = LW == 1 ? 6 : (LW == 2 ? 4 : 3);

// Coarse-to-fine refinement (param->refine, max_prob.c:110-120): frame d
// evaluates orientation r only when r's coarse cell qmap[r] is one of the
// frame's relevant coarse orientations, held as one bit per coarse
// orientation in rel[d * rwords ...]. A pair that is not evaluated never
// enters the frame's list; its log-likelihood is stored as -inf, which the
// normalisation neither keeps nor takes as a maximum. qmap == nullptr: every
// pair is evaluated.
struct RefineMask {
	const int *qmap;      // [R_pad] coarse cell per orientation, -1 past R
	const uint32_t *rel;  // [N][rwords]
	int rwords;
};

// Bit k set when orientation r0 + k (k < LW) is evaluated for frame d.
__device__ __forceinline__ unsigned refine_live(const RefineMask &rm, int d, int r0) {
	if (rm.qmap == nullptr)
		return (1u << LW) - 1u;
	const uint32_t *bits = rm.rel + (size_t)d * rm.rwords;
	unsigned live = 0;
#pragma unroll
	for (int k = 0; k < LW; ++k) {
		const int c = __ldg(rm.qmap + r0 + k);
		if (c >= 0 && (__ldg(bits + (c >> 5)) >> (c & 31) & 1u))
			live |= 1u << k;
	}
	return live;
}

// A (tile, frame) task with no evaluated pair: an empty tile maximum, which
// makes the normalisation treat the tile as dead without reading its
// log-likelihoods (so none are written).
__device__ __forceinline__ void refine_skip_tile(double *__restrict__ tmax, int *__restrict__ targ, int rt,
                                                 int Nc, int dl, int lane) {
	if (lane == 0) {
		tmax[(size_t)rt * Nc + dl] = MAX_EXP_START;
		targ[(size_t)rt * Nc + dl] = -1;
	}
}

template <bool REFINE, int MINB = ESTEP_MINB>
__global__ void __launch_bounds__(256, MINB) estep_kernel(
    const float *__restrict__ logW, const double *__restrict__ u, const double *__restrict__ logw, int R,
    const uint32_t *__restrict__ ph, const long long *__restrict__ ph_off, const long long *__restrict__ ph_mid,
    const double *__restrict__ scale, const uint8_t *__restrict__ blacklist, int d0, int Nc, int use_scale,
    const double *__restrict__ scalars, int P, int RT, double *__restrict__ pval, double *__restrict__ tmax,
    int *__restrict__ targ, RefineMask rm, int t0 = 0) {
	// RT tiles from tile t0 (orientation blocks: logW holds tiles t0 ..)
	const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (warp >= (long long)RT * Nc)
		return;
	const int rl = (int)(warp / Nc), dl = (int)(warp - (long long)rl * Nc), d = d0 + dl, rt = t0 + rl;
	if (blacklist[d])
		return;
	const int r0 = rt * TILE + lane * LW;
	unsigned live = (1u << LW) - 1u;
	if constexpr (REFINE) {
		live = refine_live(rm, d, r0);
		if (!__any_sync(FULL, live)) {
			refine_skip_tile(tmax, targ, rt, Nc, dl, lane);
			return;
		}
	}
	const float *L = logW + (size_t)rl * (P + 1) * TILE + lane * LW;
	const long long beg = ph_off[d], mid = ph_mid[d], end = ph_off[d + 1];
	// segments start at multiples of 8 words: two 16-byte loads, identical for
	// every lane (broadcast), bring 8 photon words
	const uint4 *w4 = reinterpret_cast<const uint4 *>(ph);
	float s[ECH][LW], c[ECH][LW];
#pragma unroll
	for (int h = 0; h < ECH; ++h)
#pragma unroll
		for (int k = 0; k < LW; ++k)
			s[h][k] = c[h][k] = 0.f;
	// the next 8 words are fetched while the current 8 rows are in flight
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
		const uint4 a = __ldg(w4 + (j >> 2)), b = __ldg(w4 + (j >> 2) + 1);
		const uint32_t e[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
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
	const double sd = use_scale ? scale[d] : scalars[0];
	double acc[LW];
	// tile maximum and its lowest orientation index (strict > in ascending r,
	// as the running maximum of max_prob.c:199-202)
	double m = MAX_EXP_START;
	int am = -1;
#pragma unroll
	for (int k = 0; k < LW; ++k) {
		const int r = r0 + k;
		acc[k] = 0.;
		if (r < R) {
			double ph_sum = kahan_value(s[0][k], c[0][k]);
			if (ECH == 2)
				ph_sum = dadd(ph_sum, kahan_value(s[ECH - 1][k], c[ECH - 1][k]));
			acc[k] = dadd(dsub(logw[r], dmul(u[r], sd)), ph_sum);
			if (REFINE && !(live >> k & 1u))
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

// ---------------------------------------------------------------------------
// (c) per-frame maximum, pruning, normalisation and frame reductions
// ---------------------------------------------------------------------------
// Asynchronous 16-byte global -> shared copies (cp.async, L2 only). Each
// lane copies and later reads its own bytes, so completion of the lane's own
// groups (cp.async.wait_group) is all the synchronisation needed; the waits
// are hardware waits on copies already issued and always end.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
	const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Rows of a frame's log-likelihoods in flight per warp in the normalisation
// (a ring of NORM_RING 1-KB rows in shared memory per warp).
constexpr int NORM_RING = 6;

// Streams rows 0 .. RT-1 of one lane's LW doubles (row k at src + k * stride)
// through the lane's slots of a shared-memory ring, NORM_RING - 1 rows ahead
// of the one being consumed, and calls f(rt, v) for each row in order.
template <typename F>
__device__ __forceinline__ void stream_rows(const double *__restrict__ src, size_t stride, int RT,
                                            double *ring, int lane, F &&f) {
	static_assert(LW % 2 == 0, "rows are copied 16 bytes at a time");
	double *mine = ring + lane * LW;
	auto issue = [&](int rt) {
		const double *g = src + (size_t)rt * stride;
		double *d = mine + (rt % NORM_RING) * TILE;
#pragma unroll
		for (int k = 0; k < LW; k += 2)
			cp_async16(d + k, g + k);
	};
#pragma unroll
	for (int k = 0; k < NORM_RING - 1; ++k) {
		if (k < RT)
			issue(k);
		cp_async_commit();
	}
	for (int rt = 0; rt < RT; ++rt) {
		if (rt + NORM_RING - 1 < RT)
			issue(rt + NORM_RING - 1);
		cp_async_commit();
		cp_async_wait<NORM_RING - 1>();   // the group of row rt has landed
		double v[LW];
		const double *d = mine + (rt % NORM_RING) * TILE;
#pragma unroll
		for (int k = 0; k < LW; k += 2) {
			const double2 x = *reinterpret_cast<const double2 *>(d + k);
			v[k] = x.x;
			v[k + 1] = x.y;
		}
		f(rt, v);
	}
	cp_async_wait<0>();
}

// One warp per frame. The reference visits orientations in ascending order
// with a running maximum m (max_prob.c:184-203): a pair enters the kept list
// when pval + 14/beta > m and, when pval > m, the list is pruned to entries
// > pval - 14/beta. With one thread the final list is: every r up to the first
// maximiser r* with pval > max - 14/beta, and every r after r* with
// pval + 14/beta > max. The maximiser is the lowest index reaching the maximum;
// it comes from the per-tile maxima the E-step wrote (lanes take tiles lane,
// lane + 32, ...). P_dr = exp(beta (pval - max)) / p_norm (max_update.c:96-98),
// formed as a product with 1 / p_norm; likelihood, psum_d, info and quat_norm
// follow max_update.c:105-130, with log(P / w_r * M) written as
// beta (pval - max) - log p_norm + log M - log w_r so that no pair evaluates a
// logarithm. The two passes over a frame's log-likelihoods keep UNR tile rows
// in flight per lane. With Pd given (background-aware path) P is also stored
// in FP64, with the same sign convention as Pst.
#ifndef DFG_NORM_MINB
#define DFG_NORM_MINB 4
#endif
// ONE (without tile skipping or the FP64 copy): one exp per kept pair. The
// first pass stores E = exp(beta (pval - max)) in FP32 in Pst and sums, per
// frame and in FP64, E, E pval, E u_r, E (y - log w_r) and E per mode; the
// second pass reads E back, writes P = E / p_norm with the sign gate and takes
// the pairs with P < PROB_MIN (which info and quat_norm leave out) back out of
// those sums. Then likelihood = sum E pval / p_norm - sum_fact, psum_d =
// rescale sum E u_r / p_norm and info = (sum' E (y - log w_r) + (log M -
// log p_norm) sum' E) / p_norm over the pairs with P >= PROB_MIN -- the
// reference's per-pair sums (max_update.c:96-130), regrouped.
template <bool MULTI, bool SKIP, bool ONE = false>
__global__ void __launch_bounds__(256, DFG_NORM_MINB) norm_kernel(
    const double *__restrict__ pval, const double *__restrict__ tmax, const int *__restrict__ targ, int RT,
    int Nc, int d0, int R, int M, const double *__restrict__ logw, const double *__restrict__ u,
    const double *__restrict__ beta, const double *__restrict__ sum_fact, const uint8_t *__restrict__ blacklist,
    int psum_d_on, const double *__restrict__ scalars, float *__restrict__ Pst, int *__restrict__ rmax,
    double *__restrict__ max_exp, double *__restrict__ p_norm, double *__restrict__ info,
    double *__restrict__ likelihood, double *__restrict__ psum_d, double *__restrict__ quat_norm,
    int *__restrict__ num_prob, double *__restrict__ Pd, uint8_t *__restrict__ tlive, int zero_dead) {
	constexpr int UNR = LW == 1 ? 4 : 2;
	// without tile skipping every row of the frame is read, twice: both passes
	// stream them through a per-warp ring (stream_rows)
	__shared__ __align__(16) double s_ring[SKIP ? 1 : 8][SKIP ? 1 : NORM_RING * TILE];
	const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	const size_t tstride = (size_t)Nc * TILE, pstride = (size_t)(Nc + 1) * TILE;
	float zero[LW];
#pragma unroll
	for (int k = 0; k < LW; ++k)
		zero[k] = 0.f;
	double zerod[LW];
#pragma unroll
	for (int k = 0; k < LW; ++k)
		zerod[k] = 0.;
	const size_t lstride = (size_t)Nc + 1;  // tlive [RT][Nc + 1]
	if (warp == Nc) {  // the zero row that padding words of the M-step point at
		for (int rt = 0; rt < RT; ++rt) {
			st_row(Pst + rt * pstride + (size_t)Nc * TILE + lane * LW, zero);
			if (Pd != nullptr)
				st_row(Pd + rt * pstride + (size_t)Nc * TILE + lane * LW, zerod);
			if (SKIP && lane == 0)
				tlive[rt * lstride + Nc] = 0;
		}
		return;
	}
	if (warp > Nc)
		return;
	const int dl = warp, d = d0 + dl;
	const double *pv = pval + (size_t)dl * TILE + lane * LW;
	float *ps = Pst + (size_t)dl * TILE + lane * LW;
	const bool bl = blacklist[d] != 0;

	double m = MAX_EXP_START;
	int am = -1;
	if (!bl) {
		for (int rt = lane; rt < RT; rt += 32) {
			double v = tmax[(size_t)rt * Nc + dl];
			if (v > m) {
				m = v;
				am = targ[(size_t)rt * Nc + dl];
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
		for (int rt = 0; rt < RT; ++rt) {
			if (!SKIP || zero_dead) {
				st_row(ps + rt * pstride, zero);
				if (Pd != nullptr)
					st_row(Pd + (size_t)dl * TILE + lane * LW + rt * pstride, zerod);
			}
			if (SKIP && lane == 0)
				tlive[rt * lstride + dl] = 0;
		}
		if (lane == 0) {
			rmax[d] = -1;
			max_exp[d] = MAX_EXP_START;
			p_norm[d] = 0.;
			info[d] = 0.;
			likelihood[d] = 0.;
			psum_d[d] = 0.;
			num_prob[d] = 0;
		}
		if (MULTI && lane < M)
			quat_norm[(size_t)d * M + lane] = 0.;
		return;
	}
	const double b = beta[d];
	const double thr = PDIFF_THRESH / b;
	const double lo = dsub(m, thr);
	const int rstar = am;

	// a tile whose maximum can keep no pair is dead: its log-likelihoods are
	// not read, its probabilities are zero (written only with zero_dead), and
	// tlive tells the later phases to skip it
	auto dead = [&](int rt) {
		if constexpr (!SKIP)
			return false;
		const double t = tmax[(size_t)rt * Nc + dl];
		return !(t > lo) && !(dadd(t, thr) > m);
	};
	if constexpr (ONE) {
		static_assert(!SKIP, "the one-exp form reads every row");
		double s = 0., sx = 0., su = 0., sy = 0.;
		double qe[MULTI ? MAX_MODES : 1];
#pragma unroll
		for (int k = 0; k < (MULTI ? MAX_MODES : 1); ++k)
			qe[k] = 0.;
		int cnt = 0;
		stream_rows(pv, tstride, RT, s_ring[threadIdx.x >> 5], lane, [&](int rt, const double (&v)[LW]) {
			float out[LW];
#pragma unroll
			for (int e = 0; e < LW; ++e) {
				const int r = rt * TILE + lane * LW + e;
				out[e] = 0.f;
				if (r < R) {
					const double x = v[e];
					const bool kept = (r <= rstar) ? (x > lo) : (dadd(x, thr) > m);
					if (kept) {
						const double y = dmul(b, dsub(x, m));
						const double E = exp(y);
						s += E;
						sx += E * x;
						if (psum_d_on)
							su += E * u[r];
						sy += E * (y - logw[r]);
						if (MULTI) {
							const int mode = r % M;
#pragma unroll
							for (int q = 0; q < (MULTI ? MAX_MODES : 1); ++q)
								if (q == mode)
									qe[q] += E;
						}
						cnt++;
						out[e] = (float)E;   // kept pairs have y > -14: a normal FP32 value
					}
				}
			}
			st_row(ps + rt * pstride, out);
		});
		s = warp_sum(s);
		for (int o = 16; o > 0; o >>= 1)
			cnt += __shfl_xor_sync(FULL, cnt, o);
		const double inv_s = 1. / s;
		const float inv_sf = (float)inv_s;
		// second pass: this lane's own FP32 values of the first pass, four rows
		// in flight
		double ys = 0., es = 0.;
		double qs[MULTI ? MAX_MODES : 1];
#pragma unroll
		for (int k = 0; k < (MULTI ? MAX_MODES : 1); ++k)
			qs[k] = 0.;
		constexpr int R2 = 4;
		for (int rt0 = 0; rt0 < RT; rt0 += R2) {
			float ev[R2][LW];
#pragma unroll
			for (int k = 0; k < R2; ++k)
				if (rt0 + k < RT)
					ld_row_rw(ps + (rt0 + k) * pstride, ev[k]);
#pragma unroll
			for (int k = 0; k < R2; ++k) {
				const int rt = rt0 + k;
				if (rt >= RT)
					break;
				float out[LW];
#pragma unroll
				for (int e = 0; e < LW; ++e) {
					const float E = ev[k][e];
					const float P = E * inv_sf;
					out[e] = (P > (float)PROB_MIN) ? P : -P;
					if (E > 0.f && (double)E * inv_s < PROB_MIN) {
						// a kept pair that info and quat_norm leave out
						const int r = rt * TILE + lane * LW + e;
						es += (double)E;
						ys += (double)E * ((double)logf(E) - logw[r]);
						if (MULTI) {
							const int mode = r % M;
#pragma unroll
							for (int q = 0; q < (MULTI ? MAX_MODES : 1); ++q)
								if (q == mode)
									qs[q] += (double)E;
						}
					}
				}
				st_row(ps + rt * pstride, out);
			}
		}
		sx = warp_sum(sx);
		su = warp_sum(su);
		sy = warp_sum(sy);
		ys = warp_sum(ys);
		es = warp_sum(es);
		const double rescale = scalars[0], sf = sum_fact[d];
		const double cinf = log((double)M) - log(s);
		if (MULTI) {
			for (int k = 0; k < M && k < MAX_MODES; ++k) {
				const double v = warp_sum(qe[k]) - warp_sum(qs[k]);
				if (lane == 0)
					quat_norm[(size_t)d * M + k] = v * inv_s;
			}
		}
		if (lane == 0) {
			rmax[d] = rstar;
			max_exp[d] = m;
			p_norm[d] = s;
			likelihood[d] = sx * inv_s - sf;
			info[d] = ((sy - ys) + cinf * (s - es)) * inv_s;
			psum_d[d] = psum_d_on ? rescale * su * inv_s : 0.;
			num_prob[d] = cnt;
		}
		return;
	}
	double s = 0.;
	int cnt = 0;
	if constexpr (!SKIP) {
		stream_rows(pv, tstride, RT, s_ring[threadIdx.x >> 5], lane, [&](int rt, const double (&v)[LW]) {
#pragma unroll
			for (int e = 0; e < LW; ++e) {
				const int r = rt * TILE + lane * LW + e;
				if (r < R) {
					bool kept = (r <= rstar) ? (v[e] > lo) : (dadd(v[e], thr) > m);
					if (kept) {
						s += exp(dmul(b, dsub(v[e], m)));
						cnt++;
					}
				}
			}
		});
	} else
	for (int rt0 = 0; rt0 < RT; rt0 += UNR) {
		double v[UNR][LW];
		bool dd[UNR];
#pragma unroll
		for (int k = 0; k < UNR; ++k) {
			if constexpr (SKIP) {
				dd[k] = rt0 + k >= RT || dead(rt0 + k);
				if (!dd[k])
					ld_row(pv + (rt0 + k) * tstride, v[k]);
			} else {
				dd[k] = false;
				if (rt0 + k < RT)
					ld_row(pv + (rt0 + k) * tstride, v[k]);
			}
		}
#pragma unroll
		for (int k = 0; k < UNR; ++k) {
			if (rt0 + k >= RT)
				break;
			if (SKIP && dd[k])
				continue;
#pragma unroll
			for (int e = 0; e < LW; ++e) {
				const int r = (rt0 + k) * TILE + lane * LW + e;
				if (r < R) {
					bool kept = (r <= rstar) ? (v[k][e] > lo) : (dadd(v[k][e], thr) > m);
					if (kept) {
						s += exp(dmul(b, dsub(v[k][e], m)));
						cnt++;
					}
				}
			}
		}
	}
	s = warp_sum(s);
	for (int o = 16; o > 0; o >>= 1)
		cnt += __shfl_xor_sync(FULL, cnt, o);

	const double rescale = scalars[0], sf = sum_fact[d];
	const double inv_s = 1. / s, cinf = log((double)M) - log(s);
	double ll = 0., pd = 0., inf = 0.;
	double qn[MULTI ? MAX_MODES : 1];
#pragma unroll
	for (int k = 0; k < (MULTI ? MAX_MODES : 1); ++k)
		qn[k] = 0.;
	// one kept or dropped pair of the second pass: P, the frame sums, and the
	// stored probability (sign = PROB_MIN gate)
	auto pair2 = [&](int r, double x, float &out, double &outd) {
		out = 0.f;
		outd = 0.;
		if (r < R) {
			bool kept = (r <= rstar) ? (x > lo) : (dadd(x, thr) > m);
			if (kept) {
				const double y = dmul(b, dsub(x, m));
				const double P = exp(y) * inv_s;
				ll += P * (x - sf);
				if (psum_d_on)
					pd += P * u[r] * rescale;
				if (!(P < PROB_MIN)) {
					inf += P * (y + cinf - logw[r]);
					if (MULTI) {
						int mode = r % M;
#pragma unroll
						for (int q = 0; q < (MULTI ? MAX_MODES : 1); ++q)
							if (q == mode)
								qn[q] += P;
					}
				}
				out = (P > PROB_MIN) ? (float)P : -(float)P;
				outd = (P > PROB_MIN) ? P : -P;
			}
		}
	};
	if constexpr (!SKIP) {
		stream_rows(pv, tstride, RT, s_ring[threadIdx.x >> 5], lane, [&](int rt, const double (&v)[LW]) {
			float out[LW];
			double outd[LW];
#pragma unroll
			for (int e = 0; e < LW; ++e)
				pair2(rt * TILE + lane * LW + e, v[e], out[e], outd[e]);
			st_row(ps + rt * pstride, out);
			if (Pd != nullptr)
				st_row(Pd + (size_t)dl * TILE + lane * LW + rt * pstride, outd);
		});
	} else
	for (int rt0 = 0; rt0 < RT; rt0 += UNR) {
		double v[UNR][LW];
		bool dd[UNR];
#pragma unroll
		for (int k = 0; k < UNR; ++k) {
			if constexpr (SKIP) {
				dd[k] = rt0 + k >= RT || dead(rt0 + k);
				if (!dd[k])
					ld_row(pv + (rt0 + k) * tstride, v[k]);
			} else {
				dd[k] = false;
				if (rt0 + k < RT)
					ld_row(pv + (rt0 + k) * tstride, v[k]);
			}
		}
#pragma unroll
		for (int k = 0; k < UNR; ++k) {
			const int rt = rt0 + k;
			if (rt >= RT)
				break;
			if (SKIP && lane == 0)
				tlive[rt * lstride + dl] = dd[k] ? 0 : 1;
			if (SKIP && dd[k]) {
				if (zero_dead) {
					st_row(ps + rt * pstride, zero);
					if (Pd != nullptr)
						st_row(Pd + (size_t)dl * TILE + lane * LW + rt * pstride, zerod);
				}
				continue;
			}
			float out[LW];
			double outd[LW];
#pragma unroll
			for (int e = 0; e < LW; ++e)
				pair2(rt * TILE + lane * LW + e, v[k][e], out[e], outd[e]);
			st_row(ps + rt * pstride, out);
			if (Pd != nullptr)
				st_row(Pd + (size_t)dl * TILE + lane * LW + rt * pstride, outd);
		}
	}
	ll = warp_sum(ll);
	pd = warp_sum(pd);
	inf = warp_sum(inf);
	if (MULTI) {
		for (int k = 0; k < M && k < MAX_MODES; ++k) {
			double v = warp_sum(qn[k]);
			if (lane == 0)
				quat_norm[(size_t)d * M + k] = v;
		}
	}
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

// psum_r partials: sum over a frame range of |Pst| * (phi_d or 1)
// (max_update.c:108-116). Grid (RT, splits), 8 warps per block; fixed order.
__global__ void __launch_bounds__(256) psum_r_kernel(const float *__restrict__ Pst, int Nc, int d0,
                                                      int frames_per_split, const double *__restrict__ scale,
                                                      int need_scaling, double *__restrict__ part, int R_pad,
                                                      const uint8_t *__restrict__ tlive) {
	__shared__ double s[8][TILE];
	const int rt = blockIdx.x, split = blockIdx.y, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int beg = split * frames_per_split, end = min(Nc, beg + frames_per_split);
	double acc[LW];
#pragma unroll
	for (int k = 0; k < LW; ++k)
		acc[k] = 0.;
	const float *p = Pst + (size_t)rt * (Nc + 1) * TILE + lane * LW;
	const uint8_t *live = tlive ? tlive + (size_t)rt * (Nc + 1) : nullptr;
	for (int dl = beg + w; dl < end; dl += 8) {
		if (live && !live[dl])  // dead tile: no probability (norm_kernel with tile skipping)
			continue;
		float v[LW];
		ld_row(p + (size_t)dl * TILE, v);
		const double f = need_scaling ? scale[d0 + dl] : 1.;
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
		part[(size_t)split * R_pad + rt * TILE + j] = t;
	}
}

__global__ void psum_r_reduce_kernel(const double *__restrict__ part, int nsplit, int R, int R_pad,
                                     double *__restrict__ psum_r) {
	int r = blockIdx.x * blockDim.x + threadIdx.x;
	if (r >= R)
		return;
	double s = 0.;
	for (int k = 0; k < nsplit; ++k)
		s += part[(size_t)k * R_pad + r];
	psum_r[r] += s;
}

// ---------------------------------------------------------------------------
// (e1) M-step back-projection: T[tile][p][j] += sum_(d,c) c * P_dr
// ---------------------------------------------------------------------------
// Gather form of update_tomogram_nobg (max_update.c:142-230): one warp per
// (orientation tile, pixel), walking the pixel's list of frames (pixels with
// mask < 2 only) and reading one row of P per entry (one LW-wide vector load
// per lane); count-1 and multi-photon segments as in the E-step, compensated
// FP32 sums, two orientations per paired FP32 instruction (this kernel is
// bound by instruction issue; the E-step, bound by L2, gains nothing from
// pairing). No atomics; pixels are visited heaviest first for balance.
constexpr int MSTEP_MINB = LW == 4 ? 4 : 6;

template <bool SKIP, int MINB = MSTEP_MINB>
__global__ void __launch_bounds__(256, MINB) mstep_kernel(const float *__restrict__ Pst, int Nc,
                                                     const uint32_t *__restrict__ cs,
                                                     const long long *__restrict__ cs_off,
                                                     const long long *__restrict__ cs_mid,
                                                     const int *__restrict__ pix, int npix, int P, int RT,
                                                     float *__restrict__ T, const uint8_t *__restrict__ tlive,
                                                     int t0 = 0) {
	// RT tiles from tile t0 (orientation blocks: T holds tiles t0 ..)
	const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (warp >= (long long)RT * npix)
		return;
	const int rl = (int)(warp / npix), kp = (int)(warp - (long long)rl * npix), rt = t0 + rl;
	const int p = pix[kp];
	const float *Pr = Pst + (size_t)rt * (Nc + 1) * TILE + lane * LW;
	// SKIP: frames whose tile is dead (norm_kernel) read the chunk's zero row
	// instead (cached), so their probability rows are never fetched
	const uint8_t *live = tlive + (size_t)rt * (Nc + 1);
	const uint32_t zrow = (uint32_t)Nc;
	auto lv = [&](uint32_t f) {
		if constexpr (SKIP)
			return live[f] ? f : zrow;
		else
			return f;
	};
	const long long beg = cs_off[p], mid = cs_mid[p], end = cs_off[p + 1];
	const uint4 *w4 = reinterpret_cast<const uint4 *>(cs);
	float s[ECH][LW], c[ECH][LW];
#pragma unroll
	for (int h = 0; h < ECH; ++h)
#pragma unroll
		for (int k = 0; k < LW; ++k)
			s[h][k] = c[h][k] = 0.f;
	if constexpr (LW >= 2) {
		// orientations in pairs: paired FP32 compensated additions; the next
		// 8 words are fetched while the current 8 rows are in flight
		constexpr int NP = NPAIR;
		f32x2 s2[NP], c2[NP];
#pragma unroll
		for (int h = 0; h < NP; ++h)
			s2[h] = c2[h] = 0ull;
		uint4 a = make_uint4(Nc, Nc, Nc, Nc), b = a;
		if (beg < mid) {
			a = __ldg(w4 + (beg >> 2));
			b = __ldg(w4 + (beg >> 2) + 1);
		}
		for (long long j = beg; j < mid; j += 8) {
			if constexpr (SKIP) {
				// a group of 8 frames without a live tile adds nothing
				if (!(live[a.x] | live[a.y] | live[a.z] | live[a.w] | live[b.x] | live[b.y] | live[b.z] |
				      live[b.w])) {
					if (j + 8 < mid) {
						a = __ldg(w4 + ((j + 8) >> 2));
						b = __ldg(w4 + ((j + 8) >> 2) + 1);
					}
					continue;
				}
			}
			f32x2 v[8][NP];
			ld_pairs(Pr + lv(a.x) * TILE, v[0]);
			ld_pairs(Pr + lv(a.y) * TILE, v[1]);
			ld_pairs(Pr + lv(a.z) * TILE, v[2]);
			ld_pairs(Pr + lv(a.w) * TILE, v[3]);
			ld_pairs(Pr + lv(b.x) * TILE, v[4]);
			ld_pairs(Pr + lv(b.y) * TILE, v[5]);
			ld_pairs(Pr + lv(b.z) * TILE, v[6]);
			ld_pairs(Pr + lv(b.w) * TILE, v[7]);
			if (j + 8 < mid) {
				a = __ldg(w4 + ((j + 8) >> 2));
				b = __ldg(w4 + ((j + 8) >> 2) + 1);
			}
#pragma unroll
			for (int q = 0; q < 8; ++q)
#pragma unroll
				for (int h = 0; h < NP; ++h) {
					float lo, hi;
					f2_unpack(v[q][h], lo, hi);
					kahan_add2(s2[h], c2[h], f2_pack(fmaxf(lo, 0.f), fmaxf(hi, 0.f)));
				}
		}
		for (long long j = mid; j < end; j += 8) {
			const uint4 a = __ldg(w4 + (j >> 2)), b = __ldg(w4 + (j >> 2) + 1);
			const uint32_t e[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
			if constexpr (SKIP) {
				uint32_t any = 0;
#pragma unroll
				for (int q = 0; q < 8; ++q)
					any |= live[e[q] & IDX_MASK];
				if (!any)
					continue;
			}
			f32x2 v[8][NP];
#pragma unroll
			for (int q = 0; q < 8; ++q)
				ld_pairs(Pr + lv(e[q] & IDX_MASK) * TILE, v[q]);
#pragma unroll
			for (int q = 0; q < 8; ++q)
#pragma unroll
				for (int h = 0; h < NP; ++h) {
					float lo, hi;
					f2_unpack(v[q][h], lo, hi);
					kahan_add_count2(s2[h], c2[h], e[q] >> IDX_BITS, f2_pack(fmaxf(lo, 0.f), fmaxf(hi, 0.f)));
				}
		}
#pragma unroll
		for (int h = 0; h < NP; ++h) {
			f2_unpack(s2[h], s[0][2 * h], s[0][2 * h + 1]);
			f2_unpack(c2[h], c[0][2 * h], c[0][2 * h + 1]);
		}
	} else {
#pragma unroll 2
	for (long long j = beg; j < mid; j += 8) {
		const uint4 a = __ldg(w4 + (j >> 2)), b = __ldg(w4 + (j >> 2) + 1);
		float v[8][LW];
		ld_row(Pr + lv(a.x) * TILE, v[0]);
		ld_row(Pr + lv(a.y) * TILE, v[1]);
		ld_row(Pr + lv(a.z) * TILE, v[2]);
		ld_row(Pr + lv(a.w) * TILE, v[3]);
		ld_row(Pr + lv(b.x) * TILE, v[4]);
		ld_row(Pr + lv(b.y) * TILE, v[5]);
		ld_row(Pr + lv(b.z) * TILE, v[6]);
		ld_row(Pr + lv(b.w) * TILE, v[7]);
#pragma unroll
		for (int q = 0; q < 8; ++q)
#pragma unroll
			for (int k = 0; k < LW; ++k)
				kahan_add(s[q % ECH][k], c[q % ECH][k], fmaxf(v[q][k], 0.f));
	}
	for (long long j = mid; j < end; j += 8) {
		const uint4 a = __ldg(w4 + (j >> 2)), b = __ldg(w4 + (j >> 2) + 1);
		const uint32_t e[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
		float v[8][LW];
#pragma unroll
		for (int q = 0; q < 8; ++q)
			ld_row(Pr + lv(e[q] & IDX_MASK) * TILE, v[q]);
#pragma unroll
		for (int q = 0; q < 8; ++q)
#pragma unroll
			for (int k = 0; k < LW; ++k)
				kahan_add_count(s[q % ECH][k], c[q % ECH][k], e[q] >> IDX_BITS, fmaxf(v[q][k], 0.f));
	}
	}
	float *out = T + ((size_t)rl * P + p) * TILE + lane * LW;
	float o[LW];
	ld_row_rw(out, o);
#pragma unroll
	for (int k = 0; k < LW; ++k) {
		double t = kahan_value(s[0][k], c[0][k]);
		if (ECH == 2)
			t = dadd(t, kahan_value(s[ECH - 1][k], c[ECH - 1][k]));
		o[k] = (float)((double)o[k] + t);
	}
	st_row(out, o);
}

// ---------------------------------------------------------------------------
// (e2) merge: slice_merge3d of tomo_r / psum_r for every r with psum_r > 0
// ---------------------------------------------------------------------------
// Block = orientation tile x PB pixels (same thread layout as slice_log_kernel).
// The tile's tomogram rows are staged through shared memory; each
// (pixel, orientation) with mask <= 1 and in bounds adds (f * w, f) to its 8
// corners (model.c:171-244, max_update.c:33-36). The accumulators are FP64
// (model, weight) pairs, interleaved so both atomics of a corner hit one
// 32-byte sector: FP32 sums of thousands of contributions per voxel would
// carry ~1e-6 relative error into the next iteration's likelihoods.
// The weight sum depends only on which orientations have psum_r > 0; when
// that set is the one of a cached weight grid, with_weight is 0 and only the
// model sums are accumulated. With views_final the tomograms already are the
// views (background-aware update) and are not divided by psum_r.
// INCR (pair lists): zero tomogram values add nothing and are skipped, and
// the weights are a change to the cached grid: wsign[r] = +1 / -1 adds /
// subtracts orientation r's weights (its psum_r > 0 state changed, or +1 for
// every orientation with psum_r > 0 when no grid is cached), 0 adds none.
// The full merge's scatter with warp aggregation: the 32 lanes of a warp hold
// 32 consecutive pixels of one orientation (j = g + 4 k is the same for the
// warp), and neighbouring pixels often fall in the same trilinear cell.
// Lanes whose cells coincide (__match_any_sync on the cell index) add their
// corner contributions in registers, in lane order, and the group's lowest
// lane issues one atomic per corner for the group.
template <int GEO>
__device__ __forceinline__ void merge_aggregated(const float (*s_tile)[TILE + 1], const double *s_ps,
                                                 const double (*s_rot)[9], const int *s_mode, int i, int g, int p,
                                                 int P, const double *__restrict__ qvals,
                                                 const double *__restrict__ corr, const uint8_t *__restrict__ mask,
                                                 long long S, long long V, double *__restrict__ accum,
                                                 int with_weight, int views_final) {
	const int lane = threadIdx.x & 31;
	const bool pix = p < P && mask[p] <= 1;
	const int pp = pix ? p : 0;
	const double qx = qvals[3 * (size_t)pp], qy = qvals[3 * (size_t)pp + 1], qz = qvals[3 * (size_t)pp + 2];
	const double cr = corr[pp];
	const double center = (double)(S / 2);
	constexpr int NC = GEO == MT_3D ? 8 : 4;  // corners
	// corner q's offset from the cell's first voxel (corner_offsets order)
	auto off = [S](int q) -> long long {
		if constexpr (GEO == MT_3D)
			return (long long)(q & 1) + ((q >> 1) & 1) * S + (long long)(q >> 2) * S * S;
		else
			return (long long)(q & 1) + (long long)(q >> 1) * S;
	};
	for (int k = 0; k < TILE / 4; ++k) {
		const int j = g + 4 * k;   // the same for every lane of the warp
		const double ps = s_ps[j];
		if (!(ps > 0.))
			continue;
		double fw[8];
		long long base = -1;
		bool ok = false;
		if (pix) {
			if constexpr (GEO == MT_3D) {
				Cell c = locate(s_rot[j], qx, qy, qz, center, S);
				ok = c.ok;
				if (ok) {
					corner_weights(c, fw);
					base = c.i000;
				}
			} else {
				Cell2 c = locate2d(s_rot[j], qx, qy, center, S);
				ok = c.ok;
				if (ok) {
					corner_weights2(c, fw);
					base = c.i00;
				}
			}
		}
		if (!__any_sync(FULL, ok))
			continue;
		if (!ok) {
#pragma unroll
			for (int q = 0; q < NC; ++q)
				fw[q] = 0.;
			base = -1 - lane;    // a group of its own
		}
		const double wv = views_final ? (double)s_tile[i][j] / cr : ((double)s_tile[i][j] / ps) / cr;
		const unsigned grp = __match_any_sync(FULL, base);
		const int members = __popc(grp);
		const int most = (int)__reduce_max_sync(FULL, (unsigned)members);
		const bool lead = ok && (__ffs(grp) - 1) == lane;
		double *a = accum + 2 * ((size_t)s_mode[j] * V + (ok ? base : 0));
		// model sums (slot 0), then with_weight the weights (slot 1): the
		// group's lanes in lane order, summed by the lowest lane
		for (int h = 0; h < (with_weight ? 2 : 1); ++h) {
			double v[8];
#pragma unroll
			for (int q = 0; q < NC; ++q)
				v[q] = h == 0 ? fw[q] * wv : fw[q];
			for (int m = 1; m < most; ++m) {
				// the group's m-th lane, or this lane when the group is smaller
				const int src = m < members ? (int)__fns(grp, 0, m + 1) : lane;
#pragma unroll
				for (int q = 0; q < NC; ++q) {
					const double x = __shfl_sync(FULL, h == 0 ? fw[q] * wv : fw[q], src);
					if (m < members)
						v[q] += x;
				}
			}
			if (lead) {
#pragma unroll
				for (int q = 0; q < NC; ++q)
					atomicAdd(a + 2 * off(q) + h, v[q]);
			}
		}
	}
}

template <int GEO, bool INCR = false>
__global__ void __launch_bounds__(256, 3) merge_kernel(const float *__restrict__ T,
                                                     const double *__restrict__ psum_r,
                                                     const double *__restrict__ quats, int M, int R,
                                                     const double *__restrict__ qvals,
                                                     const double *__restrict__ corr,
                                                     const uint8_t *__restrict__ mask, int P, long long S,
                                                     long long V, double *__restrict__ accum,
                                                     const int *__restrict__ weight_flag,
                                                     int views_final, const signed char *__restrict__ wsign = nullptr) {
	__shared__ double s_rot[TILE][9];
	__shared__ int s_mode[TILE];
	__shared__ double s_ps[TILE];
	__shared__ signed char s_sg[INCR ? TILE : 1];
	__shared__ float s_tile[PB][TILE + 1];
	const int t = threadIdx.x, rt = blockIdx.y, p0 = blockIdx.x * PB;
	const int with_weight = *weight_flag;
	for (int j = t; j < TILE; j += blockDim.x) {
		int r = rt * TILE + j;
		int rr = r < R ? r : 0;
		geo_setup<GEO>(quats, rr / M, s_rot[j]);
		s_mode[j] = rr % M;
		s_ps[j] = r < R ? psum_r[r] : 0.;
		if constexpr (INCR)
			s_sg[j] = r < R ? wsign[r] : 0;
	}
	{
		const int w = t >> 5, lane = t & 31;
		for (int row = w; row < PB; row += 8) {
			int pp = p0 + row;
			float v[LW];
			if (pp < P) {
				ld_row(T + ((size_t)rt * P + pp) * TILE + lane * LW, v);
			} else {
#pragma unroll
				for (int k = 0; k < LW; ++k)
					v[k] = 0.f;
			}
#pragma unroll
			for (int k = 0; k < LW; ++k)
				s_tile[row][lane * LW + k] = v[k];
		}
	}
	__syncthreads();
	const int i = t & (PB - 1), g = t >> 6, p = p0 + i;
	if constexpr (!INCR) {
		merge_aggregated<GEO>(s_tile, s_ps, s_rot, s_mode, i, g, p, P, qvals, corr, mask, S, V, accum,
		                      with_weight, views_final);
		return;
	}
	if (p >= P || mask[p] > 1)
		return;
	const double qx = qvals[3 * (size_t)p], qy = qvals[3 * (size_t)p + 1], qz = qvals[3 * (size_t)p + 2];
	const double cr = corr[p];
	const double center = (double)(S / 2);
	constexpr int NC = GEO == MT_3D ? 8 : 4;  // corners
	long long o[8];
	if constexpr (GEO == MT_3D) {
		corner_offsets(S, o);
	} else {
		o[0] = 0; o[1] = 1; o[2] = S; o[3] = S + 1;
	}
	for (int k = 0; k < TILE / 4; ++k) {
		const int j = g + 4 * k;
		const double ps = s_ps[j];
		bool model = ps > 0.;
		int sg = 0;
		if constexpr (INCR) {
			sg = s_sg[j];
			model = model && s_tile[i][j] != 0.f;
			if (!model && sg == 0)
				continue;
		} else if (!model) {
			continue;
		}
		double fw[8];
		long long base;
		if constexpr (GEO == MT_3D) {
			Cell c = locate(s_rot[j], qx, qy, qz, center, S);
			if (!c.ok)
				continue;
			corner_weights(c, fw);
			base = c.i000;
		} else {
			Cell2 c = locate2d(s_rot[j], qx, qy, center, S);
			if (!c.ok)
				continue;
			corner_weights2(c, fw);
			base = c.i00;
		}
		double *a = accum + 2 * ((size_t)s_mode[j] * V + base);
		if constexpr (INCR) {
			if (model) {
				const double wv = ((double)s_tile[i][j] / ps) / cr;
#pragma unroll
				for (int q = 0; q < NC; ++q)
					atomicAdd(a + 2 * o[q], fw[q] * wv);
			}
			if (sg != 0) {
#pragma unroll
				for (int q = 0; q < NC; ++q)
					atomicAdd(a + 2 * o[q] + 1, sg > 0 ? fw[q] : -fw[q]);
			}
			continue;
		}
		const double wv = views_final ? (double)s_tile[i][j] / cr : ((double)s_tile[i][j] / ps) / cr;
		if (with_weight) {
#pragma unroll
			for (int q = 0; q < NC; ++q) {
				atomicAdd(a + 2 * o[q], fw[q] * wv);
				atomicAdd(a + 2 * o[q] + 1, fw[q]);
			}
		} else {
#pragma unroll
			for (int q = 0; q < NC; ++q)
				atomicAdd(a + 2 * o[q], fw[q] * wv);
		}
	}
}

// ---------------------------------------------------------------------------
// model update (recon.pyx:112-149) and small per-frame kernels
// ---------------------------------------------------------------------------
// Whether the merge must accumulate weights: the set of orientations with
// psum_r > 0 (the only input of the weight grid once the geometry is fixed)
// differs from the one of the cached grid, or no grid is cached. flags[0] =
// accumulate weights, flags[1] = a grid is cached (cleared by the host when
// the geometry changes). One block; the pattern is updated in place.
__global__ void __launch_bounds__(1024) weight_pattern_kernel(const double *__restrict__ psum_r, int R,
                                                              uint8_t *__restrict__ pattern, int *__restrict__ flags) {
	int changed = 0;
	for (int r = threadIdx.x; r < R; r += blockDim.x) {
		const uint8_t p = psum_r[r] > 0. ? 1 : 0;
		if (p != pattern[r]) {
			pattern[r] = p;
			changed = 1;
		}
	}
	changed = __syncthreads_or(changed);
	if (threadIdx.x == 0) {
		flags[0] = (changed || flags[1] == 0) ? 1 : 0;
		flags[1] = 1;
	}
}

// Pair lists: the weight change of this merge. sign[r] = +1 for every
// orientation with psum_r > 0 when no grid is cached (flags[0] = 1), else
// the change of its psum_r > 0 state against the cached grid's (flags[0] =
// 2: the merge's weight sums are added to the cached grid). One block.
__global__ void __launch_bounds__(1024) weight_sign_kernel(const double *__restrict__ psum_r, int R,
                                                           uint8_t *__restrict__ pattern,
                                                           signed char *__restrict__ sign, int *__restrict__ flags) {
	const bool full = flags[1] == 0;
	for (int r = threadIdx.x; r < R; r += blockDim.x) {
		const uint8_t p = psum_r[r] > 0. ? 1 : 0;
		sign[r] = full ? (signed char)p : (signed char)((int)p - (int)pattern[r]);
		pattern[r] = p;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		flags[0] = full ? 1 : 2;
		flags[1] = 1;
	}
}

// model2 / inter_weight from the accumulators; the weights come from this
// merge (flag 1), from weight_cache (flag 0) or from weight_cache plus this
// merge's change (flag 2); weight_cache keeps the result.
__global__ void unpack_accum_kernel(const double2 *__restrict__ accum, long long n, double *__restrict__ model2,
                                    double *__restrict__ weight, double *__restrict__ weight_cache,
                                    const int *__restrict__ weight_flag) {
	long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	const int with_weight = *weight_flag;
	double2 a = accum[i];
	model2[i] = a.x;
	if (with_weight == 1) {
		weight[i] = a.y;
		weight_cache[i] = a.y;
	} else if (with_weight == 2) {
		const double w = weight_cache[i] + a.y;
		weight[i] = w;
		weight_cache[i] = w;
	} else {
		weight[i] = weight_cache[i];
	}
}

__device__ __forceinline__ double friedel_avg(double a1, double w1, double a2, double w2) {
	double a = dmul(0.5, dadd(dmul(a1, w1), dmul(a2, w2)));
	double ws = dmul(0.5, dadd(w1, w2));
	return ws > 0 ? a / ws : 0.;
}

// symmetrize_friedel (model.c:470-490) over every mode. The reference visits
// (x, y, z) for x, y in [lo, S), z in [lo, c] sequentially; pairs with z < c
// are touched once, pairs inside the z == c plane twice (the second visit
// starts from the first member's result with the roles swapped). Each thread
// owns one pair and replays exactly those visits.
__global__ void friedel_kernel(double *__restrict__ model2, const double *__restrict__ weight, int S, int M) {
	const int c = S / 2, lo = (S % 2 == 0) ? 1 : 0, n = S - lo, nz = c - lo + 1;
	const long long per_mode = (long long)n * n * nz;
	long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (id >= per_mode * M)
		return;
	const int mode = (int)(id / per_mode);
	long long k = id - (long long)mode * per_mode;
	const int z = lo + (int)(k % nz);
	k /= nz;
	const int y = lo + (int)(k % n);
	const int x = lo + (int)(k / n);
	const long long V = (long long)S * S * S;
	double *a = model2 + (size_t)mode * V;
	const double *w = weight + (size_t)mode * V;
	const long long v1 = ((long long)x * S + y) * S + z;
	const long long v2 = ((long long)(2 * c - x) * S + (2 * c - y)) * S + (2 * c - z);
	if (z < c) {
		double A = friedel_avg(a[v1], w[v1], a[v2], w[v2]);
		a[v1] = A;
		a[v2] = A;
		return;
	}
	// z == c: the member visited first owns the pair
	const int mx = 2 * c - x, my = 2 * c - y;
	const bool first = (x < mx) || (x == mx && y <= my);
	if (!first)
		return;
	double A = friedel_avg(a[v1], w[v1], a[v2], w[v2]);
	if (v1 != v2)
		A = friedel_avg(A, w[v2], A, w[v1]);
	a[v1] = A;
	a[v2] = A;
}

// symmetrize_friedel2d (model.c:495-515) over every layer: (y, z) and
// (2c - y, 2c - z) for y in [lo, S), z in [lo, c], visited as friedel_kernel
// visits its pairs (the z == c line holds the pairs touched twice).
__global__ void friedel2d_kernel(double *__restrict__ model2, const double *__restrict__ weight, int S, int M) {
	const int c = S / 2, lo = (S % 2 == 0) ? 1 : 0, n = S - lo, nz = c - lo + 1;
	const long long per_layer = (long long)n * nz;
	const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (id >= per_layer * M)
		return;
	const int layer = (int)(id / per_layer);
	const long long k = id - (long long)layer * per_layer;
	const int z = lo + (int)(k % nz), y = lo + (int)(k / nz);
	const long long A2 = (long long)S * S;
	double *a = model2 + (size_t)layer * A2;
	const double *w = weight + (size_t)layer * A2;
	const long long v1 = (long long)y * S + z, v2 = (long long)(2 * c - y) * S + (2 * c - z);
	if (z < c) {
		const double A = friedel_avg(a[v1], w[v1], a[v2], w[v2]);
		a[v1] = A;
		a[v2] = A;
		return;
	}
	// z == c: the member visited first owns the pair
	if (y > 2 * c - y)
		return;
	double A = friedel_avg(a[v1], w[v1], a[v2], w[v2]);
	if (v1 != v2)
		A = friedel_avg(A, w[v2], A, w[v1]);
	a[v1] = A;
	a[v2] = A;
}

// model2 /= weight where weight > 0; squared change against model1; model1
// <- model2 or the alpha mix (recon.pyx:136-147). Block partial sums of the
// squared change go to part[blockIdx.x] for a fixed-order reduction.
template <typename MT>
__global__ void __launch_bounds__(256) divide_update_kernel(double *__restrict__ model2,
                                                            const double *__restrict__ weight,
                                                            double *__restrict__ model1, MT *__restrict__ model1_copy,
                                                            long long n, double alpha, double *__restrict__ part) {
	__shared__ double s[8];
	long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	double d2 = 0.;
	if (i < n) {
		double m2 = model2[i];
		if (weight[i] > 0.)
			m2 = m2 / weight[i];
		model2[i] = m2;
		double m1 = model1[i];
		double diff = m2 - m1;
		d2 = diff * diff;
		double nm = alpha > 0. ? alpha * m1 + (1 - alpha) * m2 : m2;
		model1[i] = nm;
		if (model1_copy != nullptr)
			model1_copy[i] = (MT)nm;
	}
	d2 = warp_sum(d2);
	if ((threadIdx.x & 31) == 0)
		s[threadIdx.x >> 5] = d2;
	__syncthreads();
	if (threadIdx.x == 0) {
		double t = 0.;
		for (int k = 0; k < 8; ++k)
			t += s[k];
		part[blockIdx.x] = t;
	}
}

// Point-group and axial symmetrisation (symmetrize_octahedral /
// symmetrize_icosahedral / symmetrize_axial, model.c:527-757, with
// rotate_model_openmp :423-468): for every voxel v = (vx, vy, vz) - c with
// vx, vy, vz in [0, S-2], sum over the n rotations g, in list order, of the
// trilinear sample of model2 * weight and of weight at g v + c (samples
// outside [0, S-1) are skipped); out = (sum A, sum W). One thread per voxel,
// FP64 in the reference's operation order. The plane index S-1 stays zero,
// as in the reference.
__global__ void symmetrize_kernel(const double *__restrict__ model2, const double *__restrict__ weight, int S,
                                  const double *__restrict__ rots, int n, double2 *__restrict__ out) {
	const long long V = (long long)S * S * S;
	const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= V)
		return;
	const int iz = (int)(i % S), iy = (int)((i / S) % S), ix = (int)(i / ((long long)S * S));
	double sa = 0., sw = 0.;
	if (ix < S - 1 && iy < S - 1 && iz < S - 1) {
		const int c = S / 2;
		const double vx = (double)(ix - c), vy = (double)(iy - c), vz = (double)(iz - c), cd = (double)c;
		const long long SS = (long long)S * S;
		for (int g = 0; g < n; ++g) {
			const double *R = rots + 9 * g;
			double rv[3];
#pragma unroll
			for (int k = 0; k < 3; ++k)
				rv[k] = dadd(dadd(dadd(dmul(R[3 * k], vx), dmul(R[3 * k + 1], vy)), dmul(R[3 * k + 2], vz)), cd);
			if (rv[0] < 0. || rv[0] >= S - 1 || rv[1] < 0. || rv[1] >= S - 1 || rv[2] < 0. || rv[2] >= S - 1)
				continue;
			const int x = (int)rv[0], y = (int)rv[1], z = (int)rv[2];
			const double fx = dsub(rv[0], (double)x), fy = dsub(rv[1], (double)y), fz = dsub(rv[2], (double)z);
			const double cx = dsub(1., fx), cy = dsub(1., fy), cz = dsub(1., fz);
			const double wts[8] = {dmul(dmul(cx, cy), cz), dmul(dmul(cx, cy), fz), dmul(dmul(cx, fy), cz),
			                       dmul(dmul(cx, fy), fz), dmul(dmul(fx, cy), cz), dmul(dmul(fx, cy), fz),
			                       dmul(dmul(fx, fy), cz), dmul(dmul(fx, fy), fz)};
			const long long b = x * SS + (long long)y * S + z;
			const long long o[8] = {0, 1, S, S + 1, SS, SS + 1, SS + S, SS + S + 1};
			double ta = 0., tw = 0.;
#pragma unroll
			for (int q = 0; q < 8; ++q) {
				const double w = __ldg(weight + b + o[q]);
				const double a = dmul(__ldg(model2 + b + o[q]), w);
				ta = q == 0 ? dmul(wts[q], a) : dadd(ta, dmul(wts[q], a));
				tw = q == 0 ? dmul(wts[q], w) : dadd(tw, dmul(wts[q], w));
			}
			sa = dadd(sa, ta);
			sw = dadd(sw, tw);
		}
	}
	out[i] = make_double2(sa, sw);
}

// model2 = sum A / sum W where sum W > 0 (else 0), weight = sum W
// (model.c:553-569, 715-729, 751-756).
__global__ void symmetrize_finish_kernel(const double2 *__restrict__ in, long long n, double *__restrict__ model2,
                                         double *__restrict__ weight) {
	const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	const double2 v = in[i];
	model2[i] = v.y > 0. ? v.x / v.y : 0.;
	weight[i] = v.y;
}

// Fixed-order sum of n doubles by one block (second stage of reductions).
__global__ void __launch_bounds__(1024) sum_kernel(const double *__restrict__ x, long long n,
                                                   double *__restrict__ out) {
	__shared__ double s[32];
	double acc = 0.;
	for (long long i = threadIdx.x; i < n; i += blockDim.x)
		acc += x[i];
	acc = warp_sum(acc);
	if ((threadIdx.x & 31) == 0)
		s[threadIdx.x >> 5] = acc;
	__syncthreads();
	if (threadIdx.x < 32) {
		double v = threadIdx.x < (blockDim.x >> 5) ? s[threadIdx.x] : 0.;
		v = warp_sum(v);
		if (threadIdx.x == 0)
			*out = v;
	}
}

// Sums of info / likelihood over good frames, and count of good frames:
// out[0] = sum info, out[1] = sum likelihood (max_prob.c:367-371); one block.
__global__ void __launch_bounds__(1024) frame_totals_kernel(const double *__restrict__ info,
                                                            const double *__restrict__ ll,
                                                            const uint8_t *__restrict__ blacklist, int N,
                                                            double *__restrict__ out) {
	__shared__ double s[2][32];
	double a = 0., b = 0.;
	for (int d = threadIdx.x; d < N; d += blockDim.x)
		if (!blacklist[d]) {
			a += info[d];
			b += ll[d];
		}
	a = warp_sum(a);
	b = warp_sum(b);
	if ((threadIdx.x & 31) == 0) {
		s[0][threadIdx.x >> 5] = a;
		s[1][threadIdx.x >> 5] = b;
	}
	__syncthreads();
	if (threadIdx.x < 32) {
		int nw = blockDim.x >> 5;
		double x = threadIdx.x < nw ? s[0][threadIdx.x] : 0., y = threadIdx.x < nw ? s[1][threadIdx.x] : 0.;
		x = warp_sum(x);
		y = warp_sum(y);
		if (threadIdx.x == 0) {
			out[0] = x;
			out[1] = y;
		}
	}
}

// beta_d = min(1, beta_start_d * factor) for good frames (recon.pyx:165-171)
__global__ void beta_kernel(const double *__restrict__ beta_start, const uint8_t *__restrict__ blacklist,
                            int N, double factor, double *__restrict__ beta) {
	int d = blockIdx.x * blockDim.x + threadIdx.x;
	if (d >= N || blacklist[d] == 1)
		return;
	double b = beta_start[d] * factor;
	beta[d] = b > 1. ? 1. : b;
}

// phi_d = fcounts_d / psum_d for good frames (max_scale.c:13-15)
__global__ void scale_kernel(const int *__restrict__ fcounts, const double *__restrict__ psum_d,
                             const uint8_t *__restrict__ blacklist, int N, double *__restrict__ scale) {
	int d = blockIdx.x * blockDim.x + threadIdx.x;
	if (d >= N || blacklist[d])
		return;
	scale[d] = fcounts[d] / psum_d[d];
}

// Good-frame sum of phi and count, for normalize_scale (one block).
__global__ void __launch_bounds__(1024) scale_sum_kernel(const double *__restrict__ scale,
                                                         const uint8_t *__restrict__ blacklist, int N,
                                                         double *__restrict__ out) {
	__shared__ double s[2][32];
	double a = 0., c = 0.;
	for (int d = threadIdx.x; d < N; d += blockDim.x)
		if (!blacklist[d]) {
			a += scale[d];
			c += 1.;
		}
	a = warp_sum(a);
	c = warp_sum(c);
	if ((threadIdx.x & 31) == 0) {
		s[0][threadIdx.x >> 5] = a;
		s[1][threadIdx.x >> 5] = c;
	}
	__syncthreads();
	if (threadIdx.x < 32) {
		int nw = blockDim.x >> 5;
		double x = threadIdx.x < nw ? s[0][threadIdx.x] : 0., y = threadIdx.x < nw ? s[1][threadIdx.x] : 0.;
		x = warp_sum(x);
		y = warp_sum(y);
		if (threadIdx.x == 0) {
			out[0] = x;
			out[1] = y;
		}
	}
}

// a[i] += b[i]: one detector's merged sums into the shared model's.
__global__ void add_into_kernel(double *__restrict__ a, const double *__restrict__ b, long long n) {
	const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
		a[i] += b[i];
}

// phi /= mean for good frames; model1 of mode 0 *= mean (iterate.pyx:372-382);
// mean = sums[0] / sums[1] (sum and count of good frames' phi); nothing
// changes without good frames (the host reports that case).
__global__ void apply_scale_norm_kernel(double *__restrict__ scale, const uint8_t *__restrict__ blacklist,
                                        int N, double *__restrict__ model1, float *__restrict__ model1f,
                                        long long V, const double *__restrict__ sums) {
	long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (!(sums[1] > 0.))
		return;
	const double m = sums[0] / sums[1];
	if (i < V) {
		double v = model1[i] * m;
		model1[i] = v;
		if (model1f != nullptr)
			model1f[i] = (float)v;
	}
	if (i < N && !blacklist[i])
		scale[i] /= m;
}

// Captured probability mass of watched frames (learned proposals): for watched
// frame w (chunk-local frame wl[w]) the sum of |P| over the orientations whose
// coarse cell qmap[r] is among the frame's proposed cells (bits[w * rwords ..]),
// divided by the sum over all orientations. Dead tiles (tlive 0) hold no
// probability. One warp per watched frame of the chunk.
__global__ void __launch_bounds__(256) captured_mass_kernel(const float *__restrict__ Pst, int RT, int Nc,
                                                            const uint8_t *__restrict__ tlive,
                                                            const int *__restrict__ qmap, const int *__restrict__ wl,
                                                            int nw, const uint32_t *__restrict__ bits, int rwords,
                                                            double *__restrict__ mass) {
	const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
	if (w >= nw)
		return;
	const int dl = wl[w];
	const size_t pstride = (size_t)(Nc + 1) * TILE;
	const uint32_t *b = bits + (size_t)w * rwords;
	double in = 0., all = 0.;
	for (int rt = 0; rt < RT; ++rt) {
		if (tlive && !tlive[(size_t)rt * (Nc + 1) + dl])
			continue;
		float v[LW];
		ld_row(Pst + rt * pstride + (size_t)dl * TILE + lane * LW, v);
#pragma unroll
		for (int k = 0; k < LW; ++k) {
			const double p = fabs((double)v[k]);
			const int c = qmap[rt * TILE + lane * LW + k];
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

// Nearest coarse orientation of every fine one (voronoi_subset,
// quaternion.c:844-862): distance 1 - (q . q')^2 with the dot product summed
// in component order, first coarse index on ties (strict <). One thread per
// fine orientation; the coarse list is staged through shared memory.
__global__ void __launch_bounds__(256) voronoi_kernel(const double *__restrict__ coarse, int nc,
                                                      const double *__restrict__ fine, int nf,
                                                      int *__restrict__ nearest) {
	__shared__ double cq[256][4];
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	double q[4] = {0., 0., 0., 0.};
	if (i < nf)
		for (int k = 0; k < 4; ++k)
			q[k] = fine[(size_t)i * 5 + k];
	double dmin = 2.;
	int best = -1;
	for (int j0 = 0; j0 < nc; j0 += 256) {
		const int n = min(256, nc - j0);
		__syncthreads();
		if (threadIdx.x < n)
			for (int k = 0; k < 4; ++k)
				cq[threadIdx.x][k] = coarse[(size_t)(j0 + threadIdx.x) * 5 + k];
		__syncthreads();
		for (int j = 0; j < n; ++j) {
			double dot = 0.;
#pragma unroll
			for (int k = 0; k < 4; ++k)
				dot = dadd(dot, dmul(q[k], cq[j][k]));
			const double dist = dsub(1., dmul(dot, dot));
			if (dist < dmin) {
				dmin = dist;
				best = j0 + j;
			}
		}
	}
	if (i < nf)
		nearest[i] = best;
}

// One slice, un-logged (Model.slice_gen, model.c:11-59)
// (slice_gen2d / slice_genrz, model.c:65-150, for 2-D and RZ models: g holds
// the quaternion, or (cos, sin) of the angle, or the five RZ parameters)
template <int GEO>
__global__ void slice_one_kernel(const double *__restrict__ g, int mode, const double *__restrict__ qvals,
                                 const double *__restrict__ corr, int P, const double *__restrict__ model,
                                 long long S, long long V, double *__restrict__ out) {
	int p = blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= P)
		return;
	double rot[9];
	if constexpr (GEO == MT_3D)
		rot_from_quat(g, rot);
	else
		for (int k = 0; k < 5; ++k)
			rot[k] = g[k];
	out[p] = geo_sample<GEO>(rot, qvals[3 * (size_t)p], qvals[3 * (size_t)p + 1], qvals[3 * (size_t)p + 2],
	                         (double)(S / 2), S, model + (size_t)mode * V, corr[p]);
}

// One merge in FP64 (Model.slice_merge, model.c:171-244)
// (slice_merge2d / slice_mergerz, model.c:254-340, for 2-D and RZ models)
template <int GEO>
__global__ void merge_one_kernel(const double *__restrict__ g, int mode, const double *__restrict__ view,
                                 const double *__restrict__ qvals, const double *__restrict__ corr,
                                 const uint8_t *__restrict__ mask, int P, long long S, long long V,
                                 double *__restrict__ model2, double *__restrict__ weight) {
	int p = blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= P || mask[p] > 1)
		return;
	const double qx = qvals[3 * (size_t)p], qy = qvals[3 * (size_t)p + 1], qz = qvals[3 * (size_t)p + 2];
	const double center = (double)(S / 2);
	double fw[8];
	long long o[8], base;
	int nc;
	if constexpr (GEO == MT_3D) {
		double rot[9];
		rot_from_quat(g, rot);
		Cell c = locate(rot, qx, qy, qz, center, S);
		if (!c.ok)
			return;
		corner_weights(c, fw);
		corner_offsets(S, o);
		base = c.i000;
		nc = 8;
	} else {
		Cell2 c = GEO == MT_2D ? locate2d(g, qx, qy, center, S) : locate_rz(g, qx, qy, center, S);
		if (!c.ok)
			return;
		corner_weights2(c, fw);
		o[0] = 0; o[1] = 1; o[2] = S; o[3] = S + 1;
		base = c.i00;
		nc = 4;
	}
	const double w = view[p] / corr[p];
	for (int q = 0; q < nc; ++q) {
		atomicAdd(weight + (size_t)mode * V + base + o[q], fw[q]);
		atomicAdd(model2 + (size_t)mode * V + base + o[q], fw[q] * w);
	}
}

// ---------------------------------------------------------------------------
// sparse probabilities and tomograms for the result getters
// ---------------------------------------------------------------------------
// Per frame of the chunk: the number of pairs with P > PROB_MIN (positive
// Pst), i.e. the length of the frame's list after resparsify
// (max_prob.c:321-325, 429-448). One warp per frame.
__global__ void __launch_bounds__(256) count_prob_kernel(const float *__restrict__ Pst, int RT, int Nc,
                                                         int *__restrict__ count) {
	const int dl = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
	if (dl >= Nc)
		return;
	const size_t pstride = (size_t)(Nc + 1) * TILE;
	int c = 0;
	for (int rt = 0; rt < RT; ++rt) {
		float v[LW];
		ld_row(Pst + rt * pstride + (size_t)dl * TILE + lane * LW, v);
#pragma unroll
		for (int e = 0; e < LW; ++e)
			c += v[e] > 0.f;
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		c += __shfl_xor_sync(FULL, c, o);
	if (lane == 0)
		count[dl] = c;
}

// The frame's list in ascending orientation order, as the reference's
// combined and resparsified prob / place_prob (max_prob.c:306-325): P is
// formed again in FP64 from the log-likelihood exactly as the normalisation
// formed it. off [Nc + 1] holds the chunk-local list offsets. One warp per
// frame; lanes own LW consecutive orientations, so a warp-wide exclusive scan
// of the per-lane counts orders each row.
__global__ void __launch_bounds__(256) compact_prob_kernel(
    const double *__restrict__ pval, const float *__restrict__ Pst, int RT, int Nc, int d0,
    const double *__restrict__ beta, const double *__restrict__ max_exp, const double *__restrict__ p_norm,
    const long long *__restrict__ off, int *__restrict__ place, double *__restrict__ prob) {
	const int dl = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
	if (dl >= Nc)
		return;
	long long base = off[dl];
	if (off[dl + 1] == base)
		return;
	const int d = d0 + dl;
	const double m = max_exp[d], inv_s = 1. / p_norm[d], b = beta[d];
	const size_t pstride = (size_t)(Nc + 1) * TILE, tstride = (size_t)Nc * TILE;
	for (int rt = 0; rt < RT; ++rt) {
		float pv[LW];
		ld_row(Pst + rt * pstride + (size_t)dl * TILE + lane * LW, pv);
		int c = 0;
#pragma unroll
		for (int e = 0; e < LW; ++e)
			c += pv[e] > 0.f;
		int incl = c;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const int y = __shfl_up_sync(FULL, incl, o);
			if (lane >= o)
				incl += y;
		}
		const int total = __shfl_sync(FULL, incl, 31);
		if (c > 0) {
			double x[LW];
			ld_row(pval + rt * tstride + (size_t)dl * TILE + lane * LW, x);
			long long pos = base + incl - c;
#pragma unroll
			for (int e = 0; e < LW; ++e)
				if (pv[e] > 0.f) {
					place[pos] = rt * TILE + lane * LW + e;
					prob[pos] = exp(dmul(b, dsub(x[e], m))) * inv_s;
					++pos;
				}
		}
		base += total;
	}
}

// Tomograms of orientations r0 .. r0 + n - 1 divided by psum_r where it is
// positive (update_tomogram_nobg's final step, max_update.c:226-229), as
// out [n][P] FP64; with psum_r null (background path) T already holds them.
__global__ void tomogram_kernel(const float *__restrict__ T, const double *__restrict__ psum_r, int P, int r0,
                                int n, double *__restrict__ out) {
	const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= (long long)n * P)
		return;
	const int k = (int)(idx / P), p = (int)(idx - (long long)k * P), r = r0 + k;
	const double v = T[((size_t)(r / TILE) * P + p) * TILE + r % TILE];
	const double ps = psum_r != nullptr ? psum_r[r] : 0.;
	out[idx] = ps > 0. ? v / ps : v;
}

}  // namespace dfg
