// Dense form of the E-step photon term on the 5th-generation tensor cores
// (sm_100a tcgen05 + TMA). Included by emc_api.cu only.
//
// The photon term of every (orientation r, frame d) pair is a product over the
// mask-0 pixels: S[r][d] = sum_k count[d][k] * logW[r][k]. With photon counts
// of at most 256 (exact in BF16) and log-slices split as hi + lo
// (hi = bf16(x), lo = bf16(x - hi)), S = hi . count^T + lo . count^T is a pair
// of BF16 matrix products with FP32 accumulation. One CTA computes a tile of
// 128 orientations x 256 frames over all pixels:
//   warp 0     TMA producer: per 64-pixel block, the 128 x 64 hi and lo tiles
//              and the 256 x 64 count tile (128-byte swizzle) into one of
//              three shared-memory stages;
//   warp 1     one lane issues tcgen05.mma (M 128, N 256, K 16; hi then lo
//              against the same count tile), accumulating in 256 TMEM columns,
//              and releases each stage with tcgen05.commit;
//   warps 2-5  epilogue: tcgen05.ld of the accumulator (TMEM lane = orientation,
//              column = frame), pval = log w_r - u_r s_d + S (FP64) stored in
//              the sparse form's layout, and the tile maximum with its lowest
//              orientation index.
// Every wait on an mbarrier gives up after wait_cycles clock cycles (about a
// second unless a test shortens it), sets the error flag and lets the CTA
// free its TMEM and exit. withhold_kb >= 0 is a test hook that never issues
// that stage's copies, so the waits on it run out (-1 in production).
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>

#include "emc_common.cuh"
#include "tcgen05.cuh"

namespace dfg {

constexpr int DN = 256;      // frames per tile (UMMA N)
constexpr int DK = 64;       // pixels per stage: one 128-byte swizzle row of BF16
constexpr int DSTAGES = 3;
constexpr int DA_BYTES = 128 * DK * 2;                 // one 128 x 64 BF16 tile
constexpr int DB_BYTES = DN * DK * 2;                  // one 256 x 64 BF16 tile
constexpr int DSTAGE_BYTES = 2 * DA_BYTES + DB_BYTES;  // 64 KB
constexpr int DEPI_BYTES = 4 * DN * (8 + 4);            // per-warp column maxima
constexpr int DSMEM_BYTES = 1024 + DSTAGES * DSTAGE_BYTES + DEPI_BYTES + 128;
constexpr int DGROUP = 16;  // orientation tiles per rasterisation group

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), BF16 A
// and B (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t DIDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(DN >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
	asm volatile(
	    "{\n\t.reg .pred p;\n\t"
	    "setp.ne.b32 p, %4, 0;\n\t"
	    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
	    "l"(adesc), "l"(bdesc), "r"(DIDESC), "r"(accumulate)
	    : "memory");
}

// pval[tile][frame][j] for one frame chunk from the hi / lo log-slices
// [R_pad][K_pad] and the chunk's counts [Nc_pad][K_pad] (tensor maps), plus
// the per (tile, frame) maximum and its first orientation, as estep_kernel
// writes them. Grid: RT x ceil(Nc / 256) tiles, grouped by DGROUP tiles of
// orientations so that resident CTAs share operands in L2.
__global__ void __launch_bounds__(192, 1) estep_dense_kernel(
    const __grid_constant__ CUtensorMap map_hi, const __grid_constant__ CUtensorMap map_lo,
    const __grid_constant__ CUtensorMap map_cnt, int num_kb, int RT, int n_tiles, const double *__restrict__ u,
    const double *__restrict__ logw, int R, const double *__restrict__ scale, int d0, int Nc, int use_scale,
    const double *__restrict__ scalars, double *__restrict__ pval, double *__restrict__ tmax,
    int *__restrict__ targ, int *__restrict__ err, long long wait_cycles, int withhold_kb) {
	extern __shared__ uint8_t dsm_raw[];
	uint8_t *sm = (uint8_t *)(((uintptr_t)dsm_raw + 1023) & ~(uintptr_t)1023);
	double *s_max = (double *)(sm + DSTAGES * DSTAGE_BYTES);
	int *s_arg = (int *)(s_max + 4 * DN);
	uint64_t *bars = (uint64_t *)(sm + DSTAGES * DSTAGE_BYTES + DEPI_BYTES);
	uint64_t *full = bars, *empty = bars + DSTAGES, *accum = bars + 2 * DSTAGES;
	uint32_t *tmem_slot = (uint32_t *)(bars + 2 * DSTAGES + 1);
	volatile int *abort_flag = (volatile int *)(tmem_slot + 1);

	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	// grouped rasterisation of the (orientation tile, frame tile) grid
	const int per_group = DGROUP * n_tiles;
	const int grp = blockIdx.x / per_group, rem = blockIdx.x - grp * per_group;
	const int rows = min(DGROUP, RT - grp * DGROUP);
	const int rt = grp * DGROUP + rem % rows, nt = rem / rows;

	if (threadIdx.x == 0) {
		for (int s = 0; s < DSTAGES; ++s) {
			mbar_init(&full[s], 1);
			mbar_init(&empty[s], 1);
		}
		mbar_init(accum, 1);
		*abort_flag = 0;
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	if (warp == 1) {
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
		                 smem_addr(tmem_slot)),
		             "r"(DN)
		             : "memory");
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
	}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const uint32_t tmem = *tmem_slot;

	if (warp == 0) {
		if (lane == 0) {
			int issued = 0;
			for (int kb = 0; kb < num_kb; ++kb) {
				const int s = kb % DSTAGES;
				const uint32_t ph = (uint32_t)(kb / DSTAGES) & 1u;
				if (*abort_flag || !mbar_wait(&empty[s], ph ^ 1u, wait_cycles)) {
					*abort_flag = 1;
					atomicExch(err, 1);
					break;
				}
				if (kb == withhold_kb)  // test hook: this stage's copies are never issued
					continue;
				uint8_t *st = sm + s * DSTAGE_BYTES;
				mbar_expect_tx(&full[s], DSTAGE_BYTES);
				tma_load_2d(st, &map_hi, &full[s], kb * DK, rt * 128);
				tma_load_2d(st + DA_BYTES, &map_lo, &full[s], kb * DK, rt * 128);
				tma_load_2d(st + 2 * DA_BYTES, &map_cnt, &full[s], kb * DK, nt * DN);
				issued = kb + 1;
			}
			// on a give-up, let the copies still in flight land before exiting
			if (*abort_flag)
				for (int kb = max(0, issued - DSTAGES); kb < issued; ++kb)
					mbar_wait(&full[kb % DSTAGES], (uint32_t)(kb / DSTAGES) & 1u, wait_cycles);
		}
		__syncwarp();
	} else if (warp == 1) {
		if (lane == 0) {
			for (int kb = 0; kb < num_kb; ++kb) {
				const int s = kb % DSTAGES;
				const uint32_t ph = (uint32_t)(kb / DSTAGES) & 1u;
				if (*abort_flag || !mbar_wait(&full[s], ph, wait_cycles)) {
					*abort_flag = 1;
					atomicExch(err, 1);
					break;
				}
				tc_fence_after();
				const uint32_t a_hi = smem_addr(sm + s * DSTAGE_BYTES);
				const uint32_t a_lo = a_hi + DA_BYTES, b = a_hi + 2 * DA_BYTES;
#pragma unroll
				for (int k = 0; k < DK / 16; ++k) {
					const uint64_t db = sw128_desc(b + 32 * k);
					umma_bf16(tmem, sw128_desc(a_hi + 32 * k), db, (kb | k) != 0);
					umma_bf16(tmem, sw128_desc(a_lo + 32 * k), db, 1u);
				}
				umma_commit(&empty[s]);
			}
			umma_commit(accum);
		}
		__syncwarp();
	} else {
		// epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31
		const int q = warp & 3, i = q * 32 + lane, r = rt * 128 + i;
		const bool valid_r = r < R;
		const double lw = valid_r ? logw[r] : 0., ur = valid_r ? u[r] : 0.;
		const bool ok = mbar_wait(accum, 0, wait_cycles);
		if (!ok) {
			*abort_flag = 1;
			atomicExch(err, 1);
		}
		tc_fence_after();
		if (ok && !*abort_flag) {
			for (int c = 0; c < DN / 16; ++c) {
				float acc[16];
				tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(c * 16), acc);
#pragma unroll
				for (int j = 0; j < 16; ++j) {
					const int col = c * 16 + j, dl = nt * DN + col;
					double m = MAX_EXP_START;
					int am = -1;
					if (dl < Nc) {
						const double sd = use_scale ? scale[d0 + dl] : scalars[0];
						const double v = valid_r ? dadd(dsub(lw, dmul(ur, sd)), (double)acc[j]) : 0.;
						pval[((size_t)rt * Nc + dl) * 128 + i] = v;
						if (valid_r) {
							m = v;
							am = r;
						}
					}
#pragma unroll
					for (int o = 16; o > 0; o >>= 1) {
						const double om = __shfl_xor_sync(FULL, m, o);
						const int oa = __shfl_xor_sync(FULL, am, o);
						if (om > m || (om == m && oa >= 0 && (am < 0 || oa < am))) {
							m = om;
							am = oa;
						}
					}
					if (lane == 0) {
						s_max[q * DN + col] = m;
						s_arg[q * DN + col] = am;
					}
				}
			}
		}
		asm volatile("bar.sync 1, 128;" ::: "memory");
		if (ok && !*abort_flag) {
			const int t = threadIdx.x - 64;
			for (int col = t; col < DN; col += 128) {
				const int dl = nt * DN + col;
				if (dl >= Nc)
					continue;
				double m = MAX_EXP_START;
				int am = -1;
				for (int w = 0; w < 4; ++w) {  // lanes 0-31 first: lowest index wins ties
					const double v = s_max[w * DN + col];
					if (v > m) {
						m = v;
						am = s_arg[w * DN + col];
					}
				}
				tmax[(size_t)rt * Nc + dl] = m;
				targ[(size_t)rt * Nc + dl] = am;
			}
		}
	}
	tc_fence_before();
	__syncthreads();
	if (warp == 1) {
		tc_fence_after();
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(DN) : "memory");
	}
}

// ---------------------------------------------------------------------------
// dense M-step: T[r][p] += sum_d P[r][d] count[d][p] over one frame chunk
// ---------------------------------------------------------------------------
// Both operands are MN-major (orientations and pixels contiguous, frames the
// reduction): tiles of 64 elements (128 bytes) x 64 frames per TMA box,
// 8-frame groups 1024 bytes apart (SBO), 64-element blocks one box (8192
// bytes) apart (LBO); one K = 16 step is two 8-frame groups (2048 bytes).
__device__ __forceinline__ uint64_t sw128_mn_desc(uint32_t addr) {
	return (uint64_t)((addr & 0x3FFFF) >> 4) | ((uint64_t)(8192 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
	       ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}
constexpr uint32_t DIDESC_MN = DIDESC | (1u << 15) | (1u << 16);  // A and B MN-major

__device__ __forceinline__ void umma_bf16_mn(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
	asm volatile(
	    "{\n\t.reg .pred p;\n\t"
	    "setp.ne.b32 p, %4, 0;\n\t"
	    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
	    "l"(adesc), "l"(bdesc), "r"(DIDESC_MN), "r"(accumulate)
	    : "memory");
}

// One CTA per 128-orientation x 256-pixel-column tile over all frames of the
// chunk: TMA loads of the hi / lo probability tiles ([RT * Nc_pad][128] BF16,
// two 64-orientation boxes each) and of the count tile ([Nc_pad][K_pad],
// four 64-pixel boxes), tcgen05.mma into a 256-column FP32 accumulator, and
// an epilogue adding it to the tomograms T[rt][kpix[col]][j] (FP32, read and
// written as the sparse M-step does). Roles and give-up rules as
// estep_dense_kernel.
__global__ void __launch_bounds__(192, 1) mstep_dense_kernel(
    const __grid_constant__ CUtensorMap map_phi, const __grid_constant__ CUtensorMap map_plo,
    const __grid_constant__ CUtensorMap map_cnt, int num_kb, int Nc_pad, int RT, int n_tiles,
    const int *__restrict__ kpix, int K, int P, float *__restrict__ T, int *__restrict__ err, long long wait_cycles,
    int withhold_kb) {
	extern __shared__ uint8_t dsm_raw[];
	uint8_t *sm = (uint8_t *)(((uintptr_t)dsm_raw + 1023) & ~(uintptr_t)1023);
	uint64_t *bars = (uint64_t *)(sm + DSTAGES * DSTAGE_BYTES + DEPI_BYTES);
	uint64_t *full = bars, *empty = bars + DSTAGES, *accum = bars + 2 * DSTAGES;
	uint32_t *tmem_slot = (uint32_t *)(bars + 2 * DSTAGES + 1);
	volatile int *abort_flag = (volatile int *)(tmem_slot + 1);

	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int per_group = DGROUP * n_tiles;
	const int grp = blockIdx.x / per_group, rem = blockIdx.x - grp * per_group;
	const int rows = min(DGROUP, RT - grp * DGROUP);
	const int rt = grp * DGROUP + rem % rows, nt = rem / rows;

	if (threadIdx.x == 0) {
		for (int s = 0; s < DSTAGES; ++s) {
			mbar_init(&full[s], 1);
			mbar_init(&empty[s], 1);
		}
		mbar_init(accum, 1);
		*abort_flag = 0;
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	if (warp == 1) {
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
		                 smem_addr(tmem_slot)),
		             "r"(DN)
		             : "memory");
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
	}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const uint32_t tmem = *tmem_slot;

	if (warp == 0) {
		if (lane == 0) {
			int issued = 0;
			for (int kb = 0; kb < num_kb; ++kb) {
				const int s = kb % DSTAGES;
				const uint32_t ph = (uint32_t)(kb / DSTAGES) & 1u;
				if (*abort_flag || !mbar_wait(&empty[s], ph ^ 1u, wait_cycles)) {
					*abort_flag = 1;
					atomicExch(err, 1);
					break;
				}
				if (kb == withhold_kb)  // test hook: this stage's copies are never issued
					continue;
				uint8_t *st = sm + s * DSTAGE_BYTES;
				const int fy = rt * Nc_pad + kb * DK;  // probability rows of this frame block
				mbar_expect_tx(&full[s], DSTAGE_BYTES);
				for (int h = 0; h < 2; ++h) {
					tma_load_2d(st + h * (DA_BYTES / 2), &map_phi, &full[s], h * 64, fy);
					tma_load_2d(st + DA_BYTES + h * (DA_BYTES / 2), &map_plo, &full[s], h * 64, fy);
				}
				for (int h = 0; h < 4; ++h)
					tma_load_2d(st + 2 * DA_BYTES + h * (DB_BYTES / 4), &map_cnt, &full[s], nt * DN + h * 64,
					            kb * DK);
				issued = kb + 1;
			}
			if (*abort_flag)
				for (int kb = max(0, issued - DSTAGES); kb < issued; ++kb)
					mbar_wait(&full[kb % DSTAGES], (uint32_t)(kb / DSTAGES) & 1u, wait_cycles);
		}
		__syncwarp();
	} else if (warp == 1) {
		if (lane == 0) {
			for (int kb = 0; kb < num_kb; ++kb) {
				const int s = kb % DSTAGES;
				const uint32_t ph = (uint32_t)(kb / DSTAGES) & 1u;
				if (*abort_flag || !mbar_wait(&full[s], ph, wait_cycles)) {
					*abort_flag = 1;
					atomicExch(err, 1);
					break;
				}
				tc_fence_after();
				const uint32_t a_hi = smem_addr(sm + s * DSTAGE_BYTES);
				const uint32_t a_lo = a_hi + DA_BYTES, b = a_hi + 2 * DA_BYTES;
#pragma unroll
				for (int k = 0; k < DK / 16; ++k) {
					const uint64_t db = sw128_mn_desc(b + 2048 * k);
					umma_bf16_mn(tmem, sw128_mn_desc(a_hi + 2048 * k), db, (kb | k) != 0);
					umma_bf16_mn(tmem, sw128_mn_desc(a_lo + 2048 * k), db, 1u);
				}
				umma_commit(&empty[s]);
			}
			umma_commit(accum);
		}
		__syncwarp();
	} else {
		const int q = warp & 3, i = q * 32 + lane;
		const bool ok = mbar_wait(accum, 0, wait_cycles);
		if (!ok) {
			*abort_flag = 1;
			atomicExch(err, 1);
		}
		tc_fence_after();
		if (ok && !*abort_flag) {
			for (int c = 0; c < DN / 16; ++c) {
				float acc[16];
				tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(c * 16), acc);
#pragma unroll
				for (int j = 0; j < 16; ++j) {
					const int col = nt * DN + c * 16 + j;
					if (col < K) {
						float *t = T + ((size_t)rt * P + kpix[col]) * 128 + i;
						*t = (float)((double)*t + (double)acc[j]);
					}
				}
			}
		}
	}
	tc_fence_before();
	__syncthreads();
	if (warp == 1) {
		tc_fence_after();
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(DN) : "memory");
	}
}

// Probabilities of one chunk as BF16 hi / lo rows [RT][Nc_pad][128]
// (p = max(Pst, 0): pairs at or below the PROB_MIN gate do not enter the
// tomograms; rows past the chunk and of dead tiles are zero).
__global__ void split_prob_kernel(const float *__restrict__ Pst, int Nc, int Nc_pad, int RT,
                                  const uint8_t *__restrict__ tlive, __nv_bfloat16 *__restrict__ hi,
                                  __nv_bfloat16 *__restrict__ lo) {
	const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // 8 values each
	if (t >= (long long)RT * Nc_pad * 16)
		return;
	const long long row = t >> 4;
	const int rt = (int)(row / Nc_pad), dl = (int)(row - (long long)rt * Nc_pad), j0 = (int)(t & 15) * 8;
	// with tile skipping, dead tiles hold no probability (tlive)
	const bool live = dl < Nc && (tlive == nullptr || tlive[(size_t)rt * (Nc + 1) + dl]);
	__align__(16) __nv_bfloat16 h[8], l[8];
#pragma unroll
	for (int e = 0; e < 8; ++e) {
		const float p = live ? fmaxf(Pst[((size_t)rt * (Nc + 1) + dl) * TILE + j0 + e], 0.f) : 0.f;
		const __nv_bfloat16 ph = __float2bfloat16_rn(p);
		h[e] = ph;
		l[e] = __float2bfloat16_rn(p - __bfloat162float(ph));
	}
	const size_t o = (size_t)row * 128 + j0;
	*reinterpret_cast<uint4 *>(hi + o) = *reinterpret_cast<const uint4 *>(h);
	*reinterpret_cast<uint4 *>(lo + o) = *reinterpret_cast<const uint4 *>(l);
}

// hi / lo BF16 log-slices [R_pad][K_pad] (orientation rows, the mask < 2
// pixels in pixel order; zero on mask-1 pixels, which the likelihood leaves
// out, and past K) from the FP32 log-slice tiles [RT][P+1][TILE]:
// x = hi + lo + O(2^-17 |x|), hi = bf16(x), lo = bf16(x - hi). A log of zero
// (-inf) becomes -1e30 so that a zero count times it stays zero. Block = one
// orientation tile x 64 pixels, transposed through shared memory.
__global__ void __launch_bounds__(256) split_logw_kernel(const float *__restrict__ logW, int P,
                                                         const int *__restrict__ kpix,
                                                         const uint8_t *__restrict__ mask, int K, int K_pad,
                                                         __nv_bfloat16 *__restrict__ hi,
                                                         __nv_bfloat16 *__restrict__ lo) {
	__shared__ float s[DK][128 + 1];
	const int kb = blockIdx.x, rt = blockIdx.y, t = threadIdx.x;
	for (int idx = t; idx < DK * 128; idx += 256) {
		const int row = idx >> 7, col = idx & 127, k = kb * DK + row;
		float v = 0.f;
		if (k < K && mask[kpix[k]] == 0)  // mask-1 columns hold the M-step's photons only
			v = logW[((size_t)rt * (P + 1) + kpix[k]) * TILE + col];
		s[row][col] = v;
	}
	__syncthreads();
	for (int idx = t; idx < 128 * (DK / 8); idx += 256) {
		const int col = idx >> 3, c8 = idx & 7;
		__align__(16) __nv_bfloat16 h[8], l[8];
#pragma unroll
		for (int e = 0; e < 8; ++e) {
			float x = s[c8 * 8 + e][col];
			x = fmaxf(x, -1e30f);
			const __nv_bfloat16 xh = __float2bfloat16_rn(x);
			h[e] = xh;
			l[e] = __float2bfloat16_rn(x - __bfloat162float(xh));
		}
		const size_t o = ((size_t)rt * 128 + col) * K_pad + (size_t)kb * DK + c8 * 8;
		*reinterpret_cast<uint4 *>(hi + o) = *reinterpret_cast<const uint4 *>(h);
		*reinterpret_cast<uint4 *>(lo + o) = *reinterpret_cast<const uint4 *>(l);
	}
}

// Counts of one frame chunk as BF16 rows [Nc_pad][K_pad] over the mask < 2
// pixels (the buffer is zeroed before): one warp per pixel with photons
// scatters the M-step index words of the chunk (counts <= 256, so one word
// per frame and pixel; padding words name frame Nc).
__global__ void densify_counts_kernel(const uint32_t *__restrict__ cs, const long long *__restrict__ cs_off,
                                      const long long *__restrict__ cs_mid, const int *__restrict__ pix,
                                      int npix, const int *__restrict__ pcol, int Nc, int K_pad,
                                      __nv_bfloat16 *__restrict__ cnt) {
	const int w = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
	if (w >= npix)
		return;
	const int p = pix[w], col = pcol[p];
	if (col < 0)
		return;
	const long long beg = cs_off[p], mid = cs_mid[p], end = cs_off[p + 1];
	for (long long j = beg + lane; j < end; j += 32) {
		const uint32_t word = cs[j];
		const uint32_t idx = j < mid ? word : (word & IDX_MASK);
		if (idx >= (uint32_t)Nc)
			continue;
		const uint32_t c = j < mid ? 1u : (word >> IDX_BITS);
		cnt[(size_t)idx * K_pad + col] = __float2bfloat16_rn((float)c);
	}
}

}  // namespace dfg
