// Context of the B200 EMC iteration: resident inputs, work buffers and the
// error/instrumentation state behind the C ABI (include/dragonfly_b200.h).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dragonfly_b200.h"
#include "emc_common.cuh"

namespace dfg {

enum Phase { PH_SLICE, PH_ESTEP, PH_NORM, PH_PSUM, PH_MSTEP, PH_MERGE, PH_UPDATE, PH_COUNT };
constexpr int kTimingEvents = 2048;  // phase-timing events per context
static const char *kPhaseNames[PH_COUNT] = {"slice", "estep", "norm", "psum", "mstep", "merge", "update"};

// Owning device buffer; move-only.
template <typename T>
struct DevBuf {
	T *p = nullptr;
	size_t n = 0;
	DevBuf() = default;
	DevBuf(const DevBuf &) = delete;
	DevBuf &operator=(const DevBuf &) = delete;
	DevBuf(DevBuf &&o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
	DevBuf &operator=(DevBuf &&o) noexcept {
		if (this != &o) {
			release();
			p = o.p; n = o.n;
			o.p = nullptr; o.n = 0;
		}
		return *this;
	}
	~DevBuf() { release(); }
	void release() {
		if (p)
			cudaFree(p);
		p = nullptr;
		n = 0;
	}
	cudaError_t ensure(size_t count) {
		if (count <= n && p)
			return cudaSuccess;
		release();
		cudaError_t e = cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T));
		if (e == cudaSuccess)
			n = std::max<size_t>(count, 1);
		else
			p = nullptr;
		return e;
	}
};

// Page-locked host staging buffer (grow-only): large per-iteration uploads go
// through it at full copy speed, written in place by the host threads.
template <typename T>
struct HostBuf {
	T *p = nullptr;
	size_t n = 0;
	HostBuf() = default;
	HostBuf(const HostBuf &) = delete;
	HostBuf &operator=(const HostBuf &) = delete;
	~HostBuf() { release(); }
	void release() {
		if (p)
			cudaFreeHost(p);
		p = nullptr;
		n = 0;
	}
	cudaError_t ensure(size_t count) {
		if (count <= n && p)
			return cudaSuccess;
		release();
		cudaError_t e = cudaMallocHost(&p, std::max<size_t>(count, 1) * sizeof(T));
		if (e == cudaSuccess)
			n = std::max<size_t>(count, 1);
		else
			p = nullptr;
		return e;
	}
};

struct Chunk {
	int d0 = 0, nc = 0;
	DevBuf<uint32_t> cs;       // per pixel: count-1 frames, then (frame | count << 22), padded
	DevBuf<long long> cs_off;  // [P + 1]
	DevBuf<long long> cs_mid;  // [P] start of the multi-photon segment
	DevBuf<int> pix;           // pixels with non-empty lists, longest first
	int npix = 0;
	long long entries = 0;
};

}  // namespace dfg

using namespace dfg;

struct dfg_ctx {
	int device = 0;
	int num_sms = 0;  // streaming multiprocessors of the device (persistent grids)
	cudaStream_t stream = nullptr;
	std::string err;

	// detector
	int P = 0;
	DevBuf<double> qvals, corr;
	DevBuf<uint8_t> mask;
	std::vector<uint8_t> h_mask;

	// frames
	int N = 0;
	std::vector<int> h_ones, h_multi, h_place_ones, h_place_multi, h_count_multi;
	std::vector<long long> h_ones_off, h_multi_off;
	DevBuf<uint32_t> ph;       // per frame: count-1 pixels, then (pixel | count << 22), padded
	DevBuf<long long> ph_off;  // [N + 1]
	DevBuf<long long> ph_mid;  // [N] start of the multi-photon segment
	long long n_ph = 0;        // photon words without padding
	int logW_P = -1;           // detector size the zero row of logW was written for
	DevBuf<double> scale, beta, beta_start, sum_fact;
	DevBuf<int> fcounts;
	DevBuf<uint8_t> blacklist;
	double mean_count = 0.;
	bool beta_set = false;

	// orientations and model; model_type MT_2D / MT_RZ hold stacks of S x S
	// images (V = S^2) and take an angle (2-D) or (phi, beta) (RZ) per
	// orientation; cs2d [num_rot][2] = (cos, sin) of the 2-D angles, from the
	// host's libm as the reference's make_rot_angle (model.c:788-795)
	int num_rot = 0, M = 1, R = 0, RT = 0, R_pad = 0;
	int model_type = MT_3D;
	bool friedel2d = false;  // params.friedel_sym of a 2-D reconstruction
	double detd = 0.;        // detector distance (RZ geometry)
	DevBuf<double> quats, cs2d;
	long long S = 0, V = 0;
	DevBuf<double> model1, model2, weight;
	DevBuf<double2> accum;
	// inter_weight of the last merge and the psum_r > 0 pattern it was built
	// for (the weights depend on nothing else once geometry is fixed); the
	// pattern and the flags (accumulate weights, grid cached) live on the
	// device; weight_cache_valid false makes the next maximize clear them
	DevBuf<double> weight_cache;
	DevBuf<uint8_t> wpattern;
	DevBuf<int> wflags;
	bool weight_cache_valid = false;
	// the iteration as a CUDA graph (dfg_run_iteration)
	bool use_graph = true;
	bool capturing = false;  // the stream is being captured into the graph
	cudaGraphExec_t graph_exec = nullptr;
	long graph_launches = 0, graph_updates = 0, graph_instantiations = 0;

	// work buffers
	DevBuf<float> logW, Pst, T;
	DevBuf<double> u, pval, psum_r, psum_part, scalars, red_part;
	DevBuf<double> logw;  // log w_r per orientation
	DevBuf<int> rmax, num_prob, targ;
	DevBuf<double> tmax;  // per (tile, frame) maximum of pval and its first orientation
	DevBuf<uint8_t> tlive;  // [RT][Nc + 1]: the (tile, frame) has a kept pair (norm_kernel)
	bool mstep_skip = false;  // option tile_skip: skip dead (tile, frame) pairs without refinement
	DevBuf<double> info, likelihood, max_exp, p_norm, psum_d, quat_norm;
	std::vector<Chunk> chunks;
	int chunk_frames = 0;
	int chunks_R = -1;  // R the chunk layout was built for

	// options and results
	double pair_budget_mb = 0.;
	int slice_block = 0;  // orientations per slice block; 0 = automatic
	// background-aware model (per-pixel background with need_scaling):
	// background [P], powder [P] (mean mask-0 photons per frame and pixel),
	// bgscale [N], scalemax [R] and the work buffers of the scale search
	bool with_bg = false, powder_valid = false;
	bool views_final = false;  // T holds the final views (background path), not sums
	// model symmetries applied by update_model: a point group (S4 / A5) in
	// place of the Friedel average, then an axial symmetry
	DevBuf<double> group_rots, axial_rots;
	int n_group_rots = 0, n_axial_rots = 0;
	std::vector<double> h_bgscale;
	DevBuf<double> background, powder, bgscale, scalemax, smax_part, gd_part, gd_G, gd_s;
	DevBuf<double> Wd;  // slices W [RT][P+1][TILE] in FP64 (background-aware E-step)
	DevBuf<double> Pd;  // probabilities [RT][Nc+1][TILE] in FP64, sign as Pst
	DevBuf<uint8_t> gd_active;
	// sparse probabilities of the last maximize (option keep_prob): per frame
	// the pairs with P > PROB_MIN in orientation order, host-resident
	bool keep_prob = false, have_prob = false;
	std::vector<long long> h_prob_off;  // [N + 1]
	std::vector<int> h_place_prob;
	std::vector<double> h_prob;
	DevBuf<int> prob_count, d_place;
	DevBuf<long long> d_prob_off;
	DevBuf<double> d_prob, tomo_out;
	// dense (tensor-core) form of the E-step photon term. estep_form 0 =
	// sparse gathers, 1 = dense, 2 = chosen by the autotuner; dense_active is
	// this iteration's choice. K mask-0 pixels (kpix [K] their indices, pcol
	// [P] the column of each, -1 elsewhere), K_pad = K rounded up to 64; hi / lo
	// log-slices [R_pad][K_pad] and one chunk's counts [cnt_rows][K_pad] in
	// BF16 (stored as 16-bit words); their TMA tensor maps; derr = the dense
	// kernel's give-up flag
	// mstep_form likewise for the tomogram products (m_dense_active);
	// chunks_dense = the forms the chunk layout was sized for. K = mask < 2
	// pixel columns (the E-step's hi / lo rows are zero on mask-1 columns);
	// Phi / Plo = one chunk's probabilities [RT][cnt_rows][128] in BF16
	int estep_form = 0, mstep_form = 0;
	bool dense_active = false, m_dense_active = false;
	int chunks_dense = 0;
	// autotuner (option autotune): the slice block and E-step / M-step forms
	// it chose for the current inputs; tuning / tune_* while it measures
	bool autotune = false, tuned = false, tuning = false;
	int tuned_ob = 0, tuned_form = 0, tuned_mform = 0, tune_form = 0, tune_mform = 0;
	// blocks per SM of the sparse E-step and M-step (0: the build's default;
	// options estep_blocks_per_sm / mstep_blocks_per_sm override the tuner)
	int estep_minb = 0, mstep_minb = 0, tuned_estep_minb = 0, tuned_mstep_minb = 0;
	int tune_estep_minb = 0, tune_mstep_minb = 0;
	double tune_report[DFG_TUNE_REPORT] = {};
	int K = 0, K_pad = 0, dense_P = -1, cnt_rows = 0;
	int max_count0 = -1;  // largest count on a mask < 2 pixel; -1 = not known
	DevBuf<int> kpix, pcol, derr;
	// failure-detection test hooks of the dense kernels: the clock cycles
	// after which a pipeline wait gives up, and a stage whose copies are never
	// issued (-1: none)
	long long dense_wait_cycles = 2000000000LL;  // about one second, as TC_WAIT_CYCLES
	int dense_withhold = -1;
	DevBuf<uint16_t> Ahi, Alo, cnt, Phi, Plo;
	// counts read by the E-step (256-frame boxes) and the M-step (64-frame boxes)
	CUtensorMap map_hi, map_lo, map_cnt, map_phi, map_plo, map_cnt_m;
	const void *map_src[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
	// coarse-to-fine refinement: coarse cell of every orientation (qmap,
	// [R_pad], -1 past R) and per frame one bit per relevant coarse
	// orientation (rel_bits, [N][rwords])
	bool refine = false, qmap_valid = false;
	// watched frames (refinement): their proposed coarse cells as bits, and
	// the captured probability mass of each after maximize
	std::vector<int> h_watch;  // frame indices, ascending
	DevBuf<int> watch_local;
	DevBuf<uint32_t> watch_bits;
	DevBuf<double> watch_mass;
	int num_coarse = 0, rwords = 0;
	std::vector<int> h_qmap;
	DevBuf<int> qmap;
	DevBuf<uint32_t> rel_bits;
	// pair lists (option pair_lists with refinement): the live (tile, frame)
	// pairs tile-major, per-pair photon sums and probabilities, one
	// orientation block's log-slices or tomograms at a time (emc_pairs.cuh)
	bool pair_lists = false, pairs_valid = false, mw_valid = false, last_pairs = false;
	double block_budget_mb = 0.;
	std::vector<long long> h_rel_off;
	std::vector<int> h_rel;
	std::vector<uint8_t> h_rel_all;  // per frame: every coarse cell relevant (empty: none)
	HostBuf<int> stage_pairs;        // pair_tile, pair_frame, frame_pair staged for upload
	HostBuf<uint32_t> stage_bits;    // rel_bits staged for upload
	long long npairs = 0;
	std::vector<long long> h_tile_off;  // [RT + 1]
	DevBuf<long long> tile_off, frame_off;
	DevBuf<int> pair_tile, pair_frame, frame_pair;
	DevBuf<double> raw;
	DevBuf<float> blk, blkT;  // blkT: tomograms of the blocked full search
	bool blocked = false;         // the last full search ran in orientation blocks
	DevBuf<signed char> wsign;  // per orientation: weight change of the merge
	int blk_tiles = 0;
	DevBuf<uint32_t> mw;  // per frame: pixel | count << IDX_BITS on mask < 2 pixels
	DevBuf<long long> mw_off;
	bool timing = false;
	struct PhaseRec {
		int phase, ev;  // phase, begin event (end = ev + 1) in ev_pool
		long launches;
	};
	std::vector<cudaEvent_t> ev_pool;
	std::vector<PhaseRec> ev_pending;
	int ev_next = 0;
	int ev_open[PH_COUNT] = {-1, -1, -1, -1, -1, -1, -1};
	cudaEvent_t user_ev[8] = {};
	long long launches = 0;  // kernels launched by this context
	double phase_ms[PH_COUNT] = {};
	long phase_launches[PH_COUNT] = {};
	double rescale = 0., mutual_info = 0., avg_ll = 0., rms = 0.;
	bool have_results = false;

	int fail(int code, const char *fmt, ...) {
		char buf[1024];
		va_list ap;
		va_start(ap, fmt);
		vsnprintf(buf, sizeof(buf), fmt, ap);
		va_end(ap);
		err = buf;
		return code;
	}
};

#define CK(call)                                                                                  \
	do {                                                                                          \
		cudaError_t e_ = (call);                                                                  \
		if (e_ != cudaSuccess)                                                                    \
			return ctx->fail(e_ == cudaErrorMemoryAllocation ? DFG_ERR_NOMEM : DFG_ERR_CUDA,      \
			                 "%s failed: %s", #call, cudaGetErrorString(e_));                    \
	} while (0)

#define CKL(name)                                                                                 \
	do {                                                                                          \
		ctx->launches++;                                                                          \
		cudaError_t e_ = cudaGetLastError();                                                      \
		if (e_ != cudaSuccess)                                                                    \
			return ctx->fail(DFG_ERR_CUDA, "launch of %s failed: %s", name, cudaGetErrorString(e_)); \
	} while (0)

#define NEED(cond, code, ...)                                                                     \
	do {                                                                                          \
		if (!(cond))                                                                              \
			return ctx->fail(code, __VA_ARGS__);                                                  \
	} while (0)

static inline unsigned blocks_for(long long n, int per) { return (unsigned)((n + per - 1) / per); }

template <typename T>
static cudaError_t upload(DevBuf<T> &b, const T *h, size_t n, cudaStream_t s) {
	cudaError_t e = b.ensure(n);
	if (e != cudaSuccess || n == 0)
		return e;
	return cudaMemcpyAsync(b.p, h, n * sizeof(T), cudaMemcpyHostToDevice, s);
}

