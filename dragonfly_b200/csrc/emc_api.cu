// C ABI of the B200 EMC iteration (declared in include/dragonfly_b200.h).
//
// The context keeps every input resident in HBM and re-uses its work buffers
// across iterations. One iteration (dfg_maximize) is a fixed sequence of
// kernels on the context's stream:
//   slice_log -> u_reduce -> rescale                   (calculate_rescale + slices)
//   for each frame chunk:
//       estep -> norm -> psum_r -> mstep               (calculate_prob .. update_tomogram)
//   merge -> unpack -> [scale]                          (merge_tomogram, update_scale)
// The frame chunk bounds the per-pair buffers (12 bytes per orientation x frame).

#include <cudaTypedefs.h>

#include <thread>

#include "emc_ctx.cuh"
#include "emc_device.cuh"
#include "emc_bg.cuh"
#include "emc_dense.cuh"
#include "emc_pairs.cuh"

using namespace dfg;

// ---------------------------------------------------------------------------
// phase timing
// ---------------------------------------------------------------------------
// With option timing, each phase instance records a begin and an end event
// from a pool (no synchronisation, so the records can sit inside a captured
// graph); phase_collect adds the elapsed times up once the stream has
// synchronised. A pool that runs out leaves the rest of the call untimed.
static void phase_begin(dfg_ctx *ctx, int ph) {
	if (!ctx->timing || ctx->ev_next + 2 > (int)ctx->ev_pool.size())
		return;
	ctx->ev_open[ph] = ctx->ev_next;
	// under stream capture, external records become event-record nodes (the
	// flag is refused outside a capture)
	cudaEventRecordWithFlags(ctx->ev_pool[ctx->ev_next], ctx->stream,
	                         ctx->capturing ? cudaEventRecordExternal : cudaEventRecordDefault);
	ctx->ev_next += 2;
}
static void phase_end(dfg_ctx *ctx, int ph, long launches) {
	if (!ctx->timing || ctx->ev_open[ph] < 0)
		return;
	const int b = ctx->ev_open[ph];
	cudaEventRecordWithFlags(ctx->ev_pool[b + 1], ctx->stream,
	                         ctx->capturing ? cudaEventRecordExternal : cudaEventRecordDefault);
	ctx->ev_pending.push_back({ph, b, launches});
	ctx->ev_open[ph] = -1;
}
static void phase_collect(dfg_ctx *ctx) {
	for (const auto &q : ctx->ev_pending) {
		float ms = 0.f;
		if (cudaEventElapsedTime(&ms, ctx->ev_pool[q.ev], ctx->ev_pool[q.ev + 1]) == cudaSuccess)
			ctx->phase_ms[q.phase] += ms;
		ctx->phase_launches[q.phase] += q.launches;
	}
	cudaGetLastError();
	ctx->ev_pending.clear();
	ctx->ev_next = 0;
}

// ---------------------------------------------------------------------------
// lifetime
// ---------------------------------------------------------------------------
extern "C" const char *dfg_version(void) { return "dragonfly_b200 0.1 (sm_100a)"; }

extern "C" int dfg_create(int device, dfg_ctx **out) {
	if (out == nullptr)
		return DFG_ERR_ARG;
	*out = nullptr;
	int n = 0;
	if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n)
		return DFG_ERR_CUDA;
	if (cudaSetDevice(device) != cudaSuccess)
		return DFG_ERR_CUDA;
	dfg_ctx *ctx = new dfg_ctx();
	ctx->device = device;
	if (cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
	    ctx->num_sms < 1 ||
	    cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
		delete ctx;
		return DFG_ERR_CUDA;
	}
	ctx->ev_pool.assign(kTimingEvents, nullptr);
	for (auto &e : ctx->ev_pool)
		cudaEventCreate(&e);
	for (auto &e : ctx->user_ev)
		cudaEventCreate(&e);
	*out = ctx;
	return DFG_OK;
}

extern "C" void dfg_destroy(dfg_ctx *ctx) {
	if (ctx == nullptr)
		return;
	cudaSetDevice(ctx->device);
	cudaStreamSynchronize(ctx->stream);
	for (auto &e : ctx->ev_pool)
		if (e)
			cudaEventDestroy(e);
	for (auto &e : ctx->user_ev)
		if (e)
			cudaEventDestroy(e);
	if (ctx->graph_exec)
		cudaGraphExecDestroy(ctx->graph_exec);
	ctx->chunks.clear();
	cudaStreamDestroy(ctx->stream);
	delete ctx;
}

extern "C" const char *dfg_last_error(const dfg_ctx *ctx) {
	return ctx == nullptr ? "null context" : ctx->err.c_str();
}

// ---------------------------------------------------------------------------
// inputs
// ---------------------------------------------------------------------------
extern "C" int dfg_set_detector(dfg_ctx *ctx, int num_pix, const double *qvals, const double *corr,
                                const uint8_t *raw_mask) {
	if (!ctx)
		return DFG_ERR_ARG;
	NEED(num_pix > 0 && qvals && corr && raw_mask, DFG_ERR_ARG, "detector: need num_pix > 0 and arrays");
	NEED((uint32_t)num_pix <= IDX_MASK, DFG_ERR_ARG, "detector: at most %u pixels", IDX_MASK);
	for (long long i = 0; i < 3LL * num_pix; ++i)
		NEED(std::isfinite(qvals[i]), DFG_ERR_ARG, "detector: qvals[%lld] is not finite", i);
	for (int i = 0; i < num_pix; ++i)
		NEED(std::isfinite(corr[i]), DFG_ERR_ARG, "detector: corr[%d] is not finite", i);
	ctx->weight_cache_valid = false;
	CK(cudaSetDevice(ctx->device));
	if (ctx->P != 0 && ctx->P != num_pix)
		ctx->chunks_R = -1;
	ctx->P = num_pix;
	ctx->h_mask.assign(raw_mask, raw_mask + num_pix);
	ctx->tuned = false;
	ctx->dense_P = -1;  // pixel columns of the dense form follow the mask
	CK(upload(ctx->qvals, qvals, 3 * (size_t)num_pix, ctx->stream));
	CK(upload(ctx->corr, corr, (size_t)num_pix, ctx->stream));
	CK(upload(ctx->mask, raw_mask, (size_t)num_pix, ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	ctx->chunks_R = -1;  // photon lists depend on the mask
	if (ctx->N > 0) {
		int rc = dfg_set_frames(ctx, ctx->N, ctx->h_ones.data(), ctx->h_multi.data(), ctx->h_place_ones.data(),
		                        ctx->h_place_multi.data(), ctx->h_count_multi.data());
		if (rc != DFG_OK)
			return rc;
	}
	return DFG_OK;
}

// Runs fn(thread, begin, end) over [0, n) split into contiguous ranges, one
// per host thread (ascending ranges for ascending thread numbers).
template <typename F>
static void parallel_ranges(long long n, int threads, F fn) {
	std::vector<std::thread> pool;
	for (int k = 0; k < threads; ++k) {
		const long long b = n * k / threads, e = n * (k + 1) / threads;
		pool.emplace_back([=, &fn] { fn(k, b, e); });
	}
	for (auto &t : pool)
		t.join();
}

// Packs (index, count) words, splitting counts above MAX_COUNT.
static inline void push_word(std::vector<uint32_t> &v, uint32_t idx, long long count) {
	while (count > 0) {
		uint32_t c = (uint32_t)std::min<long long>(count, MAX_COUNT);
		v.push_back(idx | (c << IDX_BITS));
		count -= c;
	}
}

// Pads a segment that started at `start` to a multiple of 8 words with `pad`
// (an index whose row is all zero, count 0).
static inline void pad8(std::vector<uint32_t> &v, size_t start, uint32_t pad) {
	while ((v.size() - start) % 8)
		v.push_back(pad);
}

extern "C" int dfg_set_frames(dfg_ctx *ctx, int num_data, const int *ones, const int *multi,
                              const int *place_ones, const int *place_multi, const int *count_multi) {
	if (!ctx)
		return DFG_ERR_ARG;
	NEED(ctx->P > 0, DFG_ERR_STATE, "frames: set the detector first");
	NEED(num_data > 0 && ones && multi, DFG_ERR_ARG, "frames: need num_data > 0, ones and multi");
	NEED((uint32_t)num_data <= IDX_MASK + 1u, DFG_ERR_ARG, "frames: at most %u frames", IDX_MASK + 1u);
	CK(cudaSetDevice(ctx->device));
	const int N = num_data, P = ctx->P;
	std::vector<long long> oo(N + 1, 0), mo(N + 1, 0);
	for (int d = 0; d < N; ++d) {
		NEED(ones[d] >= 0 && multi[d] >= 0, DFG_ERR_ARG, "frames: negative ones/multi at frame %d", d);
		oo[d + 1] = oo[d] + ones[d];
		mo[d + 1] = mo[d] + multi[d];
	}
	NEED(oo[N] == 0 || place_ones, DFG_ERR_ARG, "frames: place_ones missing");
	NEED(mo[N] == 0 || (place_multi && count_multi), DFG_ERR_ARG, "frames: place_multi/count_multi missing");
	for (long long i = 0; i < oo[N]; ++i)
		NEED(place_ones[i] >= 0 && place_ones[i] < P, DFG_ERR_ARG, "frames: place_ones[%lld] = %d out of [0, %d)",
		     i, place_ones[i], P);
	for (long long i = 0; i < mo[N]; ++i) {
		NEED(place_multi[i] >= 0 && place_multi[i] < P, DFG_ERR_ARG,
		     "frames: place_multi[%lld] = %d out of [0, %d)", i, place_multi[i], P);
		NEED(count_multi[i] >= 1, DFG_ERR_ARG, "frames: count_multi[%lld] = %d < 1", i, count_multi[i]);
	}
	// host copies (the M-step index is rebuilt per frame chunk)
	if (ones != ctx->h_ones.data()) {
		ctx->h_ones.assign(ones, ones + N);
		ctx->h_multi.assign(multi, multi + N);
		ctx->h_place_ones.assign(place_ones, place_ones + oo[N]);
		ctx->h_place_multi.assign(place_multi, place_multi + mo[N]);
		ctx->h_count_multi.assign(count_multi, count_multi + mo[N]);
	}
	ctx->h_ones_off = oo;
	ctx->h_multi_off = mo;
	ctx->powder_valid = false;
	if ((int)ctx->h_bgscale.size() != N)
		ctx->h_bgscale.clear();
	ctx->N = N;

	// E-step lists: photons on mask == 0 pixels, ones then multi, per frame;
	// fcounts, sum_fact, mean_count as calc_frame_counts / calc_sum_fact
	// (iterate.c:3-117).
	const uint8_t *mk = ctx->h_mask.data();
	const uint32_t pad = (uint32_t)P;  // zero row of logW
	std::vector<uint32_t> words;
	words.reserve((size_t)(oo[N] + mo[N] + 16 * (size_t)N));
	std::vector<long long> off(N + 1, 0), midv(N, 0);
	std::vector<int> fc(N, 0);
	std::vector<double> sf(N, 0.);
	double mc = 0.;
	long long real = 0;
	for (int d = 0; d < N; ++d) {
		size_t st = words.size();
		for (long long i = oo[d]; i < oo[d + 1]; ++i) {
			int p = ctx->h_place_ones[i];
			if (mk[p] < 1) {
				words.push_back((uint32_t)p);
				fc[d]++;
				real++;
			}
		}
		pad8(words, st, pad);
		midv[d] = (long long)words.size();
		st = words.size();
		for (long long i = mo[d]; i < mo[d + 1]; ++i) {
			int p = ctx->h_place_multi[i], c = ctx->h_count_multi[i];
			if (mk[p] < 1) {
				size_t before = words.size();
				push_word(words, (uint32_t)p, c);
				real += (long long)(words.size() - before);
				fc[d] += c;
				sf[d] += std::lgamma((double)c + 1.0);
			}
		}
		pad8(words, st, pad);
		off[d + 1] = (long long)words.size();
		mc += fc[d];
	}
	ctx->mean_count = mc / N;
	ctx->n_ph = real;
	CK(upload(ctx->ph, words.data(), words.size(), ctx->stream));
	CK(upload(ctx->ph_off, off.data(), off.size(), ctx->stream));
	CK(upload(ctx->ph_mid, midv.data(), midv.size(), ctx->stream));
	CK(upload(ctx->fcounts, fc.data(), (size_t)N, ctx->stream));
	CK(upload(ctx->sum_fact, sf.data(), (size_t)N, ctx->stream));
	std::vector<double> ones_d(N, 1.);
	std::vector<uint8_t> zeros(N, 0);
	CK(upload(ctx->scale, ones_d.data(), (size_t)N, ctx->stream));
	CK(upload(ctx->blacklist, zeros.data(), (size_t)N, ctx->stream));
	CK(ctx->beta.ensure((size_t)N));
	CK(ctx->beta_start.ensure((size_t)N));
	CK(cudaStreamSynchronize(ctx->stream));
	ctx->beta_set = false;
	ctx->chunks_R = -1;
	ctx->have_results = false;
	ctx->refine = false;  // relevant orientations are per frame
	ctx->pairs_valid = ctx->mw_valid = false;
	ctx->max_count0 = -1;
	ctx->tuned = false;
	return DFG_OK;
}

extern "C" int dfg_set_quaternions(dfg_ctx *ctx, int num_rot, const double *quats) {
	if (!ctx)
		return DFG_ERR_ARG;
	NEED(num_rot > 0 && quats, DFG_ERR_ARG, "quaternions: need num_rot > 0");
	for (long long i = 0; i < 5LL * num_rot; ++i)
		NEED(std::isfinite(quats[i]), DFG_ERR_ARG, "quaternions: entry %lld is not finite", i);
	ctx->weight_cache_valid = false;
	CK(cudaSetDevice(ctx->device));
	if (num_rot != ctx->num_rot) {
		ctx->refine = false;  // the coarse map was made for the previous set
		ctx->tuned = false;
	}
	ctx->num_rot = num_rot;
	CK(upload(ctx->quats, quats, 5 * (size_t)num_rot, ctx->stream));
	std::vector<double> cs(2 * (size_t)num_rot);
	for (int r = 0; r < num_rot; ++r) {
		cs[2 * (size_t)r] = std::cos(quats[5 * (size_t)r]);
		cs[2 * (size_t)r + 1] = std::sin(quats[5 * (size_t)r]);
	}
	CK(upload(ctx->cs2d, cs.data(), cs.size(), ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	return DFG_OK;
}

extern "C" int dfg_set_model(dfg_ctx *ctx, long size, int num_modes, const double *model1) {
	if (!ctx)
		return DFG_ERR_ARG;
	NEED(size >= 3 && num_modes >= 1 && model1, DFG_ERR_ARG, "model: need size >= 3, num_modes >= 1");
	NEED(num_modes <= MAX_MODES, DFG_ERR_ARG, "model: at most %d modes", MAX_MODES);
	ctx->weight_cache_valid = false;
	CK(cudaSetDevice(ctx->device));
	if (size != ctx->S || num_modes != ctx->M)
		ctx->tuned = false;
	ctx->S = size;
	ctx->V = ctx->model_type == MT_3D ? (long long)size * size * size : (long long)size * size;
	ctx->M = num_modes;
	const size_t n = (size_t)num_modes * ctx->V;
	CK(upload(ctx->model1, model1, n, ctx->stream));
	CK(ctx->model2.ensure(n));
	CK(ctx->weight.ensure(n));
	CK(ctx->accum.ensure(n));
	CK(cudaMemsetAsync(ctx->model2.p, 0, n * sizeof(double), ctx->stream));
	CK(cudaMemsetAsync(ctx->weight.p, 0, n * sizeof(double), ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	return DFG_OK;
}

static int need_frames(dfg_ctx *ctx) {
	NEED(ctx->N > 0, DFG_ERR_STATE, "set the frames first");
	return DFG_OK;
}

extern "C" int dfg_set_model_type(dfg_ctx *ctx, int model_type, int friedel_sym) {
	if (!ctx)
		return DFG_ERR_ARG;
	NEED(model_type == MT_3D || model_type == MT_2D || model_type == MT_RZ, DFG_ERR_ARG,
	     "model_type must be 0 (3-D), 1 (2-D) or 2 (RZ)");
	if (model_type != ctx->model_type) {
		ctx->S = 0;  // the model must be set again with its new shape
		ctx->V = 0;
		ctx->weight_cache_valid = false;
	}
	ctx->model_type = model_type;
	ctx->friedel2d = friedel_sym != 0;
	return DFG_OK;
}

extern "C" int dfg_set_detector_distance(dfg_ctx *ctx, double detd) {
	if (!ctx)
		return DFG_ERR_ARG;
	NEED(std::isfinite(detd), DFG_ERR_ARG, "detector distance must be finite");
	ctx->detd = detd;
	return DFG_OK;
}

// The common end of dfg_set_refinement / dfg_set_refinement_topk: the cell
// bits go up, the coarse map is kept, the pair lists are rebuilt at the next
// iteration.
static int finish_refinement(dfg_ctx *ctx, int num_coarse, const int *quat_mapping, const uint32_t *bits,
                             size_t nbits) {
	CK(cudaSetDevice(ctx->device));
	CK(upload(ctx->rel_bits, bits, nbits, ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	ctx->h_qmap.assign(quat_mapping, quat_mapping + ctx->num_rot);
	ctx->pairs_valid = false;
	if (num_coarse != ctx->num_coarse)
		ctx->h_watch.clear();  // the cell bits were for another coarse set
	ctx->num_coarse = num_coarse;
	ctx->rwords = (num_coarse + 31) / 32;
	ctx->refine = true;
	ctx->qmap_valid = false;
	return DFG_OK;
}

extern "C" int dfg_set_refinement_topk(dfg_ctx *ctx, int num_coarse, const int *quat_mapping, int K, const int *top,
                                       int n_all, const int *all_frames) {
	if (!ctx)
		return DFG_ERR_ARG;
	if (int rc = need_frames(ctx))
		return rc;
	NEED(ctx->num_rot > 0, DFG_ERR_STATE, "refinement: set the quaternions first");
	NEED(num_coarse > 0 && quat_mapping && K >= 1 && top && n_all >= 0 && (n_all == 0 || all_frames), DFG_ERR_ARG,
	     "refinement: need num_coarse > 0, the coarse map, K >= 1 cells per frame and the full-search frames");
	const int N = ctx->N, rw = (num_coarse + 31) / 32;
	for (int r = 0; r < ctx->num_rot; ++r)
		NEED(quat_mapping[r] >= 0 && quat_mapping[r] < num_coarse, DFG_ERR_ARG,
		     "refinement: quat_mapping[%d] = %d outside [0, %d)", r, quat_mapping[r], num_coarse);
	std::vector<uint8_t> all((size_t)N, 0);
	for (int i = 0; i < n_all; ++i) {
		NEED(all_frames[i] >= 0 && all_frames[i] < N, DFG_ERR_ARG, "refinement: frame %d out of range",
		     all_frames[i]);
		all[all_frames[i]] = 1;
	}
	CK(cudaSetDevice(ctx->device));
	CK(ctx->stage_bits.ensure((size_t)N * rw));
	uint32_t *bits = ctx->stage_bits.p;
	const int nth = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
	std::vector<long long> bad((size_t)nth, -1);
	const uint32_t last = (num_coarse & 31) ? ((1u << (num_coarse & 31)) - 1u) : 0xffffffffu;
	parallel_ranges(N, std::min<int>(nth, std::max(1, N / 4096)), [&](int k, long long b, long long e) {
		for (long long d = b; d < e; ++d) {
			uint32_t *w = bits + (size_t)d * rw;
			if (all[d]) {
				for (int j = 0; j < rw; ++j)
					w[j] = j + 1 < rw ? 0xffffffffu : last;
				continue;
			}
			for (int j = 0; j < rw; ++j)
				w[j] = 0u;
			for (long long t = d * K; t < (d + 1) * K; ++t) {
				const int c = top[t];
				if (c == -1)  // an unused slot
					continue;
				if (c < 0 || c >= num_coarse) {
					if (bad[k] < 0)
						bad[k] = t;
					continue;
				}
				w[c >> 5] |= 1u << (c & 31);
			}
		}
	});
	for (long long t : bad)
		NEED(t < 0, DFG_ERR_ARG, "refinement: entry %lld lists coarse orientation %d outside [0, %d)", t, top[t],
		     num_coarse);
	ctx->h_rel_off.resize((size_t)N + 1);
	for (int d = 0; d <= N; ++d)
		ctx->h_rel_off[d] = (long long)d * K;
	ctx->h_rel.assign(top, top + (size_t)N * K);
	ctx->h_rel_all = std::move(all);
	return finish_refinement(ctx, num_coarse, quat_mapping, bits, (size_t)N * rw);
}

extern "C" int dfg_set_refinement(dfg_ctx *ctx, int num_coarse, const int *quat_mapping,
                                  const long long *rel_off, const int *rel_quat) {
	if (!ctx)
		return DFG_ERR_ARG;
	if (quat_mapping == nullptr) {
		ctx->refine = false;
		return DFG_OK;
	}
	if (int rc = need_frames(ctx))
		return rc;
	NEED(ctx->num_rot > 0, DFG_ERR_STATE, "refinement: set the quaternions first");
	NEED(num_coarse > 0 && rel_off && (rel_quat || rel_off[ctx->N] == 0), DFG_ERR_ARG,
	     "refinement: need num_coarse > 0 and the per-frame lists");
	const int N = ctx->N, rw = (num_coarse + 31) / 32;
	for (int r = 0; r < ctx->num_rot; ++r)
		NEED(quat_mapping[r] >= 0 && quat_mapping[r] < num_coarse, DFG_ERR_ARG,
		     "refinement: quat_mapping[%d] = %d outside [0, %d)", r, quat_mapping[r], num_coarse);
	NEED(rel_off[0] == 0, DFG_ERR_ARG, "refinement: rel_off[0] must be 0");
	for (int d = 0; d < N; ++d)
		NEED(rel_off[d + 1] >= rel_off[d], DFG_ERR_ARG, "refinement: rel_off decreases at frame %d", d);
	// one bit per relevant coarse orientation, frames split over the host
	// threads; the first bad entry of each range is reported
	CK(cudaSetDevice(ctx->device));
	CK(ctx->stage_bits.ensure((size_t)N * rw));
	uint32_t *bits = ctx->stage_bits.p;
	const int nth = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
	std::vector<long long> bad((size_t)nth, -1);
	parallel_ranges(N, std::min<int>(nth, std::max(1, N / 4096)), [&](int k, long long b, long long e) {
		std::fill(bits + (size_t)b * rw, bits + (size_t)e * rw, 0u);
		for (long long d = b; d < e; ++d)
			for (long long t = rel_off[d]; t < rel_off[d + 1]; ++t) {
				const int c = rel_quat[t];
				if (c < 0 || c >= num_coarse) {
					if (bad[k] < 0)
						bad[k] = t;
					continue;
				}
				bits[(size_t)d * rw + (c >> 5)] |= 1u << (c & 31);
			}
	});
	for (long long t : bad)
		NEED(t < 0, DFG_ERR_ARG, "refinement: entry %lld lists coarse orientation %d outside [0, %d)", t, rel_quat[t],
		     num_coarse);
	ctx->h_rel_off.assign(rel_off, rel_off + N + 1);
	ctx->h_rel.assign(rel_quat, rel_quat + rel_off[N]);
	ctx->h_rel_all.clear();
	return finish_refinement(ctx, num_coarse, quat_mapping, bits, (size_t)N * rw);
}

extern "C" int dfg_set_watch(dfg_ctx *ctx, int n, const int *frames, const long long *cell_off, const int *cells) {
	if (!ctx)
		return DFG_ERR_ARG;
	if (n == 0 || frames == nullptr) {
		ctx->h_watch.clear();
		return DFG_OK;
	}
	NEED(ctx->refine, DFG_ERR_STATE, "watched frames need refinement (dfg_set_refinement) first");
	NEED(n > 0 && cell_off && cells && cell_off[0] == 0, DFG_ERR_ARG, "watch: need frames and cell lists");
	const int rw = ctx->rwords;
	std::vector<uint32_t> bits((size_t)n * rw, 0u);
	for (int i = 0; i < n; ++i) {
		NEED(frames[i] >= 0 && frames[i] < ctx->N && (i == 0 || frames[i] > frames[i - 1]), DFG_ERR_ARG,
		     "watch: frames must be ascending and in range");
		for (long long t = cell_off[i]; t < cell_off[i + 1]; ++t) {
			NEED(cells[t] >= 0 && cells[t] < ctx->num_coarse, DFG_ERR_ARG, "watch: cell %d out of range", cells[t]);
			bits[(size_t)i * rw + (cells[t] >> 5)] |= 1u << (cells[t] & 31);
		}
	}
	CK(cudaSetDevice(ctx->device));
	CK(upload(ctx->watch_bits, bits.data(), bits.size(), ctx->stream));
	CK(ctx->watch_local.ensure((size_t)n));
	CK(ctx->watch_mass.ensure((size_t)n));
	CK(cudaStreamSynchronize(ctx->stream));
	ctx->h_watch.assign(frames, frames + n);
	return DFG_OK;
}

extern "C" int dfg_get_watch_mass(dfg_ctx *ctx, double *mass) {
	if (!ctx || !mass)
		return DFG_ERR_ARG;
	NEED(!ctx->h_watch.empty(), DFG_ERR_STATE, "no watched frames");
	CK(cudaSetDevice(ctx->device));
	CK(cudaMemcpy(mass, ctx->watch_mass.p, ctx->h_watch.size() * sizeof(double), cudaMemcpyDeviceToHost));
	return DFG_OK;
}

extern "C" int dfg_voronoi_subset(dfg_ctx *ctx, int num_coarse, const double *coarse, int num_fine,
                                  const double *fine, int *nearest) {
	if (!ctx)
		return DFG_ERR_ARG;
	NEED(num_coarse > 0 && num_fine >= 0 && coarse && (fine && nearest || num_fine == 0), DFG_ERR_ARG,
	     "voronoi_subset: need coarse and fine quaternions");
	if (num_fine == 0)
		return DFG_OK;
	CK(cudaSetDevice(ctx->device));
	cudaStream_t st = ctx->stream;
	DevBuf<double> c, f;
	DevBuf<int> o;
	CK(upload(c, coarse, 5 * (size_t)num_coarse, st));
	CK(upload(f, fine, 5 * (size_t)num_fine, st));
	CK(o.ensure((size_t)num_fine));
	voronoi_kernel<<<blocks_for(num_fine, 256), 256, 0, st>>>(c.p, num_coarse, f.p, num_fine, o.p);
	CKL("voronoi_kernel");
	CK(cudaMemcpyAsync(nearest, o.p, (size_t)num_fine * sizeof(int), cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	return DFG_OK;
}

extern "C" int dfg_set_scale(dfg_ctx *ctx, const double *scale) {
	if (!ctx || !scale)
		return DFG_ERR_ARG;
	if (int rc = need_frames(ctx))
		return rc;
	CK(cudaSetDevice(ctx->device));
	CK(upload(ctx->scale, scale, (size_t)ctx->N, ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	return DFG_OK;
}

extern "C" int dfg_set_background(dfg_ctx *ctx, const double *background) {
	if (!ctx)
		return DFG_ERR_ARG;
	NEED(ctx->P > 0, DFG_ERR_STATE, "background: set the detector first");
	if (background == nullptr) {
		ctx->with_bg = false;
		return DFG_OK;
	}
	const int P = ctx->P;
	for (int t = 0; t < P; ++t)
		NEED(std::isfinite(background[t]), DFG_ERR_ARG, "background[%d] is not finite", t);
	CK(cudaSetDevice(ctx->device));
	CK(upload(ctx->background, background, (size_t)P, ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	ctx->with_bg = true;
	ctx->powder_valid = false;
	return DFG_OK;
}

extern "C" int dfg_set_bgscale(dfg_ctx *ctx, const double *bgscale) {
	if (!ctx)
		return DFG_ERR_ARG;
	NEED(ctx->N > 0, DFG_ERR_STATE, "bgscale: set the frames first");
	if (bgscale == nullptr) {
		ctx->h_bgscale.clear();
		return DFG_OK;
	}
	for (int d = 0; d < ctx->N; ++d)
		NEED(std::isfinite(bgscale[d]), DFG_ERR_ARG, "bgscale[%d] is not finite", d);
	ctx->h_bgscale.assign(bgscale, bgscale + ctx->N);
	return DFG_OK;
}

// Powder sum and per-frame background scales for the background-aware path:
// powder[t] = photons on mask-0 pixel t summed over all frames / num_data
// (calc_powder, iterate.c:119-177); bgscale defaults to ones (iterate.pyx:290-296).
static int ensure_bg(dfg_ctx *ctx) {
	const int N = ctx->N, P = ctx->P;
	cudaStream_t st = ctx->stream;
	if (!ctx->powder_valid) {
		std::vector<double> pw(P, 0.);
		const uint8_t *mk = ctx->h_mask.data();
		for (int d = 0; d < N; ++d) {
			for (long long i = ctx->h_ones_off[d]; i < ctx->h_ones_off[d + 1]; ++i)
				if (mk[ctx->h_place_ones[i]] < 1)
					pw[ctx->h_place_ones[i]] += 1.;
			for (long long i = ctx->h_multi_off[d]; i < ctx->h_multi_off[d + 1]; ++i)
				if (mk[ctx->h_place_multi[i]] < 1)
					pw[ctx->h_place_multi[i]] += ctx->h_count_multi[i];
		}
		for (int t = 0; t < P; ++t)
			pw[t] /= N;
		CK(upload(ctx->powder, pw.data(), pw.size(), st));
		ctx->powder_valid = true;
	}
	std::vector<double> bs = ctx->h_bgscale;
	if ((int)bs.size() != N)
		bs.assign(N, 1.);
	CK(upload(ctx->bgscale, bs.data(), bs.size(), st));
	const int nsplit = std::max(1, std::min(64, ctx->chunk_frames / 2048));
	CK(ctx->scalemax.ensure((size_t)ctx->R_pad));
	CK(ctx->smax_part.ensure((size_t)nsplit * ctx->R_pad));
	CK(ctx->gd_part.ensure((size_t)ctx->RT * ctx->chunk_frames));
	CK(ctx->gd_G.ensure((size_t)N));
	CK(ctx->gd_s.ensure((size_t)N));
	CK(ctx->gd_active.ensure((size_t)N));
	CK(ctx->Wd.ensure((size_t)ctx->RT * (P + 1) * TILE));
	CK(ctx->Pd.ensure((size_t)ctx->R_pad * (ctx->chunk_frames + 1)));
	CK(cudaStreamSynchronize(st));
	return DFG_OK;
}

extern "C" int dfg_set_blacklist(dfg_ctx *ctx, const uint8_t *blacklist) {
	if (!ctx || !blacklist)
		return DFG_ERR_ARG;
	if (int rc = need_frames(ctx))
		return rc;
	CK(cudaSetDevice(ctx->device));
	CK(upload(ctx->blacklist, blacklist, (size_t)ctx->N, ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	return DFG_OK;
}

extern "C" int dfg_set_beta_start(dfg_ctx *ctx, const double *beta_start) {
	if (!ctx || !beta_start)
		return DFG_ERR_ARG;
	if (int rc = need_frames(ctx))
		return rc;
	for (int d = 0; d < ctx->N; ++d)
		NEED(beta_start[d] > 0. && std::isfinite(beta_start[d]), DFG_ERR_ARG, "beta_start[%d] must be > 0", d);
	CK(cudaSetDevice(ctx->device));
	CK(upload(ctx->beta_start, beta_start, (size_t)ctx->N, ctx->stream));
	CK(cudaMemcpyAsync(ctx->beta.p, beta_start, (size_t)ctx->N * sizeof(double), cudaMemcpyHostToDevice,
	                   ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	ctx->beta_set = true;
	return DFG_OK;
}

extern "C" int dfg_calc_beta(dfg_ctx *ctx, double start, int need_scaling) {
	if (!ctx)
		return DFG_ERR_ARG;
	if (int rc = need_frames(ctx))
		return rc;
	// iterate.c:66-83
	std::vector<int> fc(ctx->N);
	CK(cudaSetDevice(ctx->device));
	CK(cudaMemcpy(fc.data(), ctx->fcounts.p, (size_t)ctx->N * sizeof(int), cudaMemcpyDeviceToHost));
	if (!need_scaling && start < 0)
		start = std::exp(-6.5 * std::pow(ctx->mean_count * 1.e-5, 0.15));
	std::vector<double> b(ctx->N);
	for (int d = 0; d < ctx->N; ++d)
		b[d] = start > 0 ? start : std::exp(-6.5 * std::pow(fc[d] * 1.e-5, 0.15));
	return dfg_set_beta_start(ctx, b.data());
}

// ---------------------------------------------------------------------------
// work buffers and the frame chunks
// ---------------------------------------------------------------------------
static int build_chunks(dfg_ctx *ctx) {
	const int N = ctx->N, P = ctx->P;
	// per frame: pval and Pst of every orientation, plus its BF16 count row
	// in the dense form
	const bool any_dense = ctx->dense_active || ctx->m_dense_active;
	const size_t pair_bytes = (size_t)ctx->RT * TILE * (sizeof(double) + sizeof(float)) +
	                          (any_dense ? (size_t)ctx->K_pad * 2 : 0) +
	                          (ctx->m_dense_active ? (size_t)ctx->RT * TILE * 4 : 0);
	size_t budget;
	if (ctx->pair_budget_mb > 0.) {
		budget = (size_t)(ctx->pair_budget_mb * 1048576.);
	} else {
		size_t fr = 0, tot = 0;
		CK(cudaMemGetInfo(&fr, &tot));
		budget = (size_t)(0.6 * (double)fr);
	}
	long long nc = (long long)(budget / pair_bytes);
	NEED(nc >= 1, DFG_ERR_NOMEM, "pair buffers: %zu bytes per frame exceed the budget", pair_bytes);
	nc = std::min<long long>(nc, N);
	const int n_chunks = (int)((N + nc - 1) / nc);
	nc = (N + n_chunks - 1) / n_chunks;  // even chunks
	ctx->chunk_frames = (int)nc;
	ctx->chunks.clear();
	ctx->chunks.resize(n_chunks);

	// M-step index per chunk: photons on mask < 2 pixels grouped by pixel
	// (two counting sorts), frames ascending; per pixel a count-1 segment and
	// a multi-photon segment, each padded to 8 words with the chunk's zero
	// row Nc.
	NEED(nc <= (long long)IDX_MASK, DFG_ERR_ARG, "frame chunk of %lld frames exceeds %u", nc, IDX_MASK);
	const uint8_t *mk = ctx->h_mask.data();
	std::vector<long long> c1(P + 1), cm(P + 1);
	std::vector<uint32_t> words;
	for (int k = 0; k < n_chunks; ++k) {
		Chunk &ch = ctx->chunks[k];
		ch.d0 = (int)(k * nc);
		ch.nc = (int)std::min<long long>(nc, N - ch.d0);
		const uint32_t pad = (uint32_t)ch.nc;
		std::fill(c1.begin(), c1.end(), 0);
		std::fill(cm.begin(), cm.end(), 0);
		auto each = [&](auto fn) {
			for (int dl = 0; dl < ch.nc; ++dl) {
				int d = ch.d0 + dl;
				for (long long i = ctx->h_ones_off[d]; i < ctx->h_ones_off[d + 1]; ++i) {
					int p = ctx->h_place_ones[i];
					if (mk[p] < 2)
						fn(p, dl, 1LL);
				}
				for (long long i = ctx->h_multi_off[d]; i < ctx->h_multi_off[d + 1]; ++i) {
					int p = ctx->h_place_multi[i];
					if (mk[p] < 2)
						fn(p, dl, (long long)ctx->h_count_multi[i]);
				}
			}
		};
		each([&](int p, int, long long c) {
			if (c == 1)
				c1[p]++;
			else
				cm[p] += (c + MAX_COUNT - 1) / MAX_COUNT;
		});
		std::vector<long long> off(P + 1, 0), midv(P, 0), f1(P), fm(P);
		long long real = 0;
		for (int p = 0; p < P; ++p) {
			const long long a = (c1[p] + 7) / 8 * 8, b = (cm[p] + 7) / 8 * 8;
			f1[p] = off[p];
			midv[p] = off[p] + a;
			fm[p] = midv[p];
			off[p + 1] = off[p] + a + b;
			real += c1[p] + cm[p];
		}
		words.assign((size_t)off[P], pad);
		each([&](int p, int dl, long long c) {
			if (c == 1) {
				words[(size_t)f1[p]++] = (uint32_t)dl;
				return;
			}
			while (c > 0) {
				uint32_t cc = (uint32_t)std::min<long long>(c, MAX_COUNT);
				words[(size_t)fm[p]++] = (uint32_t)dl | (cc << IDX_BITS);
				c -= cc;
			}
		});
		std::vector<int> pix;
		for (int p = 0; p < P; ++p)
			if (off[p + 1] > off[p])
				pix.push_back(p);
		std::stable_sort(pix.begin(), pix.end(),
		                 [&](int a, int b) { return off[a + 1] - off[a] > off[b + 1] - off[b]; });
		ch.npix = (int)pix.size();
		ch.entries = real;
		CK(upload(ch.cs, words.data(), words.size(), ctx->stream));
		CK(upload(ch.cs_off, off.data(), off.size(), ctx->stream));
		CK(upload(ch.cs_mid, midv.data(), midv.size(), ctx->stream));
		CK(upload(ch.pix, pix.data(), pix.size(), ctx->stream));
		CK(cudaStreamSynchronize(ctx->stream));
	}
	ctx->chunks_R = ctx->R;
	ctx->chunks_dense = (ctx->dense_active ? 1 : 0) | (ctx->m_dense_active ? 2 : 0);
	return DFG_OK;
}

static int ensure_buffers(dfg_ctx *ctx) {
	NEED(ctx->P > 0, DFG_ERR_STATE, "detector not set");
	NEED(ctx->N > 0, DFG_ERR_STATE, "frames not set");
	NEED(ctx->num_rot > 0, DFG_ERR_STATE, "quaternions not set");
	NEED(ctx->S > 0, DFG_ERR_STATE, "model not set");
	NEED(ctx->beta_set, DFG_ERR_STATE, "beta not set (dfg_calc_beta or dfg_set_beta_start)");
	ctx->R = ctx->M * ctx->num_rot;
	ctx->RT = (ctx->R + TILE - 1) / TILE;
	ctx->R_pad = ctx->RT * TILE;
	const size_t tiles_px = (size_t)ctx->RT * ctx->P * TILE;
	const size_t logw_n = (size_t)ctx->RT * (ctx->P + 1) * TILE;
	if (ctx->logW.n < logw_n || ctx->logW_P != ctx->P) {
		CK(ctx->logW.ensure(logw_n));
		// the zero rows (pixel P of every tile) stay zero: the slice kernel
		// writes rows 0..P-1 only
		CK(cudaMemsetAsync(ctx->logW.p, 0, logw_n * sizeof(float), ctx->stream));
		ctx->logW_P = ctx->P;
	}
	CK(ctx->T.ensure(tiles_px));
	CK(ctx->u.ensure((size_t)ctx->R_pad));
	CK(ctx->logw.ensure((size_t)ctx->R_pad));
	CK(ctx->psum_r.ensure((size_t)ctx->R_pad));
	CK(ctx->scalars.ensure(8));
	CK(ctx->red_part.ensure(std::max<size_t>(blocks_for((long long)ctx->M * ctx->V, 256), 1024)));
	const size_t N = (size_t)ctx->N;
	CK(ctx->rmax.ensure(N));
	CK(ctx->num_prob.ensure(N));
	CK(ctx->info.ensure(N));
	CK(ctx->likelihood.ensure(N));
	CK(ctx->max_exp.ensure(N));
	CK(ctx->p_norm.ensure(N));
	CK(ctx->psum_d.ensure(N));
	CK(ctx->quat_norm.ensure(N * ctx->M));
	if (ctx->chunks_R != ctx->R ||
	    ctx->chunks_dense != ((ctx->dense_active ? 1 : 0) | (ctx->m_dense_active ? 2 : 0))) {
		ctx->pval.release();
		ctx->Pst.release();
		ctx->tmax.release();
		ctx->targ.release();
		if (int rc = build_chunks(ctx))
			return rc;
	}
	const size_t pairs = (size_t)ctx->R_pad * ctx->chunk_frames;
	CK(ctx->pval.ensure(pairs));
	CK(ctx->Pst.ensure((size_t)ctx->R_pad * (ctx->chunk_frames + 1)));
	CK(ctx->tmax.ensure((size_t)ctx->RT * ctx->chunk_frames));
	CK(ctx->targ.ensure((size_t)ctx->RT * ctx->chunk_frames));
	CK(ctx->tlive.ensure((size_t)ctx->RT * (ctx->chunk_frames + 1)));
	const int nsplit = std::max(1, std::min(64, ctx->chunk_frames / 2048));
	CK(ctx->psum_part.ensure((size_t)nsplit * ctx->R_pad));
	return DFG_OK;
}

// ---------------------------------------------------------------------------
// the iteration
// ---------------------------------------------------------------------------
// Sparse probabilities of one frame chunk, copied to the host lists: the
// pairs with P > PROB_MIN of every frame, in orientation order, as the
// reference's combined and resparsified prob / place_prob (max_prob.c:294-325).
// Runs after the chunk's normalisation, while its log-likelihoods are held.
static int collect_prob(dfg_ctx *ctx, const Chunk &ch) {
	cudaStream_t st = ctx->stream;
	const int Nc = ch.nc, RT = ctx->RT;
	CK(ctx->prob_count.ensure((size_t)Nc));
	count_prob_kernel<<<blocks_for(Nc, 8), 256, 0, st>>>(ctx->Pst.p, RT, Nc, ctx->prob_count.p);
	CKL("count_prob_kernel");
	std::vector<int> cnt(Nc);
	CK(cudaMemcpyAsync(cnt.data(), ctx->prob_count.p, (size_t)Nc * sizeof(int), cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	std::vector<long long> off((size_t)Nc + 1, 0);
	for (int k = 0; k < Nc; ++k)
		off[k + 1] = off[k] + cnt[k];
	const long long total = off[Nc], base = ctx->h_prob_off[ch.d0];
	for (int k = 0; k < Nc; ++k)
		ctx->h_prob_off[(size_t)ch.d0 + k + 1] = base + off[k + 1];
	if (total == 0)
		return DFG_OK;
	CK(upload(ctx->d_prob_off, off.data(), off.size(), st));
	CK(ctx->d_place.ensure((size_t)total));
	CK(ctx->d_prob.ensure((size_t)total));
	compact_prob_kernel<<<blocks_for(Nc, 8), 256, 0, st>>>(ctx->pval.p, ctx->Pst.p, RT, Nc, ch.d0, ctx->beta.p,
	                                                        ctx->max_exp.p, ctx->p_norm.p, ctx->d_prob_off.p,
	                                                        ctx->d_place.p, ctx->d_prob.p);
	CKL("compact_prob_kernel");
	ctx->h_place_prob.resize((size_t)(base + total));
	ctx->h_prob.resize((size_t)(base + total));
	CK(cudaMemcpyAsync(ctx->h_place_prob.data() + base, ctx->d_place.p, (size_t)total * sizeof(int),
	                   cudaMemcpyDeviceToHost, st));
	CK(cudaMemcpyAsync(ctx->h_prob.data() + base, ctx->d_prob.p, (size_t)total * sizeof(double),
	                   cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	return DFG_OK;
}

// G_d(phi) for the frames with mask 0 (gradient_d, max_scale.c:21-127); the
// other entries of G keep their values, as in the reference.
static int grad_d(dfg_ctx *ctx, const Chunk &ch, const std::vector<uint8_t> &mask, const std::vector<double> &phi,
                  std::vector<double> &G) {
	cudaStream_t st = ctx->stream;
	const int N = ctx->N, Nc = ch.nc, RT = ctx->RT;
	std::vector<uint8_t> active(N);
	for (int d = 0; d < N; ++d)
		active[d] = mask[d] == 0;
	CK(cudaMemcpyAsync(ctx->gd_active.p, active.data(), (size_t)N, cudaMemcpyHostToDevice, st));
	CK(cudaMemcpyAsync(ctx->gd_s.p, phi.data(), (size_t)N * sizeof(double), cudaMemcpyHostToDevice, st));
	grad_d_kernel<<<blocks_for((long long)RT * Nc, 8), 256, 0, st>>>(
	    ctx->Wd.p, ctx->Pd.p, Nc, ch.d0, RT, ctx->P, ctx->ph.p, ctx->ph_off.p, ctx->ph_mid.p, ctx->scalars.p,
	    ctx->gd_s.p, ctx->bgscale.p, ctx->background.p, ctx->gd_active.p, ctx->gd_part.p);
	CKL("grad_d_kernel");
	grad_d_reduce_kernel<<<blocks_for(Nc, 256), 256, 0, st>>>(ctx->gd_part.p, RT, Nc, ch.d0, ctx->psum_d.p,
	                                                          ctx->gd_active.p, ctx->gd_G.p);
	CKL("grad_d_reduce_kernel");
	std::vector<double> g(N);
	CK(cudaMemcpyAsync(g.data(), ctx->gd_G.p, (size_t)N * sizeof(double), cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	for (int d = 0; d < N; ++d)
		if (active[d])
			G[d] = g[d];
	return DFG_OK;
}

// Background-aware scale update (update_scale_bg, max_scale.c:129-288): per
// frame, bracket phi (start 4 phi or 32, x4 up to 5 times) and refine by
// Ridder's method (50 rounds; converged when the bracket is < 1e-5 wide or
// |G| < 1e-3); blacklisted frames get phi = -1, frames with G(0) < 1e-6 get
// 0.001. The per-frame rules run here; the sums run on the device.
static int update_scale_bg(dfg_ctx *ctx, const Chunk &ch, const dfg_iter_params *par) {
	const int N = ctx->N;
	cudaStream_t st = ctx->stream;
	std::vector<double> scale(N), so(N, 0.), sn(N, 0.), sm(N, 0.), sl(N, 0.), Go(N, 0.), Gn(N, 0.), Gm(N, 0.),
	    Gl(N, 0.);
	std::vector<uint8_t> bl(N), mask(N, 0);
	CK(cudaMemcpyAsync(scale.data(), ctx->scale.p, (size_t)N * sizeof(double), cudaMemcpyDeviceToHost, st));
	CK(cudaMemcpyAsync(bl.data(), ctx->blacklist.p, (size_t)N, cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	for (int d = 0; d < N; ++d) {
		if (bl[d]) {
			mask[d] = 255;
			scale[d] = -1.;
			continue;
		}
		sn[d] = (par->iteration > 1 || par->known_scale) ? 4. * scale[d] : 32.;
	}
	if (int rc = grad_d(ctx, ch, mask, so, Go))
		return rc;
	for (int d = 0; d < N; ++d)
		if (mask[d] != 255 && Go[d] < 1.e-6) {
			scale[d] = 0.001;
			mask[d] = 255;
		}
	for (int i = 0; i < 5; ++i) {
		if (int rc = grad_d(ctx, ch, mask, sn, Gn))
			return rc;
		int nm = 0;
		for (int d = 0; d < N; ++d) {
			if (mask[d] != 0)
				nm++;
			else if (Gn[d] < 0.) {
				mask[d] = 192;
				nm++;
			} else
				sn[d] *= 4.;
		}
		if (nm > 0.99 * N)
			break;
	}
	for (int i = 0; i < 50; ++i) {
		int nm = 0;
		for (int d = 0; d < N; ++d) {
			if (mask[d] == 255) {
				nm++;
			} else if (std::fabs(so[d] - sn[d]) < 1.e-5) {
				mask[d] = 255;
				scale[d] = 0.5 * (so[d] + sn[d]);
				nm++;
			} else {
				mask[d] = 0;
				sm[d] = 0.5 * (so[d] + sn[d]);
			}
		}
		if (nm == N)
			break;
		if (int rc = grad_d(ctx, ch, mask, sm, Gm))
			return rc;
		for (int d = 0; d < N; ++d) {
			if (mask[d] == 255)
				continue;
			if (std::fabs(Gm[d]) < BG_SCALE_TOL) {
				scale[d] = sm[d];
				mask[d] = 255;
				nm++;
				continue;
			}
			const double s = std::sqrt(Gm[d] * Gm[d] - Go[d] * Gn[d]);
			if (s < 1.e-15) {
				sl[d] = sm[d];
			} else {
				sl[d] = sm[d] + (sm[d] - so[d]) * std::copysign(1.0, Go[d]) * Gm[d] / s;
				const double lo = std::fmin(so[d], sn[d]), hi = std::fmax(so[d], sn[d]);
				if (sl[d] <= lo || sl[d] >= hi)
					sl[d] = sm[d];
			}
		}
		if (nm == N)
			break;
		if (int rc = grad_d(ctx, ch, mask, sl, Gl))
			return rc;
		for (int d = 0; d < N; ++d) {
			if (mask[d] >= 255)
				continue;
			if (std::fabs(Gl[d]) < BG_SCALE_TOL) {
				scale[d] = sl[d];
				mask[d] = 255;
				nm++;
			} else if (Gm[d] * Gl[d] < 0.) {
				so[d] = sm[d];
				Go[d] = Gm[d];
				sn[d] = sl[d];
				Gn[d] = Gl[d];
			} else if (Go[d] * Gl[d] < 0.) {
				sn[d] = sl[d];
				Gn[d] = Gl[d];
			} else {
				so[d] = sl[d];
				Go[d] = Gl[d];
			}
		}
		if (nm == N)
			break;
	}
	CK(cudaMemcpyAsync(ctx->scale.p, scale.data(), (size_t)N * sizeof(double), cudaMemcpyHostToDevice, st));
	CK(cudaStreamSynchronize(st));
	return DFG_OK;
}

// ---------------------------------------------------------------------------
// dense form of the E-step photon term (emc_dense.cuh)
// ---------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
	static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
	if (fn == nullptr) {
		void *p = nullptr;
		cudaDriverEntryPointQueryResult q;
		if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
		        cudaSuccess &&
		    q == cudaDriverEntryPointSuccess)
			fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
	}
	return fn;
}

// Tensor map of a row-major BF16 matrix [rows][K_pad] read in boxes of
// 64 columns x box_rows rows with the 128-byte swizzle.
static int encode_bf16_map(dfg_ctx *ctx, CUtensorMap *map, const void *base, long long rows, int box_rows) {
	auto fn = tensor_map_encoder();
	NEED(fn != nullptr, DFG_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
	cuuint64_t dims[2] = {(cuuint64_t)ctx->K_pad, (cuuint64_t)rows};
	cuuint64_t strides[1] = {(cuuint64_t)ctx->K_pad * 2};
	cuuint32_t box[2] = {(cuuint32_t)DK, (cuuint32_t)box_rows};
	cuuint32_t estr[2] = {1, 1};
	const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box,
	                      estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
	                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
	NEED(r == CUDA_SUCCESS, DFG_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
	return DFG_OK;
}

// Tensor map of the BF16 probability rows [rows][128] read in boxes of 64
// orientations x 64 frames with the 128-byte swizzle.
static int encode_rows_map(dfg_ctx *ctx, CUtensorMap *map, const void *base, long long rows) {
	auto fn = tensor_map_encoder();
	NEED(fn != nullptr, DFG_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
	cuuint64_t dims[2] = {128, (cuuint64_t)rows};
	cuuint64_t strides[1] = {256};
	cuuint32_t box[2] = {64, (cuuint32_t)DK};
	cuuint32_t estr[2] = {1, 1};
	const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box,
	                      estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
	                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
	NEED(r == CUDA_SUCCESS, DFG_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
	return DFG_OK;
}

// Whether this iteration may take the dense form, and why not (message).
static const char *dense_refusal(dfg_ctx *ctx, const dfg_iter_params *par) {
	if (TILE != 128)
		return "the dense form needs 128-orientation tiles (lane width 4)";
	if (ctx->with_bg && par->need_scaling)
		return "the dense form does not take the background-aware E-step";
	if (ctx->refine)
		return "the dense form does not take refinement";
	if (ctx->max_count0 < 0) {
		int m = 1;
		for (size_t i = 0; i < ctx->h_place_multi.size(); ++i)
			if (ctx->h_mask[ctx->h_place_multi[i]] < 2)
				m = std::max(m, ctx->h_count_multi[i]);
		ctx->max_count0 = m;
	}
	if (ctx->max_count0 > 256)
		return "the dense form needs photon counts of at most 256 (exact in BF16)";
	return nullptr;
}

// Pixel columns and the hi / lo log-slice buffers, before the chunk layout
// is sized (it counts the remaining memory).
static int dense_prepare_slices(dfg_ctx *ctx) {
	if (ctx->dense_P != ctx->P) {
		std::vector<int> kp, pc((size_t)ctx->P, -1);
		for (int p = 0; p < ctx->P; ++p)
			if (ctx->h_mask[p] < 2) {
				pc[p] = (int)kp.size();
				kp.push_back(p);
			}
		ctx->K = (int)kp.size();
		ctx->K_pad = std::max(DK, (ctx->K + DK - 1) / DK * DK);
		CK(upload(ctx->kpix, kp.data(), kp.size(), ctx->stream));
		CK(upload(ctx->pcol, pc.data(), pc.size(), ctx->stream));
		CK(cudaStreamSynchronize(ctx->stream));
		ctx->dense_P = ctx->P;
		std::fill(ctx->map_src, ctx->map_src + 6, nullptr);
	}
	if (!ctx->dense_active) {  // the M-step alone needs only the pixel columns
		ctx->Ahi.release();
		ctx->Alo.release();
		return DFG_OK;
	}
	const long long R_pad = (long long)(ctx->M * ctx->num_rot + TILE - 1) / TILE * TILE;
	const size_t n = (size_t)R_pad * ctx->K_pad;
	CK(ctx->Ahi.ensure(n));
	CK(ctx->Alo.ensure(n));
	if (ctx->map_src[0] != ctx->Ahi.p || ctx->map_src[1] != ctx->Alo.p) {
		if (int rc = encode_bf16_map(ctx, &ctx->map_hi, ctx->Ahi.p, R_pad, 128))
			return rc;
		if (int rc = encode_bf16_map(ctx, &ctx->map_lo, ctx->Alo.p, R_pad, 128))
			return rc;
		ctx->map_src[0] = ctx->Ahi.p;
		ctx->map_src[1] = ctx->Alo.p;
	}
	return DFG_OK;
}

// One chunk's count rows and, for the dense M-step, probability rows (after
// the chunk layout is known). The E-step reads the count tiles as 256 frame
// rows x 64 pixels; the M-step as 64 frames x 64 pixels.
static int dense_prepare_counts(dfg_ctx *ctx) {
	const int rows = (ctx->chunk_frames + DN - 1) / DN * DN;
	CK(ctx->cnt.ensure((size_t)rows * ctx->K_pad));
	if (ctx->map_src[2] != ctx->cnt.p || ctx->cnt_rows != rows) {
		if (int rc = encode_bf16_map(ctx, &ctx->map_cnt, ctx->cnt.p, rows, DN))
			return rc;
		if (int rc = encode_bf16_map(ctx, &ctx->map_cnt_m, ctx->cnt.p, rows, DK))
			return rc;
		ctx->map_src[2] = ctx->map_src[5] = ctx->cnt.p;
		ctx->cnt_rows = rows;
		ctx->map_src[3] = ctx->map_src[4] = nullptr;
	}
	if (ctx->m_dense_active) {
		const size_t n = (size_t)ctx->RT * rows * 128;
		CK(ctx->Phi.ensure(n));
		CK(ctx->Plo.ensure(n));
		if (ctx->map_src[3] != ctx->Phi.p || ctx->map_src[4] != ctx->Plo.p) {
			if (int rc = encode_rows_map(ctx, &ctx->map_phi, ctx->Phi.p, (long long)ctx->RT * rows))
				return rc;
			if (int rc = encode_rows_map(ctx, &ctx->map_plo, ctx->Plo.p, (long long)ctx->RT * rows))
				return rc;
			ctx->map_src[3] = ctx->Phi.p;
			ctx->map_src[4] = ctx->Plo.p;
		}
		CK(cudaFuncSetAttribute(mstep_dense_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, DSMEM_BYTES));
	} else {
		ctx->Phi.release();
		ctx->Plo.release();
	}
	CK(ctx->derr.ensure(1));
	CK(cudaMemsetAsync(ctx->derr.p, 0, sizeof(int), ctx->stream));
	CK(cudaFuncSetAttribute(estep_dense_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, DSMEM_BYTES));
	return DFG_OK;
}

// The dense buffers are freed when the sparse forms are in use.
static void dense_release(dfg_ctx *ctx) {
	ctx->Ahi.release();
	ctx->Alo.release();
	ctx->cnt.release();
	ctx->Phi.release();
	ctx->Plo.release();
	std::fill(ctx->map_src, ctx->map_src + 6, nullptr);
}

static int run_autotune(dfg_ctx *ctx, const dfg_iter_params *par);
static bool pair_mode(const dfg_ctx *ctx);
static int ensure_pair_buffers(dfg_ctx *ctx, const dfg_iter_params *par);
static bool blocked_wanted(dfg_ctx *ctx);
static int blocked_prepare(dfg_ctx *ctx, const dfg_iter_params *par);

// The coarse cell of every orientation on the device ([R_pad], -1 past R).
static int prepare_qmap(dfg_ctx *ctx) {
	NEED(ctx->M == 1, DFG_ERR_ARG, "refinement needs num_modes == 1");
	if (!ctx->qmap_valid || ctx->qmap.n < (size_t)ctx->R_pad) {
		std::vector<int> q((size_t)ctx->R_pad, -1);
		std::copy(ctx->h_qmap.begin(), ctx->h_qmap.end(), q.begin());
		CK(upload(ctx->qmap, q.data(), q.size(), ctx->stream));
		CK(cudaStreamSynchronize(ctx->stream));
		ctx->qmap_valid = true;
	}
	return DFG_OK;
}

// Merge weight cache: grid, psum_r > 0 pattern and flags (on the device).
static int prepare_weight_cache(dfg_ctx *ctx) {
	cudaStream_t st = ctx->stream;
	CK(ctx->weight_cache.ensure((size_t)ctx->M * ctx->V));
	CK(ctx->wpattern.ensure((size_t)ctx->R_pad));
	CK(ctx->wflags.ensure(2));
	if (!ctx->weight_cache_valid) {
		CK(cudaMemsetAsync(ctx->wflags.p, 0, 2 * sizeof(int), st));
		CK(cudaMemsetAsync(ctx->wpattern.p, 0, (size_t)ctx->R_pad, st));
		ctx->weight_cache_valid = true;  // from here on the device tracks it
	}
	return DFG_OK;
}

// max_prepare of the pair layout (no autotuner, no dense forms); watched
// frames by their global index.
static int pair_prepare(dfg_ctx *ctx, const dfg_iter_params *par) {
	ctx->dense_active = ctx->m_dense_active = false;
	ctx->blocked = false;
	if (ctx->blkT.p != nullptr) {  // block buffers sized for the blocked full search
		ctx->blkT.release();
		ctx->blk.release();
		ctx->blk_tiles = 0;
	}
	if (int rc = ensure_pair_buffers(ctx, par))
		return rc;
	if (!ctx->h_watch.empty()) {
		CK(upload(ctx->watch_local, ctx->h_watch.data(), ctx->h_watch.size(), ctx->stream));
		CK(cudaStreamSynchronize(ctx->stream));
	}
	if (int rc = prepare_qmap(ctx))
		return rc;
	return prepare_weight_cache(ctx);
}

// The part of maximize that allocates, uploads or checks on the host, done
// before any of its kernels is queued (so that the queued part can be
// captured into a CUDA graph).
static int max_prepare(dfg_ctx *ctx, const dfg_iter_params *par) {
	if (!ctx || !par)
		return DFG_ERR_ARG;
	NEED(par->beta_period > 0, DFG_ERR_ARG, "beta_period must be > 0");
	CK(cudaSetDevice(ctx->device));
	if (pair_mode(ctx))
		return pair_prepare(ctx, par);
	if (blocked_wanted(ctx))
		return blocked_prepare(ctx, par);
	ctx->blocked = false;
	// E-step form: dense tensor-core products (option estep_form 1, or the
	// autotuner's choice) where the inputs allow it
	if (ctx->autotune && !ctx->tuned && !ctx->tuning)
		if (int rc = run_autotune(ctx, par))
			return rc;
	const int form = ctx->tuning ? ctx->tune_form : (ctx->autotune ? ctx->tuned_form : ctx->estep_form);
	const int mform = ctx->tuning ? ctx->tune_mform : (ctx->autotune ? ctx->tuned_mform : ctx->mstep_form);
	ctx->dense_active = ctx->m_dense_active = false;
	if (form == 1 || mform == 1) {
		NEED(ctx->P > 0 && ctx->N > 0 && ctx->num_rot > 0, DFG_ERR_STATE, "set detector, frames and quaternions");
		const char *why = dense_refusal(ctx, par);
		NEED(why == nullptr, DFG_ERR_ARG, "%s", why);
		ctx->dense_active = form == 1;
		ctx->m_dense_active = mform == 1;
		if (int rc = dense_prepare_slices(ctx))
			return rc;
	} else if (ctx->cnt.p != nullptr || ctx->Ahi.p != nullptr) {
		dense_release(ctx);
	}
	if (int rc = ensure_buffers(ctx))
		return rc;
	if (ctx->dense_active || ctx->m_dense_active)
		if (int rc = dense_prepare_counts(ctx))
			return rc;
	cudaStream_t st = ctx->stream;
	if (ctx->refine && !ctx->h_watch.empty()) {  // chunk-local indices of the watched frames
		std::vector<int> local(ctx->h_watch.size());
		for (size_t i = 0; i < local.size(); ++i)
			local[i] = ctx->h_watch[i] % ctx->chunk_frames;
		CK(upload(ctx->watch_local, local.data(), local.size(), st));
		CK(cudaStreamSynchronize(st));
	}
	// recon.pyx:86-91 selects the 3-D or the 2-D slice functions; an RZ
	// iteration has none there
	NEED(ctx->model_type != MT_RZ, DFG_ERR_ARG, "RZ models: slice_gen / slice_merge only, no iteration");
	// background-aware path (max_prob.c:134, max_update.c:10-14, max_scale.c:8-10)
	if (ctx->with_bg && par->need_scaling) {
		NEED(ctx->chunks.size() == 1, DFG_ERR_NOMEM,
		     "background-aware updates need all %d frames in one chunk (%d chunks at the pair budget; raise "
		     "option pair_budget_mb)",
		     ctx->N, (int)ctx->chunks.size());
		if (int rc = ensure_bg(ctx))
			return rc;
	}
	// refinement: the reference indexes quat_mapping by the flat orientation
	// index over all modes (max_prob.c:114), which only covers one mode
	if (ctx->refine)
		if (int rc = prepare_qmap(ctx))
			return rc;
	return prepare_weight_cache(ctx);
}

// Whether one iteration queues its kernels without waiting on the host: the
// sparse-probability lists (keep_prob) and the background-aware scale search
// do host work between kernels.
static bool graphable(const dfg_ctx *ctx, const dfg_iter_params *par) {
	return !ctx->keep_prob && !(ctx->with_bg && par->need_scaling && par->update_scale);
}

// Orientations per slice block: the option, else whole tiles when they give
// every SM two blocks, else the largest block that does (16 at least).
static int slice_block_for(const dfg_ctx *ctx) {
	int ob = (ctx->autotune && ctx->tuned && !ctx->tuning) ? ctx->tuned_ob : ctx->slice_block;
	if (ob == 0) {
		ob = 16;
		for (int c : {TILE, 64, 32})
			if (c <= TILE && ctx->R_pad / c >= 2 * ctx->num_sms) {
				ob = c;
				break;
			}
	}
	return ob;
}

// Slices of every orientation with ob orientations per block: log W tiles (or
// W in FP64 into Wd) and u_r.
static int launch_slices(dfg_ctx *ctx, int ob, double *Wd) {
	cudaStream_t st = ctx->stream;
	const int M = ctx->M, R = ctx->R, RT = ctx->RT, P = ctx->P;
	const long long S = ctx->S, V = ctx->V;
	const int nb = ctx->R_pad / ob;
	// orientation parameters: quaternions (3-D) or (cos, sin) of the angles (2-D)
	const double *geo = ctx->model_type == MT_2D ? ctx->cs2d.p : ctx->quats.p;
#define DFG_SLICE(OBV, G)                                                                                     \
	slice_u_kernel<double, OBV, G><<<nb, 256, 0, st>>>(geo, M, R, ctx->qvals.p, ctx->corr.p, ctx->mask.p, P,     \
	                                                   ctx->model1.p, S, V, ctx->logW.p, ctx->u.p, Wd)
#define DFG_SLICE_ALL(G)                                                                                      \
	if (ob == TILE)                                                                                           \
		slice_u_tile_kernel<double, G><<<RT, 256, 0, st>>>(geo, M, R, ctx->qvals.p, ctx->corr.p, ctx->mask.p, P, \
		                                                   ctx->model1.p, S, V, ctx->logW.p, ctx->u.p, Wd);     \
	else if (ob == 64)                                                                                        \
		DFG_SLICE(TILE >= 64 ? 64 : 16, G);                                                                   \
	else if (ob == 32)                                                                                        \
		DFG_SLICE(32, G);                                                                                     \
	else                                                                                                      \
		DFG_SLICE(16, G)
	if (ctx->model_type == MT_2D) {
		DFG_SLICE_ALL(MT_2D);
	} else {
		DFG_SLICE_ALL(MT_3D);
	}
#undef DFG_SLICE_ALL
#undef DFG_SLICE
	CKL("slice_u_kernel");
	return DFG_OK;
}

// The E-step of one frame chunk: the tensor-core products (dense: counts
// densified first) or the sparse gathers (background-aware with bg).
// Tile skipping: the normalisation treats (tile, frame) pairs whose tile
// maximum can keep no pair as dead (not read, no probability written, flagged
// in tlive) and psum, the M-step and the probability split skip them. It pays
// where most tiles are dead (refinement, option tile_skip); elsewhere the
// plain kernels run and every probability row is written.
static bool tile_skipping(const dfg_ctx *ctx) { return ctx->refine || ctx->mstep_skip; }

// One chunk's photon counts as BF16 rows over the mask < 2 pixel columns
// (for the dense E-step and M-step).
static int launch_densify(dfg_ctx *ctx, const Chunk &ch) {
	cudaStream_t st = ctx->stream;
	CK(cudaMemsetAsync(ctx->cnt.p, 0, (size_t)ctx->cnt_rows * ctx->K_pad * 2, st));
	if (ch.npix > 0) {
		densify_counts_kernel<<<blocks_for((long long)ch.npix * 32, 256), 256, 0, st>>>(
		    ch.cs.p, ch.cs_off.p, ch.cs_mid.p, ch.pix.p, ch.npix, ctx->pcol.p, ch.nc, ctx->K_pad,
		    (__nv_bfloat16 *)ctx->cnt.p);
		CKL("densify_counts_kernel");
	}
	return DFG_OK;
}

// The M-step of one chunk: tomogram products on the tensor cores (the
// probabilities split into BF16 hi / lo rows first), or the sparse gathers.
static int launch_mstep(dfg_ctx *ctx, const Chunk &ch, bool dense) {
	cudaStream_t st = ctx->stream;
	const int Nc = ch.nc, P = ctx->P, RT = ctx->RT;
	if (dense) {
		const int rows = ctx->cnt_rows;
		split_prob_kernel<<<blocks_for((long long)RT * rows * 16, 256), 256, 0, st>>>(
		    ctx->Pst.p, Nc, rows, RT, tile_skipping(ctx) ? ctx->tlive.p : nullptr, (__nv_bfloat16 *)ctx->Phi.p,
		    (__nv_bfloat16 *)ctx->Plo.p);
		CKL("split_prob_kernel");
		const int n_tiles = ctx->K_pad / DN + (ctx->K_pad % DN ? 1 : 0);
		mstep_dense_kernel<<<RT * n_tiles, 192, DSMEM_BYTES, st>>>(
		    ctx->map_phi, ctx->map_plo, ctx->map_cnt_m, (Nc + DK - 1) / DK, rows, RT, n_tiles, ctx->kpix.p, ctx->K,
		    P, ctx->T.p, ctx->derr.p, ctx->dense_wait_cycles, ctx->dense_withhold);
		CKL("mstep_dense_kernel");
		return DFG_OK;
	}
	if (ch.npix > 0) {
		const long long warps = (long long)RT * ch.npix;
		const int minb = ctx->tuning ? ctx->tune_mstep_minb
		                             : (ctx->mstep_minb > 0 ? ctx->mstep_minb : ctx->tuned_mstep_minb);
#define DFG_MSTEP(SK, MB)                                                                                     \
	mstep_kernel<SK, MB><<<blocks_for(warps, 8), 256, 0, st>>>(ctx->Pst.p, Nc, ch.cs.p, ch.cs_off.p,           \
	                                                           ch.cs_mid.p, ch.pix.p, ch.npix, P, RT, ctx->T.p,  \
	                                                           ctx->tlive.p)
		if (tile_skipping(ctx))
			DFG_MSTEP(true, MSTEP_MINB);
		else if (minb == 3)
			DFG_MSTEP(false, 3);
		else if (minb == 5)
			DFG_MSTEP(false, 5);
		else
			DFG_MSTEP(false, MSTEP_MINB);
#undef DFG_MSTEP
		CKL("mstep_kernel");
	}
	return DFG_OK;
}

static int launch_estep(dfg_ctx *ctx, const Chunk &ch, int use_scale, bool bg, const RefineMask &rm, bool dense) {
	cudaStream_t st = ctx->stream;
	const int Nc = ch.nc, P = ctx->P, R = ctx->R, RT = ctx->RT;
	if (dense) {  // counts densified by launch_densify for this chunk
		const int n_tiles = (Nc + DN - 1) / DN;
		estep_dense_kernel<<<RT * n_tiles, 192, DSMEM_BYTES, st>>>(
		    ctx->map_hi, ctx->map_lo, ctx->map_cnt, ctx->K_pad / DK, RT, n_tiles, ctx->u.p, ctx->logw.p, R,
		    ctx->scale.p, ch.d0, Nc, use_scale, ctx->scalars.p, ctx->pval.p, ctx->tmax.p, ctx->targ.p,
		    ctx->derr.p, ctx->dense_wait_cycles, ctx->dense_withhold);
		CKL("estep_dense_kernel");
		return DFG_OK;
	}
	const long long warps = (long long)RT * Nc;
	if (bg) {
		estep_bg_kernel<<<blocks_for(warps, 8), 256, 0, st>>>(
		    ctx->Wd.p, ctx->u.p, ctx->logw.p, R, ctx->ph.p, ctx->ph_off.p, ctx->ph_mid.p, ctx->scale.p,
		    ctx->bgscale.p, ctx->background.p, ctx->blacklist.p, ch.d0, Nc, use_scale, ctx->scalars.p, P, RT,
		    ctx->pval.p, ctx->tmax.p, ctx->targ.p, rm);
		CKL("estep_bg_kernel");
		return DFG_OK;
	}
	// blocks per SM: the autotuner's choice (or the option), else the default
	const int minb = ctx->tuning ? ctx->tune_estep_minb : (ctx->estep_minb > 0 ? ctx->estep_minb
	                                                                           : ctx->tuned_estep_minb);
#define DFG_ESTEP(REF, MB)                                                                                    \
	estep_kernel<REF, MB><<<blocks_for(warps, 8), 256, 0, st>>>(                                              \
	    ctx->logW.p, ctx->u.p, ctx->logw.p, R, ctx->ph.p, ctx->ph_off.p, ctx->ph_mid.p, ctx->scale.p,          \
	    ctx->blacklist.p, ch.d0, Nc, use_scale, ctx->scalars.p, P, RT, ctx->pval.p, ctx->tmax.p, ctx->targ.p, rm)
	if (rm.qmap != nullptr)
		DFG_ESTEP(true, ESTEP_MINB);
	else if (minb == 2)
		DFG_ESTEP(false, 2);
	else if (minb == 4)
		DFG_ESTEP(false, 4);
	else
		DFG_ESTEP(false, ESTEP_MINB);
#undef DFG_ESTEP
	CKL("estep_kernel");
	return DFG_OK;
}

// Normalisation of one chunk (normalize_prob + the per-frame sums of
// calc_psum_r); with bg the probabilities are also kept in FP64.
static int launch_norm(dfg_ctx *ctx, const Chunk &ch, int psum_d_on, bool bg) {
	cudaStream_t st = ctx->stream;
	const int Nc = ch.nc, RT = ctx->RT, R = ctx->R, M = ctx->M;
	const int zero_dead = (ctx->keep_prob || bg) ? 1 : 0;
#define DFG_NORM(MUL, SK, ONE)                                                                                \
	norm_kernel<MUL, SK, ONE><<<blocks_for(Nc + 1, 8), 256, 0, st>>>(                                          \
	    ctx->pval.p, ctx->tmax.p, ctx->targ.p, RT, Nc, ch.d0, R, M, ctx->logw.p, ctx->u.p, ctx->beta.p,        \
	    ctx->sum_fact.p, ctx->blacklist.p, psum_d_on, ctx->scalars.p, ctx->Pst.p, ctx->rmax.p, ctx->max_exp.p, \
	    ctx->p_norm.p, ctx->info.p, ctx->likelihood.p, ctx->psum_d.p, ctx->quat_norm.p, ctx->num_prob.p,       \
	    bg ? ctx->Pd.p : nullptr, ctx->tlive.p, zero_dead)
	if (tile_skipping(ctx)) {
		if (M > 1)
			DFG_NORM(true, true, false);
		else
			DFG_NORM(false, true, false);
	} else if (bg) {  // the FP64 copy of P: two exp per pair
		if (M > 1)
			DFG_NORM(true, false, false);
		else
			DFG_NORM(false, false, false);
	} else {
		if (M > 1)
			DFG_NORM(true, false, true);
		else
			DFG_NORM(false, false, true);
	}
#undef DFG_NORM
	CKL("norm_kernel");
	return DFG_OK;
}

// Captured probability mass of the watched frames that lie in this chunk
// (their chunk-local indices were uploaded by max_prepare).
static int launch_watch(dfg_ctx *ctx, const Chunk &ch) {
	const auto &W = ctx->h_watch;
	const int lo = (int)(std::lower_bound(W.begin(), W.end(), ch.d0) - W.begin());
	const int hi = (int)(std::lower_bound(W.begin(), W.end(), ch.d0 + ch.nc) - W.begin());
	if (hi <= lo)
		return DFG_OK;
	captured_mass_kernel<<<blocks_for((long long)(hi - lo) * 32, 256), 256, 0, ctx->stream>>>(
	    ctx->Pst.p, ctx->RT, ch.nc, tile_skipping(ctx) ? ctx->tlive.p : nullptr, ctx->qmap.p,
	    ctx->watch_local.p + lo, hi - lo, ctx->watch_bits.p + (size_t)lo * ctx->rwords, ctx->rwords,
	    ctx->watch_mass.p + lo);
	CKL("captured_mass_kernel");
	return DFG_OK;
}

// ---------------------------------------------------------------------------
// pair lists (restricted searches; kernels in emc_pairs.cuh)
// ---------------------------------------------------------------------------
static bool pair_mode(const dfg_ctx *ctx) { return ctx->refine && ctx->pair_lists; }

// The live (tile, frame) pairs of the refinement: a frame's tiles are those
// holding an orientation of one of its relevant coarse cells; pair ids are
// tile-major, frames ascending within a tile. Built on the host threads over
// contiguous frame ranges: each range's tile lists and per-tile counts, then
// per-range cursors into each tile's pair range (ranges in frame order, so
// frames stay ascending within a tile).
static int build_pairs(dfg_ctx *ctx) {
	const int N = ctx->N, R = ctx->num_rot, RT = (R + TILE - 1) / TILE, nc = ctx->num_coarse;
	cudaStream_t st = ctx->stream;
	// tiles of each coarse cell, ascending
	std::vector<long long> coff((size_t)nc + 1, 0);
	std::vector<int> last((size_t)nc, -1);
	for (int r = 0; r < R; ++r) {
		const int c = ctx->h_qmap[r], t = r / TILE;
		if (last[c] != t) {
			last[c] = t;
			coff[c + 1]++;
		}
	}
	for (int c = 0; c < nc; ++c)
		coff[c + 1] += coff[c];
	std::vector<int> ctiles((size_t)coff[nc]);
	{
		std::vector<long long> cur(coff.begin(), coff.end() - 1);
		std::fill(last.begin(), last.end(), -1);
		for (int r = 0; r < R; ++r) {
			const int c = ctx->h_qmap[r], t = r / TILE;
			if (last[c] != t) {
				last[c] = t;
				ctiles[cur[c]++] = t;
			}
		}
	}
	const int TH = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
	const int nth = (int)std::min<long long>(TH, std::max(1, N / 4096));
	// pass 1: each frame's tiles (ascending) and per-range tile counts
	std::vector<std::vector<int>> ftile_th((size_t)nth);
	std::vector<std::vector<long long>> tcount_th((size_t)nth, std::vector<long long>((size_t)RT, 0));
	std::vector<long long> fcount((size_t)N);
	parallel_ranges(N, nth, [&](int k, long long b, long long e) {
		std::vector<int> stamp((size_t)RT, -1), tmp;
		auto &out = ftile_th[k];
		auto &tc = tcount_th[k];
		const bool any_all = !ctx->h_rel_all.empty();
		for (long long d = b; d < e; ++d) {
			tmp.clear();
			if (any_all && ctx->h_rel_all[d]) {  // every tile
				for (int t = 0; t < RT; ++t)
					tmp.push_back(t);
				out.insert(out.end(), tmp.begin(), tmp.end());
				fcount[d] = RT;
				for (int t = 0; t < RT; ++t)
					tc[t]++;
				continue;
			}
			for (long long j = ctx->h_rel_off[d]; j < ctx->h_rel_off[d + 1]; ++j) {
				const int c = ctx->h_rel[j];
				if (c < 0)  // an unused slot of a top-K array
					continue;
				for (long long q = coff[c]; q < coff[c + 1]; ++q)
					if (stamp[ctiles[q]] != (int)d) {
						stamp[ctiles[q]] = (int)d;
						tmp.push_back(ctiles[q]);
					}
			}
			std::sort(tmp.begin(), tmp.end());
			out.insert(out.end(), tmp.begin(), tmp.end());
			fcount[d] = (long long)tmp.size();
			for (int t : tmp)
				tc[t]++;
		}
	});
	std::vector<long long> foff((size_t)N + 1, 0);
	for (int d = 0; d < N; ++d)
		foff[d + 1] = foff[d] + fcount[d];
	const long long np = foff[N];
	NEED(np < (long long)INT32_MAX, DFG_ERR_ARG, "pair lists: %lld pairs exceed the int32 pair index", np);
	std::vector<long long> toff((size_t)RT + 1, 0);
	for (int t = 0; t < RT; ++t) {
		long long s = 0;
		for (int k = 0; k < nth; ++k)
			s += tcount_th[k][t];
		toff[t + 1] = toff[t] + s;
	}
	// pass 2: per-range cursors, then the pair arrays, written straight into
	// page-locked staging
	CK(ctx->stage_pairs.ensure((size_t)3 * std::max<long long>(np, 1)));
	int *ptile = ctx->stage_pairs.p, *pframe = ptile + np, *fpair = pframe + np;
	parallel_ranges(N, nth, [&](int k, long long b, long long e) {
		std::vector<long long> cur((size_t)RT);
		for (int t = 0; t < RT; ++t) {
			long long s = toff[t];
			for (int j = 0; j < k; ++j)
				s += tcount_th[j][t];
			cur[t] = s;
		}
		const auto &ft = ftile_th[k];
		long long i = 0;
		for (long long d = b; d < e; ++d)
			for (long long j = foff[d]; j < foff[d + 1]; ++j, ++i) {
				const int t = ft[i];
				const long long q = cur[t]++;
				ptile[q] = t;
				pframe[q] = (int)d;
				fpair[j] = (int)q;
			}
	});
	CK(upload(ctx->frame_off, foff.data(), foff.size(), st));
	CK(upload(ctx->tile_off, toff.data(), toff.size(), st));
	CK(upload(ctx->pair_tile, ptile, (size_t)np, st));
	CK(upload(ctx->pair_frame, pframe, (size_t)np, st));
	CK(upload(ctx->frame_pair, fpair, (size_t)np, st));
	CK(cudaStreamSynchronize(st));
	ctx->npairs = np;
	ctx->h_tile_off = std::move(toff);
	ctx->pairs_valid = true;
	return DFG_OK;
}

// Per frame, its photons on mask < 2 pixels as pixel | count << IDX_BITS
// words (the frame-major tomogram scatter).
static int build_mstep_words(dfg_ctx *ctx) {
	const int N = ctx->N;
	const uint8_t *mk = ctx->h_mask.data();
	std::vector<uint32_t> words;
	std::vector<long long> off((size_t)N + 1, 0);
	for (int d = 0; d < N; ++d) {
		for (long long i = ctx->h_ones_off[d]; i < ctx->h_ones_off[d + 1]; ++i)
			if (mk[ctx->h_place_ones[i]] < 2)
				push_word(words, (uint32_t)ctx->h_place_ones[i], 1);
		for (long long i = ctx->h_multi_off[d]; i < ctx->h_multi_off[d + 1]; ++i)
			if (mk[ctx->h_place_multi[i]] < 2)
				push_word(words, (uint32_t)ctx->h_place_multi[i], ctx->h_count_multi[i]);
		off[d + 1] = (long long)words.size();
	}
	CK(upload(ctx->mw, words.data(), words.size(), ctx->stream));
	CK(upload(ctx->mw_off, off.data(), off.size(), ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	ctx->mw_valid = true;
	return DFG_OK;
}

// Buffers of the pair layout. The dense layout's log-slices, tomograms and
// per-pair arrays are released (the next full search allocates them again).
static int ensure_pair_buffers(dfg_ctx *ctx, const dfg_iter_params *par) {
	NEED(ctx->P > 0 && ctx->N > 0 && ctx->num_rot > 0 && ctx->S > 0, DFG_ERR_STATE,
	     "pair lists: set detector, frames, quaternions and model first");
	NEED(ctx->beta_set, DFG_ERR_STATE, "beta not set (dfg_calc_beta or dfg_set_beta_start)");
	NEED(ctx->M == 1, DFG_ERR_ARG, "refinement needs num_modes == 1");
	NEED(ctx->model_type == MT_3D, DFG_ERR_ARG, "pair lists: 3-D models only");
	NEED(!ctx->keep_prob, DFG_ERR_ARG, "pair lists: keep_prob (sparse probability lists) is not supported");
	NEED(!(ctx->with_bg && par->need_scaling), DFG_ERR_ARG, "pair lists: no background-aware updates");
	ctx->R = ctx->num_rot;
	ctx->RT = (ctx->R + TILE - 1) / TILE;
	ctx->R_pad = ctx->RT * TILE;
	if (!ctx->pairs_valid)
		if (int rc = build_pairs(ctx))
			return rc;
	if (!ctx->mw_valid)
		if (int rc = build_mstep_words(ctx))
			return rc;
	ctx->logW.release();
	ctx->T.release();
	ctx->pval.release();
	ctx->Pst.release();
	ctx->tmax.release();
	ctx->targ.release();
	ctx->tlive.release();
	ctx->chunks_R = -1;
	dense_release(ctx);
	const size_t N = (size_t)ctx->N, P = (size_t)ctx->P;
	CK(ctx->u.ensure((size_t)ctx->R_pad));
	CK(ctx->logw.ensure((size_t)ctx->R_pad));
	CK(ctx->psum_r.ensure((size_t)ctx->R_pad));
	CK(ctx->wsign.ensure((size_t)ctx->R_pad));
	CK(ctx->scalars.ensure(8));
	CK(ctx->red_part.ensure(std::max<size_t>(blocks_for((long long)ctx->M * ctx->V, 256), 1024)));
	CK(ctx->rmax.ensure(N));
	CK(ctx->num_prob.ensure(N));
	CK(ctx->info.ensure(N));
	CK(ctx->likelihood.ensure(N));
	CK(ctx->max_exp.ensure(N));
	CK(ctx->p_norm.ensure(N));
	CK(ctx->psum_d.ensure(N));
	CK(ctx->quat_norm.ensure(N * ctx->M));
	// the per-pair buffer (FP64 sums, the probabilities written over them)
	// with 10 % headroom (the live pairs change with every new restriction);
	// the block buffer, sized from the memory left, gives way when it grows
	const size_t need = (size_t)std::max<long long>(ctx->npairs, 1) * TILE;
	if (ctx->raw.n < need) {
		ctx->blk.release();
		ctx->blk_tiles = 0;
		ctx->raw.release();
		CK(ctx->raw.ensure(need + need / 10));
	}
	// one orientation block: (P + 1) x 128 floats per tile (log-slices with
	// their zero row; the tomograms use P rows of the same space)
	const size_t tile_bytes = (P + 1) * TILE * sizeof(float);
	if (ctx->blk_tiles <= 0 || ctx->blk.n < (size_t)ctx->blk_tiles * (P + 1) * TILE) {
		size_t budget;
		if (ctx->block_budget_mb > 0.) {
			budget = (size_t)(ctx->block_budget_mb * 1048576.);
		} else {
			ctx->blk.release();
			size_t fr = 0, tot = 0;
			CK(cudaMemGetInfo(&fr, &tot));
			budget = (size_t)(0.8 * (double)fr);
		}
		ctx->blk_tiles = (int)std::max<size_t>(1, std::min<size_t>((size_t)ctx->RT, budget / tile_bytes));
		CK(ctx->blk.ensure((size_t)ctx->blk_tiles * (P + 1) * TILE));
	}
	return DFG_OK;
}

// Log-slices of the tiles [t0, t0 + nt) into the block buffer (one mode, 3-D)
// and their u_r; the zero row (pixel P) of every tile is cleared first (a
// tomogram may have been written over it).
static int launch_slices_block(dfg_ctx *ctx, int ob, int t0, int nt) {
	cudaStream_t st = ctx->stream;
	const int P = ctx->P, r0 = t0 * TILE, Rb = std::min(ctx->R - r0, nt * TILE);
	const long long S = ctx->S, V = ctx->V;
	CK(cudaMemset2DAsync(ctx->blk.p + (size_t)P * TILE, (size_t)(P + 1) * TILE * sizeof(float), 0,
	                     TILE * sizeof(float), nt, st));
	const int nb = nt * TILE / ob;
	const double *q = ctx->quats.p + 5 * (size_t)r0;
	if (ob == TILE)
		slice_u_tile_kernel<double, MT_3D><<<nt, 256, 0, st>>>(q, 1, Rb, ctx->qvals.p, ctx->corr.p, ctx->mask.p, P,
		                                                       ctx->model1.p, S, V, ctx->blk.p, ctx->u.p + r0, nullptr);
	else if (ob == 64)
		slice_u_kernel<double, TILE >= 64 ? 64 : 16, MT_3D><<<nb, 256, 0, st>>>(
		    q, 1, Rb, ctx->qvals.p, ctx->corr.p, ctx->mask.p, P, ctx->model1.p, S, V, ctx->blk.p, ctx->u.p + r0,
		    nullptr);
	else if (ob == 32)
		slice_u_kernel<double, 32, MT_3D><<<nb, 256, 0, st>>>(q, 1, Rb, ctx->qvals.p, ctx->corr.p, ctx->mask.p, P,
		                                                      ctx->model1.p, S, V, ctx->blk.p, ctx->u.p + r0,
		                                                      nullptr);
	else
		slice_u_kernel<double, 16, MT_3D><<<nb, 256, 0, st>>>(q, 1, Rb, ctx->qvals.p, ctx->corr.p, ctx->mask.p, P,
		                                                      ctx->model1.p, S, V, ctx->blk.p, ctx->u.p + r0,
		                                                      nullptr);
	CKL("slice_u_kernel");
	return DFG_OK;
}

// maximize over pair lists: per orientation block its slices and the E-step
// of its pairs; u_r and the rescale factor once every block is sliced; the
// normalisation, watched frames and psum_r over all pairs; per block the
// tomogram scatter and its merge.
static int max_enqueue_pairs(dfg_ctx *ctx, const dfg_iter_params *par) {
	cudaStream_t st = ctx->stream;
	const int N = ctx->N, P = ctx->P, M = ctx->M, R = ctx->R, RT = ctx->RT;
	const long long S = ctx->S, V = ctx->V;
	const int nblk = (P + PB - 1) / PB, BT = ctx->blk_tiles;
	const RefineMask rm{ctx->qmap.p, ctx->rel_bits.p, ctx->rwords};
	const int ob = slice_block_for(ctx);
	{
		double factor = std::pow(par->beta_jump, (double)((par->iteration - 1) / par->beta_period));
		factor *= par->beta_factor;
		beta_kernel<<<blocks_for(N, 256), 256, 0, st>>>(ctx->beta_start.p, ctx->blacklist.p, N, factor,
		                                                 ctx->beta.p);
		CKL("beta_kernel");
	}
	for (int t0 = 0; t0 < RT; t0 += BT) {
		const int nt = std::min(BT, RT - t0);
		phase_begin(ctx, PH_SLICE);
		if (int rc = launch_slices_block(ctx, ob, t0, nt))
			return rc;
		phase_end(ctx, PH_SLICE, 1);
		phase_begin(ctx, PH_ESTEP);
		const long long q0 = ctx->h_tile_off[t0], nq = ctx->h_tile_off[t0 + nt] - q0;
		if (nq > 0) {
			estep_pairs_kernel<<<blocks_for(nq, 8), 256, 0, st>>>(
			    ctx->blk.p, t0, q0, nq, ctx->pair_tile.p, ctx->pair_frame.p, ctx->ph.p, ctx->ph_off.p,
			    ctx->ph_mid.p, ctx->blacklist.p, R, P, rm, ctx->raw.p);
			CKL("estep_pairs_kernel");
		}
		phase_end(ctx, PH_ESTEP, nq > 0 ? 1 : 0);
	}
	phase_begin(ctx, PH_SLICE);
	rescale_kernel<<<1, 256, 0, st>>>(ctx->u.p, ctx->quats.p, M, R, ctx->mean_count, ctx->scalars.p);
	CKL("rescale_kernel");
	logw_kernel<<<blocks_for(R, 256), 256, 0, st>>>(ctx->quats.p, M, R, ctx->logw.p);
	CKL("logw_kernel");
	phase_end(ctx, PH_SLICE, 2);

	const int use_scale = par->need_scaling && (par->iteration > 1 || par->known_scale);
	const int psum_d_on = par->need_scaling && par->update_scale;
	phase_begin(ctx, PH_NORM);
	norm_pairs_kernel<<<blocks_for((long long)N * 32, 256), 256, 0, st>>>(
	    ctx->raw.p, ctx->frame_off.p, ctx->frame_pair.p, ctx->pair_tile.p, N, R, ctx->logw.p, ctx->u.p,
	    ctx->scale.p, use_scale, ctx->beta.p, ctx->sum_fact.p, ctx->blacklist.p, psum_d_on, ctx->scalars.p,
	    (float *)ctx->raw.p, ctx->rmax.p, ctx->max_exp.p, ctx->p_norm.p, ctx->info.p, ctx->likelihood.p, ctx->psum_d.p,
	    ctx->num_prob.p);
	CKL("norm_pairs_kernel");
	const int nw = (int)ctx->h_watch.size();
	if (nw > 0) {
		captured_mass_pairs_kernel<<<blocks_for((long long)nw * 32, 256), 256, 0, st>>>(
		    (float *)ctx->raw.p, ctx->frame_off.p, ctx->frame_pair.p, ctx->pair_tile.p, ctx->qmap.p, ctx->watch_local.p, nw,
		    ctx->watch_bits.p, ctx->rwords, ctx->watch_mass.p);
		CKL("captured_mass_pairs_kernel");
	}
	phase_end(ctx, PH_NORM, nw > 0 ? 2 : 1);
	phase_begin(ctx, PH_PSUM);
	psum_pairs_kernel<<<RT, 256, 0, st>>>((float *)ctx->raw.p, ctx->tile_off.p, ctx->pair_frame.p, ctx->scale.p,
	                                      par->need_scaling, R, ctx->psum_r.p);
	CKL("psum_pairs_kernel");
	phase_end(ctx, PH_PSUM, 1);

	weight_sign_kernel<<<1, 1024, 0, st>>>(ctx->psum_r.p, R, ctx->wpattern.p, ctx->wsign.p, ctx->wflags.p);
	CKL("weight_sign_kernel");
	CK(cudaMemsetAsync(ctx->accum.p, 0, (size_t)M * V * sizeof(double2), st));
	for (int t0 = 0; t0 < RT; t0 += BT) {
		const int nt = std::min(BT, RT - t0), r0 = t0 * TILE, Rb = std::min(R - r0, nt * TILE);
		phase_begin(ctx, PH_MSTEP);
		CK(cudaMemsetAsync(ctx->blk.p, 0, (size_t)nt * P * TILE * sizeof(float), st));
		const long long q0 = ctx->h_tile_off[t0], nq = ctx->h_tile_off[t0 + nt] - q0;
		if (nq > 0) {
			mstep_pairs_kernel<<<blocks_for(nq, 8), 256, 0, st>>>((float *)ctx->raw.p, t0, q0, nq, ctx->pair_tile.p,
			                                                       ctx->pair_frame.p, ctx->mw.p, ctx->mw_off.p, P,
			                                                       ctx->blk.p);
			CKL("mstep_pairs_kernel");
		}
		phase_end(ctx, PH_MSTEP, nq > 0 ? 1 : 0);
		phase_begin(ctx, PH_MERGE);
		merge_kernel<MT_3D, true><<<dim3(nblk, nt), 256, 0, st>>>(
		    ctx->blk.p, ctx->psum_r.p + r0, ctx->quats.p + 5 * (size_t)r0, 1, Rb, ctx->qvals.p, ctx->corr.p,
		    ctx->mask.p, P, S, V, (double *)ctx->accum.p, ctx->wflags.p, 0, ctx->wsign.p + r0);
		CKL("merge_kernel");
		phase_end(ctx, PH_MERGE, 1);
	}
	phase_begin(ctx, PH_UPDATE);
	unpack_accum_kernel<<<blocks_for((long long)M * V, 256), 256, 0, st>>>(
	    ctx->accum.p, (long long)M * V, ctx->model2.p, ctx->weight.p, ctx->weight_cache.p, ctx->wflags.p);
	CKL("unpack_accum_kernel");
	frame_totals_kernel<<<1, 1024, 0, st>>>(ctx->info.p, ctx->likelihood.p, ctx->blacklist.p, N,
	                                        ctx->scalars.p + 1);
	CKL("frame_totals_kernel");
	if (par->need_scaling && par->update_scale) {
		scale_kernel<<<blocks_for(N, 256), 256, 0, st>>>(ctx->fcounts.p, ctx->psum_d.p, ctx->blacklist.p, N,
		                                                  ctx->scale.p);
		CKL("scale_kernel");
	}
	phase_end(ctx, PH_UPDATE, par->need_scaling && par->update_scale ? 3 : 2);
	ctx->views_final = false;
	return DFG_OK;
}

// ---------------------------------------------------------------------------
// orientation-blocked full search (log-slices and tomograms too large to keep
// for every orientation)
// ---------------------------------------------------------------------------
// Whether a full search runs in orientation blocks: option block_budget_mb
// (without refinement), or the log-slices and tomograms of every orientation
// would take more than half of the device memory.
static bool blocked_wanted(dfg_ctx *ctx) {
	if (ctx->refine || ctx->P <= 0 || ctx->num_rot <= 0 || ctx->M <= 0)
		return false;
	if (ctx->block_budget_mb > 0.)
		return true;
	const size_t RT = ((size_t)ctx->M * ctx->num_rot + TILE - 1) / TILE;
	const size_t need = RT * ((size_t)2 * ctx->P + 1) * TILE * sizeof(float);
	size_t fr = 0, tot = 0;
	if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
		cudaGetLastError();
		return false;
	}
	const size_t held = (ctx->logW.n + ctx->T.n + ctx->blk.n + ctx->blkT.n) * sizeof(float);
	return need > (fr + held) / 2;
}

// Buffers of the blocked full search: one block of log-slices (blk) and one
// of tomograms (blkT), then the frame chunks from the memory left.
static int blocked_prepare(dfg_ctx *ctx, const dfg_iter_params *par) {
	NEED(ctx->P > 0 && ctx->N > 0 && ctx->num_rot > 0 && ctx->S > 0, DFG_ERR_STATE,
	     "set detector, frames, quaternions and model first");
	NEED(ctx->beta_set, DFG_ERR_STATE, "beta not set (dfg_calc_beta or dfg_set_beta_start)");
	NEED(ctx->M == 1 && ctx->model_type == MT_3D, DFG_ERR_ARG,
	     "orientation blocks (the full search's log-slices and tomograms exceed the memory, or block_budget_mb): "
	     "one mode, 3-D models only");
	NEED(!(ctx->with_bg && par->need_scaling), DFG_ERR_ARG, "orientation blocks: no background-aware updates");
	ctx->dense_active = ctx->m_dense_active = false;
	ctx->blocked = true;
	ctx->R = ctx->num_rot;
	ctx->RT = (ctx->R + TILE - 1) / TILE;
	ctx->R_pad = ctx->RT * TILE;
	ctx->logW.release();
	ctx->T.release();
	ctx->raw.release();  // per-pair buffer of the pair lists
	dense_release(ctx);
	const size_t N = (size_t)ctx->N, P = (size_t)ctx->P;
	CK(ctx->u.ensure((size_t)ctx->R_pad));
	CK(ctx->logw.ensure((size_t)ctx->R_pad));
	CK(ctx->psum_r.ensure((size_t)ctx->R_pad));
	CK(ctx->scalars.ensure(8));
	CK(ctx->red_part.ensure(std::max<size_t>(blocks_for((long long)ctx->M * ctx->V, 256), 1024)));
	CK(ctx->rmax.ensure(N));
	CK(ctx->num_prob.ensure(N));
	CK(ctx->info.ensure(N));
	CK(ctx->likelihood.ensure(N));
	CK(ctx->max_exp.ensure(N));
	CK(ctx->p_norm.ensure(N));
	CK(ctx->psum_d.ensure(N));
	CK(ctx->quat_norm.ensure(N * ctx->M));
	const size_t tile_bytes = ((size_t)2 * P + 1) * TILE * sizeof(float);
	if (ctx->blk_tiles <= 0 || ctx->blkT.n < (size_t)ctx->blk_tiles * P * TILE ||
	    ctx->blk.n < (size_t)ctx->blk_tiles * (P + 1) * TILE) {
		ctx->blk.release();
		ctx->blkT.release();
		size_t budget;
		if (ctx->block_budget_mb > 0.) {
			budget = (size_t)(ctx->block_budget_mb * 1048576.);
		} else {
			size_t fr = 0, tot = 0;
			CK(cudaMemGetInfo(&fr, &tot));
			budget = (size_t)(0.35 * (double)fr);
		}
		ctx->blk_tiles = (int)std::max<size_t>(1, std::min<size_t>((size_t)ctx->RT, budget / tile_bytes));
		CK(ctx->blk.ensure((size_t)ctx->blk_tiles * (P + 1) * TILE));
		CK(ctx->blkT.ensure((size_t)ctx->blk_tiles * P * TILE));
	}
	if (ctx->chunks_R != ctx->R || ctx->chunks_dense != 0) {
		ctx->pval.release();
		ctx->Pst.release();
		ctx->tmax.release();
		ctx->targ.release();
		if (int rc = build_chunks(ctx))
			return rc;
	}
	const size_t pairs = (size_t)ctx->R_pad * ctx->chunk_frames;
	CK(ctx->pval.ensure(pairs));
	CK(ctx->Pst.ensure((size_t)ctx->R_pad * (ctx->chunk_frames + 1)));
	CK(ctx->tmax.ensure((size_t)ctx->RT * ctx->chunk_frames));
	CK(ctx->targ.ensure((size_t)ctx->RT * ctx->chunk_frames));
	CK(ctx->tlive.ensure((size_t)ctx->RT * (ctx->chunk_frames + 1)));
	const int nsplit = std::max(1, std::min(64, ctx->chunk_frames / 2048));
	CK(ctx->psum_part.ensure((size_t)nsplit * ctx->R_pad));
	return prepare_weight_cache(ctx);
}

// E-step of the tiles [t0, t0 + nt) for one chunk from the block buffer.
static int launch_estep_block(dfg_ctx *ctx, const Chunk &ch, int t0, int nt, int use_scale) {
	const RefineMask none{nullptr, nullptr, 0};
	estep_kernel<false><<<blocks_for((long long)nt * ch.nc, 8), 256, 0, ctx->stream>>>(
	    ctx->blk.p, ctx->u.p, ctx->logw.p, ctx->R, ctx->ph.p, ctx->ph_off.p, ctx->ph_mid.p, ctx->scale.p,
	    ctx->blacklist.p, ch.d0, ch.nc, use_scale, ctx->scalars.p, ctx->P, nt, ctx->pval.p, ctx->tmax.p, ctx->targ.p,
	    none, t0);
	CKL("estep_kernel");
	return DFG_OK;
}

// maximize with the orientations in blocks of whole tiles, in two passes.
// Pass 1, per frame chunk: every block's slices and E-step into the chunk's
// log-likelihoods, then the normalisation over all orientations (exact: the
// per-frame maximum, first argmax, kept sum and frame sums as the one-chunk
// path) and psum_r. Pass 2, per block: its slices once, then per chunk its
// E-step again, its probabilities from the pass-1 per-frame results
// (prob_block_kernel) and its tomograms; the block is merged once all chunks
// are in. u_r (and the rescale factor the E-step needs) come from a slice
// pass over every block first.
static int max_enqueue_blocked(dfg_ctx *ctx, const dfg_iter_params *par) {
	cudaStream_t st = ctx->stream;
	const int N = ctx->N, P = ctx->P, M = ctx->M, R = ctx->R, RT = ctx->RT, R_pad = ctx->R_pad;
	const long long S = ctx->S, V = ctx->V;
	const int nblk = (P + PB - 1) / PB, BT = ctx->blk_tiles;
	const int ob = slice_block_for(ctx);
	{
		double factor = std::pow(par->beta_jump, (double)((par->iteration - 1) / par->beta_period));
		factor *= par->beta_factor;
		beta_kernel<<<blocks_for(N, 256), 256, 0, st>>>(ctx->beta_start.p, ctx->blacklist.p, N, factor,
		                                                 ctx->beta.p);
		CKL("beta_kernel");
	}
	phase_begin(ctx, PH_SLICE);
	for (int t0 = 0; t0 < RT; t0 += BT)
		if (int rc = launch_slices_block(ctx, ob, t0, std::min(BT, RT - t0)))
			return rc;
	rescale_kernel<<<1, 256, 0, st>>>(ctx->u.p, ctx->quats.p, M, R, ctx->mean_count, ctx->scalars.p);
	CKL("rescale_kernel");
	logw_kernel<<<blocks_for(R, 256), 256, 0, st>>>(ctx->quats.p, M, R, ctx->logw.p);
	CKL("logw_kernel");
	phase_end(ctx, PH_SLICE, (RT + BT - 1) / BT + 2);
	CK(cudaMemsetAsync(ctx->psum_r.p, 0, (size_t)R_pad * sizeof(double), st));
	CK(cudaMemsetAsync(ctx->accum.p, 0, (size_t)M * V * sizeof(double2), st));
	const int use_scale = par->need_scaling && (par->iteration > 1 || par->known_scale);
	const int psum_d_on = par->need_scaling && par->update_scale;
	if (ctx->keep_prob) {
		ctx->h_prob_off.assign((size_t)N + 1, 0);
		ctx->h_place_prob.clear();
		ctx->h_prob.clear();
	}
	ctx->have_prob = false;
	// pass 1
	for (Chunk &ch : ctx->chunks) {
		const int Nc = ch.nc;
		for (int t0 = 0; t0 < RT; t0 += BT) {
			const int nt = std::min(BT, RT - t0);
			phase_begin(ctx, PH_SLICE);
			if (int rc = launch_slices_block(ctx, ob, t0, nt))
				return rc;
			phase_end(ctx, PH_SLICE, 1);
			phase_begin(ctx, PH_ESTEP);
			if (int rc = launch_estep_block(ctx, ch, t0, nt, use_scale))
				return rc;
			phase_end(ctx, PH_ESTEP, 1);
		}
		phase_begin(ctx, PH_NORM);
		if (int rc = launch_norm(ctx, ch, psum_d_on, false))
			return rc;
		phase_end(ctx, PH_NORM, 1);
		if (ctx->keep_prob)
			if (int rc = collect_prob(ctx, ch))
				return rc;
		phase_begin(ctx, PH_PSUM);
		const int nsplit = std::max(1, std::min(64, ctx->chunk_frames / 2048));
		const int fps = (Nc + nsplit - 1) / nsplit;
		psum_r_kernel<<<dim3(RT, nsplit), 256, 0, st>>>(ctx->Pst.p, Nc, ch.d0, fps, ctx->scale.p, par->need_scaling,
		                                                ctx->psum_part.p, R_pad,
		                                                tile_skipping(ctx) ? ctx->tlive.p : nullptr);
		CKL("psum_r_kernel");
		psum_r_reduce_kernel<<<blocks_for(R, 256), 256, 0, st>>>(ctx->psum_part.p, nsplit, R, R_pad, ctx->psum_r.p);
		CKL("psum_r_reduce_kernel");
		phase_end(ctx, PH_PSUM, 2);
	}
	weight_pattern_kernel<<<1, 1024, 0, st>>>(ctx->psum_r.p, R, ctx->wpattern.p, ctx->wflags.p);
	CKL("weight_pattern_kernel");
	// pass 2
	for (int t0 = 0; t0 < RT; t0 += BT) {
		const int nt = std::min(BT, RT - t0), r0 = t0 * TILE, Rb = std::min(R - r0, nt * TILE);
		phase_begin(ctx, PH_SLICE);
		if (int rc = launch_slices_block(ctx, ob, t0, nt))
			return rc;
		phase_end(ctx, PH_SLICE, 1);
		CK(cudaMemsetAsync(ctx->blkT.p, 0, (size_t)nt * P * TILE * sizeof(float), st));
		for (Chunk &ch : ctx->chunks) {
			const int Nc = ch.nc;
			phase_begin(ctx, PH_ESTEP);
			if (int rc = launch_estep_block(ctx, ch, t0, nt, use_scale))
				return rc;
			phase_end(ctx, PH_ESTEP, 1);
			phase_begin(ctx, PH_NORM);
			prob_block_kernel<<<blocks_for((long long)nt * (Nc + 1), 8), 256, 0, st>>>(
			    ctx->pval.p, t0, nt, Nc, ch.d0, R, ctx->beta.p, ctx->max_exp.p, ctx->rmax.p, ctx->p_norm.p,
			    ctx->blacklist.p, ctx->Pst.p);
			CKL("prob_block_kernel");
			phase_end(ctx, PH_NORM, 1);
			phase_begin(ctx, PH_MSTEP);
			if (ch.npix > 0) {
				mstep_kernel<false><<<blocks_for((long long)nt * ch.npix, 8), 256, 0, st>>>(
				    ctx->Pst.p, Nc, ch.cs.p, ch.cs_off.p, ch.cs_mid.p, ch.pix.p, ch.npix, P, nt, ctx->blkT.p,
				    ctx->tlive.p, t0);
				CKL("mstep_kernel");
			}
			phase_end(ctx, PH_MSTEP, ch.npix > 0 ? 1 : 0);
		}
		phase_begin(ctx, PH_MERGE);
		merge_kernel<MT_3D><<<dim3(nblk, nt), 256, 0, st>>>(ctx->blkT.p, ctx->psum_r.p + r0,
		                                                     ctx->quats.p + 5 * (size_t)r0, 1, Rb, ctx->qvals.p,
		                                                     ctx->corr.p, ctx->mask.p, P, S, V,
		                                                     (double *)ctx->accum.p, ctx->wflags.p, 0);
		CKL("merge_kernel");
		phase_end(ctx, PH_MERGE, 1);
	}
	phase_begin(ctx, PH_UPDATE);
	unpack_accum_kernel<<<blocks_for((long long)M * V, 256), 256, 0, st>>>(
	    ctx->accum.p, (long long)M * V, ctx->model2.p, ctx->weight.p, ctx->weight_cache.p, ctx->wflags.p);
	CKL("unpack_accum_kernel");
	frame_totals_kernel<<<1, 1024, 0, st>>>(ctx->info.p, ctx->likelihood.p, ctx->blacklist.p, N,
	                                        ctx->scalars.p + 1);
	CKL("frame_totals_kernel");
	if (par->need_scaling && par->update_scale) {
		scale_kernel<<<blocks_for(N, 256), 256, 0, st>>>(ctx->fcounts.p, ctx->psum_d.p, ctx->blacklist.p, N,
		                                                  ctx->scale.p);
		CKL("scale_kernel");
	}
	phase_end(ctx, PH_UPDATE, par->need_scaling && par->update_scale ? 3 : 2);
	ctx->views_final = false;
	return DFG_OK;
}

// Queues maximize's kernels (after max_prepare). Synchronises only where
// graphable() is false.
static int max_enqueue(dfg_ctx *ctx, const dfg_iter_params *par) {
	ctx->last_pairs = pair_mode(ctx);
	if (ctx->last_pairs)
		return max_enqueue_pairs(ctx, par);
	if (ctx->blocked)
		return max_enqueue_blocked(ctx, par);
	cudaStream_t st = ctx->stream;
	const int N = ctx->N, P = ctx->P, M = ctx->M, R = ctx->R, RT = ctx->RT, R_pad = ctx->R_pad;
	const long long S = ctx->S, V = ctx->V;
	const int nblk = (P + PB - 1) / PB;
	const bool bg = ctx->with_bg && par->need_scaling;
	double *const Wd = bg ? ctx->Wd.p : nullptr;  // FP64 slices for the background path
	const bool two_d = ctx->model_type == MT_2D;
	const RefineMask rm = ctx->refine ? RefineMask{ctx->qmap.p, ctx->rel_bits.p, ctx->rwords}
	                                  : RefineMask{nullptr, nullptr, 0};

	// update_beta (recon.pyx:161-171)
	{
		double factor = std::pow(par->beta_jump, (double)((par->iteration - 1) / par->beta_period));
		factor *= par->beta_factor;
		beta_kernel<<<blocks_for(N, 256), 256, 0, st>>>(ctx->beta_start.p, ctx->blacklist.p, N, factor,
		                                                 ctx->beta.p);
		CKL("beta_kernel");
	}

	// slices, u_r, rescale (calculate_rescale, max_prob.c:3-64)
	phase_begin(ctx, PH_SLICE);
	if (int rc = launch_slices(ctx, slice_block_for(ctx), Wd))
		return rc;
	rescale_kernel<<<1, 256, 0, st>>>(ctx->u.p, ctx->quats.p, M, R, ctx->mean_count, ctx->scalars.p);
	CKL("rescale_kernel");
	logw_kernel<<<blocks_for(R, 256), 256, 0, st>>>(ctx->quats.p, M, R, ctx->logw.p);
	CKL("logw_kernel");
	if (ctx->dense_active) {
		split_logw_kernel<<<dim3(ctx->K_pad / DK, RT), 256, 0, st>>>(
		    ctx->logW.p, P, ctx->kpix.p, ctx->mask.p, ctx->K, ctx->K_pad, (__nv_bfloat16 *)ctx->Ahi.p,
		    (__nv_bfloat16 *)ctx->Alo.p);
		CKL("split_logw_kernel");
	}
	phase_end(ctx, PH_SLICE, ctx->dense_active ? 4 : 3);

	CK(cudaMemsetAsync(ctx->T.p, 0, (size_t)RT * P * TILE * sizeof(float), st));
	CK(cudaMemsetAsync(ctx->psum_r.p, 0, (size_t)R_pad * sizeof(double), st));
	CK(cudaMemsetAsync(ctx->accum.p, 0, (size_t)M * V * sizeof(double2), st));
	const int use_scale = par->need_scaling && (par->iteration > 1 || par->known_scale);
	const int psum_d_on = par->need_scaling && par->update_scale;

	if (ctx->keep_prob) {
		ctx->h_prob_off.assign((size_t)N + 1, 0);
		ctx->h_place_prob.clear();
		ctx->h_prob.clear();
	}
	ctx->have_prob = false;
	for (Chunk &ch : ctx->chunks) {
		const int Nc = ch.nc;
		// E-step (calculate_prob, max_prob.c:66-213)
		phase_begin(ctx, PH_ESTEP);
		if (ctx->dense_active || ctx->m_dense_active)
			if (int rc = launch_densify(ctx, ch))
				return rc;
		if (int rc = launch_estep(ctx, ch, use_scale, bg, rm, ctx->dense_active))
			return rc;
		phase_end(ctx, PH_ESTEP, (ctx->dense_active || ctx->m_dense_active ? 1 : 0) + 1);
		// normalisation and per-frame sums (normalize_prob + calc_psum_r)
		phase_begin(ctx, PH_NORM);
		if (int rc = launch_norm(ctx, ch, psum_d_on, bg))
			return rc;
		if (ctx->refine && !ctx->h_watch.empty())
			if (int rc = launch_watch(ctx, ch))
				return rc;
		phase_end(ctx, PH_NORM, 1);
		if (ctx->keep_prob)
			if (int rc = collect_prob(ctx, ch))
				return rc;
		// psum_r (calc_psum_r, max_update.c:108-116)
		phase_begin(ctx, PH_PSUM);
		{
			const int nsplit = std::max(1, std::min(64, ctx->chunk_frames / 2048));
			const int fps = (Nc + nsplit - 1) / nsplit;
			psum_r_kernel<<<dim3(RT, nsplit), 256, 0, st>>>(ctx->Pst.p, Nc, ch.d0, fps, ctx->scale.p,
			                                                par->need_scaling, ctx->psum_part.p, R_pad,
			                                                tile_skipping(ctx) ? ctx->tlive.p : nullptr);
			CKL("psum_r_kernel");
			psum_r_reduce_kernel<<<blocks_for(R, 256), 256, 0, st>>>(ctx->psum_part.p, nsplit, R, R_pad,
			                                                          ctx->psum_r.p);
			CKL("psum_r_reduce_kernel");
			if (bg) {
				scalemax_kernel<<<dim3(RT, nsplit), 256, 0, st>>>(ctx->Pd.p, Nc, ch.d0, fps, ctx->scale.p,
				                                                  ctx->smax_part.p, R_pad);
				CKL("scalemax_kernel");
				scalemax_reduce_kernel<<<blocks_for(R, 256), 256, 0, st>>>(ctx->smax_part.p, nsplit, R, R_pad,
				                                                            ctx->scalemax.p);
				CKL("scalemax_reduce_kernel");
			}
		}
		phase_end(ctx, PH_PSUM, bg ? 4 : 2);
		// tomograms (update_tomogram_nobg, max_update.c:142-230)
		phase_begin(ctx, PH_MSTEP);
		if (!bg) {
			if (int rc = launch_mstep(ctx, ch, ctx->m_dense_active))
				return rc;
		} else if (ch.npix > 0) {
			long long warps = (long long)RT * ch.npix;
			{
				// update_tomogram_bg (max_update.c:343-543); the mean photons per
				// pixel bound the first search window (:397-400)
				mstep_bg_kernel<<<blocks_for(warps, 8), 256, 0, st>>>(
				    ctx->Pd.p, Nc, ch.d0, ch.cs.p, ch.cs_off.p, ch.cs_mid.p, ch.pix.p, ch.npix, P, RT, R,
				    ctx->psum_r.p, ctx->scalemax.p, ctx->scale.p, ctx->bgscale.p, ctx->background.p, ctx->powder.p,
				    ctx->mean_count / P, ctx->T.p);
				CKL("mstep_bg_kernel");
			}
		}
		phase_end(ctx, PH_MSTEP, ctx->m_dense_active ? 2 : (ch.npix > 0 ? 1 : 0));
	}

	// merge (merge_tomogram -> slice_merge3d); the weight grid is rebuilt only
	// when the set of orientations with psum_r > 0 changed (decided on the device)
	weight_pattern_kernel<<<1, 1024, 0, st>>>(ctx->psum_r.p, R, ctx->wpattern.p, ctx->wflags.p);
	CKL("weight_pattern_kernel");
	phase_begin(ctx, PH_MERGE);
	if (two_d)
		merge_kernel<MT_2D><<<dim3(nblk, RT), 256, 0, st>>>(ctx->T.p, ctx->psum_r.p, ctx->cs2d.p, M, R, ctx->qvals.p,
		                                                     ctx->corr.p, ctx->mask.p, P, S, V, (double *)ctx->accum.p,
		                                                     ctx->wflags.p, bg ? 1 : 0);
	else
		merge_kernel<MT_3D><<<dim3(nblk, RT), 256, 0, st>>>(ctx->T.p, ctx->psum_r.p, ctx->quats.p, M, R, ctx->qvals.p,
		                                                     ctx->corr.p, ctx->mask.p, P, S, V, (double *)ctx->accum.p,
		                                                     ctx->wflags.p, bg ? 1 : 0);
	CKL("merge_kernel");
	phase_end(ctx, PH_MERGE, 1);

	phase_begin(ctx, PH_UPDATE);
	unpack_accum_kernel<<<blocks_for((long long)M * V, 256), 256, 0, st>>>(
	    ctx->accum.p, (long long)M * V, ctx->model2.p, ctx->weight.p, ctx->weight_cache.p, ctx->wflags.p);
	CKL("unpack_accum_kernel");
	// averages over good frames; the packaged Iterate never sets num_blacklist,
	// so they divide by N (max_prob.c:373-374, iterate.pyx:35)
	frame_totals_kernel<<<1, 1024, 0, st>>>(ctx->info.p, ctx->likelihood.p, ctx->blacklist.p, N,
	                                        ctx->scalars.p + 1);
	CKL("frame_totals_kernel");
	if (par->need_scaling && par->update_scale) {
		if (bg) {
			if (int rc = update_scale_bg(ctx, ctx->chunks[0], par))
				return rc;
		} else {
			scale_kernel<<<blocks_for(N, 256), 256, 0, st>>>(ctx->fcounts.p, ctx->psum_d.p, ctx->blacklist.p, N,
			                                                  ctx->scale.p);
			CKL("scale_kernel");
		}
	}
	phase_end(ctx, PH_UPDATE, par->need_scaling && par->update_scale ? 3 : 2);
	ctx->views_final = bg;
	return DFG_OK;
}

// Project autotuner. On the context's own inputs it times (CUDA events, best
// of two after a warm-up launch) the slice kernel with 128, 64, 32 and 16 orientations per block and
// both forms of the E-step photon term and of the M-step (sparse gathers,
// dense tensor-core products where the inputs allow them) on the first frame
// chunk, and keeps the fastest of each; then, where the sparse gathers won,
// their resident blocks per SM. tune_report: as dfg_autotune's report (the
// dense E-step time includes the count densification).
static int run_autotune(dfg_ctx *ctx, const dfg_iter_params *par) {
	NEED(ctx->P > 0 && ctx->N > 0 && ctx->num_rot > 0 && ctx->S > 0, DFG_ERR_STATE,
	     "autotune: set detector, frames, quaternions and model first");
	double rep[DFG_TUNE_REPORT];
	std::fill(rep, rep + DFG_TUNE_REPORT, -1.);
	const bool dense_ok = dense_refusal(ctx, par) == nullptr;
	const bool save_timing = ctx->timing;
	ctx->timing = false;
	ctx->tuning = true;
	ctx->tune_estep_minb = ESTEP_MINB;
	ctx->tune_mstep_minb = MSTEP_MINB;
	ctx->tune_form = ctx->tune_mform = dense_ok ? 1 : 0;
	int rc = max_prepare(ctx, par);
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	if (rc == DFG_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
		rc = ctx->fail(DFG_ERR_CUDA, "autotune: cudaEventCreate failed");
	cudaStream_t st = ctx->stream;
	// one untimed launch (module loading, shared-memory carve-out), then the
	// best of two timed ones
	auto timed = [&](auto &&launch, double &out) -> int {
		if (int r = launch())
			return r;
		float best = 1e30f;
		for (int k = 0; k < 2; ++k) {
			CK(cudaEventRecord(e0, st));
			if (int r = launch())
				return r;
			CK(cudaEventRecord(e1, st));
			CK(cudaEventSynchronize(e1));
			float ms = 0.f;
			CK(cudaEventElapsedTime(&ms, e0, e1));
			best = std::min(best, ms);
		}
		out = best;
		return DFG_OK;
	};
	const bool bg = ctx->with_bg && par->need_scaling;
	double *const Wd = bg ? ctx->Wd.p : nullptr;
	const RefineMask rm = ctx->refine ? RefineMask{ctx->qmap.p, ctx->rel_bits.p, ctx->rwords}
	                                  : RefineMask{nullptr, nullptr, 0};
	const int obs[4] = {128, 64, 32, 16};
	int bi = -1;
	for (int i = 0; i < 4 && rc == DFG_OK; ++i) {
		const int ob = obs[i];
		if (ob > TILE || TILE % ob != 0)
			continue;
		rc = timed([&] { return launch_slices(ctx, ob, Wd); }, rep[i]);
		if (rc == DFG_OK && (bi < 0 || rep[i] < rep[bi]))
			bi = i;
	}
	const int best_ob = bi >= 0 ? obs[bi] : 0;
	const int use_scale = par->need_scaling && (par->iteration > 1 || par->known_scale);
	if (rc == DFG_OK) {
		// the E-step's other inputs
		rescale_kernel<<<1, 256, 0, st>>>(ctx->u.p, ctx->quats.p, ctx->M, ctx->R, ctx->mean_count, ctx->scalars.p);
		CKL("rescale_kernel");
		logw_kernel<<<blocks_for(ctx->R, 256), 256, 0, st>>>(ctx->quats.p, ctx->M, ctx->R, ctx->logw.p);
		CKL("logw_kernel");
		rc = timed([&] { return launch_estep(ctx, ctx->chunks[0], use_scale, bg, rm, false); }, rep[4]);
	}
	const Chunk &c0 = ctx->chunks[0];
	if (rc == DFG_OK && dense_ok) {
		split_logw_kernel<<<dim3(ctx->K_pad / DK, ctx->RT), 256, 0, st>>>(
		    ctx->logW.p, ctx->P, ctx->kpix.p, ctx->mask.p, ctx->K, ctx->K_pad, (__nv_bfloat16 *)ctx->Ahi.p,
		    (__nv_bfloat16 *)ctx->Alo.p);
		CKL("split_logw_kernel");
		// the densification counts to the dense E-step (when the M-step stays
		// sparse it is needed for the E-step alone)
		rc = timed(
		    [&] {
			    if (int r = launch_densify(ctx, c0))
				    return r;
			    return launch_estep(ctx, c0, use_scale, bg, rm, true);
		    },
		    rep[5]);
	}
	// the M-step forms on the first chunk's probabilities
	const int psum_d_on = par->need_scaling && par->update_scale;
	if (rc == DFG_OK)
		rc = launch_norm(ctx, c0, psum_d_on, bg);
	if (rc == DFG_OK && !bg)
		rc = timed([&] { return launch_mstep(ctx, c0, false); }, rep[8]);
	if (rc == DFG_OK && dense_ok)
		rc = timed([&] { return launch_mstep(ctx, c0, true); }, rep[9]);
	// resident blocks per SM of the sparse gathers (the plain 3-D path), when
	// the sparse form is the faster; the chunk's probabilities are still those
	// of its normalisation above
	const bool plain = !bg && rm.qmap == nullptr && !tile_skipping(ctx);
	const bool e_sparse = !(dense_ok && rep[5] >= 0. && rep[5] < rep[4]);
	const bool m_sparse = !(dense_ok && rep[9] >= 0. && (rep[8] < 0. || rep[9] < rep[8]));
	int e_minb = ESTEP_MINB, m_minb = MSTEP_MINB;
	if (rc == DFG_OK && plain && e_sparse) {
		const int cand[3] = {2, 3, 4};
		for (int i = 0; i < 3 && rc == DFG_OK; ++i) {
			ctx->tune_estep_minb = cand[i];
			rc = timed([&] { return launch_estep(ctx, c0, use_scale, bg, rm, false); }, rep[10 + i]);
		}
		for (int i = 0; i < 3; ++i)
			if (rep[10 + i] >= 0. && rep[10 + i] < rep[10 + (e_minb - 2)])
				e_minb = cand[i];
		ctx->tune_estep_minb = ESTEP_MINB;
		// the last variant overwrote the chunk's log-likelihoods with equal values
	}
	if (rc == DFG_OK && plain && m_sparse && c0.npix > 0) {
		const int cand[3] = {3, 4, 5};
		for (int i = 0; i < 3 && rc == DFG_OK; ++i) {
			ctx->tune_mstep_minb = cand[i];
			rc = timed([&] { return launch_mstep(ctx, c0, false); }, rep[13 + i]);
		}
		for (int i = 0; i < 3; ++i)
			if (rep[13 + i] >= 0. && rep[13 + i] < rep[13 + (m_minb - 3)])
				m_minb = cand[i];
		ctx->tune_mstep_minb = MSTEP_MINB;
	}
	if (rc == DFG_OK && dense_ok) {
		int derr = 0;
		CK(cudaMemcpy(&derr, ctx->derr.p, sizeof(int), cudaMemcpyDeviceToHost));
		if (derr)
			rc = ctx->fail(DFG_ERR_CUDA, "autotune: a dense kernel gave up");
	}
	if (e0)
		cudaEventDestroy(e0);
	if (e1)
		cudaEventDestroy(e1);
	ctx->tuning = false;
	ctx->timing = save_timing;
	if (rc != DFG_OK)
		return rc;
	ctx->tuned_ob = best_ob;
	ctx->tuned_form = (dense_ok && rep[5] >= 0. && rep[5] < rep[4]) ? 1 : 0;
	ctx->tuned_mform = (dense_ok && rep[9] >= 0. && (rep[8] < 0. || rep[9] < rep[8])) ? 1 : 0;
	ctx->tuned_estep_minb = e_minb;
	ctx->tuned_mstep_minb = m_minb;
	ctx->tuned = true;
	rep[6] = best_ob;
	rep[7] = ctx->tuned_form + 2 * ctx->tuned_mform;
	rep[16] = e_minb;
	rep[17] = m_minb;
	std::copy(rep, rep + DFG_TUNE_REPORT, ctx->tune_report);
	return DFG_OK;
}

extern "C" int dfg_get_autotune_report(dfg_ctx *ctx, double *report) {
	if (!ctx || !report)
		return DFG_ERR_ARG;
	NEED(ctx->tuned, DFG_ERR_STATE, "not tuned for the current inputs");
	std::copy(ctx->tune_report, ctx->tune_report + DFG_TUNE_REPORT, report);
	return DFG_OK;
}

extern "C" int dfg_autotune(dfg_ctx *ctx, const dfg_iter_params *par, double *report) {
	if (!ctx || !par)
		return DFG_ERR_ARG;
	CK(cudaSetDevice(ctx->device));
	NEED(!pair_mode(ctx), DFG_ERR_STATE, "autotune: not with pair lists (their kernels have one form)");
	if (int rc = run_autotune(ctx, par))
		return rc;
	if (report)
		std::copy(ctx->tune_report, ctx->tune_report + DFG_TUNE_REPORT, report);
	return DFG_OK;
}

// maximize's scalar results from h = scalars[0..2] (rescale, sum info, sum
// log-likelihood), read back after its kernels completed.
static void max_finish(dfg_ctx *ctx, const double *h) {
	ctx->rescale = h[0];
	ctx->mutual_info = h[1] / ctx->N;
	ctx->avg_ll = h[2] / ctx->N;
	ctx->have_results = true;
	ctx->have_prob = ctx->keep_prob;
}

extern "C" int dfg_maximize(dfg_ctx *ctx, const dfg_iter_params *par, double *avg_likelihood) {
	if (int rc = max_prepare(ctx, par))
		return rc;
	if (int rc = max_enqueue(ctx, par))
		return rc;
	double h[3];
	int derr = 0;
	CK(cudaMemcpyAsync(h, ctx->scalars.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
	if (ctx->dense_active || ctx->m_dense_active)
		CK(cudaMemcpyAsync(&derr, ctx->derr.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	phase_collect(ctx);
	NEED(derr == 0, DFG_ERR_CUDA, "dense E-step / M-step: a pipeline wait gave up (results invalid)");
	max_finish(ctx, h);
	if (avg_likelihood)
		*avg_likelihood = ctx->avg_ll;
	return DFG_OK;
}

// Rotation lists of the model symmetries, row-major 3x3 each.
// S4 (octahedral, symmetrize_octahedral model.c:636-729): the 48 signed
// permutation matrices. A5 (icosahedral, symmetrize_icosahedral model.c:573-757):
// the 60 rotations of the icosahedron whose vertices are the cyclic
// permutations of (0, +-tau, +-1), the one the reference's table preserves,
// generated by the cyclic axis permutation, diag(-1, -1, 1) and the 72-degree
// rotation about the vertex axis (0, tau, 1), entries snapped to their exact
// values (the reference's table gives them to 11 decimals). Axial (symmetrize_axial model.c:527-571): rotations by
// 2 pi i / order about z, from cos / sin as the reference forms them.
static std::vector<double> octahedral_rotations() {
	std::vector<double> out;
	const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
	for (const auto &pm : perms)
		for (int sg = 0; sg < 8; ++sg) {
			double R[9] = {0};
			for (int i = 0; i < 3; ++i)
				R[3 * i + pm[i]] = (sg >> (2 - i)) & 1 ? -1. : 1.;
			out.insert(out.end(), R, R + 9);
		}
	return out;
}

static std::vector<double> icosahedral_rotations() {
	const double t = (1. + std::sqrt(5.)) / 2.;
	const double exact[5] = {0., 0.5, 1., t / 2., 1. / (2. * t)};
	auto snap = [&](double x) {
		double best = x, bd = 1e300;
		for (double e : exact)
			for (double sg : {1., -1.})
				if (std::fabs(x - sg * e) < bd) {
					bd = std::fabs(x - sg * e);
					best = sg * e;
				}
		return best;
	};
	auto mul = [&](const double *A, const double *B, double *C) {
		for (int i = 0; i < 3; ++i)
			for (int j = 0; j < 3; ++j) {
				double v = 0.;
				for (int k = 0; k < 3; ++k)
					v += A[3 * i + k] * B[3 * k + j];
				C[3 * i + j] = snap(v);
			}
	};
	// 72-degree rotation about the unit axis along (0, tau, 1) (Rodrigues)
	const double nrm = std::sqrt(1. + t * t), ax[3] = {0., t / nrm, 1. / nrm};
	const double c5 = std::cos(2. * M_PI / 5.), s5 = std::sin(2. * M_PI / 5.);
	double F[9];
	for (int i = 0; i < 3; ++i)
		for (int j = 0; j < 3; ++j) {
			double v = (i == j ? c5 : 0.) + (1. - c5) * ax[i] * ax[j];
			const int k = 3 - i - j;  // the remaining axis for the cross-product term
			if (i != j) {
				const double sgn = ((i + 1) % 3 == j) ? -1. : 1.;
				v += sgn * s5 * ax[k];
			}
			F[3 * i + j] = snap(v);
		}
	const double P[9] = {0, 0, 1, 1, 0, 0, 0, 1, 0}, D[9] = {-1, 0, 0, 0, -1, 0, 0, 0, 1};
	std::vector<std::vector<double>> group = {{1, 0, 0, 0, 1, 0, 0, 0, 1}};
	const double *gens[3] = {P, D, F};
	for (size_t i = 0; i < group.size() && group.size() < 60; ++i)
		for (const double *g : gens) {
			std::vector<double> C(9);
			mul(group[i].data(), g, C.data());
			bool found = false;
			for (const auto &h : group) {
				double d = 0.;
				for (int k = 0; k < 9; ++k)
					d += std::fabs(h[k] - C[k]);
				if (d < 1e-9) {
					found = true;
					break;
				}
			}
			if (!found)
				group.push_back(C);
		}
	std::vector<double> out;
	for (const auto &g : group)
		out.insert(out.end(), g.begin(), g.end());
	return out;
}

extern "C" int dfg_set_symmetry(dfg_ctx *ctx, int point_group, int axial_order) {
	if (!ctx)
		return DFG_ERR_ARG;
	NEED(point_group >= 0 && point_group <= 2, DFG_ERR_ARG, "point_group must be 0 (none), 1 (S4) or 2 (A5)");
	NEED(axial_order >= 0, DFG_ERR_ARG, "axial_order must be >= 0");
	CK(cudaSetDevice(ctx->device));
	ctx->n_group_rots = 0;
	if (point_group > 0) {
		std::vector<double> r = point_group == 1 ? octahedral_rotations() : icosahedral_rotations();
		NEED(r.size() == (point_group == 1 ? 48u : 60u) * 9u, DFG_ERR_STATE, "symmetry group generation failed");
		CK(upload(ctx->group_rots, r.data(), r.size(), ctx->stream));
		ctx->n_group_rots = (int)(r.size() / 9);
	}
	ctx->n_axial_rots = 0;
	if (axial_order > 1) {
		std::vector<double> r;
		for (int i = 0; i < axial_order; ++i) {
			const double angle = 2. * M_PI * i / axial_order, c = std::cos(angle), s = std::sin(angle);
			const double R[9] = {c, -s, 0., s, c, 0., 0., 0., 1.};
			r.insert(r.end(), R, R + 9);
		}
		CK(upload(ctx->axial_rots, r.data(), r.size(), ctx->stream));
		ctx->n_axial_rots = axial_order;
	}
	CK(cudaStreamSynchronize(ctx->stream));
	return DFG_OK;
}

// Model.rotate_model (dragonfly/model.pyx:226-254 -> rotate_model,
// model.c:381-425): one thread per voxel v of the cube [-max_r, max_r)^3
// around the centre adds the trilinear interpolation of m at rot v + c to
// rotmodel[v + c], in the reference's operation order (no contraction).
namespace dfg {
__global__ void rotate_model_kernel(const double *__restrict__ rot, const double *__restrict__ m, int s, int max_r,
                                    double *__restrict__ rotmodel) {
	const long long side = 2LL * max_r, n = side * side * side;
	const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	const int c = s / 2;
	const int vx = (int)(i / (side * side)) - max_r, vy = (int)((i / side) % side) - max_r,
	          vz = (int)(i % side) - max_r;
	double rv[3];
#pragma unroll
	for (int k = 0; k < 3; ++k)
		rv[k] = dadd(dadd(dadd(dmul(rot[3 * k], (double)vx), dmul(rot[3 * k + 1], (double)vy)),
		                  dmul(rot[3 * k + 2], (double)vz)), (double)c);
	if (rv[0] < 0 || rv[0] >= s - 1 || rv[1] < 0 || rv[1] >= s - 1 || rv[2] < 0 || rv[2] >= s - 1)
		return;
	const int x = (int)rv[0], y = (int)rv[1], z = (int)rv[2];
	const double fx = dsub(rv[0], (double)x), fy = dsub(rv[1], (double)y), fz = dsub(rv[2], (double)z);
	const double cx = dsub(1., fx), cy = dsub(1., fy), cz = dsub(1., fz);
	const long long ss = (long long)s * s, x1 = (x + 1) % s, y1 = (y + 1) % s, z1 = (z + 1) % s;
	double v = dmul(dmul(dmul(cx, cy), cz), m[x * ss + (long long)y * s + z]);
	v = dadd(v, dmul(dmul(dmul(cx, cy), fz), m[x * ss + (long long)y * s + z1]));
	v = dadd(v, dmul(dmul(dmul(cx, fy), cz), m[x * ss + y1 * s + z]));
	v = dadd(v, dmul(dmul(dmul(cx, fy), fz), m[x * ss + y1 * s + z1]));
	v = dadd(v, dmul(dmul(dmul(fx, cy), cz), m[x1 * ss + (long long)y * s + z]));
	v = dadd(v, dmul(dmul(dmul(fx, cy), fz), m[x1 * ss + (long long)y * s + z1]));
	v = dadd(v, dmul(dmul(dmul(fx, fy), cz), m[x1 * ss + y1 * s + z]));
	v = dadd(v, dmul(dmul(dmul(fx, fy), fz), m[x1 * ss + y1 * s + z1]));
	double *o = rotmodel + (long long)(vx + c) * ss + (long long)(vy + c) * s + (vz + c);
	*o = dadd(*o, v);
}
}  // namespace dfg

extern "C" int dfg_model_rotate(dfg_ctx *ctx, const double *rot, int size, int max_r, const double *model,
                                double *rotmodel) {
	if (!ctx || !rot || !model || !rotmodel)
		return DFG_ERR_ARG;
	NEED(size >= 3 && size <= 2048, DFG_ERR_ARG, "model_rotate: size %d out of [3, 2048]", size);
	if (max_r == 0)
		max_r = size / 2;   // model.c:385-386
	NEED(max_r > 0 && max_r <= size / 2, DFG_ERR_ARG, "model_rotate: max_r %d out of [1, size / 2]", max_r);
	for (int k = 0; k < 9; ++k)
		NEED(std::isfinite(rot[k]), DFG_ERR_ARG, "model_rotate: rotation entry %d is not finite", k);
	CK(cudaSetDevice(ctx->device));
	cudaStream_t st = ctx->stream;
	const size_t V = (size_t)size * size * size;
	DevBuf<double> d_rot, d_m, d_out;
	CK(upload(d_rot, rot, 9, st));
	CK(upload(d_m, model, V, st));
	CK(upload(d_out, rotmodel, V, st));
	const long long n = 8LL * max_r * max_r * max_r;
	rotate_model_kernel<<<blocks_for(n, 256), 256, 0, st>>>(d_rot.p, d_m.p, size, max_r, d_out.p);
	CKL("rotate_model_kernel");
	CK(cudaMemcpyAsync(rotmodel, d_out.p, V * sizeof(double), cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	return DFG_OK;
}

extern "C" int dfg_model_symmetrize(dfg_ctx *ctx, int group, int order, int size, double *model,
                                    double *weights) {
	if (!ctx || !model || !weights)
		return DFG_ERR_ARG;
	NEED(group >= 1 && group <= 3, DFG_ERR_ARG, "model_symmetrize: group must be 1 (S4), 2 (A5) or 3 (axial)");
	NEED(group != 3 || (order >= 1 && order <= 1024), DFG_ERR_ARG, "model_symmetrize: axial order %d", order);
	NEED(size >= 3 && size <= 2048, DFG_ERR_ARG, "model_symmetrize: size %d out of [3, 2048]", size);
	CK(cudaSetDevice(ctx->device));
	cudaStream_t st = ctx->stream;
	std::vector<double> r;
	if (group == 1)
		r = octahedral_rotations();
	else if (group == 2)
		r = icosahedral_rotations();
	else
		for (int i = 0; i < order; ++i) {   // symmetrize_axial, model.c:540-549
			const double angle = 2. * M_PI * i / order, c = std::cos(angle), sn = std::sin(angle);
			const double R[9] = {c, -sn, 0., sn, c, 0., 0., 0., 1.};
			r.insert(r.end(), R, R + 9);
		}
	const long long V = (long long)size * size * size;
	DevBuf<double> d_rot, d_m, d_w;
	DevBuf<double2> d_acc;
	CK(upload(d_rot, r.data(), r.size(), st));
	CK(upload(d_m, model, (size_t)V, st));
	CK(upload(d_w, weights, (size_t)V, st));
	CK(d_acc.ensure((size_t)V));
	symmetrize_kernel<<<blocks_for(V, 256), 256, 0, st>>>(d_m.p, d_w.p, size, d_rot.p, (int)(r.size() / 9), d_acc.p);
	CKL("symmetrize_kernel");
	symmetrize_finish_kernel<<<blocks_for(V, 256), 256, 0, st>>>(d_acc.p, V, d_m.p, d_w.p);
	CKL("symmetrize_finish_kernel");
	CK(cudaMemcpyAsync(model, d_m.p, (size_t)V * sizeof(double), cudaMemcpyDeviceToHost, st));
	CK(cudaMemcpyAsync(weights, d_w.p, (size_t)V * sizeof(double), cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	return DFG_OK;
}

// Queues update_model's kernels; the squared change lands in scalars[3].
static int update_enqueue(dfg_ctx *ctx, double alpha) {
	cudaStream_t st = ctx->stream;
	const long long n = (long long)ctx->M * ctx->V;
	const int S = (int)ctx->S, lo = (S % 2 == 0) ? 1 : 0;
	const long long pairs = (long long)ctx->M * (S - lo) * (S - lo) * (S / 2 - lo + 1);
	phase_begin(ctx, PH_UPDATE);
	int launched = 3;
	// recon.pyx:120-134: the point group replaces the Friedel average; the
	// axial symmetry applies after either
	auto symmetrize = [&](const DevBuf<double> &rots, int nrot) -> int {
		for (int mode = 0; mode < ctx->M; ++mode) {
			double *m2 = ctx->model2.p + (size_t)mode * ctx->V, *w = ctx->weight.p + (size_t)mode * ctx->V;
			symmetrize_kernel<<<blocks_for(ctx->V, 256), 256, 0, st>>>(m2, w, S, rots.p, nrot, ctx->accum.p);
			CKL("symmetrize_kernel");
			symmetrize_finish_kernel<<<blocks_for(ctx->V, 256), 256, 0, st>>>(ctx->accum.p, ctx->V, m2, w);
			CKL("symmetrize_finish_kernel");
			launched += 2;
		}
		return DFG_OK;
	};
	if (ctx->model_type != MT_3D) {
		// image stacks: the 2-D Friedel average for RZ, or for 2-D with
		// params.friedel_sym (recon.pyx:118-119); no volume symmetries
		NEED(ctx->n_group_rots == 0 && ctx->n_axial_rots <= 1, DFG_ERR_ARG,
		     "point-group and axial symmetries apply to 3-D models only");
		if (ctx->model_type == MT_RZ || ctx->friedel2d) {
			const long long pairs2 = (long long)ctx->M * (S - lo) * (S / 2 - lo + 1);
			friedel2d_kernel<<<blocks_for(pairs2, 256), 256, 0, st>>>(ctx->model2.p, ctx->weight.p, S, ctx->M);
			CKL("friedel2d_kernel");
			launched++;
		}
	} else if (ctx->n_group_rots > 0) {
		if (int rc = symmetrize(ctx->group_rots, ctx->n_group_rots))
			return rc;
	} else {
		friedel_kernel<<<blocks_for(pairs, 256), 256, 0, st>>>(ctx->model2.p, ctx->weight.p, S, ctx->M);
		CKL("friedel_kernel");
		launched++;
	}
	if (ctx->model_type == MT_3D && ctx->n_axial_rots > 1)
		if (int rc = symmetrize(ctx->axial_rots, ctx->n_axial_rots))
			return rc;
	const unsigned nb = blocks_for(n, 256);
	divide_update_kernel<float><<<nb, 256, 0, st>>>(ctx->model2.p, ctx->weight.p, ctx->model1.p, nullptr, n,
	                                                alpha, ctx->red_part.p);
	CKL("divide_update_kernel");
	sum_kernel<<<1, 1024, 0, st>>>(ctx->red_part.p, nb, ctx->scalars.p + 3);
	CKL("sum_kernel");
	phase_end(ctx, PH_UPDATE, launched - 1);
	return DFG_OK;
}

extern "C" int dfg_update_model(dfg_ctx *ctx, double alpha, double *rms_change) {
	if (!ctx)
		return DFG_ERR_ARG;
	NEED(ctx->have_results, DFG_ERR_STATE, "update_model: run dfg_maximize first");
	CK(cudaSetDevice(ctx->device));
	if (int rc = update_enqueue(ctx, alpha))
		return rc;
	double change = 0.;
	CK(cudaMemcpyAsync(&change, ctx->scalars.p + 3, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	phase_collect(ctx);
	ctx->rms = std::sqrt(change / ctx->M / (double)ctx->V);
	if (rms_change)
		*rms_change = ctx->rms;
	return DFG_OK;
}

// Queues normalize_scale's kernels: sum and count of the good frames' phi
// into scalars[4..5], then phi /= mean and model1 (mode 0) *= mean.
static int normalize_enqueue(dfg_ctx *ctx) {
	cudaStream_t st = ctx->stream;
	scale_sum_kernel<<<1, 1024, 0, st>>>(ctx->scale.p, ctx->blacklist.p, ctx->N, ctx->scalars.p + 4);
	CKL("scale_sum_kernel");
	const long long n = std::max<long long>(ctx->V, ctx->N);
	apply_scale_norm_kernel<<<blocks_for(n, 256), 256, 0, st>>>(ctx->scale.p, ctx->blacklist.p, ctx->N,
	                                                             ctx->model1.p, nullptr, ctx->V,
	                                                             ctx->scalars.p + 4);
	CKL("apply_scale_norm_kernel");
	return DFG_OK;
}

// The mean from h = scalars[4..5], after normalize_enqueue's kernels ran.
static int normalize_finish(dfg_ctx *ctx, const double *h, double *mean_scale) {
	NEED(h[1] > 0, DFG_ERR_STATE, "normalize_scale: no good frames");
	const double mean = h[0] / h[1];
	ctx->rms *= mean;
	if (mean_scale)
		*mean_scale = mean;
	return DFG_OK;
}

extern "C" int dfg_normalize_scale(dfg_ctx *ctx, double *mean_scale) {
	if (!ctx)
		return DFG_ERR_ARG;
	if (int rc = need_frames(ctx))
		return rc;
	NEED(ctx->S > 0, DFG_ERR_STATE, "model not set");
	CK(cudaSetDevice(ctx->device));
	CK(ctx->scalars.ensure(8));
	if (int rc = normalize_enqueue(ctx))
		return rc;
	double h[2];
	CK(cudaMemcpyAsync(h, ctx->scalars.p + 4, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	return normalize_finish(ctx, h, mean_scale);
}

// One whole iteration (EMCRecon.run_iteration's compute, recon.pyx:94-104):
// maximize, update_model and, when need_scaling (volumes only, recon.pyx:
// 102-103), normalize_scale, with one synchronisation at the end. Where no
// step needs the host in between (graphable) and option graph is on, the
// queued kernels are captured into a CUDA graph and launched as one; the
// graph of the previous iteration is updated in place when only kernel
// arguments changed (beta factor, alpha), else instantiated again.
static int iteration_enqueue(dfg_ctx *ctx, const dfg_iter_params *par, double alpha, bool normalize) {
	if (int rc = max_enqueue(ctx, par))
		return rc;
	if (int rc = update_enqueue(ctx, alpha))
		return rc;
	if (normalize)
		if (int rc = normalize_enqueue(ctx))
			return rc;
	return DFG_OK;
}

// A captured graph replaces *exec in place when only kernel arguments
// changed, else it is instantiated again.
static cudaError_t graph_commit(cudaGraphExec_t *exec, cudaGraph_t g, long *updates, long *instantiations) {
	if (*exec) {
		cudaGraphExecUpdateResultInfo info;
		if (cudaGraphExecUpdate(*exec, g, &info) == cudaSuccess) {
			++*updates;
			return cudaSuccess;
		}
		cudaGetLastError();
		cudaGraphExecDestroy(*exec);
		*exec = nullptr;
	}
	const cudaError_t e = cudaGraphInstantiate(exec, g, 0);
	if (e != cudaSuccess)
		*exec = nullptr;
	else
		++*instantiations;
	return e;
}

static bool iteration_normalizes(const dfg_ctx *ctx, const dfg_iter_params *par) {
	return par->need_scaling && ctx->model_type == MT_3D;
}

// Reads an iteration's scalars back (the one synchronisation) and completes
// its host-side results; out[5] as dfg_run_iteration.
static int iteration_finish(dfg_ctx *ctx, const dfg_iter_params *par, double *out) {
	cudaStream_t st = ctx->stream;
	double h[6];
	int derr = 0;
	CK(cudaMemcpyAsync(h, ctx->scalars.p, 6 * sizeof(double), cudaMemcpyDeviceToHost, st));
	if (ctx->dense_active || ctx->m_dense_active)
		CK(cudaMemcpyAsync(&derr, ctx->derr.p, sizeof(int), cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	phase_collect(ctx);
	NEED(derr == 0, DFG_ERR_CUDA, "dense E-step / M-step: a pipeline wait gave up (results invalid)");
	max_finish(ctx, h);
	ctx->rms = std::sqrt(h[3] / ctx->M / (double)ctx->V);
	double mean = 1.;
	if (iteration_normalizes(ctx, par))
		if (int rc = normalize_finish(ctx, h + 4, &mean))
			return rc;
	if (out) {
		out[0] = ctx->avg_ll;
		out[1] = ctx->rms;
		out[2] = ctx->mutual_info;
		out[3] = ctx->rescale;
		out[4] = mean;
	}
	return DFG_OK;
}

extern "C" int dfg_run_iteration(dfg_ctx *ctx, const dfg_iter_params *par, double alpha, double *out) {
	if (int rc = max_prepare(ctx, par))
		return rc;
	cudaStream_t st = ctx->stream;
	const bool normalize = iteration_normalizes(ctx, par);
	if (ctx->use_graph && graphable(ctx, par)) {
		CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
		ctx->capturing = true;
		const int rc = iteration_enqueue(ctx, par, alpha, normalize);
		cudaGraph_t g = nullptr;
		const cudaError_t e = cudaStreamEndCapture(st, &g);
		ctx->capturing = false;
		if (rc != DFG_OK || e != cudaSuccess) {
			if (g)
				cudaGraphDestroy(g);
			cudaGetLastError();
			return rc != DFG_OK ? rc : ctx->fail(DFG_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
		}
		const cudaError_t ei = graph_commit(&ctx->graph_exec, g, &ctx->graph_updates, &ctx->graph_instantiations);
		cudaGraphDestroy(g);
		NEED(ei == cudaSuccess, DFG_ERR_CUDA, "cudaGraphInstantiate failed: %s", cudaGetErrorString(ei));
		CK(cudaGraphLaunch(ctx->graph_exec, st));
		ctx->graph_launches++;
	} else {
		if (int rc = iteration_enqueue(ctx, par, alpha, normalize))
			return rc;
	}
	return iteration_finish(ctx, par, out);
}

// ---------------------------------------------------------------------------
// batches of independent reconstructions
// ---------------------------------------------------------------------------
struct dfg_batch {
	std::vector<dfg_ctx *> ctxs;
	int lanes = 1;  // concurrent branches; each runs its reconstructions in turn
	int device = 0;
	cudaStream_t stream = nullptr;
	cudaEvent_t fork = nullptr;
	std::vector<cudaEvent_t> joins;
	cudaGraphExec_t exec = nullptr;
	long launches = 0, updates = 0, instantiations = 0;
	std::string err;
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

extern "C" void dfg_batch_destroy(dfg_batch *b) {
	if (!b)
		return;
	cudaSetDevice(b->device);
	if (b->stream)
		cudaStreamSynchronize(b->stream);
	if (b->exec)
		cudaGraphExecDestroy(b->exec);
	for (auto e : b->joins)
		if (e)
			cudaEventDestroy(e);
	if (b->fork)
		cudaEventDestroy(b->fork);
	if (b->stream)
		cudaStreamDestroy(b->stream);
	delete b;
}

extern "C" int dfg_batch_create(dfg_ctx *const *ctxs, int n, dfg_batch **out) {
	if (!ctxs || n < 1 || !out)
		return DFG_ERR_ARG;
	*out = nullptr;
	for (int i = 0; i < n; ++i) {
		if (!ctxs[i] || ctxs[i]->device != ctxs[0]->device)
			return DFG_ERR_ARG;
		for (int j = 0; j < i; ++j)
			if (ctxs[j] == ctxs[i])
				return DFG_ERR_ARG;
	}
	dfg_batch *b = new dfg_batch();
	b->ctxs.assign(ctxs, ctxs + n);
	b->device = ctxs[0]->device;
	b->joins.assign((size_t)n, nullptr);
	b->lanes = 1;
	bool ok = cudaSetDevice(b->device) == cudaSuccess &&
	          cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
	          cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess;
	for (int i = 0; i < n && ok; ++i)
		ok = cudaEventCreateWithFlags(&b->joins[i], cudaEventDisableTiming) == cudaSuccess;
	if (!ok) {
		dfg_batch_destroy(b);
		return DFG_ERR_CUDA;
	}
	*out = b;
	return DFG_OK;
}

extern "C" const char *dfg_batch_last_error(const dfg_batch *b) { return b ? b->err.c_str() : "null batch"; }

extern "C" int dfg_batch_set_lanes(dfg_batch *b, int lanes) {
	if (!b || lanes < 1)
		return DFG_ERR_ARG;
	b->lanes = std::min<int>(lanes, (int)b->ctxs.size());
	return DFG_OK;
}

extern "C" int dfg_batch_stats(dfg_batch *b, long *out) {
	if (!b || !out)
		return DFG_ERR_ARG;
	out[0] = b->launches;
	out[1] = b->instantiations;
	out[2] = b->updates;
	return DFG_OK;
}

extern "C" int dfg_batch_run(dfg_batch *b, const dfg_iter_params *pars, const double *alphas, double *out) {
	if (!b || !pars)
		return DFG_ERR_ARG;
	const int n = (int)b->ctxs.size();
	if (cudaSetDevice(b->device) != cudaSuccess)
		return b->fail(DFG_ERR_CUDA, "cudaSetDevice failed");
	bool graph = true;
	for (int i = 0; i < n; ++i) {
		dfg_ctx *c = b->ctxs[i];
		if (int rc = max_prepare(c, &pars[i]))
			return b->fail(rc, "reconstruction %d: %s", i, c->err.c_str());
		graph = graph && c->use_graph && graphable(c, &pars[i]);
	}
	auto alpha = [&](int i) { return alphas ? alphas[i] : 0.; };
	if (graph) {
		// one graph: a branch per reconstruction on its own stream, forked
		// from and joined back into the batch stream, so their kernels run
		// side by side
		if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
			return b->fail(DFG_ERR_CUDA, "cudaStreamBeginCapture failed");
		// lanes: reconstructions dealt out in decreasing pair count to the
		// least-loaded lane; within a lane each waits for the one before
		std::vector<int> order(n), lane_of(n), prev(n, -1), last((size_t)b->lanes, -1);
		std::vector<double> load((size_t)b->lanes, 0.);
		for (int i = 0; i < n; ++i)
			order[i] = i;
		auto work = [&](int i) { return (double)b->ctxs[i]->R * b->ctxs[i]->N; };
		std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return work(x) > work(y); });
		for (int i : order) {
			const int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
			lane_of[i] = l;
			prev[i] = last[l];
			last[l] = i;
			load[l] += work(i);
		}
		int rc = DFG_OK, bad = -1;
		cudaError_t e = cudaEventRecord(b->fork, b->stream);
		for (int i : order) {
			if (e != cudaSuccess)
				break;
			dfg_ctx *c = b->ctxs[i];
			e = cudaStreamWaitEvent(c->stream, prev[i] < 0 ? b->fork : b->joins[prev[i]], 0);
			if (e != cudaSuccess)
				break;
			if (rc == DFG_OK) {
				c->capturing = true;
				rc = iteration_enqueue(c, &pars[i], alpha(i), iteration_normalizes(c, &pars[i]));
				c->capturing = false;
				if (rc != DFG_OK)
					bad = i;
			}
			e = cudaEventRecord(b->joins[i], c->stream);
		}
		for (int l = 0; l < b->lanes && e == cudaSuccess; ++l)
			if (last[l] >= 0)
				e = cudaStreamWaitEvent(b->stream, b->joins[last[l]], 0);
		cudaGraph_t g = nullptr;
		const cudaError_t ee = cudaStreamEndCapture(b->stream, &g);
		if (rc != DFG_OK || e != cudaSuccess || ee != cudaSuccess) {
			if (g)
				cudaGraphDestroy(g);
			cudaGetLastError();
			if (rc != DFG_OK)
				return b->fail(rc, "reconstruction %d: %s", bad, b->ctxs[bad]->err.c_str());
			return b->fail(DFG_ERR_CUDA, "batch capture failed: %s",
			               cudaGetErrorString(e != cudaSuccess ? e : ee));
		}
		const cudaError_t ei = graph_commit(&b->exec, g, &b->updates, &b->instantiations);
		cudaGraphDestroy(g);
		if (ei != cudaSuccess)
			return b->fail(DFG_ERR_CUDA, "cudaGraphInstantiate failed: %s", cudaGetErrorString(ei));
		if (cudaGraphLaunch(b->exec, b->stream) != cudaSuccess || cudaStreamSynchronize(b->stream) != cudaSuccess)
			return b->fail(DFG_ERR_CUDA, "batch graph launch failed: %s", cudaGetErrorString(cudaGetLastError()));
		b->launches++;
		for (int i = 0; i < n; ++i)
			b->ctxs[i]->graph_launches++;
	} else {
		// some reconstruction needs the host between kernels: queue each on
		// its own stream without a graph
		for (int i = 0; i < n; ++i) {
			dfg_ctx *c = b->ctxs[i];
			if (int rc = iteration_enqueue(c, &pars[i], alpha(i), iteration_normalizes(c, &pars[i])))
				return b->fail(rc, "reconstruction %d: %s", i, c->err.c_str());
		}
	}
	for (int i = 0; i < n; ++i) {
		dfg_ctx *c = b->ctxs[i];
		if (int rc = iteration_finish(c, &pars[i], out ? out + 5 * (size_t)i : nullptr))
			return b->fail(rc, "reconstruction %d: %s", i, c->err.c_str());
	}
	return DFG_OK;
}

extern "C" int dfg_run_iteration_host(dfg_ctx *ctx, const dfg_iter_params *par, double alpha,
                                      double *model1_inout, int *rmax, double *likelihood,
                                      double *avg_likelihood, double *rms_change) {
	if (!ctx || !par || !model1_inout)
		return DFG_ERR_ARG;
	NEED(ctx->S > 0, DFG_ERR_STATE, "model not set");
	CK(cudaSetDevice(ctx->device));
	const size_t n = (size_t)ctx->M * ctx->V;
	CK(cudaMemcpyAsync(ctx->model1.p, model1_inout, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
	double out[5];
	if (int rc = dfg_run_iteration(ctx, par, alpha, out))
		return rc;
	const double ll = out[0], rms = out[1];
	CK(cudaMemcpyAsync(model1_inout, ctx->model1.p, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
	if (rmax)
		CK(cudaMemcpyAsync(rmax, ctx->rmax.p, (size_t)ctx->N * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
	if (likelihood)
		CK(cudaMemcpyAsync(likelihood, ctx->likelihood.p, (size_t)ctx->N * sizeof(double), cudaMemcpyDeviceToHost,
		                   ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	if (avg_likelihood)
		*avg_likelihood = ll;
	if (rms_change)
		*rms_change = rms;
	return DFG_OK;
}

// ---------------------------------------------------------------------------
// several detectors in one reconstruction
// ---------------------------------------------------------------------------
// Iterate with an in_detector_list (iterate.pyx:432-456): member k is a
// context holding detector k and the frames it sees. The reference's
// per-detector quantities (u, rescale, psum_r, the tomograms: max_prob.c:
// 31-60, max_update.c:33-36, 55-128, 153-229) live in the members; what the
// detectors share is the model: the merged sums of every member are added
// into member 0's (the reference merges all detectors into one model2 /
// inter_weight), member 0 updates the model and every member gets a copy.
// Frame-wide quantities (average log-likelihood, mutual information, the
// mean scale of normalize_scale) are taken over the frames of all members.
struct dfg_group {
	std::vector<dfg_ctx *> m;
	std::string err;
	bool have_results = false;
	double avg_ll = 0., mutual_info = 0., rms = 0.;
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

#define GNEED(cond, code, ...)                  \
	do {                                        \
		if (!(cond))                            \
			return g->fail(code, __VA_ARGS__);  \
	} while (0)
#define GCK(call)                                                                                   \
	do {                                                                                            \
		cudaError_t e_ = (call);                                                                    \
		if (e_ != cudaSuccess)                                                                      \
			return g->fail(DFG_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
	} while (0)

extern "C" void dfg_group_destroy(dfg_group *g) { delete g; }

extern "C" const char *dfg_group_last_error(const dfg_group *g) { return g ? g->err.c_str() : "null group"; }

extern "C" int dfg_group_create(dfg_ctx *const *members, int n, dfg_group **out) {
	if (!members || n < 1 || !out)
		return DFG_ERR_ARG;
	*out = nullptr;
	for (int i = 0; i < n; ++i)
		if (!members[i])
			return DFG_ERR_ARG;
	dfg_group *g = new dfg_group;
	g->m.assign(members, members + n);
	*out = g;
	return DFG_OK;
}

// The members must agree on everything but their detector and frames.
static int group_check(dfg_group *g) {
	dfg_ctx *a = g->m[0];
	for (size_t k = 0; k < g->m.size(); ++k) {
		dfg_ctx *c = g->m[k];
		GNEED(c->device == a->device, DFG_ERR_ARG, "detector %d: another device", (int)k);
		GNEED(c->P > 0 && c->N > 0, DFG_ERR_STATE, "detector %d: set detector and frames", (int)k);
		GNEED(c->S > 0 && c->S == a->S && c->M == a->M && c->model_type == a->model_type, DFG_ERR_ARG,
		      "detector %d: the model must have the same shape and type as detector 0's", (int)k);
		GNEED(c->num_rot == a->num_rot, DFG_ERR_ARG, "detector %d: another orientation count", (int)k);
		GNEED(c->refine == a->refine, DFG_ERR_ARG, "detector %d: refinement on some detectors only", (int)k);
		// the background-aware updates couple the detectors (scalemax over
		// all frames, mean_count averaged over the detectors: max_update.c:
		// 350-356); not built for several detectors
		GNEED(!c->with_bg || g->m.size() == 1, DFG_ERR_ARG,
		      "background-aware updates with several detectors are not supported");
		for (size_t j = 0; j < k; ++j)
			GNEED(g->m[j] != c, DFG_ERR_ARG, "detector %d repeats detector %d", (int)k, (int)j);
	}
	return DFG_OK;
}

extern "C" int dfg_group_maximize(dfg_group *g, const dfg_iter_params *par, double *avg_likelihood) {
	if (!g || !par)
		return DFG_ERR_ARG;
	if (int rc = group_check(g))
		return rc;
	dfg_ctx *m0 = g->m[0];
	GCK(cudaSetDevice(m0->device));
	// every member's iteration on its own stream
	for (size_t k = 0; k < g->m.size(); ++k) {
		dfg_ctx *c = g->m[k];
		if (int rc = max_prepare(c, par))
			return g->fail(rc, "detector %d: %s", (int)k, c->err.c_str());
		if (int rc = max_enqueue(c, par))
			return g->fail(rc, "detector %d: %s", (int)k, c->err.c_str());
	}
	double sum_mi = 0., sum_ll = 0.;
	long long n = 0;
	std::vector<double> h(3 * g->m.size());
	for (size_t k = 0; k < g->m.size(); ++k) {
		dfg_ctx *c = g->m[k];
		int derr = 0;
		GCK(cudaMemcpyAsync(&h[3 * k], c->scalars.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
		if (c->dense_active || c->m_dense_active)
			GCK(cudaMemcpyAsync(&derr, c->derr.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
		GCK(cudaStreamSynchronize(c->stream));
		phase_collect(c);
		GNEED(derr == 0, DFG_ERR_CUDA, "detector %d: dense E-step / M-step: a pipeline wait gave up", (int)k);
		max_finish(c, &h[3 * k]);
		sum_mi += h[3 * k + 1];
		sum_ll += h[3 * k + 2];
		n += c->N;
	}
	// one model: the other members' merged sums added into member 0's
	const long long mv = (long long)m0->M * m0->V;
	for (size_t k = 1; k < g->m.size(); ++k) {
		add_into_kernel<<<blocks_for(mv, 256), 256, 0, m0->stream>>>(m0->model2.p, g->m[k]->model2.p, mv);
		add_into_kernel<<<blocks_for(mv, 256), 256, 0, m0->stream>>>(m0->weight.p, g->m[k]->weight.p, mv);
		GCK(cudaGetLastError());
	}
	GCK(cudaStreamSynchronize(m0->stream));
	g->mutual_info = sum_mi / (double)n;
	g->avg_ll = sum_ll / (double)n;
	g->have_results = true;
	if (avg_likelihood)
		*avg_likelihood = g->avg_ll;
	return DFG_OK;
}

// member 0's model to the others (after an update or a scale normalisation)
static int group_share_model(dfg_group *g) {
	dfg_ctx *m0 = g->m[0];
	const size_t n = (size_t)m0->M * m0->V;
	for (size_t k = 1; k < g->m.size(); ++k)
		GCK(cudaMemcpyAsync(g->m[k]->model1.p, m0->model1.p, n * sizeof(double), cudaMemcpyDeviceToDevice,
		                    m0->stream));
	GCK(cudaStreamSynchronize(m0->stream));
	return DFG_OK;
}

extern "C" int dfg_group_update_model(dfg_group *g, double alpha, double *rms_change) {
	if (!g)
		return DFG_ERR_ARG;
	GNEED(g->have_results, DFG_ERR_STATE, "update_model: run dfg_group_maximize first");
	dfg_ctx *m0 = g->m[0];
	if (int rc = dfg_update_model(m0, alpha, &g->rms))
		return g->fail(rc, "%s", m0->err.c_str());
	if (int rc = group_share_model(g))
		return rc;
	if (rms_change)
		*rms_change = g->rms;
	return DFG_OK;
}

// normalize_scale over the frames of all detectors (iterate.pyx:361-384):
// the mean of the good frames' scale factors divides each member's factors;
// member 0's model (mode 0) is multiplied by it and shared.
extern "C" int dfg_group_normalize_scale(dfg_group *g, double *mean_scale) {
	if (!g)
		return DFG_ERR_ARG;
	if (int rc = group_check(g))
		return rc;
	dfg_ctx *m0 = g->m[0];
	GCK(cudaSetDevice(m0->device));
	double tot[2] = {0., 0.};
	for (dfg_ctx *c : g->m) {
		GCK(c->scalars.ensure(8));
		scale_sum_kernel<<<1, 1024, 0, c->stream>>>(c->scale.p, c->blacklist.p, c->N, c->scalars.p + 4);
		GCK(cudaGetLastError());
		double h[2];
		GCK(cudaMemcpyAsync(h, c->scalars.p + 4, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
		GCK(cudaStreamSynchronize(c->stream));
		tot[0] += h[0];
		tot[1] += h[1];
	}
	GNEED(tot[1] > 0, DFG_ERR_STATE, "normalize_scale: no good frames");
	for (size_t k = 0; k < g->m.size(); ++k) {
		dfg_ctx *c = g->m[k];
		GCK(cudaMemcpyAsync(c->scalars.p + 4, tot, 2 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
		const long long V = k == 0 ? m0->V : 0;  // the model once, in member 0
		const long long nn = std::max<long long>(V, c->N);
		apply_scale_norm_kernel<<<blocks_for(nn, 256), 256, 0, c->stream>>>(c->scale.p, c->blacklist.p, c->N,
		                                                                   c->model1.p, nullptr, V, c->scalars.p + 4);
		GCK(cudaGetLastError());
		GCK(cudaStreamSynchronize(c->stream));
	}
	if (int rc = group_share_model(g))
		return rc;
	const double mean = tot[0] / tot[1];
	g->rms *= mean;
	for (dfg_ctx *c : g->m)
		c->rms = g->rms;
	if (mean_scale)
		*mean_scale = mean;
	return DFG_OK;
}

// One iteration over all detectors: maximize, update_model and, when
// need_scaling (volumes only, recon.pyx:102-103), normalize_scale. out[5]:
// average log-likelihood, rms change, mutual information, detector 0's
// rescale factor, mean scale (1 without normalisation).
extern "C" int dfg_group_run_iteration(dfg_group *g, const dfg_iter_params *par, double alpha, double *out) {
	if (!g || !par)
		return DFG_ERR_ARG;
	if (int rc = dfg_group_maximize(g, par, nullptr))
		return rc;
	if (int rc = dfg_group_update_model(g, alpha, nullptr))
		return rc;
	double mean = 1.;
	if (iteration_normalizes(g->m[0], par))
		if (int rc = dfg_group_normalize_scale(g, &mean))
			return rc;
	if (out) {
		out[0] = g->avg_ll;
		out[1] = g->rms;
		out[2] = g->mutual_info;
		out[3] = g->m[0]->rescale;
		out[4] = mean;
	}
	return DFG_OK;
}

#undef GNEED
#undef GCK

// ---------------------------------------------------------------------------
// results
// ---------------------------------------------------------------------------
template <typename T>
static cudaError_t fetch(T *h, const DevBuf<T> &b, size_t n, cudaStream_t s) {
	if (h == nullptr || n == 0)
		return cudaSuccess;
	return cudaMemcpyAsync(h, b.p, n * sizeof(T), cudaMemcpyDeviceToHost, s);
}

extern "C" int dfg_get_frame_results(dfg_ctx *ctx, int *rmax, double *info, double *likelihood,
                                     double *max_exp, double *p_norm, double *psum_d) {
	if (!ctx)
		return DFG_ERR_ARG;
	NEED(ctx->have_results, DFG_ERR_STATE, "no results yet");
	CK(cudaSetDevice(ctx->device));
	const size_t N = (size_t)ctx->N;
	CK(fetch(rmax, ctx->rmax, N, ctx->stream));
	CK(fetch(info, ctx->info, N, ctx->stream));
	CK(fetch(likelihood, ctx->likelihood, N, ctx->stream));
	CK(fetch(max_exp, ctx->max_exp, N, ctx->stream));
	CK(fetch(p_norm, ctx->p_norm, N, ctx->stream));
	CK(fetch(psum_d, ctx->psum_d, N, ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	return DFG_OK;
}

extern "C" int dfg_get_num_prob(dfg_ctx *ctx, int *num_prob) {
	if (!ctx || !num_prob)
		return DFG_ERR_ARG;
	NEED(ctx->have_results, DFG_ERR_STATE, "no results yet");
	CK(cudaSetDevice(ctx->device));
	CK(fetch(num_prob, ctx->num_prob, (size_t)ctx->N, ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	return DFG_OK;
}

extern "C" int dfg_get_sparse_prob_offsets(dfg_ctx *ctx, long long *offsets) {
	if (!ctx || !offsets)
		return DFG_ERR_ARG;
	NEED(ctx->have_prob, DFG_ERR_STATE, "no sparse probabilities: set option keep_prob and run dfg_maximize");
	std::memcpy(offsets, ctx->h_prob_off.data(), ctx->h_prob_off.size() * sizeof(long long));
	return DFG_OK;
}

extern "C" int dfg_get_sparse_prob(dfg_ctx *ctx, int *place_prob, double *prob) {
	if (!ctx)
		return DFG_ERR_ARG;
	NEED(ctx->have_prob, DFG_ERR_STATE, "no sparse probabilities: set option keep_prob and run dfg_maximize");
	if (place_prob)
		std::memcpy(place_prob, ctx->h_place_prob.data(), ctx->h_place_prob.size() * sizeof(int));
	if (prob)
		std::memcpy(prob, ctx->h_prob.data(), ctx->h_prob.size() * sizeof(double));
	return DFG_OK;
}

extern "C" int dfg_get_tomograms(dfg_ctx *ctx, int r0, int n, double *out) {
	if (!ctx || !out)
		return DFG_ERR_ARG;
	NEED(ctx->have_results, DFG_ERR_STATE, "no results yet");
	NEED(!ctx->last_pairs && !ctx->blocked, DFG_ERR_STATE,
	     "tomograms are not kept with pair lists or orientation blocks (one block at a time)");
	NEED(r0 >= 0 && n >= 1 && (long long)r0 + n <= ctx->R, DFG_ERR_ARG,
	     "orientations %d..%lld outside 0..%d", r0, (long long)r0 + n - 1, ctx->R - 1);
	CK(cudaSetDevice(ctx->device));
	const size_t count = (size_t)n * ctx->P;
	CK(ctx->tomo_out.ensure(count));
	tomogram_kernel<<<blocks_for((long long)count, 256), 256, 0, ctx->stream>>>(
	    ctx->T.p, ctx->views_final ? nullptr : ctx->psum_r.p, ctx->P, r0, n, ctx->tomo_out.p);
	CKL("tomogram_kernel");
	CK(fetch(out, ctx->tomo_out, count, ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	return DFG_OK;
}

extern "C" int dfg_get_quat_norm(dfg_ctx *ctx, double *quat_norm) {
	if (!ctx || !quat_norm)
		return DFG_ERR_ARG;
	NEED(ctx->have_results, DFG_ERR_STATE, "no results yet");
	const size_t n = (size_t)ctx->N * ctx->M;
	if (ctx->M == 1) {
		memset(quat_norm, 0, n * sizeof(double));
		return DFG_OK;
	}
	CK(cudaSetDevice(ctx->device));
	CK(fetch(quat_norm, ctx->quat_norm, n, ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	return DFG_OK;
}

extern "C" int dfg_get_orientation_results(dfg_ctx *ctx, double *u, double *psum_r) {
	if (!ctx)
		return DFG_ERR_ARG;
	NEED(ctx->have_results, DFG_ERR_STATE, "no results yet");
	CK(cudaSetDevice(ctx->device));
	CK(fetch(u, ctx->u, (size_t)ctx->R, ctx->stream));
	CK(fetch(psum_r, ctx->psum_r, (size_t)ctx->R, ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	return DFG_OK;
}

extern "C" int dfg_get_model(dfg_ctx *ctx, double *model1, double *model2, double *inter_weight) {
	if (!ctx)
		return DFG_ERR_ARG;
	NEED(ctx->S > 0, DFG_ERR_STATE, "model not set");
	CK(cudaSetDevice(ctx->device));
	const size_t n = (size_t)ctx->M * ctx->V;
	CK(fetch(model1, ctx->model1, n, ctx->stream));
	CK(fetch(model2, ctx->model2, n, ctx->stream));
	CK(fetch(inter_weight, ctx->weight, n, ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	return DFG_OK;
}

extern "C" int dfg_get_frame_params(dfg_ctx *ctx, double *scale, double *beta, double *beta_start, int *fcounts,
                                    double *sum_fact, uint8_t *blacklist) {
	if (!ctx)
		return DFG_ERR_ARG;
	if (int rc = need_frames(ctx))
		return rc;
	CK(cudaSetDevice(ctx->device));
	const size_t N = (size_t)ctx->N;
	CK(fetch(scale, ctx->scale, N, ctx->stream));
	if (ctx->beta_set) {
		CK(fetch(beta, ctx->beta, N, ctx->stream));
		CK(fetch(beta_start, ctx->beta_start, N, ctx->stream));
	}
	CK(fetch(fcounts, ctx->fcounts, N, ctx->stream));
	CK(fetch(sum_fact, ctx->sum_fact, N, ctx->stream));
	CK(fetch(blacklist, ctx->blacklist, N, ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	return DFG_OK;
}

extern "C" int dfg_get_scalars(dfg_ctx *ctx, double *out) {
	if (!ctx || !out)
		return DFG_ERR_ARG;
	out[0] = ctx->rescale;
	out[1] = ctx->mutual_info;
	out[2] = ctx->avg_ll;
	out[3] = ctx->mean_count;
	out[4] = ctx->rms;
	return DFG_OK;
}

// ---------------------------------------------------------------------------
// one-slice operations
// ---------------------------------------------------------------------------
// Orientation parameters of one slice for slice_one_kernel / merge_one_kernel:
// the quaternion (3-D); cos, sin of the angle quat[0] (2-D); cos, sin of phi =
// quat[0] and of beta = quat[1] and the detector distance (RZ). cos and sin
// come from the host's libm, as make_rot_angle's (model.c:788-795).
static int orientation_params(const dfg_ctx *ctx, const double *quat, double *g) {
	if (ctx->model_type == MT_2D) {
		g[0] = std::cos(quat[0]);
		g[1] = std::sin(quat[0]);
		return 2;
	}
	if (ctx->model_type == MT_RZ) {
		g[0] = std::cos(quat[0]);
		g[1] = std::sin(quat[0]);
		g[2] = std::cos(quat[1]);
		g[3] = std::sin(quat[1]);
		g[4] = ctx->detd;
		return 5;
	}
	for (int k = 0; k < 5; ++k)
		g[k] = quat[k];
	return 5;
}

extern "C" int dfg_slice_gen(dfg_ctx *ctx, const double *quat, int mode, double *out) {
	if (!ctx || !quat || !out)
		return DFG_ERR_ARG;
	NEED(ctx->P > 0 && ctx->S > 0, DFG_ERR_STATE, "slice_gen: detector and model must be set");
	NEED(mode >= 0 && mode < ctx->M, DFG_ERR_ARG, "slice_gen: mode %d out of range", mode);
	CK(cudaSetDevice(ctx->device));
	CK(ctx->scalars.ensure(8));
	DevBuf<double> q, o;
	double g[8];
	const int ng = orientation_params(ctx, quat, g);
	CK(upload(q, g, (size_t)ng, ctx->stream));
	CK(o.ensure((size_t)ctx->P));
	const unsigned nb = blocks_for(ctx->P, 256);
	if (ctx->model_type == MT_2D)
		slice_one_kernel<MT_2D><<<nb, 256, 0, ctx->stream>>>(q.p, mode, ctx->qvals.p, ctx->corr.p, ctx->P,
		                                                     ctx->model1.p, ctx->S, ctx->V, o.p);
	else if (ctx->model_type == MT_RZ)
		slice_one_kernel<MT_RZ><<<nb, 256, 0, ctx->stream>>>(q.p, mode, ctx->qvals.p, ctx->corr.p, ctx->P,
		                                                     ctx->model1.p, ctx->S, ctx->V, o.p);
	else
		slice_one_kernel<MT_3D><<<nb, 256, 0, ctx->stream>>>(q.p, mode, ctx->qvals.p, ctx->corr.p, ctx->P,
		                                                     ctx->model1.p, ctx->S, ctx->V, o.p);
	CKL("slice_one_kernel");
	CK(cudaMemcpyAsync(out, o.p, (size_t)ctx->P * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	return DFG_OK;
}

extern "C" int dfg_slice_merge(dfg_ctx *ctx, const double *quat, int mode, const double *view, double *model2,
                               double *inter_weight) {
	if (!ctx || !quat || !view || !model2 || !inter_weight)
		return DFG_ERR_ARG;
	NEED(ctx->P > 0 && ctx->S > 0, DFG_ERR_STATE, "slice_merge: detector and model must be set");
	NEED(mode >= 0 && mode < ctx->M, DFG_ERR_ARG, "slice_merge: mode %d out of range", mode);
	CK(cudaSetDevice(ctx->device));
	const size_t n = (size_t)ctx->M * ctx->V;
	DevBuf<double> q, v, m2, w;
	double g[8];
	const int ng = orientation_params(ctx, quat, g);
	CK(upload(q, g, (size_t)ng, ctx->stream));
	CK(upload(v, view, (size_t)ctx->P, ctx->stream));
	CK(upload(m2, model2, n, ctx->stream));
	CK(upload(w, inter_weight, n, ctx->stream));
	const unsigned nb = blocks_for(ctx->P, 256);
#define DFG_MERGE_ONE(G)                                                                                       \
	merge_one_kernel<G><<<nb, 256, 0, ctx->stream>>>(q.p, mode, v.p, ctx->qvals.p, ctx->corr.p, ctx->mask.p, ctx->P, \
	                                                 ctx->S, ctx->V, m2.p, w.p)
	if (ctx->model_type == MT_2D)
		DFG_MERGE_ONE(MT_2D);
	else if (ctx->model_type == MT_RZ)
		DFG_MERGE_ONE(MT_RZ);
	else
		DFG_MERGE_ONE(MT_3D);
#undef DFG_MERGE_ONE
	CKL("merge_one_kernel");
	CK(cudaMemcpyAsync(model2, m2.p, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
	CK(cudaMemcpyAsync(inter_weight, w.p, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
	CK(cudaStreamSynchronize(ctx->stream));
	return DFG_OK;
}

// ---------------------------------------------------------------------------
// options and instrumentation
// ---------------------------------------------------------------------------
extern "C" int dfg_set_option(dfg_ctx *ctx, const char *key, double value) {
	if (!ctx || !key)
		return DFG_ERR_ARG;
	if (!strcmp(key, "pair_budget_mb")) {
		NEED(value >= 0., DFG_ERR_ARG, "pair_budget_mb must be >= 0");
		ctx->pair_budget_mb = value;
		ctx->chunks_R = -1;
		return DFG_OK;
	}
	if (!strcmp(key, "timing")) {
		ctx->timing = value != 0.;
		return DFG_OK;
	}
	if (!strcmp(key, "keep_prob")) {
		ctx->keep_prob = value != 0.;
		return DFG_OK;
	}
	if (!strcmp(key, "graph")) {
		ctx->use_graph = value != 0.;
		return DFG_OK;
	}
	if (!strcmp(key, "autotune")) {
		ctx->autotune = value != 0.;
		return DFG_OK;
	}
	if (!strcmp(key, "estep_form")) {
		const int v = (int)value;
		NEED(v == 0 || v == 1, DFG_ERR_ARG, "estep_form must be 0 (sparse) or 1 (dense)");
		ctx->estep_form = v;
		return DFG_OK;
	}
	if (!strcmp(key, "pair_lists")) {
		ctx->pair_lists = value != 0.;
		return DFG_OK;
	}
	if (!strcmp(key, "block_budget_mb")) {
		NEED(value >= 0., DFG_ERR_ARG, "block_budget_mb must be >= 0");
		ctx->block_budget_mb = value;
		ctx->blk_tiles = 0;
		return DFG_OK;
	}
	if (!strcmp(key, "tile_skip")) {
		ctx->mstep_skip = value != 0.;
		return DFG_OK;
	}
	if (!strcmp(key, "estep_blocks_per_sm")) {
		NEED(value == 0 || value == 2 || value == 3 || value == 4, DFG_ERR_ARG,
		     "estep_blocks_per_sm must be 0 (tuned / default), 2, 3 or 4");
		ctx->estep_minb = (int)value;
		return DFG_OK;
	}
	if (!strcmp(key, "mstep_blocks_per_sm")) {
		NEED(value == 0 || value == 3 || value == 4 || value == 5, DFG_ERR_ARG,
		     "mstep_blocks_per_sm must be 0 (tuned / default), 3, 4 or 5");
		ctx->mstep_minb = (int)value;
		return DFG_OK;
	}
	if (!strcmp(key, "dense_wait_cycles")) {
		NEED(value >= 1e4 && value <= 1e11, DFG_ERR_ARG, "dense_wait_cycles must be in [1e4, 1e11]");
		ctx->dense_wait_cycles = (long long)value;
		return DFG_OK;
	}
	if (!strcmp(key, "dense_withhold_stage")) {
		NEED(value >= -1 && value < 1e6, DFG_ERR_ARG, "dense_withhold_stage must be -1 or a stage index");
		ctx->dense_withhold = (int)value;
		return DFG_OK;
	}
	if (!strcmp(key, "mstep_form")) {
		const int v = (int)value;
		NEED(v == 0 || v == 1, DFG_ERR_ARG, "mstep_form must be 0 (sparse) or 1 (dense)");
		ctx->mstep_form = v;
		return DFG_OK;
	}
	if (!strcmp(key, "slice_block")) {
		const int v = (int)value;
		NEED(v == 0 || ((v == 16 || v == 32 || v == 64 || v == TILE) && v <= TILE), DFG_ERR_ARG,
		     "slice_block must be 0 (automatic), 16, 32, 64 (at most %d) or %d", TILE, TILE);
		ctx->slice_block = v;
		return DFG_OK;
	}
	return ctx->fail(DFG_ERR_ARG, "unknown option '%s'", key);
}

extern "C" int dfg_get_graph_stats(dfg_ctx *ctx, long *out) {
	if (!ctx || !out)
		return DFG_ERR_ARG;
	out[0] = ctx->graph_launches;
	out[1] = ctx->graph_instantiations;
	out[2] = ctx->graph_updates;
	return DFG_OK;
}

extern "C" int dfg_get_phase_times(dfg_ctx *ctx, double *ms, long *launches, int n) {
	if (!ctx)
		return DFG_ERR_ARG;
	for (int i = 0; i < n && i < PH_COUNT; ++i) {
		if (ms)
			ms[i] = ctx->phase_ms[i];
		if (launches)
			launches[i] = ctx->phase_launches[i];
	}
	return PH_COUNT;
}

extern "C" const char *dfg_phase_name(int i) { return (i >= 0 && i < PH_COUNT) ? kPhaseNames[i] : ""; }

extern "C" int dfg_reset_phase_times(dfg_ctx *ctx) {
	if (!ctx)
		return DFG_ERR_ARG;
	for (int i = 0; i < PH_COUNT; ++i) {
		ctx->phase_ms[i] = 0.;
		ctx->phase_launches[i] = 0;
	}
	return DFG_OK;
}

extern "C" int dfg_event_record(dfg_ctx *ctx, int slot) {
	if (!ctx || slot < 0 || slot >= 8)
		return DFG_ERR_ARG;
	CK(cudaSetDevice(ctx->device));
	CK(cudaEventRecord(ctx->user_ev[slot], ctx->stream));
	return DFG_OK;
}

extern "C" int dfg_event_elapsed(dfg_ctx *ctx, int a, int b, double *ms) {
	if (!ctx || !ms || a < 0 || a >= 8 || b < 0 || b >= 8)
		return DFG_ERR_ARG;
	CK(cudaSetDevice(ctx->device));
	CK(cudaEventSynchronize(ctx->user_ev[b]));
	float f = 0.f;
	CK(cudaEventElapsedTime(&f, ctx->user_ev[a], ctx->user_ev[b]));
	*ms = f;
	return DFG_OK;
}

extern "C" int dfg_get_workload(dfg_ctx *ctx, long long *out) {
	if (!ctx || !out)
		return DFG_ERR_ARG;
	long long ms = 0;
	for (auto &c : ctx->chunks)
		ms += c.entries;
	out[0] = ctx->R;
	out[1] = ctx->N;
	out[2] = ctx->n_ph;
	out[3] = ms;
	out[4] = (long long)ctx->chunks.size();
	out[5] = ctx->chunk_frames;
	out[6] = ctx->launches;
	out[7] = ctx->K_pad;
	out[8] = (ctx->dense_active ? 1 : 0) | (ctx->m_dense_active ? 2 : 0);
	out[9] = ctx->last_pairs ? ctx->npairs : 0;
	out[10] = ctx->last_pairs ? ctx->blk_tiles : 0;
	return DFG_OK;
}
