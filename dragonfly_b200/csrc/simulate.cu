// Frame simulator on the GPU: Poisson photon frames from slices of an
// intensity model, in the sparse .emc layout.
//
// The reference simulates data on the CPU (dragonfly/utils/src/make_data.c:
// gen_and_save_dataset 115-326: a slice at a random orientation times the
// frame's scale, a Poisson count per pixel with mask <= 1, frames written as
// ones / multi / place_ones / place_multi / count_multi). This kernel does the
// same per frame, one block per frame; random numbers come from a counter-based
// Philox stream keyed by (seed, frame, pixel), so the counting pass and the
// writing pass draw identical counts. Pixels are visited in ascending order,
// so place_ones / place_multi are sorted inside each frame like the
// reference writer's np.where (dragonfly/emcfile.pyx:395-397).

#include <curand_kernel.h>

#include "emc_ctx.cuh"

namespace dfg {

template <bool WRITE>
__global__ void __launch_bounds__(256) simulate_kernel(
    const double *__restrict__ quats4, const double *__restrict__ phi, const double *__restrict__ qvals,
    const double *__restrict__ corr, const uint8_t *__restrict__ mask, int P, const double *__restrict__ intens,
    long long S, unsigned long long seed, int *__restrict__ ones, int *__restrict__ multi,
    const long long *__restrict__ ones_off, const long long *__restrict__ multi_off, int *__restrict__ place_ones,
    int *__restrict__ place_multi, int *__restrict__ count_multi) {
	__shared__ double s_rot[9];
	__shared__ int s_w1[8], s_wm[8];
	__shared__ int s_base[2];
	const int d = blockIdx.x, t = threadIdx.x, lane = t & 31, w = t >> 5;
	if (t == 0) {
		rot_from_quat(&quats4[4 * (size_t)d], s_rot);
		s_base[0] = s_base[1] = 0;
	}
	__syncthreads();
	const double f = phi[d], center = (double)(S / 2);
	const long long ob = WRITE ? ones_off[d] : 0, mb = WRITE ? multi_off[d] : 0;
	for (int p0 = 0; p0 < P; p0 += 256) {
		const int p = p0 + t;
		unsigned c = 0;
		if (p < P && mask[p] <= 1) {
			Cell cell = locate(s_rot, qvals[3 * (size_t)p], qvals[3 * (size_t)p + 1], qvals[3 * (size_t)p + 2],
			                   center, S);
			double lam = cell.ok ? f * interp(cell, intens, S, corr[p]) : 0.;
			if (lam > 0.) {
				curandStatePhilox4_32_10_t st;
				curand_init(seed, (unsigned long long)d * (unsigned long long)P + p, 0, &st);
				c = curand_poisson(&st, lam);
			}
		}
		const unsigned b1 = __ballot_sync(FULL, c == 1), bm = __ballot_sync(FULL, c > 1);
		const unsigned below = (1u << lane) - 1u;
		if (lane == 0) {
			s_w1[w] = __popc(b1);
			s_wm[w] = __popc(bm);
		}
		__syncthreads();
		int o1 = s_base[0], om = s_base[1];
		for (int k = 0; k < w; ++k) {
			o1 += s_w1[k];
			om += s_wm[k];
		}
		if (WRITE) {
			if (c == 1)
				place_ones[ob + o1 + __popc(b1 & below)] = p;
			else if (c > 1) {
				long long i = mb + om + __popc(bm & below);
				place_multi[i] = p;
				count_multi[i] = (int)c;
			}
		}
		__syncthreads();
		if (t == 0) {
			int a = 0, b = 0;
			for (int k = 0; k < 8; ++k) {
				a += s_w1[k];
				b += s_wm[k];
			}
			s_base[0] += a;
			s_base[1] += b;
		}
		__syncthreads();
	}
	if (!WRITE && t == 0) {
		ones[d] = s_base[0];
		multi[d] = s_base[1];
	}
}

}  // namespace dfg

extern "C" int dfg_simulate_frames(dfg_ctx *ctx, long size, const double *intens, int num_data,
                                   const double *quats4, const double *phi, unsigned long long seed,
                                   long long *totals) {
	if (!ctx)
		return DFG_ERR_ARG;
	NEED(ctx->P > 0, DFG_ERR_STATE, "simulate: set the detector first");
	NEED(size >= 3 && intens && num_data > 0 && quats4 && phi, DFG_ERR_ARG, "simulate: bad arguments");
	for (int d = 0; d < num_data; ++d)
		NEED(std::isfinite(phi[d]) && phi[d] >= 0. && std::isfinite(quats4[4 * (size_t)d]), DFG_ERR_ARG,
		     "simulate: frame %d has a bad scale or orientation", d);
	CK(cudaSetDevice(ctx->device));
	cudaStream_t st = ctx->stream;
	const long long V = (long long)size * size * size;
	DevBuf<double> d_int, d_q, d_phi;
	DevBuf<int> d_ones, d_multi, d_po, d_pm, d_cm;
	DevBuf<long long> d_oo, d_mo;
	CK(upload(d_int, intens, (size_t)V, st));
	CK(upload(d_q, quats4, 4 * (size_t)num_data, st));
	CK(upload(d_phi, phi, (size_t)num_data, st));
	CK(d_ones.ensure((size_t)num_data));
	CK(d_multi.ensure((size_t)num_data));
	simulate_kernel<false><<<num_data, 256, 0, st>>>(d_q.p, d_phi.p, ctx->qvals.p, ctx->corr.p, ctx->mask.p, ctx->P,
	                                                 d_int.p, size, seed, d_ones.p, d_multi.p, nullptr, nullptr,
	                                                 nullptr, nullptr, nullptr);
	CKL("simulate_kernel<count>");
	std::vector<int> ones(num_data), multi(num_data);
	CK(cudaMemcpyAsync(ones.data(), d_ones.p, num_data * sizeof(int), cudaMemcpyDeviceToHost, st));
	CK(cudaMemcpyAsync(multi.data(), d_multi.p, num_data * sizeof(int), cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	std::vector<long long> oo(num_data + 1, 0), mo(num_data + 1, 0);
	for (int d = 0; d < num_data; ++d) {
		oo[d + 1] = oo[d] + ones[d];
		mo[d + 1] = mo[d] + multi[d];
	}
	CK(upload(d_oo, oo.data(), oo.size(), st));
	CK(upload(d_mo, mo.data(), mo.size(), st));
	CK(d_po.ensure((size_t)oo[num_data]));
	CK(d_pm.ensure((size_t)mo[num_data]));
	CK(d_cm.ensure((size_t)mo[num_data]));
	simulate_kernel<true><<<num_data, 256, 0, st>>>(d_q.p, d_phi.p, ctx->qvals.p, ctx->corr.p, ctx->mask.p, ctx->P,
	                                                d_int.p, size, seed, nullptr, nullptr, d_oo.p, d_mo.p, d_po.p,
	                                                d_pm.p, d_cm.p);
	CKL("simulate_kernel<write>");
	std::vector<int> po((size_t)oo[num_data]), pm((size_t)mo[num_data]), cm((size_t)mo[num_data]);
	CK(cudaMemcpyAsync(po.data(), d_po.p, po.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
	CK(cudaMemcpyAsync(pm.data(), d_pm.p, pm.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
	CK(cudaMemcpyAsync(cm.data(), d_cm.p, cm.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	long long photons = oo[num_data];
	for (int c : cm)
		photons += c;
	if (totals) {
		totals[0] = oo[num_data];
		totals[1] = mo[num_data];
		totals[2] = photons;
	}
	return dfg_set_frames(ctx, num_data, ones.data(), multi.data(), po.data(), pm.data(), cm.data());
}

extern "C" int dfg_get_frames(dfg_ctx *ctx, int *ones, int *multi, int *place_ones, int *place_multi,
                              int *count_multi) {
	if (!ctx)
		return DFG_ERR_ARG;
	NEED(ctx->N > 0, DFG_ERR_STATE, "no frames set");
	auto cp = [](int *dst, const std::vector<int> &src) {
		if (dst && !src.empty())
			memcpy(dst, src.data(), src.size() * sizeof(int));
	};
	cp(ones, ctx->h_ones);
	cp(multi, ctx->h_multi);
	cp(place_ones, ctx->h_place_ones);
	cp(place_multi, ctx->h_place_multi);
	cp(count_multi, ctx->h_count_multi);
	return DFG_OK;
}

// ---------------------------------------------------------------------------
// .emc files (binary): a 1024-byte header of int32 num_data, num_pix, ftype,
// then for ftype 0 (sparse) int32 ones[num_data], multi[num_data],
// place_ones[], place_multi[], count_multi[] (emcfile.c:3-57,
// emcfile.pyx:491-532); for ftype 1 int32 frames [num_data][num_pix].
// ---------------------------------------------------------------------------
extern "C" int dfg_load_emc(dfg_ctx *ctx, int num_files, const char *const *paths) {
	if (!ctx || num_files < 1 || !paths)
		return DFG_ERR_ARG;
	NEED(ctx->P > 0, DFG_ERR_STATE, "load_emc: set the detector first");
	std::vector<int> ones, multi, po, pm, cm;
	for (int f = 0; f < num_files; ++f) {
		FILE *fp = fopen(paths[f], "rb");
		NEED(fp != nullptr, DFG_ERR_ARG, "load_emc: cannot open %s", paths[f]);
		int hdr[3] = {0, 0, -1};
		bool ok = fread(hdr, sizeof(int), 3, fp) == 3 && fseek(fp, 1024, SEEK_SET) == 0;
		const int nd = hdr[0], npx = hdr[1], ftype = hdr[2];
		if (!ok || nd < 0 || npx != ctx->P || (ftype != 0 && ftype != 1)) {
			fclose(fp);
			return ctx->fail(DFG_ERR_ARG,
			                 "load_emc: %s: %d frames x %d pixels, type %d (need %d pixels, type 0 sparse or 1 "
			                 "dense integer)",
			                 paths[f], nd, npx, ftype, ctx->P);
		}
		auto rd = [&](std::vector<int> &v, size_t n) {
			const size_t o = v.size();
			v.resize(o + n);
			return n == 0 || fread(v.data() + o, sizeof(int), n, fp) == n;
		};
		if (ftype == 0) {
			const size_t o0 = ones.size(), m0 = multi.size();
			ok = rd(ones, (size_t)nd) && rd(multi, (size_t)nd);
			long long so = 0, sm = 0;
			for (int d = 0; ok && d < nd; ++d) {
				so += ones[o0 + d];
				sm += multi[m0 + d];
			}
			ok = ok && rd(po, (size_t)so) && rd(pm, (size_t)sm) && rd(cm, (size_t)sm);
		} else {
			// dense integer frames become sparse (count 1 -> ones, > 1 -> multi)
			std::vector<int> fr((size_t)npx);
			for (int d = 0; ok && d < nd; ++d) {
				ok = fread(fr.data(), sizeof(int), (size_t)npx, fp) == (size_t)npx;
				int n1 = 0, nm = 0;
				for (int t = 0; ok && t < npx; ++t) {
					if (fr[t] == 1) {
						po.push_back(t);
						n1++;
					} else if (fr[t] > 1) {
						pm.push_back(t);
						cm.push_back(fr[t]);
						nm++;
					}
				}
				ones.push_back(n1);
				multi.push_back(nm);
			}
		}
		fclose(fp);
		NEED(ok, DFG_ERR_ARG, "load_emc: %s is truncated", paths[f]);
	}
	NEED(!ones.empty(), DFG_ERR_ARG, "load_emc: no frames");
	return dfg_set_frames(ctx, (int)ones.size(), ones.data(), multi.data(), po.data(), pm.data(), cm.data());
}

extern "C" int dfg_save_emc(dfg_ctx *ctx, const char *path) {
	if (!ctx || !path)
		return DFG_ERR_ARG;
	NEED(ctx->N > 0, DFG_ERR_STATE, "save_emc: no frames set");
	FILE *fp = fopen(path, "wb");
	NEED(fp != nullptr, DFG_ERR_ARG, "save_emc: cannot create %s", path);
	std::vector<char> hdr(1024, 0);
	const int h[3] = {ctx->N, ctx->P, 0};
	memcpy(hdr.data(), h, sizeof(h));
	auto wr = [&](const void *p, size_t bytes) { return bytes == 0 || fwrite(p, 1, bytes, fp) == bytes; };
	const bool ok = wr(hdr.data(), hdr.size()) && wr(ctx->h_ones.data(), ctx->h_ones.size() * sizeof(int)) &&
	                wr(ctx->h_multi.data(), ctx->h_multi.size() * sizeof(int)) &&
	                wr(ctx->h_place_ones.data(), ctx->h_place_ones.size() * sizeof(int)) &&
	                wr(ctx->h_place_multi.data(), ctx->h_place_multi.size() * sizeof(int)) &&
	                wr(ctx->h_count_multi.data(), ctx->h_count_multi.size() * sizeof(int));
	const bool closed = fclose(fp) == 0;
	NEED(ok && closed, DFG_ERR_ARG, "save_emc: writing %s failed", path);
	return DFG_OK;
}
