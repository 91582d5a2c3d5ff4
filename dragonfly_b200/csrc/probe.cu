// Gather-rate probe: the ceiling of the access pattern of the E-step and
// M-step gathers, measured on the device the context runs on.
//
// Both gather kernels read, per photon entry, one 512-byte row (128 FP32
// orientations or probabilities, a 16-byte load per lane) of a table that
// stays resident in L2 while the warps of one orientation tile run: the
// log-slice tile [P + 1][128] (34 MB on the 66820-pixel detector) or the
// probability tile [Nc + 1][128]. The rows are served by L2 and L1, not by
// HBM, so the copy bandwidth of HBM is not their roofline. This probe reads
// uniformly random rows of a table of the same size with nothing else to do
// (row indices from a register hash, eight rows in flight per lane, full
// occupancy), which bounds what any kernel with this access pattern can
// reach on the device.

#include "emc_ctx.cuh"

namespace {

constexpr int kProbeRowsInFlight = 8;
constexpr int kProbeSteps = 1024;       // groups of 8 rows per warp
constexpr int kProbeBlocksPerSM = 8;    // 8 x 256 threads: the SM's 2048-thread limit

__global__ void probe_fill_kernel(float4 *__restrict__ buf, long long n) {
	const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
		buf[i] = make_float4(1.f, 0.5f, 0.25f, 0.125f);
}

__device__ __forceinline__ unsigned probe_hash(unsigned x) {
	x ^= x >> 16;
	x *= 0x7feb352du;
	x ^= x >> 15;
	x *= 0x846ca68bu;
	x ^= x >> 16;
	return x;
}

// Each warp reads kProbeSteps x 8 rows; all lanes of a warp compute the same
// row index (the hash depends on the warp only), each lane loads its 16 bytes.
__global__ void __launch_bounds__(256) probe_gather_kernel(const float4 *__restrict__ buf, unsigned rows,
                                                           unsigned seed, float *__restrict__ sink) {
	const unsigned warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	unsigned x = probe_hash(warp * 0x9e3779b9u ^ seed);
	float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
	for (int i = 0; i < kProbeSteps; ++i) {
		float4 v[kProbeRowsInFlight];
#pragma unroll
		for (int q = 0; q < kProbeRowsInFlight; ++q) {
			x = x * 1664525u + 1013904223u;
			const unsigned row = __umulhi(probe_hash(x), rows);
			v[q] = __ldg(buf + (size_t)row * 32 + lane);
		}
#pragma unroll
		for (int q = 0; q < kProbeRowsInFlight; ++q) {
			acc.x += v[q].x;
			acc.y += v[q].y;
			acc.z += v[q].z;
			acc.w += v[q].w;
		}
	}
	// never true for the fill values (keeps the loads live)
	if (acc.x + acc.y + acc.z + acc.w == -1.f)
		sink[warp * 32 + lane] = acc.x;
}

}  // namespace

extern "C" int dfg_measure_gather_rate(dfg_ctx *ctx, long long rows, int reps, double *gbs) {
	if (!ctx || !gbs)
		return DFG_ERR_ARG;
	NEED(rows >= 1 && rows <= (1LL << 26), DFG_ERR_ARG, "measure_gather_rate: rows %lld out of [1, 2^26]", rows);
	NEED(reps >= 1 && reps <= 100, DFG_ERR_ARG, "measure_gather_rate: reps %d out of [1, 100]", reps);
	CK(cudaSetDevice(ctx->device));
	cudaStream_t st = ctx->stream;
	const unsigned blocks = (unsigned)(ctx->num_sms * kProbeBlocksPerSM);
	const long long warps = (long long)blocks * 8;
	DevBuf<float4> buf;
	DevBuf<float> sink;
	CK(buf.ensure((size_t)rows * 32));
	CK(sink.ensure((size_t)warps * 32));
	probe_fill_kernel<<<blocks_for(rows * 32, 256), 256, 0, st>>>(buf.p, rows * 32);
	CKL("probe_fill_kernel");
	cudaEvent_t e0, e1;
	CK(cudaEventCreate(&e0));
	CK(cudaEventCreate(&e1));
	double best = 0.;
	cudaError_t err = cudaSuccess;
	for (int k = 0; k <= reps && err == cudaSuccess; ++k) {   // launch 0 warms up
		cudaEventRecord(e0, st);
		probe_gather_kernel<<<blocks, 256, 0, st>>>(buf.p, (unsigned)rows, 0x51ed27u + 977u * k, sink.p);
		ctx->launches++;
		err = cudaGetLastError();
		cudaEventRecord(e1, st);
		if (err == cudaSuccess)
			err = cudaEventSynchronize(e1);
		float ms = 0.f;
		if (err == cudaSuccess)
			err = cudaEventElapsedTime(&ms, e0, e1);
		if (err == cudaSuccess && k > 0 && ms > 0.f)
			best = std::max(best, (double)warps * kProbeSteps * kProbeRowsInFlight * 512. / (ms * 1e-3) / 1e9);
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	CK(err);
	*gbs = best;
	return DFG_OK;
}
