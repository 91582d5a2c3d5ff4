// Slice generation without device allocation.
//
// dfg_slice_gen (emc_api.cu) allocates two small device buffers per call (the
// quaternion and the output slice). Some callers cannot allow that: an
// application that has handed its whole device memory budget to its own pool
// allocator and forbids other allocations once it is running, or a real-time
// loop where a cudaMalloc / cudaFree (which synchronise the device) would
// stall other streams. dfg_slice_gen_noalloc serves them: its scratch is one
// file-scope device array, sized for at most DFG_NOALLOC_MAX_PIXELS pixels,
// that every GPU loading this library holds until the process exits.
//
// In host code the array's name only stands for it; its device address comes
// from cudaGetSymbolAddress, looked up once per device with that device
// current, on the first call on that device (make that first call before any
// stream capture), and kept for the life of the process: the entry point must
// not be used across a cudaDeviceReset (or another teardown of the device's
// primary context) in the host process, after which the kept address would
// point into freed memory. All calls share the array: calls that overlap on the GPU
// (other threads, other contexts on the same device) race and must be
// serialised by the caller. Every call writes the quaternion slots and all
// num_pix output slots before reading them, so nothing has to be cleared.

#include <mutex>

#include "emc_ctx.cuh"

namespace {

constexpr int kQuatSlots = 8;  // quaternion (5 doubles), padded to 64 bytes
static __device__ __align__(256) double g_slice_scratch[kQuatSlots + DFG_NOALLOC_MAX_PIXELS];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_lock;
double *g_scratch_addr[kMaxDevices] = {};

// The device address of g_slice_scratch on the current device (looked up once).
cudaError_t scratch_address(int device, double **out) {
	std::lock_guard<std::mutex> guard(g_scratch_lock);
	if (g_scratch_addr[device] == nullptr) {
		void *p = nullptr;
		cudaError_t e = cudaGetSymbolAddress(&p, g_slice_scratch);
		if (e != cudaSuccess)
			return e;
		g_scratch_addr[device] = static_cast<double *>(p);
	}
	*out = g_scratch_addr[device];
	return cudaSuccess;
}

// slice_one_kernel of emc_api.cu with the quaternion read from, and the slice
// written to, the scratch array (which device code names directly).
__global__ void slice_one_scratch_kernel(int mode, const double *__restrict__ qvals,
                                         const double *__restrict__ corr, int P, const double *__restrict__ model,
                                         long long S, long long V) {
	int p = blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= P)
		return;
	double rot[9];
	rot_from_quat(g_slice_scratch, rot);
	Cell c = locate(rot, qvals[3 * (size_t)p], qvals[3 * (size_t)p + 1], qvals[3 * (size_t)p + 2],
	                (double)(S / 2), S);
	g_slice_scratch[kQuatSlots + p] = interp(c, model + (size_t)mode * V, S, corr[p]);
}

}  // namespace

extern "C" int dfg_slice_gen_noalloc(dfg_ctx *ctx, const double *quat, int mode, double *out) {
	if (!ctx || !quat || !out)
		return DFG_ERR_ARG;
	NEED(ctx->P > 0 && ctx->S > 0, DFG_ERR_STATE, "slice_gen_noalloc: detector and model must be set");
	NEED(mode >= 0 && mode < ctx->M, DFG_ERR_ARG, "slice_gen_noalloc: mode %d out of range", mode);
	NEED(ctx->model_type == MT_3D, DFG_ERR_ARG, "slice_gen_noalloc: 3-D models only");
	NEED(ctx->P <= DFG_NOALLOC_MAX_PIXELS, DFG_ERR_ARG,
	     "slice_gen_noalloc: the detector has %d pixels, more than the maximum of %d", ctx->P,
	     DFG_NOALLOC_MAX_PIXELS);
	NEED(ctx->device >= 0 && ctx->device < kMaxDevices, DFG_ERR_ARG, "slice_gen_noalloc: device %d unsupported",
	     ctx->device);
	CK(cudaSetDevice(ctx->device));
	double *scratch = nullptr;
	CK(scratch_address(ctx->device, &scratch));
	cudaStream_t st = ctx->stream;
	CK(cudaMemcpyAsync(scratch, quat, 5 * sizeof(double), cudaMemcpyHostToDevice, st));
	slice_one_scratch_kernel<<<(ctx->P + 255) / 256, 256, 0, st>>>(mode, ctx->qvals.p, ctx->corr.p, ctx->P,
	                                                                ctx->model1.p, ctx->S, ctx->V);
	CKL("slice_one_scratch_kernel");
	CK(cudaMemcpyAsync(out, scratch + kQuatSlots, (size_t)ctx->P * sizeof(double), cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	return DFG_OK;
}
