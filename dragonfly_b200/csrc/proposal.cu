// Learned orientation proposals: a small convolutional network that maps a
// frame's binned photon image to logits over the coarse orientations, trained
// and evaluated on the GPU by the kernels below (BF16 weights for the
// products, FP32 activations, accumulation and optimiser state).
//
// Network (NHWC activations, batch B):
//   image [B][32][32][1] = log(1 + photons binned on a 32 x 32 grid of q)
//   conv1 3x3 stride 1 -> [B][32][32][32], ReLU
//   conv2 3x3 stride 2 -> [B][16][16][32], ReLU
//   conv3 3x3 stride 1 -> [B][16][16][64], ReLU
//   conv4 3x3 stride 2 -> [B][8][8][64],  ReLU   (= [B][4096])
//   fc1 4096 -> 256, ReLU
//   fc2 256 -> num_classes (logits)
// Convolutions are products of im2col matrices [B*Ho*Wo][9*C] with the
// weights [Cout][9*C] (rows ordered ky, kx, c); the backward pass forms the
// weight gradients as dY^T . cols, the input gradients as dY . W followed by a
// gather (col2im, deterministic). Loss: softmax cross-entropy against a class
// label per frame. Optimiser: Adam on FP32 master weights, BF16 copies for the
// products. No counterpart in the reference (its E-step searches every
// orientation).
#include <cuda_bf16.h>

#include <cmath>
#include <random>

#include <cudaTypedefs.h>

#include "emc_ctx.cuh"
#include "tcgen05.cuh"

namespace {

constexpr int IMG = 32;  // image side
constexpr int NL = 6;    // layers

struct LayerShape {
	int kind;  // 0 conv 3x3, 1 fully connected
	int cin, cout, hin, stride, hout;
	int fan_in() const { return kind == 0 ? 9 * cin : cin; }
	long long nw() const { return (long long)cout * fan_in(); }
};

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ float to_f(T x);
template <>
__device__ __forceinline__ float to_f<float>(float x) {
	return x;
}
template <>
__device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 x) {
	return __bfloat162float(x);
}

// C[M][N] = alpha * op(A) op(B) + beta * C, op(A) [M][K], op(B) [K][N]; A is
// stored [M][K] (or [K][M] with TA), B [K][N] (or [N][K] with TB). 64 x 64
// tiles, 16-deep k steps through shared memory, 4 x 4 outputs per thread,
// FP32 accumulation. Split k: block z covers k in [z kchunk, (z + 1) kchunk)
// and writes its partial product to C + z cstride.
template <typename TAe, typename TBe, bool TA, bool TB>
__global__ void __launch_bounds__(256) gemm_kernel(int M, int N, int K, float alpha, const TAe *__restrict__ A,
                                                   int lda, const TBe *__restrict__ B, int ldb, float beta,
                                                   float *__restrict__ C, int ldc, int kchunk, long long cstride) {
	__shared__ float As[16][64 + 4], Bs[16][64 + 4];
	const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
	const int i0 = blockIdx.y * 64, j0 = blockIdx.x * 64;
	const int kb = blockIdx.z * kchunk, ke = min(K, kb + kchunk);
	C += blockIdx.z * cstride;
	float acc[4][4] = {};
	for (int k0 = kb; k0 < ke; k0 += 16) {
		// consecutive threads read consecutive addresses: along k for A
		// [M][K] and B^T [N][K], along the 64-wide tile for A^T and B
		for (int e = t; e < 64 * 16; e += 256) {
			const int r = TA ? (e & 63) : (e >> 4), kk = TA ? (e >> 6) : (e & 15);
			const int i = i0 + r, k = k0 + kk;
			float a = 0.f;
			if (i < M && k < ke)
				a = to_f(TA ? A[(size_t)k * lda + i] : A[(size_t)i * lda + k]);
			As[kk][r] = a;
		}
		for (int e = t; e < 64 * 16; e += 256) {
			const int r = TB ? (e >> 4) : (e & 63), kk = TB ? (e & 15) : (e >> 6);
			const int j = j0 + r, k = k0 + kk;
			float b = 0.f;
			if (j < N && k < ke)
				b = to_f(TB ? B[(size_t)j * ldb + k] : B[(size_t)k * ldb + j]);
			Bs[kk][r] = b;
		}
		__syncthreads();
#pragma unroll
		for (int kk = 0; kk < 16; ++kk) {
			float a[4], b[4];
#pragma unroll
			for (int q = 0; q < 4; ++q) {
				a[q] = As[kk][ty * 4 + q];
				b[q] = Bs[kk][tx * 4 + q];
			}
#pragma unroll
			for (int p = 0; p < 4; ++p)
#pragma unroll
				for (int q = 0; q < 4; ++q)
					acc[p][q] = fmaf(a[p], b[q], acc[p][q]);
		}
		__syncthreads();
	}
#pragma unroll
	for (int p = 0; p < 4; ++p) {
		const int i = i0 + ty * 4 + p;
		if (i >= M)
			continue;
#pragma unroll
		for (int q = 0; q < 4; ++q) {
			const int j = j0 + tx * 4 + q;
			if (j >= N)
				continue;
			float *c = C + (size_t)i * ldc + j;
			*c = alpha * acc[p][q] + (beta != 0.f ? beta * *c : 0.f);
		}
	}
}

// cols[(b, ho, wo)][(ky, kx, c)] = X[b][ho s + ky - 1][wo s + kx - 1][c]
// (zero outside the image).
__global__ void im2col_kernel(const float *__restrict__ X, int B, int H, int C, int s, int Ho,
                              float *__restrict__ cols) {
	const long long n = (long long)B * Ho * Ho * 9 * C;
	for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
		const int c = (int)(e % C);
		long long r = e / C;
		const int kx = (int)(r % 3);
		r /= 3;
		const int ky = (int)(r % 3);
		r /= 3;
		const int wo = (int)(r % Ho);
		r /= Ho;
		const int ho = (int)(r % Ho);
		const int b = (int)(r / Ho);
		const int y = ho * s + ky - 1, x = wo * s + kx - 1;
		cols[e] = (y >= 0 && y < H && x >= 0 && x < H) ? X[(((size_t)b * H + y) * H + x) * C + c] : 0.f;
	}
}

// dX[b][y][x][c] = sum of dcols over the (ho, wo, ky, kx) that read it.
// col2im_kernel for C a multiple of 4 and stride S (1 or 2): four channels
// per thread (16-byte loads and stores), the taps added in the same order.
template <int S>
__global__ void col2im4_kernel(const float *__restrict__ dcols, int B, int H, int C, int Ho,
                               float *__restrict__ dX) {
	const unsigned C4 = (unsigned)C >> 2;
	const unsigned n = (unsigned)B * H * H * C4;
	for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
		const unsigned c4 = e % C4;
		unsigned r = e / C4;
		const int x = (int)(r % (unsigned)H);
		r /= (unsigned)H;
		const int y = (int)(r % (unsigned)H);
		const int b = (int)(r / (unsigned)H);
		float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
		for (int ky = 0; ky < 3; ++ky) {
			const int yy = y + 1 - ky;
			if (yy < 0 || (S == 2 && (yy & 1)))
				continue;
			const int ho = yy / S;
			if (ho >= Ho)
				continue;
			for (int kx = 0; kx < 3; ++kx) {
				const int xx = x + 1 - kx;
				if (xx < 0 || (S == 2 && (xx & 1)))
					continue;
				const int wo = xx / S;
				if (wo >= Ho)
					continue;
				const float4 v = *reinterpret_cast<const float4 *>(
				    dcols + ((((size_t)b * Ho + ho) * Ho + wo) * 9 + ky * 3 + kx) * C + 4 * c4);
				acc.x += v.x;
				acc.y += v.y;
				acc.z += v.z;
				acc.w += v.w;
			}
		}
		*reinterpret_cast<float4 *>(dX + (size_t)e * 4) = acc;
	}
}

__global__ void col2im_kernel(const float *__restrict__ dcols, int B, int H, int C, int s, int Ho,
                              float *__restrict__ dX) {
	// 32-bit index arithmetic (B H H C < 2^31 for every layer and batch)
	const unsigned n = (unsigned)B * H * H * C;
	for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
		const int c = (int)(e % (unsigned)C);
		unsigned r = e / (unsigned)C;
		const int x = (int)(r % (unsigned)H);
		r /= (unsigned)H;
		const int y = (int)(r % (unsigned)H);
		const int b = (int)(r / (unsigned)H);
		float acc = 0.f;
		for (int ky = 0; ky < 3; ++ky) {
			const int yy = y + 1 - ky;
			if (yy < 0 || yy % s)
				continue;
			const int ho = yy / s;
			if (ho >= Ho)
				continue;
			for (int kx = 0; kx < 3; ++kx) {
				const int xx = x + 1 - kx;
				if (xx < 0 || xx % s)
					continue;
				const int wo = xx / s;
				if (wo >= Ho)
					continue;
				acc += dcols[((((size_t)b * Ho + ho) * Ho + wo) * 9 + ky * 3 + kx) * C + c];
			}
		}
		dX[e] = acc;
	}
}

// Y[r][c] += bias[c], then ReLU when relu.
__global__ void bias_act_kernel(float *__restrict__ Y, long long rows, int cols, const float *__restrict__ bias,
                                int relu) {
	const long long n = rows * cols;
	for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
		float v = Y[e] + bias[e % cols];
		Y[e] = relu ? fmaxf(v, 0.f) : v;
	}
}

// out[e] = sum over z of part[z n + e]: block (32, 8) per 32 elements, row y
// of the block adds the splits y, y + 8, ... in order and the 8 rows are
// added in order (deterministic; the 8 rows keep loads in flight when S is
// large and n small).
__global__ void __launch_bounds__(256) sum_splits_kernel(const float *__restrict__ part, int S, long long n,
                                                         float *__restrict__ out) {
	__shared__ float s[8][32];
	const long long e = (long long)blockIdx.x * 32 + threadIdx.x;
	float acc = 0.f;
	if (e < n)
		for (int z = threadIdx.y; z < S; z += 8)
			acc += part[z * n + e];
	s[threadIdx.y][threadIdx.x] = acc;
	__syncthreads();
	if (threadIdx.y == 0 && e < n) {
		float t = 0.f;
#pragma unroll
		for (int k = 0; k < 8; ++k)
			t += s[k][threadIdx.x];
		out[e] = t;
	}
}

// *acc += sum of loss[0, n) (one block, fixed-order tree).
__global__ void __launch_bounds__(256) loss_sum_kernel(const float *__restrict__ loss, int n, double *__restrict__ acc) {
	__shared__ double s[256];
	double v = 0.;
	for (int k = threadIdx.x; k < n; k += 256)
		v += loss[k];
	s[threadIdx.x] = v;
	__syncthreads();
	for (int h = 128; h > 0; h >>= 1) {
		if (threadIdx.x < h)
			s[threadIdx.x] += s[threadIdx.x + h];
		__syncthreads();
	}
	if (threadIdx.x == 0)
		*acc += s[0];
}

// dY *= (Y > 0) (ReLU backward, Y the forward output).
__global__ void relu_back_kernel(float *__restrict__ dY, const float *__restrict__ Y, long long n) {
	for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
		if (!(Y[e] > 0.f))
			dY[e] = 0.f;
}

// db[c] = sum_r dY[r][c]: one block per column, a fixed-order tree over
// per-thread strided partial sums.
// Column sums of dY [rows][cols] (bias gradients), first stage: block b adds
// its rows [b chunk, (b + 1) chunk) into part[b][cols]. With cols dividing
// 256, thread t keeps column t % cols and every (256 / cols)-th row from
// t / cols on, so each step reads 256 consecutive floats (coalesced); the
// threads of a column are then added in thread order. Otherwise thread t
// keeps columns t, t + 256, ... over all the block's rows. Fixed order
// throughout: the sums are deterministic.
__global__ void __launch_bounds__(256) colsum_part_kernel(const float *__restrict__ dY, long long rows, int cols,
                                                          long long chunk, float *__restrict__ part) {
	__shared__ float s[256];
	const long long r0 = (long long)blockIdx.x * chunk, r1 = min(rows, r0 + chunk);
	float *out = part + (size_t)blockIdx.x * cols;
	if (256 % cols == 0) {
		const int c = threadIdx.x % cols, j = threadIdx.x / cols, step = 256 / cols;
		float acc = 0.f;
		for (long long r = r0 + j; r < r1; r += step)
			acc += dY[r * cols + c];
		s[threadIdx.x] = acc;
		__syncthreads();
		if (threadIdx.x < cols) {
			float t = 0.f;
			for (int k = 0; k < step; ++k)
				t += s[k * cols + threadIdx.x];
			out[threadIdx.x] = t;
		}
	} else {
		for (int c = threadIdx.x; c < cols; c += 256) {
			float acc = 0.f;
			for (long long r = r0; r < r1; ++r)
				acc += dY[r * cols + c];
			out[c] = acc;
		}
	}
}

// out[c] = sum over b < nb of part[b][c], b in order.
__global__ void colsum_final_kernel(const float *__restrict__ part, int nb, int cols, float *__restrict__ out) {
	const int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= cols)
		return;
	float t = 0.f;
	for (int b = 0; b < nb; ++b)
		t += part[(size_t)b * cols + c];
	out[c] = t;
}

// Layer 0's weight and bias gradients (cout 32, K = 9 taps of one channel),
// first stage: block b takes rows [b chunk, (b + 1) chunk) of dY [rows][32]
// and the FP32 im2col rows X [rows][9]; thread t keeps output channel t % 32
// over every 8th row from t / 32 on (each step reads 256 consecutive floats
// of dY; the 9 taps of a row are read by the 32 threads of its channel group
// from the same 36 bytes). part[b][c][0 .. 8] = weight sums, [9] = bias sum,
// the 8 row phases added in order.
__global__ void __launch_bounds__(256) wgrad0_part_kernel(const float *__restrict__ dY, const float *__restrict__ X,
                                                          long long rows, long long chunk, float *__restrict__ part) {
	__shared__ float s[8][32][10];
	const int c = threadIdx.x & 31, j = threadIdx.x >> 5;
	const long long r0 = (long long)blockIdx.x * chunk, r1 = min(rows, r0 + chunk);
	float acc[10];
#pragma unroll
	for (int k = 0; k < 10; ++k)
		acc[k] = 0.f;
	for (long long r = r0 + j; r < r1; r += 8) {
		const float g = dY[r * 32 + c];
		const float *x = X + r * 9;
#pragma unroll
		for (int k = 0; k < 9; ++k)
			acc[k] += g * x[k];
		acc[9] += g;
	}
#pragma unroll
	for (int k = 0; k < 10; ++k)
		s[j][c][k] = acc[k];
	__syncthreads();
	for (int e = threadIdx.x; e < 320; e += 256) {
		const int cc = e / 10, k = e % 10;
		float t = 0.f;
		for (int jj = 0; jj < 8; ++jj)
			t += s[jj][cc][k];
		part[(size_t)blockIdx.x * 320 + e] = t;
	}
}

// Second stage: gw[c][k] and gb[c] from the blocks' partial sums, in block order.
__global__ void wgrad0_final_kernel(const float *__restrict__ part, int nb, float *__restrict__ gw,
                                    float *__restrict__ gb) {
	const int e = threadIdx.x;  // c * 10 + k
	if (e >= 320)
		return;
	float t = 0.f;
	for (int b = 0; b < nb; ++b)
		t += part[(size_t)b * 320 + e];
	const int c = e / 10, k = e % 10;
	if (k < 9)
		gw[c * 9 + k] = t;
	else
		gb[c] = t;
}

// Softmax cross-entropy per row (one warp per row): loss[b] =
// logsumexp(z) - z[label]; dz = (softmax(z) - onehot) / B.
__global__ void softmax_xent_kernel(const float *__restrict__ z, const int *__restrict__ label, int B, int n,
                                    float *__restrict__ dz, float *__restrict__ loss) {
	const int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
	if (b >= B)
		return;
	const float *r = z + (size_t)b * n;
	float m = -INFINITY;
	for (int j = lane; j < n; j += 32)
		m = fmaxf(m, r[j]);
	for (int o = 16; o > 0; o >>= 1)
		m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
	float s = 0.f;
	for (int j = lane; j < n; j += 32)
		s += expf(r[j] - m);
	for (int o = 16; o > 0; o >>= 1)
		s += __shfl_xor_sync(FULL, s, o);
	const int y = label[b];
	for (int j = lane; j < n; j += 32)
		dz[(size_t)b * n + j] = (expf(r[j] - m) / s - (j == y ? 1.f : 0.f)) / (float)B;
	if (lane == 0)
		loss[b] = logf(s) + m - r[y];
}

// Softmax cross-entropy against a target distribution per row (one warp per
// row): row b is image img[b], whose targets are classes t_cls[t_off[img] ..
// t_off[img + 1]) with weights t_w (distinct classes, weights summing to 1):
// loss[b] = logsumexp(z) - sum_t w_t z[c_t]; dz = (softmax(z) - q) / B.
__global__ void softmax_xent_soft_kernel(const float *__restrict__ z, const int *__restrict__ img,
                                         const long long *__restrict__ t_off, const int *__restrict__ t_cls,
                                         const float *__restrict__ t_w, int B, int n, float *__restrict__ dz,
                                         float *__restrict__ loss) {
	const int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
	if (b >= B)
		return;
	const float *r = z + (size_t)b * n;
	float m = -INFINITY;
	for (int j = lane; j < n; j += 32)
		m = fmaxf(m, r[j]);
	for (int o = 16; o > 0; o >>= 1)
		m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
	float s = 0.f;
	for (int j = lane; j < n; j += 32)
		s += expf(r[j] - m);
	for (int o = 16; o > 0; o >>= 1)
		s += __shfl_xor_sync(FULL, s, o);
	for (int j = lane; j < n; j += 32)
		dz[(size_t)b * n + j] = expf(r[j] - m) / s / (float)B;
	__syncwarp();
	const long long t0 = t_off[img[b]], t1 = t_off[img[b] + 1];
	float zt = 0.f;
	for (long long t = t0 + lane; t < t1; t += 32) {
		const int c = t_cls[t];
		dz[(size_t)b * n + c] -= t_w[t] / (float)B;
		zt += t_w[t] * r[c];
	}
	for (int o = 16; o > 0; o >>= 1)
		zt += __shfl_xor_sync(FULL, zt, o);
	if (lane == 0)
		loss[b] = logf(s) + m - zt;
}

// Adam on FP32 master weights; the BF16 copy is refreshed.
__global__ void adam_kernel(float *__restrict__ w, float *__restrict__ m, float *__restrict__ v,
                            const float *__restrict__ g, __nv_bfloat16 *__restrict__ wb, long long n, float lr,
                            float b1, float b2, float c1, float c2, float eps) {
	for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
		const float gg = g[e];
		const float mm = b1 * m[e] + (1.f - b1) * gg, vv = b2 * v[e] + (1.f - b2) * gg * gg;
		m[e] = mm;
		v[e] = vv;
		const float ww = w[e] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
		w[e] = ww;
		if (wb)
			wb[e] = __float2bfloat16_rn(ww);
	}
}

__global__ void to_bf16_kernel(const float *__restrict__ x, __nv_bfloat16 *__restrict__ y, long long n) {
	for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
		y[e] = __float2bfloat16_rn(x[e]);
}

// Image of each frame: photons of its mask-0 pixels (the E-step lists) summed
// per bin (pixel_bin[p] in [0, 1024), -1 outside the grid), then log(1 + n).
// One block per frame; the image is built in shared memory.
__global__ void frame_image_kernel(const uint32_t *__restrict__ ph, const long long *__restrict__ ph_off,
                                   const long long *__restrict__ ph_mid, const int *__restrict__ pixel_bin, int P,
                                   int d0, int n, float *__restrict__ img) {
	__shared__ float s[IMG * IMG];
	const int dl = blockIdx.x, d = d0 + dl;
	if (dl >= n)
		return;
	for (int k = threadIdx.x; k < IMG * IMG; k += blockDim.x)
		s[k] = 0.f;
	__syncthreads();
	const long long beg = ph_off[d], mid = ph_mid[d], end = ph_off[d + 1];
	for (long long j = beg + threadIdx.x; j < end; j += blockDim.x) {
		const uint32_t w = ph[j];
		const uint32_t idx = j < mid ? w : (w & IDX_MASK);
		if (idx >= (uint32_t)P)
			continue;
		const int b = pixel_bin[idx];
		if (b >= 0)
			atomicAdd(&s[b], (float)(j < mid ? 1u : (w >> IDX_BITS)));
	}
	__syncthreads();
	for (int k = threadIdx.x; k < IMG * IMG; k += blockDim.x)
		img[(size_t)dl * IMG * IMG + k] = log1pf(s[k]);
}

// The largest logits of each row, in decreasing order (first index on ties;
// one warp per row, one warp-wide arg-max per pick): K_min picks, then more
// until the picks' softmax probabilities (over the whole row) sum to `mass`,
// at most K_max; unused slots of out [B][K_max] are -1. K_min = K_max gives
// the plain top-K.
__global__ void topk_kernel(const float *__restrict__ z, int B, int n, int K_min, int K_max, float mass,
                            int *__restrict__ out) {
	const int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
	if (b >= B)
		return;
	const float *r = z + (size_t)b * n;
	// softmax normaliser of the row: its maximum and sum of exp(z - max)
	float zmax = -INFINITY;
	for (int j = lane; j < n; j += 32)
		zmax = fmaxf(zmax, r[j]);
	for (int o = 16; o > 0; o >>= 1)
		zmax = fmaxf(zmax, __shfl_xor_sync(FULL, zmax, o));
	float den = 0.f;
	for (int j = lane; j < n; j += 32)
		den += __expf(r[j] - zmax);
	for (int o = 16; o > 0; o >>= 1)
		den += __shfl_xor_sync(FULL, den, o);
	float last = INFINITY, cum = 0.f;
	int last_i = -1;
	for (int k = 0; k < K_max; ++k) {
		if (k >= K_min && cum >= mass) {   // covered: the rest of the row stays out
			if (lane == 0)
				out[(size_t)b * K_max + k] = -1;
			continue;
		}
		float m = -INFINITY;
		int mi = n;
		for (int j = lane; j < n; j += 32) {
			const float v = r[j];
			// strictly after the previous pick in (value desc, index asc) order
			const bool after = v < last || (v == last && j > last_i);
			if (after && (v > m || (v == m && j < mi))) {
				m = v;
				mi = j;
			}
		}
		for (int o = 16; o > 0; o >>= 1) {
			const float om = __shfl_xor_sync(FULL, m, o);
			const int oi = __shfl_xor_sync(FULL, mi, o);
			if (om > m || (om == m && oi < mi)) {
				m = om;
				mi = oi;
			}
		}
		if (lane == 0)
			out[(size_t)b * K_max + k] = mi < n ? mi : -1;
		cum += mi < n ? __expf(m - zmax) / den : 0.f;
		last = m;
		last_i = mi;
	}
}

// Order-preserving key of a finite float (larger float, larger key); -0 and
// +0 share a key, as they compare equal.
__device__ __forceinline__ uint32_t order_key(float v) {
	const uint32_t b = v == 0.f ? 0u : __float_as_uint(v);
	return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// topk_kernel's picks for K_max <= SELK, one warp per row, without a row scan
// per pick: a radix select (four passes of 8 bits, a per-warp histogram in
// shared memory) finds the K_max-th largest key, the K_max largest entries
// (ties at the boundary by ascending index) are compacted into shared memory
// in index order, sorted by (value descending, index ascending) with a
// bitonic network, and the mass rule is applied to them in that order with
// topk_kernel's arithmetic, so the output is the same.
constexpr int SELK = 256;
__global__ void __launch_bounds__(256) topk_select_kernel(const float *__restrict__ z, int B, int n, int K_min,
                                                          int K_max, float mass, int *__restrict__ out) {
	__shared__ uint32_t s_hist[8][256];
	__shared__ uint32_t s_key[8][SELK];
	__shared__ int s_idx[8][SELK];
	const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int b = blockIdx.x * 8 + w;
	if (b >= B)
		return;
	const float *r = z + (size_t)b * n;
	uint32_t *hist = s_hist[w], *key = s_key[w];
	int *idx = s_idx[w];
	// softmax normaliser, as topk_kernel
	float zmax = -INFINITY;
	for (int j = lane; j < n; j += 32)
		zmax = fmaxf(zmax, r[j]);
	for (int o = 16; o > 0; o >>= 1)
		zmax = fmaxf(zmax, __shfl_xor_sync(FULL, zmax, o));
	float den = 0.f;
	for (int j = lane; j < n; j += 32)
		den += __expf(r[j] - zmax);
	for (int o = 16; o > 0; o >>= 1)
		den += __shfl_xor_sync(FULL, den, o);
	// radix select of the K_max-th largest key
	uint32_t prefix = 0;
	int need = K_max;
	for (int shift = 24; shift >= 0; shift -= 8) {
		for (int k = lane; k < 256; k += 32)
			hist[k] = 0;
		__syncwarp();
		const uint32_t hi_mask = shift == 24 ? 0u : (0xffffffffu << (shift + 8));
		for (int j = lane; j < n; j += 32) {
			const uint32_t u = order_key(r[j]);
			if ((u & hi_mask) == (prefix & hi_mask))
				atomicAdd(&hist[(u >> shift) & 255u], 1u);
		}
		__syncwarp();
		// lane L holds digits 255 - 8 L down to 248 - 8 L
		int lsum = 0;
#pragma unroll
		for (int q = 0; q < 8; ++q)
			lsum += (int)hist[255 - 8 * lane - q];
		int incl = lsum;
		for (int o = 1; o < 32; o <<= 1) {
			const int t = __shfl_up_sync(FULL, incl, o);
			if (lane >= o)
				incl += t;
		}
		const unsigned hit = __ballot_sync(FULL, incl >= need);
		const int src = __ffs(hit) - 1;  // need <= the group's count, so some lane crosses
		int d = 0, above = 0;
		if (lane == src) {
			int c = incl - lsum;
			for (int q = 0; q < 8; ++q) {
				const int dig = 255 - 8 * lane - q, h = (int)hist[dig];
				if (c + h >= need) {
					d = dig;
					above = c;
					break;
				}
				c += h;
			}
		}
		d = __shfl_sync(FULL, d, src);
		above = __shfl_sync(FULL, above, src);
		need -= above;
		prefix |= (uint32_t)d << shift;
		__syncwarp();
	}
	// the entries above the boundary key, and the first `need` at it by index,
	// compacted in index order
	int base = 0, ties = 0;
	for (int j0 = 0; j0 < n; j0 += 32) {
		const int j = j0 + lane;
		const uint32_t u = j < n ? order_key(r[j]) : 0u;
		const bool tie = j < n && u == prefix;
		const unsigned tm = __ballot_sync(FULL, tie);
		const int trank = ties + __popc(tm & ((1u << lane) - 1u));
		const bool sel = j < n && (u > prefix || (tie && trank < need));
		const unsigned sm = __ballot_sync(FULL, sel);
		if (sel) {
			const int pos = base + __popc(sm & ((1u << lane) - 1u));
			key[pos] = u;
			idx[pos] = j;
		}
		base += __popc(sm);
		ties += __popc(tm);
	}
	int P = 1;
	while (P < K_max)
		P <<= 1;
	for (int k = K_max + lane; k < P; k += 32) {  // pads sort last
		key[k] = 0u;
		idx[k] = 0x7fffffff;
	}
	__syncwarp();
	for (int k = 2; k <= P; k <<= 1)
		for (int jj = k >> 1; jj > 0; jj >>= 1) {
			for (int i = lane; i < P; i += 32) {
				const int ixj = i ^ jj;
				if (ixj > i) {
					const uint32_t ka = key[i], kb = key[ixj];
					const int ia = idx[i], ib = idx[ixj];
					const bool a_first = ka > kb || (ka == kb && ia < ib);
					if (((i & k) == 0) != a_first) {
						key[i] = kb;
						key[ixj] = ka;
						idx[i] = ib;
						idx[ixj] = ia;
					}
				}
			}
			__syncwarp();
		}
	if (lane == 0) {
		float cum = 0.f;
		for (int k = 0; k < K_max; ++k) {
			if (k >= K_min && cum >= mass) {
				out[(size_t)b * K_max + k] = -1;
				continue;
			}
			const int i = idx[k];
			out[(size_t)b * K_max + k] = i;
			cum += __expf(r[i] - zmax) / den;
		}
	}
}

// ---------------------------------------------------------------------------
// inference products on the tensor cores
// ---------------------------------------------------------------------------
constexpr int GK = 64;  // K per stage: one 128-byte swizzle row of BF16
constexpr int GSTAGES = 4;

template <int BN>
struct GemmCfg {
	static constexpr int A_BYTES = 128 * GK * 2;
	static constexpr int B_BYTES = BN * GK * 2;
	static constexpr int STAGE = A_BYTES + B_BYTES;
	static constexpr int SMEM = 1024 + GSTAGES * STAGE + 128;
	// kind::f16: FP32 accumulator, BF16 A and B, both K-major, N = BN, M = 128
	static constexpr uint32_t IDESC =
	    (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((128u >> 4) << 24);
};

// C[M][N] = act(A B^T + bias) for A [M][K] and B [N][K] in BF16 (K a multiple
// of 64; both read by TMA with the 128-byte swizzle, rows past M or N read as
// zero; bias may be null), accumulated in FP32 in TMEM. One CTA per 128 x BN tile: warp 0
// issues the TMA loads (GSTAGES-deep ring), warp 1 the MMAs (and owns the
// TMEM allocation), warps 2-5 read their 32 TMEM lanes, add the bias, apply
// the ReLU and store FP32 rows. Every wait gives up after wait_cycles clock
// cycles (about a second unless a test shortens it), sets *err and lets the
// CTA free its TMEM and exit; withhold_kb >= 0 is a test hook that never
// issues that stage's copies (-1 in production).
template <int BN>
__global__ void __launch_bounds__(192, 1) pnet_gemm_tc_kernel(const __grid_constant__ CUtensorMap map_a,
                                                              const __grid_constant__ CUtensorMap map_b, int num_kb,
                                                              int M, int N, const float *__restrict__ bias, int relu,
                                                              float *__restrict__ C, int ldc, int *__restrict__ err,
                                                              long long wait_cycles, int withhold_kb,
                                                              int kb_split = 0) {
	using G = GemmCfg<BN>;
	// split-k (kb_split > 0): CTA z takes K blocks [z kb_split, +kb_split)
	// and writes its partial product to C + z M ldc (every split has at
	// least one block: the grid has ceil(num_kb / kb_split) of them)
	const int kb0 = kb_split > 0 ? (int)blockIdx.z * kb_split : 0;
	const int nkb = kb_split > 0 ? min(kb_split, num_kb - kb0) : num_kb;
	if (kb_split > 0)
		C += (size_t)blockIdx.z * M * ldc;
	extern __shared__ uint8_t gsm_raw[];
	uint8_t *sm = (uint8_t *)(((uintptr_t)gsm_raw + 1023) & ~(uintptr_t)1023);
	uint64_t *bars = (uint64_t *)(sm + GSTAGES * G::STAGE);
	uint64_t *full = bars, *empty = bars + GSTAGES, *accum = bars + 2 * GSTAGES;
	uint32_t *tmem_slot = (uint32_t *)(bars + 2 * GSTAGES + 1);
	volatile int *abort_flag = (volatile int *)(tmem_slot + 1);
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int mt = blockIdx.x, nt = blockIdx.y;
	if (threadIdx.x == 0) {
		for (int s = 0; s < GSTAGES; ++s) {
			mbar_init(&full[s], 1);
			mbar_init(&empty[s], 1);
		}
		mbar_init(accum, 1);
		*abort_flag = 0;
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	if (warp == 1) {
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
		             "r"(BN)
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
			for (int kb = 0; kb < nkb; ++kb) {
				const int s = kb % GSTAGES;
				const uint32_t ph = (uint32_t)(kb / GSTAGES) & 1u;
				if (*abort_flag || !mbar_wait(&empty[s], ph ^ 1u, wait_cycles)) {
					*abort_flag = 1;
					atomicExch(err, 1);
					break;
				}
				if (kb == withhold_kb)  // test hook: this stage's copies are never issued
					continue;
				uint8_t *st = sm + s * G::STAGE;
				mbar_expect_tx(&full[s], G::STAGE);
				tma_load_2d(st, &map_a, &full[s], (kb0 + kb) * GK, mt * 128);
				tma_load_2d(st + G::A_BYTES, &map_b, &full[s], (kb0 + kb) * GK, nt * BN);
				issued = kb + 1;
			}
			// on a give-up, let the copies still in flight land before exiting
			if (*abort_flag)
				for (int kb = max(0, issued - GSTAGES); kb < issued; ++kb)
					mbar_wait(&full[kb % GSTAGES], (uint32_t)(kb / GSTAGES) & 1u, wait_cycles);
		}
		__syncwarp();
	} else if (warp == 1) {
		if (lane == 0) {
			for (int kb = 0; kb < nkb; ++kb) {
				const int s = kb % GSTAGES;
				const uint32_t ph = (uint32_t)(kb / GSTAGES) & 1u;
				if (*abort_flag || !mbar_wait(&full[s], ph, wait_cycles)) {
					*abort_flag = 1;
					atomicExch(err, 1);
					break;
				}
				tc_fence_after();
				const uint32_t a = smem_addr(sm + s * G::STAGE), b = a + G::A_BYTES;
#pragma unroll
				for (int k = 0; k < GK / 16; ++k)
					umma_f16(tmem, sw128_desc(a + 32 * k), sw128_desc(b + 32 * k), G::IDESC, (kb | k) != 0);
				umma_commit(&empty[s]);
			}
			umma_commit(accum);
		}
		__syncwarp();
	} else {
		// warp w reads TMEM lanes 32 (w % 4) .. + 31
		const int q = warp & 3, row = mt * 128 + q * 32 + lane;
		const bool ok = mbar_wait(accum, 0, wait_cycles);
		if (!ok) {
			*abort_flag = 1;
			atomicExch(err, 1);
		}
		tc_fence_after();
		if (ok && !*abort_flag) {
			for (int c = 0; c < BN / 16; ++c) {
				float v[16];
				tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(c * 16), v);
				if (row < M) {
#pragma unroll
					for (int j = 0; j < 16; ++j) {
						const int col = nt * BN + c * 16 + j;
						if (col < N) {
							const float x = bias != nullptr ? v[j] + bias[col] : v[j];
							C[(size_t)row * ldc + col] = relu ? fmaxf(x, 0.f) : x;
						}
					}
				}
			}
		}
	}
	tc_fence_before();
	__syncthreads();
	if (warp == 1) {
		tc_fence_after();
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN) : "memory");
	}
}

// cols[(b, ho, wo)][k] in BF16, k = (ky, kx, c) < 9 C as im2col_kernel, zero
// for 9 C <= k < Kp (the products' K padding). C and Kp are multiples of 8:
// each thread writes 8 consecutive k (8 channels of one input pixel: two
// 16-byte loads, one 16-byte store).
__global__ void im2col_bf16_kernel(const float *__restrict__ X, int B, int H, int C, int s, int Ho, int Kp,
                                   __nv_bfloat16 *__restrict__ cols) {
	const int groups = Kp >> 3, K = 9 * C;
	const long long n = (long long)B * Ho * Ho * groups;
	for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
		const unsigned r = (unsigned)(e / groups), k0 = (unsigned)(e - (long long)r * groups) * 8u;
		float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
		if ((int)k0 < K) {
			const unsigned tap = k0 / (unsigned)C, c0 = k0 - tap * (unsigned)C;
			const unsigned ky = tap / 3u, kx = tap - ky * 3u;
			const unsigned wo = r % (unsigned)Ho, t = r / (unsigned)Ho;
			const unsigned ho = t % (unsigned)Ho, b = t / (unsigned)Ho;
			const int y = (int)(ho * s + ky) - 1, x = (int)(wo * s + kx) - 1;
			if (y >= 0 && y < H && x >= 0 && x < H) {
				const float4 *src = reinterpret_cast<const float4 *>(X + (((size_t)b * H + y) * H + x) * C + c0);
				const float4 p = src[0], q = src[1];
				v[0] = p.x; v[1] = p.y; v[2] = p.z; v[3] = p.w;
				v[4] = q.x; v[5] = q.y; v[6] = q.z; v[7] = q.w;
			}
		}
		__align__(16) __nv_bfloat16 o[8];
#pragma unroll
		for (int j = 0; j < 8; ++j)
			o[j] = __float2bfloat16_rn(v[j]);
		*reinterpret_cast<uint4 *>(cols + (size_t)r * Kp + k0) = *reinterpret_cast<const uint4 *>(o);
	}
}

// Layer 0 of the inference pass (conv 3x3, 1 -> 32 channels, stride 1 on the
// 32 x 32 image) directly: one thread per output pixel, its 9 inputs times
// the BF16 weights in tap order with fmaf from zero (the operation order of
// the FP32 product path), + bias, ReLU; 32 channels stored as 8 16-byte
// vectors.
__global__ void __launch_bounds__(256) conv0_kernel(const float *__restrict__ X, int B,
                                                    const __nv_bfloat16 *__restrict__ w,
                                                    const float *__restrict__ bias, float *__restrict__ Y) {
	__shared__ float ws[32 * 9], bs[32];
	for (int i = threadIdx.x; i < 32 * 9; i += blockDim.x)
		ws[i] = __bfloat162float(w[i]);
	for (int i = threadIdx.x; i < 32; i += blockDim.x)
		bs[i] = bias[i];
	__syncthreads();
	const long long n = (long long)B * IMG * IMG;
	for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
		const int x = (int)(p & (IMG - 1)), y = (int)((p >> 5) & (IMG - 1));
		const float *img = X + (p - (long long)y * IMG - x);
		float in[9];
#pragma unroll
		for (int ky = 0; ky < 3; ++ky)
#pragma unroll
			for (int kx = 0; kx < 3; ++kx) {
				const int yy = y + ky - 1, xx = x + kx - 1;
				in[ky * 3 + kx] = (yy >= 0 && yy < IMG && xx >= 0 && xx < IMG) ? img[yy * IMG + xx] : 0.f;
			}
		float4 *out = reinterpret_cast<float4 *>(Y + p * 32);
#pragma unroll
		for (int o4 = 0; o4 < 8; ++o4) {
			float r[4];
#pragma unroll
			for (int j = 0; j < 4; ++j) {
				const int o = o4 * 4 + j;
				float acc = 0.f;
#pragma unroll
				for (int k = 0; k < 9; ++k)
					acc = fmaf(in[k], ws[o * 9 + k], acc);
				r[j] = fmaxf(acc + bs[o], 0.f);
			}
			out[o4] = make_float4(r[0], r[1], r[2], r[3]);
		}
	}
}

// W [rows][K] BF16 -> [rows][Kp] with zero columns K .. Kp - 1.
__global__ void pad_rows_bf16_kernel(const __nv_bfloat16 *__restrict__ W, long long rows, int K, int Kp,
                                     __nv_bfloat16 *__restrict__ out) {
	const long long n = rows * Kp;
	for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
		const int k = (int)(e % Kp);
		out[e] = k < K ? W[(e / Kp) * K + k] : __float2bfloat16_rn(0.f);
	}
}

// X [rows][K] FP32 -> [rows][Kp] BF16 with zero columns K .. Kp - 1.
__global__ void rows_bf16_kernel(const float *__restrict__ X, long long rows, int K, int Kp,
                                 __nv_bfloat16 *__restrict__ out) {
	// 32-bit index arithmetic (rows Kp < 2^31 for every layer and batch)
	const unsigned n = (unsigned)(rows * Kp);
	for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
		const unsigned r = e / (unsigned)Kp, k = e - r * (unsigned)Kp;
		out[e] = __float2bfloat16_rn((int)k < K ? X[(size_t)r * K + k] : 0.f);
	}
}

}  // namespace

// ---------------------------------------------------------------------------
// the network object
// ---------------------------------------------------------------------------
// A training batch: dst row k = src row idx[k], lab_out[k] = lab[idx[k]].
__global__ void gather_rows_kernel(const float *__restrict__ src, const int *__restrict__ idx, int n, int row,
                                   float *__restrict__ dst, const int *__restrict__ lab, int *__restrict__ lab_out) {
	const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (e < (long long)n * row)
		dst[e] = src[(size_t)idx[e / row] * row + e % row];
	if (lab != nullptr && e < n)
		lab_out[e] = lab[idx[e]];
}

// Y[c][r] = bf16(X[r][c]) for r < rows, 0 for rows <= r < rows_p: a 32 x 32
// tile through shared memory per block (coalesced reads of X's rows and
// writes of Y's rows). Grid: ceil(cols / 32) x ceil(rows_p / 32), 32 x 8
// threads.
template <typename T>
__global__ void transpose_bf16_kernel(const T *__restrict__ X, long long rows, int cols, long long rows_p,
                                      __nv_bfloat16 *__restrict__ Y) {
	__shared__ float tile[32][33];
	const int c0 = blockIdx.x * 32;
	const long long r0 = (long long)blockIdx.y * 32;
	for (int k = threadIdx.y; k < 32; k += 8) {
		const long long r = r0 + k;
		const int c = c0 + threadIdx.x;
		float v = 0.f;
		if (r < rows && c < cols)
			v = (float)X[r * cols + c];
		tile[k][threadIdx.x] = v;
	}
	__syncthreads();
	for (int k = threadIdx.y; k < 32; k += 8) {
		const int c = c0 + k;
		const long long r = r0 + threadIdx.x;
		if (c < cols && r < rows_p)
			Y[(size_t)c * rows_p + r] = __float2bfloat16(tile[threadIdx.x][k]);
	}
}

// Wt[k][c] = W[c][k] for a BF16 weight matrix W [cout][K], c padded with
// zeros to coutp: the B operand of the input-gradient product.
__global__ void transpose_pad_weights_kernel(const __nv_bfloat16 *__restrict__ W, int cout, int K, int coutp,
                                             __nv_bfloat16 *__restrict__ Wt) {
	const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= (long long)K * coutp)
		return;
	const int k = (int)(i / coutp), c = (int)(i % coutp);
	Wt[i] = c < cout ? W[(size_t)c * K + k] : __float2bfloat16(0.f);
}

struct dfg_pnet {
	int device = 0;
	cudaStream_t stream = nullptr;
	std::string err;
	int num_classes = 0, batch = 0;
	int infer_batch = 0;  // images per forward pass outside training (>= batch)
	LayerShape L[NL];
	DevBuf<float> w[NL], b[NL], mw[NL], vw[NL], mb[NL], vb[NL], gw[NL], gb[NL];
	DevBuf<__nv_bfloat16> wb[NL];
	DevBuf<float> act[NL + 1], dact[NL + 1], cols[4], dcols[4], loss, xbatch;
	DevBuf<int> labels, idx, perm, lab_all;
	DevBuf<float> wsplit;  // split-k partial weight gradients
	DevBuf<float> gpart;   // per-block partial sums of the bias and layer-0 gradients
	DevBuf<double> loss_acc;
	DevBuf<float> images;
	long long n_images = 0;
	DevBuf<int> pixel_bin;
	int P = 0;
	// tensor-core inference: BF16 operands with K padded to 64, error flag
	bool use_tc = true;
	DevBuf<__nv_bfloat16> colsb, wbp[NL];
	// tensor-core training (mixed precision): every layer's BF16 input rows
	// of the training batch (kept for its weight gradient), the transposed
	// operands of the gradient products, BF16 output gradients, transposed
	// padded weights and split-k partials
	bool tc_train = true;
	DevBuf<__nv_bfloat16> colsbl[NL], dyt, colst, dyb, wtp[NL];
	DevBuf<float> tsplit;
	DevBuf<int> terr;
	// failure-detection test hooks of the tensor-core products (as the
	// context's dense_wait_cycles / dense_withhold_stage options)
	long long wait_cycles = 2000000000LL;
	int withhold = -1;
	// soft targets of the loaded images (dfg_pnet_set_targets)
	DevBuf<long long> t_off;
	DevBuf<int> t_cls, iota;
	DevBuf<float> t_w;
	long long n_targets_images = -1;
	long long step = 0;
	int fail(int code, const char *fmt, ...) {
		char buf[1024];
		va_list ap;
		va_start(ap, fmt);
		vsnprintf(buf, sizeof(buf), fmt, ap);
		va_end(ap);
		err = buf;
		return code;
	}
	long long rows(int l, int n) const {  // output rows of layer l for n images
		return L[l].kind == 0 ? (long long)n * L[l].hout * L[l].hout : n;
	}
};

#define PK(call)                                                                                  \
	do {                                                                                          \
		cudaError_t e_ = (call);                                                                  \
		if (e_ != cudaSuccess)                                                                    \
			return net->fail(e_ == cudaErrorMemoryAllocation ? DFG_ERR_NOMEM : DFG_ERR_CUDA,      \
			                 "%s failed: %s", #call, cudaGetErrorString(e_));                    \
	} while (0)
#define PKL(name)                                                                                 \
	do {                                                                                          \
		cudaError_t e_ = cudaGetLastError();                                                      \
		if (e_ != cudaSuccess)                                                                    \
			return net->fail(DFG_ERR_CUDA, "launch of %s failed: %s", name, cudaGetErrorString(e_)); \
	} while (0)

static unsigned grid_for(long long n) { return (unsigned)std::min<long long>((n + 255) / 256, 1 << 20); }

// Split of the k range of an M x N product so that the grid fills about two
// blocks per SM (chunks of at least 512, multiples of 16): (splits, chunk).
static void k_split(int M, int N, long long K, int *S, int *chunk) {
	const long long blocks = (long long)((N + 63) / 64) * ((M + 63) / 64);
	long long s = std::min<long long>(K / 512, (296 + blocks - 1) / blocks);
	s = std::max<long long>(1, std::min<long long>(s, 1024));
	long long c = (K + s - 1) / s;
	c = (c + 15) / 16 * 16;
	*chunk = (int)c;
	*S = (int)((K + c - 1) / c);
}

template <typename TAe, typename TBe, bool TA, bool TB>
static int gemm(dfg_pnet *net, int M, int N, int K, float alpha, const TAe *A, int lda, const TBe *B, int ldb,
                float beta, float *C, int ldc) {
	dim3 grid((N + 63) / 64, (M + 63) / 64);
	gemm_kernel<TAe, TBe, TA, TB><<<grid, 256, 0, net->stream>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, K, 0);
	PKL("gemm_kernel");
	return DFG_OK;
}

// Weight gradient C [M][N] = A^T B with A [K][M], B [K][N] and a long k range
// (the batch's output positions): split-k partials, summed in split order.
static int gemm_wgrad(dfg_pnet *net, int M, int N, int K, const float *A, const float *B, float *C) {
	int S, chunk;
	k_split(M, N, K, &S, &chunk);
	if (S == 1)
		return gemm<float, float, true, false>(net, M, N, K, 1.f, A, M, B, N, 0.f, C, N);
	dim3 grid((N + 63) / 64, (M + 63) / 64, S);
	gemm_kernel<float, float, true, false><<<grid, 256, 0, net->stream>>>(M, N, K, 1.f, A, M, B, N, 0.f,
	                                                                      net->wsplit.p, N, chunk,
	                                                                      (long long)M * N);
	PKL("gemm_kernel");
	sum_splits_kernel<<<(unsigned)(((long long)M * N + 31) / 32), dim3(32, 8), 0, net->stream>>>(net->wsplit.p, S,
	                                                                                          (long long)M * N, C);
	PKL("sum_splits_kernel");
	return DFG_OK;
}

// dX [B][H][H][C] from the column gradients of a 3 x 3 convolution.
static int col2im(dfg_pnet *net, const float *dcols, int B, int H, int C, int s, int Ho, float *dX) {
	cudaStream_t st = net->stream;
	if (C % 4 == 0 && (s == 1 || s == 2)) {
		const long long n4 = (long long)B * H * H * (C / 4);
		if (s == 1)
			col2im4_kernel<1><<<grid_for(n4), 256, 0, st>>>(dcols, B, H, C, Ho, dX);
		else
			col2im4_kernel<2><<<grid_for(n4), 256, 0, st>>>(dcols, B, H, C, Ho, dX);
		PKL("col2im4_kernel");
		return DFG_OK;
	}
	col2im_kernel<<<grid_for((long long)B * H * H * C), 256, 0, st>>>(dcols, B, H, C, s, Ho, dX);
	PKL("col2im_kernel");
	return DFG_OK;
}

// Bias gradients db[c] = sum over rows of dY[r][c] (two-stage, deterministic).
static int bias_grad(dfg_pnet *net, const float *dY, long long rows, int cols, float *db) {
	const long long chunk = std::max<long long>(64, (rows + 295) / 296);
	const int nb = (int)((rows + chunk - 1) / chunk);
	if ((size_t)nb * cols > net->gpart.n)
		PK(net->gpart.ensure((size_t)nb * cols));
	colsum_part_kernel<<<nb, 256, 0, net->stream>>>(dY, rows, cols, chunk, net->gpart.p);
	PKL("colsum_part_kernel");
	colsum_final_kernel<<<(cols + 255) / 256, 256, 0, net->stream>>>(net->gpart.p, nb, cols, db);
	PKL("colsum_final_kernel");
	return DFG_OK;
}

// Layer 0's weight and bias gradients from its FP32 im2col rows (K = 9).
static int wgrad0(dfg_pnet *net, const float *dY, const float *X, long long rows, float *gw, float *gb) {
	if (net->L[0].cout != 32 || net->L[0].fan_in() != 9)
		return net->fail(DFG_ERR_STATE, "layer 0 must map 1 channel to 32 (3 x 3)");
	const long long chunk = std::max<long long>(64, (rows + 295) / 296);
	const int nb = (int)((rows + chunk - 1) / chunk);
	if ((size_t)nb * 320 > net->gpart.n)
		PK(net->gpart.ensure((size_t)nb * 320));
	wgrad0_part_kernel<<<nb, 256, 0, net->stream>>>(dY, X, rows, chunk, net->gpart.p);
	PKL("wgrad0_part_kernel");
	wgrad0_final_kernel<<<1, 320, 0, net->stream>>>(net->gpart.p, nb, gw, gb);
	PKL("wgrad0_final_kernel");
	return DFG_OK;
}

// Forward pass of n images at X (device, [n][1024]); logits in act[NL].
static int forward(dfg_pnet *net, const float *X, int n) {
	cudaStream_t st = net->stream;
	const float *in = X;
	for (int l = 0; l < NL; ++l) {
		const LayerShape &s = net->L[l];
		const long long rows = net->rows(l, n);
		float *out = net->act[l + 1].p;
		if (s.kind == 0) {
			const long long nc = rows * 9 * s.cin;
			im2col_kernel<<<grid_for(nc), 256, 0, st>>>(in, n, s.hin, s.cin, s.stride, s.hout, net->cols[l].p);
			PKL("im2col_kernel");
			if (int rc = gemm<float, __nv_bfloat16, false, true>(net, (int)rows, s.cout, 9 * s.cin, 1.f,
			                                                       net->cols[l].p, 9 * s.cin, net->wb[l].p,
			                                                       9 * s.cin, 0.f, out, s.cout))
				return rc;
		} else {
			if (int rc = gemm<float, __nv_bfloat16, false, true>(net, n, s.cout, s.cin, 1.f, in, s.cin,
			                                                       net->wb[l].p, s.cin, 0.f, out, s.cout))
				return rc;
		}
		bias_act_kernel<<<grid_for(rows * s.cout), 256, 0, st>>>(out, rows, s.cout, net->b[l].p, l < NL - 1);
		PKL("bias_act_kernel");
		in = out;
	}
	return DFG_OK;
}

// ---------------------------------------------------------------------------
// tensor-core forward pass (inference)
// ---------------------------------------------------------------------------
static int kpad64(int k) { return (k + GK - 1) / GK * GK; }

static PFN_cuTensorMapEncodeTiled_v12000 pnet_map_encoder() {
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

// Tensor map of a row-major BF16 matrix [rows][K] (K a multiple of 64) read in
// boxes of 64 columns x box_rows rows with the 128-byte swizzle.
static int pnet_map(dfg_pnet *net, CUtensorMap *map, const void *base, long long rows, int K, int box_rows) {
	auto fn = pnet_map_encoder();
	if (fn == nullptr)
		return net->fail(DFG_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
	cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
	cuuint64_t strides[1] = {(cuuint64_t)K * 2};
	cuuint32_t box[2] = {(cuuint32_t)GK, (cuuint32_t)box_rows};
	cuuint32_t estr[2] = {1, 1};
	const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box, estr,
	                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
	                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
	if (r != CUDA_SUCCESS)
		return net->fail(DFG_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
	return DFG_OK;
}

template <int BN>
static int launch_tc_gemm(dfg_pnet *net, const CUtensorMap &ma, const CUtensorMap &mb, int num_kb, int M, int N,
                          const float *bias, int relu, float *C) {
	dim3 grid((M + 127) / 128, (N + BN - 1) / BN);
	pnet_gemm_tc_kernel<BN><<<grid, 192, GemmCfg<BN>::SMEM, net->stream>>>(ma, mb, num_kb, M, N, bias, relu, C, N,
	                                                                     net->terr.p, net->wait_cycles,
	                                                                     net->withhold);
	PKL("pnet_gemm_tc_kernel");
	return DFG_OK;
}

// BF16 weight copies with K padded to 64 for the tensor-core products (after
// any change of the weights), and the products' shared-memory limits on this
// network's device.
static int pad_weights(dfg_pnet *net) {
	PK(cudaFuncSetAttribute(pnet_gemm_tc_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, GemmCfg<32>::SMEM));
	PK(cudaFuncSetAttribute(pnet_gemm_tc_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, GemmCfg<64>::SMEM));
	PK(cudaFuncSetAttribute(pnet_gemm_tc_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                        GemmCfg<256>::SMEM));
	for (int l = 1; l < NL; ++l) {
		const LayerShape &sh = net->L[l];
		const int K = sh.fan_in(), Kp = kpad64(K);
		pad_rows_bf16_kernel<<<grid_for((long long)sh.cout * Kp), 256, 0, net->stream>>>(net->wb[l].p, sh.cout, K,
		                                                                                Kp, net->wbp[l].p);
		PKL("pad_rows_bf16_kernel");
	}
	return DFG_OK;
}

// Forward pass of n <= infer_batch images with the products of layers 1-5 on
// the tensor cores (BF16 activations and weights, FP32 accumulation); layer 0
// (K = 9) stays in FP32 (conv0_kernel, the FP32 path's arithmetic). Logits
// in act[NL].
static int forward_tc(dfg_pnet *net, const float *X, int n) {
	cudaStream_t st = net->stream;
	conv0_kernel<<<grid_for((long long)n * IMG * IMG), 256, 0, st>>>(X, n, net->wb[0].p, net->b[0].p, net->act[1].p);
	PKL("conv0_kernel");
	for (int l = 1; l < NL; ++l) {
		const LayerShape &s = net->L[l];
		const long long rows = net->rows(l, n);
		const int K = s.fan_in(), Kp = kpad64(K);
		const float *in = net->act[l].p;
		if (s.kind == 0) {
			im2col_bf16_kernel<<<grid_for(rows * Kp / 8), 256, 0, st>>>(in, n, s.hin, s.cin, s.stride, s.hout, Kp,
			                                                            net->colsb.p);
			PKL("im2col_bf16_kernel");
		} else {
			rows_bf16_kernel<<<grid_for(rows * Kp), 256, 0, st>>>(in, rows, K, Kp, net->colsb.p);
			PKL("rows_bf16_kernel");
		}
		CUtensorMap ma, mb;
		if (int rc = pnet_map(net, &ma, net->colsb.p, rows, Kp, 128))
			return rc;
		const int BN = s.cout <= 32 ? 32 : (s.cout <= 64 ? 64 : 256);
		if (int rc = pnet_map(net, &mb, net->wbp[l].p, s.cout, Kp, BN))
			return rc;
		const int relu = l < NL - 1;
		int rc;
		if (BN == 32)
			rc = launch_tc_gemm<32>(net, ma, mb, Kp / GK, (int)rows, s.cout, net->b[l].p, relu, net->act[l + 1].p);
		else if (BN == 64)
			rc = launch_tc_gemm<64>(net, ma, mb, Kp / GK, (int)rows, s.cout, net->b[l].p, relu, net->act[l + 1].p);
		else
			rc = launch_tc_gemm<256>(net, ma, mb, Kp / GK, (int)rows, s.cout, net->b[l].p, relu, net->act[l + 1].p);
		if (rc)
			return rc;
	}
	return DFG_OK;
}

// Loss and gradients of n images at X with labels (device), or with the soft
// targets of the loaded images img (device, lab == nullptr); per-image losses
// in loss.
static int backward(dfg_pnet *net, const float *X, const int *lab, int n, const int *img = nullptr) {
	cudaStream_t st = net->stream;
	if (lab != nullptr) {
		softmax_xent_kernel<<<(n * 32 + 255) / 256, 256, 0, st>>>(net->act[NL].p, lab, n, net->num_classes,
		                                                          net->dact[NL].p, net->loss.p);
		PKL("softmax_xent_kernel");
	} else {
		softmax_xent_soft_kernel<<<(n * 32 + 255) / 256, 256, 0, st>>>(
		    net->act[NL].p, img, net->t_off.p, net->t_cls.p, net->t_w.p, n, net->num_classes, net->dact[NL].p,
		    net->loss.p);
		PKL("softmax_xent_soft_kernel");
	}
	for (int l = NL - 1; l >= 0; --l) {
		const LayerShape &s = net->L[l];
		const long long rows = net->rows(l, n);
		float *dY = net->dact[l + 1].p;
		if (l < NL - 1) {
			relu_back_kernel<<<grid_for(rows * s.cout), 256, 0, st>>>(dY, net->act[l + 1].p, rows * s.cout);
			PKL("relu_back_kernel");
		}
		const float *in = l == 0 ? X : net->act[l].p;
		if (l == 0) {
			if (int rc = wgrad0(net, dY, net->cols[0].p, rows, net->gw[0].p, net->gb[0].p))
				return rc;
			continue;
		}
		if (int rc = bias_grad(net, dY, rows, s.cout, net->gb[l].p))
			return rc;
		if (s.kind == 0) {
			if (int rc = gemm_wgrad(net, s.cout, 9 * s.cin, (int)rows, dY, net->cols[l].p, net->gw[l].p))
				return rc;
			if (l > 0) {
				if (int rc = gemm<float, __nv_bfloat16, false, false>(net, (int)rows, 9 * s.cin, s.cout, 1.f, dY,
				                                                        s.cout, net->wb[l].p, 9 * s.cin, 0.f,
				                                                        net->dcols[l].p, 9 * s.cin))
					return rc;
				if (int rc = col2im(net, net->dcols[l].p, n, s.hin, s.cin, s.stride, s.hout, net->dact[l].p))
					return rc;
			}
		} else {
			if (int rc = gemm_wgrad(net, s.cout, s.cin, n, dY, in, net->gw[l].p))
				return rc;
			if (int rc = gemm<float, __nv_bfloat16, false, false>(net, n, s.cin, s.cout, 1.f, dY, s.cout,
			                                                        net->wb[l].p, s.cin, 0.f, net->dact[l].p,
			                                                        s.cin))
				return rc;
		}
	}
	return DFG_OK;
}

// ---------------------------------------------------------------------------
// tensor-core training: mixed precision (BF16 operands, FP32 accumulation)
// ---------------------------------------------------------------------------
// C[M][N] (row stride N) = A[M][Kp] B[N][Kp]^T (+ bias, ReLU) on the tensor
// cores; when the (M, N) tiles alone would leave most SMs idle, the K blocks
// are split over a third grid dimension and the partial products summed in
// split order (deterministic).
static long long round128(long long m) { return (m + 127) / 128 * 128; }

static int tc_product(dfg_pnet *net, const __nv_bfloat16 *A, long long M, int Kp, const __nv_bfloat16 *B, int N,
                      float *C, const float *bias, int relu) {
	// A holds round128(M) rows (the rows past M are never stored), so that
	// every 128-row box lies inside the tensor
	const int BN = N <= 32 ? 32 : (N <= 64 ? 64 : 256);
	const int num_kb = Kp / GK;
	const long long tiles = ((M + 127) / 128) * (long long)((N + BN - 1) / BN);
	int S = (int)std::max<long long>(1, std::min<long long>(num_kb, 296 / std::max<long long>(1, tiles)));
	const int kbs = (num_kb + S - 1) / S;
	S = (num_kb + kbs - 1) / kbs;  // every split holds at least one K block
	if (S > 1 && (size_t)S * M * N > net->tsplit.n)
		PK(net->tsplit.ensure((size_t)S * M * N));
	CUtensorMap ma, mb;
	if (int rc = pnet_map(net, &ma, A, round128(M), Kp, 128))
		return rc;
	if (int rc = pnet_map(net, &mb, B, N, Kp, BN))
		return rc;
	float *out = S > 1 ? net->tsplit.p : C;
	const float *b = S > 1 ? nullptr : bias;
	const int rl = S > 1 ? 0 : relu;
	dim3 grid((unsigned)((M + 127) / 128), (unsigned)((N + BN - 1) / BN), (unsigned)S);
#define DFG_TC(BNV)                                                                                           \
	pnet_gemm_tc_kernel<BNV><<<grid, 192, GemmCfg<BNV>::SMEM, net->stream>>>(                                 \
	    ma, mb, num_kb, (int)M, N, b, rl, out, N, net->terr.p, net->wait_cycles, net->withhold, S > 1 ? kbs : 0)
	if (BN == 32)
		DFG_TC(32);
	else if (BN == 64)
		DFG_TC(64);
	else
		DFG_TC(256);
#undef DFG_TC
	PKL("pnet_gemm_tc_kernel");
	if (S > 1) {
		sum_splits_kernel<<<(unsigned)((M * N + 31) / 32), dim3(32, 8), 0, net->stream>>>(net->tsplit.p, S, M * N, C);
		PKL("sum_splits_kernel");
		if (bias != nullptr) {
			bias_act_kernel<<<grid_for(M * N), 256, 0, net->stream>>>(C, M, N, bias, relu);
			PKL("bias_act_kernel");
		}
	}
	return DFG_OK;
}

// The BF16 copies of the current weights the tensor-core products read: K
// padded to 64 (forward) and transposed with the outputs padded to 64 (input
// gradients).
static int refresh_tc_weights(dfg_pnet *net) {
	if (int rc = pad_weights(net))
		return rc;
	for (int l = 1; l < NL; ++l) {
		const LayerShape &sh = net->L[l];
		const int K = sh.fan_in(), cp = kpad64(sh.cout);
		transpose_pad_weights_kernel<<<grid_for((long long)K * cp), 256, 0, net->stream>>>(net->wb[l].p, sh.cout,
		                                                                                    K, cp, net->wtp[l].p);
		PKL("transpose_pad_weights_kernel");
	}
	return DFG_OK;
}

// Training forward pass of n <= batch images: layer 0 as the FP32 path (its
// im2col rows kept for its weight gradient), layers 1-5 as tensor-core
// products of BF16 input rows (kept per layer) and the padded weights;
// FP32 outputs in act.
static int forward_train_tc(dfg_pnet *net, const float *X, int n) {
	cudaStream_t st = net->stream;
	const LayerShape &s0 = net->L[0];
	const long long rows0 = net->rows(0, n);
	im2col_kernel<<<grid_for(rows0 * 9 * s0.cin), 256, 0, st>>>(X, n, s0.hin, s0.cin, s0.stride, s0.hout,
	                                                           net->cols[0].p);
	PKL("im2col_kernel");
	conv0_kernel<<<grid_for((long long)n * IMG * IMG), 256, 0, st>>>(X, n, net->wb[0].p, net->b[0].p, net->act[1].p);
	PKL("conv0_kernel");
	for (int l = 1; l < NL; ++l) {
		const LayerShape &s = net->L[l];
		const long long rows = net->rows(l, n);
		const int K = s.fan_in(), Kp = kpad64(K);
		const float *in = net->act[l].p;
		if (s.kind == 0) {
			im2col_bf16_kernel<<<grid_for(rows * Kp / 8), 256, 0, st>>>(in, n, s.hin, s.cin, s.stride, s.hout, Kp,
			                                                            net->colsbl[l].p);
			PKL("im2col_bf16_kernel");
		} else {
			rows_bf16_kernel<<<grid_for(rows * Kp), 256, 0, st>>>(in, rows, K, Kp, net->colsbl[l].p);
			PKL("rows_bf16_kernel");
		}
		if (int rc = tc_product(net, net->colsbl[l].p, rows, Kp, net->wbp[l].p, s.cout, net->act[l + 1].p,
		                        net->b[l].p, l < NL - 1))
			return rc;
	}
	return DFG_OK;
}

// Gradients of the training forward pass: per layer the FP32 output
// gradient (ReLU mask, bias gradient as the FP32 path), then in BF16 on the
// tensor cores the weight gradient dW = dY^T X (dY and the layer's BF16
// input rows transposed so that the batch's rows are the reduction, split-k)
// and the input gradient dX = dY W (dY rows against the transposed weights);
// layer 0's weight gradient (K = 9) stays on the FP32 path.
static int backward_tc(dfg_pnet *net, const float *X, const int *lab, int n, const int *img) {
	cudaStream_t st = net->stream;
	(void)X;
	if (lab != nullptr) {
		softmax_xent_kernel<<<(n * 32 + 255) / 256, 256, 0, st>>>(net->act[NL].p, lab, n, net->num_classes,
		                                                          net->dact[NL].p, net->loss.p);
		PKL("softmax_xent_kernel");
	} else {
		softmax_xent_soft_kernel<<<(n * 32 + 255) / 256, 256, 0, st>>>(
		    net->act[NL].p, img, net->t_off.p, net->t_cls.p, net->t_w.p, n, net->num_classes, net->dact[NL].p,
		    net->loss.p);
		PKL("softmax_xent_soft_kernel");
	}
	for (int l = NL - 1; l >= 0; --l) {
		const LayerShape &s = net->L[l];
		const long long rows = net->rows(l, n);
		float *dY = net->dact[l + 1].p;
		if (l < NL - 1) {
			relu_back_kernel<<<grid_for(rows * s.cout), 256, 0, st>>>(dY, net->act[l + 1].p, rows * s.cout);
			PKL("relu_back_kernel");
		}
		if (l == 0) {
			if (int rc = wgrad0(net, dY, net->cols[0].p, rows, net->gw[0].p, net->gb[0].p))
				return rc;
			continue;
		}
		if (int rc = bias_grad(net, dY, rows, s.cout, net->gb[l].p))
			return rc;
		const int K = s.fan_in(), Kp = kpad64(K), cp = kpad64(s.cout);
		const long long rows_p = (rows + 63) / 64 * 64;
		// dW [cout][K] = dY^T X: both operands with the batch rows as the reduction
		dim3 tb(32, 8);
		transpose_bf16_kernel<float><<<dim3((s.cout + 31) / 32, (unsigned)(rows_p / 32)), tb, 0, st>>>(
		    dY, rows, s.cout, rows_p, net->dyt.p);
		PKL("transpose_bf16_kernel");
		transpose_bf16_kernel<__nv_bfloat16><<<dim3((Kp + 31) / 32, (unsigned)(rows_p / 32)), tb, 0, st>>>(
		    net->colsbl[l].p, rows, Kp, rows_p, net->colst.p);
		PKL("transpose_bf16_kernel");
		if (int rc = tc_product(net, net->dyt.p, s.cout, (int)rows_p, net->colst.p, K, net->gw[l].p, nullptr, 0))
			return rc;
		// dX = dY W: dY rows in BF16 (outputs padded to 64) against W^T
		rows_bf16_kernel<<<grid_for(rows * cp), 256, 0, st>>>(dY, rows, s.cout, cp, net->dyb.p);
		PKL("rows_bf16_kernel");
		if (s.kind == 0) {
			if (int rc = tc_product(net, net->dyb.p, rows, cp, net->wtp[l].p, K, net->dcols[l].p, nullptr, 0))
				return rc;
			if (int rc = col2im(net, net->dcols[l].p, n, s.hin, s.cin, s.stride, s.hout, net->dact[l].p))
				return rc;
		} else {
			if (int rc = tc_product(net, net->dyb.p, rows, cp, net->wtp[l].p, K, net->dact[l].p, nullptr, 0))
				return rc;
		}
	}
	return DFG_OK;
}

static int check_tc_flag(dfg_pnet *net);

// Loss and gradients of one training batch: on the tensor cores (BF16
// operands from the current weights) or on the FP32 path. The products'
// pipeline flag is read by the caller at its next synchronisation.
static int train_pass(dfg_pnet *net, const float *X, const int *lab, int m, const int *img) {
	if (net->tc_train) {
		if (int rc = refresh_tc_weights(net))
			return rc;
		if (int rc = forward_train_tc(net, X, m))
			return rc;
		return backward_tc(net, X, lab, m, img);
	}
	if (int rc = forward(net, X, m))
		return rc;
	return backward(net, X, lab, m, img);
}

static int adam_step(dfg_pnet *net, float lr) {
	const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
	net->step++;
	const float c1 = 1.f - powf(b1, (float)net->step), c2 = 1.f - powf(b2, (float)net->step);
	for (int l = 0; l < NL; ++l) {
		const long long nw = net->L[l].nw();
		adam_kernel<<<grid_for(nw), 256, 0, net->stream>>>(net->w[l].p, net->mw[l].p, net->vw[l].p, net->gw[l].p,
		                                                    net->wb[l].p, nw, lr, b1, b2, c1, c2, eps);
		PKL("adam_kernel");
		adam_kernel<<<grid_for(net->L[l].cout), 256, 0, net->stream>>>(net->b[l].p, net->mb[l].p, net->vb[l].p,
		                                                                net->gb[l].p, nullptr, net->L[l].cout, lr,
		                                                                b1, b2, c1, c2, eps);
		PKL("adam_kernel");
	}
	return DFG_OK;
}

static int upload_params(dfg_pnet *net, const float *h) {
	size_t o = 0;
	for (int l = 0; l < NL; ++l) {
		const long long nw = net->L[l].nw();
		PK(cudaMemcpyAsync(net->w[l].p, h + o, nw * sizeof(float), cudaMemcpyHostToDevice, net->stream));
		o += nw;
		PK(cudaMemcpyAsync(net->b[l].p, h + o, net->L[l].cout * sizeof(float), cudaMemcpyHostToDevice, net->stream));
		o += net->L[l].cout;
		to_bf16_kernel<<<grid_for(nw), 256, 0, net->stream>>>(net->w[l].p, net->wb[l].p, nw);
		PKL("to_bf16_kernel");
	}
	PK(cudaStreamSynchronize(net->stream));
	return DFG_OK;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" void dfg_pnet_destroy(dfg_pnet *net) {
	if (!net)
		return;
	cudaSetDevice(net->device);
	if (net->stream) {
		cudaStreamSynchronize(net->stream);
		cudaStreamDestroy(net->stream);
	}
	delete net;
}

extern "C" int dfg_pnet_create(int device, int num_classes, int batch, unsigned long long seed, dfg_pnet **out) {
	if (!out || num_classes < 2 || batch < 1)
		return DFG_ERR_ARG;
	*out = nullptr;
	if (cudaSetDevice(device) != cudaSuccess)
		return DFG_ERR_CUDA;
	dfg_pnet *net = new dfg_pnet();
	net->device = device;
	net->num_classes = num_classes;
	net->batch = batch;
	if (cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking) != cudaSuccess) {
		delete net;
		return DFG_ERR_CUDA;
	}
	const LayerShape shapes[NL] = {{0, 1, 32, 32, 1, 32},   {0, 32, 32, 32, 2, 16}, {0, 32, 64, 16, 1, 16},
	                               {0, 64, 64, 16, 2, 8},   {1, 4096, 256, 0, 0, 0}, {1, 256, num_classes, 0, 0, 0}};
	std::mt19937_64 rng(seed);
	std::vector<float> params;
	for (int l = 0; l < NL; ++l) {
		net->L[l] = shapes[l];
		// He initialisation (unit variance for the logits' layer)
		std::normal_distribution<float> nd(0.f, std::sqrt((l < NL - 1 ? 2.f : 1.f) / shapes[l].fan_in()));
		for (long long k = 0; k < shapes[l].nw(); ++k)
			params.push_back(nd(rng));
		for (int k = 0; k < shapes[l].cout; ++k)
			params.push_back(0.f);
	}
	auto bad = [&](int rc) {
		dfg_pnet_destroy(net);
		return rc;
	};
	// forward buffers for the inference batch, backward ones for the
	// training batch
	net->infer_batch = std::max(batch, 2048);
	for (int l = 0; l < NL; ++l) {
		const LayerShape &s = net->L[l];
		const long long nw = s.nw(), rows = net->rows(l, batch), irows = net->rows(l, net->infer_batch);
		bool ok = net->w[l].ensure(nw) == cudaSuccess && net->mw[l].ensure(nw) == cudaSuccess &&
		          net->vw[l].ensure(nw) == cudaSuccess && net->gw[l].ensure(nw) == cudaSuccess &&
		          net->wb[l].ensure(nw) == cudaSuccess && net->b[l].ensure(s.cout) == cudaSuccess &&
		          net->mb[l].ensure(s.cout) == cudaSuccess && net->vb[l].ensure(s.cout) == cudaSuccess &&
		          net->gb[l].ensure(s.cout) == cudaSuccess && net->act[l + 1].ensure(irows * s.cout) == cudaSuccess &&
		          net->dact[l + 1].ensure(rows * s.cout) == cudaSuccess;
		if (ok && s.kind == 0)
			ok = net->cols[l].ensure(irows * 9 * s.cin) == cudaSuccess &&
			     net->dcols[l].ensure(rows * 9 * s.cin) == cudaSuccess;
		if (!ok)
			return bad(DFG_ERR_NOMEM);
		cudaMemsetAsync(net->mw[l].p, 0, nw * sizeof(float), net->stream);
		cudaMemsetAsync(net->vw[l].p, 0, nw * sizeof(float), net->stream);
		cudaMemsetAsync(net->mb[l].p, 0, s.cout * sizeof(float), net->stream);
		cudaMemsetAsync(net->vb[l].p, 0, s.cout * sizeof(float), net->stream);
	}
	long long ws = 0;
	for (int l = 0; l < NL; ++l) {
		int S, chunk;
		k_split(net->L[l].cout, net->L[l].fan_in(), net->rows(l, batch), &S, &chunk);
		if (S > 1)
			ws = std::max(ws, (long long)S * net->L[l].nw());
	}
	if (ws > 0 && net->wsplit.ensure(ws) != cudaSuccess)
		return bad(DFG_ERR_NOMEM);
	// tensor-core inference: BF16 operand rows (the largest layer) and padded weights
	long long cb = 0;
	for (int l = 1; l < NL; ++l) {
		const int Kp = (net->L[l].fan_in() + 63) / 64 * 64;
		cb = std::max(cb, net->rows(l, net->infer_batch) * Kp);
		if (net->wbp[l].ensure((size_t)net->L[l].cout * Kp) != cudaSuccess)
			return bad(DFG_ERR_NOMEM);
	}
	if (net->colsb.ensure((size_t)cb) != cudaSuccess || net->terr.ensure(1) != cudaSuccess)
		return bad(DFG_ERR_NOMEM);
	// tensor-core training: per layer the BF16 input rows of a training batch
	// and the transposed padded weights; the transposed output gradients (the
	// output count padded to 128 rows, zero past it), transposed input rows
	// and BF16 output gradients of the largest layer
	{
		long long dyt = 0, colst = 0, dyb = 0;
		for (int l = 1; l < NL; ++l) {
			const LayerShape &sh = net->L[l];
			const int K = sh.fan_in(), Kp = kpad64(K), cp = kpad64(sh.cout);
			const long long rows = net->rows(l, batch), rows_p = (rows + 63) / 64 * 64;
			if (net->colsbl[l].ensure((size_t)round128(rows) * Kp) != cudaSuccess ||
			    net->wtp[l].ensure((size_t)K * cp) != cudaSuccess)
				return bad(DFG_ERR_NOMEM);
			dyt = std::max(dyt, round128(sh.cout) * rows_p);
			colst = std::max(colst, (long long)Kp * rows_p);
			dyb = std::max(dyb, round128(rows) * cp);
		}
		if (net->dyt.ensure((size_t)dyt) != cudaSuccess || net->colst.ensure((size_t)colst) != cudaSuccess ||
		    net->dyb.ensure((size_t)dyb) != cudaSuccess)
			return bad(DFG_ERR_NOMEM);
		cudaMemsetAsync(net->dyt.p, 0, (size_t)dyt * sizeof(__nv_bfloat16), net->stream);
		for (int l = 1; l < NL; ++l)
			cudaMemsetAsync(net->colsbl[l].p, 0, net->colsbl[l].n * sizeof(__nv_bfloat16), net->stream);
		cudaMemsetAsync(net->dyb.p, 0, (size_t)dyb * sizeof(__nv_bfloat16), net->stream);
	}
	cudaMemsetAsync(net->terr.p, 0, sizeof(int), net->stream);
	if (net->loss_acc.ensure(1) != cudaSuccess)
		return bad(DFG_ERR_NOMEM);
	if (net->dact[0].ensure((long long)batch * IMG * IMG) != cudaSuccess ||
	    net->loss.ensure(batch) != cudaSuccess || net->labels.ensure(batch) != cudaSuccess ||
	    net->idx.ensure(batch) != cudaSuccess || net->xbatch.ensure((long long)batch * IMG * IMG) != cudaSuccess)
		return bad(DFG_ERR_NOMEM);
	if (upload_params(net, params.data()) != DFG_OK)
		return bad(DFG_ERR_CUDA);
	*out = net;
	return DFG_OK;
}

extern "C" const char *dfg_pnet_last_error(const dfg_pnet *net) { return net ? net->err.c_str() : "null network"; }

extern "C" int dfg_pnet_set_tensor_cores(dfg_pnet *net, int on) {
	if (!net)
		return DFG_ERR_ARG;
	net->use_tc = on != 0;
	return DFG_OK;
}

extern "C" int dfg_pnet_set_option(dfg_pnet *net, const char *key, double value) {
	if (!net || !key)
		return DFG_ERR_ARG;
	if (!strcmp(key, "tensor_cores"))
		return dfg_pnet_set_tensor_cores(net, value != 0.);
	if (!strcmp(key, "tensor_core_training")) {
		net->tc_train = value != 0.;
		return DFG_OK;
	}
	if (!strcmp(key, "wait_cycles")) {
		if (!(value >= 1e4 && value <= 1e11))
			return net->fail(DFG_ERR_ARG, "wait_cycles must be in [1e4, 1e11]");
		net->wait_cycles = (long long)value;
		return DFG_OK;
	}
	if (!strcmp(key, "withhold_stage")) {
		if (!(value >= -1 && value < 1e6))
			return net->fail(DFG_ERR_ARG, "withhold_stage must be -1 or a stage index");
		net->withhold = (int)value;
		return DFG_OK;
	}
	return net->fail(DFG_ERR_ARG, "unknown option %s", key);
}

extern "C" long long dfg_pnet_num_params(const dfg_pnet *net) {
	if (!net)
		return 0;
	long long n = 0;
	for (int l = 0; l < NL; ++l)
		n += net->L[l].nw() + net->L[l].cout;
	return n;
}

extern "C" int dfg_pnet_get_params(dfg_pnet *net, float *out) {
	if (!net || !out)
		return DFG_ERR_ARG;
	PK(cudaSetDevice(net->device));
	size_t o = 0;
	for (int l = 0; l < NL; ++l) {
		const long long nw = net->L[l].nw();
		PK(cudaMemcpyAsync(out + o, net->w[l].p, nw * sizeof(float), cudaMemcpyDeviceToHost, net->stream));
		o += nw;
		PK(cudaMemcpyAsync(out + o, net->b[l].p, net->L[l].cout * sizeof(float), cudaMemcpyDeviceToHost,
		                   net->stream));
		o += net->L[l].cout;
	}
	PK(cudaStreamSynchronize(net->stream));
	return DFG_OK;
}

extern "C" int dfg_pnet_set_params(dfg_pnet *net, const float *in) {
	if (!net || !in)
		return DFG_ERR_ARG;
	PK(cudaSetDevice(net->device));
	return upload_params(net, in);
}

extern "C" int dfg_pnet_set_bins(dfg_pnet *net, int num_pix, const int *pixel_bin) {
	if (!net || num_pix < 1 || !pixel_bin)
		return DFG_ERR_ARG;
	for (int p = 0; p < num_pix; ++p)
		if (pixel_bin[p] < -1 || pixel_bin[p] >= IMG * IMG)
			return net->fail(DFG_ERR_ARG, "pixel_bin[%d] = %d outside [-1, %d)", p, pixel_bin[p], IMG * IMG);
	PK(cudaSetDevice(net->device));
	PK(upload(net->pixel_bin, pixel_bin, (size_t)num_pix, net->stream));
	PK(cudaStreamSynchronize(net->stream));
	net->P = num_pix;
	return DFG_OK;
}

extern "C" int dfg_pnet_load_frames(dfg_pnet *net, dfg_ctx *ctx) {
	if (!net || !ctx)
		return DFG_ERR_ARG;
	if (ctx->N <= 0 || ctx->P != net->P)
		return net->fail(DFG_ERR_STATE, "the context's frames and detector (%d pixels) must match the bins (%d)",
		                 ctx->P, net->P);
	if (ctx->device != net->device)
		return net->fail(DFG_ERR_ARG, "context and network on different devices");
	PK(cudaSetDevice(net->device));
	PK(net->images.ensure((size_t)ctx->N * IMG * IMG));
	PK(cudaStreamSynchronize(ctx->stream));
	frame_image_kernel<<<ctx->N, 256, 0, net->stream>>>(ctx->ph.p, ctx->ph_off.p, ctx->ph_mid.p, net->pixel_bin.p,
	                                                    ctx->P, 0, ctx->N, net->images.p);
	PKL("frame_image_kernel");
	PK(cudaStreamSynchronize(net->stream));
	net->n_images = ctx->N;
	net->n_targets_images = -1;
	return DFG_OK;
}

extern "C" int dfg_pnet_set_images(dfg_pnet *net, long long n, const float *images) {
	if (!net || n < 1 || !images)
		return DFG_ERR_ARG;
	PK(cudaSetDevice(net->device));
	PK(upload(net->images, images, (size_t)n * IMG * IMG, net->stream));
	PK(cudaStreamSynchronize(net->stream));
	net->n_images = n;
	net->n_targets_images = -1;
	return DFG_OK;
}

extern "C" int dfg_pnet_get_images(dfg_pnet *net, float *out) {
	if (!net || !out)
		return DFG_ERR_ARG;
	PK(cudaSetDevice(net->device));
	PK(cudaMemcpy(out, net->images.p, (size_t)net->n_images * IMG * IMG * sizeof(float), cudaMemcpyDeviceToHost));
	return DFG_OK;
}

// Soft targets of the loaded images: image i's classes t_cls[t_off[i] ..
// t_off[i + 1]) with weights t_w (distinct classes, weights >= 0 summing to
// 1); used by dfg_pnet_train / dfg_pnet_gradients called without labels.
extern "C" int dfg_pnet_set_targets(dfg_pnet *net, const long long *t_off, const int *t_cls, const float *t_w) {
	if (!net || !t_off)
		return DFG_ERR_ARG;
	const long long n = net->n_images;
	if (n < 1)
		return net->fail(DFG_ERR_STATE, "no images loaded");
	if (t_off[0] != 0 || (t_off[n] > 0 && (!t_cls || !t_w)))
		return net->fail(DFG_ERR_ARG, "targets: t_off[0] must be 0 and classes / weights given");
	std::vector<long long> stamp((size_t)net->num_classes, -1);
	for (long long i = 0; i < n; ++i) {
		if (t_off[i + 1] < t_off[i])
			return net->fail(DFG_ERR_ARG, "targets: t_off decreases at image %lld", i);
		for (long long t = t_off[i]; t < t_off[i + 1]; ++t) {
			const int c = t_cls[t];
			if (c < 0 || c >= net->num_classes || stamp[c] == i || !(t_w[t] >= 0.f) || !std::isfinite(t_w[t]))
				return net->fail(DFG_ERR_ARG, "targets: image %lld: class %d repeated, out of range or bad weight", i,
				                 c);
			stamp[c] = i;
		}
	}
	PK(cudaSetDevice(net->device));
	PK(upload(net->t_off, t_off, (size_t)n + 1, net->stream));
	PK(upload(net->t_cls, t_cls ? t_cls : nullptr, (size_t)std::max<long long>(t_off[n], 0), net->stream));
	PK(upload(net->t_w, t_w ? t_w : nullptr, (size_t)std::max<long long>(t_off[n], 0), net->stream));
	std::vector<int> io((size_t)net->batch);
	for (int k = 0; k < net->batch; ++k)
		io[k] = k;
	PK(upload(net->iota, io.data(), io.size(), net->stream));
	PK(cudaStreamSynchronize(net->stream));
	net->n_targets_images = n;
	return DFG_OK;
}

extern "C" int dfg_pnet_train(dfg_pnet *net, const int *labels, int epochs, double lr, unsigned long long seed,
                              double *mean_loss) {
	if (!net || epochs < 1 || !(lr > 0.))
		return DFG_ERR_ARG;
	if (net->n_images < 1)
		return net->fail(DFG_ERR_STATE, "no images loaded");
	if (labels == nullptr && net->n_targets_images != net->n_images)
		return net->fail(DFG_ERR_STATE, "no labels and no soft targets for the loaded images");
	for (long long i = 0; labels && i < net->n_images; ++i)
		if (labels[i] < 0 || labels[i] >= net->num_classes)
			return net->fail(DFG_ERR_ARG, "label %d of image %lld outside [0, %d)", labels[i], i, net->num_classes);
	PK(cudaSetDevice(net->device));
	cudaStream_t st = net->stream;
	const long long n = net->n_images;
	// each epoch's shuffled order goes up once; batches are gathered on the
	// device and the losses summed there (one synchronisation per epoch)
	std::vector<int> perm((size_t)n);
	for (long long i = 0; i < n; ++i)
		perm[(size_t)i] = (int)i;
	if (labels)
		PK(upload(net->lab_all, labels, (size_t)n, st));
	PK(net->perm.ensure((size_t)n));
	std::mt19937_64 rng(seed);
	double last = 0.;
	for (int ep = 0; ep < epochs; ++ep) {
		std::shuffle(perm.begin(), perm.end(), rng);
		PK(cudaMemcpyAsync(net->perm.p, perm.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, st));
		PK(cudaMemsetAsync(net->loss_acc.p, 0, sizeof(double), st));
		for (long long b0 = 0; b0 < n; b0 += net->batch) {
			const int m = (int)std::min<long long>(net->batch, n - b0);
			gather_rows_kernel<<<grid_for((long long)m * IMG * IMG), 256, 0, st>>>(
			    net->images.p, net->perm.p + b0, m, IMG * IMG, net->xbatch.p, labels ? net->lab_all.p : nullptr,
			    net->labels.p);
			PKL("gather_rows_kernel");
			if (int rc = train_pass(net, net->xbatch.p, labels ? net->labels.p : nullptr, m, net->perm.p + b0))
				return rc;
			if (int rc = adam_step(net, (float)lr))
				return rc;
			loss_sum_kernel<<<1, 256, 0, st>>>(net->loss.p, m, net->loss_acc.p);
			PKL("loss_sum_kernel");
		}
		double sum = 0.;
		PK(cudaMemcpyAsync(&sum, net->loss_acc.p, sizeof(double), cudaMemcpyDeviceToHost, st));
		PK(cudaStreamSynchronize(st));
		if (net->tc_train)
			if (int rc = check_tc_flag(net))
				return rc;
		last = sum / (double)n;
	}
	if (mean_loss)
		*mean_loss = last;
	return DFG_OK;
}

// Runs fn(b0, m) over the loaded images in inference batches after a
// forward pass.
template <typename F>
static int for_batches(dfg_pnet *net, F fn) {
	if (net->use_tc)
		if (int rc = pad_weights(net))
			return rc;
	for (long long b0 = 0; b0 < net->n_images; b0 += net->infer_batch) {
		const int m = (int)std::min<long long>(net->infer_batch, net->n_images - b0);
		const float *X = net->images.p + (size_t)b0 * IMG * IMG;
		if (int rc = net->use_tc ? forward_tc(net, X, m) : forward(net, X, m))
			return rc;
		if (int rc = fn(b0, m))
			return rc;
	}
	return DFG_OK;
}

// After tensor-core products: a pipeline wait that gave up makes the results
// invalid (the flag is cleared for the next call).
static int check_tc(dfg_pnet *net) {
	if (!net->use_tc)
		return DFG_OK;
	return check_tc_flag(net);
}

static int check_tc_flag(dfg_pnet *net) {
	int e = 0;
	PK(cudaMemcpyAsync(&e, net->terr.p, sizeof(int), cudaMemcpyDeviceToHost, net->stream));
	PK(cudaStreamSynchronize(net->stream));
	if (e) {
		PK(cudaMemsetAsync(net->terr.p, 0, sizeof(int), net->stream));
		return net->fail(DFG_ERR_CUDA, "tensor-core product: a pipeline wait gave up (results invalid)");
	}
	return DFG_OK;
}

extern "C" int dfg_pnet_topk_mass(dfg_pnet *net, int K_min, int K_max, double mass, int *out) {
	if (!net || K_min < 1 || K_max < K_min || K_max > net->num_classes || !out || !(mass >= 0.))
		return DFG_ERR_ARG;
	PK(cudaSetDevice(net->device));
	DevBuf<int> d;  // every image's picks, read back once
	PK(d.ensure((size_t)net->n_images * K_max));
	if (int rc = for_batches(net, [&](long long b0, int m) -> int {
		    if (K_max <= SELK) {
			    topk_select_kernel<<<(m + 7) / 8, 256, 0, net->stream>>>(
			        net->act[NL].p, m, net->num_classes, K_min, K_max, (float)mass, d.p + (size_t)b0 * K_max);
			    PKL("topk_select_kernel");
		    } else {
			    topk_kernel<<<(m * 32 + 255) / 256, 256, 0, net->stream>>>(
			        net->act[NL].p, m, net->num_classes, K_min, K_max, (float)mass, d.p + (size_t)b0 * K_max);
			    PKL("topk_kernel");
		    }
		    return DFG_OK;
	    }))
		return rc;
	PK(cudaMemcpyAsync(out, d.p, (size_t)net->n_images * K_max * sizeof(int), cudaMemcpyDeviceToHost,
	                   net->stream));
	PK(cudaStreamSynchronize(net->stream));
	return check_tc(net);
}

extern "C" int dfg_pnet_topk(dfg_pnet *net, int K, int *out) {
	if (!net || K < 1 || !out)
		return DFG_ERR_ARG;
	return dfg_pnet_topk_mass(net, K, K, 2., out);
}

extern "C" int dfg_pnet_logits(dfg_pnet *net, float *out) {
	if (!net || !out)
		return DFG_ERR_ARG;
	PK(cudaSetDevice(net->device));
	if (int rc = for_batches(net, [&](long long b0, int m) -> int {
		    PK(cudaMemcpyAsync(out + (size_t)b0 * net->num_classes, net->act[NL].p,
		                       (size_t)m * net->num_classes * sizeof(float), cudaMemcpyDeviceToHost, net->stream));
		    PK(cudaStreamSynchronize(net->stream));
		    return DFG_OK;
	    }))
		return rc;
	return check_tc(net);
}

// Mean loss and gradients (flat, as dfg_pnet_get_params) of the first
// min(n_images, batch) loaded images with the given labels; no update.
extern "C" int dfg_pnet_gradients(dfg_pnet *net, const int *labels, float *grads, double *mean_loss) {
	if (!net || !grads)
		return DFG_ERR_ARG;
	if (net->n_images < 1)
		return net->fail(DFG_ERR_STATE, "no images loaded");
	if (labels == nullptr && net->n_targets_images != net->n_images)
		return net->fail(DFG_ERR_STATE, "no labels and no soft targets for the loaded images");
	PK(cudaSetDevice(net->device));
	const int m = (int)std::min<long long>(net->batch, net->n_images);
	if (labels)
		PK(cudaMemcpyAsync(net->labels.p, labels, m * sizeof(int), cudaMemcpyHostToDevice, net->stream));
	if (int rc = train_pass(net, net->images.p, labels ? net->labels.p : nullptr, m, net->iota.p))
		return rc;
	size_t o = 0;
	for (int l = 0; l < NL; ++l) {
		const long long nw = net->L[l].nw();
		PK(cudaMemcpyAsync(grads + o, net->gw[l].p, nw * sizeof(float), cudaMemcpyDeviceToHost, net->stream));
		o += nw;
		PK(cudaMemcpyAsync(grads + o, net->gb[l].p, net->L[l].cout * sizeof(float), cudaMemcpyDeviceToHost,
		                   net->stream));
		o += net->L[l].cout;
	}
	std::vector<float> loss((size_t)m);
	PK(cudaMemcpyAsync(loss.data(), net->loss.p, m * sizeof(float), cudaMemcpyDeviceToHost, net->stream));
	PK(cudaStreamSynchronize(net->stream));
	if (net->tc_train)
		if (int rc = check_tc_flag(net))
			return rc;
	double s = 0.;
	for (float v : loss)
		s += v;
	if (mean_loss)
		*mean_loss = s / m;
	return DFG_OK;
}
