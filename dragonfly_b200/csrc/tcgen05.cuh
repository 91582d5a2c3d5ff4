// tcgen05 / TMA building blocks shared by the tensor-core kernels (the dense
// E-step and M-step, the proposal network's products): mbarriers with
// bounded waits, 2-D tiled TMA loads, shared-memory matrix descriptors with
// the 128-byte swizzle, kind::f16 MMAs with TMEM accumulators and TMEM loads.
#pragma once

#include <cuda.h>
#include <cstdint>

namespace dfg {

constexpr long long TC_WAIT_CYCLES = 2000000000LL;  // about one second

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
	return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
	             : "memory");
}

// Waits for the phase of the given parity to complete; false after `limit`
// clock cycles (about a second by default; the caller then gives up).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit = TC_WAIT_CYCLES) {
	const long long t0 = clock64();
	while (true) {
		uint32_t done;
		asm volatile(
		    "{\n\t.reg .pred p;\n\t"
		    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		    "selp.u32 %0, 1, 0, p;\n\t}"
		    : "=r"(done)
		    : "r"(smem_addr(bar)), "r"(parity)
		    : "memory");
		if (done)
			return true;
		if (clock64() - t0 > limit)
			return false;
	}
}

// 2-D tiled TMA load into this CTA's shared memory, completing on bar.
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y) {
	asm volatile(
	    "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], "
	    "[%2];" ::"r"(smem_addr(dst)),
	    "l"((uint64_t)map), "r"(smem_addr(bar)), "r"(x), "r"(y)
	    : "memory");
}

// Shared-memory matrix descriptor of a K-major tile with 128-byte swizzle:
// rows of 128 bytes, 8-row groups 1024 bytes apart (SBO), version 1,
// layout type 2 (SWIZZLE_128B).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
	return (uint64_t)((addr & 0x3FFFF) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
	       ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// One tcgen05.mma of kind::f16 (cta_group::1) with instruction descriptor
// idesc; accumulate = 0 overwrites the accumulator.
__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
	asm volatile(
	    "{\n\t.reg .pred p;\n\t"
	    "setp.ne.b32 p, %4, 0;\n\t"
	    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
	    "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
	    : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
	                 smem_addr(bar))
	             : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive 32-bit TMEM columns of this thread's lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
	uint32_t r[16];
	asm volatile(
	    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
	    "%14, %15}, [%16];"
	    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
	      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
	    : "r"(taddr));
	asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
	for (int k = 0; k < 16; ++k)
		v[k] = __uint_as_float(r[k]);
}

}  // namespace dfg
