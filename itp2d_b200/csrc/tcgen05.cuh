// Device helpers shared by the tensor-core contraction kernels (tc.cu: BF16
// planes; oz.cu: int8 slices): shared-memory and instruction descriptors,
// tcgen05.mma issue and commit, mbarriers with bounded waits, bulk copies and
// tensor-memory loads. All operands are K-major without swizzle: 8-row x
// 16-byte core matrices, the two 16-byte K halves of a row group 128 B apart
// (LBO), row groups 256 B apart (SBO).
#pragma once

#include <stdint.h>

namespace itp2d {
namespace tcg {

constexpr long long kSpinLimit = 1LL << 24;            // back-stop on the number of polls
constexpr unsigned long long kWaitNs = 1000000000ULL;  // a wait gives up after 1 s

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: K-major, no swizzle, version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
	const uint64_t lbo = 128, sbo = 256;
	uint64_t d = 0;
	d |= (uint64_t)((saddr >> 4) & 0x3FFF);
	d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
	d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
	d |= (uint64_t)1 << 46;
	return d;
}

// Instruction descriptors, K-major A and B, M = 128:
//   BF16 x BF16 -> F32 (kind::f16), optional negation of A;
//   S8 x S8 -> S32 (kind::i8).
__host__ __device__ constexpr uint32_t idesc_bf16(int n, bool negate_a) {
	return (1u << 4) | (1u << 7) | (1u << 10) | ((negate_a ? 1u : 0u) << 13) | ((uint32_t)(n >> 3) << 17) |
	       ((uint32_t)(128 >> 4) << 24);
}
__host__ __device__ constexpr uint32_t idesc_s8(int n) {
	return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

// D (tensor memory) = A B (+ D when acc != 0); one thread issues.
__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
	const uint32_t z = 0;
	asm volatile(
			"{\n\t.reg .pred p;\n\t"
			"setp.ne.b32 p, %4, 0;\n\t"
			"tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
			:
			: "r"(tmem_d), "l"(a), "l"(b), "r"(id), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}
__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
	const uint32_t z = 0;
	asm volatile(
			"{\n\t.reg .pred p;\n\t"
			"setp.ne.b32 p, %4, 0;\n\t"
			"tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
			:
			: "r"(tmem_d), "l"(a), "l"(b), "r"(id), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

// The mbarrier completes once every MMA issued before it by this thread has.
__device__ __forceinline__ void umma_commit(uint32_t mbar) {
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
	unsigned long long t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

// Bounded wait for the phase with the given parity: false once kWaitNs of
// wall time (or kSpinLimit polls) passed without the phase completing.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
	const unsigned long long t0 = global_ns();
	for (long long i = 0; i < kSpinLimit; i++) {
		uint32_t done;
		asm volatile(
				"{\n\t.reg .pred P1;\n\t"
				"mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
				"selp.b32 %0, 1, 0, P1;\n\t}\n"
				: "=r"(done)
				: "r"(mbar), "r"(parity)
				: "memory");
		if (done) return true;
		if (i > 64) {
			__nanosleep(64);
			if ((i & 255) == 0 && global_ns() - t0 > kWaitNs) return false;
		}
	}
	return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

// Contiguous global -> shared copy (16-byte aligned, size a multiple of 16)
// completing on an mbarrier's transaction count.
__device__ __forceinline__ void bulk_copy(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
			"l"(src), "r"(bytes), "r"(mbar)
			: "memory");
}

// 32 consecutive 32-bit columns of this warp's 32 tensor-memory lanes.
__device__ __forceinline__ void tmem_ld32_raw(uint32_t taddr, uint32_t* r) {
	asm volatile(
			"tcgen05.ld.sync.aligned.32x32b.x32.b32 "
			"{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
			"%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
			: "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
			  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
			  "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
			  "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
			: "r"(taddr));
	asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
	uint32_t r[32];
	tmem_ld32_raw(taddr, r);
#pragma unroll
	for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// Tensor-memory allocation of `cols` columns by warp 0 (address into *slot).
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {
	asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(cols)
			: "memory");
	asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t cols) {
	asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols) : "memory");
}

}  // namespace tcg
}  // namespace itp2d
