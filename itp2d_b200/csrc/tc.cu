// Orthonormalisation contractions of the FP32 form on the 5th-generation
// tensor cores (tcgen05.mma kind::f16, BF16 operands, FP32 accumulation in
// tensor memory).
//
//   overlap:  S_ij = sum_g conj(psi_i[g]) psi_j[g]        (stateset.cpp:146-154)
//   rotation: out_n[g] = sum_i W[i][n] psi_i[g]           (stateset.cpp:214-228)
//
// Every FP32 operand value x is split into three BF16 parts x = h + m + l
// (24 significant bits), and each real product x*y is formed from the six
// partial products h h, h m, m h, h l, l h, m m; the dropped terms are below
// 2^-24 relative. A complex product takes four real products; the imaginary
// part's "- Ai Br" term uses the instruction descriptor's negate-A bit.
//
// Each MMA rounds its FP32 accumulator once, with an error relative to the
// accumulator's magnitude, so the h h products (the bulk of the sum) go to
// their own accumulator and the five smaller products to a second one, whose
// rounding errors are 2^-8 smaller relative to the result; the epilogue adds
// the two in FP64. The overlap bounds the K range one accumulator sees (grid
// chunks, summed in FP64 afterwards).
//
// One CTA (8 warps) owns a 128 x 128 output tile in tensor memory (512
// columns: large-part real, imaginary, small-part real, imaginary). K
// advances 16 per step (one MMA depth).
//
// Two engines issue the same MMAs in the same order (bit-identical results):
//   * pre-split (the default): split_psi_rows_kernel / split_psi_cols_kernel
//     write the planes of the states once per contraction, in the MMA block
//     layout; overlap_tc2_kernel / rotate_tc2_kernel then run their K loop in
//     one thread: a cp.async.bulk of each 24 KB block into a ring of four
//     slots (full mbarrier), the 24 MMAs, tcgen05.commit to the slot's empty
//     mbarrier, and the refill of the previous step's slot;
//   * staged (ITP2D_CONTRACT_TC_STAGED): overlap_tc_kernel / rotate_tc_kernel
//     split inside the CTA. Per step:
//   * cp.async fetches the FP32 operand tiles of step s + 2 into a ring of
//     three raw slots (16-byte pieces, XOR-swizzled against bank conflicts);
//   * all threads split the raw tile of step s into six BF16 planes in the
//     K-major canonical layout without swizzle (8 x 16-byte core matrices,
//     LBO 128 B between the two K halves, SBO 256 B between 8-row groups),
//     one core matrix per warp store;
//   * one thread issues the 24 MMAs and commits them to an mbarrier; two
//     plane buffers let the split of step s + 1 overlap the MMAs of step s.
// The rotation's A operand W^T is split once per call by split_w_kernel into
// global memory in exactly the shared-memory plane layout, and cp.async copies
// it into a ring of four plane slots that the MMAs read in place.
//
// Waits on mbarriers are bounded: on time-out the kernel records
// ITP2D_E_TIMEOUT, waits (bounded) for its MMAs, frees its tensor memory and
// returns.
#include <cuda_bf16.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/itp2d_gpu.h"
#include "contract.cuh"
#include "tcgen05.cuh"

namespace itp2d {

namespace {

using namespace tcg;

constexpr int TM = 128;                                // tile rows (M)
constexpr int TN = 128;                                // tile cols (N)
constexpr int KT = 16;                                 // K per step
constexpr int kThreads = 256;
constexpr int kPlaneBytes = TM * KT * 2;               // 4 KB: one BF16 plane of a 128 x 16 operand
constexpr int kOperandBytes = 6 * kPlaneBytes;         // 24 KB: re/im x hi/mid/lo
constexpr int kRawRowBytes = KT * 8;                   // 128 B: 16 complex FP32
constexpr int kTmemCols = 512;

// Shared memory map (bytes from the 1024-aligned base).
//   overlap:  planes[2] x (A, B) 96 KB | raw[3] x (A, B) 96 KB
//   rotation: B planes[2] 48 KB | A plane ring[4] 96 KB | raw psi[3] 48 KB
constexpr int kBufBytes = 192 * 1024;
constexpr int kOvPlanes = 0;
constexpr int kOvRaw = 2 * 2 * kOperandBytes;
constexpr int kOvRawSlot = 2 * TM * kRawRowBytes;      // 32 KB
constexpr int kRoB = 0;
constexpr int kRoA = 2 * kOperandBytes;
constexpr int kRoRaw = kRoA + 4 * kOperandBytes;
constexpr int kRoRawSlot = KT * TN * 8;                // 16 KB: 16 rows (i) x 128 complex (g)
static_assert(kOvRaw + 3 * kOvRawSlot <= kBufBytes, "overlap shared memory");
static_assert(kRoRaw + 3 * kRoRawSlot <= kBufBytes, "rotation shared memory");
static_assert(8 * 32 * 33 * 16 <= kBufBytes, "epilogue staging");

// Instruction descriptor: BF16 x BF16 -> F32, K-major A and B, M = 128, N = 128.
__host__ __device__ constexpr uint32_t idesc(bool negate_a) { return idesc_bf16(TN, negate_a); }

// 16-byte global -> shared copy; src_bytes = 0 writes zeros without reading.
__device__ __forceinline__ void cp16(uint32_t dst, const void* src, int src_bytes) {
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Byte offset of element (row r, k) of a K-major no-swizzle 128 x 16 plane:
// core matrix (r / 8, k / 8) at ((r / 8) * 2 + k / 8) * 128, rows 16 B apart.
__host__ __device__ __forceinline__ uint32_t kmaj_off(int r, int k) {
	return (uint32_t)((((r >> 3) << 1) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// Three-way BF16 split of two FP32 values at once (x = h + m + l exactly:
// each remainder is exact in FP32), with packed round-to-nearest
// conversions; returns the h, m and l parts as bf16x2 words, x0 in the low
// half.
__device__ __forceinline__ void split3x2(float x0, float x1, uint32_t& h, uint32_t& m, uint32_t& l) {
	const __nv_bfloat162 bh = __floats2bfloat162_rn(x0, x1);
	const float2 fh = __bfloat1622float2(bh);
	const float r0 = x0 - fh.x, r1 = x1 - fh.y;
	const __nv_bfloat162 bm = __floats2bfloat162_rn(r0, r1);
	const float2 fm = __bfloat1622float2(bm);
	const __nv_bfloat162 bl = __floats2bfloat162_rn(r0 - fm.x, r1 - fm.y);
	h = *reinterpret_cast<const uint32_t*>(&bh);
	m = *reinterpret_cast<const uint32_t*>(&bm);
	l = *reinterpret_cast<const uint32_t*>(&bl);
}

// Writes two consecutive K elements (k even) of row r, split into the six
// planes of one operand: planes 0..2 real hi/mid/lo, 3..5 imaginary.
__device__ __forceinline__ void put2(unsigned char* op, uint32_t off, float re0, float im0, float re1, float im1) {
	uint32_t h, m, l;
	split3x2(re0, re1, h, m, l);
	*reinterpret_cast<uint32_t*>(op + 0 * kPlaneBytes + off) = h;
	*reinterpret_cast<uint32_t*>(op + 1 * kPlaneBytes + off) = m;
	*reinterpret_cast<uint32_t*>(op + 2 * kPlaneBytes + off) = l;
	split3x2(im0, im1, h, m, l);
	*reinterpret_cast<uint32_t*>(op + 3 * kPlaneBytes + off) = h;
	*reinterpret_cast<uint32_t*>(op + 4 * kPlaneBytes + off) = m;
	*reinterpret_cast<uint32_t*>(op + 5 * kPlaneBytes + off) = l;
}

// The 24 MMAs of one step. Accumulators: h h products in columns 0..255
// (real 0..127, imaginary 128..255), the other five in 256..511 likewise.
// conjA selects conj(A) B (overlap) instead of A B (rotation).
__device__ __forceinline__ void issue_step(uint32_t tmem, uint32_t abase, uint32_t bbase, bool conjA, bool first) {
	const uint32_t id = idesc(false), idn = idesc(true);
#pragma unroll
	for (int t = 0; t < 6; t++) {
		// split pairs (p, q): hh, hm, mh, hl, lh, mm
		const int p = (t == 2 || t == 5) ? 1 : (t == 4 ? 2 : 0);
		const int q = (t == 1 || t == 5) ? 1 : (t == 3 ? 2 : 0);
		const uint32_t cre = tmem + (t == 0 ? 0 : 2 * TN), cim = cre + TN;
		const uint32_t acc = (first && t <= 1) ? 0u : 1u;
		const uint64_t ar = sdesc(abase + p * kPlaneBytes), ai = sdesc(abase + (3 + p) * kPlaneBytes);
		const uint64_t br = sdesc(bbase + q * kPlaneBytes), bi = sdesc(bbase + (3 + q) * kPlaneBytes);
		// (a) A B:        re = ar br - ai bi,  im = ar bi + ai br
		// (b) conj(A) B:  re = ar br + ai bi,  im = ar bi - ai br
		umma_f16(cre, ar, br, id, acc);
		umma_f16(cre, ai, bi, conjA ? id : idn, 1u);
		umma_f16(cim, ar, bi, id, acc);
		umma_f16(cim, ai, br, conjA ? idn : id, 1u);
	}
}

struct TcShared {
	alignas(1024) unsigned char buf[kBufBytes];
	alignas(8) unsigned long long mbar[2];
	uint32_t tmem_base;
	int abort;
};

__device__ TcShared& tc_shared() {
	extern __shared__ __align__(1024) unsigned char smem_raw[];
	return *reinterpret_cast<TcShared*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
}

__device__ void tc_setup(TcShared& sh) {
	if (threadIdx.x < 32) tmem_alloc(&sh.tmem_base, kTmemCols);
	if (threadIdx.x == 0) {
		mbar_init(smem_u32(&sh.mbar[0]), 1);
		mbar_init(smem_u32(&sh.mbar[1]), 1);
		sh.abort = 0;
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
}

__device__ void tc_teardown(TcShared& sh) {
	tc_fence_before();
	__syncthreads();
	if (threadIdx.x < 32) tmem_dealloc(sh.tmem_base, kTmemCols);
}

// The step pipeline. prefetch(s) issues the cp.async copies of step s (called
// for s < nsteps only; one group is committed per step whether or not it
// copies, so that group counting stays uniform). convert(s) turns the raw
// slot of step s into the plane buffer s & 1. a_addr(s) / b_addr(s) give the
// shared-memory bases the MMAs of step s read. Returns with the accumulators
// complete, or with sh.abort set.
template <class Prefetch, class Convert, class AAddr, class BAddr>
__device__ void run_pipeline(TcShared& sh, int nsteps, bool conjA, Prefetch prefetch, Convert convert, AAddr a_addr,
		BAddr b_addr, int* err) {
	const int tid = threadIdx.x;
	const uint32_t mb0 = smem_u32(&sh.mbar[0]), mb1 = smem_u32(&sh.mbar[1]);
	if (nsteps > 0) prefetch(0);
	cp_commit();
	if (nsteps > 1) prefetch(1);
	cp_commit();
	int ran = 0;
	for (int s = 0; s < nsteps; s++) {
		if (s >= 2) {  // the MMAs of step s - 2 read the plane buffer (and ring slot) reused now
			const bool ok = mbar_wait((s & 1) ? mb1 : mb0, (uint32_t)(((s >> 1) - 1) & 1));
			if (!__syncthreads_and(ok)) {
				if (tid == 0) {
					sh.abort = 1;
					atomicExch(err, ITP2D_E_TIMEOUT);
				}
				break;
			}
		}
		if (s + 2 < nsteps) prefetch(s + 2);
		cp_commit();
		cp_wait<2>();  // this thread's copies of step s have landed
		__syncthreads();
		convert(s);
		proxy_fence();
		__syncthreads();
		if (tid == 0) {
			tc_fence_after();
			issue_step(sh.tmem_base, a_addr(s), b_addr(s), conjA, s == 0);
			umma_commit((s & 1) ? mb1 : mb0);
		}
		ran = s + 1;
	}
	cp_wait<0>();
	// drain: the last commit of each barrier (bounded, also after an abort)
	for (int b = 0; b < 2; b++) {
		const int commits = (ran - b + 1) / 2;
		if (commits <= 0) continue;
		const bool ok = mbar_wait(b ? mb1 : mb0, (uint32_t)((commits - 1) & 1));
		if (!__syncthreads_and(ok) && tid == 0) {
			sh.abort = 1;
			atomicExch(err, ITP2D_E_TIMEOUT);
		}
	}
	tc_fence_after();
	__syncthreads();
}

// Epilogue: the tile (large and small accumulators added in FP64) leaves
// through a per-warp 32 x 32 staging square in the idle pipeline buffers, so
// that each global store of a warp covers 32 consecutive columns of one row.
// Warp w reads TMEM lanes 32 (w % 4) .. + 31 and columns 64 (w / 4) .. + 63.
// emit(r, c, re, im) stores one element.
template <class Emit>
__device__ void store_tile(TcShared& sh, Emit emit) {
	const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int q = w & 3, half = w >> 2;
	double2* buf = reinterpret_cast<double2*>(sh.buf) + w * 32 * 33;
	const uint32_t trow = sh.tmem_base + ((uint32_t)(q * 32) << 16);
	for (int c = half * 64; c < half * 64 + 64; c += 32) {
		float big[32], small[32];
		tmem_ld32(trow + c, big);
		tmem_ld32(trow + 2 * TN + c, small);
#pragma unroll
		for (int j = 0; j < 32; j++) buf[lane * 33 + j].x = (double)big[j] + (double)small[j];
		tmem_ld32(trow + TN + c, big);
		tmem_ld32(trow + 3 * TN + c, small);
#pragma unroll
		for (int j = 0; j < 32; j++) buf[lane * 33 + j].y = (double)big[j] + (double)small[j];
		__syncwarp();
		for (int r = 0; r < 32; r++) {
			const double2 v = buf[r * 33 + lane];
			emit(q * 32 + r, c + lane, v.x, v.y);
		}
		__syncwarp();
	}
}

// Overlap tile pair (ti <= tj) from blockIdx.x, K range [g0, g1) from
// blockIdx.y; writes the partial S block of split blockIdx.y.
__global__ void __launch_bounds__(kThreads, 1) overlap_tc_kernel(const float2* __restrict__ psi, int k, long long G,
		int ntiles, long long chunk, double2* __restrict__ part, int* err) {
	TcShared& sh = tc_shared();
	int p = blockIdx.x, ti = 0;
	while (p >= ntiles - ti) {
		p -= ntiles - ti;
		ti++;
	}
	const int tj = ti + p;
	const int i0 = ti * TM, j0 = tj * TN;
	const long long g0 = (long long)blockIdx.y * chunk;
	const long long g1 = min(G, g0 + chunk);
	const int nsteps = (int)((g1 - g0 + KT - 1) / KT);
	tc_setup(sh);
	const int tid = threadIdx.x;
	unsigned char* const base = sh.buf;
	// a diagonal tile pair (ti == tj) has one operand: B reads A's planes
	const bool diag = ti == tj;
	// raw slot: operand o (0 = rows i0.., 1 = rows j0..), row r, 16-byte piece
	// pc (two complex) stored at slot pc ^ 4 (r & 1)
	auto fetch = [&](unsigned char* slot, long long gb, int it) {
		const int idx = it * kThreads + tid;  // 0..2047
		const int o = idx >> 10, r = (idx >> 3) & 127, pc = idx & 7;
		const int row = (o ? j0 : i0) + r;
		const long long g = gb + 2 * pc;
		const bool in = row < k && g < g1;  // g even, g1 even: both complex in range
		const float2* src = in ? psi + (long long)row * G + g : psi;
		cp16(smem_u32(slot + o * (TM * kRawRowBytes) + r * kRawRowBytes + ((pc ^ ((r & 1) << 2)) << 4)), src,
				in ? 16 : 0);
	};
	auto prefetch = [&](int s) {
		unsigned char* slot = base + kOvRaw + (s % 3) * kOvRawSlot;
		const long long gb = g0 + (long long)s * KT;
#pragma unroll
		for (int it = 0; it < 4; it++) fetch(slot, gb, it);
		if (!diag) {
#pragma unroll
			for (int it = 4; it < 8; it++) fetch(slot, gb, it);
		}
	};
	// convert: warp w handles core matrices m = w, w + 8, ... of the 64 (two
	// operands x 16 row groups x 2 K halves); lane = (row in group) * 4 + pair
	auto convert_one = [&](const unsigned char* slot, unsigned char* planes, int it) {
		const int w = tid >> 5, lane = tid & 31;
		const int m = it * 8 + w;
		const int o = m >> 5, rg = (m >> 1) & 15, kc = m & 1;
		const int r = rg * 8 + (lane >> 2), kk = kc * 8 + (lane & 3) * 2;
		const int pc = kk >> 1;
		const float4 v = *reinterpret_cast<const float4*>(
				slot + o * (TM * kRawRowBytes) + r * kRawRowBytes + ((pc ^ ((r & 1) << 2)) << 4));
		put2(planes + o * kOperandBytes, kmaj_off(r, kk), v.x, v.y, v.z, v.w);
	};
	auto convert = [&](int s) {
		const unsigned char* slot = base + kOvRaw + (s % 3) * kOvRawSlot;
		unsigned char* planes = base + kOvPlanes + (s & 1) * 2 * kOperandBytes;
#pragma unroll
		for (int it = 0; it < 4; it++) convert_one(slot, planes, it);
		if (!diag) {
#pragma unroll
			for (int it = 4; it < 8; it++) convert_one(slot, planes, it);
		}
	};
	auto a_addr = [&](int s) { return smem_u32(base + kOvPlanes + (s & 1) * 2 * kOperandBytes); };
	auto b_addr = [&](int s) {
		return smem_u32(base + kOvPlanes + (s & 1) * 2 * kOperandBytes + (diag ? 0 : kOperandBytes));
	};
	run_pipeline(sh, nsteps, true, prefetch, convert, a_addr, b_addr, err);
	if (!sh.abort) {
		double2* out = part + (size_t)blockIdx.y * k * k;
		store_tile(sh, [&](int r, int c, double re, double im) {
			const int i = i0 + r, j = j0 + c;
			if (i < k && j < k) out[(size_t)i * k + j] = make_double2(re, im);
		});
	}
	tc_teardown(sh);
}

// W^T split into BF16 planes, in the shared-memory layout of the rotation's A
// operand: block (n tile nt, K step s) of kOperandBytes at
// (nt * ksteps + s) * kOperandBytes; rows n, K index i; zero outside k x k.
// One warp per core matrix (lane = row in group * 4 + K pair).
__global__ void split_w_kernel(const double2* __restrict__ W, int k, int ksteps, int ntiles,
		unsigned char* __restrict__ out) {
	const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	const long long total = (long long)ntiles * ksteps * 32;  // 32 core matrices per block
	if (warp >= total) return;
	const int m = (int)(warp & 31);
	const long long blk = warp >> 5;
	const int s = (int)(blk % ksteps);
	const int nt = (int)(blk / ksteps);
	const int rg = m >> 1, kc = m & 1;
	const int r = rg * 8 + (lane >> 2), kk = kc * 8 + (lane & 3) * 2;
	const int n = nt * TM + r, i = s * KT + kk;
	double2 w0 = make_double2(0.0, 0.0), w1 = w0;
	if (n < k) {
		if (i < k) w0 = W[(size_t)i * k + n];
		if (i + 1 < k) w1 = W[(size_t)(i + 1) * k + n];
	}
	put2(out + blk * kOperandBytes, kmaj_off(r, kk), (float)w0.x, (float)w0.y, (float)w1.x, (float)w1.y);
}

// ---------------------------------------------------------------------------
// Pre-split operands. The FP32 states are split into the six BF16 planes once
// per contraction, in the same block layout as split_w_kernel's W^T, so that
// the contraction kernels only copy 24 KB blocks (one cp.async.bulk each) and
// issue MMAs: no split work and no block-wide barrier per K step.
//   rows layout (overlap): block (state tile ti, grid step gs) at
//     (ti * gsteps + gs) * kOperandBytes; rows = states, K = grid points;
//   cols layout (rotation's B): block (grid tile gt, state step s) at
//     (gt * ksteps + s) * kOperandBytes; rows = grid points, K = states.
// Zero outside k x G. One warp per core matrix (lane = row in group * 4 + K
// pair), as in split_w_kernel.

__global__ void split_psi_rows_kernel(const float2* __restrict__ psi, int k, long long G, int ntiles,
		long long gsteps, unsigned char* __restrict__ out) {
	const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (warp >= (long long)ntiles * gsteps * 32) return;
	const int m = (int)(warp & 31);
	const long long blk = warp >> 5;
	const long long gs = blk % gsteps;
	const int ti = (int)(blk / gsteps);
	const int rg = m >> 1, kc = m & 1;
	const int r = rg * 8 + (lane >> 2), kk = kc * 8 + (lane & 3) * 2;
	const int i = ti * TM + r;
	const long long g = gs * KT + kk;  // even; G even: g and g + 1 in range together
	float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
	if (i < k && g < G) v = *reinterpret_cast<const float4*>(psi + (long long)i * G + g);
	put2(out + blk * kOperandBytes, kmaj_off(r, kk), v.x, v.y, v.z, v.w);
}

__global__ void split_psi_cols_kernel(const float2* __restrict__ psi, int k, long long G, long long gtiles,
		int ksteps, unsigned char* __restrict__ out) {
	const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (warp >= gtiles * ksteps * 32) return;
	const int m = (int)(warp & 31);
	const long long blk = warp >> 5;
	const int s = (int)(blk % ksteps);
	const long long gt = blk / ksteps;
	const int rg = m >> 1, kc = m & 1;
	const int r = rg * 8 + (lane >> 2), kk = kc * 8 + (lane & 3) * 2;
	const long long g = gt * TN + r;
	const int i = s * KT + kk;
	float2 a = make_float2(0.f, 0.f), b = a;
	if (g < G) {
		if (i < k) a = psi[(long long)i * G + g];
		if (i + 1 < k) b = psi[(long long)(i + 1) * G + g];
	}
	put2(out + blk * kOperandBytes, kmaj_off(r, kk), a.x, a.y, b.x, b.y);
}

constexpr int kRing = 4;                      // slots of (A, B) block pairs
constexpr int kSlotBytes = 2 * kOperandBytes;  // 48 KB
static_assert(kRing * kSlotBytes <= kBufBytes, "pre-split ring");

// The K loop over pre-split blocks, run by thread 0 alone: block pair s is
// copied into slot s mod kRing (full[slot] completes when it has landed),
// its MMAs are issued and committed to empty[slot]; after the MMAs of step s
// are issued, the slot of step s - 1 is refilled with step s - 1 + kRing once
// those MMAs have finished reading it. src_a(s) / src_b(s) give the global
// blocks (src_b null: B reads A's planes). Returns with every MMA complete or
// with sh.abort set (copies and MMAs in flight drained, bounded).
template <class SrcA, class SrcB>
__device__ void run_bulk_pipeline(TcShared& sh, unsigned long long* full, unsigned long long* empty, int nsteps,
		bool conjA, SrcA src_a, SrcB src_b, int* err) {
	if (threadIdx.x != 0 || nsteps <= 0) return;
	unsigned char* const base = sh.buf;
	auto copy = [&](int st) {
		const int slot = st % kRing;
		unsigned char* dst = base + slot * kSlotBytes;
		const unsigned char* b = src_b(st);
		const uint32_t fb = smem_u32(&full[slot]);
		mbar_expect_tx(fb, b ? 2 * kOperandBytes : kOperandBytes);
		bulk_copy(smem_u32(dst), src_a(st), kOperandBytes, fb);
		if (b) bulk_copy(smem_u32(dst + kOperandBytes), b, kOperandBytes, fb);
	};
	int copied = 0, issued = 0;  // steps copied / whose MMAs were issued
	for (; copied < nsteps && copied < kRing; copied++) copy(copied);
	bool ok = true;
	for (int st = 0; st < nsteps; st++) {
		const int slot = st % kRing;
		if (!mbar_wait(smem_u32(&full[slot]), (uint32_t)((st / kRing) & 1))) {
			ok = false;
			break;
		}
		tc_fence_after();
		const uint32_t a = smem_u32(base + slot * kSlotBytes);
		issue_step(sh.tmem_base, a, src_b(st) ? a + kOperandBytes : a, conjA, st == 0);
		umma_commit(smem_u32(&empty[slot]));
		issued = st + 1;
		if (st >= 1 && copied < nsteps) {
			const int ps = (st - 1) % kRing;
			if (!mbar_wait(smem_u32(&empty[ps]), (uint32_t)(((st - 1) / kRing) & 1))) {
				ok = false;
				break;
			}
			copy(copied++);
		}
	}
	if (!ok) {
		sh.abort = 1;
		atomicExch(err, ITP2D_E_TIMEOUT);
		// copies not yet waited for land before the CTA leaves
		for (int st = issued; st < copied; st++) mbar_wait(smem_u32(&full[st % kRing]), (uint32_t)((st / kRing) & 1));
	}
	// the last commit covers every MMA issued before it
	if (issued > 0 && !mbar_wait(smem_u32(&empty[(issued - 1) % kRing]), (uint32_t)(((issued - 1) / kRing) & 1))) {
		sh.abort = 1;
		atomicExch(err, ITP2D_E_TIMEOUT);
	}
}

__device__ void init_ring(unsigned long long* full, unsigned long long* empty) {
	if (threadIdx.x == 0)
		for (int i = 0; i < kRing; i++) {
			mbar_init(smem_u32(&full[i]), 1);
			mbar_init(smem_u32(&empty[i]), 1);
		}
}

// Overlap from the rows layout: tile pair (ti <= tj) from blockIdx.x, grid
// steps [g0 / KT, g1 / KT) from blockIdx.y; the same MMAs in the same order
// as overlap_tc_kernel.
__global__ void __launch_bounds__(kThreads, 1) overlap_tc2_kernel(const unsigned char* __restrict__ rows, int k,
		long long G, int ntiles, long long gsteps, long long chunk, double2* __restrict__ part, int* err) {
	TcShared& sh = tc_shared();
	__shared__ alignas(8) unsigned long long full[kRing], empty[kRing];
	int p = blockIdx.x, ti = 0;
	while (p >= ntiles - ti) {
		p -= ntiles - ti;
		ti++;
	}
	const int tj = ti + p;
	const int i0 = ti * TM, j0 = tj * TN;
	const long long g0 = (long long)blockIdx.y * chunk;
	const long long g1 = min(G, g0 + chunk);
	const int nsteps = (int)((g1 - g0 + KT - 1) / KT);
	const long long gs0 = g0 / KT;
	init_ring(full, empty);
	tc_setup(sh);
	const bool diag = ti == tj;
	run_bulk_pipeline(sh, full, empty, nsteps, true,
			[&](int st) { return rows + ((long long)ti * gsteps + gs0 + st) * kOperandBytes; },
			[&](int st) -> const unsigned char* {
				return diag ? nullptr : rows + ((long long)tj * gsteps + gs0 + st) * kOperandBytes;
			},
			err);
	__syncthreads();
	tc_fence_after();
	if (!sh.abort) {
		double2* out = part + (size_t)blockIdx.y * k * k;
		store_tile(sh, [&](int r, int c, double re, double im) {
			const int i = i0 + r, j = j0 + c;
			if (i < k && j < k) out[(size_t)i * k + j] = make_double2(re, im);
		});
	}
	tc_teardown(sh);
}

// Rotation from pre-split W^T (A) and the cols layout of psi (B); the same
// MMAs in the same order as rotate_tc_kernel.
__global__ void __launch_bounds__(kThreads, 1) rotate_tc2_kernel(const unsigned char* __restrict__ wsplit,
		const unsigned char* __restrict__ cols, int k, long long G, float2* __restrict__ out, int* err, int upper) {
	TcShared& sh = tc_shared();
	__shared__ alignas(8) unsigned long long full[kRing], empty[kRing];
	const int n0 = blockIdx.x * TM;
	const long long gt = blockIdx.y;
	const long long gt0 = gt * TN;
	const int nsteps = (k + KT - 1) / KT;
	const int nrun = upper ? (min(k, n0 + TM) + KT - 1) / KT : nsteps;
	const unsigned char* wblk = wsplit + (size_t)blockIdx.x * nsteps * kOperandBytes;
	const unsigned char* cblk = cols + (size_t)gt * nsteps * kOperandBytes;
	init_ring(full, empty);
	tc_setup(sh);
	run_bulk_pipeline(sh, full, empty, nrun, false, [&](int st) { return wblk + (size_t)st * kOperandBytes; },
			[&](int st) -> const unsigned char* { return cblk + (size_t)st * kOperandBytes; }, err);
	__syncthreads();
	tc_fence_after();
	if (!sh.abort) {
		store_tile(sh, [&](int r, int c, double re, double im) {
			const int n = n0 + r;
			const long long g = gt0 + c;
			if (n < k && g < G) out[(long long)n * G + g] = make_float2((float)re, (float)im);
		});
	}
	tc_teardown(sh);
}

// Rotation tile: out rows n0.. (state index n), columns gt0.. (grid points).
// A = W^T from the pre-split planes, B[g][i] = psi_i[g].
__global__ void __launch_bounds__(kThreads, 1) rotate_tc_kernel(const unsigned char* __restrict__ wsplit,
		const float2* __restrict__ psi, int k, long long G, float2* __restrict__ out, int* err, int upper) {
	TcShared& sh = tc_shared();
	const int n0 = blockIdx.x * TM;
	const long long gt0 = (long long)blockIdx.y * TN;
	const int nsteps = (k + KT - 1) / KT;
	// upper-triangular W (Cholesky): states i >= n0 + TM do not contribute
	const int nrun = upper ? (min(k, n0 + TM) + KT - 1) / KT : nsteps;
	tc_setup(sh);
	const int tid = threadIdx.x;
	unsigned char* const base = sh.buf;
	const unsigned char* wblk = wsplit + (size_t)blockIdx.x * nsteps * kOperandBytes;
	// raw psi slot: row r = K index within the step (16 rows of 128 complex),
	// 16-byte piece pg (64 per row) stored at slot pg ^ 2 ((r >> 1) & 3): the
	// four rows a half-warp of the split reads land in distinct 32-byte banks
	auto prefetch = [&](int s) {
		unsigned char* ring = base + kRoA + (s & 3) * kOperandBytes;
		const unsigned char* src = wblk + (size_t)s * kOperandBytes;
#pragma unroll
		for (int it = 0; it < kOperandBytes / 16 / kThreads; it++) {
			const int idx = it * kThreads + tid;
			cp16(smem_u32(ring + idx * 16), src + idx * 16, 16);
		}
		unsigned char* slot = base + kRoRaw + (s % 3) * kRoRawSlot;
#pragma unroll
		for (int it = 0; it < 4; it++) {
			const int idx = it * kThreads + tid;  // 0..1023
			const int r = idx >> 6, pg = idx & 63;
			const int i = s * KT + r;
			const long long g = gt0 + 2 * pg;
			const bool in = i < k && g < G;  // g even, G even: both complex in range
			const float2* p = in ? psi + (long long)i * G + g : psi;
			cp16(smem_u32(slot + r * (TN * 8) + ((pg ^ (((r >> 1) & 3) << 1)) << 4)), p, in ? 16 : 0);
		}
	};
	// convert: warp w handles core matrices m = w, w + 8, w + 16, w + 24 of the
	// 32 (16 row groups of g x 2 K halves of i)
	auto convert = [&](int s) {
		const unsigned char* slot = base + kRoRaw + (s % 3) * kRoRawSlot;
		unsigned char* planes = base + kRoB + (s & 1) * kOperandBytes;
		const int w = tid >> 5, lane = tid & 31;
#pragma unroll
		for (int it = 0; it < 4; it++) {
			const int m = it * 8 + w;
			const int rg = m >> 1, kc = m & 1;
			const int r = rg * 8 + (lane >> 2), kk = kc * 8 + (lane & 3) * 2;
			const int pg = r >> 1, sub = r & 1;
			const float2 p0 = reinterpret_cast<const float2*>(
					slot + kk * (TN * 8) + ((pg ^ (((kk >> 1) & 3) << 1)) << 4))[sub];
			const float2 p1 = reinterpret_cast<const float2*>(
					slot + (kk + 1) * (TN * 8) + ((pg ^ ((((kk + 1) >> 1) & 3) << 1)) << 4))[sub];
			put2(planes, kmaj_off(r, kk), p0.x, p0.y, p1.x, p1.y);
		}
	};
	auto a_addr = [&](int s) { return smem_u32(base + kRoA + (s & 3) * kOperandBytes); };
	auto b_addr = [&](int s) { return smem_u32(base + kRoB + (s & 1) * kOperandBytes); };
	run_pipeline(sh, nrun, false, prefetch, convert, a_addr, b_addr, err);
	if (!sh.abort) {
		store_tile(sh, [&](int r, int c, double re, double im) {
			const int n = n0 + r;
			const long long g = gt0 + c;
			if (n < k && g < G) out[(long long)n * G + g] = make_float2((float)re, (float)im);
		});
	}
	tc_teardown(sh);
}

// Diagnostic of the bounded waits: one CTA sets up exactly like the
// tensor-core kernels (tensor memory allocated, mbarriers initialised), waits
// on a barrier that nothing completes, records ITP2D_E_TIMEOUT when the wait
// gives up, frees its tensor memory and returns.
__global__ void __launch_bounds__(kThreads, 1) tc_wait_probe_kernel(int* err) {
	TcShared& sh = tc_shared();
	tc_setup(sh);
	const bool ok = mbar_wait(smem_u32(&sh.mbar[0]), 0);  // phase 0 is never completed
	if (!__syncthreads_and(ok) && threadIdx.x == 0) atomicExch(err, ITP2D_E_TIMEOUT);
	tc_teardown(sh);
}

size_t tc_smem() { return sizeof(TcShared) + 1024; }

void set_tc_attributes() {
	cudaFuncSetAttribute(overlap_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc_smem());
	cudaFuncSetAttribute(rotate_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc_smem());
	cudaFuncSetAttribute(overlap_tc2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc_smem());
	cudaFuncSetAttribute(rotate_tc2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc_smem());
	cudaFuncSetAttribute(tc_wait_probe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc_smem());
}

}  // namespace

bool tc_supported(int k, long long G) { return k >= 2 && G >= KT && G % 2 == 0; }

int tc_overlap_splits(int k, long long G, int num_sms) {
	const int nt = (k + TM - 1) / TM;
	const int npairs = nt * (nt + 1) / 2;
	// enough CTAs to cover the SMs; chunks of at most 2048 grid points bound
	// the FP32 accumulation in tensor memory (the splits add up in FP64); then
	// the first count (up to twice that) whose grid fills its last wave of one
	// CTA per SM to 90% or more, else the best-filled one
	const long long by_sms = (num_sms + npairs - 1) / npairs;
	const long long by_len = (G + 2047) / 2048;
	const long long most = std::max(1LL, G / (4 * KT));
	const long long lo = std::max(1LL, std::min(std::max(by_sms, by_len), most));
	long long best = lo;
	double best_fill = 0.0;
	for (long long ns = lo; ns <= std::min(2 * lo, most); ns++) {
		const long long ctas = npairs * ns;
		const long long waves = (ctas + num_sms - 1) / num_sms;
		const double fill = (double)ctas / (double)(waves * num_sms);
		if (fill > best_fill + 1e-9) {
			best = ns;
			best_fill = fill;
		}
		if (fill >= 0.9) break;
	}
	return (int)best;
}

size_t tc_wsplit_bytes(int k) {
	const size_t nt = (k + TM - 1) / TM, ks = (k + KT - 1) / KT;
	return nt * ks * kOperandBytes;
}

void launch_overlap_tc(const float2* psi, int k, long long G, int nsplit, double2* part, double dx2, double2* S,
		int* err, cudaStream_t s) {
	const int nt = (k + TM - 1) / TM;
	const int npairs = nt * (nt + 1) / 2;
	long long chunk = (G + nsplit - 1) / nsplit;
	chunk = ((chunk + KT - 1) / KT) * KT;
	const int used = (int)((G + chunk - 1) / chunk);
	set_tc_attributes();
	overlap_tc_kernel<<<dim3(npairs, used), kThreads, tc_smem(), s>>>(psi, k, G, nt, chunk, part, err);
	launch_overlap_finish(part, k, used, dx2, S, s);
}

void launch_rotate_tc(const double2* W, const float2* psi, int k, long long G, unsigned char* wsplit, float2* out,
		int* err, cudaStream_t s, bool upper) {
	const int nt = (k + TM - 1) / TM, ks = (k + KT - 1) / KT;
	const long long threads = (long long)nt * ks * 32 * 32;
	split_w_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(W, k, ks, nt, wsplit);
	set_tc_attributes();
	const dim3 grid(nt, (unsigned)((G + TN - 1) / TN));
	rotate_tc_kernel<<<grid, kThreads, tc_smem(), s>>>(wsplit, psi, k, G, out, err, upper ? 1 : 0);
}

size_t tc_rows_bytes(int k, long long G) {
	return (size_t)((k + TM - 1) / TM) * (size_t)((G + KT - 1) / KT) * kOperandBytes;
}

size_t tc_cols_bytes(int k, long long G) {
	return (size_t)((G + TN - 1) / TN) * (size_t)((k + KT - 1) / KT) * kOperandBytes;
}

void launch_overlap_tc_presplit(const float2* psi, int k, long long G, int nsplit, unsigned char* rows, double2* part,
		double dx2, double2* S, int* err, cudaStream_t s) {
	const int nt = (k + TM - 1) / TM;
	const int npairs = nt * (nt + 1) / 2;
	const long long gsteps = (G + KT - 1) / KT;
	const long long threads = (long long)nt * gsteps * 32 * 32;
	split_psi_rows_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(psi, k, G, nt, gsteps, rows);
	long long chunk = (G + nsplit - 1) / nsplit;
	chunk = ((chunk + KT - 1) / KT) * KT;
	const int used = (int)((G + chunk - 1) / chunk);
	set_tc_attributes();
	overlap_tc2_kernel<<<dim3(npairs, used), kThreads, tc_smem(), s>>>(rows, k, G, nt, gsteps, chunk, part, err);
	launch_overlap_finish(part, k, used, dx2, S, s);
}

void launch_rotate_tc_presplit(const double2* W, const float2* psi, int k, long long G, unsigned char* wsplit,
		unsigned char* cols, float2* out, int* err, cudaStream_t s, bool upper) {
	const int nt = (k + TM - 1) / TM, ks = (k + KT - 1) / KT;
	const long long gtiles = (G + TN - 1) / TN;
	long long threads = (long long)nt * ks * 32 * 32;
	split_w_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(W, k, ks, nt, wsplit);
	threads = gtiles * ks * 32 * 32;
	split_psi_cols_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(psi, k, G, gtiles, ks, cols);
	set_tc_attributes();
	rotate_tc2_kernel<<<dim3(nt, (unsigned)gtiles), kThreads, tc_smem(), s>>>(wsplit, cols, k, G, out, err,
			upper ? 1 : 0);
}

}  // namespace itp2d

int itp2d_tc_wait_probe(void) {
	int* err = nullptr;
	if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) return ITP2D_E_OOM;
	int st = ITP2D_E_CUDA;
	if (cudaMemset(err, 0, sizeof(int)) == cudaSuccess) {
		itp2d::set_tc_attributes();
		itp2d::tc_wait_probe_kernel<<<1, itp2d::kThreads, itp2d::tc_smem()>>>(err);
		int h = -1;
		if (cudaGetLastError() == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess &&
				cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess)
			st = h;
	}
	cudaFree(err);
	return st;
}
