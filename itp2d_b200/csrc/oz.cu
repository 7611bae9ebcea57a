// FP64 rotation of the states on the int8 tensor cores (tcgen05.mma
// kind::i8, exact 32-bit integer accumulation in tensor memory):
//
//   out_n[g] = sum_i W[i][n] psi_i[g]                     (stateset.cpp:214-228)
//
// Both operands are split into int8 slices under a power-of-two scale shared
// by a row of the product (the Ozaki scheme): each value x of a row with
// max |x| < 2^e is written x = 2^e sum_s d_s 2^{-7 (s + 1)}, digits d_s in
// [-127, 127] from repeated truncation (v <- 128 v, d = trunc(v), v <- v - d,
// all exact in FP64), kSlices = 8 of them: 56 bits of the row maximum. The
// product of two slices is an exact integer matrix; slice pairs (s, t) with
// s + t = d share the weight 2^{-7 (d + 2)}, so the pairs of one diagonal d
// accumulate into one S32 accumulator (at most 8 x 127^2 x 2k < 2^31 for
// k < 8300 states), and pairs with s + t >= kSlices are dropped (terms below
// 2^-56 of the row maxima; the result agrees with FP64 products to about
// 1e-15 of the largest output of its row). The FP64 result is sum_d 2^{-7 (d + 2)} acc_d,
// times the two row scales.
//
// Operands (K = 2 i + c: state i, component c = re, im):
//   A[n][(i, c)]      = W[i][n].c                      scale per output state n
//   B[2 m][(i, c)]    = (psi_i[g].re, -psi_i[g].im)    real part of out_n[g]
//   B[2 m + 1][(i, c)] = (psi_i[g].im,  psi_i[g].re)   imaginary part
// with g = g0 + m, scale per grid point g (over all states). One MMA of
// M = 128 states, N = 128 columns (64 grid points x re/im), K = 32 (16 states)
// per slice pair. The slices are written once per rotation into the MMA's
// K-major block layout (slice_w_kernel, slice_psi_kernel), so the kernel only
// copies blocks: one cp.async.bulk per operand and step into a ring of three
// slots, issued with the MMAs by one thread.
//
// Tensor memory holds four 128-column accumulators, so the 8 diagonals run in
// two passes over K: diagonals 0..3 (slices 0..3 copied), then 4..7 (all 8),
// 36 MMAs per step.
// After each pass all threads add their accumulator columns into FP64
// registers. Waits on mbarriers are bounded (tcgen05.cuh).
#include <stdint.h>

#include <algorithm>

#include "../../include/itp2d_gpu.h"
#include "contract.cuh"
#include "tcgen05.cuh"

namespace itp2d {

namespace {

using namespace tcg;

constexpr int TM = 128;                     // output states per tile (M)
constexpr int TN = 128;                     // accumulator columns (N): 64 grid points x re/im
constexpr int GT = TN / 2;                  // grid points per tile
constexpr int KS = 16;                      // states per K step (32 int8 K values)
constexpr int kSlices = 8;
constexpr int kBlock = TM * 32;             // 4 KB: one slice of a 128-row x 32-byte block
constexpr int kThreads = 256;
constexpr int kRing = 3;
constexpr int kSlotBytes = 2 * kSlices * kBlock;  // 64 KB: the A and B slices of one step
constexpr int kTmemCols = 512;
constexpr int kDiagPerPass = 4;             // 128-column accumulators in tensor memory
static_assert(kDiagPerPass * TN <= kTmemCols, "accumulators");

struct OzShared {
	alignas(128) unsigned char ring[kRing * kSlotBytes];
	alignas(8) unsigned long long full[kRing], empty[kRing];
	uint32_t tmem_base;
	int abort;
};

// Byte offset of element (row r, K index kk < 32) in a 128 x 32 int8 block:
// core matrix (r / 8, kk / 16) at ((r / 8) * 2 + kk / 16) * 128, rows 16 B apart.
__host__ __device__ __forceinline__ uint32_t kmaj8_off(int r, int kk) {
	return (uint32_t)((((r >> 3) << 1) + (kk >> 4)) * 128 + (r & 7) * 16 + (kk & 15));
}

// Exponent e with m < 2^e (m >= 0; 0 for m = 0, whose digits are all zero),
// at least -1000 so that the scalings below stay normal (a row whose largest
// value is below 2^-1000 keeps fewer digits).
__device__ __forceinline__ int scale_exp(double m) {
	int e = 0;
	if (m > 0.0) frexp(m, &e);  // m = f 2^e, f in [0.5, 1)
	return e < -1000 ? -1000 : e;
}

// 2^p for -1022 <= p <= 1023, from the IEEE-754 bit pattern.
__device__ __forceinline__ double pow2(int p) { return __longlong_as_double((long long)(1023 + p) << 52); }

// The kSlices digits of x 2^{-e} (|x| < 2^e), packed 4 per word: word s of
// dst gets digit s of four values, lane (byte) b from v[b].
__device__ __forceinline__ void digits4(const double* v, int e, uint32_t* dst) {
	double r[4];
	const double sc = pow2(-e);
#pragma unroll
	for (int b = 0; b < 4; b++) r[b] = v[b] * sc;
#pragma unroll
	for (int s = 0; s < kSlices; s++) {
		uint32_t w = 0;
#pragma unroll
		for (int b = 0; b < 4; b++) {
			const double t = trunc(r[b] * 128.0);
			r[b] = r[b] * 128.0 - t;
			w |= ((uint32_t)(int)t & 0xFFu) << (8 * b);
		}
		dst[s] = w;
	}
}

// 16 values (one 16-byte core-matrix row) into the kSlices blocks of one
// step: value j of vals goes to byte j of the row at byte offset off.
__device__ __forceinline__ void put_row16(unsigned char* blocks, uint32_t off, const double* vals, int e) {
	uint32_t w[4][kSlices];
#pragma unroll
	for (int q = 0; q < 4; q++) digits4(vals + 4 * q, e, w[q]);
#pragma unroll
	for (int s = 0; s < kSlices; s++)
		*reinterpret_cast<uint4*>(blocks + s * kBlock + off) = make_uint4(w[0][s], w[1][s], w[2][s], w[3][s]);
}

// eA[n] for the rows of A (n < k; W[i][n] over i): one thread per n, the
// loads of a warp along n coalesced. Rows n >= k (to the tile edge) get 0.
__global__ void w_exp_kernel(const double2* __restrict__ W, int k, int rows, int* __restrict__ eA) {
	const int n = blockIdx.x * blockDim.x + threadIdx.x;
	if (n >= rows) return;
	double m = 0.0;
	if (n < k)
		for (int i = 0; i < k; i++) {
			const double2 w = W[(size_t)i * k + n];
			m = fmax(m, fmax(fabs(w.x), fabs(w.y)));
		}
	eA[n] = scale_exp(m);
}

// eB[g] for the grid points (g < G; psi_i[g] over i): one thread per g.
__global__ void psi_exp_kernel(const double2* __restrict__ psi, int k, long long G, long long cols,
		int* __restrict__ eB) {
	const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (g >= cols) return;
	double m = 0.0;
	if (g < G)
		for (int i = 0; i < k; i++) {
			const double2 v = __ldcs(psi + (long long)i * G + g);
			m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
		}
	eB[g] = scale_exp(m);
}

// A slices: block group (n tile nt, step s) at ((nt * ksteps + s) * kSlices)
// * kBlock; thread t of 256 writes row r = t / 2, K half kc = t % 2 (states
// s * 16 + kc * 8 + j / 2, component j % 2, j < 16).
__global__ void slice_w_kernel(const double2* __restrict__ W, int k, int ksteps, const int* __restrict__ eA,
		unsigned char* __restrict__ out) {
	const int nt = blockIdx.x, st = blockIdx.y;
	const int r = threadIdx.x >> 1, kc = threadIdx.x & 1;
	const int n = nt * TM + r;
	double v[16];
#pragma unroll
	for (int j = 0; j < 16; j += 2) {
		const int i = st * KS + kc * 8 + j / 2;
		double2 w = make_double2(0.0, 0.0);
		if (n < k && i < k) w = W[(size_t)i * k + n];
		v[j] = w.x;
		v[j + 1] = w.y;
	}
	put_row16(out + ((size_t)nt * ksteps + st) * kSlices * kBlock, kmaj8_off(r, kc * 16), v, eA[n]);
}

// B slices: block group (grid tile gt, step s) at ((gt * ksteps + s) *
// kSlices) * kBlock. The 16 states x 64 grid points of the step are staged in
// shared memory (coalesced rows of psi); thread t writes row r = t / 2 (grid
// point m = r / 2, real row for r even, imaginary for r odd), K half t % 2.
__global__ void slice_psi_kernel(const double2* __restrict__ psi, int k, long long G, int ksteps,
		const int* __restrict__ eB, unsigned char* __restrict__ out) {
	__shared__ double2 tile[KS][GT + 1];
	const long long gt = blockIdx.x;
	const int st = blockIdx.y;
	for (int idx = threadIdx.x; idx < KS * GT; idx += blockDim.x) {
		const int ii = idx / GT, m = idx % GT;
		const int i = st * KS + ii;
		const long long g = gt * GT + m;
		tile[ii][m] = (i < k && g < G) ? __ldcs(psi + (long long)i * G + g) : make_double2(0.0, 0.0);
	}
	__syncthreads();
	const int r = threadIdx.x >> 1, kc = threadIdx.x & 1;
	const int m = r >> 1;
	const bool imag = r & 1;
	double v[16];
#pragma unroll
	for (int j = 0; j < 16; j += 2) {
		const double2 p = tile[kc * 8 + j / 2][m];
		v[j] = imag ? p.y : p.x;       // c = re: psi.re (real row), psi.im (imaginary row)
		v[j + 1] = imag ? p.x : -p.y;  // c = im: -psi.im (real row), psi.re (imaginary row)
	}
	put_row16(out + ((size_t)gt * ksteps + st) * kSlices * kBlock, kmaj8_off(r, kc * 16), v, eB[gt * GT + m]);
}

// Overlap operands. State exponents e[i] (max over the grid of both
// components of psi_i < 2^e[i]; 0 for the padding rows up to the tile edge):
// one block per state.
__global__ void state_exp_kernel(const double2* __restrict__ psi, int k, long long G, int* __restrict__ e) {
	__shared__ double red[32];
	const int i = blockIdx.x;
	double m = 0.0;
	if (i < k)
		for (long long g = threadIdx.x; g < G; g += blockDim.x) {
			const double2 v = __ldcs(psi + (long long)i * G + g);
			m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
		}
	for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
	if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
	__syncthreads();
	if (threadIdx.x < 32) {
		m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
		for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
		if (threadIdx.x == 0) e[i] = scale_exp(m);
	}
}

// A slices of the overlap: block group (state tile ti of 128, grid step gs of
// 16 points) at ((ti * gsteps + gs) * kSlices) * kBlock; row r = state
// ti * 128 + r, K index 2 (g - 16 gs) + c: (psi.re, psi.im). Thread t writes
// row t / 2, grid points 16 gs + 8 (t % 2) .. + 7.
__global__ void slice_rows_kernel(const double2* __restrict__ psi, int k, long long G, long long gsteps,
		const int* __restrict__ e, unsigned char* __restrict__ out) {
	const int ti = blockIdx.y;
	const long long gs = blockIdx.x;
	const int r = threadIdx.x >> 1, kc = threadIdx.x & 1;
	const int i = ti * TM + r;
	double v[16];
#pragma unroll
	for (int j = 0; j < 16; j += 2) {
		const long long g = gs * 16 + kc * 8 + j / 2;
		const double2 p = (i < k && g < G) ? __ldcs(psi + (long long)i * G + g) : make_double2(0.0, 0.0);
		v[j] = p.x;
		v[j + 1] = p.y;
	}
	put_row16(out + ((size_t)ti * gsteps + gs) * kSlices * kBlock, kmaj8_off(r, kc * 16), v, e[i]);
}

// B slices of the overlap: block group (state tile tj of 64, grid step gs) at
// ((tj * gsteps + gs) * kSlices) * kBlock; row 2 m = X of state tj * 64 + m
// (psi.re, psi.im: the real part of the overlap), row 2 m + 1 = Y (psi.im,
// -psi.re: the imaginary part).
__global__ void slice_xy_kernel(const double2* __restrict__ psi, int k, long long G, long long gsteps,
		const int* __restrict__ e, unsigned char* __restrict__ out) {
	const int tj = blockIdx.y;
	const long long gs = blockIdx.x;
	const int r = threadIdx.x >> 1, kc = threadIdx.x & 1;
	const int j = tj * GT + (r >> 1);
	const bool y = r & 1;
	double v[16];
#pragma unroll
	for (int jj = 0; jj < 16; jj += 2) {
		const long long g = gs * 16 + kc * 8 + jj / 2;
		const double2 p = (j < k && g < G) ? __ldcs(psi + (long long)j * G + g) : make_double2(0.0, 0.0);
		v[jj] = y ? p.y : p.x;
		v[jj + 1] = y ? -p.x : p.y;
	}
	put_row16(out + ((size_t)tj * gsteps + gs) * kSlices * kBlock, kmaj8_off(r, kc * 16), v, e[j]);
}

// The MMAs of one step of pass p (diagonals 4p .. 4p + 3 below kSlices):
// slice pair (s, d - s) into accumulator d - 4p. first: the step opens its
// segment (the first pair of each diagonal overwrites its accumulator).
__device__ __forceinline__ void issue_oz_step(uint32_t tmem, uint32_t abase, uint32_t bbase, int pass, bool first) {
	constexpr uint32_t id = idesc_s8(TN);
#pragma unroll
	for (int dd = 0; dd < kDiagPerPass; dd++) {
		const int d = pass * kDiagPerPass + dd;
		if (d >= kSlices) break;
		const uint32_t acc = tmem + (uint32_t)(dd * TN);
		for (int s = 0; s <= d; s++)
			umma_i8(acc, sdesc(abase + s * kBlock), sdesc(bbase + (d - s) * kBlock), id,
					(first && s == 0) ? 0u : 1u);
	}
}

// Slices copied for pass p: all slices up to its largest diagonal.
__host__ __device__ constexpr int pass_slices(int pass) {
	return (pass + 1) * kDiagPerPass < kSlices ? (pass + 1) * kDiagPerPass : kSlices;
}

// Step u of a CTA's sequence over K steps [s0, s0 + n) in chunks of L steps:
// chunk c runs pass 0 over its steps, then pass 1 over the same steps (the
// S32 sums of a chunk stay below 2^31); a segment is one pass over one chunk,
// after which the accumulators are added into FP64 registers.
struct OzStep {
	int pass, st, seg_begin, seg_end;  // pass, absolute K step, the segment's u range
};
__device__ __forceinline__ OzStep oz_step(int u, int s0, int n, int L) {
	const int c = u / (2 * L), r = u - c * 2 * L;
	const int len = min(L, n - c * L);
	const int pass = r / len, off = r - pass * len;
	OzStep o;
	o.pass = pass;
	o.st = s0 + c * L + off;
	o.seg_begin = u - off;
	o.seg_end = o.seg_begin + len;
	return o;
}

// Tensor memory, mbarriers and the abort flag of a CTA (all threads).
__device__ __forceinline__ void oz_setup(OzShared& sh) {
	if (threadIdx.x < 32) tmem_alloc(&sh.tmem_base, kTmemCols);
	if (threadIdx.x == 0) {
		for (int i = 0; i < kRing; i++) {
			mbar_init(smem_u32(&sh.full[i]), 1);
			mbar_init(smem_u32(&sh.empty[i]), 1);
		}
		sh.abort = 0;
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
}

__device__ __forceinline__ void oz_teardown(OzShared& sh) {
	tc_fence_before();
	__syncthreads();
	if (threadIdx.x < 32) tmem_dealloc(sh.tmem_base, kTmemCols);
}

// The K loop of a CTA (all threads call it): thread 0 copies the slice blocks
// of step u (src_a(st), src_b(st): the kSlices blocks of absolute step st)
// into ring slot u % kRing and issues the MMAs; at the end of each segment
// all threads add their 64 accumulator columns (warp w: tensor-memory lanes
// 32 (w % 4) .., columns 64 (w / 4) ..) weighted 2^{-7 d} into acc. Returns
// with sh.abort set if a bounded wait gave up (then acc is incomplete).
template <class SrcA, class SrcB>
__device__ __forceinline__ void oz_run(OzShared& sh, int s0, int n, int L, SrcA src_a, SrcB src_b, double (&acc)[64],
		int* err) {
	const int tid = threadIdx.x;
	const uint32_t tmem = sh.tmem_base;
	const int total = 2 * n;
	auto copy = [&](int u) {
		const OzStep o = oz_step(u, s0, n, L);
		const uint32_t bytes = (uint32_t)(pass_slices(o.pass) * kBlock);
		unsigned char* dst = sh.ring + (u % kRing) * kSlotBytes;
		const uint32_t fb = smem_u32(&sh.full[u % kRing]);
		mbar_expect_tx(fb, 2 * bytes);
		bulk_copy(smem_u32(dst), src_a(o.st), bytes, fb);
		bulk_copy(smem_u32(dst + kSlices * kBlock), src_b(o.st), bytes, fb);
	};
	int copied = 0, issued = 0;  // thread 0: steps copied / whose MMAs were issued
	if (tid == 0)
		for (; copied < total && copied < kRing; copied++) copy(copied);
#pragma unroll
	for (int j = 0; j < 64; j++) acc[j] = 0.0;
	const int w = tid >> 5;
	const uint32_t trow = tmem + ((uint32_t)((w & 3) * 32) << 16) + (uint32_t)((w >> 2) * 64);
	int u0 = 0;
	while (u0 < total) {
		const OzStep seg = oz_step(u0, s0, n, L);
		if (tid == 0 && !sh.abort) {
			bool ok = true;
			for (int u = seg.seg_begin; u < seg.seg_end; u++) {
				const int slot = u % kRing;
				if (!mbar_wait(smem_u32(&sh.full[slot]), (uint32_t)((u / kRing) & 1))) {
					ok = false;
					break;
				}
				tc_fence_after();
				const uint32_t a = smem_u32(sh.ring + slot * kSlotBytes);
				issue_oz_step(tmem, a, a + kSlices * kBlock, seg.pass, u == seg.seg_begin);
				umma_commit(smem_u32(&sh.empty[slot]));
				issued = u + 1;
				// refill the slot of step u - 1 once its MMAs have read it (a
				// completed phase: the wait returns at once after a segment end)
				if (u >= 1 && copied < total) {
					const int pu = u - 1;
					if (!mbar_wait(smem_u32(&sh.empty[pu % kRing]), (uint32_t)((pu / kRing) & 1))) {
						ok = false;
						break;
					}
					copy(copied++);
				}
			}
			// the last commit covers every MMA of the segment
			if (ok && issued > 0 &&
					!mbar_wait(smem_u32(&sh.empty[(issued - 1) % kRing]), (uint32_t)(((issued - 1) / kRing) & 1)))
				ok = false;
			if (!ok) {
				sh.abort = 1;
				atomicExch(err, ITP2D_E_TIMEOUT);
				// copies not yet waited for land before the CTA leaves
				for (int u = issued; u < copied; u++)
					mbar_wait(smem_u32(&sh.full[u % kRing]), (uint32_t)((u / kRing) & 1));
				if (issued > 0)
					mbar_wait(smem_u32(&sh.empty[(issued - 1) % kRing]), (uint32_t)(((issued - 1) / kRing) & 1));
			}
		}
		u0 = seg.seg_end;
		__syncthreads();
		tc_fence_after();
		if (sh.abort) break;
#pragma unroll
		for (int dd = 0; dd < kDiagPerPass; dd++) {
			const int d = seg.pass * kDiagPerPass + dd;
			if (d >= kSlices) break;
			const double f = pow2(-7 * d);
#pragma unroll
			for (int c = 0; c < 64; c += 32) {
				uint32_t r[32];
				tmem_ld32_raw(trow + (uint32_t)(dd * TN + c), r);
#pragma unroll
				for (int j = 0; j < 32; j++) acc[c + j] += (double)(int)r[j] * f;
			}
		}
		tc_fence_before();
		__syncthreads();
		tc_fence_after();
	}
}

__device__ __forceinline__ OzShared& oz_shared() {
	extern __shared__ __align__(128) unsigned char smem_raw[];
	return *reinterpret_cast<OzShared*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
}

// Rotation tile: states n0 .. n0 + 127 (blockIdx.x), grid points g0 .. g0 + 63
// (blockIdx.y). upper: W is upper triangular (Cholesky), states i >= n0 + 128
// do not contribute. K = 2k stays below 2^31 / (8 127^2) for k < 8300: one
// chunk.
__global__ void __launch_bounds__(kThreads, 1) rotate_oz_kernel(const unsigned char* __restrict__ wsl,
		const unsigned char* __restrict__ psl, const int* __restrict__ eA, const int* __restrict__ eB, int k,
		long long G, double2* __restrict__ out, int* err, int upper) {
	OzShared& sh = oz_shared();
	const int n0 = blockIdx.x * TM;
	const long long gt = blockIdx.y;
	const long long g0 = gt * GT;
	const int ksteps = (k + KS - 1) / KS;
	const int nrun = upper ? (min(k, n0 + TM) + KS - 1) / KS : ksteps;
	const unsigned char* ablk = wsl + (size_t)blockIdx.x * ksteps * kSlices * kBlock;
	const unsigned char* bblk = psl + (size_t)gt * ksteps * kSlices * kBlock;
	oz_setup(sh);
	double acc[64];
	oz_run(sh, 0, nrun, nrun, [&](int st) { return ablk + (size_t)st * kSlices * kBlock; },
			[&](int st) { return bblk + (size_t)st * kSlices * kBlock; }, acc, err);
	if (!sh.abort) {
		// row n, grid points g0 + 32 (w / 4) + jj (columns 2 jj, 2 jj + 1: re, im)
		const int w = threadIdx.x >> 5;
		const int n = n0 + (w & 3) * 32 + (threadIdx.x & 31);
		if (n < k) {
			const int ea = eA[n] - 14;
			double2* dst = out + (long long)n * G;
#pragma unroll
			for (int jj = 0; jj < 32; jj++) {
				const long long g = g0 + (w >> 2) * 32 + jj;
				if (g < G) {
					const double sc = ldexp(1.0, ea + eB[g]);
					dst[g] = make_double2(acc[2 * jj] * sc, acc[2 * jj + 1] * sc);
				}
			}
		}
	}
	oz_teardown(sh);
}

// Overlap tile pair: states i0 .. i0 + 127 (A rows) x states j0 .. j0 + 63 (B:
// X and Y rows), pair index blockIdx.x over the pairs with j0 + 63 >= i0 (the
// upper triangle), grid steps [s0, s0 + n) of split blockIdx.y in chunks of
// kOvChunk steps (2 x 16 x 512 = 16384 K values: 8 x 127^2 x 16384 < 2^31).
// Writes part[split][i][j] = sum over the split's grid points of
// conj(psi_i) psi_j (before dx^2).
constexpr int kOvChunk = 512;
__global__ void __launch_bounds__(kThreads, 1) overlap_oz_kernel(const unsigned char* __restrict__ asl,
		const unsigned char* __restrict__ bsl, const int* __restrict__ e, int k, long long gsteps, int ntj,
		long long split_steps, double2* __restrict__ part, int* err) {
	OzShared& sh = oz_shared();
	int p = blockIdx.x, ti = 0;
	while (p >= ntj - 2 * ti) {
		p -= ntj - 2 * ti;
		ti++;
	}
	const int tj = 2 * ti + p;
	const int i0 = ti * TM, j0 = tj * GT;
	const long long s0 = (long long)blockIdx.y * split_steps;
	const int n = (int)min(split_steps, gsteps - s0);
	const unsigned char* ablk = asl + (size_t)ti * gsteps * kSlices * kBlock;
	const unsigned char* bblk = bsl + (size_t)tj * gsteps * kSlices * kBlock;
	oz_setup(sh);
	double acc[64];
	oz_run(sh, (int)0, n, kOvChunk, [&](int st) { return ablk + (size_t)(s0 + st) * kSlices * kBlock; },
			[&](int st) { return bblk + (size_t)(s0 + st) * kSlices * kBlock; }, acc, err);
	if (!sh.abort) {
		const int w = threadIdx.x >> 5;
		const int i = i0 + (w & 3) * 32 + (threadIdx.x & 31);
		if (i < k) {
			const int ei = e[i] - 14;
			double2* dst = part + (size_t)blockIdx.y * k * k + (size_t)i * k;
#pragma unroll
			for (int jj = 0; jj < 32; jj++) {
				const int j = j0 + (w >> 2) * 32 + jj;
				if (j < k) {
					const double sc = ldexp(1.0, ei + e[j]);
					dst[j] = make_double2(acc[2 * jj] * sc, acc[2 * jj + 1] * sc);
				}
			}
		}
	}
	oz_teardown(sh);
}

size_t oz_smem() { return sizeof(OzShared) + 128; }

}  // namespace

bool oz_supported(int k, long long G) { return k >= 2 && k < 8300 && G >= 1; }

size_t oz_w_bytes(int k) {
	return (size_t)((k + TM - 1) / TM) * (size_t)((k + KS - 1) / KS) * kSlices * kBlock;
}

// Slice scratch: the rotation's state slices, or the overlap's A and B
// slices (never needed at the same time).
static size_t ov_rows_bytes(int k, long long G) {
	return (size_t)((k + TM - 1) / TM) * (size_t)((G + 15) / 16) * kSlices * kBlock;
}
static size_t ov_xy_bytes(int k, long long G) {
	return (size_t)((k + GT - 1) / GT) * (size_t)((G + 15) / 16) * kSlices * kBlock;
}

size_t oz_scratch_bytes(int k, long long G) {
	const size_t rot = (size_t)((G + GT - 1) / GT) * (size_t)((k + KS - 1) / KS) * kSlices * kBlock;
	return std::max(rot, ov_rows_bytes(k, G) + ov_xy_bytes(k, G));
}

size_t oz_exp_ints(int k, long long G) {
	return (size_t)((k + TM - 1) / TM) * TM + (size_t)((G + GT - 1) / GT) * GT;
}

static void oz_attributes() {
	static bool attr = false;
	if (!attr) {
		cudaFuncSetAttribute(rotate_oz_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)oz_smem());
		cudaFuncSetAttribute(overlap_oz_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)oz_smem());
		attr = true;
	}
}

void launch_rotate_oz(const double2* W, const double2* psi, int k, long long G, unsigned char* wsl,
		unsigned char* scratch, int* ebuf, double2* out, int* err, cudaStream_t s, bool upper) {
	const int nt = (k + TM - 1) / TM, ks = (k + KS - 1) / KS;
	const long long gtiles = (G + GT - 1) / GT;
	int* eA = ebuf;
	int* eB = ebuf + (size_t)nt * TM;
	unsigned char* psl = scratch;
	w_exp_kernel<<<(nt * TM + 255) / 256, 256, 0, s>>>(W, k, nt * TM, eA);
	psi_exp_kernel<<<(unsigned)((gtiles * GT + 255) / 256), 256, 0, s>>>(psi, k, G, gtiles * GT, eB);
	slice_w_kernel<<<dim3(nt, ks), 256, 0, s>>>(W, k, ks, eA, wsl);
	slice_psi_kernel<<<dim3((unsigned)gtiles, ks), 256, 0, s>>>(psi, k, G, ks, eB, psl);
	oz_attributes();
	rotate_oz_kernel<<<dim3(nt, (unsigned)gtiles), kThreads, oz_smem(), s>>>(wsl, psl, eA, eB, k, G, out, err,
			upper ? 1 : 0);
}

int oz_overlap_splits(int k, long long G, int num_sms, int max_splits) {
	const int nti = (k + TM - 1) / TM, ntj = (k + GT - 1) / GT;
	int pairs = 0;
	for (int ti = 0; ti < nti; ti++) pairs += ntj - 2 * ti;
	const long long gsteps = (G + 15) / 16;
	const int most = (int)std::max(1LL, std::min<long long>(max_splits, gsteps));
	const int lo = std::min(most, std::max(1, (4 * num_sms + pairs - 1) / pairs));
	// the first count up to 4 lo whose last wave of one CTA per SM is 95% full
	int best = lo;
	double best_fill = 0.0;
	for (int ns = lo; ns <= std::min(most, 4 * lo); ns++) {
		const long long ctas = (long long)pairs * ns;
		const double fill = (double)ctas / (double)(((ctas + num_sms - 1) / num_sms) * num_sms);
		if (fill > best_fill + 1e-9) {
			best = ns;
			best_fill = fill;
		}
		if (fill >= 0.95) break;
	}
	return best;
}

void launch_overlap_oz(const double2* psi, int k, long long G, int nsplit, unsigned char* scratch, int* ebuf,
		double2* part, double dx2, double2* S, int* err, cudaStream_t s) {
	const int nti = (k + TM - 1) / TM, ntj = (k + GT - 1) / GT;
	int pairs = 0;
	for (int ti = 0; ti < nti; ti++) pairs += ntj - 2 * ti;
	const long long gsteps = (G + 15) / 16;
	unsigned char* asl = scratch;
	unsigned char* bsl = scratch + ov_rows_bytes(k, G);
	state_exp_kernel<<<nti * TM, 256, 0, s>>>(psi, k, G, ebuf);
	slice_rows_kernel<<<dim3((unsigned)gsteps, nti), 256, 0, s>>>(psi, k, G, gsteps, ebuf, asl);
	slice_xy_kernel<<<dim3((unsigned)gsteps, ntj), 256, 0, s>>>(psi, k, G, gsteps, ebuf, bsl);
	const long long split_steps = (gsteps + nsplit - 1) / nsplit;
	const int used = (int)((gsteps + split_steps - 1) / split_steps);
	oz_attributes();
	overlap_oz_kernel<<<dim3(pairs, used), kThreads, oz_smem(), s>>>(asl, bsl, ebuf, k, gsteps, ntj, split_steps,
			part, err);
	launch_overlap_finish(part, k, used, dx2, S, s);
}

int oz_launches() { return 5; }

}  // namespace itp2d
