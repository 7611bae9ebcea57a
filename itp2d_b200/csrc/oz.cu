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
constexpr int kPasses = (kSlices + kDiagPerPass - 1) / kDiagPerPass;
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

// The MMAs of one step of pass p (diagonals 4p .. 4p + 3 below kSlices):
// slice pair (s, d - s) into accumulator d - 4p. first: the step opens the
// pass (the first pair of each diagonal overwrites its accumulator).
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

// Rotation tile: states n0 .. n0 + 127 (blockIdx.x), grid points g0 .. g0 + 63
// (blockIdx.y). upper: W is upper triangular (Cholesky), states i >= n0 + 128
// do not contribute.
__global__ void __launch_bounds__(kThreads, 1) rotate_oz_kernel(const unsigned char* __restrict__ wsl,
		const unsigned char* __restrict__ psl, const int* __restrict__ eA, const int* __restrict__ eB, int k,
		long long G, double2* __restrict__ out, int* err, int upper) {
	extern __shared__ __align__(128) unsigned char smem_raw[];
	OzShared& sh = *reinterpret_cast<OzShared*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
	const int tid = threadIdx.x;
	const int nt = blockIdx.x;
	const long long gt = blockIdx.y;
	const int n0 = nt * TM;
	const long long g0 = gt * GT;
	const int ksteps = (k + KS - 1) / KS;
	const int nrun = upper ? (min(k, n0 + TM) + KS - 1) / KS : ksteps;
	const int total = kPasses * nrun;
	const unsigned char* ablk = wsl + (size_t)nt * ksteps * kSlices * kBlock;
	const unsigned char* bblk = psl + (size_t)gt * ksteps * kSlices * kBlock;
	if (tid < 32) tmem_alloc(&sh.tmem_base, kTmemCols);
	if (tid == 0) {
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
	const uint32_t tmem = sh.tmem_base;
	// step u = pass * nrun + st lives in slot u % kRing
	auto copy = [&](int u) {
		const int pass = u / nrun, st = u % nrun;
		const uint32_t bytes = (uint32_t)(pass_slices(pass) * kBlock);
		unsigned char* dst = sh.ring + (u % kRing) * kSlotBytes;
		const uint32_t fb = smem_u32(&sh.full[u % kRing]);
		mbar_expect_tx(fb, 2 * bytes);
		bulk_copy(smem_u32(dst), ablk + (size_t)st * kSlices * kBlock, bytes, fb);
		bulk_copy(smem_u32(dst + kSlices * kBlock), bblk + (size_t)st * kSlices * kBlock, bytes, fb);
	};
	int copied = 0, issued = 0;  // thread 0: steps copied / whose MMAs were issued
	if (tid == 0)
		for (; copied < total && copied < kRing; copied++) copy(copied);
	double acc[64];
#pragma unroll
	for (int j = 0; j < 64; j++) acc[j] = 0.0;
	const int w = tid >> 5, lane = tid & 31;
	const int q = w & 3, half = w >> 2;
	const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(half * 64);
	for (int pass = 0; pass < kPasses; pass++) {
		if (tid == 0 && !sh.abort) {
			bool ok = true;
			for (int st = 0; st < nrun; st++) {
				const int u = pass * nrun + st;
				const int slot = u % kRing;
				if (!mbar_wait(smem_u32(&sh.full[slot]), (uint32_t)((u / kRing) & 1))) {
					ok = false;
					break;
				}
				tc_fence_after();
				const uint32_t a = smem_u32(sh.ring + slot * kSlotBytes);
				issue_oz_step(tmem, a, a + kSlices * kBlock, pass, st == 0);
				umma_commit(smem_u32(&sh.empty[slot]));
				issued = u + 1;
				if (u >= 1 && copied < total) {
					const int pu = u - 1;
					if (!mbar_wait(smem_u32(&sh.empty[pu % kRing]), (uint32_t)((pu / kRing) & 1))) {
						ok = false;
						break;
					}
					copy(copied++);
				}
			}
			// the last commit covers every MMA of the pass
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
		__syncthreads();
		tc_fence_after();
		if (sh.abort) break;
		// this thread's 64 columns of each accumulator of the pass, weighted 2^{-7 d}
#pragma unroll
		for (int dd = 0; dd < kDiagPerPass; dd++) {
			const int d = pass * kDiagPerPass + dd;
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
	if (!sh.abort) {
		// row n, grid points g0 + 32 half + jj (columns 2 jj, 2 jj + 1: re, im)
		const int n = n0 + q * 32 + lane;
		if (n < k) {
			const int ea = eA[n] - 14;
			double2* dst = out + (long long)n * G;
#pragma unroll
			for (int jj = 0; jj < 32; jj++) {
				const long long g = g0 + half * 32 + jj;
				if (g < G) {
					const double sc = ldexp(1.0, ea + eB[g]);
					dst[g] = make_double2(acc[2 * jj] * sc, acc[2 * jj + 1] * sc);
				}
			}
		}
	}
	tc_fence_before();
	__syncthreads();
	if (tid < 32) tmem_dealloc(tmem, kTmemCols);
}

size_t oz_smem() { return sizeof(OzShared) + 128; }

}  // namespace

bool oz_supported(int k, long long G) { return k >= 2 && k < 8300 && G >= 1; }

size_t oz_w_bytes(int k) {
	return (size_t)((k + TM - 1) / TM) * (size_t)((k + KS - 1) / KS) * kSlices * kBlock;
}

size_t oz_psi_bytes(int k, long long G) {
	return (size_t)((G + GT - 1) / GT) * (size_t)((k + KS - 1) / KS) * kSlices * kBlock;
}

size_t oz_exp_ints(int k, long long G) {
	return (size_t)((k + TM - 1) / TM) * TM + (size_t)((G + GT - 1) / GT) * GT;
}

void launch_rotate_oz(const double2* W, const double2* psi, int k, long long G, unsigned char* wsl,
		unsigned char* psl, int* ebuf, double2* out, int* err, cudaStream_t s, bool upper) {
	const int nt = (k + TM - 1) / TM, ks = (k + KS - 1) / KS;
	const long long gtiles = (G + GT - 1) / GT;
	int* eA = ebuf;
	int* eB = ebuf + (size_t)nt * TM;
	w_exp_kernel<<<(nt * TM + 255) / 256, 256, 0, s>>>(W, k, nt * TM, eA);
	psi_exp_kernel<<<(unsigned)((gtiles * GT + 255) / 256), 256, 0, s>>>(psi, k, G, gtiles * GT, eB);
	slice_w_kernel<<<dim3(nt, ks), 256, 0, s>>>(W, k, ks, eA, wsl);
	slice_psi_kernel<<<dim3((unsigned)gtiles, ks), 256, 0, s>>>(psi, k, G, ks, eB, psl);
	static bool attr = false;
	if (!attr) {
		cudaFuncSetAttribute(rotate_oz_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)oz_smem());
		attr = true;
	}
	rotate_oz_kernel<<<dim3(nt, (unsigned)gtiles), kThreads, oz_smem(), s>>>(wsl, psl, eA, eB, k, G, out, err,
			upper ? 1 : 0);
}

int oz_launches() { return 5; }

}  // namespace itp2d
