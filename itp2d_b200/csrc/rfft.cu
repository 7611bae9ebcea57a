// Row and column passes of the split operator for periodic lines of
// N = A * B points (N = 32 ... 1024, powers of two), with the line FFTs held
// in registers.
//
// One line is owned by B threads of one warp; thread t holds the A elements at
// positions t + B a (a = 0..A-1). A forward or backward DFT of the line is the
// two-stage (four-step) factorisation
//   Y[b][k1]      = sum_a x[B a + b] w_A^(a k1)                 (registers)
//   Y[b][k1]     *= w_N^(b k1)
//   X[k1 + A k2]  = sum_b Y[b][k1] w_B^(b k2)                   (registers)
// with one exchange of Y through shared memory between the stages (warp
// barriers only). Thread t then holds X at k1 = t + B i, all k2, that is at
// positions t + B (i + (A/B) k2): the same position set it started with, so an
// inverse transform, a pointwise table and a forward transform chain without
// any further data movement. The exchange index of Y[b][k1] is
// k1 B + (b xor (k1 mod B)), which makes both the writes (fixed k1) and the
// reads (fixed b) free of shared-memory bank conflicts for 8- and 16-byte
// elements. The in-register DFTs are radix-2 decimation in time with
// compile-time twiddle factors.
//
// Same arithmetic contract as the shared-memory Stockham passes in split.cu:
// unnormalised transforms with FFTW's sign convention (forward exp(-2 pi i jk/N)),
// tables applied as in RowPassArgs / ColPassArgs.
#include "split.cuh"

#include "../../include/itp2d_gpu.h"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>
#include <set>
#include <type_traits>
#include <utility>

namespace itp2d {

namespace {

constexpr int kThreads = 256;

// cos(2 pi j / 32) and sin(2 pi j / 32), j = 0..31.
__host__ __device__ constexpr double cos32(int j) {
	constexpr double c[32] = {
			1.0, 0.98078528040323044913, 0.92387953251128675613, 0.83146961230254523708,
			0.70710678118654752440, 0.55557023301960222474, 0.38268343236508977173, 0.19509032201612826785,
			0.0, -0.19509032201612826785, -0.38268343236508977173, -0.55557023301960222474,
			-0.70710678118654752440, -0.83146961230254523708, -0.92387953251128675613, -0.98078528040323044913,
			-1.0, -0.98078528040323044913, -0.92387953251128675613, -0.83146961230254523708,
			-0.70710678118654752440, -0.55557023301960222474, -0.38268343236508977173, -0.19509032201612826785,
			0.0, 0.19509032201612826785, 0.38268343236508977173, 0.55557023301960222474,
			0.70710678118654752440, 0.83146961230254523708, 0.92387953251128675613, 0.98078528040323044913};
	return c[j & 31];
}
__host__ __device__ constexpr double sin32(int j) { return cos32(j - 8); }

__host__ __device__ constexpr int bitrev(int i, int n) {
	int r = 0;
	for (int m = n >> 1; m > 0; m >>= 1, i >>= 1) r = (r << 1) | (i & 1);
	return r;
}

__host__ __device__ constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n >> 1); }

// Compile-time loop: f(std::integral_constant<int, I>) for I = 0 .. N-1, so
// that register-array indices inside f are constants.
template <class F, int... I>
__device__ __forceinline__ void sfor_impl(F&& f, std::integer_sequence<int, I...>) {
	(f(std::integral_constant<int, I>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void sfor(F&& f) {
	sfor_impl(f, std::make_integer_sequence<int, N>{});
}

// In-register DFT of length M (power of two, <= 32) of v[0..M), in place,
// natural order in and out: v[k] = sum_j v[j] exp(SIGN 2 pi i jk / M).
template <class R, int M, int SIGN>
__device__ __forceinline__ void dft_reg(c2<R>* v) {
	sfor<M>([&](auto I) {
		constexpr int i = I;
		constexpr int r = bitrev(i, M);
		if constexpr (r > i) {
			const c2<R> x = v[i];
			v[i] = v[r];
			v[r] = x;
		}
	});
	sfor<ilog2(M)>([&](auto S) {
		constexpr int m = 2 << S;
		constexpr int h = m >> 1;
		sfor<M / m>([&](auto G) {
			constexpr int base = G * m;
			sfor<h>([&](auto J) {
				constexpr int j = J;
				c2<R> x = v[base + j + h];
				if constexpr (j == 0) {
				} else if constexpr (4 * j == m) {
					x = cmul_i(x, SIGN);  // exp(SIGN i pi / 2)
				} else {
					constexpr double cr = cos32(j * (32 / m));
					constexpr double ci = SIGN * sin32(j * (32 / m));
					x = cmul(x, mk<R>((R)cr, (R)ci));
				}
				const c2<R> u = v[base + j];
				v[base + j] = cadd(u, x);
				v[base + j + h] = csub(u, x);
			});
		});
	});
}

// Transform of one line held as v[a] = x[t + B a]. xb(i): the line's
// exchange area, element i = 0..N-1 (a reference into shared memory); xtw:
// w_N^(b k1) at [k1 * B + b] (forward sign). On return v[a] = X[t + B a].
template <class R, int A, int B, int SIGN, class XB>
__device__ __forceinline__ void line_fft_x(c2<R>* v, int t, XB&& xb, const c2<R>* xtw) {
	constexpr int S2 = A / B;
	dft_reg<R, A, SIGN>(v);
	sfor<A - 1>([&](auto K) {
		constexpr int k1 = K + 1;
		c2<R> w = xtw[k1 * B + t];
		if (SIGN > 0) w.y = -w.y;
		v[k1] = cmul(v[k1], w);
	});
	__syncwarp();  // earlier readers of xb are done
	sfor<A>([&](auto K) {
		constexpr int k1 = K;
		xb(k1 * B + (t ^ (k1 & (B - 1)))) = v[k1];
	});
	__syncwarp();
	c2<R> u[A];
	sfor<S2>([&](auto I) {
		constexpr int i = I;
		const int k1 = t + B * i;
		sfor<B>([&](auto Bi) {
			constexpr int b = Bi;
			u[i * B + b] = xb(k1 * B + (b ^ t));
		});
		dft_reg<R, B, SIGN>(u + i * B);
	});
	sfor<S2>([&](auto I) {
		sfor<B>([&](auto K2) { v[I + S2 * K2] = u[I * B + K2]; });
	});
}

// The same with the exchange area at xb[i * es].
template <class R, int A, int B, int SIGN>
__device__ __forceinline__ void line_fft(c2<R>* v, int t, c2<R>* xb, int es, const c2<R>* xtw) {
	line_fft_x<R, A, B, SIGN>(v, t, [=](int i) -> c2<R>& { return xb[i * es]; }, xtw);
}

template <class R, int A, int B>
__device__ __forceinline__ void load_xtw(c2<R>* xtw, const c2<R>* tw) {
	constexpr int N = A * B;
	for (int i = threadIdx.x; i < N; i += blockDim.x) {
		const int k1 = i / B, b = i - k1 * B;
		xtw[i] = tw[(b * k1) & (N - 1)];
	}
}

// Row pass: 256 / B rows of one state per tile, tiles ordered state-fastest.
template <class R, int A, int B>
__global__ void __launch_bounds__(kThreads) row_reg_kernel(RowPassArgs a, int k) {
	using T = c2<R>;
	constexpr int N = A * B, LPI = kThreads / B;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	T* xtw = reinterpret_cast<T*>(smem_raw);
	T* xb = xtw + N;
	load_xtw<R, A, B>(xtw, reinterpret_cast<const T*>(a.lp.fft.tw));
	__syncthreads();
	const int line = threadIdx.x / B, t = threadIdx.x % B;
	T* lxb = xb + line * N;
	const int sx = a.sx;
	const int ntr = (a.sy + LPI - 1) / LPI;
	const long long total = (long long)k * ntr;
	const R* mpre = reinterpret_cast<const R*>(a.mul_pre);
	const R* mmid = reinterpret_cast<const R*>(a.mul_mid);
	const R* mpost = reinterpret_cast<const R*>(a.mul_post);
	const T* in = reinterpret_cast<const T*>(a.in);
	T* out = reinterpret_cast<T*>(a.out);
	const T* acc = reinterpret_cast<const T*>(a.acc);
	for (long long tile = blockIdx.x; tile < total; tile += gridDim.x) {
		const long long state = tile % k;
		const int y = (int)(tile / k) * LPI + line;
		const bool valid = y < a.sy;  // the whole warp runs the transforms
		const long long base = state * a.G + (long long)y * sx + t;
		const int toff = y * sx + t;
		T v[A];
#pragma unroll
		for (int i = 0; i < A; i++) v[i] = valid ? in[base + B * i] : mk<R>(0, 0);
		const R* m0 = a.do_inv ? mpre : mmid;
		if (m0 && valid) {
#pragma unroll
			for (int i = 0; i < A; i++) v[i] = cscale(v[i], m0[toff + B * i]);
		}
		if (a.do_inv) {
			line_fft<R, A, B, 1>(v, t, lxb, 1, xtw);
			if (mmid && valid) {
#pragma unroll
				for (int i = 0; i < A; i++) v[i] = cscale(v[i], mmid[toff + B * i]);
			}
		}
		if (a.do_fwd) {
			line_fft<R, A, B, -1>(v, t, lxb, 1, xtw);
			if (mpost && valid) {
#pragma unroll
				for (int i = 0; i < A; i++) v[i] = cscale(v[i], mpost[toff + B * i]);
			}
		}
		if (valid) {
			if (acc) {
#pragma unroll
				for (int i = 0; i < A; i++) v[i] = cadd(v[i], acc[base + B * i]);
			}
#pragma unroll
			for (int i = 0; i < A; i++) out[base + B * i] = v[i];
		}
	}
}

// Asynchronous global -> shared copy of one complex element.
template <class T> __device__ __forceinline__ void cp_async_elem(T* dst, const T* src);
template <> __device__ __forceinline__ void cp_async_elem<double2>(double2* dst, const double2* src) {
	const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
template <> __device__ __forceinline__ void cp_async_elem<float2>(float2* dst, const float2* src) {
	const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
	asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Column pass, in place: tiles of W = 256 / B columns x N rows of one state
// staged in shared memory ([y][c], row stride W + 1); tile tl covers columns
// (tl mod nct) W .. of state tl / nct, so the CTAs running at one time read
// the neighbouring column strips of the same rows (whole DRAM rows rather
// than one W-column strip of many states); each column line is
// transformed by B threads of one warp, using the line's own column of the
// tile as its exchange area. Persistent; with NBUF = 2 the next tile is copied
// in by cp.async while the current one is transformed (NBUF = 1 where two
// tiles do not fit in shared memory).
// FP32 lines of up to 256 points fit in 80 registers without spills: three
// CTAs per SM (the shared-memory tiles allow three as well). FP32 lines of
// 512 and 1024 points (32 values per thread) fit in 128 registers without
// spills when asked to: two CTAs per SM, each with a single tile buffer (two
// double-buffered CTAs would not fit in shared memory), so one CTA's loads
// overlap the other's transforms.
template <class R, int A, int B, int NBUF>
__global__ void __launch_bounds__(kThreads, (sizeof(R) == 4 && A <= 16) ? 3 : (sizeof(R) == 4 ? 2 : 0))
		col_reg_kernel(ColPassArgs a, int k) {
	using T = c2<R>;
	constexpr int N = A * B, W = kThreads / B, LD = W + 1, TS = N * LD;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	T* xtw = reinterpret_cast<T*>(smem_raw);
	T* tiles = xtw + N;
	load_xtw<R, A, B>(xtw, reinterpret_cast<const T*>(a.lp.fft.tw));
	const int line = threadIdx.x / B, t = threadIdx.x % B;
	const int sx = a.sx;
	const int nct = (sx + W - 1) / W;
	const long long total = (long long)k * nct;
	const R* m2 = reinterpret_cast<const R*>(a.mul2d);
	const R* m1 = reinterpret_cast<const R*>(a.mul1d);
	T* data = reinterpret_cast<T*>(a.data);
	// copies tile tl into dst (asynchronously when NBUF = 2); columns beyond sx read as zero
	auto fetch = [&](T* dst, long long tl) {
		const long long state = tl / nct;
		const int col0 = (int)(tl % nct) * W;
		const int ncols = min(W, sx - col0);
		const T* src = data + state * a.G + col0;
#pragma unroll
		for (int it = 0; it < N * W / kThreads; it++) {
			const int i = it * kThreads + threadIdx.x;
			const int y = i / W, c = i - y * W;
			if (c >= ncols) dst[y * LD + c] = mk<R>(0, 0);
			else if (NBUF == 2) cp_async_elem<T>(dst + y * LD + c, src + (long long)y * sx + c);
			else dst[y * LD + c] = src[(long long)y * sx + c];
		}
	};
	long long tl = blockIdx.x;
	int cur = 0;
	if (NBUF == 2) {
		if (tl < total) fetch(tiles, tl);
		cp_async_commit();
	}
	for (; tl < total; tl += gridDim.x) {
		T* tile = tiles + cur * TS;
		if (NBUF == 2) {
			const long long nx = tl + gridDim.x;
			if (nx < total) fetch(tiles + (cur ^ 1) * TS, nx);
			cp_async_commit();
			cp_async_wait<1>();  // this thread's copies of the current tile have landed
			__syncthreads();
		} else {
			fetch(tile, tl);
			__syncthreads();
		}
		const long long state = tl / nct;
		const int col0 = (int)(tl % nct) * W;
		const int ncols = min(W, sx - col0);
		T v[A];
#pragma unroll
		for (int i = 0; i < A; i++) v[i] = tile[(t + B * i) * LD + line];
		T* lxb = tile + line;
		if (a.mode == 0 || a.mode == 1) line_fft<R, A, B, -1>(v, t, lxb, LD, xtw);
		if (a.mode == 0) {
			const bool valid = line < ncols;
#pragma unroll
			for (int i = 0; i < A; i++) {
				const int y = t + B * i;
				const R f = !valid ? (R)0 : (m2 ? m2[y * sx + col0 + line] : m1[y]);
				v[i] = cscale(v[i], f);
			}
		}
		if (a.mode == 0 || a.mode == 2) line_fft<R, A, B, 1>(v, t, lxb, LD, xtw);
		__syncwarp();
#pragma unroll
		for (int i = 0; i < A; i++) tile[(t + B * i) * LD + line] = v[i];
		__syncthreads();
		T* dst = data + state * a.G + col0;
#pragma unroll
		for (int it = 0; it < N * W / kThreads; it++) {
			const int i = it * kThreads + threadIdx.x;
			const int y = i / W, c = i - y * W;
			if (c < ncols) dst[(long long)y * sx + c] = tile[y * LD + c];
		}
		__syncthreads();  // the tile buffer is refilled by a later fetch
		if (NBUF == 2) cur ^= 1;
	}
	if (NBUF == 2) cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// Column pass with TMA tile movement (kColTma).
//
// A tile is one 128-byte wide strip of a state: W = 128 / sizeof(complex)
// columns (16 FP32, 8 FP64) by all N rows, brought into shared memory by
// cp.async.bulk.tensor (a 3-D tensor map over k x sy x sx in 8-byte units,
// boxes of 16 units x min(N, 256) rows, 128-byte swizzle) and written back by
// the same engine after the in-place transform. S = 3 slots form a ring: the
// tile two steps ahead is in flight while one is transformed. One thread
// (the leader, thread 0, also a transform thread) issues the copies: after
// every transform thread has written tile j back (mbarrier `done`), it
// stores tile j, then refills the slot of tile j - 1 (whose store has
// finished reading) with tile j - 1 + S. Transform threads only wait for
// `full` of their next tile, so no block-wide barrier sits in the loop.
// Column line `line` of a tile is transformed by B threads of one warp as in
// col_reg_kernel, using its own column of the slot as the exchange area.
// Every wait is bounded (one second of global time); on time-out the kernel
// records ITP2D_E_TIMEOUT in *err, waits (bounded) for its copies in flight
// and returns.

constexpr unsigned long long kTmaWaitNs = 1000000000ULL;

__device__ __forceinline__ uint32_t sh_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long gtime_ns() {
	unsigned long long t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

__device__ __forceinline__ bool mbar_try(uint32_t mb, uint32_t parity) {
	uint32_t ok;
	asm volatile(
			"{\n\t.reg .pred P1;\n\t"
			"mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
			"selp.b32 %0, 1, 0, P1;\n\t}\n"
			: "=r"(ok)
			: "r"(mb), "r"(parity)
			: "memory");
	return ok != 0;
}

// Bounded wait for the phase with the given parity; false on time-out.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t mb, uint32_t parity) {
	if (mbar_try(mb, parity)) return true;
	const unsigned long long t0 = gtime_ns();
	for (long long i = 0; i < (1LL << 26); i++) {
		if (mbar_try(mb, parity)) return true;
		__nanosleep(32);
		if ((i & 63) == 0 && gtime_ns() - t0 > kTmaWaitNs) return false;
	}
	return false;
}

__device__ __forceinline__ void tma_load3(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t mb) {
	asm volatile(
			"cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
			"[%5];" ::"r"(dst),
			"l"(map), "r"(x), "r"(y), "r"(z), "r"(mb)
			: "memory");
}

__device__ __forceinline__ void tma_store3(const CUtensorMap* map, int x, int y, int z, uint32_t src) {
	asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(map),
			"r"(x), "r"(y), "r"(z), "r"(src)
			: "memory");
}

// Byte offset of element (row r, column c) of a tile: 128-byte rows, the
// 16-byte chunk index of row r XORed with r mod 8 (the TMA 128-byte swizzle).
template <int ES>
__device__ __forceinline__ uint32_t swz(int r, int c) {
	const int byte = c * ES;
	return (uint32_t)(r * 128 + ((((byte >> 4) ^ (r & 7))) << 4) + (byte & 15));
}

template <class R, int A, int B, int S>
__global__ void __launch_bounds__((128 / (2 * (int)sizeof(R))) * B)
		col_tma_kernel(const __grid_constant__ CUtensorMap map, ColPassArgs a, int k) {
	using T = c2<R>;
	constexpr int ES = (int)sizeof(T), N = A * B, W = 128 / ES, NT = W * B;
	constexpr int TILE = N * 128, BOX = N < 256 ? N : 256, U = ES / 8;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	unsigned char* base =
			reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
	T* xtw = reinterpret_cast<T*>(base + S * TILE);
	unsigned long long* full = reinterpret_cast<unsigned long long*>(xtw + N);
	unsigned long long* done = full + S;
	load_xtw<R, A, B>(xtw, reinterpret_cast<const T*>(a.lp.fft.tw));
	const bool leader = threadIdx.x == 0;
	if (leader) {
		for (int s = 0; s < S; s++) {
			asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sh_u32(full + s)), "r"(1) : "memory");
			asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sh_u32(done + s)), "r"(NT) : "memory");
		}
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	__syncthreads();
	const int sx = a.sx;
	const int nct = (sx + W - 1) / W;
	const long long total = (long long)k * nct;
	auto tile_of = [&](long long j) { return (long long)blockIdx.x + j * gridDim.x; };
	int issued[S], seen[S];  // leader: loads issued and done phases seen per slot
#pragma unroll
	for (int s = 0; s < S; s++) issued[s] = seen[s] = 0;
	auto load = [&](int s, long long tl) {
		const int st = (int)(tl / nct), x = (int)(tl % nct) * W * U;
		asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sh_u32(full + s)), "r"(TILE)
				: "memory");
#pragma unroll
		for (int h = 0; h < N / BOX; h++) tma_load3(sh_u32(base + s * TILE + h * BOX * 128), &map, x, h * BOX, st,
				sh_u32(full + s));
		issued[s]++;
	};
	if (leader) {
		asm volatile("prefetch.tensormap [%0];" ::"l"(&map) : "memory");
		for (int s = 0; s < S; s++)
			if (tile_of(s) < total) load(s, tile_of(s));
	}
	const int line = threadIdx.x / B, t = threadIdx.x % B;
	const R* m2 = reinterpret_cast<const R*>(a.mul2d);
	const R* m1 = reinterpret_cast<const R*>(a.mul1d);
	bool ok = true;
	long long j = 0;
	for (; tile_of(j) < total; j++) {
		const long long tl = tile_of(j);
		const int s = (int)(j % S);
		const uint32_t par = (uint32_t)((j / S) & 1);
		if (!mbar_wait_bounded(sh_u32(full + s), par)) {
			ok = false;
			break;
		}
		unsigned char* tile = base + s * TILE;
		auto X = [&](int r) -> T& { return *reinterpret_cast<T*>(tile + swz<ES>(r, line)); };
		const int col0 = (int)(tl % nct) * W;
		T v[A];
#pragma unroll
		for (int i = 0; i < A; i++) v[i] = X(t + B * i);
		if (a.mode == 0 || a.mode == 1) line_fft_x<R, A, B, -1>(v, t, X, xtw);
		if (a.mode == 0) {
			const bool valid = col0 + line < sx;
#pragma unroll
			for (int i = 0; i < A; i++) {
				const int y = t + B * i;
				const R f = !valid ? (R)0 : (m2 ? m2[y * sx + col0 + line] : m1[y]);
				v[i] = cscale(v[i], f);
			}
		}
		if (a.mode == 0 || a.mode == 2) line_fft_x<R, A, B, 1>(v, t, X, xtw);
		__syncwarp();
#pragma unroll
		for (int i = 0; i < A; i++) X(t + B * i) = v[i];
		asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
		asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(sh_u32(done + s)) : "memory");
		if (leader) {
			if (!mbar_wait_bounded(sh_u32(done + s), par)) {
				ok = false;
				break;
			}
			seen[s]++;
			const int st = (int)(tl / nct), x = (int)(tl % nct) * W * U;
#pragma unroll
			for (int h = 0; h < N / BOX; h++) tma_store3(&map, x, h * BOX, st, sh_u32(tile + h * BOX * 128));
			asm volatile("cp.async.bulk.commit_group;" ::: "memory");
			if (j >= 1) {
				// the slot of tile j - 1: its store (the older group) has read it
				asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
				const int s1 = (int)((j - 1) % S);
				if (tile_of(j - 1 + S) < total) load(s1, tile_of(j - 1 + S));
			}
		}
	}
	if (!ok) atomicExch(a.err, ITP2D_E_TIMEOUT);
	if (leader) {
		// copies still in flight: loads not yet consumed (error path only), then
		// every store
		for (int s = 0; s < S; s++)
			if (issued[s] > seen[s]) mbar_wait_bounded(sh_u32(full + s), (uint32_t)((issued[s] - 1) & 1));
		asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
	}
}

// Energy sums of one element: Re, Im <psi|h>, <h|h>, |h - es psi|^2, <psi|psi>.
template <class T>
__device__ __forceinline__ void esums(double* s, T p, T h, double es) {
	const double pr = p.x, pi = p.y, hr = h.x, hi = h.y;
	s[0] += pr * hr + pi * hi;
	s[1] += pr * hi - pi * hr;
	s[2] += hr * hr + hi * hi;
	const double dr = hr - es * pr, di = hi - es * pi;
	s[3] += dr * dr + di * di;
	s[4] += pr * pr + pi * pi;
}

// Deterministic CTA reduction of the five sums into out[0..5) (thread 0).
__device__ __forceinline__ void reduce5(double* s, double* red, double* out) {
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
	for (int j = 0; j < 5; j++)
		for (int o = 16; o > 0; o >>= 1) s[j] += __shfl_xor_sync(0xffffffffu, s[j], o);
	__syncthreads();
	if (lane == 0)
		for (int j = 0; j < 5; j++) red[warp * 5 + j] = s[j];
	__syncthreads();
	if (threadIdx.x == 0)
		for (int j = 0; j < 5; j++) {
			double v = 0.0;
			for (int w = 0; w < kThreads / 32; w++) v += red[w * 5 + j];
			out[j] = v;
		}
}

// Energy row pass (grid: states x row tiles of 256 / B rows):
//   t = Tinv_x(tmul .* Tfwd_x(src_t)) (do_fwd) or Tinv_x(src_t);
//   h = t + V .* psi; h -> h_out; per-tile sums.
template <class R, int A, int B>
__global__ void __launch_bounds__(kThreads) energy_row_reg_kernel(EnergyRowArgs a) {
	using T = c2<R>;
	constexpr int N = A * B, LPI = kThreads / B;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	T* xtw = reinterpret_cast<T*>(smem_raw);
	T* xb = xtw + N;
	double* red = reinterpret_cast<double*>(xb + LPI * N);
	load_xtw<R, A, B>(xtw, reinterpret_cast<const T*>(a.lp.fft.tw));
	__syncthreads();
	const int line = threadIdx.x / B, t = threadIdx.x % B;
	const long long state = blockIdx.x;
	const int y = blockIdx.y * LPI + line;
	const bool valid = y < a.sy;
	const long long base = state * a.G + (long long)y * a.sx + t;
	const int toff = y * a.sx + t;
	const T* src = reinterpret_cast<const T*>(a.src_t);
	T v[A];
#pragma unroll
	for (int i = 0; i < A; i++) v[i] = valid ? src[base + B * i] : mk<R>(0, 0);
	if (a.do_fwd) {
		line_fft<R, A, B, -1>(v, t, xb + line * N, 1, xtw);
		const R* tm = reinterpret_cast<const R*>(a.tmul);
		if (valid) {
#pragma unroll
			for (int i = 0; i < A; i++) v[i] = cscale(v[i], tm[toff + B * i]);
		}
	}
	line_fft<R, A, B, 1>(v, t, xb + line * N, 1, xtw);
	double s[5] = {0, 0, 0, 0, 0};
	if (valid) {
		const T* psi = reinterpret_cast<const T*>(a.psi);
		const R* V = reinterpret_cast<const R*>(a.V);
		T* hout = reinterpret_cast<T*>(a.h_out);
		const double es = a.Eshift ? a.Eshift[state] : 0.0;
#pragma unroll
		for (int i = 0; i < A; i++) {
			T h = v[i];
			const T p = psi[base + B * i];
			if (V) {
				const R w = V[toff + B * i];
				h.x += w * p.x;
				h.y += w * p.y;
			}
			if (hout) hout[base + B * i] = h;
			if (a.sums) esums(s, p, h, es);
		}
	}
	if (a.sums) reduce5(s, red, a.sums + ((size_t)state * gridDim.y + blockIdx.y) * 5);
}

// Energy column pass (magnetic field): t = Tinv_y(ty .* Tfwd_y(src)),
// h = t + add_in; h -> h_out; per-tile sums against psi at
// sums[(state * ntiles + tile) * 5]. Persistent over tiles of 256 / B columns
// of one state, with the next tile's src copied in by cp.async while the
// current one is transformed (NBUF = 2; NBUF = 1 where two tiles do not fit).
template <class R, int A, int B, int NBUF>
__global__ void __launch_bounds__(kThreads, (sizeof(R) == 4 && A <= 16) ? 3 : 0)
		energy_col_reg_kernel(EnergyColArgs a, int k) {
	using T = c2<R>;
	constexpr int N = A * B, W = kThreads / B, LD = W + 1, TS = N * LD;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	T* xtw = reinterpret_cast<T*>(smem_raw);
	T* tiles = xtw + N;
	double* red = reinterpret_cast<double*>(tiles + NBUF * TS);
	load_xtw<R, A, B>(xtw, reinterpret_cast<const T*>(a.lp.fft.tw));
	const int line = threadIdx.x / B, t = threadIdx.x % B;
	const int sx = a.sx;
	const int nct = (sx + W - 1) / W;
	const long long total = (long long)k * nct;
	const T* psi_all = reinterpret_cast<const T*>(a.psi);
	const T* src_all = a.src ? reinterpret_cast<const T*>(a.src) : psi_all;
	auto fetch = [&](T* dst, long long tl) {
		const long long state = tl / nct;
		const int col0 = (int)(tl % nct) * W;
		const int ncols = min(W, sx - col0);
		const T* src = src_all + state * a.G + col0;
#pragma unroll
		for (int it = 0; it < N * W / kThreads; it++) {
			const int i = it * kThreads + threadIdx.x;
			const int y = i / W, c = i - y * W;
			if (c >= ncols) dst[y * LD + c] = mk<R>(0, 0);
			else if (NBUF == 2) cp_async_elem<T>(dst + y * LD + c, src + (long long)y * sx + c);
			else dst[y * LD + c] = src[(long long)y * sx + c];
		}
	};
	const R* ty = reinterpret_cast<const R*>(a.ty);
	long long tl = blockIdx.x;
	int cur = 0;
	if (NBUF == 2) {
		if (tl < total) fetch(tiles, tl);
		cp_async_commit();
	}
	for (; tl < total; tl += gridDim.x) {
		T* tile = tiles + cur * TS;
		if (NBUF == 2) {
			const long long nx = tl + gridDim.x;
			if (nx < total) fetch(tiles + (cur ^ 1) * TS, nx);
			cp_async_commit();
			cp_async_wait<1>();
			__syncthreads();
		} else {
			fetch(tile, tl);
			__syncthreads();
		}
		const long long state = tl / nct;
		const int ct = (int)(tl % nct);
		const int col0 = ct * W;
		const int ncols = min(W, sx - col0);
		const long long base = state * a.G + col0;
		T v[A];
#pragma unroll
		for (int i = 0; i < A; i++) v[i] = tile[(t + B * i) * LD + line];
		line_fft<R, A, B, -1>(v, t, tile + line, LD, xtw);
#pragma unroll
		for (int i = 0; i < A; i++) v[i] = cscale(v[i], ty[t + B * i]);
		line_fft<R, A, B, 1>(v, t, tile + line, LD, xtw);
		__syncwarp();
#pragma unroll
		for (int i = 0; i < A; i++) tile[(t + B * i) * LD + line] = v[i];
		__syncthreads();
		const T* add = reinterpret_cast<const T*>(a.add_in) + base;
		const T* psi = psi_all + base;
		T* hout = a.h_out ? reinterpret_cast<T*>(a.h_out) + base : nullptr;
		const double es = a.Eshift ? a.Eshift[state] : 0.0;
		double s[5] = {0, 0, 0, 0, 0};
		// the global loads of EB rows at once (the compiler cannot move them
		// across the hout stores): one latency per EB rows instead of per row
		constexpr int NE = N * W / kThreads, EB = NE < 8 ? NE : 8;
		static_assert(NE % EB == 0, "epilogue batches");
#pragma unroll
		for (int b0 = 0; b0 < NE; b0 += EB) {
			T av[EB], pv[EB];
#pragma unroll
			for (int e = 0; e < EB; e++) {
				const int i = (b0 + e) * kThreads + threadIdx.x;
				const int y = i / W, c = i - y * W;
				const long long off = (long long)y * sx + c;
				av[e] = c < ncols ? add[off] : mk<R>(0, 0);
				pv[e] = c < ncols ? psi[off] : mk<R>(0, 0);
			}
#pragma unroll
			for (int e = 0; e < EB; e++) {
				const int i = (b0 + e) * kThreads + threadIdx.x;
				const int y = i / W, c = i - y * W;
				if (c < ncols) {
					const long long off = (long long)y * sx + c;
					const T h = cadd(tile[y * LD + c], av[e]);
					if (hout) hout[off] = h;
					if (a.sums) esums(s, pv[e], h, es);
				}
			}
		}
		if (a.sums) reduce5(s, red, a.sums + ((size_t)state * nct + ct) * 5);
		__syncthreads();  // the tile buffer is refilled by a later fetch
		if (NBUF == 2) cur ^= 1;
	}
	if (NBUF == 2) cp_async_wait<0>();
}

template <class K>
void opt_in_smem(K kernel, size_t bytes) {
	static std::mutex mu;
	static std::set<const void*> done;
	std::lock_guard<std::mutex> g(mu);
	if (bytes > 48 * 1024 && done.insert((const void*)kernel).second)
		cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
}

template <class K>
int grid_for(K kernel, size_t smem, long long tiles) {
	static int sms = 0;
	if (!sms) {
		int dev = 0;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	}
	int per_sm = 0;
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, smem);
	const long long b = (long long)std::max(1, per_sm) * std::max(1, sms);
	return (int)std::max(1LL, std::min(b, tiles));
}

template <class R, int A, int B>
void row_reg(const RowPassArgs& a, int k, cudaStream_t s) {
	constexpr int N = A * B;
	const size_t sm = (size_t)(N + (kThreads / B) * N) * sizeof(c2<R>);
	opt_in_smem(row_reg_kernel<R, A, B>, sm);
	const long long tiles = (long long)k * ((a.sy + kThreads / B - 1) / (kThreads / B));
	row_reg_kernel<R, A, B><<<grid_for(row_reg_kernel<R, A, B>, sm, tiles), kThreads, sm, s>>>(a, k);
}

template <class R, int A, int B>
void col_reg(const ColPassArgs& a, int k, cudaStream_t s) {
	constexpr int N = A * B, W = kThreads / B;
	constexpr size_t tile_bytes = (size_t)N * (W + 1) * sizeof(c2<R>);
	// FP32 lines of 32 values per thread run two single-buffered CTAs per SM
	constexpr bool two_ctas = sizeof(R) == 4 && A > 16;
	constexpr int NBUF = (!two_ctas && 2 * tile_bytes + N * sizeof(c2<R>) <= 220 * 1024) ? 2 : 1;
	const size_t sm = N * sizeof(c2<R>) + NBUF * tile_bytes;
	opt_in_smem(col_reg_kernel<R, A, B, NBUF>, sm);
	const long long tiles = (long long)k * ((a.sx + W - 1) / W);
	col_reg_kernel<R, A, B, NBUF><<<grid_for(col_reg_kernel<R, A, B, NBUF>, sm, tiles), kThreads, sm, s>>>(a, k);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
	static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
	static std::once_flag once;
	std::call_once(once, [] {
		void* p = nullptr;
		cudaDriverEntryPointQueryResult q;
		if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
				q == cudaDriverEntryPointSuccess)
			fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
	});
	return fn;
}

constexpr int kTmaStages = 3;

// Tensor map of a k x sy x sx complex state array in 8-byte units, boxes of
// 16 units (128 bytes) by min(N, 256) rows, 128-byte swizzle.
template <class R>
bool encode_state_map(CUtensorMap* m, void* data, int sx, int sy, int k) {
	auto enc = tensor_map_encoder();
	if (!enc) return false;
	constexpr int U = (int)sizeof(c2<R>) / 8;
	const cuuint64_t dims[3] = {(cuuint64_t)sx * U, (cuuint64_t)sy, (cuuint64_t)k};
	const cuuint64_t strides[2] = {(cuuint64_t)sx * U * 8, (cuuint64_t)sx * sy * U * 8};
	const cuuint32_t box[3] = {16, (cuuint32_t)std::min(sy, 256), 1};
	const cuuint32_t estr[3] = {1, 1, 1};
	return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, data, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
	               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
	               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The TMA column pass (lines of 256 or 512 points); false when it does not
// apply (no tensor-map encoder, data not 16-byte aligned, rows not a
// multiple of 16 bytes, no error word).
template <class R, int A, int B>
bool col_tma(const ColPassArgs& a, int k, cudaStream_t s) {
	constexpr int N = A * B, ES = (int)sizeof(c2<R>), W = 128 / ES, S = kTmaStages;
	static_assert(N <= 512, "three 128-byte tiles of the line must fit in shared memory");
	if (a.sy != N || !a.err || (reinterpret_cast<uintptr_t>(a.data) & 15) || ((long long)a.sx * ES) % 16) return false;
	CUtensorMap map;
	if (!encode_state_map<R>(&map, a.data, a.sx, a.sy, k)) return false;
	const size_t sm = 1024 + (size_t)S * N * 128 + N * sizeof(c2<R>) + 2 * S * sizeof(unsigned long long);
	opt_in_smem(col_tma_kernel<R, A, B, S>, sm);
	const long long tiles = (long long)k * ((a.sx + W - 1) / W);
	static int sms = 0;
	if (!sms) {
		int dev = 0;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	}
	int per_sm = 0;
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, col_tma_kernel<R, A, B, S>, W * B, sm);
	const int grid = (int)std::max(1LL, std::min((long long)std::max(1, per_sm) * std::max(1, sms), tiles));
	col_tma_kernel<R, A, B, S><<<grid, W * B, sm, s>>>(map, a, k);
	return true;
}

template <class R, int A, int B>
void energy_row_reg(const EnergyRowArgs& a, int k, cudaStream_t s) {
	constexpr int N = A * B, LPI = kThreads / B;
	const size_t sm = (size_t)(N + LPI * N) * sizeof(c2<R>) + 5 * (kThreads / 32) * sizeof(double);
	opt_in_smem(energy_row_reg_kernel<R, A, B>, sm);
	energy_row_reg_kernel<R, A, B><<<dim3(k, (a.sy + LPI - 1) / LPI), kThreads, sm, s>>>(a);
}

template <class R, int A, int B>
void energy_col_reg(const EnergyColArgs& a, int k, cudaStream_t s) {
	constexpr int N = A * B, W = kThreads / B;
	constexpr size_t tile_bytes = (size_t)N * (W + 1) * sizeof(c2<R>);
	constexpr int NBUF = (2 * tile_bytes + N * sizeof(c2<R>) <= 220 * 1024) ? 2 : 1;
	const size_t sm = N * sizeof(c2<R>) + NBUF * tile_bytes + 5 * (kThreads / 32) * sizeof(double);
	opt_in_smem(energy_col_reg_kernel<R, A, B, NBUF>, sm);
	const long long tiles = (long long)k * ((a.sx + W - 1) / W);
	energy_col_reg_kernel<R, A, B, NBUF>
			<<<grid_for(energy_col_reg_kernel<R, A, B, NBUF>, sm, tiles), kThreads, sm, s>>>(a, k);
}

// Threads per line (B) of the register path for line length N, 0 if none.
int reg_threads(int N) {
	switch (N) {
		case 32: return 4;
		case 64: return 8;
		case 128: return 8;
		case 256: return 16;
		case 512: return 16;
		case 1024: return 32;
		default: return 0;
	}
}

}  // namespace

int energy_row_tile_reg(const LinePlan& lp, int) {
	const int B = lp.kind == 0 ? reg_threads(lp.N) : 0;
	return B ? kThreads / B : 0;
}

int energy_col_tile_reg(const LinePlan& lp, int) {
	const int B = lp.kind == 0 ? reg_threads(lp.N) : 0;
	return B ? kThreads / B : 0;
}

template <class R>
bool launch_energy_row_reg(const EnergyRowArgs& a, int k, cudaStream_t s) {
	if (a.lp.kind != 0 || a.rows_per_tile == 0 || a.rows_per_tile != energy_row_tile_reg(a.lp, a.sy)) return false;
	switch (a.sx) {
		case 32: energy_row_reg<R, 8, 4>(a, k, s); return true;
		case 64: energy_row_reg<R, 8, 8>(a, k, s); return true;
		case 128: energy_row_reg<R, 16, 8>(a, k, s); return true;
		case 256: energy_row_reg<R, 16, 16>(a, k, s); return true;
		case 512: energy_row_reg<R, 32, 16>(a, k, s); return true;
		case 1024: energy_row_reg<R, 32, 32>(a, k, s); return true;
		default: return false;
	}
}

template <class R>
bool launch_energy_col_reg(const EnergyColArgs& a, int k, cudaStream_t s) {
	if (a.lp.kind != 0 || a.cols_per_tile == 0 || a.cols_per_tile != energy_col_tile_reg(a.lp, a.sx)) return false;
	switch (a.sy) {
		case 32: energy_col_reg<R, 8, 4>(a, k, s); return true;
		case 64: energy_col_reg<R, 8, 8>(a, k, s); return true;
		case 128: energy_col_reg<R, 16, 8>(a, k, s); return true;
		case 256: energy_col_reg<R, 16, 16>(a, k, s); return true;
		case 512: energy_col_reg<R, 32, 16>(a, k, s); return true;
		case 1024: energy_col_reg<R, 32, 32>(a, k, s); return true;
		default: return false;
	}
}

template <class R>
bool launch_row_pass_reg(const RowPassArgs& a, int k, cudaStream_t s) {
	if (a.lp.kind != 0) return false;
	switch (a.sx) {
		case 32: row_reg<R, 8, 4>(a, k, s); return true;
		case 64: row_reg<R, 8, 8>(a, k, s); return true;
		case 128: row_reg<R, 16, 8>(a, k, s); return true;
		case 256: row_reg<R, 16, 16>(a, k, s); return true;
		case 512: row_reg<R, 32, 16>(a, k, s); return true;
		case 1024: row_reg<R, 32, 32>(a, k, s); return true;
		default: return false;
	}
}

template <class R>
bool launch_col_pass_reg(const ColPassArgs& a, int k, cudaStream_t s) {
	if (a.lp.kind != 0) return false;
	if (a.variant == kColTma) {
		if (a.sy == 256 && col_tma<R, 16, 16>(a, k, s)) return true;
		if (a.sy == 512 && col_tma<R, 32, 16>(a, k, s)) return true;
	}
	switch (a.sy) {
		case 32: col_reg<R, 8, 4>(a, k, s); return true;
		case 64: col_reg<R, 8, 8>(a, k, s); return true;
		case 128: col_reg<R, 16, 8>(a, k, s); return true;
		case 256: col_reg<R, 16, 16>(a, k, s); return true;
		case 512: col_reg<R, 32, 16>(a, k, s); return true;
		case 1024: col_reg<R, 32, 32>(a, k, s); return true;
		default: return false;
	}
}

template <class R>
int tune_col_pass_reg(ColPassArgs a, int k, cudaStream_t s) {
	if (a.lp.kind != 0 || reg_threads(a.sy) == 0) return -1;
	if (a.sy != 256 && a.sy != 512) return kColRegSmem;  // the only register variant at other sizes
	cudaEvent_t e0, e1;
	if (cudaEventCreate(&e0) != cudaSuccess) return kColRegSmem;
	if (cudaEventCreate(&e1) != cudaSuccess) {
		cudaEventDestroy(e0);
		return kColRegSmem;
	}
	int best = kColRegSmem;
	float best_ms = 0.0f;
	for (int v = 0; v < kColVariants; v++) {
		a.variant = v;
		float ms = 0.0f;
		bool ran = true;
		for (int rep = 0; rep < 4 && ran; rep++) {  // the first run is a warm-up
			cudaEventRecord(e0, s);
			if (v == kColTma) {
				ran = (a.sy == 256) ? col_tma<R, 16, 16>(a, k, s) : col_tma<R, 32, 16>(a, k, s);
			} else {
				if (a.sy == 256) col_reg<R, 16, 16>(a, k, s);
				else col_reg<R, 32, 16>(a, k, s);
			}
			cudaEventRecord(e1, s);
			if (cudaEventSynchronize(e1) != cudaSuccess) ran = false;
			float t = 0.0f;
			cudaEventElapsedTime(&t, e0, e1);
			if (rep > 0) ms += t;
		}
		if (!ran || cudaGetLastError() != cudaSuccess) continue;
		if (v == kColRegSmem || ms < best_ms) {
			best = v;
			best_ms = ms;
		}
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	return best;
}

template int tune_col_pass_reg<double>(ColPassArgs, int, cudaStream_t);
template int tune_col_pass_reg<float>(ColPassArgs, int, cudaStream_t);
template bool launch_row_pass_reg<double>(const RowPassArgs&, int, cudaStream_t);
template bool launch_row_pass_reg<float>(const RowPassArgs&, int, cudaStream_t);
template bool launch_col_pass_reg<double>(const ColPassArgs&, int, cudaStream_t);
template bool launch_col_pass_reg<float>(const ColPassArgs&, int, cudaStream_t);
template bool launch_energy_row_reg<double>(const EnergyRowArgs&, int, cudaStream_t);
template bool launch_energy_row_reg<float>(const EnergyRowArgs&, int, cudaStream_t);
template bool launch_energy_col_reg<double>(const EnergyColArgs&, int, cudaStream_t);
template bool launch_energy_col_reg<float>(const EnergyColArgs&, int, cudaStream_t);

}  // namespace itp2d
