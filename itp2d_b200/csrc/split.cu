// Split-operator row/column passes and Hamiltonian energy passes.
//
// Each CTA stages one tile (a few rows, or a few columns of one state) in
// shared memory, transforms it along x or y (fft.cuh), applies the fused
// pointwise tables and writes it back: one HBM round trip per pass. The grid
// is (k states, tiles) with the state index fastest so that CTAs running at the
// same time read the same rows of the (state-independent) tables from L2.
#include "fft.cuh"
#include "split.cuh"

#include <algorithm>
#include <mutex>
#include <set>

namespace itp2d {

namespace {

constexpr int kThreads = 256;
constexpr int kTileBytes = 32768;  // shared-memory bytes per ping-pong buffer

template <class R>
__device__ __forceinline__ void load_twiddles(c2<R>* tw, const LinePlan& lp) {
	const c2<R>* g = reinterpret_cast<const c2<R>*>(lp.fft.tw);
	for (int i = threadIdx.x; i < lp.fft.n; i += blockDim.x) tw[i] = g[i];
}

// Asynchronous global -> shared copy of one complex element (cp.async: the
// data does not pass through registers, so a CTA can have the next tile in
// flight while it transforms the current one).
template <class R> __device__ __forceinline__ void cp_elem(c2<R>* dst, const c2<R>* src);
template <> __device__ __forceinline__ void cp_elem<double>(double2* dst, const double2* src) {
	const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
template <> __device__ __forceinline__ void cp_elem<float>(float2* dst, const float2* src) {
	const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
	asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Row pass, persistent and double-buffered: tile t (rows_per_tile rows of one
// state; tiles ordered state-fastest) is transformed while tile t + grid is
// being copied in. Shared memory: two tile buffers, one scratch buffer for the
// FFT ping-pong, the twiddles.
template <class R>
__global__ void __launch_bounds__(kThreads) row_pass_kernel(RowPassArgs a, int k) {
	using T = c2<R>;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int L = a.lp.kind == 0 ? a.sx : 2 * a.sx;
	const int rows = a.rows_per_tile;
	const int tsz = rows * L;
	T* tiles = reinterpret_cast<T*>(smem_raw);
	T* scr = tiles + 2 * tsz;
	T* tw = scr + tsz;
	load_twiddles<R>(tw, a.lp);
	const int sx = a.sx;
	const int ntr = (a.sy + rows - 1) / rows;
	const long long total = (long long)k * ntr;
	const R* mpre = reinterpret_cast<const R*>(a.mul_pre);
	const R* mmid = reinterpret_cast<const R*>(a.mul_mid);
	const R* mpost = reinterpret_cast<const R*>(a.mul_post);

	long long t = blockIdx.x;
	int cur = 0;
	auto issue = [&](T* dst, long long tt) {
		const long long state = tt % k;
		const int row0 = (int)(tt / k) * rows;
		const int nrows = min(rows, a.sy - row0);
		const T* in = reinterpret_cast<const T*>(a.in) + state * a.G + (long long)row0 * sx;
		for (int i = threadIdx.x; i < nrows * sx; i += blockDim.x) {
			const int r = i / sx;
			cp_elem<R>(dst + r * L + (i - r * sx), in + i);
		}
	};
	if (t < total) issue(tiles, t);
	cp_commit();
	for (; t < total; t += gridDim.x) {
		const long long tn = t + gridDim.x;
		if (tn < total) issue(tiles + (cur ^ 1) * tsz, tn);
		cp_commit();
		cp_wait<1>();
		__syncthreads();

		T* buf0 = tiles + cur * tsz;
		const long long state = t % k;
		const int row0 = (int)(t / k) * rows;
		const int nrows = min(rows, a.sy - row0);
		const long long base = state * a.G + (long long)row0 * sx;
		const int toff = row0 * sx;
		const int cnt = nrows * sx;
		const R* m0 = a.do_inv ? mpre : mmid;
		if (m0) {
			for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
				const int r = i / sx;
				T& v = buf0[r * L + (i - r * sx)];
				v = cscale(v, m0[toff + i]);
			}
			__syncthreads();
		}
		T* cur_b = buf0;
		T* oth = scr;
		if (a.do_inv) {
			cur_b = line_transform<R, false>(buf0, scr, a.lp, tw, nrows, 1, L, true);
			oth = (cur_b == buf0) ? scr : buf0;
			if (mmid) {
				for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
					const int r = i / sx;
					const int x = i - r * sx;
					cur_b[r * L + x] = cscale(cur_b[r * L + x], mmid[toff + i]);
				}
				__syncthreads();
			}
		}
		if (a.do_fwd) cur_b = line_transform<R, false>(cur_b, oth, a.lp, tw, nrows, 1, L, false);

		T* out = reinterpret_cast<T*>(a.out) + base;
		const T* acc = reinterpret_cast<const T*>(a.acc);
		if (acc) acc += base;
		for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
			const int r = i / sx;
			const int x = i - r * sx;
			T v = cur_b[r * L + x];
			if (a.do_fwd && mpost) v = cscale(v, mpost[toff + i]);
			if (acc) v = cadd(v, acc[i]);
			out[i] = v;
		}
		__syncthreads();  // the tile buffers are reused by the copy issued next iteration
		cur ^= 1;
	}
	cp_wait<0>();
}

// Column pass, persistent and double-buffered like the row pass; tiles are
// cols_per_tile columns x sy rows of one state, in place.
template <class R>
__global__ void __launch_bounds__(kThreads) col_pass_kernel(ColPassArgs a, int k) {
	using T = c2<R>;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int L = a.lp.kind == 0 ? a.sy : 2 * a.sy;
	const int C = a.cols_per_tile;
	const int tsz = L * C;
	T* tiles = reinterpret_cast<T*>(smem_raw);
	T* scr = tiles + 2 * tsz;
	T* tw = scr + tsz;
	load_twiddles<R>(tw, a.lp);
	const int sx = a.sx, sy = a.sy;
	const int nct = (sx + C - 1) / C;
	const long long total = (long long)k * nct;
	const R* m2 = reinterpret_cast<const R*>(a.mul2d);
	const R* m1 = reinterpret_cast<const R*>(a.mul1d);

	long long t = blockIdx.x;
	int cur = 0;
	auto issue = [&](T* dst, long long tt) {
		const long long state = tt % k;
		const int col0 = (int)(tt / k) * C;
		const int ncols = min(C, sx - col0);
		const T* src = reinterpret_cast<const T*>(a.data) + state * a.G + col0;
		for (int i = threadIdx.x; i < sy * C; i += blockDim.x) {
			const int y = i / C;
			const int c = i - y * C;
			if (c < ncols) cp_elem<R>(dst + y * C + c, src + (long long)y * sx + c);
			else dst[y * C + c] = mk<R>(0, 0);
		}
	};
	if (t < total) issue(tiles, t);
	cp_commit();
	for (; t < total; t += gridDim.x) {
		const long long tn = t + gridDim.x;
		if (tn < total) issue(tiles + (cur ^ 1) * tsz, tn);
		cp_commit();
		cp_wait<1>();
		__syncthreads();

		T* cur_b = tiles + cur * tsz;
		T* oth = scr;
		const long long state = t % k;
		const int col0 = (int)(t / k) * C;
		const int ncols = min(C, sx - col0);
		if (a.mode == 0 || a.mode == 1) {
			T* r0 = line_transform<R, true>(cur_b, oth, a.lp, tw, C, C, 1, false);
			oth = (r0 == cur_b) ? oth : cur_b;
			cur_b = r0;
		}
		if (a.mode == 0) {
			for (int i = threadIdx.x; i < sy * C; i += blockDim.x) {
				const int y = i / C;
				const int c = i - y * C;
				if (c < ncols) {
					const R f = m2 ? m2[y * sx + col0 + c] : m1[y];
					cur_b[y * C + c] = cscale(cur_b[y * C + c], f);
				}
			}
			__syncthreads();
		}
		if (a.mode == 0 || a.mode == 2) cur_b = line_transform<R, true>(cur_b, oth, a.lp, tw, C, C, 1, true);

		T* data = reinterpret_cast<T*>(a.data) + state * a.G + col0;
		for (int i = threadIdx.x; i < sy * C; i += blockDim.x) {
			const int y = i / C;
			const int c = i - y * C;
			if (c < ncols) data[(long long)y * sx + c] = cur_b[y * C + c];
		}
		__syncthreads();
		cur ^= 1;
	}
	cp_wait<0>();
}

// Dirichlet magnetic row pass (DmRowArgs). One CTA per (state, tile of rows);
// four line buffers of 2 sx elements per row: P0/P1 carry the main (sine)
// branch and its FFT scratch, Q0/Q1 the shifted (cosine) branch.
template <class R>
__global__ void __launch_bounds__(kThreads) dm_row_kernel(DmRowArgs a) {
	using T = c2<R>;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int N = a.sx, L = 2 * N, rows = a.rows_per_tile, tsz = rows * L;
	T* P0 = reinterpret_cast<T*>(smem_raw);
	T* P1 = P0 + tsz;
	T* Q0 = P1 + tsz;
	T* Q1 = Q0 + tsz;
	T* tw = Q1 + tsz;
	load_twiddles<R>(tw, a.lp_dst);  // the 2 sx-point FFT of both line kinds
	const long long state = blockIdx.x;
	const int row0 = blockIdx.y * rows;
	const int nrows = min(rows, a.sy - row0);
	const long long base = state * a.G + (long long)row0 * N;
	const int toff = row0 * N;
	const int cnt = nrows * N;
	const T* in = reinterpret_cast<const T*>(a.in) + base;
	for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
		const int r = i / N;
		P0[r * L + (i - r * N)] = in[i];
	}
	__syncthreads();
	const R* x1 = reinterpret_cast<const R*>(a.x1);
	const R* x2 = reinterpret_cast<const R*>(a.x2);
	auto other = [&](T* b) { return b == P0 ? P1 : P0; };
	auto fwd = [&](T* b) { return line_transform<R, false>(b, other(b), a.lp_dst, tw, nrows, 1, L, false); };
	auto xop = [&](T* b) -> T* {
		for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
			const int r = i / N, x = i - r * N;
			T u = mk<R>(0, 0);
			if (x >= 1) {
				const T v = b[r * L + x - 1];
				const R w = x2[toff + i - 1];
				u = mk<R>(-w * v.y, w * v.x);  // i w v
			}
			Q0[r * L + x] = u;
		}
		__syncthreads();
		for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
			const int r = i / N, x = i - r * N;
			b[r * L + x] = cscale(b[r * L + x], x1[toff + i]);
		}
		__syncthreads();
		T* ra = line_transform<R, false>(b, other(b), a.lp_dst, tw, nrows, 1, L, true);
		T* rb = line_transform<R, false>(Q0, Q1, a.lp_dct, tw, nrows, 1, L, true);
		for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
			const int r = i / N, x = i - r * N;
			ra[r * L + x] = cadd(ra[r * L + x], rb[r * L + x]);
		}
		__syncthreads();
		return ra;
	};
	T* cur = P0;
	if (a.lead_fwd) cur = fwd(cur);
	if (a.do_inv) cur = xop(cur);
	const R* mid = reinterpret_cast<const R*>(a.mul_mid);
	if (mid) {
		for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
			const int r = i / N, x = i - r * N;
			cur[r * L + x] = cscale(cur[r * L + x], mid[toff + i]);
		}
		__syncthreads();
	}
	if (a.do_fwd) {
		cur = fwd(cur);
		cur = xop(cur);
		cur = fwd(cur);
	}
	T* out = reinterpret_cast<T*>(a.out) + base;
	const T* acc = a.acc ? reinterpret_cast<const T*>(a.acc) + base : nullptr;
	const R* vadd = reinterpret_cast<const R*>(a.vadd);
	for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
		const int r = i / N, x = i - r * N;
		T v = cur[r * L + x];
		if (vadd) {
			const T p = in[i];
			const R w = vadd[toff + i];
			v.x += w * p.x;
			v.y += w * p.y;
		}
		if (acc) v = cadd(v, acc[i]);
		out[i] = v;
	}
}

// Deterministic block reduction of NV doubles; result valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_reduce(double* v, double* red) {
	const int lane = threadIdx.x & 31;
	const int warp = threadIdx.x >> 5;
#pragma unroll
	for (int j = 0; j < NV; j++)
		for (int o = 16; o > 0; o >>= 1) v[j] += __shfl_xor_sync(0xffffffffu, v[j], o);
	if (lane == 0)
		for (int j = 0; j < NV; j++) red[warp * NV + j] = v[j];
	__syncthreads();
	if (threadIdx.x == 0) {
		const int nw = blockDim.x >> 5;
		for (int j = 0; j < NV; j++) {
			double s = 0.0;
			for (int w = 0; w < nw; w++) s += red[w * NV + j];
			v[j] = s;
		}
	}
}

template <class T>
__device__ __forceinline__ void accumulate_sums(double* s, T psi, T h, double es) {
	const double pr = psi.x, pi = psi.y, hr = h.x, hi = h.y;
	s[0] += pr * hr + pi * hi;  // Re conj(psi) h
	s[1] += pr * hi - pi * hr;  // Im conj(psi) h
	s[2] += hr * hr + hi * hi;
	const double dr = hr - es * pr, di = hi - es * pi;
	s[3] += dr * dr + di * di;
	s[4] += pr * pr + pi * pi;
}

template <class R>
__global__ void __launch_bounds__(kThreads) energy_row_kernel(EnergyRowArgs a) {
	using T = c2<R>;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int L = a.lp.kind == 0 ? a.sx : 2 * a.sx;
	const int rows = a.rows_per_tile;
	T* buf0 = reinterpret_cast<T*>(smem_raw);
	T* buf1 = buf0 + rows * L;
	T* tw = buf1 + rows * L;
	double* red = reinterpret_cast<double*>(tw + a.lp.fft.n);
	load_twiddles<R>(tw, a.lp);

	const long long state = blockIdx.x;
	const int row0 = blockIdx.y * rows;
	const int nrows = min(rows, a.sy - row0);
	const int sx = a.sx;
	const long long base = state * a.G + (long long)row0 * sx;
	const int toff = row0 * sx;
	const int cnt = nrows * sx;
	const T* src = reinterpret_cast<const T*>(a.src_t) + base;
	for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
		const int r = i / sx;
		buf0[r * L + (i - r * sx)] = src[i];
	}
	__syncthreads();
	T* cur = buf0;
	T* oth = buf1;
	if (a.do_fwd) {
		cur = line_transform<R, false>(cur, oth, a.lp, tw, nrows, 1, L, false);
		oth = (cur == buf0) ? buf1 : buf0;
		const R* tm = reinterpret_cast<const R*>(a.tmul);
		for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
			const int r = i / sx;
			const int x = i - r * sx;
			cur[r * L + x] = cscale(cur[r * L + x], tm[toff + i]);
		}
		__syncthreads();
	}
	cur = line_transform<R, false>(cur, oth, a.lp, tw, nrows, 1, L, true);

	const T* psi = reinterpret_cast<const T*>(a.psi) + base;
	const R* V = reinterpret_cast<const R*>(a.V);
	T* hout = a.h_out ? reinterpret_cast<T*>(a.h_out) + base : nullptr;
	const double es = a.Eshift ? a.Eshift[state] : 0.0;
	double s[5] = {0, 0, 0, 0, 0};
	for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
		const int r = i / sx;
		const int x = i - r * sx;
		T h = cur[r * L + x];
		const T p = psi[i];
		if (V) {
			const R v = V[toff + i];
			h.x += v * p.x;
			h.y += v * p.y;
		}
		if (hout) hout[i] = h;
		if (a.sums) accumulate_sums(s, p, h, es);
	}
	if (a.sums) {
		block_reduce<5>(s, red);
		if (threadIdx.x == 0) {
			double* o = a.sums + ((size_t)state * gridDim.y + blockIdx.y) * 5;
			for (int j = 0; j < 5; j++) o[j] = s[j];
		}
	}
}

template <class R>
__global__ void __launch_bounds__(kThreads) energy_col_kernel(EnergyColArgs a) {
	using T = c2<R>;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int L = a.lp.kind == 0 ? a.sy : 2 * a.sy;
	const int C = a.cols_per_tile;
	T* buf0 = reinterpret_cast<T*>(smem_raw);
	T* buf1 = buf0 + L * C;
	T* tw = buf1 + L * C;
	double* red = reinterpret_cast<double*>(tw + a.lp.fft.n);
	load_twiddles<R>(tw, a.lp);

	const long long state = blockIdx.x;
	const int col0 = blockIdx.y * C;
	const int ncols = min(C, a.sx - col0);
	const int sx = a.sx, sy = a.sy;
	const long long base = state * a.G + col0;
	const T* psi = reinterpret_cast<const T*>(a.psi) + base;
	const T* src = a.src ? reinterpret_cast<const T*>(a.src) + base : psi;
	for (int i = threadIdx.x; i < sy * C; i += blockDim.x) {
		const int y = i / C;
		const int c = i - y * C;
		buf0[y * C + c] = (c < ncols) ? src[(long long)y * sx + c] : mk<R>(0, 0);
	}
	__syncthreads();
	T* cur = line_transform<R, true>(buf0, buf1, a.lp, tw, C, C, 1, false);
	T* oth = (cur == buf0) ? buf1 : buf0;
	const R* ty = reinterpret_cast<const R*>(a.ty);
	for (int i = threadIdx.x; i < sy * C; i += blockDim.x) {
		const int y = i / C;
		cur[i] = cscale(cur[i], ty[y]);
	}
	__syncthreads();
	cur = line_transform<R, true>(cur, oth, a.lp, tw, C, C, 1, true);

	const T* add = reinterpret_cast<const T*>(a.add_in) + base;
	T* hout = a.h_out ? reinterpret_cast<T*>(a.h_out) + base : nullptr;
	const double es = a.Eshift ? a.Eshift[state] : 0.0;
	double s[5] = {0, 0, 0, 0, 0};
	for (int i = threadIdx.x; i < sy * C; i += blockDim.x) {
		const int y = i / C;
		const int c = i - y * C;
		if (c < ncols) {
			const long long off = (long long)y * sx + c;
			const T h = cadd(cur[i], add[off]);
			if (hout) hout[off] = h;
			if (a.sums) accumulate_sums(s, psi[off], h, es);
		}
	}
	if (a.sums) {
		block_reduce<5>(s, red);
		if (threadIdx.x == 0) {
			double* o = a.sums + ((size_t)state * gridDim.y + blockIdx.y) * 5;
			for (int j = 0; j < 5; j++) o[j] = s[j];
		}
	}
}

__global__ void energy_finish_kernel(const double* __restrict__ sums, const double* __restrict__ sums2, int k,
		int ntiles, double dx2, const double* __restrict__ Eshift, int normalize, double* E, double* sigma,
		double* sigma_res, double* E_imag) {
	const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (warp >= k) return;
	double s[5] = {0, 0, 0, 0, 0};
	for (int t = lane; t < ntiles; t += 32)
		for (int j = 0; j < 5; j++) s[j] += sums[((size_t)warp * ntiles + t) * 5 + j];
	double q[2] = {0, 0};
	if (sums2)
		for (int t = lane; t < ntiles; t += 32)
			for (int j = 0; j < 2; j++) q[j] += sums2[((size_t)warp * ntiles + t) * 5 + j];
	for (int j = 0; j < 5; j++)
		for (int o = 16; o > 0; o >>= 1) s[j] += __shfl_xor_sync(0xffffffffu, s[j], o);
	for (int j = 0; j < 2; j++)
		for (int o = 16; o > 0; o >>= 1) q[j] += __shfl_xor_sync(0xffffffffu, q[j], o);
	if (lane == 0) {
		// normalize: Rayleigh quotients <psi|H psi> / <psi|psi> (and <H^2> likewise)
		const double inv = normalize ? 1.0 / (s[4] * dx2) : 1.0;
		const double er = s[0] * dx2 * inv, ei = s[1] * dx2 * inv;
		// <H^2>: <psi|H H psi> from the second pass, else |H psi|^2 (H Hermitian)
		const double m2r = (sums2 ? q[0] : s[2]) * dx2 * inv;
		const double m2i = sums2 ? q[1] * dx2 * inv : 0.0;
		// sigma = Re sqrt(<H^2> - <H>^2) with complex <H> (operators.cpp:46-49)
		const double zr = m2r - (er * er - ei * ei);
		const double zi = m2i - 2.0 * er * ei;
		const double az = hypot(zr, zi);
		const double sg = sqrt(fmax(0.0, 0.5 * (az + zr)));
		const double es = Eshift ? Eshift[warp] : 0.0;
		const double de = er - es;
		const double res2 = normalize ? s[3] * dx2 * inv - de * de : s[3] * dx2 - de * de * (s[4] * dx2);
		E[warp] = er;
		sigma[warp] = sg;
		if (sigma_res) sigma_res[warp] = sqrt(fmax(0.0, res2));
		if (E_imag) E_imag[warp] = ei;
	}
}

// Opts a kernel into the full 227 KB of dynamic shared memory once per
// kernel (keyed by its address: float and double instantiations share a type).
template <class K>
void set_smem_limit(K kernel) {
	static std::mutex mu;
	static std::set<const void*> done;
	std::lock_guard<std::mutex> g(mu);
	if (done.insert((const void*)kernel).second)
		cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
}

}  // namespace

int row_tile_rows(int L, int elem_bytes, int sy) {
	int r = kTileBytes / (elem_bytes * L);
	r = std::max(1, std::min(r, 32));
	return std::min(r, sy);
}

int col_tile_cols(int L, int elem_bytes, int sx) {
	int c = kTileBytes / (elem_bytes * L);
	c = std::max(1, std::min(c, 16));
	return std::min(c, sx);
}

size_t row_pass_smem(int L, int rows, int n_fft, int elem_bytes) {
	return (size_t)(2 * rows * L + n_fft) * elem_bytes + 5 * sizeof(double) * (kThreads / 32);
}

size_t pipe_smem(int L, int lines, int n_fft, int elem_bytes) {
	return (size_t)(3 * lines * L + n_fft) * elem_bytes;
}

size_t col_pass_smem(int L, int cols, int n_fft, int elem_bytes) {
	return (size_t)(2 * cols * L + n_fft) * elem_bytes + 5 * sizeof(double) * (kThreads / 32);
}

// Persistent grid: as many CTAs as fit on the device, at most one per tile.
template <class K>
int persistent_blocks(K kernel, size_t smem, long long tiles) {
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

int dm_row_tile_rows(int sx, int elem_bytes, int sy) {
	const size_t row_bytes = (size_t)4 * 2 * sx * elem_bytes;
	const size_t room = 200 * 1024 - (size_t)2 * sx * elem_bytes;
	const int r = (int)std::max<size_t>(1, room / row_bytes);
	return std::min(std::min(r, 32), sy);
}

template <class R>
void launch_dm_row_pass(const DmRowArgs& a, int k, cudaStream_t s) {
	const size_t es = sizeof(c2<R>);
	const size_t sm = (size_t)4 * a.rows_per_tile * 2 * a.sx * es + (size_t)a.lp_dst.fft.n * es;
	set_smem_limit(dm_row_kernel<R>);
	const dim3 grid(k, (a.sy + a.rows_per_tile - 1) / a.rows_per_tile);
	dm_row_kernel<R><<<grid, kThreads, sm, s>>>(a);
}

template <class R>
void launch_row_pass(const RowPassArgs& a, int k, const void*, cudaStream_t s) {
	if (launch_row_pass_reg<R>(a, k, s)) return;
	const int L = a.lp.kind == 0 ? a.sx : 2 * a.sx;
	const size_t sm = pipe_smem(L, a.rows_per_tile, a.lp.fft.n, sizeof(c2<R>));
	set_smem_limit(row_pass_kernel<R>);
	const long long tiles = (long long)k * ((a.sy + a.rows_per_tile - 1) / a.rows_per_tile);
	row_pass_kernel<R><<<persistent_blocks(row_pass_kernel<R>, sm, tiles), kThreads, sm, s>>>(a, k);
}

template <class R>
void launch_col_pass(const ColPassArgs& a, int k, const void*, cudaStream_t s) {
	if (launch_col_pass_reg<R>(a, k, s)) return;
	const int L = a.lp.kind == 0 ? a.sy : 2 * a.sy;
	const size_t sm = pipe_smem(L, a.cols_per_tile, a.lp.fft.n, sizeof(c2<R>));
	set_smem_limit(col_pass_kernel<R>);
	const long long tiles = (long long)k * ((a.sx + a.cols_per_tile - 1) / a.cols_per_tile);
	col_pass_kernel<R><<<persistent_blocks(col_pass_kernel<R>, sm, tiles), kThreads, sm, s>>>(a, k);
}

template <class R>
void launch_energy_row(const EnergyRowArgs& a, int k, const void*, cudaStream_t s) {
	if (launch_energy_row_reg<R>(a, k, s)) return;
	const int L = a.lp.kind == 0 ? a.sx : 2 * a.sx;
	const dim3 grid(k, (a.sy + a.rows_per_tile - 1) / a.rows_per_tile);
	const size_t sm = row_pass_smem(L, a.rows_per_tile, a.lp.fft.n, sizeof(c2<R>));
	set_smem_limit(energy_row_kernel<R>);
	energy_row_kernel<R><<<grid, kThreads, sm, s>>>(a);
}

template <class R>
void launch_energy_col(const EnergyColArgs& a, int k, const void*, cudaStream_t s) {
	if (launch_energy_col_reg<R>(a, k, s)) return;
	const int L = a.lp.kind == 0 ? a.sy : 2 * a.sy;
	const dim3 grid(k, (a.sx + a.cols_per_tile - 1) / a.cols_per_tile);
	const size_t sm = col_pass_smem(L, a.cols_per_tile, a.lp.fft.n, sizeof(c2<R>));
	set_smem_limit(energy_col_kernel<R>);
	energy_col_kernel<R><<<grid, kThreads, sm, s>>>(a);
}

void launch_energy_finish(const double* sums, const double* sums2, int k, int ntiles, double dx2,
		const double* Eshift, int normalize, double* E, double* sigma, double* sigma_res, double* E_imag,
		cudaStream_t s) {
	const int threads = 128;
	const int blocks = (k * 32 + threads - 1) / threads;
	energy_finish_kernel<<<blocks, threads, 0, s>>>(sums, sums2, k, ntiles, dx2, Eshift, normalize, E, sigma,
			sigma_res, E_imag);
}

template void launch_dm_row_pass<double>(const DmRowArgs&, int, cudaStream_t);
template void launch_dm_row_pass<float>(const DmRowArgs&, int, cudaStream_t);
template void launch_row_pass<double>(const RowPassArgs&, int, const void*, cudaStream_t);
template void launch_row_pass<float>(const RowPassArgs&, int, const void*, cudaStream_t);
template void launch_col_pass<double>(const ColPassArgs&, int, const void*, cudaStream_t);
template void launch_col_pass<float>(const ColPassArgs&, int, const void*, cudaStream_t);
template void launch_energy_row<double>(const EnergyRowArgs&, int, const void*, cudaStream_t);
template void launch_energy_row<float>(const EnergyRowArgs&, int, const void*, cudaStream_t);
template void launch_energy_col<double>(const EnergyColArgs&, int, const void*, cudaStream_t);
template void launch_energy_col<float>(const EnergyColArgs&, int, const void*, cudaStream_t);

}  // namespace itp2d
