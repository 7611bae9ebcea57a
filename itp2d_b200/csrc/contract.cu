// Dense contractions of the orthonormalisation on FP64 tensor cores.
//
//   overlap:  S_ij = dx^2 sum_g conj(psi_i[g]) psi_j[g]     (stateset.cpp:146-154)
//   rotation: out_n[g] = sum_i W[i][n] psi_i[g]             (stateset.cpp:214-228)
//
// tcgen05 has no f64 kind, so the FP64 path issues DMMA (mma.sync m8n8k4 f64)
// from register fragments staged through shared memory. A complex product is
// four real MMAs. The overlap computes only upper-triangle 64x64 tiles and
// splits the long g dimension across CTAs; a second kernel sums the splits in
// a fixed order and fills the Hermitian matrix from the upper triangle, as
// ZHEEV("U") reads it (eigensolver.hpp:44-53).
#include "contract.cuh"

#include <algorithm>

namespace itp2d {

namespace {

constexpr int kBM = 64;   // tile rows
constexpr int kBN = 64;   // tile cols
constexpr int kBK = 16;   // k step
constexpr int kPad = 20;  // padded row length (doubles) of a staged plane: conflict-free fragments

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
	asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
			: "+d"(d0), "+d"(d1)
			: "d"(a), "d"(b));
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

// Overlap: A rows i (conjugated side) and B rows j, both rows of psi (k x G).
// The g range of the split advances kBK per step through two shared-memory
// stages of complex-interleaved rows (pitch kPad elements: conflict-free
// fragment loads): cp.async fetches step s + 1 while the DMMAs of step s run.
template <class T>
__global__ void __launch_bounds__(256) overlap_kernel(const T* __restrict__ psi, const T* __restrict__ psib, int k,
		long long G, const int2* __restrict__ pairs, long long chunk, double2* __restrict__ part) {
	extern __shared__ __align__(16) unsigned char smem_raw[];
	T* stage = reinterpret_cast<T*>(smem_raw);  // [2][A rows kBM | B rows kBN][kPad]
	constexpr int SS = (kBM + kBN) * kPad;
	const int2 tp = pairs[blockIdx.x];
	const int i0 = tp.x * kBM, j0 = tp.y * kBN;
	const long long g0 = (long long)blockIdx.y * chunk;
	const long long g1 = min(G, g0 + chunk);
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int wi = warp >> 2;  // 0..1 : 32 rows each
	const int wj = warp & 3;   // 0..3 : 16 cols each
	double accr[4][2][2], acci[4][2][2];
#pragma unroll
	for (int a = 0; a < 4; a++)
#pragma unroll
		for (int b = 0; b < 2; b++) {
			accr[a][b][0] = accr[a][b][1] = 0.0;
			acci[a][b][0] = acci[a][b][1] = 0.0;
		}
	// loader mapping: row = tid / 4, 4 consecutive complex at seg*4, for A and B
	const int lrow = tid >> 2, lseg = (tid & 3) * 4;
	auto fetch = [&](T* st, long long g) {
		const int ia = i0 + lrow, jb = j0 + lrow;
#pragma unroll
		for (int q = 0; q < 4; q++) {
			const long long gg = g + lseg + q;
			T* da = st + lrow * kPad + lseg + q;
			T* db = st + (kBM + lrow) * kPad + lseg + q;
			if (gg < g1 && ia < k) cp_async_elem<T>(da, psi + (long long)ia * G + gg);
			else *da = T{0, 0};
			if (gg < g1 && jb < k) cp_async_elem<T>(db, psib + (long long)jb * G + gg);
			else *db = T{0, 0};
		}
	};
	int cur = 0;
	if (g0 < g1) fetch(stage, g0);
	cp_async_commit();
	for (long long g = g0; g < g1; g += kBK) {
		if (g + kBK < g1) fetch(stage + (cur ^ 1) * SS, g + kBK);
		cp_async_commit();
		cp_async_wait<1>();
		__syncthreads();
		const T* sa = stage + cur * SS;
		const T* sb = sa + kBM * kPad;
#pragma unroll
		for (int kk = 0; kk < kBK; kk += 4) {
			double far[4], fai[4], fbr[2], fbi[2];
#pragma unroll
			for (int a = 0; a < 4; a++) {
				const T v = sa[(wi * 32 + a * 8 + (lane >> 2)) * kPad + kk + (lane & 3)];
				far[a] = v.x;
				fai[a] = v.y;
			}
#pragma unroll
			for (int b = 0; b < 2; b++) {
				const T v = sb[(wj * 16 + b * 8 + (lane >> 2)) * kPad + kk + (lane & 3)];
				fbr[b] = v.x;
				fbi[b] = v.y;
			}
#pragma unroll
			for (int a = 0; a < 4; a++)
#pragma unroll
				for (int b = 0; b < 2; b++) {
					// conj(a) b = (ar br + ai bi) + i (ar bi - ai br)
					dmma(accr[a][b][0], accr[a][b][1], far[a], fbr[b]);
					dmma(accr[a][b][0], accr[a][b][1], fai[a], fbi[b]);
					dmma(acci[a][b][0], acci[a][b][1], far[a], fbi[b]);
					dmma(acci[a][b][0], acci[a][b][1], -fai[a], fbr[b]);
				}
		}
		__syncthreads();  // this stage is refilled by the fetch of the next step
		cur ^= 1;
	}
	cp_async_wait<0>();
	// write the partial tile: part[split][i][j]
	double2* out = part + (size_t)blockIdx.y * k * k;
#pragma unroll
	for (int a = 0; a < 4; a++)
#pragma unroll
		for (int b = 0; b < 2; b++) {
			const int i = i0 + wi * 32 + a * 8 + (lane >> 2);
			const int j = j0 + wj * 16 + b * 8 + 2 * (lane & 3);
			if (i < k) {
				if (j < k) out[(size_t)i * k + j] = make_double2(accr[a][b][0], acci[a][b][0]);
				if (j + 1 < k) out[(size_t)i * k + j + 1] = make_double2(accr[a][b][1], acci[a][b][1]);
			}
		}
}

// Sum the splits (fixed order), scale, and build the Hermitian matrix from the
// upper triangle. One thread per (i, j) with i <= j of the full matrix.
__global__ void overlap_finish_kernel(const double2* __restrict__ part, int k, int nsplit, double dx2,
		double2* __restrict__ S) {
	const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= (long long)k * k) return;
	const int i = (int)(idx / k), j = (int)(idx % k);
	if (i > j) return;
	double sr = 0.0, si = 0.0;
	for (int s = 0; s < nsplit; s++) {
		const double2 v = part[(size_t)s * k * k + idx];
		sr += v.x;
		si += v.y;
	}
	sr *= dx2;
	si *= dx2;
	if (i == j) {
		S[idx] = make_double2(sr, 0.0);
	} else {
		S[idx] = make_double2(sr, si);
		S[(size_t)j * k + i] = make_double2(sr, -si);
	}
}

// Rotation: out[n][g] = sum_i W[i][n] psi[i][g]; tile 64 n x 64 g. The i range
// advances kBK per step through two shared-memory stages holding the W rows
// [i][n] and the psi rows [i][g] as in global memory (cp.async fetches step
// s + 1 while the DMMAs of step s run); row pitches of 66 (16-byte elements)
// and 68 (8-byte elements) make the transposed fragment reads conflict-free.
template <class T>
__global__ void __launch_bounds__(256) rotate_kernel(const double2* __restrict__ W, const T* __restrict__ psi,
		int k, long long G, T* __restrict__ out, int upper) {
	constexpr int PW = 66, PP = sizeof(T) == 16 ? 66 : 68;
	constexpr int SW = kBK * PW * (int)sizeof(double2), SP = kBK * PP * (int)sizeof(T);
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int n0 = blockIdx.x * kBM;
	const long long g0 = (long long)blockIdx.y * kBN;
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int wn = warp >> 2, wg = warp & 3;
	double accr[4][2][2], acci[4][2][2];
#pragma unroll
	for (int a = 0; a < 4; a++)
#pragma unroll
		for (int b = 0; b < 2; b++) {
			accr[a][b][0] = accr[a][b][1] = 0.0;
			acci[a][b][0] = acci[a][b][1] = 0.0;
		}
	auto sw = [&](int buf) { return reinterpret_cast<double2*>(smem_raw + buf * (SW + SP)); };
	auto sp = [&](int buf) { return reinterpret_cast<T*>(smem_raw + buf * (SW + SP) + SW); };
	// W tile 16 i x 64 n and psi tile 16 i x 64 g: 4 elements each per thread
	auto fetch = [&](int buf, int i0) {
		double2* dw = sw(buf);
		T* dp = sp(buf);
#pragma unroll
		for (int q = 0; q < 4; q++) {
			const int e = tid + q * 256;
			const int ii = e >> 6, cc = e & 63;
			const int i = i0 + ii, n = n0 + cc;
			const long long g = g0 + cc;
			if (i < k && n < k) cp_async_elem<double2>(dw + ii * PW + cc, W + (size_t)i * k + n);
			else dw[ii * PW + cc] = make_double2(0, 0);
			if (i < k && g < G) cp_async_elem<T>(dp + ii * PP + cc, psi + (long long)i * G + g);
			else dp[ii * PP + cc] = T{0, 0};
		}
	};
	// upper-triangular W (Cholesky): rows i > n are zero, so the i range ends
	// with this tile's last output state
	const int kend = upper ? min(k, n0 + kBM) : k;
	int cur = 0;
	fetch(0, 0);
	cp_async_commit();
	for (int i0 = 0; i0 < kend; i0 += kBK) {
		if (i0 + kBK < kend) fetch(cur ^ 1, i0 + kBK);
		cp_async_commit();
		cp_async_wait<1>();
		__syncthreads();
		const double2* a_s = sw(cur);
		const T* b_s = sp(cur);
#pragma unroll
		for (int kk = 0; kk < kBK; kk += 4) {
			double far[4], fai[4], fbr[2], fbi[2];
			const int ii = kk + (lane & 3);
#pragma unroll
			for (int a = 0; a < 4; a++) {
				const double2 v = a_s[ii * PW + wn * 32 + a * 8 + (lane >> 2)];
				far[a] = v.x;
				fai[a] = v.y;
			}
#pragma unroll
			for (int b = 0; b < 2; b++) {
				const T v = b_s[ii * PP + wg * 16 + b * 8 + (lane >> 2)];
				fbr[b] = v.x;
				fbi[b] = v.y;
			}
#pragma unroll
			for (int a = 0; a < 4; a++)
#pragma unroll
				for (int b = 0; b < 2; b++) {
					// (ar + i ai)(br + i bi)
					dmma(accr[a][b][0], accr[a][b][1], far[a], fbr[b]);
					dmma(accr[a][b][0], accr[a][b][1], -fai[a], fbi[b]);
					dmma(acci[a][b][0], acci[a][b][1], far[a], fbi[b]);
					dmma(acci[a][b][0], acci[a][b][1], fai[a], fbr[b]);
				}
		}
		__syncthreads();  // this stage is refilled by the fetch of the next step
		cur ^= 1;
	}
	cp_async_wait<0>();
#pragma unroll
	for (int a = 0; a < 4; a++)
#pragma unroll
		for (int b = 0; b < 2; b++) {
			const int n = n0 + wn * 32 + a * 8 + (lane >> 2);
			const long long g = g0 + wg * 16 + b * 8 + 2 * (lane & 3);
			if (n < k) {
				T o;
				if (g < G) { o.x = accr[a][b][0]; o.y = acci[a][b][0]; out[(long long)n * G + g] = o; }
				if (g + 1 < G) { o.x = accr[a][b][1]; o.y = acci[a][b][1]; out[(long long)n * G + g + 1] = o; }
			}
		}
}

// Norm of a single state (the N = 1 branch of stateset.cpp:138-144).
template <class T>
__global__ void norm1_kernel(const T* __restrict__ psi, long long G, double dx, double* out) {
	__shared__ double red[32];
	double s = 0.0;
	for (long long g = threadIdx.x; g < G; g += blockDim.x) {
		const T v = psi[g];
		s += (double)v.x * v.x + (double)v.y * v.y;
	}
	for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
	if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
	__syncthreads();
	if (threadIdx.x == 0) {
		double t = 0.0;
		for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
		*out = sqrt(t) * dx;
	}
}

template <class T>
__global__ void scale1_kernel(T* psi, long long G, const double* nrm) {
	const double f = 1.0 / *nrm;
	for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < G; g += (long long)gridDim.x * blockDim.x) {
		T v = psi[g];
		v.x = v.x * f;
		v.y = v.y * f;
		psi[g] = v;
	}
}

template <class TI, class TO>
__global__ void convert_kernel(const TI* __restrict__ in, TO* __restrict__ out, long long n) {
	for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
		const TI v = in[i];
		TO o;
		o.x = v.x;
		o.y = v.y;
		out[i] = o;
	}
}

}  // namespace

int overlap_tiles(int k) { return (k + kBM - 1) / kBM; }

int overlap_splits(int k, long long G, int num_sms) {
	const int nt = overlap_tiles(k);
	const long long npairs = (long long)nt * (nt + 1) / 2;
	// two CTAs per SM (80 KB of stages each for FP64 states); splits of at
	// least 512 grid points, up to enough for two waves (at least 16); the
	// first count whose grid fills its last wave to 95 % or more, else the
	// best-filled one (k = 2000: 528 tile pairs fill 1.78 waves unsplit, 5
	// splits fill 8.92 waves; a few tile pairs take as many splits as fill
	// the GPU)
	const long long slots = 2LL * num_sms;
	const long long most = std::max(1LL, std::min(G / 512, std::max(16LL, 2 * slots / npairs)));
	long long best = 1;
	double best_fill = 0.0;
	for (long long ns = 1; ns <= most; ns++) {
		const long long ctas = npairs * ns;
		const long long waves = (ctas + slots - 1) / slots;
		const double fill = (double)ctas / (double)(waves * slots);
		if (fill > best_fill + 1e-9) {
			best = ns;
			best_fill = fill;
		}
		if (fill >= 0.95) break;
	}
	return (int)best;
}

template <class T>
void launch_overlap(const T* psi, int k, long long G, const int2* pairs, int npairs, int nsplit,
		double2* part, double dx2, double2* S, cudaStream_t s, const T* psib) {
	long long chunk = (G + nsplit - 1) / nsplit;
	chunk = ((chunk + kBK - 1) / kBK) * kBK;
	const int used = (int)((G + chunk - 1) / chunk);
	const size_t sm = (size_t)2 * (kBM + kBN) * kPad * sizeof(T);
	cudaFuncSetAttribute(overlap_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
	overlap_kernel<T><<<dim3(npairs, used), 256, sm, s>>>(psi, psib ? psib : psi, k, G, pairs, chunk, part);
	launch_overlap_finish(part, k, used, dx2, S, s);
}

void launch_overlap_finish(const double2* part, int k, int nsplit, double dx2, double2* S, cudaStream_t s) {
	const long long kk = (long long)k * k;
	overlap_finish_kernel<<<(unsigned)((kk + 255) / 256), 256, 0, s>>>(part, k, nsplit, dx2, S);
}

template <class T>
void launch_rotate(const double2* W, const T* psi, int k, long long G, T* out, cudaStream_t s, bool upper) {
	const dim3 grid((k + kBM - 1) / kBM, (unsigned)((G + kBN - 1) / kBN));
	const size_t sm = (size_t)2 * kBK * (66 * sizeof(double2) + (sizeof(T) == 16 ? 66 : 68) * sizeof(T));
	cudaFuncSetAttribute(rotate_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
	rotate_kernel<T><<<grid, 256, sm, s>>>(W, psi, k, G, out, upper ? 1 : 0);
}

template <class T>
void launch_normalize1(T* psi, long long G, double dx, double* tmp, cudaStream_t s) {
	norm1_kernel<T><<<1, 1024, 0, s>>>(psi, G, dx, tmp);
	scale1_kernel<T><<<148, 256, 0, s>>>(psi, G, tmp);
}

void launch_convert(const void* in, int in_fp64, void* out, long long n, cudaStream_t s) {
	const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 148 * 16);
	if (in_fp64)
		convert_kernel<double2, float2><<<blocks, 256, 0, s>>>((const double2*)in, (float2*)out, n);
	else
		convert_kernel<float2, double2><<<blocks, 256, 0, s>>>((const float2*)in, (double2*)out, n);
}

template void launch_overlap<double2>(const double2*, int, long long, const int2*, int, int, double2*, double,
		double2*, cudaStream_t, const double2*);
template void launch_overlap<float2>(const float2*, int, long long, const int2*, int, int, double2*, double,
		double2*, cudaStream_t, const float2*);
template void launch_rotate<double2>(const double2*, const double2*, int, long long, double2*, cudaStream_t, bool);
template void launch_rotate<float2>(const double2*, const float2*, int, long long, float2*, cudaStream_t, bool);
template void launch_normalize1<double2>(double2*, long long, double, double*, cudaStream_t);
template void launch_normalize1<float2>(float2*, long long, double, double*, cudaStream_t);

}  // namespace itp2d
