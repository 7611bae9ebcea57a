// Second-order Löwdin orthonormalisation for the FP32 form.
//
// With S the overlap of the states, D = diag(S)^{-1/2} and the
// diagonal-normalised overlap D S D = I + E (E Hermitian, zero diagonal),
// W = D (I + E)^{-1/2} makes the states orthonormal: W^H S W = I. The series
// (I + E)^{-1/2} = I - E/2 + 3/8 E^2 - 5/16 E^3 + ... is cut after E^2, so
// the result is orthonormal up to 5/16 |E|^3. After the first iterations of
// an imaginary-time solve the states entering an orthonormalisation are the
// previous iteration's orthonormal states propagated by one step, E is small,
// and this replaces the k x k eigendecomposition of the canonical form by one
// k x k product. No reference counterpart: the reference always orthonormalises
// canonically (stateset.cpp:136-232); the FP32 form alternates the two and
// keeps the canonical one for every FP64 iteration.
#include "../../include/itp2d_gpu.h"
#include "contract.cuh"

namespace itp2d {

namespace {

// D_i = S_ii^{-1/2}; E (row-major, stride k) and its complex conjugate;
// stats[0] = max |E_ij|, stats[1] = sum |E_ij|^2, stats[2] = 1 if a diagonal
// element is not a positive normal number.
__global__ void lowdin_prep_kernel(const double2* __restrict__ S, int k, double* __restrict__ D,
		double2* __restrict__ E, double2* __restrict__ Ec, double* stats) {
	__shared__ double smax[32], ssum[32];
	const long long n2 = (long long)k * k;
	double mx = 0.0, sq = 0.0;
	int bad = 0;
	for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n2;
			idx += (long long)gridDim.x * blockDim.x) {
		const int i = (int)(idx / k), j = (int)(idx % k);
		const double si = S[(long long)i * k + i].x, sj = S[(long long)j * k + j].x;
		if (!(si > 0.0) || !(sj > 0.0) || !isfinite(si) || !isfinite(sj)) {
			bad = 1;
			continue;
		}
		const double di = rsqrt(si), dj = rsqrt(sj);
		if (j == i) D[i] = di;
		double2 e = make_double2(0.0, 0.0);
		if (i != j) {
			const double2 s = S[idx];
			e = make_double2(s.x * di * dj, s.y * di * dj);
		}
		E[idx] = e;
		Ec[idx] = make_double2(e.x, -e.y);
		const double a2 = e.x * e.x + e.y * e.y;
		if (!isfinite(a2)) bad = 1;
		mx = fmax(mx, a2);
		sq += a2;
	}
	for (int o = 16; o > 0; o >>= 1) {
		mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
		sq += __shfl_xor_sync(0xffffffffu, sq, o);
		bad |= __shfl_xor_sync(0xffffffffu, bad, o);
	}
	const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
	if (lane == 0) {
		smax[w] = mx;
		ssum[w] = sq;
	}
	if (bad && lane == 0) stats[2] = 1.0;
	__syncthreads();
	if (threadIdx.x == 0) {
		double m = 0.0, t = 0.0;
		for (int q = 0; q < (int)(blockDim.x >> 5); q++) {
			m = fmax(m, smax[q]);
			t += ssum[q];
		}
		// non-negative doubles order like their bit patterns
		atomicMax(reinterpret_cast<unsigned long long*>(stats), (unsigned long long)__double_as_longlong(sqrt(m)));
		atomicAdd(stats + 1, t);
	}
}

// W[i * k + n] (coefficient of state i in output state n, the layout of the
// rotation kernels) = D_i (delta_in - E_in / 2 + 3/8 (E^2)_in), with E and E^2
// row-major (E[i * k + n] = E_in).
__global__ void lowdin_w_kernel(const double* __restrict__ D, const double2* __restrict__ E,
		const double2* __restrict__ E2, int k, double2* __restrict__ W) {
	const long long n2 = (long long)k * k;
	for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n2;
			idx += (long long)gridDim.x * blockDim.x) {
		const int i = (int)(idx / k), n = (int)(idx % k);
		const double2 e = E[idx];
		const double2 q = E2[idx];
		double re = -0.5 * e.x + 0.375 * q.x;
		double im = -0.5 * e.y + 0.375 * q.y;
		if (i == n) re += 1.0;
		const double d = D[i];
		W[idx] = make_double2(d * re, d * im);
	}
}

}  // namespace

void launch_lowdin_prep(const double2* S, int k, double* D, double2* E, double2* Ec, double* stats,
		cudaStream_t s) {
	const long long n2 = (long long)k * k;
	cudaMemsetAsync(stats, 0, 3 * sizeof(double), s);
	lowdin_prep_kernel<<<(unsigned)std::min<long long>((n2 + 255) / 256, 2048), 256, 0, s>>>(S, k, D, E, Ec, stats);
}

// W from D, E and E^2. The rotation kernel computes
// out[n][g] = sum_i Wr[i * k + n] P[i][g]; with Wr = conj(E) and P = E that is
// sum_i conj(E_in) E_ig = sum_i E_ni E_ig = (E^2)_ng, row-major.
void launch_lowdin_w(const double* D, const double2* E, const double2* Ec, double2* E2, int k, double2* W,
		cudaStream_t s) {
	launch_rotate<double2>(Ec, E, k, k, E2, s);
	const long long n2 = (long long)k * k;
	lowdin_w_kernel<<<(unsigned)std::min<long long>((n2 + 255) / 256, 4096), 256, 0, s>>>(D, E, E2, k, W);
}

}  // namespace itp2d
