// Common device/host helpers for the itp2d B200 kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace itp2d {

template <class R> struct V2;
template <> struct V2<double> { using T = double2; };
template <> struct V2<float> { using T = float2; };

template <class R> using c2 = typename V2<R>::T;

template <class R>
__host__ __device__ __forceinline__ c2<R> mk(R a, R b) {
	c2<R> r;
	r.x = a;
	r.y = b;
	return r;
}

template <class T> __host__ __device__ __forceinline__ T cadd(T a, T b) { T r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <class T> __host__ __device__ __forceinline__ T csub(T a, T b) { T r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <class T> __host__ __device__ __forceinline__ T cmul(T a, T b) {
	T r;
	r.x = a.x * b.x - a.y * b.y;
	r.y = a.x * b.y + a.y * b.x;
	return r;
}
// a * conj(b)
template <class T> __host__ __device__ __forceinline__ T cmulc(T a, T b) {
	T r;
	r.x = a.x * b.x + a.y * b.y;
	r.y = a.y * b.x - a.x * b.y;
	return r;
}
template <class T, class R> __host__ __device__ __forceinline__ T cscale(T a, R s) { T r; r.x = a.x * s; r.y = a.y * s; return r; }
// multiply by -i (sign < 0) or +i (sign > 0)
template <class T> __host__ __device__ __forceinline__ T cmul_i(T a, int sign) {
	T r;
	if (sign < 0) { r.x = a.y; r.y = -a.x; } else { r.x = -a.y; r.y = a.x; }
	return r;
}

// Plan of one complex FFT length: radix stages and twiddle table
// exp(-2 pi i t / n), t in [0, n), in the working precision.
constexpr int kMaxStages = 16;
struct FftPlan {
	int n;
	int nstages;
	int radix[kMaxStages];
	const void* tw;
};

// Plan of one line transform of N grid points.
//   kind 0: DFT of length N.
//   kind 1: DST-II forward / DST-III inverse through a 2N-point complex FFT.
//   kind 2: DCT-II forward / DCT-III inverse through a 2N-point complex FFT.
// ext: exp(-i pi m / (2N)), m in [0, 2N], for kinds 1 and 2.
struct LinePlan {
	int N;
	int kind;
	FftPlan fft;
	const void* ext;
};

}  // namespace itp2d
