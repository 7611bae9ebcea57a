// Gaussian impurity potentials built on the device (V and the impurity list in
// device memory; host pointers are rejected before any launch).
//
// V(x, y) += sum_j A_j exp(-r_j^2 / (2 w_j^2)), r_j the distance of the grid
// point from impurity j: GaussianImpurities::add_noise (noise.cpp:24-40)
// applied to a whole impurity list, in list order at every grid point as the
// reference's loop over impurities does. Grid positions are cell-centred,
// x_i = (2i + 1 - sx) dx / 2 (DataLayout, datalayout.cpp:21-35); V is stored
// [y][x] like the potential arrays of the path. The products and sums are
// rounded one at a time (no fused multiply-add), so the result differs from
// the reference's host loop only through exp().
#include <cuda_runtime.h>

#include "../../include/itp2d_gpu.h"

namespace {

constexpr int kThreads = 256;  // also the impurities staged in shared memory per pass

__global__ void __launch_bounds__(kThreads) gaussian_impurities_kernel(int sx, int sy, double dx, int n,
		const double* __restrict__ imp, double* __restrict__ V) {
	__shared__ double4 st[kThreads];  // (x, y, A, w)
	const long long G = (long long)sx * sy;
	const long long idx = (long long)blockIdx.x * kThreads + threadIdx.x;
	const bool in = idx < G;
	const int x = in ? (int)(idx % sx) : 0, y = in ? (int)(idx / sx) : 0;
	const double px = (2.0 * x + 1.0 - sx) * 0.5 * dx;
	const double py = (2.0 * y + 1.0 - sy) * 0.5 * dx;
	double v = in ? V[idx] : 0.0;
	for (int c0 = 0; c0 < n; c0 += kThreads) {
		const int m = min(kThreads, n - c0);
		__syncthreads();  // the previous chunk has been read
		if ((int)threadIdx.x < m) {
			const double* p = imp + 4LL * (c0 + threadIdx.x);
			st[threadIdx.x] = make_double4(p[0], p[1], p[2], p[3]);
		}
		__syncthreads();
		for (int j = 0; j < m; j++) {
			const double4 p = st[j];
			const double rx = __dsub_rn(p.x, px), ry = __dsub_rn(p.y, py);
			const double r2 = __dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry));
			const double w2 = __dmul_rn(p.w, p.w);
			v = __dadd_rn(v, __dmul_rn(p.z, exp(__dmul_rn(-0.5, __ddiv_rn(r2, w2)))));
		}
	}
	if (in) V[idx] = v;
}

// True when p is device (or managed) memory the kernel can dereference.
bool device_pointer(const void* p) {
	cudaPointerAttributes a;
	if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
		cudaGetLastError();  // clear the error an unknown pointer leaves behind
		return false;
	}
	return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" int itp2d_add_gaussian_impurities(int sx, int sy, double dx, int n, const double* impurities, double* V,
		void* cuda_stream) {
	if (sx < 1 || sy < 1 || !(dx > 0.0) || n < 0 || !V || (n > 0 && !impurities)) return ITP2D_E_INVALID;
	if (n == 0) return ITP2D_OK;
	if (!device_pointer(V) || !device_pointer(impurities)) return ITP2D_E_INVALID;
	const long long G = (long long)sx * sy;
	const unsigned blocks = (unsigned)((G + kThreads - 1) / kThreads);
	gaussian_impurities_kernel<<<blocks, kThreads, 0, (cudaStream_t)cuda_stream>>>(sx, sy, dx, n, impurities, V);
	return cudaGetLastError() == cudaSuccess ? ITP2D_OK : ITP2D_E_CUDA;
}
