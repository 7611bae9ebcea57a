// Device peak probe: throughput of FP64 DMMA (mma.sync m8n8k4 f64) from
// register operands, no memory traffic. The FP64 contractions of the
// orthonormalisation are measured against this number, since tcgen05 has no
// f64 kind and the driver-measured peaks cover HBM and BF16 only.
#include <cuda_runtime.h>

#include "../../include/itp2d_gpu.h"

namespace {

__global__ void dmma_peak_kernel(double* out, int iters) {
	double d[8][2];
	for (int i = 0; i < 8; i++) d[i][0] = d[i][1] = 0.0;
	const double a = 1.0 + threadIdx.x * 1e-9, b = 1.0 - threadIdx.x * 1e-9;
	for (int it = 0; it < iters; it++) {
#pragma unroll
		for (int i = 0; i < 8; i++)
			asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
					: "+d"(d[i][0]), "+d"(d[i][1])
					: "d"(a), "d"(b));
	}
	double s = 0.0;
	for (int i = 0; i < 8; i++) s += d[i][0] + d[i][1];
	out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // one store per thread, index < blocks * threads
}

// FP32 FFMA throughput: 16 independent dependency chains per thread.
__global__ void ffma_peak_kernel(float* out, int iters) {
	float x[16];
	const float a = 1.0f - threadIdx.x * 1e-7f, b = 1e-3f + threadIdx.x * 1e-9f;
#pragma unroll
	for (int i = 0; i < 16; i++) x[i] = 1.0f + i * 1e-3f;
	for (int it = 0; it < iters; it++) {
#pragma unroll
		for (int i = 0; i < 16; i++) x[i] = fmaf(x[i], a, b);
	}
	float s = 0.f;
#pragma unroll
	for (int i = 0; i < 16; i++) s += x[i];
	out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // one store per thread, index < blocks * threads
}

// Best of three timed launches (after one warm-up) of kern<<<blocks, threads>>>(out, iters), in ms.
template <class T>
int time_peak(void (*kern)(T*, int), int blocks, int threads, int iters, float* best_ms) {
	T* out = nullptr;
	if (cudaMalloc(&out, sizeof(T) * blocks * threads) != cudaSuccess) return ITP2D_E_OOM;
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	float best = 1e30f;
	for (int rep = 0; rep < 4; rep++) {
		cudaEventRecord(e0);
		kern<<<blocks, threads>>>(out, iters);
		cudaEventRecord(e1);
		cudaEventSynchronize(e1);
		float ms = 0.f;
		cudaEventElapsedTime(&ms, e0, e1);
		if (rep > 0 && ms < best) best = ms;
	}
	const cudaError_t err = cudaGetLastError();
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	cudaFree(out);
	if (err != cudaSuccess) return ITP2D_E_CUDA;
	*best_ms = best;
	return ITP2D_OK;
}

}  // namespace

extern "C" int itp2d_device_fp32_peak(double* tflops) {
	if (!tflops) return ITP2D_E_INVALID;
	int dev = 0, sms = 0;
	if (cudaGetDevice(&dev) != cudaSuccess) return ITP2D_E_CUDA;
	if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return ITP2D_E_CUDA;
	const int blocks = sms * 4, threads = 256, iters = 8192;
	float ms = 0.f;
	const int st = time_peak(ffma_peak_kernel, blocks, threads, iters, &ms);
	if (st != ITP2D_OK) return st;
	const double flops = 2.0 * 16 * (double)iters * blocks * threads;
	*tflops = flops / (ms * 1e-3) / 1e12;
	return ITP2D_OK;
}

extern "C" int itp2d_device_fp64_peak(double* tflops) {
	if (!tflops) return ITP2D_E_INVALID;
	int dev = 0, sms = 0;
	if (cudaGetDevice(&dev) != cudaSuccess) return ITP2D_E_CUDA;
	if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return ITP2D_E_CUDA;
	const int blocks = sms * 4, threads = 256, iters = 4096;
	double* out = nullptr;
	if (cudaMalloc(&out, sizeof(double) * blocks * threads) != cudaSuccess) return ITP2D_E_OOM;
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	float best = 1e30f;
	for (int rep = 0; rep < 4; rep++) {
		cudaEventRecord(e0);
		dmma_peak_kernel<<<blocks, threads>>>(out, iters);
		cudaEventRecord(e1);
		cudaEventSynchronize(e1);
		float ms = 0.f;
		cudaEventElapsedTime(&ms, e0, e1);
		if (rep > 0 && ms < best) best = ms;
	}
	const cudaError_t err = cudaGetLastError();
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	cudaFree(out);
	if (err != cudaSuccess) return ITP2D_E_CUDA;
	const double flops = 2.0 * 8 * 8 * 4 * 8.0 * iters * ((double)blocks * threads / 32);
	*tflops = flops / (best * 1e-3) / 1e12;
	return ITP2D_OK;
}
