// Allocation-free Hermitian eigensolver entry point.
//
// Some callers of this library cannot create device memory: a host
// application whose memory manager has already taken the whole device for its
// own pool (a cudaMalloc then fails or fragments that pool), or a
// latency-sensitive loop where the device-wide synchronisation that
// cudaMalloc/cudaFree can imply would stall other streams. For them,
// itp2d_hermitian_eigensolve_noalloc does the same work as
// itp2d_hermitian_eigensolve but keeps every temporary in one fixed array of
// device memory that belongs to this library file, so a call allocates
// nothing, on the device or on the host.
//
// The array holds at most ITP2D_NOALLOC_MAX_N x ITP2D_NOALLOC_MAX_N matrices
// (about 1.6 MB in total) and stays resident on every GPU that loads the
// library until the process exits. Every call uses the same array, so calls
// that overlap on the GPU (from several host threads, or on several streams)
// race and must be serialised by the caller. Every call looks up the array's
// device address (cudaGetSymbolAddress) with the calling device current, so a
// device reset or a re-created primary context never leaves a stale address;
// the first call on a device also loads this library's device code there, so
// make that first call before any stream capture begins.
#include "../../include/itp2d_gpu.h"
#include "contract.cuh"

namespace {

using itp2d::EigStatus;
using itp2d::JacobiWork;

constexpr int kMaxN = ITP2D_NOALLOC_MAX_N;
constexpr int kMaxSweeps = 60;
constexpr size_t kAlign = 256;
constexpr size_t align_up(size_t b) { return (b + kAlign - 1) / kAlign * kAlign; }
constexpr size_t kMatBytes = align_up((size_t)kMaxN * kMaxN * sizeof(double2));
// input, S, A0, A1, V, eigenvector output, eigenvalues, permutation, counters, status
constexpr size_t kOffIn = 0;
constexpr size_t kOffS = kOffIn + kMatBytes;
constexpr size_t kOffA0 = kOffS + kMatBytes;
constexpr size_t kOffA1 = kOffA0 + kMatBytes;
constexpr size_t kOffV = kOffA1 + kMatBytes;
constexpr size_t kOffVec = kOffV + kMatBytes;
constexpr size_t kOffEval = kOffVec + kMatBytes;
constexpr size_t kOffPerm = kOffEval + align_up(kMaxN * sizeof(double));
constexpr size_t kOffCnt = kOffPerm + align_up(kMaxN * sizeof(int));
constexpr size_t kOffStat = kOffCnt + align_up(itp2d::jacobi_counter_ints(kMaxSweeps) * sizeof(int));
constexpr size_t kScratchBytes = kOffStat + align_up(sizeof(EigStatus));

// The scratch array. In host code its name is a host-side stand-in, not a
// device address: only the address returned by cudaGetSymbolAddress is passed
// to kernels.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of the scratch array on the current device, looked up on
// every call (no allocation once the module is loaded on the device).
int scratch_address(unsigned char** out) {
	void* p = nullptr;
	const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
	if (e != cudaSuccess || !p) return ITP2D_E_CUDA;
	*out = static_cast<unsigned char*>(p);
	return ITP2D_OK;
}

// Full Hermitian matrix (row-major) from the upper triangle of the
// column-major input, the part ZHEEV("U") reads.
__global__ void expand_upper_kernel(const double2* __restrict__ in, int n, double2* __restrict__ S) {
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= n * n) return;
	const int i = idx / n, j = idx % n;
	if (i > j) return;
	const double2 v = in[(size_t)j * n + i];
	if (i == j) {
		S[(size_t)i * n + i] = make_double2(v.x, 0.0);
	} else {
		S[(size_t)i * n + j] = v;
		S[(size_t)j * n + i] = make_double2(v.x, -v.y);
	}
}

// out[m*n + i] = element i of the m-th eigenvector (ascending eigenvalues).
__global__ void gather_vectors_kernel(const double2* __restrict__ V, int n, int kp, const int* __restrict__ perm,
		double2* __restrict__ out) {
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= n * n) return;
	const int m = idx / n, i = idx % n;
	out[idx] = V[(size_t)i * kp + perm[m]];
}

int status_of(cudaError_t e) { return e == cudaSuccess ? ITP2D_OK : ITP2D_E_CUDA; }

}  // namespace

extern "C" int itp2d_hermitian_eigensolve_noalloc(int n, const double* A, double* evals, double* evecs) {
	if (!A || !evals || !evecs || n < 1) return ITP2D_E_INVALID;
	if (n > kMaxN) return ITP2D_E_INVALID;  // beyond the fixed scratch
	int dev = 0, sms = 0;
	if (cudaGetDevice(&dev) != cudaSuccess) return ITP2D_E_CUDA;
	if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return ITP2D_E_CUDA;
	unsigned char* base = nullptr;
	int st = scratch_address(&base);
	if (st != ITP2D_OK) return st;
	itp2d::CoopUser user;
	double2* in = reinterpret_cast<double2*>(base + kOffIn);
	double2* S = reinterpret_cast<double2*>(base + kOffS);
	double2* vec = reinterpret_cast<double2*>(base + kOffVec);
	EigStatus* dstat = reinterpret_cast<EigStatus*>(base + kOffStat);
	JacobiWork w;
	w.A0 = reinterpret_cast<double2*>(base + kOffA0);
	w.A1 = reinterpret_cast<double2*>(base + kOffA1);
	w.V = reinterpret_cast<double2*>(base + kOffV);
	w.evals = reinterpret_cast<double*>(base + kOffEval);
	w.perm = reinterpret_cast<int*>(base + kOffPerm);
	w.counters = reinterpret_cast<int*>(base + kOffCnt);  // cleared by launch_eigh on every call
	w.max_sweeps = kMaxSweeps;
	const int kp = (n + 1) & ~1;
	const int nn = n * n;
	cudaError_t e = cudaMemcpy(in, A, (size_t)nn * sizeof(double2), cudaMemcpyHostToDevice);
	if (e != cudaSuccess) return status_of(e);
	expand_upper_kernel<<<(nn + 255) / 256, 256>>>(in, n, S);
	e = itp2d::launch_eigh(S, n, w, dstat, sms, 0, 0);
	if (e != cudaSuccess) return status_of(e);
	gather_vectors_kernel<<<(nn + 255) / 256, 256>>>(w.V, n, kp, w.perm, vec);
	e = cudaGetLastError();
	if (e == cudaSuccess) e = cudaMemcpy(evals, w.evals, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
	if (e == cudaSuccess) e = cudaMemcpy(evecs, vec, (size_t)nn * sizeof(double2), cudaMemcpyDeviceToHost);
	EigStatus hs;
	if (e == cudaSuccess) e = cudaMemcpy(&hs, dstat, sizeof(EigStatus), cudaMemcpyDeviceToHost);
	if (e != cudaSuccess) return status_of(e);
	return hs.status;
}
