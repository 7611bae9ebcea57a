// Batched Hermitian eigensolver: the k x k overlap eigenproblems of many
// independent state sets (each the ZHEEV call of StateSet::orthonormalize,
// stateset.cpp:156-176) in one persistent launch, one CTA per instance at a
// time (a work queue hands out the instances). Instances of
// different k share the launch; no CTA waits for another, so the launch can
// share the GPU with any other work (unlike the cooperative solvers of
// jacobi.cu / bjacobi.cu, which serve one large matrix at a time).
//
// Method: cyclic Jacobi with the round-robin parallel ordering. In a round
// the k_p / 2 disjoint index pairs (p, q) are rotated together: thread j sets
// up the 2 x 2 unitary Q_j = [[c, s u], [-s conj(u), c]] (u = A_pq / |A_pq|,
// t = s / c the smaller root of the real 2 x 2 problem) that zeroes A_pq,
// then A <- Q^H A Q is applied as a row pass and a column pass over the CTA,
// and V <- V Q. A and V live in global memory (the instance's own work
// matrices, L2-resident at these sizes). A sweep is k_p - 1 rounds; the solve
// stops after the first sweep whose largest rotation tangent is below tau.
// The epilogue sorts the eigenvalues ascending, applies the checks of
// stateset.cpp:158-172 (first non-positive or non-normal eigenvalue) and
// writes W = U Lambda^{-1/2} in the rotation kernels' layout
// (W[i * k + n]: coefficient of state i in output state n).
#include "../../include/itp2d_gpu.h"
#include "contract.cuh"

#include <algorithm>

namespace itp2d {

namespace {

constexpr int kBThreads = 512;
constexpr int kMaxPairs = 2048;  // k_p / 2 for k up to 4096
// A pair is not rotated when |A_pq| <= kSkipBelow sqrt(|A_pp A_qq|): such an
// element is at the rounding level of the diagonal. A lower threshold never
// ends for (numerically) degenerate diagonal pairs, whose rotation is a
// 45-degree one that leaves an off-diagonal element of the same rounding size.
constexpr double kSkipBelow = 1e-15;

__device__ __forceinline__ int rr_player(int pos, int r, int npos) {
	return pos == 0 ? 0 : ((pos - 1 + r) % (npos - 1)) + 1;
}

struct Rot {
	double c, s, ur, ui;  // Q = [[c, s u], [-s conj(u), c]]
	int p, q;             // p < q; p < 0: no rotation
};

// One instance, by the whole CTA.
__device__ void solve_item(const BatchEigItem& it, int max_sweeps, int smem_bytes) {
	__shared__ Rot rot[kMaxPairs / 4];  // pairs handled per chunk (see below)
	__shared__ double red[kBThreads / 32];
	__shared__ int s_bad, s_sweeps;
	extern __shared__ __align__(16) double2 work[];
	const int k = it.k;
	const int kp = (k + 1) & ~1;
	const int np = kp / 2;
	const int tid = threadIdx.x;
	// A (and V) in shared memory when they fit in this launch's dynamic
	// shared memory, else the instance's work matrices in global memory
	const size_t mat = (size_t)kp * kp * sizeof(double2);
	double2* A = mat <= (size_t)smem_bytes ? work : it.A;
	double2* V = 2 * mat <= (size_t)smem_bytes ? work + (size_t)kp * kp : it.V;
	// A = S (row-major, stride kp), V = I
	for (int idx = tid; idx < kp * kp; idx += blockDim.x) {
		const int i = idx / kp, j = idx % kp;
		A[idx] = (i < k && j < k) ? it.S[(size_t)i * k + j] : make_double2(0.0, 0.0);
		V[idx] = make_double2(i == j ? 1.0 : 0.0, 0.0);
	}
	if (tid == 0) s_sweeps = -1;
	__syncthreads();
	// pairs are processed in chunks of kMaxPairs / 4 (the rotation table in
	// shared memory); for k <= 1024 one chunk holds a whole round
	constexpr int kChunk = kMaxPairs / 4;
	for (int sweep = 0; sweep < max_sweeps; sweep++) {
		double tmax = 0.0;
		for (int r = 0; r < kp - 1; r++) {
			for (int j0 = 0; j0 < np; j0 += kChunk) {
				const int nj = min(kChunk, np - j0);
				for (int jj = tid; jj < nj; jj += blockDim.x) {
					const int j = j0 + jj;
					int p = rr_player(j, r, kp), q = rr_player(kp - 1 - j, r, kp);
					if (p > q) {
						const int x = p;
						p = q;
						q = x;
					}
					Rot R;
					R.p = -1;
					R.q = q;
					if (q < k) {
						const double a = A[(size_t)p * kp + p].x, b = A[(size_t)q * kp + q].x;
						const double2 cpq = A[(size_t)p * kp + q];
						const double g = hypot(cpq.x, cpq.y);
						if (g > 1e-300 && g > kSkipBelow * sqrt(fabs(a) * fabs(b))) {
							// real problem [[a, g], [g, b]]: t = sign(z) / (|z| + sqrt(1 + z^2)), z = (b - a) / 2g
							const double z = 0.5 * (b - a) / g;
							const double t = (z >= 0 ? 1.0 : -1.0) / (fabs(z) + sqrt(1.0 + z * z));
							const double c = 1.0 / sqrt(1.0 + t * t);
							R.c = c;
							R.s = t * c;
							R.ur = cpq.x / g;
							R.ui = cpq.y / g;
							R.p = p;
							tmax = fmax(tmax, fabs(t));
						}
					}
					rot[jj] = R;
				}
				__syncthreads();
				// rows p, q of A: A <- Q^H A
				for (int idx = tid; idx < nj * kp; idx += blockDim.x) {
					const Rot R = rot[idx / kp];
					if (R.p < 0) continue;
					const int col = idx % kp;
					double2* xp = A + (size_t)R.p * kp + col;
					double2* xq = A + (size_t)R.q * kp + col;
					const double2 ap = *xp, aq = *xq;
					// row p: c a_p - s u a_q ; row q: s conj(u) a_p + c a_q
					const double sur = R.s * R.ur, sui = R.s * R.ui;
					xp->x = R.c * ap.x - (sur * aq.x - sui * aq.y);
					xp->y = R.c * ap.y - (sur * aq.y + sui * aq.x);
					xq->x = (sur * ap.x + sui * ap.y) + R.c * aq.x;
					xq->y = (sur * ap.y - sui * ap.x) + R.c * aq.y;
				}
				__syncthreads();
				// columns p, q of A and V: X <- X Q
				for (int idx = tid; idx < nj * kp * 2; idx += blockDim.x) {
					const int half = idx / (nj * kp);
					const int rest = idx - half * nj * kp;
					const Rot R = rot[rest / kp];
					if (R.p < 0) continue;
					const int row = rest % kp;
					double2* X = half ? V : A;
					double2* xp = X + (size_t)row * kp + R.p;
					double2* xq = X + (size_t)row * kp + R.q;
					const double2 ap = *xp, aq = *xq;
					// col p: c a_p - s conj(u) a_q ; col q: s u a_p + c a_q
					const double sur = R.s * R.ur, sui = R.s * R.ui;
					xp->x = R.c * ap.x - (sur * aq.x + sui * aq.y);
					xp->y = R.c * ap.y - (sur * aq.y - sui * aq.x);
					xq->x = (sur * ap.x - sui * ap.y) + R.c * aq.x;
					xq->y = (sur * ap.y + sui * ap.x) + R.c * aq.y;
				}
				__syncthreads();
			}
		}
		// largest tangent of the sweep over the CTA
		for (int o = 16; o > 0; o >>= 1) tmax = fmax(tmax, __shfl_xor_sync(0xffffffffu, tmax, o));
		if ((tid & 31) == 0) red[tid >> 5] = tmax;
		__syncthreads();
		if (tid == 0) {
			double m = 0.0;
			for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmax(m, red[w]);
			red[0] = m;
		}
		__syncthreads();
		const double m = red[0];
		__syncthreads();
		if (m < it.tau) {
			if (tid == 0) s_sweeps = sweep + 1;
			break;
		}
	}
	__syncthreads();
	// ascending eigenvalues: rank of each diagonal element (ties by index)
	for (int i = tid; i < k; i += blockDim.x) {
		const double ei = A[(size_t)i * kp + i].x;
		int rank = 0;
		for (int j = 0; j < k; j++) {
			const double ej = A[(size_t)j * kp + j].x;
			rank += (ej < ei || (ej == ei && j < i)) ? 1 : 0;
		}
		it.perm[rank] = i;
		it.evals[rank] = ei;
	}
	if (tid == 0) s_bad = k;
	__syncthreads();
	// first offending eigenvalue in ascending order (stateset.cpp:158-172)
	for (int r = tid; r < k; r += blockDim.x) {
		const double e = it.evals[r];
		if (!(e > 0.0) || !(e >= 2.2250738585072014e-308) || isinf(e) || e != e) atomicMin(&s_bad, r);
	}
	__syncthreads();
	if (tid == 0) {
		EigStatus st;
		st.sweeps = s_sweeps;
		st.pad = 0;
		st.bad_index = -1;
		st.bad_value = 0.0;
		st.status = ITP2D_OK;
		if (s_sweeps < 0) st.status = ITP2D_E_EIGENSOLVER;
		if (s_bad < k) {
			const double e = it.evals[s_bad];
			st.status = e <= 0.0 ? ITP2D_E_NONPOSITIVE_EIGENVALUE : ITP2D_E_NONNORMAL_EIGENVALUE;
			st.bad_index = s_bad;
			st.bad_value = e;
		}
		*it.st = st;
	}
	__syncthreads();
	if (s_bad < k) return;
	for (int idx = tid; idx < k * k; idx += blockDim.x) {
		const int i = idx / k, m = idx % k;
		const int src = it.perm[m];
		const double f = 1.0 / sqrt(it.evals[m]);
		const double2 v = V[(size_t)i * kp + src];
		it.W[idx] = make_double2(v.x * f, v.y * f);
	}
}

// Persistent work queue: every CTA takes the next instance from *next until
// none is left. The host orders the instances by decreasing k (the longest
// first), so uneven sizes finish together.
__global__ void __launch_bounds__(kBThreads) batched_jacobi_kernel(const BatchEigItem* __restrict__ items, int n,
		int max_sweeps, int smem_bytes, int* next) {
	__shared__ int s_next;
	for (;;) {
		if (threadIdx.x == 0) s_next = atomicAdd(next, 1);
		__syncthreads();
		const int q = s_next;
		__syncthreads();  // every thread has read s_next before it changes
		if (q >= n) return;
		const BatchEigItem it = items[q];
		solve_item(it, max_sweeps, smem_bytes);
		__syncthreads();
	}
}

}  // namespace

cudaError_t launch_batched_eigensolve(const BatchEigItem* items, int n, int max_sweeps, int max_k, int* next,
		cudaStream_t s) {
	if (n <= 0) return cudaSuccess;
	// dynamic shared memory for A and V of the largest instance, up to 200 KB
	// (instances whose matrices do not fit use their global work matrices)
	const size_t kp = (size_t)((max_k + 1) & ~1);
	const size_t want = 2 * kp * kp * sizeof(double2);
	const size_t one = kp * kp * sizeof(double2);
	const size_t cap = 200 * 1024;
	const int smem = (int)(want <= cap ? want : (one <= cap ? one : 0));
	if (smem > 48 * 1024) {
		const cudaError_t e = cudaFuncSetAttribute(batched_jacobi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
				smem);
		if (e != cudaSuccess) return e;
	}
	static int sms = 0;
	if (!sms) {
		int dev = 0;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	}
	int per_sm = 0;
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batched_jacobi_kernel, kBThreads, smem);
	const int grid = std::max(1, std::min(n, std::max(1, per_sm) * std::max(1, sms)));
	cudaError_t e = cudaMemsetAsync(next, 0, sizeof(int), s);
	if (e != cudaSuccess) return e;
	batched_jacobi_kernel<<<grid, kBThreads, smem, s>>>(items, n, max_sweeps, smem, next);
	return cudaGetLastError();
}

int batched_eigensolve_max_k() { return 2 * kMaxPairs; }

}  // namespace itp2d
