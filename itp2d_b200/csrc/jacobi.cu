// Hermitian eigen-decomposition of the k x k overlap matrix on the GPU.
//
// Replaces EigenSolver::solve (ZHEEV, eigensolver.hpp:80-84) and the checks
// and scaling of StateSet::orthonormalize (stateset.cpp:155-176). Method:
// parallel cyclic two-sided Jacobi. Each round applies kp/2 disjoint complex
// plane rotations J_pq (round-robin "circle" pairing, every pair once per
// sweep), A <- J^H A J and V <- V J, with A double-buffered so a round needs
// one grid-wide barrier. Rotation angles follow the classical Jacobi
// formulas (tan of the smaller angle), lifted to the Hermitian case by the
// phase of A_pq. A rotation is skipped when |A_pq| <= tol sqrt(|A_pp A_qq|),
// which gives the high relative accuracy Jacobi is known for on positive
// definite matrices; a sweep without rotations ends the iteration.
#include <cooperative_groups.h>

#include "contract.cuh"
#include "../../include/itp2d_gpu.h"

namespace cg = cooperative_groups;

namespace itp2d {

namespace {

constexpr int TP = 16;        // pair slots per tile side
constexpr int kVRows = 32;    // V rows per work item
constexpr int kThreads = 256;

struct Rot {
	double c, s, er, ei;  // J = [[c, s e], [-s conj(e), c]], e = er + i ei
	double ap, aq;        // rotated diagonal
	int p, q;
	int rotated;
};

__device__ __forceinline__ int player(int pos, int r, int kp) {
	return pos == 0 ? 0 : ((pos - 1 + r) % (kp - 1)) + 1;
}

__device__ __forceinline__ double2 ldA(const double2* A, long long idx) { return __ldcg(A + idx); }

__device__ void make_rot(Rot& R, const double2* A, int kp, int slot, int r, double tol) {
	const int p = player(slot, r, kp);
	const int q = player(kp - 1 - slot, r, kp);
	R.p = p;
	R.q = q;
	const double a = ldA(A, (long long)p * kp + p).x;
	const double b = ldA(A, (long long)q * kp + q).x;
	const double2 c = ldA(A, (long long)p * kp + q);
	const double cabs = hypot(c.x, c.y);
	R.c = 1.0; R.s = 0.0; R.er = 1.0; R.ei = 0.0; R.ap = a; R.aq = b; R.rotated = 0;
	if (cabs > 0.0 && cabs > tol * sqrt(fabs(a) * fabs(b))) {
		const double th = (b - a) / (2.0 * cabs);
		const double ath = fabs(th);
		double t = (ath > 1e150) ? 0.5 / ath : 1.0 / (ath + sqrt(th * th + 1.0));
		if (th < 0) t = -t;
		if (t != 0.0) {
			R.c = 1.0 / sqrt(t * t + 1.0);
			R.s = t * R.c;
			R.er = c.x / cabs;
			R.ei = c.y / cabs;
			R.ap = a - t * cabs;
			R.aq = b + t * cabs;
			R.rotated = 1;
		}
	}
}

__device__ __forceinline__ double2 cm(double2 a, double2 b) {
	return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd2(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csc(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// Rows of J^H X for J = [[c, s e], [-s conj(e), c]], written as corrections
// of the old values (tau = s / (1 + c)), which keeps small rotations accurate.
__device__ __forceinline__ void rot_rows(const Rot& R, double2 xp, double2 xq, double2& yp, double2& yq) {
	const double tau = R.s / (1.0 + R.c);
	const double2 e = make_double2(R.er, R.ei);
	yp = cadd2(xp, csc(cadd2(cm(e, xq), csc(xp, tau)), -R.s));
	yq = cadd2(xq, csc(cadd2(cm(cconj(e), xp), csc(xq, -tau)), R.s));
}

// Columns of X J in the same correction form.
__device__ __forceinline__ void rot_cols(const Rot& C, double2 xs, double2 xt, double2& ys, double2& yt) {
	const double tau = C.s / (1.0 + C.c);
	const double2 e = make_double2(C.er, C.ei);
	ys = cadd2(xs, csc(cadd2(cm(cconj(e), xt), csc(xs, tau)), -C.s));
	yt = cadd2(xt, csc(cadd2(cm(e, xs), csc(xt, -tau)), C.s));
}

__global__ void __launch_bounds__(kThreads) jacobi_kernel(double2* A0, double2* A1, double2* V, int kp,
		int max_sweeps, double tol, int* counters) {
	cg::grid_group grid = cg::this_grid();
	__shared__ Rot rr[TP];
	__shared__ Rot rc[TP];
	const int np = kp / 2;
	const int nt = (np + TP - 1) / TP;
	const int nA = nt * nt;
	const int nVr = (kp + kVRows - 1) / kVRows;
	const int nW = nA + nVr * nt;
	double2* Acur = A0;
	double2* Anext = A1;
	int sweep = 0;
	for (; sweep < max_sweeps; sweep++) {
		for (int r = 0; r < kp - 1; r++) {
			for (int w = blockIdx.x; w < nW; w += gridDim.x) {
				if (w < nA) {
					const int TI = w / nt, TJ = w % nt;
					if (threadIdx.x < TP) {
						const int sl = TI * TP + threadIdx.x;
						if (sl < np) make_rot(rr[threadIdx.x], Acur, kp, sl, r, tol);
					} else if (threadIdx.x < 2 * TP) {
						const int sl = TJ * TP + threadIdx.x - TP;
						if (sl < np) make_rot(rc[threadIdx.x - TP], Acur, kp, sl, r, tol);
					}
					__syncthreads();
					for (int e = threadIdx.x; e < TP * TP; e += blockDim.x) {
						const int a = e / TP, b = e % TP;
						const int sa = TI * TP + a, sb = TJ * TP + b;
						if (sa >= np || sb >= np) continue;
						const Rot& R = rr[a];
						const Rot& C = rc[b];
						const int p = R.p, q = R.q, s = C.p, t = C.q;
						if (sa == sb) {
							Anext[(long long)p * kp + p] = make_double2(R.ap, 0.0);
							Anext[(long long)q * kp + q] = make_double2(R.aq, 0.0);
							if (R.rotated) {
								Anext[(long long)p * kp + q] = make_double2(0.0, 0.0);
								Anext[(long long)q * kp + p] = make_double2(0.0, 0.0);
								atomicAdd(&counters[sweep], 1);
							} else {
								Anext[(long long)p * kp + q] = ldA(Acur, (long long)p * kp + q);
								Anext[(long long)q * kp + p] = ldA(Acur, (long long)q * kp + p);
							}
							continue;
						}
						const double2 xps = ldA(Acur, (long long)p * kp + s);
						const double2 xpt = ldA(Acur, (long long)p * kp + t);
						const double2 xqs = ldA(Acur, (long long)q * kp + s);
						const double2 xqt = ldA(Acur, (long long)q * kp + t);
						// Y = Jr^H X in the tau form y_p = x_p - s(e x_q + tau x_p),
						// y_q = x_q + s(conj(e) x_p - tau x_q), tau = s / (1 + c)
						double2 y1s, y1t, y2s, y2t;
						rot_rows(R, xps, xqs, y1s, y2s);
						rot_rows(R, xpt, xqt, y1t, y2t);
						// X' = Y Jc: x_s' = x_s - s(conj(e) x_t + tau x_s), x_t' = x_t + s(e x_s - tau x_t)
						double2 o;
						rot_cols(C, y1s, y1t, o, Anext[(long long)p * kp + t]);
						Anext[(long long)p * kp + s] = o;
						rot_cols(C, y2s, y2t, o, Anext[(long long)q * kp + t]);
						Anext[(long long)q * kp + s] = o;
					}
					__syncthreads();
				} else {
					const int v = w - nA;
					const int RC = v / nt, TJ = v % nt;
					if (threadIdx.x < TP) {
						const int sl = TJ * TP + threadIdx.x;
						if (sl < np) make_rot(rc[threadIdx.x], Acur, kp, sl, r, tol);
					}
					__syncthreads();
					for (int e = threadIdx.x; e < kVRows * TP; e += blockDim.x) {
						const int ii = e / TP, b = e % TP;
						const int i = RC * kVRows + ii, sb = TJ * TP + b;
						if (i >= kp || sb >= np) continue;
						const Rot& C = rc[b];
						if (!C.rotated) continue;
						const long long is = (long long)i * kp + C.p, it = (long long)i * kp + C.q;
						const double2 vs = ldA(V, is), vt = ldA(V, it);
						double2 ns, nt2;
						rot_cols(C, vs, vt, ns, nt2);
						V[is] = ns;
						V[it] = nt2;
					}
					__syncthreads();
				}
			}
			grid.sync();
			double2* tmp = Acur;
			Acur = Anext;
			Anext = tmp;
		}
		const int cnt = *((volatile int*)&counters[sweep]);
		if (cnt == 0) break;
	}
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		counters[max_sweeps] = (sweep < max_sweeps) ? sweep + 1 : -1;  // sweeps used, -1: no convergence
		counters[max_sweeps + 1] = (Acur == A0) ? 0 : 1;                // buffer holding the result
	}
}

// Copy S (k x k) into the padded kp x kp work matrix; V = I.
__global__ void jacobi_init_kernel(const double2* __restrict__ S, int k, int kp, double2* A, double2* V) {
	const long long n = (long long)kp * kp;
	for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
			idx += (long long)gridDim.x * blockDim.x) {
		const int i = (int)(idx / kp), j = (int)(idx % kp);
		A[idx] = (i < k && j < k) ? S[(long long)i * k + j] : make_double2(0.0, 0.0);
		V[idx] = make_double2(i == j ? 1.0 : 0.0, 0.0);
	}
}

// Normalises the first k columns of V in place (removes the norm drift that
// the accumulated rotations leave). 32 columns per CTA, 8 row groups.
__global__ void __launch_bounds__(256) normalize_columns_kernel(double2* V, int k, int kp) {
	__shared__ double part[8][32];
	const int cl = threadIdx.x & 31, rg = threadIdx.x >> 5;
	const int j = blockIdx.x * 32 + cl;
	double sum = 0.0;
	if (j < k)
		for (int i = rg; i < kp; i += 8) {
			const double2 v = __ldcg(V + (long long)i * kp + j);
			sum += v.x * v.x + v.y * v.y;
		}
	part[rg][cl] = sum;
	__syncthreads();
	if (rg == 0) {
		double t = 0.0;
		for (int r = 0; r < 8; r++) t += part[r][cl];
		part[0][cl] = t > 0.0 ? 1.0 / sqrt(t) : 1.0;
	}
	__syncthreads();
	const double f = part[0][cl];
	if (j < k)
		for (int i = rg; i < kp; i += 8) {
			const long long o = (long long)i * kp + j;
			const double2 v = __ldcg(V + o);
			V[o] = make_double2(v.x * f, v.y * f);
		}
}

// Sort the k eigenvalues ascending (bitonic, one CTA) and run the checks of
// stateset.cpp:158-173 in that order.
__global__ void eig_sort_kernel(const double2* __restrict__ A0, const double2* __restrict__ A1, int k, int kp,
		const int* counters, int max_sweeps, double* evals, int* perm, EigStatus* st, int check) {
	extern __shared__ unsigned char sm[];
	int P = 1;
	while (P < k) P <<= 1;
	double* key = reinterpret_cast<double*>(sm);
	int* idx = reinterpret_cast<int*>(key + P);
	const double2* A = counters[max_sweeps + 1] == 0 ? A0 : A1;
	for (int i = threadIdx.x; i < P; i += blockDim.x) {
		if (i < k) {
			double v = __ldcg(A + (long long)i * kp + i).x;
			if (v != v) v = -INFINITY;  // NaN sorts first so the check below reports it
			key[i] = v;
		} else {
			key[i] = INFINITY;
		}
		idx[i] = i;
	}
	__syncthreads();
	for (int size = 2; size <= P; size <<= 1) {
		for (int stride = size >> 1; stride > 0; stride >>= 1) {
			for (int i = threadIdx.x; i < P; i += blockDim.x) {
				const int j = i ^ stride;
				if (j > i) {
					const bool up = (i & size) == 0;
					const double ki = key[i], kj = key[j];
					const bool swap = up ? (ki > kj || (ki == kj && idx[i] > idx[j]))
					                     : (ki < kj || (ki == kj && idx[i] < idx[j]));
					if (swap) {
						key[i] = kj;
						key[j] = ki;
						const int t = idx[i];
						idx[i] = idx[j];
						idx[j] = t;
					}
				}
			}
			__syncthreads();
		}
	}
	for (int i = threadIdx.x; i < k; i += blockDim.x) {
		perm[i] = idx[i];
		evals[i] = __ldcg(A + (long long)idx[i] * kp + idx[i]).x;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		EigStatus s;
		s.status = ITP2D_OK;
		s.bad_index = -1;
		s.bad_value = 0.0;
		s.pad = 0;
		s.sweeps = counters[max_sweeps];
		if (s.sweeps < 0) s.status = ITP2D_E_EIGENSOLVER;
		for (int n = 0; n < k && s.status == ITP2D_OK && check; n++) {
			const double v = evals[n];
			if (v <= 0.0) {
				s.status = ITP2D_E_NONPOSITIVE_EIGENVALUE;
				s.bad_index = n;
				s.bad_value = v;
			} else if (!(v >= 2.2250738585072014e-308) || isinf(v) || v != v) {
				s.status = ITP2D_E_NONNORMAL_EIGENVALUE;
				s.bad_index = n;
				s.bad_value = v;
			}
		}
		*st = s;
	}
}

// W[i][n] = V[i][perm[n]] / sqrt(l_n) (the zdscal of stateset.cpp:175).
__global__ void build_w_kernel(const double2* __restrict__ V, int k, int kp, const double* __restrict__ evals,
		const int* __restrict__ perm, double2* W) {
	const long long n2 = (long long)k * k;
	for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n2;
			idx += (long long)gridDim.x * blockDim.x) {
		const int i = (int)(idx / k), n = (int)(idx % k);
		const double f = 1.0 / sqrt(evals[n]);
		const double2 v = __ldcg(V + (long long)i * kp + perm[n]);
		W[idx] = make_double2(v.x * f, v.y * f);
	}
}

}  // namespace

size_t jacobi_counters(int max_sweeps) { return (size_t)max_sweeps + 4; }

cudaError_t launch_eigensolve(double2* S, int k, JacobiWork& w, double2* W, EigStatus* st, int num_sms,
		cudaStream_t s) {
	cudaError_t e = launch_eigh(S, k, w, st, num_sms, s, 1);
	if (e != cudaSuccess) return e;
	const long long n2 = (long long)k * k;
	const int kp = (k + 1) & ~1;
	build_w_kernel<<<(unsigned)std::min<long long>((n2 + 255) / 256, 4096), 256, 0, s>>>(w.V, k, kp, w.evals,
			w.perm, W);
	return cudaGetLastError();
}

cudaError_t launch_eigh(double2* S, int k, JacobiWork& w, EigStatus* st, int num_sms, cudaStream_t s, int check) {
	const int kp = (k + 1) & ~1;
	const long long n = (long long)kp * kp;
	cudaError_t e = cudaMemsetAsync(w.counters, 0, jacobi_counters(w.max_sweeps) * sizeof(int), s);
	if (e != cudaSuccess) return e;
	jacobi_init_kernel<<<(unsigned)std::min<long long>((n + 255) / 256, 4096), 256, 0, s>>>(S, k, kp, w.A0, w.V);
	int per_sm = 0;
	e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, jacobi_kernel, kThreads, 0);
	if (e != cudaSuccess) return e;
	if (per_sm < 1) return cudaErrorLaunchOutOfResources;
	const int np = kp / 2;
	const int nt = (np + TP - 1) / TP;
	const int nW = nt * nt + ((kp + kVRows - 1) / kVRows) * nt;
	int blocks = std::min(num_sms * std::min(per_sm, 2), nW);
	if (blocks < 1) blocks = 1;
	double tol = 1e-15;
	int ms = w.max_sweeps;
	void* args[] = {&w.A0, &w.A1, &w.V, (void*)&kp, &ms, &tol, &w.counters};
	e = cudaLaunchCooperativeKernel((void*)jacobi_kernel, dim3(blocks), dim3(kThreads), args, 0, s);
	if (e != cudaSuccess) return e;
	normalize_columns_kernel<<<(k + 31) / 32, 256, 0, s>>>(w.V, k, kp);
	int P = 1;
	while (P < k) P <<= 1;
	const size_t smem = (size_t)P * (sizeof(double) + sizeof(int));
	if (smem > 48 * 1024) cudaFuncSetAttribute(eig_sort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
	eig_sort_kernel<<<1, 1024, smem, s>>>(w.A0, w.A1, k, kp, w.counters, w.max_sweeps, w.evals, w.perm, st,
			check);
	return cudaGetLastError();
}

}  // namespace itp2d
