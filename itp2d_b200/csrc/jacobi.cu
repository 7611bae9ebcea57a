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
#include <atomic>
#include <mutex>

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
	double t;             // |tan| of the rotation angle (0 when skipped)
	int rotated;
};

__device__ __forceinline__ int player(int pos, int r, int kp) {
	return pos == 0 ? 0 : ((pos - 1 + r) % (kp - 1)) + 1;
}

__device__ __forceinline__ double2 ldA(const double2* A, long long idx) { return __ldcg(A + idx); }

__device__ void make_rot(Rot& R, const double2* A, int kp, int slot, int r, double tol) {
	const int p = player(slot, r, kp);
	const int q = player(kp - 1 - slot, r, kp);
	const double a = ldA(A, (long long)p * kp + p).x;
	const double b = ldA(A, (long long)q * kp + q).x;
	const double2 c = ldA(A, (long long)p * kp + q);
	const double cabs = hypot(c.x, c.y);
	R.c = 1.0; R.s = 0.0; R.er = 1.0; R.ei = 0.0; R.ap = a; R.aq = b; R.t = 0.0; R.rotated = 0;
	if (cabs > 0.0 && cabs > tol * sqrt(fabs(a) * fabs(b))) {
		const double th = (b - a) / (2.0 * cabs);
		const double ath = fabs(th);
		const double t = (ath > 1e150) ? 0.5 / ath : 1.0 / (ath + sqrt(th * th + 1.0));
		if (t != 0.0) {
			R.c = 1.0 / sqrt(t * t + 1.0);
			R.s = (th < 0 ? -t : t) * R.c;
			R.er = c.x / cabs;
			R.ei = c.y / cabs;
			R.ap = a - (th < 0 ? -t : t) * cabs;
			R.aq = b + (th < 0 ? -t : t) * cabs;
			R.t = t;
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

constexpr int kItems = 2;  // work items per CTA between two CTA barriers

// Tangent below which a sweep is final: the next sweep could only change
// off-diagonal elements by O(k tau^2) relative to the eigenvalue gaps.
constexpr double kTauFinal = 1e-10;

// One cooperative launch = the whole eigensolve. Per round, each CTA takes up
// to kItems work items (an A tile of TP x TP pair blocks, or a V tile of
// kVRows rows x TP pairs), issues all of their global loads together with the
// loads of the rotation inputs, then applies the rotations after one CTA
// barrier; the round ends with one grid barrier.
__global__ void __launch_bounds__(kThreads) jacobi_kernel(double2* A0, double2* A1, double2* V, int kp,
		int max_sweeps, double tol, double tau_final, int* counters, unsigned long long* tmax) {
	cg::grid_group grid = cg::this_grid();
	__shared__ Rot rr[kItems][TP];
	__shared__ Rot rc[kItems][TP];
	__shared__ int s_cnt;                 // rotations applied by this CTA in the sweep
	__shared__ unsigned long long s_tmax;  // largest tangent (bit pattern of a non-negative double)
	const int tid = threadIdx.x;
	if (tid == 0) {
		s_cnt = 0;
		s_tmax = 0ULL;
	}
	__syncthreads();
	const int np = kp / 2;
	const int nt = (np + TP - 1) / TP;
	const int nA = nt * nt;
	const int nVr = (kp + kVRows - 1) / kVRows;
	const int nW = nA + nVr * nt;
	double2* Acur = A0;
	double2* Anext = A1;
	int sweep = 0;
	bool converged = false;
	for (; sweep < max_sweeps && !converged; sweep++) {
		for (int r = 0; r < kp - 1; r++) {
			for (int w0 = blockIdx.x * kItems; w0 < nW; w0 += gridDim.x * kItems) {
				double2 x[kItems][4];
				// phase 1: rotation set-up and all loads
#pragma unroll
				for (int it = 0; it < kItems; it++) {
					const int w = w0 + it;
					if (w >= nW) break;
					if (w < nA) {
						const int TI = w / nt, TJ = w % nt;
						if (tid < TP) {
							const int sl = TI * TP + tid;
							if (sl < np) make_rot(rr[it][tid], Acur, kp, sl, r, tol);
						} else if (tid < 2 * TP) {
							const int sl = TJ * TP + tid - TP;
							if (sl < np) make_rot(rc[it][tid - TP], Acur, kp, sl, r, tol);
						}
						const int sa = TI * TP + tid / TP, sb = TJ * TP + tid % TP;
						if (sa < np && sb < np) {
							const int p = player(sa, r, kp), q = player(kp - 1 - sa, r, kp);
							const int s2 = player(sb, r, kp), t2 = player(kp - 1 - sb, r, kp);
							if (sa == sb) {
								x[it][0] = ldA(Acur, (long long)p * kp + q);
								x[it][1] = ldA(Acur, (long long)q * kp + p);
							} else {
								x[it][0] = ldA(Acur, (long long)p * kp + s2);
								x[it][1] = ldA(Acur, (long long)p * kp + t2);
								x[it][2] = ldA(Acur, (long long)q * kp + s2);
								x[it][3] = ldA(Acur, (long long)q * kp + t2);
							}
						}
					} else {
						const int v = w - nA;
						const int RC = v / nt, TJ = v % nt;
						if (tid < TP) {
							const int sl = TJ * TP + tid;
							if (sl < np) make_rot(rc[it][tid], Acur, kp, sl, r, tol);
						}
#pragma unroll
						for (int h = 0; h < 2; h++) {
							const int e = tid + h * kThreads;
							const int i = RC * kVRows + e / TP, sb = TJ * TP + e % TP;
							if (i < kp && sb < np) {
								const int s2 = player(sb, r, kp), t2 = player(kp - 1 - sb, r, kp);
								x[it][2 * h] = ldA(V, (long long)i * kp + s2);
								x[it][2 * h + 1] = ldA(V, (long long)i * kp + t2);
							}
						}
					}
				}
				__syncthreads();
				// phase 2: apply
#pragma unroll
				for (int it = 0; it < kItems; it++) {
					const int w = w0 + it;
					if (w >= nW) break;
					if (w < nA) {
						const int TI = w / nt, TJ = w % nt;
						const int a = tid / TP, b = tid % TP;
						const int sa = TI * TP + a, sb = TJ * TP + b;
						if (sa >= np || sb >= np) continue;
						const Rot& R = rr[it][a];
						const Rot& C = rc[it][b];
						const int p = player(sa, r, kp), q = player(kp - 1 - sa, r, kp);
						if (sa == sb) {
							Anext[(long long)p * kp + p] = make_double2(R.ap, 0.0);
							Anext[(long long)q * kp + q] = make_double2(R.aq, 0.0);
							if (R.rotated) {
								Anext[(long long)p * kp + q] = make_double2(0.0, 0.0);
								Anext[(long long)q * kp + p] = make_double2(0.0, 0.0);
								atomicAdd(&s_cnt, 1);
								atomicMax(&s_tmax, (unsigned long long)__double_as_longlong(R.t));
							} else {
								Anext[(long long)p * kp + q] = x[it][0];
								Anext[(long long)q * kp + p] = x[it][1];
							}
							continue;
						}
						const int s2 = player(sb, r, kp), t2 = player(kp - 1 - sb, r, kp);
						double2 y1s, y1t, y2s, y2t, o1, o2;
						rot_rows(R, x[it][0], x[it][2], y1s, y2s);
						rot_rows(R, x[it][1], x[it][3], y1t, y2t);
						rot_cols(C, y1s, y1t, o1, o2);
						Anext[(long long)p * kp + s2] = o1;
						Anext[(long long)p * kp + t2] = o2;
						rot_cols(C, y2s, y2t, o1, o2);
						Anext[(long long)q * kp + s2] = o1;
						Anext[(long long)q * kp + t2] = o2;
					} else {
						const int v = w - nA;
						const int RC = v / nt, TJ = v % nt;
#pragma unroll
						for (int h = 0; h < 2; h++) {
							const int e = tid + h * kThreads;
							const int i = RC * kVRows + e / TP, b = e % TP, sb = TJ * TP + b;
							if (i >= kp || sb >= np) continue;
							const Rot& C = rc[it][b];
							if (!C.rotated) continue;
							const int s2 = player(sb, r, kp), t2 = player(kp - 1 - sb, r, kp);
							double2 ns, nt2;
							rot_cols(C, x[it][2 * h], x[it][2 * h + 1], ns, nt2);
							V[(long long)i * kp + s2] = ns;
							V[(long long)i * kp + t2] = nt2;
						}
					}
				}
				__syncthreads();
			}
			grid.sync();
			double2* tmp = Acur;
			Acur = Anext;
			Anext = tmp;
		}
		// one global update per CTA and sweep, then a grid barrier so every CTA
		// reads the final totals
		if (tid == 0) {
			if (s_cnt) atomicAdd(&counters[sweep], s_cnt);
			if (s_tmax) atomicMax(&tmax[sweep], s_tmax);
			s_cnt = 0;
			s_tmax = 0ULL;
		}
		grid.sync();
		// uniform across the grid: everything below reads values final after grid.sync
		const int cnt = *((volatile int*)&counters[sweep]);
		const double tm = __longlong_as_double((long long)*((volatile unsigned long long*)&tmax[sweep]));
		if (cnt == 0 || tm < tau_final) converged = true;
	}
	if (blockIdx.x == 0 && threadIdx.x == 0) {
		counters[max_sweeps] = converged ? sweep : -1;   // sweeps used, -1: no convergence
		counters[max_sweeps + 1] = (Acur == A0) ? 0 : 1;  // buffer holding the result
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
// Columns j of V scaled to unit norm: 32 columns per CTA, 32 row groups; the
// row loops are unrolled by 4 so that several loads are in flight per thread.
__global__ void __launch_bounds__(1024) normalize_columns_kernel(double2* V, int k, int kp) {
	__shared__ double part[32][33];
	const int cl = threadIdx.x & 31, rg = threadIdx.x >> 5;
	const int j = blockIdx.x * 32 + cl;
	double sum = 0.0;
	if (j < k) {
#pragma unroll 4
		for (int i = rg; i < kp; i += 32) {
			const double2 v = __ldcg(V + (long long)i * kp + j);
			sum += v.x * v.x + v.y * v.y;
		}
	}
	part[rg][cl] = sum;
	__syncthreads();
	if (rg == 0) {
		double t = 0.0;
		for (int r = 0; r < 32; r++) t += part[r][cl];
		part[0][cl] = t > 0.0 ? 1.0 / sqrt(t) : 1.0;
	}
	__syncthreads();
	const double f = part[0][cl];
	if (j < k) {
#pragma unroll 4
		for (int i = rg; i < kp; i += 32) {
			const long long o = (long long)i * kp + j;
			const double2 v = __ldcg(V + o);
			V[o] = make_double2(v.x * f, v.y * f);
		}
	}
}

// Sort the k eigenvalues ascending (bitonic, one CTA) and run the checks of
// stateset.cpp:158-173 in that order.
__global__ void eig_sort_kernel(const double2* __restrict__ A0, const double2* __restrict__ A1,
		const double2* __restrict__ A2, int k, int kp, const int* counters, int max_sweeps, double* evals, int* perm,
		EigStatus* st, int check) {
	extern __shared__ unsigned char sm[];
	int P = 1;
	while (P < k) P <<= 1;
	double* key = reinterpret_cast<double*>(sm);
	int* idx = reinterpret_cast<int*>(key + P);
	const int which = counters[max_sweeps + 1];
	const double2* A = which == 0 ? A0 : (which == 1 ? A1 : A2);
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
	// the checks in eigenvalue order: the first failing n, found in parallel
	__shared__ int first_bad;
	if (threadIdx.x == 0) first_bad = k;
	__syncthreads();
	for (int i = threadIdx.x; i < k; i += blockDim.x) {
		perm[i] = idx[i];
		const double v = __ldcg(A + (long long)idx[i] * kp + idx[i]).x;
		evals[i] = v;
		if (check && (v <= 0.0 || !(v >= 2.2250738585072014e-308) || isinf(v) || v != v)) atomicMin(&first_bad, i);
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		EigStatus s;
		s.status = ITP2D_OK;
		s.bad_index = -1;
		s.bad_value = 0.0;
		s.pad = 0;
		s.sweeps = counters[max_sweeps];
		if (s.sweeps < 0 && check == 2) {
			s.sweeps = max_sweeps;  // a capped solve: the caller finishes it
		} else if (s.sweeps < 0) {
			s.status = ITP2D_E_EIGENSOLVER;
		} else if (first_bad < k) {
			const int n = first_bad;
			const double v = __ldcg(A + (long long)idx[n] * kp + idx[n]).x;
			s.status = v <= 0.0 ? ITP2D_E_NONPOSITIVE_EIGENVALUE : ITP2D_E_NONNORMAL_EIGENVALUE;
			s.bad_index = n;
			s.bad_value = v;
		}
		*st = s;
	}
}

// S_out[a][b] = (A[p(a)][p(b)] + conj(A[p(b)][p(a)])) / 2 and VT[a][i] =
// V[i][p(a)], p(a) = perm[k - 1 - a]: the overlap of the states rotated onto
// the columns of V, largest eigenvalue (lowest energy) first.
__global__ void eig_cholesky_prep_kernel(const double2* __restrict__ A0, const double2* __restrict__ A1,
		const double2* __restrict__ A2, const double2* __restrict__ V, const int* __restrict__ perm,
		const int* __restrict__ counters, int max_sweeps, int k, int kp, double2* __restrict__ S_out,
		double2* __restrict__ VT) {
	const int which = counters[max_sweeps + 1];
	const double2* A = which == 0 ? A0 : (which == 1 ? A1 : A2);
	const long long n2 = (long long)k * k;
	for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n2;
			idx += (long long)gridDim.x * blockDim.x) {
		const int a = (int)(idx / k), b = (int)(idx % k);
		const int pa = perm[k - 1 - a], pb = perm[k - 1 - b];
		const double2 x = __ldcg(A + (long long)pa * kp + pb), y = __ldcg(A + (long long)pb * kp + pa);
		S_out[idx] = make_double2(0.5 * (x.x + y.x), 0.5 * (x.y - y.y));
		VT[idx] = __ldcg(V + (long long)b * kp + pa);
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

// W[i][n] = V[i][perm[n]]: the Ritz vectors' coefficients, ascending Ritz values.
__global__ void ritz_w_kernel(const double2* __restrict__ V, int k, int kp, const int* __restrict__ perm, double2* W) {
	const long long n2 = (long long)k * k;
	for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n2;
			idx += (long long)gridDim.x * blockDim.x) {
		const int i = (int)(idx / k), n = (int)(idx % k);
		W[idx] = __ldcg(V + (long long)i * kp + perm[n]);
	}
}

}  // namespace

size_t jacobi_counters(int max_sweeps) { return jacobi_counter_ints(max_sweeps); }

namespace {
std::atomic<int> g_coop_users{0};
std::mutex g_coop_mu;
}  // namespace

void coop_user_enter() { g_coop_users.fetch_add(1); }
void coop_user_leave() { g_coop_users.fetch_sub(1); }

cudaError_t launch_eigensolve(double2* S, int k, JacobiWork& w, double2* W, EigStatus* st, int num_sms,
		cudaStream_t s) {
	cudaError_t e = launch_eigh(S, k, w, st, num_sms, s, 1);
	if (e != cudaSuccess) return e;
	const long long n2 = (long long)k * k;
	const int kp = jacobi_kp(w, k);
	build_w_kernel<<<(unsigned)std::min<long long>((n2 + 255) / 256, 4096), 256, 0, s>>>(w.V, k, kp, w.evals,
			w.perm, W);
	return cudaGetLastError();
}

cudaError_t launch_ritz(double2* H, int k, JacobiWork& w, double2* W, EigStatus* st, int num_sms, cudaStream_t s) {
	cudaError_t e = launch_eigh(H, k, w, st, num_sms, s, 0);
	if (e != cudaSuccess) return e;
	const long long n2 = (long long)k * k;
	ritz_w_kernel<<<(unsigned)std::min<long long>((n2 + 255) / 256, 4096), 256, 0, s>>>(w.V, k, jacobi_kp(w, k),
			w.perm, W);
	return cudaGetLastError();
}

cudaError_t launch_eig_cholesky_prep(const JacobiWork& w, int k, double2* S_out, double2* VT, cudaStream_t s) {
	const long long n2 = (long long)k * k;
	eig_cholesky_prep_kernel<<<(unsigned)std::min<long long>((n2 + 255) / 256, 4096), 256, 0, s>>>(w.A0, w.A1, w.A2,
			w.V, w.perm, w.counters, w.max_sweeps, k, jacobi_kp(w, k), S_out, VT);
	return cudaGetLastError();
}

int jacobi_kp(const JacobiWork& w, int k) {
	return (w.Qbuf && w.A2 && k >= kBlockJacobiMinK) ? bjacobi_padded(k) : ((k + 1) & ~1);
}

cudaError_t launch_eigh(double2* S, int k, JacobiWork& w, EigStatus* st, int num_sms, cudaStream_t s, int check) {
	const int kp = jacobi_kp(w, k);
	const long long n = (long long)kp * kp;
	cudaError_t e = cudaMemsetAsync(w.counters, 0, jacobi_counters(w.max_sweeps) * sizeof(int), s);
	if (e != cudaSuccess) return e;
	// one cooperative kernel at a time while several users share the device:
	// held until the kernel below has finished
	std::unique_lock<std::mutex> serial;
	if (g_coop_users.load() > 1) serial = std::unique_lock<std::mutex>(g_coop_mu);
	if (w.f32.A0 && w.Qbuf && w.A2 && k >= kBlockJacobiMinK) {
		e = launch_bjacobi32(S, k, w, num_sms, s);
		if (e != cudaSuccess) return e;
	} else if (w.Qbuf && w.A2 && k >= kBlockJacobiMinK) {
		jacobi_init_kernel<<<(unsigned)std::min<long long>((n + 255) / 256, 4096), 256, 0, s>>>(S, k, kp, w.A0,
				w.V);
		e = launch_bjacobi(w.A0, w.A1, w.A2, w.V, w.Qbuf, kp, w.max_sweeps, w.tau_final, w.counters, num_sms, s);
		if (e != cudaSuccess) return e;
	} else {
		jacobi_init_kernel<<<(unsigned)std::min<long long>((n + 255) / 256, 4096), 256, 0, s>>>(S, k, kp, w.A0,
				w.V);
		int per_sm = 0;
		e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, jacobi_kernel, kThreads, 0);
		if (e != cudaSuccess) return e;
		if (per_sm < 1) return cudaErrorLaunchOutOfResources;
		const int np = kp / 2;
		const int nt = (np + TP - 1) / TP;
		const int nW = nt * nt + ((kp + kVRows - 1) / kVRows) * nt;
		int blocks = std::min(num_sms * std::min(per_sm, 2), (nW + kItems - 1) / kItems);
		if (blocks < 1) blocks = 1;
		double tol = 1e-15;
		double tau_final = w.tau_final > 0.0 ? w.tau_final : kTauFinal;
		int ms = w.max_sweeps;
		int kpv = kp;
		unsigned long long* tmax = reinterpret_cast<unsigned long long*>(w.counters + jacobi_tmax_offset(ms));
		void* args[] = {&w.A0, &w.A1, &w.V, (void*)&kpv, &ms, &tol, &tau_final, &w.counters, &tmax};
		e = cudaLaunchCooperativeKernel((void*)jacobi_kernel, dim3(blocks), dim3(kThreads), args, 0, s);
		if (e != cudaSuccess) return e;
	}
	if (serial.owns_lock()) {
		e = cudaStreamSynchronize(s);
		serial.unlock();
		if (e != cudaSuccess) return e;
	}
	normalize_columns_kernel<<<(k + 31) / 32, 1024, 0, s>>>(w.V, k, kp);
	int P = 1;
	while (P < k) P <<= 1;
	const size_t smem = (size_t)P * (sizeof(double) + sizeof(int));
	if (smem > 48 * 1024) cudaFuncSetAttribute(eig_sort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
	eig_sort_kernel<<<1, 1024, smem, s>>>(w.A0, w.A1, w.A2, k, kp, w.counters, w.max_sweeps, w.evals, w.perm,
			st, check);
	return cudaGetLastError();
}

}  // namespace itp2d
