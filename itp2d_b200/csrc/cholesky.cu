// Cholesky (Gram-Schmidt order) orthonormalisation.
//
// With S = Psi^H Psi dx^2 Hermitian positive definite and S = L L^H its
// Cholesky factorisation (L lower triangular, real positive diagonal),
// W = L^{-H} is upper triangular and W^H S W = I: output state n is a
// combination of the input states 0..n only, the result of Gram-Schmidt in
// storage order. The eigendecomposition of the canonical form is replaced by
// about k^3 / 2 complex multiply-adds in three kinds of launches per panel of
// 32 columns:
//
//   1. one CTA factors the diagonal block S_jj = L_jj L_jj^H in shared memory
//      and inverts L_jj;
//   2. the panel below becomes L_21 = A_21 L_jj^{-H}, and the rows of the
//      running inverse X (L X = I, block forward substitution) that belong to
//      this panel become L_jj^{-1} X_j;
//   3. the trailing lower triangle takes A_22 -= L_21 L_21^H and the rows of X
//      below the panel take X_2 -= L_21 X_j (64 x 64 output tiles, FP64).
//
// Finally W[i k + n] = conj(X[n k + i]) for i <= n and 0 below. A pivot that
// is not a positive finite number stops the factorisation with
// ITP2D_E_NONPOSITIVE_EIGENVALUE (bad index = the pivot's row). No reference
// counterpart: the reference orthonormalises canonically (stateset.cpp:136-232).
#include "../../include/itp2d_gpu.h"
#include "contract.cuh"

#include <algorithm>

namespace itp2d {

namespace {

constexpr int NB = 32;   // panel width
constexpr int TU = 64;   // trailing-update output tile

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
	return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
	return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

// X = I (row-major k x k)
__global__ void chol_identity_kernel(double2* X, int k) {
	const long long n2 = (long long)k * k;
	for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += (long long)gridDim.x * blockDim.x)
		X[i] = make_double2(i / k == i % k ? 1.0 : 0.0, 0.0);
}

// Step 1: L_jj and L_jj^{-1} of the diagonal block at (j, j); 1024 threads.
__global__ void __launch_bounds__(1024) chol_diag_kernel(double2* A, int k, int j, double2* Linv, EigStatus* st) {
	__shared__ double2 L[NB][NB + 1];
	__shared__ double2 M[NB][NB + 1];
	if (st->status != 0) return;
	const int nb = min(NB, k - j);
	const int r = threadIdx.x / NB, c = threadIdx.x % NB;
	L[r][c] = (r < nb && c < nb && c <= r) ? A[(long long)(j + r) * k + j + c] : make_double2(0.0, 0.0);
	M[r][c] = make_double2(0.0, 0.0);
	for (int p = 0; p < nb; p++) {
		__syncthreads();
		const double pivot = L[p][p].x;
		if (!(pivot > 0.0) || !isfinite(pivot)) {
			if (threadIdx.x == 0) {
				st->status = ITP2D_E_NONPOSITIVE_EIGENVALUE;
				st->bad_index = j + p;
				st->bad_value = pivot;
			}
			return;  // every thread read the same pivot: the whole CTA leaves here
		}
		const double d = sqrt(pivot);
		__syncthreads();
		if (c == p && r >= p && r < nb) {
			const double2 v = L[r][p];
			L[r][p] = r == p ? make_double2(d, 0.0) : make_double2(v.x / d, v.y / d);
		}
		__syncthreads();
		if (c > p && r >= c && r < nb) L[r][c] = csub(L[r][c], cmulc(L[r][p], L[c][p]));
	}
	__syncthreads();
	if (r < nb && c <= r) A[(long long)(j + r) * k + j + c] = L[r][c];
	// L^{-1} column by column (one thread per column, forward substitution)
	if (threadIdx.x < nb) {
		const int col = threadIdx.x;
		for (int row = col; row < nb; row++) {
			double2 s = make_double2(row == col ? 1.0 : 0.0, 0.0);
			for (int m = col; m < row; m++) s = csub(s, cmul(L[row][m], M[m][col]));
			const double inv = 1.0 / L[row][row].x;
			M[row][col] = make_double2(s.x * inv, s.y * inv);
		}
	}
	__syncthreads();
	Linv[r * NB + c] = M[r][c];  // zero above the diagonal and beyond nb
}

// Step 2: blocks [0, nrb) turn 32 rows of the panel below the diagonal block
// into L_21 = A_21 L_jj^{-H}; blocks [nrb, ...) turn 32 columns of X's panel
// rows into L_jj^{-1} X_j. 256 threads.
__global__ void __launch_bounds__(256) chol_panel_kernel(double2* A, double2* X, int k, int j, const double2* Linv,
		int nrb, const EigStatus* st) {
	__shared__ double2 Li[NB][NB + 1];
	__shared__ double2 T[NB][NB + 1];
	if (st->status != 0) return;
	const int nb = min(NB, k - j), r0 = j + nb;
	for (int i = threadIdx.x; i < NB * NB; i += blockDim.x) Li[i / NB][i % NB] = Linv[i];
	if ((int)blockIdx.x < nrb) {
		const int row0 = r0 + NB * blockIdx.x;
		for (int i = threadIdx.x; i < NB * NB; i += blockDim.x) {
			const int rr = i / NB, p = i % NB, row = row0 + rr;
			T[rr][p] = (row < k && p < nb) ? A[(long long)row * k + j + p] : make_double2(0.0, 0.0);
		}
		__syncthreads();
		for (int i = threadIdx.x; i < NB * NB; i += blockDim.x) {
			const int rr = i / NB, q = i % NB, row = row0 + rr;
			if (row >= k || q >= nb) continue;
			double2 s = make_double2(0.0, 0.0);
			for (int p = 0; p <= q; p++) {
				const double2 a = T[rr][p], l = Li[q][p];
				s.x += a.x * l.x + a.y * l.y;  // a * conj(l)
				s.y += a.y * l.x - a.x * l.y;
			}
			A[(long long)row * k + j + q] = s;
		}
		return;
	}
	const int c0 = NB * (blockIdx.x - nrb);
	if (c0 >= j) {
		// the panel's own columns: X_j = L_jj^{-1} there (identity before)
		for (int i = threadIdx.x; i < NB * NB; i += blockDim.x) {
			const int q = i / NB, cc = i % NB;
			if (q < nb && cc < nb) X[(long long)(j + q) * k + j + cc] = Li[q][cc];
		}
		return;
	}
	for (int i = threadIdx.x; i < NB * NB; i += blockDim.x) {
		const int q = i / NB, cc = i % NB;
		T[q][cc] = q < nb ? X[(long long)(j + q) * k + c0 + cc] : make_double2(0.0, 0.0);
	}
	__syncthreads();
	for (int i = threadIdx.x; i < NB * NB; i += blockDim.x) {
		const int q = i / NB, cc = i % NB;
		if (q >= nb) continue;
		double2 s = make_double2(0.0, 0.0);
		for (int p = 0; p <= q; p++) {
			const double2 l = Li[q][p], x = T[p][cc];
			s.x += l.x * x.x - l.y * x.y;
			s.y += l.x * x.y + l.y * x.x;
		}
		X[(long long)(j + q) * k + c0 + cc] = s;
	}
}

// Step 3: rows [r0, k) of the trailing part. Column tiles [0, ncx) cover X's
// columns [0, r0) (X_2 -= L_21 X_j); the rest cover A's columns [r0, k)
// aligned with the row tiles (A_22 -= L_21 L_21^H, lower triangle only).
// 256 threads, 4 x 4 outputs each.
__global__ void __launch_bounds__(256) chol_update_kernel(double2* A, double2* X, int k, int j, int ncx,
		const EigStatus* st) {
	extern __shared__ __align__(16) unsigned char smem_raw[];
	double2(*Lt)[NB + 1] = reinterpret_cast<double2(*)[NB + 1]>(smem_raw);             // [TU][NB + 1]
	double2(*Bt)[TU + 1] = reinterpret_cast<double2(*)[TU + 1]>(smem_raw + sizeof(double2) * TU * (NB + 1));
	if (st->status != 0) return;
	const int nb = min(NB, k - j), r0 = j + nb;
	const int rt = blockIdx.y, ct = blockIdx.x;
	const bool xpart = ct < ncx;
	if (!xpart && ct - ncx > rt) return;  // strictly above the diagonal
	const int row0 = r0 + TU * rt;
	const int col0 = xpart ? TU * ct : r0 + TU * (ct - ncx);
	const int col_end = xpart ? r0 : k;
	for (int i = threadIdx.x; i < TU * NB; i += blockDim.x) {
		const int rr = i / NB, q = i % NB, row = row0 + rr;
		Lt[rr][q] = (row < k && q < nb) ? A[(long long)row * k + j + q] : make_double2(0.0, 0.0);
	}
	for (int i = threadIdx.x; i < TU * NB; i += blockDim.x) {
		const int q = i / TU, cc = i % TU, col = col0 + cc;
		double2 b = make_double2(0.0, 0.0);
		if (q < nb && col < col_end) {
			if (xpart) b = X[(long long)(j + q) * k + col];
			else {
				const double2 l = A[(long long)col * k + j + q];
				b = make_double2(l.x, -l.y);
			}
		}
		Bt[q][cc] = b;
	}
	__syncthreads();
	const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
	double2 acc[4][4];
#pragma unroll
	for (int a = 0; a < 4; a++)
#pragma unroll
		for (int b = 0; b < 4; b++) acc[a][b] = make_double2(0.0, 0.0);
	for (int q = 0; q < nb; q++) {
		double2 l[4], r[4];
#pragma unroll
		for (int a = 0; a < 4; a++) l[a] = Lt[ty + 16 * a][q];
#pragma unroll
		for (int b = 0; b < 4; b++) r[b] = Bt[q][tx + 16 * b];
#pragma unroll
		for (int a = 0; a < 4; a++)
#pragma unroll
			for (int b = 0; b < 4; b++) {
				acc[a][b].x += l[a].x * r[b].x - l[a].y * r[b].y;
				acc[a][b].y += l[a].x * r[b].y + l[a].y * r[b].x;
			}
	}
	double2* out = xpart ? X : A;
#pragma unroll
	for (int a = 0; a < 4; a++) {
		const int row = row0 + ty + 16 * a;
		if (row >= k) continue;
#pragma unroll
		for (int b = 0; b < 4; b++) {
			const int col = col0 + tx + 16 * b;
			if (col >= col_end || (!xpart && col > row)) continue;
			double2* o = out + (long long)row * k + col;
			*o = csub(*o, acc[a][b]);
		}
	}
}

// W[i k + n] = conj(X[n k + i]) for i <= n, 0 below (32 x 32 tiles through
// shared memory, coalesced both ways). 32 x 8 threads.
__global__ void chol_w_kernel(const double2* X, int k, double2* W, const EigStatus* st) {
	__shared__ double2 t[32][33];
	if (st->status != 0) return;
	const int bi = blockIdx.y * 32, bn = blockIdx.x * 32;  // W tile rows i, columns n
	for (int yy = threadIdx.y; yy < 32; yy += 8) {
		const int n = bn + yy, i = bi + threadIdx.x;
		t[yy][threadIdx.x] = (n < k && i < k) ? X[(long long)n * k + i] : make_double2(0.0, 0.0);
	}
	__syncthreads();
	for (int yy = threadIdx.y; yy < 32; yy += 8) {
		const int i = bi + yy, n = bn + threadIdx.x;
		if (i >= k || n >= k) continue;
		const double2 x = t[threadIdx.x][yy];
		W[(long long)i * k + n] = i <= n ? make_double2(x.x, -x.y) : make_double2(0.0, 0.0);
	}
}

}  // namespace

size_t cholesky_update_smem() { return sizeof(double2) * (TU * (NB + 1) + NB * (TU + 1)); }

int launch_cholesky_w(const double2* S, int k, double2* A, double2* X, double2* Linv, double2* W, EigStatus* st,
		cudaStream_t s) {
	static bool attr = false;
	if (!attr) {
		if (cudaFuncSetAttribute(chol_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
				    (int)cholesky_update_smem()) != cudaSuccess)
			return ITP2D_E_CUDA;
		attr = true;
	}
	cudaError_t e = cudaMemsetAsync(st, 0, sizeof(EigStatus), s);
	if (e == cudaSuccess) e = cudaMemcpyAsync(A, S, (size_t)k * k * sizeof(double2), cudaMemcpyDeviceToDevice, s);
	if (e != cudaSuccess) return ITP2D_E_CUDA;
	chol_identity_kernel<<<std::min(1184, (int)(((long long)k * k + 255) / 256)), 256, 0, s>>>(X, k);
	for (int j = 0; j < k; j += NB) {
		const int nb = std::min(NB, k - j), r0 = j + nb;
		chol_diag_kernel<<<1, 1024, 0, s>>>(A, k, j, Linv, st);
		const int nrb = (k - r0 + NB - 1) / NB, ncb = (r0 + NB - 1) / NB;
		chol_panel_kernel<<<nrb + ncb, 256, 0, s>>>(A, X, k, j, Linv, nrb, st);
		if (r0 < k) {
			const int nrt = (k - r0 + TU - 1) / TU, ncx = (r0 + TU - 1) / TU;
			chol_update_kernel<<<dim3(ncx + nrt, nrt), 256, cholesky_update_smem(), s>>>(A, X, k, j, ncx, st);
		}
	}
	const int nt = (k + 31) / 32;
	chol_w_kernel<<<dim3(nt, nt), dim3(32, 8), 0, s>>>(X, k, W, st);
	return cudaGetLastError() == cudaSuccess ? ITP2D_OK : ITP2D_E_CUDA;
}

int cholesky_launches(int k) { return 2 + 3 * ((k + NB - 1) / NB); }

}  // namespace itp2d
