// Orthonormalisation contractions and eigensolver entry points.
#pragma once

#include <cuda_runtime.h>

namespace itp2d {

int overlap_tiles(int k);
// Grid splits of the FP64 overlap for k states on G points.
int overlap_splits(int k, long long G, int num_sms);
// T = double2 (FP64 states) or float2 (FP32 states); products and sums in FP64.
// S = Psi^H Psib dx^2 from its upper triangle, mirrored Hermitian (psib null:
// Psi itself; otherwise Psib = H Psi for a Hermitian H).
template <class T>
void launch_overlap(const T* psi, int k, long long G, const int2* pairs, int npairs, int nsplit,
		double2* part, double dx2, double2* S, cudaStream_t s, const T* psib = nullptr);
// out = psi W (FP64 DMMA); upper: W is upper triangular (Cholesky), so output
// tile n reads only states i < n0 + 64.
template <class T>
void launch_rotate(const double2* W, const T* psi, int k, long long G, T* out, cudaStream_t s, bool upper = false);
// Sums the nsplit partial k x k blocks of part (upper triangle i <= j used),
// scales by dx2 and writes the full Hermitian S.
void launch_overlap_finish(const double2* part, int k, int nsplit, double dx2, double2* S, cudaStream_t s);

// Tensor-core (tcgen05, split-BF16, FP32 accumulation) contractions of FP32
// states; *err receives ITP2D_E_TIMEOUT if a bounded wait ran out.
bool tc_supported(int k, long long G);
int tc_overlap_splits(int k, long long G, int num_sms);
void launch_overlap_tc(const float2* psi, int k, long long G, int nsplit, double2* part, double dx2, double2* S,
		int* err, cudaStream_t s);
// wsplit: tc_wsplit_bytes(k) bytes of device scratch (W^T split into BF16 planes).
size_t tc_wsplit_bytes(int k);
void launch_rotate_tc(const double2* W, const float2* psi, int k, long long G, unsigned char* wsplit, float2* out,
		int* err, cudaStream_t s, bool upper = false);
// The same contractions from pre-split operands (split once per call into
// device scratch: tc_rows_bytes for the overlap, tc_cols_bytes for the
// rotation's psi), copied block by block by cp.async.bulk; bit-identical
// results to launch_overlap_tc / launch_rotate_tc.
size_t tc_rows_bytes(int k, long long G);
size_t tc_cols_bytes(int k, long long G);
void launch_overlap_tc_presplit(const float2* psi, int k, long long G, int nsplit, unsigned char* rows, double2* part,
		double dx2, double2* S, int* err, cudaStream_t s);
void launch_rotate_tc_presplit(const double2* W, const float2* psi, int k, long long G, unsigned char* wsplit,
		unsigned char* cols, float2* out, int* err, cudaStream_t s, bool upper = false);

template <class T>
void launch_normalize1(T* psi, long long G, double dx, double* tmp, cudaStream_t s);
// Converts n complex values between double2 (in_fp64 = 1) and float2.
void launch_convert(const void* in, int in_fp64, void* out, long long n, cudaStream_t s);

// Status block written by the eigensolver (device memory).
struct EigStatus {
	int status;      // 0 ok, ITP2D_E_* otherwise
	int bad_index;   // first offending eigenvalue (ascending order)
	int sweeps;      // Jacobi sweeps used
	int pad;
	double bad_value;
};

struct JacobiWork {
	double2* A0;      // k x k working matrix (input S, overwritten)
	double2* A1;      // k x k second buffer
	double2* V;       // k x k eigenvectors (columns)
	double* evals;    // k
	int* perm;        // k
	int* counters;    // jacobi_counter_ints(max_sweeps) ints
	int max_sweeps;
	double2* Qbuf = nullptr;  // block Jacobi unitaries (bjacobi_qbuf_elems); null: scalar Jacobi only
	double2* A2 = nullptr;    // third kp x kp buffer of the block path (required with Qbuf)
	// Stop after a sweep whose largest rotation tangent is below tau_final;
	// 0 selects the FP64 default of the kernel. The remaining off-diagonal
	// elements are then of order tau_final^2 relative to the eigenvalue gaps.
	double tau_final = 0.0;
	// FP32 block path (launch_bjacobi32): set, with k >= kBlockJacobiMinK, the
	// solve runs in single precision on these kp x kp buffers and widens its
	// result into A0 (diagonal) and V. They may alias A1, A2 and Qbuf, which
	// that path does not use otherwise; none may alias A0 or V.
	struct F32 {
		float2* A0 = nullptr;
		float2* A1 = nullptr;
		float2* A2 = nullptr;
		float2* V = nullptr;
		float2* Qbuf = nullptr;  // bjacobi_qbuf_elems(k) elements
	} f32;
	// FP32 block path: widen all of the final A into A0 (the rotated overlap
	// that launch_eig_cholesky_prep reads), not only its diagonal.
	bool full_result = false;
};

// Smallest k solved by block Jacobi (when JacobiWork::Qbuf is set).
constexpr int kBlockJacobiMinK = 256;
// Padded dimension of the block path (multiple of 32) and its Q buffer size
// (the unitaries of two rounds).
int bjacobi_padded(int k);
size_t bjacobi_qbuf_elems(int k);
// Padded dimension the eigensolver uses for (w, k); A0/A1/V are kp x kp.
int jacobi_kp(const JacobiWork& w, int k);
cudaError_t launch_bjacobi(double2* A0, double2* A1, double2* A2, double2* V, double2* Qbuf, int kp,
		int max_sweeps, double tau_final, int* counters, int num_sms, cudaStream_t s);
// Single-precision block Jacobi of S (k x k, FP64) on w.f32; leaves the
// eigenvalues on the diagonal of w.A0, the eigenvectors in w.V and the result
// fields of w.counters as the FP64 path does (result index 0).
cudaError_t launch_bjacobi32(const double2* S, int k, JacobiWork& w, int num_sms, cudaStream_t s);

// Eigen-decomposition of the Hermitian S (k x k, row-major, full storage) by
// parallel cyclic Jacobi, then W[:, n] = V[:, p(n)] / sqrt(l_n) with l
// ascending, and the eigenvalue checks of stateset.cpp:158-173. S is
// consumed. Returns a CUDA error code of the launches (status goes to *st).
cudaError_t launch_eigensolve(double2* S, int k, JacobiWork& w, double2* W, EigStatus* st, int num_sms,
		cudaStream_t s);
// Eigenvalues (ascending, w.evals), permutation (w.perm) and eigenvectors
// (columns of w.V, kp x kp with kp = k rounded up to even) without the
// overlap checks unless check != 0; check 2 also accepts a solve that ended
// at w.max_sweeps without converging (sweeps reported as w.max_sweeps).
cudaError_t launch_eigh(double2* S, int k, JacobiWork& w, EigStatus* st, int num_sms, cudaStream_t s, int check);
// Finish of a sweep-capped eigensolve (launch_eigh with check 2): with the
// order p(a) = perm[k - 1 - a] (descending eigenvalue), S_out[a][b] =
// A[p(a)][p(b)] (the final Jacobi matrix V^H S V, Hermitian part, k x k) and
// VT[a][i] = V[i][p(a)] (k x k), for W = V_p L^{-H} with S_out = L L^H.
cudaError_t launch_eig_cholesky_prep(const JacobiWork& w, int k, double2* S_out, double2* VT, cudaStream_t s);
// Rayleigh-Ritz: eigenpairs of the Hermitian H (k x k, consumed) with
// W[:, n] = V[:, p(n)] (unit columns, ascending eigenvalues in w.evals, any
// sign) for the rotation psi' = psi W.
cudaError_t launch_ritz(double2* H, int k, JacobiWork& w, double2* W, EigStatus* st, int num_sms, cudaStream_t s);

// FP64 rotation out_n[g] = sum_i W[i][n] psi_i[g] and overlap S = Psi^H Psi
// dx^2 on the int8 tensor cores (oz.cu): both operands split into 8 int8
// slices under per-row power-of-two scales, slice products accumulated
// exactly in 32 bits, combined in FP64. wsl (oz_w_bytes), scratch
// (oz_scratch_bytes) and ebuf (oz_exp_ints) are scratch; a bounded wait that
// gives up sets *err to ITP2D_E_TIMEOUT. upper: W upper triangular. The
// overlap writes nsplit (oz_overlap_splits, at most max_splits) partial
// blocks into part and sums them into S (launch_overlap_finish).
// oz_launches() kernels per call of either.
bool oz_supported(int k, long long G);
size_t oz_w_bytes(int k);
size_t oz_scratch_bytes(int k, long long G);
size_t oz_exp_ints(int k, long long G);
void launch_rotate_oz(const double2* W, const double2* psi, int k, long long G, unsigned char* wsl,
		unsigned char* scratch, int* ebuf, double2* out, int* err, cudaStream_t s, bool upper);
int oz_overlap_splits(int k, long long G, int num_sms, int max_splits);
void launch_overlap_oz(const double2* psi, int k, long long G, int nsplit, unsigned char* scratch, int* ebuf,
		double2* part, double dx2, double2* S, int* err, cudaStream_t s);
int oz_launches();

// Second-order Lowdin orthonormalisation (lowdin.cu): D = diag(S)^{-1/2},
// E = D S D - I (row-major) and conj(E), stats = {max |E_ij|, sum |E_ij|^2,
// bad diagonal}; then W = D (I - E/2 + 3/8 E^2) in the rotation layout, with
// E2 (k x k) as the product's scratch.
void launch_lowdin_prep(const double2* S, int k, double* D, double2* E, double2* Ec, double* stats,
		cudaStream_t s);
void launch_lowdin_w(const double* D, const double2* E, const double2* Ec, double2* E2, int k, double2* W,
		cudaStream_t s);
// Largest normalised off-diagonal overlap element and Frobenius norm for which
// a Lowdin step is taken: the series error 5/16 |E|^3 stays below 5e-3 in the
// worst case (|E|_2 <= |E|_F) and far below it for the noise-like E of
// near-converged states.
constexpr double kLowdinMaxElement = 0.05;
constexpr double kLowdinMaxFrobenius = 0.25;

// Cholesky orthonormalisation (cholesky.cu): W = L^{-H} with S = L L^H, in
// k x k buffers A (factor, overwritten) and X (inverse), Linv 32 x 32; st
// receives ITP2D_E_NONPOSITIVE_EIGENVALUE and the pivot on failure.
int launch_cholesky_w(const double2* S, int k, double2* A, double2* X, double2* Linv, double2* W, EigStatus* st,
		cudaStream_t s);
int cholesky_launches(int k);

// One instance of the batched eigensolver (batch.cu): the k x k overlap S
// (row-major), work matrices A and V ((k + 1) & ~1 squared), the result
// W = U Lambda^{-1/2} (rotation layout), ascending eigenvalues and their
// source indices, the status, and the tangent at which the sweeps stop.
struct BatchEigItem {
	const double2* S;
	double2* A;
	double2* V;
	double2* W;
	double* evals;
	int* perm;
	EigStatus* st;
	int k;
	int pad;
	double tau;
};
// max_k: the largest k among the items (sizes the shared-memory work area);
// next: a device int, the work queue's position (reset by the launch). Items
// in decreasing k balance the CTAs best.
cudaError_t launch_batched_eigensolve(const BatchEigItem* items, int n, int max_sweeps, int max_k, int* next,
		cudaStream_t s);
int batched_eigensolve_max_k();

// Users of the cooperative eigensolvers (contexts and the standalone
// eigensolve entry points). The Jacobi kernels are cooperative launches whose
// CTAs wait for each other at grid barriers; two of them on different streams
// could each hold part of the GPU while waiting for the rest. While more than
// one user is alive, launch_eigh therefore serialises the cooperative kernel
// process-wide and waits for it before returning.
void coop_user_enter();
void coop_user_leave();
struct CoopUser {
	CoopUser() { coop_user_enter(); }
	~CoopUser() { coop_user_leave(); }
	CoopUser(const CoopUser&) = delete;
	CoopUser& operator=(const CoopUser&) = delete;
};
// Counter block of the Jacobi kernel, in ints: per-sweep rotation counts, the
// result fields at [max_sweeps] and [max_sweeps + 1], then per-sweep maxima of
// the rotation tangents as 64-bit words starting at jacobi_tmax_offset(), then
// the four phase-2 item counters of the block path (round r in slot r & 3).
constexpr size_t jacobi_tmax_offset(int max_sweeps) { return ((size_t)max_sweeps + 4 + 1) & ~(size_t)1; }
constexpr size_t jacobi_p2ctr_offset(int max_sweeps) { return jacobi_tmax_offset(max_sweeps) + 2 * (size_t)max_sweeps + 2; }
constexpr size_t jacobi_counter_ints(int max_sweeps) { return jacobi_p2ctr_offset(max_sweeps) + 4; }
size_t jacobi_counters(int max_sweeps);

}  // namespace itp2d
