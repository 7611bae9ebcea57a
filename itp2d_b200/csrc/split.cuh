// Row / column pass kernels of the split-operator propagation and of the
// Hamiltonian used for energies.
#pragma once

#include "common.cuh"

namespace itp2d {

// One row pass over a k x sy x sx state array:
//   v = in[row]
//   if do_inv:  v = Tinv_x( mul_pre .* v )        (X table then inverse transform)
//   v = mul_mid .* v                              (potential exponential)
//   if do_fwd:  v = mul_post .* Tfwd_x(v)         (forward transform then X table)
//   out[row] = v (+ acc[row])
// Tables are [sy][sx] in the working precision; null pointers skip a multiply.
struct RowPassArgs {
	const void* in;
	void* out;
	const void* acc;
	const void* mul_pre;
	const void* mul_mid;
	const void* mul_post;
	int do_inv;
	int do_fwd;
	int sx, sy;
	long long G;
	int rows_per_tile;
	LinePlan lp;
};

// One column pass, in place:
//   mode 0: v = Tinv_y( mul .* Tfwd_y(v) ), mul = mul2d[y][x] or mul1d[y]
//   mode 1: v = Tfwd_y(v)      mode 2: v = Tinv_y(v)
struct ColPassArgs {
	void* data;
	const void* mul2d;
	const void* mul1d;
	int mode;
	int sx, sy;
	long long G;
	int cols_per_tile;
	LinePlan lp;
	// register-FFT column pass variant (rfft.cu): kColRegSmem stages tiles
	// through registers, kColTma by TMA (tune_col_pass_reg picks one per size)
	int variant = 0;
	int* err = nullptr;  // device status word for the TMA variant's bounded waits
};

enum { kColRegSmem = 0, kColTma = 1, kColVariants = 2 };

// Energy pass over rows, producing h = H psi pieces and per-tile sums.
//   src_t: array whose rows are transformed (psi or a partially transformed
//          scratch). if do_fwd: t = Tinv_x( tmul .* Tfwd_x(src_t) )
//          else: t = Tinv_x(src_t) (the column pass already multiplied).
//   h = t + V .* psi (V may be null) (+ add_in when non-null)
//   write h to h_out when non-null; when sums is non-null accumulate
//   <psi|h>, <h|h>, <h - Eshift psi|h - Eshift psi>, <psi|psi> per tile.
struct EnergyRowArgs {
	const void* src_t;
	const void* psi;
	const void* tmul;
	const void* V;
	void* h_out;
	double* sums;  // [k][ntiles][5]
	const double* Eshift;
	int do_fwd;
	int sx, sy;
	long long G;
	int rows_per_tile;
	LinePlan lp;
};

// Energy pass over columns (magnetic field): t = Tinv_y(ty .* Tfwd_y(src)),
// h = t + add_in; sums as above against psi. src null: src = psi.
struct EnergyColArgs {
	const void* src = nullptr;
	const void* psi;
	const void* add_in;
	const void* ty;
	void* h_out;
	double* sums;
	const double* Eshift;
	int sx, sy;
	long long G;
	int cols_per_tile;
	LinePlan lp;
};

// Row pass of the Dirichlet kinetic factor with a magnetic field, whose
// x-part maps a sine series to sines and cosines (expkinetic.cpp:108-133,
// 173-194; kinetic.cpp:66-80,126-138):
//   Xop(s) = iDSTx(x1 .* s) + iDCTx(shift(i x2 .* s)),
//   shift(u)[x] = u[x - 1] for x >= 1, shift(u)[0] = 0 (state.hpp:192-201).
//   v = in[row]
//   if lead_fwd: v = DSTx(v)
//   if do_inv:   v = Xop(v)                 (v arrives as a DSTx series)
//   v = mul_mid .* v                        (when non-null)
//   if do_fwd:   v = DSTx(Xop(DSTx(v)))     (start of the next kinetic factor)
//   out[row] = v (+ vadd .* in[row]) (+ acc[row])
// Tables are [sy][sx] in the working precision.
struct DmRowArgs {
	const void* in;
	void* out;
	const void* acc;
	const void* x1;
	const void* x2;
	const void* mul_mid;
	const void* vadd;
	int lead_fwd;
	int do_inv;
	int do_fwd;
	int sx, sy;
	long long G;
	int rows_per_tile;
	LinePlan lp_dst;  // x-lines, DST-II / DST-III
	LinePlan lp_dct;  // x-lines, DCT-II / DCT-III
};

template <class R> void launch_dm_row_pass(const DmRowArgs& a, int k, cudaStream_t s);
int dm_row_tile_rows(int sx, int elem_bytes, int sy);

template <class R> void launch_row_pass(const RowPassArgs& a, int k, const void* tw, cudaStream_t s);
// Register-FFT passes (rfft.cu) for periodic lines of 32..1024 points (powers
// of two); return false, launching nothing, for other lines.
template <class R> bool launch_row_pass_reg(const RowPassArgs& a, int k, cudaStream_t s);
template <class R> bool launch_col_pass_reg(const ColPassArgs& a, int k, cudaStream_t s);
// Times the register-FFT column pass variants of `a` (its data pointer is a
// scratch state array of k states, overwritten) and returns the fastest, or
// -1 if the size has no register path.
template <class R> int tune_col_pass_reg(ColPassArgs a, int k, cudaStream_t s);
// Register-FFT energy passes; they run when the tile size equals
// energy_row_tile_reg / energy_col_tile_reg (non-zero for supported lines).
int energy_row_tile_reg(const LinePlan& lp, int sy);
int energy_col_tile_reg(const LinePlan& lp, int sx);
template <class R> bool launch_energy_row_reg(const EnergyRowArgs& a, int k, cudaStream_t s);
template <class R> bool launch_energy_col_reg(const EnergyColArgs& a, int k, cudaStream_t s);
template <class R> void launch_col_pass(const ColPassArgs& a, int k, const void* tw, cudaStream_t s);
template <class R> void launch_energy_row(const EnergyRowArgs& a, int k, const void* tw, cudaStream_t s);
template <class R> void launch_energy_col(const EnergyColArgs& a, int k, const void* tw, cudaStream_t s);

// Per-state reduction of the energy partial sums into E, sigma and the
// residual deviation (deterministic order). normalize != 0 divides by
// <psi|psi> (Rayleigh quotients; used by the FP32 form, whose contractions
// leave norms exact only to FP32 accuracy).
// sums2 (may be null): tile sums of a second energy pass whose h is H(H psi);
// then <H^2> = <psi|H H psi> (complex) as operators.cpp:40-50 computes it,
// instead of |H psi|^2.
void launch_energy_finish(const double* sums, const double* sums2, int k, int ntiles, double dx2,
		const double* Eshift, int normalize,
		double* E, double* sigma, double* sigma_res, double* E_imag, cudaStream_t s);

// Tile sizes (rows or columns per CTA) for a line length L (complex entries).
int row_tile_rows(int L, int elem_bytes, int sy);
int col_tile_cols(int L, int elem_bytes, int sx);
size_t row_pass_smem(int L, int rows, int n_fft, int elem_bytes);
size_t col_pass_smem(int L, int cols, int n_fft, int elem_bytes);
// Shared memory of the persistent double-buffered row/column passes.
size_t pipe_smem(int L, int lines, int n_fft, int elem_bytes);

}  // namespace itp2d
