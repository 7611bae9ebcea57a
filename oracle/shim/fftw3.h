/*
 * Oracle-only substitute for the subset of the FFTW 3 API that the itp2d
 * reference sources call (transformer.cpp:97-151, transformer.hpp:132-158,
 * itp2d_common.hpp:51-61). This is test infrastructure: it lets the
 * unmodified reference hot-path sources compile into the CPU oracle when
 * libfftw3 is absent. The transforms follow FFTW's documented definitions:
 *
 *   FFTW_FORWARD (-1):  Y_k = sum_j X_j exp(-2 pi i j k / n)   (unnormalised)
 *   FFTW_BACKWARD (+1): Y_k = sum_j X_j exp(+2 pi i j k / n)   (unnormalised)
 *   FFTW_RODFT10 (DST-II):  Y_k = 2 sum_j X_j sin(pi (j+1/2)(k+1) / n)
 *   FFTW_RODFT01 (DST-III): Y_k = (-1)^k X_{n-1} + 2 sum_{j<n-1} X_j sin(pi (j+1)(k+1/2) / n)
 *   FFTW_REDFT10 (DCT-II):  Y_k = 2 sum_j X_j cos(pi (j+1/2) k / n)
 *   FFTW_REDFT01 (DCT-III): Y_k = X_0 + 2 sum_{j>0} X_j cos(pi j (k+1/2) / n)
 *
 * Multi-dimensional transforms are separable products of the 1-D ones, with
 * the row-major index convention of FFTW (last dimension contiguous).
 * Planner flags are accepted and ignored; wisdom calls are no-ops.
 */
#ifndef ITP2D_ORACLE_FFTW3_SHIM_H
#define ITP2D_ORACLE_FFTW3_SHIM_H

#include <stddef.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct itp2d_shim_plan_s* fftw_plan;

typedef enum {
	FFTW_R2HC = 0, FFTW_HC2R = 1, FFTW_DHT = 2,
	FFTW_REDFT00 = 3, FFTW_REDFT01 = 4, FFTW_REDFT10 = 5, FFTW_REDFT11 = 6,
	FFTW_RODFT00 = 7, FFTW_RODFT01 = 8, FFTW_RODFT10 = 9, FFTW_RODFT11 = 10
} fftw_r2r_kind;

typedef struct {
	int n;
	int is;
	int os;
} fftw_iodim;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)

#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_UNALIGNED (1U << 1)
#define FFTW_CONSERVE_MEMORY (1U << 2)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_WISDOM_ONLY (1U << 21)

void* fftw_malloc(size_t n);
void fftw_free(void* p);

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out,
		int sign, unsigned flags);
fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany,
		fftw_complex* in, const int* inembed, int istride, int idist,
		fftw_complex* out, const int* onembed, int ostride, int odist,
		int sign, unsigned flags);
fftw_plan fftw_plan_many_r2r(int rank, const int* n, int howmany,
		double* in, const int* inembed, int istride, int idist,
		double* out, const int* onembed, int ostride, int odist,
		const fftw_r2r_kind* kind, unsigned flags);
fftw_plan fftw_plan_guru_r2r(int rank, const fftw_iodim* dims,
		int howmany_rank, const fftw_iodim* howmany_dims,
		double* in, double* out, const fftw_r2r_kind* kind, unsigned flags);

void fftw_execute(const fftw_plan p);
void fftw_execute_dft(const fftw_plan p, fftw_complex* in, fftw_complex* out);
void fftw_execute_r2r(const fftw_plan p, double* in, double* out);
void fftw_destroy_plan(fftw_plan p);

int fftw_import_wisdom_from_file(FILE* f);
void fftw_export_wisdom_to_file(FILE* f);
void fftw_cleanup(void);

#ifdef __cplusplus
}
#endif

#endif /* ITP2D_ORACLE_FFTW3_SHIM_H */
