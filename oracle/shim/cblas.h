/*
 * Oracle-only CBLAS prototypes for the routines the itp2d reference sources
 * call (state.hpp:130-240, stateset.cpp:199-226, eigensolver.hpp:76-78).
 * Test infrastructure: the symbols resolve to the OpenBLAS runtime that ships
 * in this image; the oracle build links it by path.
 */
#ifndef ITP2D_ORACLE_CBLAS_SHIM_H
#define ITP2D_ORACLE_CBLAS_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

/* BLAS threading policy of the oracle (shim/blas_threads.c). The reference
 * calls ZGEMM (HighMem lincomb, stateset.cpp:216-224) and ZHEEV
 * (eigensolver.hpp:80-84) from one thread, outside its OpenMP loops, and the
 * level-1/2 routines from inside them. A BLAS built for OpenMP programs runs
 * the former on every core and the latter on one; the runtime linked here is
 * a pthreads OpenBLAS, so these two calls are routed through wrappers that
 * raise its thread count to oracle_blas_threads for the call (and only when
 * no OpenMP region is active), while everything else stays single-threaded
 * (OPENBLAS_NUM_THREADS=1). The renaming also applies to the reference's own
 * zheev_ declaration, which follows the cblas.h include (eigensolver.hpp:41-46). */
#define cblas_zgemm oracle_cblas_zgemm
#define zheev_ oracle_zheev
void oracle_set_blas_threads(int threads);
int oracle_get_blas_threads(void);

enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };

void cblas_zaxpy(const int n, const void* alpha, const void* x, const int incx, void* y, const int incy);
void cblas_zcopy(const int n, const void* x, const int incx, void* y, const int incy);
void cblas_zdscal(const int n, const double alpha, void* x, const int incx);
void cblas_zscal(const int n, const void* alpha, void* x, const int incx);
double cblas_dznrm2(const int n, const void* x, const int incx);
void cblas_zdotc_sub(const int n, const void* x, const int incx, const void* y, const int incy, void* dotc);
void cblas_zgemv(const enum CBLAS_ORDER order, const enum CBLAS_TRANSPOSE trans,
		const int m, const int n, const void* alpha, const void* a, const int lda,
		const void* x, const int incx, const void* beta, void* y, const int incy);
void cblas_zgemm(const enum CBLAS_ORDER order, const enum CBLAS_TRANSPOSE transa,
		const enum CBLAS_TRANSPOSE transb, const int m, const int n, const int k,
		const void* alpha, const void* a, const int lda, const void* b, const int ldb,
		const void* beta, void* c, const int ldc);

#ifdef __cplusplus
}
#endif

#endif /* ITP2D_ORACLE_CBLAS_SHIM_H */
