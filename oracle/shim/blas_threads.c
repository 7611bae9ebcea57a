/*
 * Oracle-only BLAS threading wrappers (see the policy note in cblas.h).
 * Test infrastructure: the CPU oracle and the reference CPU baseline. The
 * wrapped routines resolve to the OpenBLAS runtime that the oracle links.
 */
#include <omp.h>

typedef struct { double re, im; } oracle_z;

/* the OpenBLAS runtime's own entry points */
void cblas_zgemm(const int order, const int transa, const int transb, const int m, const int n, const int k,
		const void* alpha, const void* a, const int lda, const void* b, const int ldb, const void* beta, void* c,
		const int ldc);
void zheev_(char* jobz, char* uplo, const int* n, oracle_z* a, const int* lda, double* w, oracle_z* work,
		const int* lwork, double* rwork, int* info);
void openblas_set_num_threads(int n);

static int blas_threads = 1;

void oracle_set_blas_threads(int threads) { blas_threads = threads > 0 ? threads : 1; }
int oracle_get_blas_threads(void) { return blas_threads; }

static int enter(void) {
	const int n = omp_in_parallel() ? 1 : blas_threads;
	if (n > 1) openblas_set_num_threads(n);
	return n;
}

static void leave(int n) {
	if (n > 1) openblas_set_num_threads(1);
}

void oracle_cblas_zgemm(const int order, const int transa, const int transb, const int m, const int n, const int k,
		const void* alpha, const void* a, const int lda, const void* b, const int ldb, const void* beta, void* c,
		const int ldc) {
	const int t = enter();
	cblas_zgemm(order, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
	leave(t);
}

void oracle_zheev(char* jobz, char* uplo, const int* n, oracle_z* a, const int* lda, double* w, oracle_z* work,
		const int* lwork, double* rwork, int* info) {
	const int t = enter();
	zheev_(jobz, uplo, n, a, lda, w, work, lwork, rwork, info);
	leave(t);
}
