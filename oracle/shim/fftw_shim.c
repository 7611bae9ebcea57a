/*
 * Oracle-only implementation of the FFTW-API subset declared in fftw3.h.
 * Test infrastructure for compiling the itp2d reference sources into the CPU
 * oracle; never linked into the product.
 *
 * Complex transforms: self-sorting (Stockham) mixed-radix FFT, radices 4, 2,
 * 3, 5, 7 and a direct O(p^2) butterfly for any other prime factor. Twiddles
 * come from a per-length table exp(-2 pi i t / n) computed with long-double
 * sin/cos. Real-to-real kinds (DST-II/III, DCT-II/III, FFTW's RODFT10/01 and
 * REDFT10/01) are evaluated through a complex FFT of length 2n of an odd or
 * even extension of the line, which is exact in real arithmetic.
 */
#define _POSIX_C_SOURCE 200112L
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define SHIM_MAXDIMS 4

typedef struct {
	int n;
	int radix[64];
	int nradix;
	double* tw; /* 2*n doubles: cos, -sin of 2 pi t / n */
} cfft_t;

typedef struct itp2d_shim_plan_s {
	int is_r2r;
	int sign;
	int rank;
	fftw_iodim dims[SHIM_MAXDIMS];
	int kind[SHIM_MAXDIMS];
	int nloops;
	fftw_iodim loops[SHIM_MAXDIMS];
	cfft_t* eng[SHIM_MAXDIMS]; /* complex engine: length n (dft) or 2n (r2r) */
	double* ext[SHIM_MAXDIMS]; /* r2r: exp(-i pi m / (2n)), m = 0..2n */
	double* in;
	double* out;
} shim_plan;

static cfft_t* cfft_new(int n) {
	cfft_t* e = (cfft_t*)calloc(1, sizeof(cfft_t));
	int m = n, t;
	e->n = n;
	e->tw = (double*)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
	for (t = 0; t < n; t++) {
		long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)t / (long double)n;
		e->tw[2 * t] = (double)cosl(a);
		e->tw[2 * t + 1] = (double)(-sinl(a));
	}
	while (m > 1) {
		int p;
		if (m % 4 == 0) p = 4;
		else if (m % 2 == 0) p = 2;
		else {
			p = 3;
			while (m % p != 0) p += 2;
		}
		e->radix[e->nradix++] = p;
		m /= p;
	}
	return e;
}

static void cfft_free(cfft_t* e) {
	if (!e) return;
	free(e->tw);
	free(e);
}

/* In-place transform of x (n complex, interleaved) using scratch y (n complex).
 * sign = -1 forward, +1 backward. */
static void cfft_exec(const cfft_t* e, double* x, double* y, int sign) {
	const int n = e->n;
	const double* tw = e->tw;
	double* src = x;
	double* dst = y;
	int Ns = 1, s;
	double vr[64], vi[64];
	for (s = 0; s < e->nradix; s++) {
		const int R = e->radix[s];
		const int nR = n / R;
		const int step = n / (Ns * R);
		int j;
		for (j = 0; j < nR; j++) {
			const int k = j % Ns;
			const int idxD = (j / Ns) * Ns * R + k;
			int r, q;
			for (r = 0; r < R; r++) {
				const double ar = src[2 * (j + r * nR)];
				const double ai = src[2 * (j + r * nR) + 1];
				const int ti = ((k * r) % (Ns * R)) * step;
				const double wr = tw[2 * ti];
				const double wi = sign < 0 ? tw[2 * ti + 1] : -tw[2 * ti + 1];
				vr[r] = ar * wr - ai * wi;
				vi[r] = ar * wi + ai * wr;
			}
			if (R == 2) {
				dst[2 * idxD] = vr[0] + vr[1];
				dst[2 * idxD + 1] = vi[0] + vi[1];
				dst[2 * (idxD + Ns)] = vr[0] - vr[1];
				dst[2 * (idxD + Ns) + 1] = vi[0] - vi[1];
			} else if (R == 4) {
				/* multiply by -i (forward) or +i (backward) for the odd term */
				const double t0r = vr[0] + vr[2], t0i = vi[0] + vi[2];
				const double t1r = vr[0] - vr[2], t1i = vi[0] - vi[2];
				const double t2r = vr[1] + vr[3], t2i = vi[1] + vi[3];
				double t3r = vr[1] - vr[3], t3i = vi[1] - vi[3];
				double rr, ri;
				if (sign < 0) { rr = t3i; ri = -t3r; } else { rr = -t3i; ri = t3r; }
				t3r = rr; t3i = ri;
				dst[2 * idxD] = t0r + t2r;
				dst[2 * idxD + 1] = t0i + t2i;
				dst[2 * (idxD + Ns)] = t1r + t3r;
				dst[2 * (idxD + Ns) + 1] = t1i + t3i;
				dst[2 * (idxD + 2 * Ns)] = t0r - t2r;
				dst[2 * (idxD + 2 * Ns) + 1] = t0i - t2i;
				dst[2 * (idxD + 3 * Ns)] = t1r - t3r;
				dst[2 * (idxD + 3 * Ns) + 1] = t1i - t3i;
			} else {
				for (q = 0; q < R; q++) {
					double sr = 0.0, si = 0.0;
					for (r = 0; r < R; r++) {
						const int ti = ((r * q) % R) * nR;
						const double wr = tw[2 * ti];
						const double wi = sign < 0 ? tw[2 * ti + 1] : -tw[2 * ti + 1];
						sr += vr[r] * wr - vi[r] * wi;
						si += vr[r] * wi + vi[r] * wr;
					}
					dst[2 * (idxD + q * Ns)] = sr;
					dst[2 * (idxD + q * Ns) + 1] = si;
				}
			}
		}
		{
			double* t = src;
			src = dst;
			dst = t;
		}
		Ns *= R;
	}
	if (src != x) memcpy(x, src, sizeof(double) * 2 * (size_t)n);
}

void* fftw_malloc(size_t n) {
	void* p = NULL;
	if (posix_memalign(&p, 64, n ? n : 1) != 0) return NULL;
	return p;
}

void fftw_free(void* p) { free(p); }

static shim_plan* plan_new(void) { return (shim_plan*)calloc(1, sizeof(shim_plan)); }

static void plan_init_engines(shim_plan* p) {
	int d;
	for (d = 0; d < p->rank; d++) {
		const int n = p->dims[d].n;
		if (!p->is_r2r) {
			p->eng[d] = cfft_new(n);
		} else {
			int m;
			p->eng[d] = cfft_new(2 * n);
			p->ext[d] = (double*)malloc(sizeof(double) * 2 * (size_t)(2 * n + 1));
			for (m = 0; m <= 2 * n; m++) {
				long double a = 3.14159265358979323846264338327950288L * (long double)m / (long double)(2 * n);
				p->ext[d][2 * m] = (double)cosl(a);
				p->ext[d][2 * m + 1] = (double)(-sinl(a));
			}
		}
	}
}

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out, int sign, unsigned flags) {
	shim_plan* p = plan_new();
	(void)flags;
	p->is_r2r = 0;
	p->sign = sign;
	p->rank = 2;
	p->dims[0].n = n0; p->dims[0].is = n1; p->dims[0].os = n1;
	p->dims[1].n = n1; p->dims[1].is = 1; p->dims[1].os = 1;
	p->nloops = 0;
	p->in = (double*)in;
	p->out = (double*)out;
	plan_init_engines(p);
	return p;
}

/* Row-major strides for an advanced-interface plan (inembed/onembed NULL). */
static void fill_many_dims(shim_plan* p, int rank, const int* n, int howmany,
		int istride, int idist, int ostride, int odist) {
	int d;
	int ist = istride, ost = ostride;
	p->rank = rank;
	for (d = rank - 1; d >= 0; d--) {
		p->dims[d].n = n[d];
		p->dims[d].is = ist;
		p->dims[d].os = ost;
		ist *= n[d];
		ost *= n[d];
	}
	p->nloops = 1;
	p->loops[0].n = howmany;
	p->loops[0].is = idist;
	p->loops[0].os = odist;
}

fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany,
		fftw_complex* in, const int* inembed, int istride, int idist,
		fftw_complex* out, const int* onembed, int ostride, int odist,
		int sign, unsigned flags) {
	shim_plan* p = plan_new();
	(void)inembed; (void)onembed; (void)flags;
	p->is_r2r = 0;
	p->sign = sign;
	fill_many_dims(p, rank, n, howmany, istride, idist, ostride, odist);
	p->in = (double*)in;
	p->out = (double*)out;
	plan_init_engines(p);
	return p;
}

fftw_plan fftw_plan_many_r2r(int rank, const int* n, int howmany,
		double* in, const int* inembed, int istride, int idist,
		double* out, const int* onembed, int ostride, int odist,
		const fftw_r2r_kind* kind, unsigned flags) {
	shim_plan* p = plan_new();
	int d;
	(void)inembed; (void)onembed; (void)flags;
	p->is_r2r = 1;
	fill_many_dims(p, rank, n, howmany, istride, idist, ostride, odist);
	for (d = 0; d < rank; d++) p->kind[d] = (int)kind[d];
	p->in = in;
	p->out = out;
	plan_init_engines(p);
	return p;
}

fftw_plan fftw_plan_guru_r2r(int rank, const fftw_iodim* dims, int howmany_rank,
		const fftw_iodim* howmany_dims, double* in, double* out,
		const fftw_r2r_kind* kind, unsigned flags) {
	shim_plan* p = plan_new();
	int d;
	(void)flags;
	p->is_r2r = 1;
	p->rank = rank;
	for (d = 0; d < rank; d++) {
		p->dims[d] = dims[d];
		p->kind[d] = (int)kind[d];
	}
	p->nloops = howmany_rank;
	for (d = 0; d < howmany_rank; d++) p->loops[d] = howmany_dims[d];
	p->in = in;
	p->out = out;
	plan_init_engines(p);
	return p;
}

/* Real-to-real transform of one line (n real values in line[0..n)) through the
 * 2n-point complex engine. buf and scr each hold 2n complex values. */
static void r2r_line(const cfft_t* e, const double* ext, int kind, int n,
		double* line, double* buf, double* scr) {
	int j, m;
	const int n2 = 2 * n;
	memset(buf, 0, sizeof(double) * 2 * (size_t)n2);
	switch (kind) {
		case FFTW_RODFT10: /* DST-II: odd extension, forward FFT */
		case FFTW_REDFT10: { /* DCT-II: even extension, forward FFT */
			const double sgn = (kind == FFTW_RODFT10) ? -1.0 : 1.0;
			for (j = 0; j < n; j++) {
				buf[2 * j] = line[j];
				buf[2 * (n2 - 1 - j)] = sgn * line[j];
			}
			cfft_exec(e, buf, scr, -1);
			if (kind == FFTW_RODFT10) {
				/* Y_{m-1} = Re(i * exp(-i pi m/2n) * U_m) */
				for (m = 1; m <= n; m++) {
					const double ur = buf[2 * m], ui = buf[2 * m + 1];
					const double cr = ext[2 * m], ci = ext[2 * m + 1];
					const double pi_ = ur * ci + ui * cr; /* Im(c * U) */
					line[m - 1] = -pi_;
				}
			} else {
				for (m = 0; m < n; m++) {
					const double ur = buf[2 * m], ui = buf[2 * m + 1];
					const double cr = ext[2 * m], ci = ext[2 * m + 1];
					line[m] = ur * cr - ui * ci;
				}
			}
			break;
		}
		case FFTW_RODFT01: { /* DST-III */
			for (m = 1; m < n; m++) {
				const double x = 2.0 * line[m - 1];
				/* exp(+i pi m / 2n) = conj(ext[m]) */
				buf[2 * m] = x * ext[2 * m];
				buf[2 * m + 1] = -x * ext[2 * m + 1];
				buf[2 * (n2 - m)] = -x * ext[2 * m];
				buf[2 * (n2 - m) + 1] = -x * ext[2 * m + 1];
			}
			buf[2 * n] = 0.0;
			buf[2 * n + 1] = 2.0 * line[n - 1];
			cfft_exec(e, buf, scr, +1);
			for (m = 0; m < n; m++) line[m] = 0.5 * buf[2 * m + 1];
			break;
		}
		case FFTW_REDFT01: { /* DCT-III */
			buf[0] = 2.0 * line[0];
			for (m = 1; m < n; m++) {
				const double x = 2.0 * line[m];
				buf[2 * m] = x * ext[2 * m];
				buf[2 * m + 1] = -x * ext[2 * m + 1];
				buf[2 * (n2 - m)] = x * ext[2 * m];
				buf[2 * (n2 - m) + 1] = x * ext[2 * m + 1];
			}
			cfft_exec(e, buf, scr, +1);
			for (m = 0; m < n; m++) line[m] = 0.5 * buf[2 * m];
			break;
		}
		default:
			abort();
	}
}

/* Visit every index tuple over a list of (n, stride) pairs, calling fn with
 * the accumulated offset. */
typedef struct {
	int n[2 * SHIM_MAXDIMS];
	long st[2 * SHIM_MAXDIMS];
	int cnt;
} odo_t;

static void apply_dim(const shim_plan* p, int d, double* data) {
	odo_t o;
	int idx[2 * SHIM_MAXDIMS];
	int i, q;
	const int n = p->dims[d].n;
	const long st = p->dims[d].os;
	const cfft_t* e = p->eng[d];
	const int nl = p->is_r2r ? 2 * n : n;
	double* line = (double*)malloc(sizeof(double) * 2 * (size_t)nl);
	double* buf = (double*)malloc(sizeof(double) * 2 * (size_t)nl);
	double* scr = (double*)malloc(sizeof(double) * 2 * (size_t)nl);
	o.cnt = 0;
	for (i = 0; i < p->rank; i++)
		if (i != d) { o.n[o.cnt] = p->dims[i].n; o.st[o.cnt] = p->dims[i].os; o.cnt++; }
	for (i = 0; i < p->nloops; i++) { o.n[o.cnt] = p->loops[i].n; o.st[o.cnt] = p->loops[i].os; o.cnt++; }
	for (i = 0; i < o.cnt; i++) idx[i] = 0;
	for (;;) {
		long off = 0;
		for (i = 0; i < o.cnt; i++) off += (long)idx[i] * o.st[i];
		if (!p->is_r2r) {
			for (q = 0; q < n; q++) {
				line[2 * q] = data[2 * (off + q * st)];
				line[2 * q + 1] = data[2 * (off + q * st) + 1];
			}
			cfft_exec(e, line, scr, p->sign);
			for (q = 0; q < n; q++) {
				data[2 * (off + q * st)] = line[2 * q];
				data[2 * (off + q * st) + 1] = line[2 * q + 1];
			}
		} else {
			for (q = 0; q < n; q++) line[q] = data[off + q * st];
			r2r_line(e, p->ext[d], p->kind[d], n, line, buf, scr);
			for (q = 0; q < n; q++) data[off + q * st] = line[q];
		}
		/* advance odometer */
		for (i = 0; i < o.cnt; i++) {
			if (++idx[i] < o.n[i]) break;
			idx[i] = 0;
		}
		if (i == o.cnt) break;
	}
	free(line);
	free(buf);
	free(scr);
}

static void shim_execute(const shim_plan* p, double* in, double* out) {
	int d;
	if (in != out) {
		/* Out-of-place: not used by the reference; copy then transform. */
		abort();
	}
	/* Separable: transform the last (contiguous) dimension first, like a
	 * row-column decomposition. */
	for (d = p->rank - 1; d >= 0; d--) apply_dim(p, d, out);
}

void fftw_execute(const fftw_plan p) { shim_execute(p, p->in, p->out); }

void fftw_execute_dft(const fftw_plan p, fftw_complex* in, fftw_complex* out) {
	shim_execute(p, (double*)in, (double*)out);
}

void fftw_execute_r2r(const fftw_plan p, double* in, double* out) { shim_execute(p, in, out); }

void fftw_destroy_plan(fftw_plan p) {
	int d;
	if (!p) return;
	for (d = 0; d < p->rank; d++) {
		cfft_free(p->eng[d]);
		free(p->ext[d]);
	}
	free(p);
}

int fftw_import_wisdom_from_file(FILE* f) { (void)f; return 0; }
void fftw_export_wisdom_to_file(FILE* f) { (void)f; }
void fftw_cleanup(void) {}
