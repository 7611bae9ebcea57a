// Block-cooperative FFT / DST / DCT on lines staged in shared memory.
//
// A tile of `nlines` lines lives in shared memory; element e of line l is at
// l*lstride + e*estride (rows: estride 1, lstride L; column tiles: estride C,
// lstride 1). Complex FFTs use the self-sorting Stockham formulation with
// mixed radices 8, 4, 2, 3, 5, 7 (each stage reads src and writes dst, so
// two buffers ping-pong). The real-to-real kinds of the reference
// Transformer (FFTW RODFT10/RODFT01 = DST-II/III and REDFT10/REDFT01 =
// DCT-II/III, transformer.cpp:108-151) act on complex data directly through a
// 2N-point complex FFT of the odd (sine) or even (cosine) extension of each
// line; both transforms have real coefficients, so applying them to the
// complex line equals transforming Re and Im separately as the reference does.
#pragma once

#include "common.cuh"

namespace itp2d {

template <class T>
__device__ __forceinline__ void dft4(T* v, int sign) {
	const T t0 = cadd(v[0], v[2]);
	const T t1 = csub(v[0], v[2]);
	const T t2 = cadd(v[1], v[3]);
	const T t3 = cmul_i(csub(v[1], v[3]), sign);
	v[0] = cadd(t0, t2);
	v[1] = cadd(t1, t3);
	v[2] = csub(t0, t2);
	v[3] = csub(t1, t3);
}

template <class R>
__device__ __forceinline__ void dft8(c2<R>* v, int sign) {
	using T = c2<R>;
	const R s = (R)0.70710678118654752440;
	T b[4], c[4];
#pragma unroll
	for (int r = 0; r < 4; r++) {
		b[r] = cadd(v[r], v[r + 4]);
		c[r] = csub(v[r], v[r + 4]);
	}
	const R sg = sign < 0 ? (R)-1 : (R)1;
	c[1] = cmul(c[1], mk<R>(s, sg * s));
	c[2] = cmul_i(c[2], sign);
	c[3] = cmul(c[3], mk<R>(-s, sg * s));
	dft4(b, sign);
	dft4(c, sign);
	v[0] = b[0]; v[2] = b[1]; v[4] = b[2]; v[6] = b[3];
	v[1] = c[0]; v[3] = c[1]; v[5] = c[2]; v[7] = c[3];
}

// Direct DFT of odd prime size RD using roots from the length-n table.
template <class R, int RD>
__device__ __forceinline__ void dft_generic(c2<R>* v, const c2<R>* tw, int nR, int sign) {
	using T = c2<R>;
	T u[RD];
#pragma unroll
	for (int q = 0; q < RD; q++) {
		T acc = v[0];
#pragma unroll
		for (int r = 1; r < RD; r++) {
			T w = tw[((r * q) % RD) * nR];
			if (sign > 0) w.y = -w.y;
			acc = cadd(acc, cmul(v[r], w));
		}
		u[q] = acc;
	}
#pragma unroll
	for (int q = 0; q < RD; q++) v[q] = u[q];
}

template <class R, int RD, bool LINES_FAST>
__device__ __forceinline__ void stockham_stage(const c2<R>* __restrict__ src, c2<R>* __restrict__ dst,
		const c2<R>* tw, int n, int Ns, int nlines, int estride, int lstride, int sign) {
	using T = c2<R>;
	const int nR = n / RD;
	const int step = n / (Ns * RD);
	const int total = nlines * nR;
	for (int f = threadIdx.x; f < total; f += blockDim.x) {
		int line, j;
		if (LINES_FAST) {
			line = f % nlines;
			j = f / nlines;
		} else {
			j = f % nR;
			line = f / nR;
		}
		const T* in = src + line * lstride;
		T* out = dst + line * lstride;
		const int k = j % Ns;
		T v[RD];
		v[0] = in[j * estride];
#pragma unroll
		for (int r = 1; r < RD; r++) {
			const T a = in[(j + r * nR) * estride];
			T w = tw[k * r * step];
			if (sign > 0) w.y = -w.y;
			v[r] = cmul(a, w);
		}
		if (RD == 2) {
			const T a = v[0], b = v[1];
			v[0] = cadd(a, b);
			v[1] = csub(a, b);
		} else if (RD == 4) {
			dft4(v, sign);
		} else if (RD == 8) {
			dft8<R>(v, sign);
		} else {
			dft_generic<R, RD>(v, tw, nR, sign);
		}
		const int idxD = (j / Ns) * Ns * RD + k;
#pragma unroll
		for (int q = 0; q < RD; q++) out[(idxD + q * Ns) * estride] = v[q];
	}
}

// Complex FFT of every line (length p.n). sign -1: exp(-2 pi i jk/n) (FFTW
// forward), +1: backward, both unnormalised. Input in src; returns the buffer
// holding the result (src or dst). Ends with __syncthreads().
template <class R, bool LINES_FAST>
__device__ c2<R>* fft_lines(c2<R>* src, c2<R>* dst, const FftPlan& p, const c2<R>* tw, int nlines,
		int estride, int lstride, int sign) {
	int Ns = 1;
	for (int s = 0; s < p.nstages; s++) {
		const int rd = p.radix[s];
		switch (rd) {
			case 2: stockham_stage<R, 2, LINES_FAST>(src, dst, tw, p.n, Ns, nlines, estride, lstride, sign); break;
			case 3: stockham_stage<R, 3, LINES_FAST>(src, dst, tw, p.n, Ns, nlines, estride, lstride, sign); break;
			case 4: stockham_stage<R, 4, LINES_FAST>(src, dst, tw, p.n, Ns, nlines, estride, lstride, sign); break;
			case 5: stockham_stage<R, 5, LINES_FAST>(src, dst, tw, p.n, Ns, nlines, estride, lstride, sign); break;
			case 7: stockham_stage<R, 7, LINES_FAST>(src, dst, tw, p.n, Ns, nlines, estride, lstride, sign); break;
			default: stockham_stage<R, 8, LINES_FAST>(src, dst, tw, p.n, Ns, nlines, estride, lstride, sign); break;
		}
		__syncthreads();
		c2<R>* t = src;
		src = dst;
		dst = t;
		Ns *= rd;
	}
	return src;
}

// Forward (DFT forward / DST-II / DCT-II) or inverse (DFT backward / DST-III /
// DCT-III) transform of every line. The line data is in buf0[0, N) of each
// line; both buffers must hold L = N (kind 0) or 2N (kinds 1, 2) elements per
// line. Returns the buffer holding the N results. Ends with __syncthreads().
template <class R, bool LINES_FAST>
__device__ c2<R>* line_transform(c2<R>* buf0, c2<R>* buf1, const LinePlan& lp, const c2<R>* tw,
		int nlines, int estride, int lstride, bool inverse) {
	using T = c2<R>;
	if (lp.kind == 0)
		return fft_lines<R, LINES_FAST>(buf0, buf1, lp.fft, tw, nlines, estride, lstride, inverse ? 1 : -1);
	const int N = lp.N;
	const int N2 = 2 * N;
	const bool sine = lp.kind == 1;
	const T* ext = reinterpret_cast<const T*>(lp.ext);
	if (!inverse) {
		// odd (sine) or even (cosine) extension of length 2N
		for (int f = threadIdx.x; f < nlines * N; f += blockDim.x) {
			int line, j;
			if (LINES_FAST) { line = f % nlines; j = f / nlines; } else { j = f % N; line = f / N; }
			const T x = buf0[line * lstride + j * estride];
			buf1[line * lstride + j * estride] = x;
			buf1[line * lstride + (N2 - 1 - j) * estride] = sine ? mk<R>(-x.x, -x.y) : x;
		}
		__syncthreads();
		T* res = fft_lines<R, LINES_FAST>(buf1, buf0, lp.fft, tw, nlines, estride, lstride, -1);
		T* oth = (res == buf1) ? buf0 : buf1;
		// sine:   Y_{m-1} = i exp(-i pi m/2N) U_m, m = 1..N
		// cosine: Y_m     =   exp(-i pi m/2N) U_m, m = 0..N-1
		for (int f = threadIdx.x; f < nlines * N; f += blockDim.x) {
			int line, j;
			if (LINES_FAST) { line = f % nlines; j = f / nlines; } else { j = f % N; line = f / N; }
			const int m = sine ? j + 1 : j;
			const T u = res[line * lstride + m * estride];
			T y = cmul(u, __ldg(&ext[m]));
			if (sine) y = cmul_i(y, +1);
			oth[line * lstride + j * estride] = y;
		}
		__syncthreads();
		return oth;
	}
	// inverse: build V (length 2N) from x in buf0, backward FFT, scale.
	for (int f = threadIdx.x; f < nlines * N2; f += blockDim.x) {
		int line, m;
		if (LINES_FAST) { line = f % nlines; m = f / nlines; } else { m = f % N2; line = f / N2; }
		const T* x = buf0 + line * lstride;
		T v;
		if (sine) {
			if (m == 0) {
				v = mk<R>(0, 0);
			} else if (m < N) {
				const T e = __ldg(&ext[m]);  // exp(-i pi m/2N)
				v = cscale(cmulc(x[(m - 1) * estride], e), (R)2);  // 2 x exp(+i pi m/2N)
			} else if (m == N) {
				const T xv = x[(N - 1) * estride];
				v = mk<R>(-2 * xv.y, 2 * xv.x);  // 2i x
			} else {
				const int mm = N2 - m;
				const T e = __ldg(&ext[mm]);
				v = cscale(cmul(x[(mm - 1) * estride], e), (R)-2);  // -2 x exp(-i pi m'/2N)
			}
		} else {
			if (m == 0) {
				v = cscale(x[0], (R)2);
			} else if (m < N) {
				const T e = __ldg(&ext[m]);
				v = cscale(cmulc(x[m * estride], e), (R)2);
			} else if (m == N) {
				v = mk<R>(0, 0);
			} else {
				const int mm = N2 - m;
				const T e = __ldg(&ext[mm]);
				v = cscale(cmul(x[mm * estride], e), (R)2);
			}
		}
		buf1[line * lstride + m * estride] = v;
	}
	__syncthreads();
	T* res = fft_lines<R, LINES_FAST>(buf1, buf0, lp.fft, tw, nlines, estride, lstride, +1);
	T* oth = (res == buf1) ? buf0 : buf1;
	for (int f = threadIdx.x; f < nlines * N; f += blockDim.x) {
		int line, j;
		if (LINES_FAST) { line = f % nlines; j = f / nlines; } else { j = f % N; line = f / N; }
		const T y = res[line * lstride + j * estride];
		// sine: y / (2i) = -i y / 2; cosine: y / 2
		oth[line * lstride + j * estride] = sine ? cscale(cmul_i(y, -1), (R)0.5) : cscale(y, (R)0.5);
	}
	__syncthreads();
	return oth;
}

}  // namespace itp2d
