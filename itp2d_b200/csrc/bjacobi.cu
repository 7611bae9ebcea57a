// Block Jacobi eigensolver for the overlap matrix at large k.
//
// Same decomposition as the scalar kernel in jacobi.cu (and the same output
// conventions), organised for fewer grid-wide rounds: the padded index range
// is cut into blocks of BS, blocks are paired round-robin (k/BS - 1 rounds per
// sweep), and each round r has two phases:
//   1. one CTA per block pair sweeps the 2BS x 2BS Hermitian subproblem in
//      shared memory with cyclic Jacobi (CTA barriers only), leaving its
//      2BS x 2BS unitary Q_r in global memory and the rotated subproblem as
//      the diagonal pair block of A_r;
//   2. every other 2BS x 2BS block of A_r becomes Q_r^H A_{r-1} Q_r (row and
//      column pairs) and every slab of 2BS rows of V becomes V Q_r, both as
//      FP64 DMMA products staged in shared memory.
// The phases are pipelined: one grid barrier separates supersteps, and
// superstep t runs phase 1 of round t on one set of CTAs while the others run
// phase 2 of round t - 1. Phase 1 of round t therefore builds its subproblem
// itself: its diagonal blocks are parts of round t - 1's rotated subproblems
// (already in A_{t-1}), and its off-diagonal block (P', Q') is taken from
// Q_a^H A_{t-2}(a, b) Q_b for the round t - 1 pairs a, b that held P' and Q'.
// Three matrix buffers rotate (A_{t-2} read, A_{t-1} completed by phase 2,
// A_t's diagonal pair blocks written by phase 1) and Q alternates between two
// buffers.
// In every 16th round of an outer sweep (starting with the first) every
// subproblem gets one full inner sweep (all pairs of its 2BS indices, so every
// within-block pair is rotated at least once per outer sweep); in the other
// rounds only the BS x BS cross pairs (p in block P, q in block Q) are
// rotated, in BS inner rounds. Over an outer sweep every index pair is thus
// rotated at least once, a block-cyclic ordering of cyclic Jacobi. A rotation is applied when |A_pq| > tol sqrt(|A_pp A_qq|).
// Rotations whose relative off-diagonal |A_pq| / sqrt(|A_pp A_qq|) is at the
// rounding level of the phase-2 products (below 1e-13) do not count against
// convergence; the iteration stops after a sweep whose largest counted
// rotation tangent is below tau_final (3e-9 by default: quadratic convergence
// then leaves off-diagonal elements of order k * 1e-17 relative to the gaps).
#include <cooperative_groups.h>

#include "../../include/itp2d_gpu.h"
#include "contract.cuh"

namespace cg = cooperative_groups;

namespace itp2d {

namespace {

constexpr int BS = 16;        // block size
constexpr int MS = 32;        // subproblem size: two blocks
constexpr int NR = MS / 2;    // rotations per inner round
constexpr int LD = MS + 4;    // padded row length (doubles): conflict-free DMMA fragments
constexpr int PL = MS * LD;   // doubles per plane
// 512 threads, one CTA per SM: in an inner round, threads [0, 256) update the
// 256 2 x 2 blocks of M while threads [256, 512) rotate the columns of Q; the
// two halves of a phase-2 CTA work on separate products.
constexpr int kThreads = 512;
constexpr int kMThreads = NR * NR;
constexpr double kTauFinal = 3e-9;
// Rounds between full inner sweeps (within-block pairs rotated again); every
// 16th round measured best on k = 500 (fewer outer sweeps for little cost).
constexpr int kFullEvery = 16;
constexpr double kNoiseRel = 1e-13;  // relative off-diagonal treated as rounding noise

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
	asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
			: "+d"(d0), "+d"(d1)
			: "d"(a), "d"(b));
}

// Round-robin pairing of npos positions (circle method): position 0 fixed.
__device__ __forceinline__ int rr_player(int pos, int r, int npos) {
	return pos == 0 ? 0 : ((pos - 1 + r) % (npos - 1)) + 1;
}

// Global index of local subproblem index i (< 64) for the block pair (P, Q).
__device__ __forceinline__ int gidx(int i, int P, int Q) { return i < BS ? P * BS + i : Q * BS + (i - BS); }

struct Shared {
	// phase 1: [0,1] M, [2,3] Q, [4,5] formation operands; phase 2: half h of
	// the CTA uses [6h, 6h + 6): X/T, Q_r, Q_c
	double pl[12][PL];
	// rotations of two consecutive inner rounds (round r in buffer r & 1)
	double2 rst[2][NR];                          // (sin, tau)
	double2 re[2][NR];                           // e = c / |c|
	double rap[2][NR], raq[2][NR];               // M(p, p), M(q, q) after the round
	int rpq[2][NR];                              // p | q << 8 | applied << 16
	int next[2];  // phase-2 item of each CTA half
	int cnt;                                     // counted rotations of the current outer sweep
	unsigned long long tmax;                     // largest tangent (bits of a non-negative double)
};

// Reciprocal and reciprocal square root in double precision by Newton-Raphson
// refinement of the single-precision hardware estimates: each step squares the
// relative error (about 1e-7 -> 1e-14 -> below double rounding). Valid for
// positive normal arguments inside the float exponent range, which the
// rotation set-up below guarantees by scaling.
__device__ __forceinline__ double rcp_nr(double x) {
	double y = (double)__frcp_rn((float)x);
	y = y * fma(-x, y, 2.0);
	y = y * fma(-x, y, 2.0);
	return y;
}
__device__ __forceinline__ double rsqrt_nr(double x) {
	double y = (double)rsqrtf((float)x);
	y = y * fma(-0.5 * x * y, y, 1.5);
	y = y * fma(-0.5 * x * y, y, 1.5);
	return y;
}

// Exponent of a positive normal double, and 2^e for -1022 <= e <= 1023, by
// bit manipulation (exact).
__device__ __forceinline__ int exp2i(double x) { return (int)((__double_as_longlong(x) >> 52) & 0x7ff) - 1023; }
__device__ __forceinline__ double pow2i(int e) { return __longlong_as_double((long long)(e + 1023) << 52); }

// Rotation of the local pair (p, q) of the subproblem in planes (mr, mi).
// With d = (b - a) / 2, r = sqrt(d^2 + |c|^2), u = |d| + r and w = 2 r u, the
// rotation of the smaller angle has tan = |c| / u, cos = u / sqrt(w) and
// |sin| = |c| / sqrt(w) (cos^2 + sin^2 = (u^2 + |c|^2) / w = 1), and
// tau = sin / (1 + cos) = |c| / (sqrt(w) + u): three dependent Newton-refined
// reciprocal (square root) steps. d and c are scaled by the power of two of
// max(|d|, |c|), and c alone by its own for e = c / |c|, so that every refined
// estimate starts inside float range; exponents beyond +-1000 take the same
// formulas through scalbn.
// The pair has M(p, p) = a, M(q, q) = b, M(p, q) = (cr, ci); the rotation
// goes to rotation buffer buf, slot j. Counted rotations and the largest
// counted tangent accumulate in the caller's registers (cnt, tmax) and are
// reduced once per inner sweep.
__device__ __forceinline__ void inner_rotation(Shared& sh, int buf, int j, int p, int q, double a, double b,
		double cr, double ci, double tol, int& cnt, double& tmax) {
	const double c2 = cr * cr + ci * ci;
	const double scale2 = fabs(a) * fabs(b);
	sh.rap[buf][j] = a;
	sh.raq[buf][j] = b;
	sh.rpq[buf][j] = p | q << 8;
	if (!(c2 > 0.0 && c2 > tol * tol * scale2)) return;
	const double d = 0.5 * (b - a);
	const double ad = fabs(d);
	const double mc = fmax(fabs(cr), fabs(ci));
	const double m = fmax(ad, mc);
	int ex = exp2i(m), exc = exp2i(mc);
	const bool fast = ex > -1000 && ex < 1000 && exc > -1000 && exc < 1000;
	if (!fast) {
		ex = ilogb(m);
		exc = ilogb(mc);
	}
	const double sc = fast ? pow2i(-ex) : scalbn(1.0, -ex);
	const double scc = fast ? pow2i(-exc) : scalbn(1.0, -exc);
	// ratios in units of 2^ex: max(dn, |crn|, |cin|) in [1, 2)
	const double dn = ad * sc, crn = cr * sc, cin = ci * sc;
	const double cn2 = crn * crn + cin * cin;
	const double rn2 = dn * dn + cn2;         // [1, 12)
	const double rn = rn2 * rsqrt_nr(rn2);
	const double un = dn + rn;                // [1, 5.5)
	const double wn = 2.0 * rn * un;          // [2, 38)
	const double qn = rsqrt_nr(wn);
	const double cn = sqrt(cn2);
	const double t = cn * rcp_nr(un);
	if (t == 0.0) return;
	// e = c / |c| from c scaled by its own exponent: crs^2 + cis^2 in [1, 8)
	const double crs = cr * scc, cis = ci * scc;
	const double ec = rsqrt_nr(crs * crs + cis * cis);
	const double sg = d < 0 ? -1.0 : 1.0;
	const double sw = wn * qn;                 // sqrt(w)
	const double cabs = fast ? cn * pow2i(ex) : scalbn(cn, ex);
	sh.rst[buf][j] = make_double2(sg * cn * qn, sg * cn * rcp_nr(sw + un));  // sw + un in [2.4, 12)
	sh.re[buf][j] = make_double2(crs * ec, cis * ec);
	sh.rap[buf][j] = a - sg * t * cabs;
	sh.raq[buf][j] = b + sg * t * cabs;
	sh.rpq[buf][j] = p | q << 8 | 1 << 16;
	if (c2 > kNoiseRel * kNoiseRel * scale2) {
		cnt++;
		tmax = fmax(tmax, t);
	}
}

// Rotation j of an inner round from the subproblem in shared memory.
__device__ __forceinline__ void inner_rotation_sm(Shared& sh, int buf, int j, int p, int q, double tol, int& cnt,
		double& tmax) {
	const double* mr = sh.pl[0];
	const double* mi = sh.pl[1];
	inner_rotation(sh, buf, j, p, q, mr[p * LD + p], mr[q * LD + q], mr[p * LD + q], mi[p * LD + q], tol, cnt,
			tmax);
}

// Rows p, q of J^H X with J = [[c, s e], [-s conj(e), c]] (correction form,
// tau = s / (1 + c)).
__device__ __forceinline__ void rows2(double s, double tau, double er, double ei, double& xpr, double& xpi,
		double& xqr, double& xqi) {
	// yp = xp - s (e xq + tau xp)
	const double ypr = xpr - s * (er * xqr - ei * xqi + tau * xpr);
	const double ypi = xpi - s * (er * xqi + ei * xqr + tau * xpi);
	// yq = xq + s (conj(e) xp - tau xq)
	const double yqr = xqr + s * (er * xpr + ei * xpi - tau * xqr);
	const double yqi = xqi + s * (er * xpi - ei * xpr - tau * xqi);
	xpr = ypr; xpi = ypi; xqr = yqr; xqi = yqi;
}

// Columns s, t of X J (correction form, tau = s / (1 + c)).
__device__ __forceinline__ void cols2(double s, double tau, double er, double ei, double& xsr, double& xsi,
		double& xtr, double& xti) {
	// ys = xs - s (conj(e) xt + tau xs)
	const double ysr = xsr - s * (er * xtr + ei * xti + tau * xsr);
	const double ysi = xsi - s * (er * xti - ei * xtr + tau * xsi);
	// yt = xt + s (e xs - tau xt)
	const double ytr = xtr + s * (er * xsr - ei * xsi - tau * xtr);
	const double yti = xti + s * (er * xsi + ei * xsr - tau * xti);
	xsr = ysr; xsi = ysi; xtr = ytr; xti = yti;
}

// One inner sweep on the MS x MS subproblem in planes 0/1, accumulating Q in
// planes 2/3: full (MS - 1 rounds of NR rotations over all pairs) or cross
// (BS rounds: round r pairs p with BS + (p + r) % BS). Each round updates
// every 2 x 2 block {p,q} x {s,t} in place as J_pq^H X J_st (threads
// [0, 256)) while threads [256, 512) rotate the columns of Q, so the
// subproblem crosses shared memory once per round.
// In a cross sweep, round r + 1 pairs p with q' = BS + (p + r + 1) % BS, the
// second index of pair p + 1 in round r; so the thread updating the block
// (pair p, pair p + 1) of round r holds M(p, q') and finds M(p, p) and
// M(q', q') among round r's results, and sets up rotation p of round r + 1
// right away: one barrier per inner round.
__device__ void inner_sweep(Shared& sh, double tol, bool full) {
	double* mr = sh.pl[0];
	double* mi = sh.pl[1];
	double* qr = sh.pl[2];
	double* qi = sh.pl[3];
	const int tid = threadIdx.x;
	const int rounds = full ? MS - 1 : BS;
	int cnt = 0;
	double tmax = 0.0;
	if (tid < NR) {
		const int p = full ? rr_player(tid, 0, MS) : tid;
		const int q = full ? rr_player(MS - 1 - tid, 0, MS) : BS + tid;
		inner_rotation_sm(sh, 0, tid, p, q, tol, cnt, tmax);
	}
	__syncthreads();
	for (int r = 0; r < rounds; r++) {
		const int cur = r & 1;
		if (full && r > 0) {
			if (tid < NR)
				inner_rotation_sm(sh, cur, tid, rr_player(tid, r, MS), rr_player(MS - 1 - tid, r, MS), tol, cnt, tmax);
			__syncthreads();
		}
		if (tid < kMThreads) {
			const int ja = tid / NR, jb = tid % NR;
			const int pa = sh.rpq[cur][ja], pb = sh.rpq[cur][jb];
			const bool ra = pa >> 16, rb = pb >> 16;
			const bool nx = !full && r + 1 < rounds && jb == ((ja + 1) & (NR - 1));
			const int p = pa & 255, q = (pa >> 8) & 255, s2 = pb & 255, t2 = (pb >> 8) & 255;
			if (ja == jb) {
				if (ra) {
					mr[p * LD + p] = sh.rap[cur][ja]; mi[p * LD + p] = 0.0;
					mr[q * LD + q] = sh.raq[cur][ja]; mi[q * LD + q] = 0.0;
					mr[p * LD + q] = 0.0; mi[p * LD + q] = 0.0;
					mr[q * LD + p] = 0.0; mi[q * LD + p] = 0.0;
				}
			} else if (ra || rb || nx) {
				double psr = mr[p * LD + s2], psi = mi[p * LD + s2], ptr = mr[p * LD + t2], pti = mi[p * LD + t2];
				double qsr = mr[q * LD + s2], qsi = mi[q * LD + s2], qtr = mr[q * LD + t2], qti = mi[q * LD + t2];
				if (ra) {
					const double2 st = sh.rst[cur][ja], e = sh.re[cur][ja];
					rows2(st.x, st.y, e.x, e.y, psr, psi, qsr, qsi);
					rows2(st.x, st.y, e.x, e.y, ptr, pti, qtr, qti);
				}
				if (rb) {
					const double2 st = sh.rst[cur][jb], e = sh.re[cur][jb];
					cols2(st.x, st.y, e.x, e.y, psr, psi, ptr, pti);
					cols2(st.x, st.y, e.x, e.y, qsr, qsi, qtr, qti);
				}
				if (ra || rb) {
					mr[p * LD + s2] = psr; mi[p * LD + s2] = psi; mr[p * LD + t2] = ptr; mi[p * LD + t2] = pti;
					mr[q * LD + s2] = qsr; mi[q * LD + s2] = qsi; mr[q * LD + t2] = qtr; mi[q * LD + t2] = qti;
				}
				if (nx)
					inner_rotation(sh, cur ^ 1, ja, p, t2, sh.rap[cur][ja], sh.raq[cur][jb], ptr, pti, tol, cnt, tmax);
			}
		} else {
			for (int e = tid - kMThreads; e < MS * NR; e += kThreads - kMThreads) {
				const int i = e / NR, j = e % NR;
				const int pj = sh.rpq[cur][j];
				if (!(pj >> 16)) continue;
				const int p = pj & 255, q = (pj >> 8) & 255;
				double ysr = qr[i * LD + p], ysi = qi[i * LD + p], ytr = qr[i * LD + q], yti = qi[i * LD + q];
				const double2 st = sh.rst[cur][j], ev = sh.re[cur][j];
				cols2(st.x, st.y, ev.x, ev.y, ysr, ysi, ytr, yti);
				qr[i * LD + p] = ysr; qi[i * LD + p] = ysi; qr[i * LD + q] = ytr; qi[i * LD + q] = yti;
			}
		}
		__syncthreads();
	}
	// counts and tangents of every thread that set up rotations
	for (int o = 16; o > 0; o >>= 1) {
		cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
		tmax = fmax(tmax, __shfl_xor_sync(0xffffffffu, tmax, o));
	}
	if ((tid & 31) == 0 && cnt) {
		atomicAdd(&sh.cnt, cnt);
		atomicMax(&sh.tmax, (unsigned long long)__double_as_longlong(tmax));
	}
}

// One 8 x 8 tile of the complex product A B (32-deep operands given as plane
// pairs) by one warp with FP64 DMMA: acc (h) of lane holds output row
// row0 + (lane >> 2), column col0 + 2 (lane & 3) + h. A element (i, m) at
// a_re[i * as_i + m * as_m], B element (m, l) at b_re[m * LD + l]; conjA
// conjugates A.
__device__ __forceinline__ void ctile(int lane, const double* ar, const double* ai, int as_i, int as_m, bool conjA,
		const double* br, const double* bi, int row0, int col0, double (&cr)[2], double (&ci)[2]) {
	const int i = row0 + (lane >> 2);
	const int l = col0 + (lane >> 2);
	cr[0] = cr[1] = ci[0] = ci[1] = 0.0;
#pragma unroll
	for (int kk = 0; kk < MS; kk += 4) {
		const int m = kk + (lane & 3);
		const double far = ar[i * as_i + m * as_m];
		const double fai = conjA ? -ai[i * as_i + m * as_m] : ai[i * as_i + m * as_m];
		const double fbr = br[m * LD + l], fbi = bi[m * LD + l];
		dmma(cr[0], cr[1], far, fbr);
		dmma(cr[0], cr[1], -fai, fbi);
		dmma(ci[0], ci[1], far, fbi);
		dmma(ci[0], ci[1], fai, fbr);
	}
}

// Full 32 x 32 product on one half of the CTA (local warp lw of 8): warp lw
// owns rows (lw >> 1) * 8 .. + 8 and columns (lw & 1) * 16 .. + 16 (tiles b).
__device__ __forceinline__ void half_gemm(int lt, const double* ar, const double* ai, int as_i, int as_m,
		bool conjA, const double* br, const double* bi, double (&cr)[2][2], double (&ci)[2][2]) {
	const int lane = lt & 31, lw = lt >> 5;
#pragma unroll
	for (int b = 0; b < 2; b++)
		ctile(lane, ar, ai, as_i, as_m, conjA, br, bi, (lw >> 1) * 8, (lw & 1) * 16 + b * 8, cr[b], ci[b]);
}

// Output coordinates of accumulator (b, h) of half_gemm for local thread lt.
__device__ __forceinline__ void half_rc(int lt, int b, int h, int& row, int& col) {
	const int lane = lt & 31, lw = lt >> 5;
	row = (lw >> 1) * 8 + (lane >> 2);
	col = (lw & 1) * 16 + b * 8 + 2 * (lane & 3) + h;
}

// Barrier of one half of the CTA (named barrier 1 + half, 256 threads).
__device__ __forceinline__ void half_sync(int half) {
	asm volatile("bar.sync %0, %1;\n" ::"r"(1 + half), "r"(kThreads / 2) : "memory");
}

// Position of player p in round r of the circle method (inverse of rr_player).
__device__ __forceinline__ int rr_position(int p, int r, int npos) {
	if (p == 0) return 0;
	const int m = npos - 1;
	return ((p - 1 - r) % m + m) % m + 1;
}

// Phase 1 for pair j of round t (within-sweep round rr): forms the subproblem
// in planes 0/1 (Q in planes 2/3 = I), sweeps it, stores Q_t and the rotated
// subproblem. prev: A_{t-1} (diagonal pair blocks of round t - 1), prev2:
// A_{t-2}, Qprev: the Q buffer of round t - 1 (t >= 1). For t = 0 the
// subproblem is read from prev = A_{-1}, the initial matrix.
__device__ void phase1_item(Shared& sh, int j, long long t, int rounds, int nb, int np, int kp, double tol,
		const double2* prev, const double2* prev2, const double2* Qprev, double2* Qout, double2* out) {
	const int tid = threadIdx.x;
	const int rr = (int)(t % rounds);
	const int P = rr_player(j, rr, nb), Q = rr_player(nb - 1 - j, rr, nb);
	double* mr = sh.pl[0];
	double* mi = sh.pl[1];
	if (t == 0) {
		for (int e = tid; e < MS * MS; e += kThreads) {
			const int i = e / MS, l = e % MS;
			const double2 v = __ldcg(prev + (long long)gidx(i, P, Q) * kp + gidx(l, P, Q));
			mr[i * LD + l] = v.x;
			mi[i * LD + l] = v.y;
		}
	} else {
		// the round t - 1 pairs (a, b) holding P and Q, and the halves they sit in
		const int ro = (int)((t - 1) % rounds);
		const int posP = rr_position(P, ro, nb), posQ = rr_position(Q, ro, nb);
		const int a = posP < np ? posP : nb - 1 - posP, hP = posP < np ? 0 : 1;
		const int b = posQ < np ? posQ : nb - 1 - posQ, hQ = posQ < np ? 0 : 1;
		const int Pa = rr_player(a, ro, nb), Qa = rr_player(nb - 1 - a, ro, nb);
		const int Pb = rr_player(b, ro, nb), Qb = rr_player(nb - 1 - b, ro, nb);
		// all global loads of the formation at once: A_{t-2}(a, b), Q_a, Q_b
		// and the diagonal blocks (P, P), (Q, Q) of A_{t-1} (kept in registers);
		// then T = A_{t-2}(a, b) Q_b and C = Q_a^H T
		static_assert(MS * MS % kThreads == 0 && 2 * BS * BS % kThreads == 0, "formation tiling");
		constexpr int NL = MS * MS / kThreads, ND = 2 * BS * BS / kThreads;
		double2 la[NL], lqa[NL], lqb[NL], ld[ND];
#pragma unroll
		for (int it = 0; it < NL; it++) {
			const int e = it * kThreads + tid, i = e / MS, l = e % MS;
			la[it] = __ldcg(prev2 + (long long)gidx(i, Pa, Qa) * kp + gidx(l, Pb, Qb));
			lqa[it] = __ldcg(Qprev + (size_t)a * MS * MS + e);
			lqb[it] = __ldcg(Qprev + (size_t)b * MS * MS + e);
		}
#pragma unroll
		for (int it = 0; it < ND; it++) {
			const int e = it * kThreads + tid;
			const int half = e / (BS * BS), i = (e / BS) % BS, l = e % BS;
			const int g0 = (half ? Q : P) * BS;
			ld[it] = __ldcg(prev + (long long)(g0 + i) * kp + g0 + l);
		}
#pragma unroll
		for (int it = 0; it < NL; it++) {
			const int e = it * kThreads + tid, i = e / MS, l = e % MS;
			mr[i * LD + l] = la[it].x;
			mi[i * LD + l] = la[it].y;
			sh.pl[2][i * LD + l] = lqa[it].x;
			sh.pl[3][i * LD + l] = lqa[it].y;
			sh.pl[4][i * LD + l] = lqb[it].x;
			sh.pl[5][i * LD + l] = lqb[it].y;
		}
		__syncthreads();
		// only the (hP, hQ) quadrant of Q_a^H A_{t-2}(a, b) Q_b enters the
		// subproblem: T = A_{t-2}(a, b) Q_b[:, hQ half] (32 x 16: eight 8 x 8
		// tiles, warps 0-7), then C = Q_a[:, hP half]^H T (16 x 16: four tiles,
		// warps 0-3)
		{
			const int lane = tid & 31, warp = tid >> 5;
			double cr[2], ci[2];
			if (warp < 8)
				ctile(lane, sh.pl[0], sh.pl[1], LD, 1, false, sh.pl[4] + hQ * BS, sh.pl[5] + hQ * BS, (warp >> 1) * 8,
						(warp & 1) * 8, cr, ci);
			__syncthreads();
			if (warp < 8)
#pragma unroll
				for (int h = 0; h < 2; h++) {
					const int row = (warp >> 1) * 8 + (lane >> 2), col = (warp & 1) * 8 + 2 * (lane & 3) + h;
					mr[row * LD + col] = cr[h];
					mi[row * LD + col] = ci[h];
				}
			__syncthreads();
			if (warp < 4)
				ctile(lane, sh.pl[2] + hP * BS, sh.pl[3] + hP * BS, 1, LD, true, sh.pl[0], sh.pl[1], (warp >> 1) * 8,
						(warp & 1) * 8, cr, ci);
			__syncthreads();
			if (warp < 4)
#pragma unroll
				for (int h = 0; h < 2; h++) {
					const int i = (warp >> 1) * 8 + (lane >> 2), l = BS + (warp & 1) * 8 + 2 * (lane & 3) + h;
					mr[i * LD + l] = cr[h];
					mi[i * LD + l] = ci[h];
					mr[l * LD + i] = cr[h];
					mi[l * LD + i] = -ci[h];
				}
		}
		// diagonal blocks (P, P) and (Q, Q) of A_{t-1}
#pragma unroll
		for (int it = 0; it < ND; it++) {
			const int e = it * kThreads + tid;
			const int half = e / (BS * BS), i = (e / BS) % BS, l = e % BS;
			mr[(half * BS + i) * LD + half * BS + l] = ld[it].x;
			mi[(half * BS + i) * LD + half * BS + l] = ld[it].y;
		}
	}
	for (int e = tid; e < MS * MS; e += kThreads) {
		const int i = e / MS, l = e % MS;
		sh.pl[2][i * LD + l] = (i == l) ? 1.0 : 0.0;
		sh.pl[3][i * LD + l] = 0.0;
	}
	__syncthreads();
	inner_sweep(sh, tol, rr % kFullEvery == 0);
	double2* Qg = Qout + (size_t)j * MS * MS;
	for (int e = tid; e < MS * MS; e += kThreads) {
		const int i = e / MS, l = e % MS;
		Qg[e] = make_double2(sh.pl[2][i * LD + l], sh.pl[3][i * LD + l]);
		out[(long long)gidx(i, P, Q) * kp + gidx(l, P, Q)] = make_double2(mr[i * LD + l], mi[i * LD + l]);
	}
	__syncthreads();
}

// Phase 2 item w of round ro: an off-diagonal pair block of A (w < nA2) or a
// slab of V, read from src / V, written to dst / V; on one half of the CTA
// (the two halves take alternate items, each with its own planes and named
// barrier).
__device__ void phase2_item(Shared& sh, int half, int w, int ro, int nb, int np, int kp, const double2* src,
		double2* dst, double2* V, const double2* Qr) {
	const int lt = threadIdx.x & (kThreads / 2 - 1);
	double* xr = sh.pl[6 * half + 0];
	double* xi = sh.pl[6 * half + 1];
	double* ar = sh.pl[6 * half + 2];
	double* ai = sh.pl[6 * half + 3];
	double* br = sh.pl[6 * half + 4];
	double* bi = sh.pl[6 * half + 5];
	const int nA2 = np * (np - 1);
	constexpr int NH = MS * MS / (kThreads / 2);  // elements per thread and operand
	double cr[2][2], ci[2][2];
	if (w < nA2) {
		const int jr = w / (np - 1);
		int jc = w % (np - 1);
		if (jc >= jr) jc++;
		const int Pr = rr_player(jr, ro, nb), Qr_ = rr_player(nb - 1 - jr, ro, nb);
		const int Pc = rr_player(jc, ro, nb), Qc = rr_player(nb - 1 - jc, ro, nb);
		// all global loads of the item at once, then the shared-memory stores
		double2 lx[NH], la[NH], lb[NH];
#pragma unroll
		for (int it = 0; it < NH; it++) {
			const int e = it * (kThreads / 2) + lt, i = e / MS, l = e % MS;
			lx[it] = __ldcg(src + (long long)gidx(i, Pr, Qr_) * kp + gidx(l, Pc, Qc));
			la[it] = __ldcg(Qr + (size_t)jr * MS * MS + e);
			lb[it] = __ldcg(Qr + (size_t)jc * MS * MS + e);
		}
#pragma unroll
		for (int it = 0; it < NH; it++) {
			const int e = it * (kThreads / 2) + lt, o = (e / MS) * LD + e % MS;
			xr[o] = lx[it].x;
			xi[o] = lx[it].y;
			ar[o] = la[it].x;
			ai[o] = la[it].y;
			br[o] = lb[it].x;
			bi[o] = lb[it].y;
		}
		half_sync(half);
		half_gemm(lt, xr, xi, LD, 1, false, br, bi, cr, ci);  // T = X Qc
		half_sync(half);
#pragma unroll
		for (int b = 0; b < 2; b++)
#pragma unroll
			for (int h = 0; h < 2; h++) {
				int row, col;
				half_rc(lt, b, h, row, col);
				xr[row * LD + col] = cr[b][h];
				xi[row * LD + col] = ci[b][h];
			}
		half_sync(half);
		// C = Qr^H T: A(i, m) = conj(Qr(m, i))
		half_gemm(lt, ar, ai, 1, LD, true, xr, xi, cr, ci);
#pragma unroll
		for (int b = 0; b < 2; b++)
#pragma unroll
			for (int h = 0; h < 2; h++) {
				int row, col;
				half_rc(lt, b, h, row, col);
				dst[(long long)gidx(row, Pr, Qr_) * kp + gidx(col, Pc, Qc)] = make_double2(cr[b][h], ci[b][h]);
			}
	} else {
		const int v = w - nA2;
		const int rb = v / np, jc = v % np;
		const int Pc = rr_player(jc, ro, nb), Qc = rr_player(nb - 1 - jc, ro, nb);
		double2 lx[NH], lb[NH];
#pragma unroll
		for (int it = 0; it < NH; it++) {
			const int e = it * (kThreads / 2) + lt, i = e / MS, l = e % MS;
			lx[it] = __ldcg(V + (long long)(rb * MS + i) * kp + gidx(l, Pc, Qc));
			lb[it] = __ldcg(Qr + (size_t)jc * MS * MS + e);
		}
#pragma unroll
		for (int it = 0; it < NH; it++) {
			const int e = it * (kThreads / 2) + lt, o = (e / MS) * LD + e % MS;
			xr[o] = lx[it].x;
			xi[o] = lx[it].y;
			br[o] = lb[it].x;
			bi[o] = lb[it].y;
		}
		half_sync(half);
		half_gemm(lt, xr, xi, LD, 1, false, br, bi, cr, ci);  // V Qc
#pragma unroll
		for (int b = 0; b < 2; b++)
#pragma unroll
			for (int h = 0; h < 2; h++) {
				int row, col;
				half_rc(lt, b, h, row, col);
				V[(long long)(rb * MS + row) * kp + gidx(col, Pc, Qc)] = make_double2(cr[b][h], ci[b][h]);
			}
	}
	half_sync(half);
}

// Buffers: A_r lives in bufs[(r + 1) % 3] (A_{-1} = the input in A0); Q_r in
// Qbuf + (r & 1) * np * MS * MS.
__global__ void __launch_bounds__(kThreads, 1) bjacobi_kernel(double2* A0, double2* A1, double2* A2, double2* V,
		double2* Qbuf, int kp, int max_sweeps, double tol, double tau_final, int* counters,
		unsigned long long* tmax, int* p2ctr) {
	cg::grid_group grid = cg::this_grid();
	extern __shared__ __align__(16) unsigned char smem_raw[];
	Shared& sh = *reinterpret_cast<Shared*>(smem_raw);
	const int tid = threadIdx.x;
	const int nb = kp / BS;
	const int np = nb / 2;
	const int rounds = nb - 1;
	const int nrb = kp / MS;
	const int nW = np * (np - 1) + nrb * np;
	double2* const bufs[3] = {A0, A1, A2};
	const size_t qstride = (size_t)np * MS * MS;
	// CTAs [0, p1) take phase 1 items, the rest phase 2 items (all CTAs take
	// both kinds when the grid is not larger than the pair count)
	const bool split = (int)gridDim.x > np;
	const int p1 = split ? np : (int)gridDim.x;
	const int p2first = split ? np : 0;
	const int p2count = split ? (int)gridDim.x - np : (int)gridDim.x;
	// with many phase-2 items the phase-1 CTAs take items too once their own
	// subproblems are done (phase 2 is then the longer phase)
	const bool join = split && nW > 8 * p2count;

	if (tid == 0) {
		sh.cnt = 0;
		sh.tmax = 0ULL;
	}
	__syncthreads();

	int sweep = 0;
	bool stop = false, converged = false;
	long long t = 0;
	for (;;) {
		const bool do_p1 = !stop;  // phase 1 of round t
		// round t + 1's item counter (its last use, round t - 3, is complete)
		if (blockIdx.x == 0 && tid == 0) p2ctr[(t + 1) & 3] = 0;
		const bool do_p2 = t >= 1;  // phase 2 of round t - 1
		if (do_p1 && (int)blockIdx.x < p1) {
			const double2* prev = bufs[t % 3];
			const double2* prev2 = bufs[(t + 2) % 3];
			double2* out = bufs[(t + 1) % 3];
			for (int j = blockIdx.x; j < np; j += p1)
				phase1_item(sh, j, t, rounds, nb, np, kp, tol, prev, prev2, Qbuf + ((t + 1) & 1) * qstride,
						Qbuf + (t & 1) * qstride, out);
		}
		if (do_p2 && ((int)blockIdx.x >= p2first || join)) {
			const int ro = (int)((t - 1) % rounds);
			const double2* src = bufs[(t + 2) % 3];
			double2* dst = bufs[t % 3];
			// items handed out by the round's counter; the next index is fetched
			// while the current item is processed
			const int half = tid / (kThreads / 2), lt = tid & (kThreads / 2 - 1);
			int* ctr = p2ctr + ((t - 1) & 3);
			if (lt == 0) sh.next[half] = atomicAdd(ctr, 1);
			half_sync(half);
			int w = sh.next[half];
			while (w < nW) {
				int wn = 0;
				if (lt == 0) wn = atomicAdd(ctr, 1);
				phase2_item(sh, half, w, ro, nb, np, kp, src, dst, V, Qbuf + ((t + 1) & 1) * qstride);
				if (lt == 0) sh.next[half] = wn;
				half_sync(half);
				w = sh.next[half];
			}
		}
		const bool sweep_end = do_p1 && (t % rounds == rounds - 1);
		if (sweep_end && tid == 0) {
			if (sh.cnt) atomicAdd(&counters[sweep], sh.cnt);
			if (sh.tmax) atomicMax(&tmax[sweep], sh.tmax);
			sh.cnt = 0;
			sh.tmax = 0ULL;
		}
		grid.sync();
		if (!do_p1) break;  // that was the last phase 2
		if (sweep_end) {
			// uniform across the grid: the counters are final after grid.sync
			const int cnt = *((volatile int*)&counters[sweep]);
			const double tm = __longlong_as_double((long long)*((volatile unsigned long long*)&tmax[sweep]));
			if (cnt == 0 || tm < tau_final) {
				converged = true;
				stop = true;
			}
			sweep++;
			if (sweep >= max_sweeps) stop = true;
		}
		t++;
	}
	// the last round completed is t - 1; A_{t-1} lives in bufs[t % 3]
	if (blockIdx.x == 0 && tid == 0) {
		counters[max_sweeps] = converged ? sweep : -1;
		counters[max_sweeps + 1] = (int)(t % 3);
	}
}

}  // namespace

int bjacobi_padded(int k) { return ((k + MS - 1) / MS) * MS; }
size_t bjacobi_qbuf_elems(int k) { return 2 * (size_t)(bjacobi_padded(k) / MS) * MS * MS; }

cudaError_t launch_bjacobi(double2* A0, double2* A1, double2* A2, double2* V, double2* Qbuf, int kp,
		int max_sweeps, double tau_final, int* counters, int num_sms, cudaStream_t s) {
	const size_t smem = sizeof(Shared);
	cudaError_t e = cudaFuncSetAttribute(bjacobi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
	if (e != cudaSuccess) return e;
	int per_sm = 0;
	e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bjacobi_kernel, kThreads, smem);
	if (e != cudaSuccess) return e;
	if (per_sm < 1) return cudaErrorLaunchOutOfResources;
	const int blocks = num_sms * std::min(per_sm, 1);
	double tol = 1e-15;
	if (!(tau_final > 0.0)) tau_final = kTauFinal;
	unsigned long long* tmax = reinterpret_cast<unsigned long long*>(counters + jacobi_tmax_offset(max_sweeps));
	int* p2ctr = counters + jacobi_p2ctr_offset(max_sweeps);
	void* args[] = {&A0, &A1, &A2, &V, &Qbuf, &kp, &max_sweeps, &tol, &tau_final, &counters, &tmax, &p2ctr};
	return cudaLaunchCooperativeKernel((void*)bjacobi_kernel, dim3(blocks), dim3(kThreads), args, smem, s);
}

}  // namespace itp2d
