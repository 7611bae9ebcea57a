// Single-precision block Jacobi for the overlap matrix of the FP32 form.
//
// The FP32 form's overlap is accurate to about 1e-5 (split-BF16 tensor-core
// contraction) and its eigensolve stops at a largest rotation tangent of 1e-3,
// so FP64 arithmetic buys nothing there. This is the schedule of bjacobi.cu —
// round-robin pairs of 16-index blocks, 32 x 32 subproblems swept by one CTA
// per pair (k_p / 32 of them; cross pairs only except every 16th round),
// phase 1 of round t pipelined against phase 2 of round t - 1 (here on four
// 128-thread groups per CTA), one grid barrier per round — in single
// precision: the rotation set-up uses the hardware square root and reciprocal
// square root directly (no Newton refinement), and the block products are
// FFMA. Its latency chains are the short ones of FP32, which is what the
// latency-bound subproblem sweeps need.
//
// Accuracy: rotations are unitary to a few FP32 units, so the eigenvector
// matrix is orthonormal to about 1e-6; normalize_columns_kernel (jacobi.cu)
// renormalises its columns in FP64 afterwards. Rotations whose relative
// off-diagonal element is below 1e-7 are not applied, those below 1e-6 do not
// count toward convergence.
#include <cooperative_groups.h>

#include "../../include/itp2d_gpu.h"
#include "contract.cuh"

namespace cg = cooperative_groups;

namespace itp2d {

namespace {

constexpr int BS = 16;        // block size
constexpr int MS = 32;        // subproblem size: two blocks
constexpr int NR = MS / 2;    // rotations per inner round
// Row pitch 48 floats: rows p and p + 1 fall 16 banks apart, so the half-warps
// of the cross-pair updates (consecutive p, 16 consecutive columns) and of the
// block products (two consecutive rows per warp) never share a bank.
constexpr int LD = 48;
constexpr int PL = MS * LD;   // floats per plane
// 512 threads, one CTA per SM: in an inner round, threads [0, 256) update the
// 256 2 x 2 blocks of M while threads [256, 512) rotate the columns of Q.
constexpr int kThreads = 512;
constexpr int kMThreads = NR * NR;
// Phase 2 runs on four groups of 128 threads, each on its own block product:
// four DRAM-latency-bound products in flight per SM.
constexpr int kGroups = 4;
constexpr int kGT = kThreads / kGroups;
constexpr int kFullEvery = 16;
constexpr float kSkipRel = 1e-7f;
constexpr float kNoiseRel = 1e-6f;

__device__ __forceinline__ int rr_player(int pos, int r, int npos) {
	return pos == 0 ? 0 : ((pos - 1 + r) % (npos - 1)) + 1;
}

__device__ __forceinline__ int gidx(int i, int P, int Q) { return i < BS ? P * BS + i : Q * BS + (i - BS); }

struct Shared32 {
	// phase 1: [0,1] M, [2,3] Q, [4,5] formation operands; phase 2: group g
	// of the CTA uses [6g, 6g + 6): X/T, Q_r, Q_c
	float pl[6 * kGroups][PL];
	// rotations of two consecutive inner rounds (round r in buffer r & 1)
	float4 rot[2][NR];  // rotation j: (sin, tau, Re e, Im e)
	float rap[2][NR], raq[2][NR];  // M(p, p), M(q, q) after the round
	int rpq[2][NR];     // p | q << 8 | applied << 16
	int next[kGroups];  // phase-2 item of each thread group
	int cnt;
	unsigned long long tmax;  // bits of a non-negative double
};

// Rotation j of an inner round (into rotation buffer buf) of the local pair
// (p, q) with M(p, p) = a, M(q, q) = b, M(p, q) = (cr, ci): with
// d = (b - a) / 2, r = sqrt(d^2 + |c|^2), u = |d| + r and w = 2 r u:
// cos = u / sqrt(w), |sin| = |c| / sqrt(w), tau = |sin| / (1 + cos),
// tan = |c| / u (the formulas of bjacobi.cu).
__device__ __forceinline__ void inner_rotation32(Shared32& sh, int buf, int j, int p, int q, float a, float b,
		float cr, float ci, int& cnt, float& tmax) {
	const float c2 = cr * cr + ci * ci;
	const float scale2 = fabsf(a) * fabsf(b);
	if (!(c2 > 0.f && c2 > kSkipRel * kSkipRel * scale2)) {
		sh.rap[buf][j] = a;
		sh.raq[buf][j] = b;
		sh.rpq[buf][j] = p | q << 8;
		return;
	}
	const float d = 0.5f * (b - a);
	const float ad = fabsf(d);
	const float rn = sqrtf(fmaf(d, d, c2));
	const float un = ad + rn;
	const float wn = 2.f * rn * un;
	const float qn = rsqrtf(wn);
	const float cabs = sqrtf(c2);
	const float t = __fdividef(cabs, un);
	const float ic = rsqrtf(c2);
	const float sg = d < 0.f ? -1.f : 1.f;
	sh.rot[buf][j] = make_float4(sg * cabs * qn, sg * __fdividef(cabs, wn * qn + un), cr * ic, ci * ic);
	sh.rap[buf][j] = a - sg * t * cabs;
	sh.raq[buf][j] = b + sg * t * cabs;
	sh.rpq[buf][j] = p | q << 8 | 1 << 16;
	if (c2 > kNoiseRel * kNoiseRel * scale2) {
		cnt++;
		tmax = fmaxf(tmax, t);
	}
}

// Rotation j of an inner round from the subproblem in shared memory.
__device__ __forceinline__ void inner_rotation32_sm(Shared32& sh, int buf, int j, int p, int q, int& cnt,
		float& tmax) {
	const float* mr = sh.pl[0];
	const float* mi = sh.pl[1];
	inner_rotation32(sh, buf, j, p, q, mr[p * LD + p], mr[q * LD + q], mr[p * LD + q], mi[p * LD + q], cnt, tmax);
}

__device__ __forceinline__ void rows2f(float s, float tau, float er, float ei, float& xpr, float& xpi, float& xqr,
		float& xqi) {
	const float ypr = xpr - s * (er * xqr - ei * xqi + tau * xpr);
	const float ypi = xpi - s * (er * xqi + ei * xqr + tau * xpi);
	const float yqr = xqr + s * (er * xpr + ei * xpi - tau * xqr);
	const float yqi = xqi + s * (er * xpi - ei * xpr - tau * xqi);
	xpr = ypr; xpi = ypi; xqr = yqr; xqi = yqi;
}

__device__ __forceinline__ void cols2f(float s, float tau, float er, float ei, float& xsr, float& xsi, float& xtr,
		float& xti) {
	const float ysr = xsr - s * (er * xtr + ei * xti + tau * xsr);
	const float ysi = xsi - s * (er * xti - ei * xtr + tau * xsi);
	const float ytr = xtr + s * (er * xsr - ei * xsi - tau * xtr);
	const float yti = xti + s * (er * xsi + ei * xsr - tau * xti);
	xsr = ysr; xsi = ysi; xtr = ytr; xti = yti;
}

// One inner sweep (full: MS - 1 rounds over all pairs; cross: BS rounds of the
// BS x BS cross pairs, round r pairing p < BS with BS + (p + r) % BS) on the
// subproblem in planes 0/1, Q in planes 2/3. In each round the M blocks and
// the Q columns are rotated by separate threads at the same time.
// In a cross sweep, round r + 1 pairs p with q' = BS + (p + r + 1) % BS, the
// second index of pair p + 1 in round r; so the thread updating the block
// (pair p, pair p + 1) of round r holds M(p, q') and finds M(p, p) and
// M(q', q') among round r's results, and sets up rotation p of round r + 1
// right away: one barrier per inner round.
__device__ void inner_sweep32(Shared32& sh, bool full) {
	float* mr = sh.pl[0];
	float* mi = sh.pl[1];
	float* qr = sh.pl[2];
	float* qi = sh.pl[3];
	const int tid = threadIdx.x;
	const int rounds = full ? MS - 1 : BS;
	int cnt = 0;
	float tmax = 0.f;
	if (tid < NR) {
		const int p = full ? rr_player(tid, 0, MS) : tid;
		const int q = full ? rr_player(MS - 1 - tid, 0, MS) : BS + tid;
		inner_rotation32_sm(sh, 0, tid, p, q, cnt, tmax);
	}
	__syncthreads();
	for (int r = 0; r < rounds; r++) {
		const int cur = r & 1;
		if (full && r > 0) {
			if (tid < NR) inner_rotation32_sm(sh, cur, tid, rr_player(tid, r, MS), rr_player(MS - 1 - tid, r, MS), cnt,
					tmax);
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
					mr[p * LD + p] = sh.rap[cur][ja]; mi[p * LD + p] = 0.f;
					mr[q * LD + q] = sh.raq[cur][ja]; mi[q * LD + q] = 0.f;
					mr[p * LD + q] = 0.f; mi[p * LD + q] = 0.f;
					mr[q * LD + p] = 0.f; mi[q * LD + p] = 0.f;
				}
			} else if (ra || rb || nx) {
				float psr = mr[p * LD + s2], psi = mi[p * LD + s2], ptr = mr[p * LD + t2], pti = mi[p * LD + t2];
				float qsr = mr[q * LD + s2], qsi = mi[q * LD + s2], qtr = mr[q * LD + t2], qti = mi[q * LD + t2];
				if (ra) {
					const float4 R = sh.rot[cur][ja];
					rows2f(R.x, R.y, R.z, R.w, psr, psi, qsr, qsi);
					rows2f(R.x, R.y, R.z, R.w, ptr, pti, qtr, qti);
				}
				if (rb) {
					const float4 R = sh.rot[cur][jb];
					cols2f(R.x, R.y, R.z, R.w, psr, psi, ptr, pti);
					cols2f(R.x, R.y, R.z, R.w, qsr, qsi, qtr, qti);
				}
				if (ra || rb) {
					mr[p * LD + s2] = psr; mi[p * LD + s2] = psi; mr[p * LD + t2] = ptr; mi[p * LD + t2] = pti;
					mr[q * LD + s2] = qsr; mi[q * LD + s2] = qsi; mr[q * LD + t2] = qtr; mi[q * LD + t2] = qti;
				}
				if (nx)
					inner_rotation32(sh, cur ^ 1, ja, p, t2, sh.rap[cur][ja], sh.raq[cur][jb], ptr, pti, cnt, tmax);
			}
		} else {
			for (int e = tid - kMThreads; e < MS * NR; e += kThreads - kMThreads) {
				const int i = e / NR, j = e % NR;
				const int pj = sh.rpq[cur][j];
				if (!(pj >> 16)) continue;
				const int p = pj & 255, q = (pj >> 8) & 255;
				float ysr = qr[i * LD + p], ysi = qi[i * LD + p], ytr = qr[i * LD + q], yti = qi[i * LD + q];
				const float4 R = sh.rot[cur][j];
				cols2f(R.x, R.y, R.z, R.w, ysr, ysi, ytr, yti);
				qr[i * LD + p] = ysr; qi[i * LD + p] = ysi; qr[i * LD + q] = ytr; qi[i * LD + q] = yti;
			}
		}
		__syncthreads();
	}
	// counts and tangents of every thread that set up rotations
	for (int o = 16; o > 0; o >>= 1) {
		cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
		tmax = fmaxf(tmax, __shfl_xor_sync(0xffffffffu, tmax, o));
	}
	if ((tid & 31) == 0 && cnt) {
		atomicAdd(&sh.cnt, cnt);
		atomicMax(&sh.tmax, (unsigned long long)__double_as_longlong((double)tmax));
	}
}

// Complex products of 32-deep operands given as plane pairs, FFMA: the thread
// accumulates rows row0 + r * rstep (r < NRW) by columns col0 + c * cstep
// (c < NCL). A element (i, m) at a_re[i * as_i + m * as_m], B element (m, l)
// at b_re[m * LD + l]; conjA conjugates A.
template <int NRW, int NCL>
__device__ __forceinline__ void cmm32(const float* ar, const float* ai, int as_i, int as_m, bool conjA,
		const float* br, const float* bi, int row0, int rstep, int col0, int cstep, float (&cr)[NRW][NCL],
		float (&ci)[NRW][NCL]) {
#pragma unroll
	for (int r = 0; r < NRW; r++)
#pragma unroll
		for (int c = 0; c < NCL; c++) cr[r][c] = ci[r][c] = 0.f;
#pragma unroll 4
	for (int m = 0; m < MS; m++) {
		float xr[NRW], xi[NRW], yr[NCL], yi[NCL];
#pragma unroll
		for (int r = 0; r < NRW; r++) {
			const int o = (row0 + r * rstep) * as_i + m * as_m;
			xr[r] = ar[o];
			xi[r] = conjA ? -ai[o] : ai[o];
		}
#pragma unroll
		for (int c = 0; c < NCL; c++) {
			yr[c] = br[m * LD + col0 + c * cstep];
			yi[c] = bi[m * LD + col0 + c * cstep];
		}
#pragma unroll
		for (int r = 0; r < NRW; r++)
#pragma unroll
			for (int c = 0; c < NCL; c++) {
				cr[r][c] = fmaf(xr[r], yr[c], fmaf(-xi[r], yi[c], cr[r][c]));
				ci[r][c] = fmaf(xr[r], yi[c], fmaf(xi[r], yr[c], ci[r][c]));
			}
	}
}

// Group products of phase 2: thread lt of 128, warp lw = lt >> 5 owns rows
// 8 lw .. 8 lw + 7; lane (h, l) computes rows 8 lw + h + 2r at columns l + 16c.
__device__ __forceinline__ void group_rc(int lt, int r, int c, int& row, int& col) {
	const int lane = lt & 31, lw = lt >> 5;
	row = 8 * lw + (lane >> 4) + 2 * r;
	col = (lane & 15) + 16 * c;
}

__device__ __forceinline__ void group_gemm(int lt, const float* ar, const float* ai, int as_i, int as_m, bool conjA,
		const float* br, const float* bi, float (&cr)[4][2], float (&ci)[4][2]) {
	int row0, col0;
	group_rc(lt, 0, 0, row0, col0);
	cmm32<4, 2>(ar, ai, as_i, as_m, conjA, br, bi, row0, 2, col0, 16, cr, ci);
}

// Barrier of one thread group (named barrier 1 + g, 128 threads).
__device__ __forceinline__ void group_sync(int g) {
	asm volatile("bar.sync %0, %1;\n" ::"r"(1 + g), "r"(kGT) : "memory");
}

__device__ __forceinline__ int rr_position(int p, int r, int npos) {
	if (p == 0) return 0;
	const int m = npos - 1;
	return ((p - 1 - r) % m + m) % m + 1;
}

// Phase 1 for pair j of round t (bjacobi.cu phase1_item in FP32).
__device__ void phase1_item32(Shared32& sh, int j, long long t, int rounds, int nb, int np, int kp,
		const float2* prev, const float2* prev2, const float2* Qprev, float2* Qout, float2* out) {
	const int tid = threadIdx.x;
	const int rr = (int)(t % rounds);
	const int P = rr_player(j, rr, nb), Q = rr_player(nb - 1 - j, rr, nb);
	float* mr = sh.pl[0];
	float* mi = sh.pl[1];
	if (t == 0) {
		for (int e = tid; e < MS * MS; e += kThreads) {
			const int i = e / MS, l = e % MS;
			const float2 v = __ldcg(prev + (long long)gidx(i, P, Q) * kp + gidx(l, P, Q));
			mr[i * LD + l] = v.x;
			mi[i * LD + l] = v.y;
		}
	} else {
		const int ro = (int)((t - 1) % rounds);
		const int posP = rr_position(P, ro, nb), posQ = rr_position(Q, ro, nb);
		const int a = posP < np ? posP : nb - 1 - posP, hP = posP < np ? 0 : 1;
		const int b = posQ < np ? posQ : nb - 1 - posQ, hQ = posQ < np ? 0 : 1;
		const int Pa = rr_player(a, ro, nb), Qa = rr_player(nb - 1 - a, ro, nb);
		const int Pb = rr_player(b, ro, nb), Qb = rr_player(nb - 1 - b, ro, nb);
		constexpr int NL = MS * MS / kThreads, ND = 2 * BS * BS / kThreads;
		float2 la[NL], lqa[NL], lqb[NL], ldg[ND];
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
			ldg[it] = __ldcg(prev + (long long)(g0 + i) * kp + g0 + l);
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
		// subproblem: T = A_{t-2}(a, b) Q_b[:, hQ half] (32 x 16, one element per
		// thread), then C = Q_a[:, hP half]^H T (16 x 16, threads [0, 256))
		{
			const int lane = tid & 31, warp = tid >> 5;
			const int trow = 2 * warp + (lane >> 4), tcol = lane & 15;
			float tr[1][1], ti[1][1];
			cmm32<1, 1>(sh.pl[0], sh.pl[1], LD, 1, false, sh.pl[4], sh.pl[5], trow, 0, hQ * BS + tcol, 0, tr, ti);
			__syncthreads();
			mr[trow * LD + tcol] = tr[0][0];
			mi[trow * LD + tcol] = ti[0][0];
			__syncthreads();
			float cr[1][1], ci[1][1];
			const int i = (tid >> 4) & (BS - 1), l = tid & 15;
			if (tid < BS * BS)
				cmm32<1, 1>(sh.pl[2] + hP * BS, sh.pl[3] + hP * BS, 1, LD, true, sh.pl[0], sh.pl[1], i, 0, l, 0, cr,
						ci);
			__syncthreads();
			if (tid < BS * BS) {
				mr[i * LD + BS + l] = cr[0][0];
				mi[i * LD + BS + l] = ci[0][0];
				mr[(BS + l) * LD + i] = cr[0][0];
				mi[(BS + l) * LD + i] = -ci[0][0];
			}
		}
#pragma unroll
		for (int it = 0; it < ND; it++) {
			const int e = it * kThreads + tid;
			const int half = e / (BS * BS), i = (e / BS) % BS, l = e % BS;
			mr[(half * BS + i) * LD + half * BS + l] = ldg[it].x;
			mi[(half * BS + i) * LD + half * BS + l] = ldg[it].y;
		}
	}
	for (int e = tid; e < MS * MS; e += kThreads) {
		const int i = e / MS, l = e % MS;
		sh.pl[2][i * LD + l] = (i == l) ? 1.f : 0.f;
		sh.pl[3][i * LD + l] = 0.f;
	}
	__syncthreads();
	inner_sweep32(sh, rr % kFullEvery == 0);
	float2* Qg = Qout + (size_t)j * MS * MS;
	for (int e = tid; e < MS * MS; e += kThreads) {
		const int i = e / MS, l = e % MS;
		Qg[e] = make_float2(sh.pl[2][i * LD + l], sh.pl[3][i * LD + l]);
		out[(long long)gidx(i, P, Q) * kp + gidx(l, P, Q)] = make_float2(mr[i * LD + l], mi[i * LD + l]);
	}
	__syncthreads();
}

// Phase 2 item w of round ro (bjacobi.cu phase2_item in FP32), on one thread
// group of the CTA, with its own planes and named barrier.
__device__ void phase2_item32(Shared32& sh, int g, int w, int ro, int nb, int np, int kp, const float2* src,
		float2* dst, float2* V, const float2* Qr) {
	const int lt = threadIdx.x & (kGT - 1);
	float* xr = sh.pl[6 * g + 0];
	float* xi = sh.pl[6 * g + 1];
	float* ar = sh.pl[6 * g + 2];
	float* ai = sh.pl[6 * g + 3];
	float* br = sh.pl[6 * g + 4];
	float* bi = sh.pl[6 * g + 5];
	const int nA2 = np * (np - 1);
	constexpr int NH = MS * MS / kGT;  // elements per thread and operand
	float cr[4][2], ci[4][2];
	if (w < nA2) {
		const int jr = w / (np - 1);
		int jc = w % (np - 1);
		if (jc >= jr) jc++;
		const int Pr = rr_player(jr, ro, nb), Qr_ = rr_player(nb - 1 - jr, ro, nb);
		const int Pc = rr_player(jc, ro, nb), Qc = rr_player(nb - 1 - jc, ro, nb);
		// all global loads of the item at once, then the shared-memory stores
		float2 lx[NH], la[NH], lb[NH];
#pragma unroll
		for (int it = 0; it < NH; it++) {
			const int e = it * kGT + lt, i = e / MS, l = e % MS;
			lx[it] = __ldcg(src + (long long)gidx(i, Pr, Qr_) * kp + gidx(l, Pc, Qc));
			la[it] = __ldcg(Qr + (size_t)jr * MS * MS + e);
			lb[it] = __ldcg(Qr + (size_t)jc * MS * MS + e);
		}
#pragma unroll
		for (int it = 0; it < NH; it++) {
			const int e = it * kGT + lt, o = (e / MS) * LD + e % MS;
			xr[o] = lx[it].x;
			xi[o] = lx[it].y;
			ar[o] = la[it].x;
			ai[o] = la[it].y;
			br[o] = lb[it].x;
			bi[o] = lb[it].y;
		}
		group_sync(g);
		group_gemm(lt, xr, xi, LD, 1, false, br, bi, cr, ci);  // T = X Qc
		group_sync(g);
#pragma unroll
		for (int r = 0; r < 4; r++)
#pragma unroll
			for (int c = 0; c < 2; c++) {
				int row, col;
				group_rc(lt, r, c, row, col);
				xr[row * LD + col] = cr[r][c];
				xi[row * LD + col] = ci[r][c];
			}
		group_sync(g);
		group_gemm(lt, ar, ai, 1, LD, true, xr, xi, cr, ci);  // Qr^H T
#pragma unroll
		for (int r = 0; r < 4; r++)
#pragma unroll
			for (int c = 0; c < 2; c++) {
				int row, col;
				group_rc(lt, r, c, row, col);
				dst[(long long)gidx(row, Pr, Qr_) * kp + gidx(col, Pc, Qc)] = make_float2(cr[r][c], ci[r][c]);
			}
	} else {
		const int v = w - nA2;
		const int rb = v / np, jc = v % np;
		const int Pc = rr_player(jc, ro, nb), Qc = rr_player(nb - 1 - jc, ro, nb);
		float2 lx[NH], lb[NH];
#pragma unroll
		for (int it = 0; it < NH; it++) {
			const int e = it * kGT + lt, i = e / MS, l = e % MS;
			lx[it] = __ldcg(V + (long long)(rb * MS + i) * kp + gidx(l, Pc, Qc));
			lb[it] = __ldcg(Qr + (size_t)jc * MS * MS + e);
		}
#pragma unroll
		for (int it = 0; it < NH; it++) {
			const int e = it * kGT + lt, o = (e / MS) * LD + e % MS;
			xr[o] = lx[it].x;
			xi[o] = lx[it].y;
			br[o] = lb[it].x;
			bi[o] = lb[it].y;
		}
		group_sync(g);
		group_gemm(lt, xr, xi, LD, 1, false, br, bi, cr, ci);  // V Qc
#pragma unroll
		for (int r = 0; r < 4; r++)
#pragma unroll
			for (int c = 0; c < 2; c++) {
				int row, col;
				group_rc(lt, r, c, row, col);
				V[(long long)(rb * MS + row) * kp + gidx(col, Pc, Qc)] = make_float2(cr[r][c], ci[r][c]);
			}
	}
	group_sync(g);
}

// The cooperative solve: bjacobi_kernel of bjacobi.cu in FP32 (one CTA per SM). A_r lives in
// bufs[(r + 1) % 3] (A_{-1} = the input in A0); Q_r in Qbuf + (r & 1) * np * MS^2.
__global__ void __launch_bounds__(kThreads, 1) bjacobi32_kernel(float2* A0, float2* A1, float2* A2, float2* V,
		float2* Qbuf, int kp, int max_sweeps, double tau_final, int* counters, unsigned long long* tmaxg,
		int* p2ctr) {
	cg::grid_group grid = cg::this_grid();
	extern __shared__ __align__(16) unsigned char smem_raw[];
	Shared32& sh = *reinterpret_cast<Shared32*>(smem_raw);
	const int tid = threadIdx.x;
	const int nb = kp / BS;
	const int np = nb / 2;
	const int rounds = nb - 1;
	const int nrb = kp / MS;
	const int nW = np * (np - 1) + nrb * np;
	float2* const bufs[3] = {A0, A1, A2};
	const size_t qstride = (size_t)np * MS * MS;
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
		const bool do_p1 = !stop;
		// round t + 1's item counter (its last use, round t - 3, is complete)
		if (blockIdx.x == 0 && tid == 0) p2ctr[(t + 1) & 3] = 0;
		const bool do_p2 = t >= 1;
		if (do_p1 && (int)blockIdx.x < p1) {
			const float2* prev = bufs[t % 3];
			const float2* prev2 = bufs[(t + 2) % 3];
			float2* out = bufs[(t + 1) % 3];
			for (int j = blockIdx.x; j < np; j += p1)
				phase1_item32(sh, j, t, rounds, nb, np, kp, prev, prev2, Qbuf + ((t + 1) & 1) * qstride,
						Qbuf + (t & 1) * qstride, out);
		}
		if (do_p2 && ((int)blockIdx.x >= p2first || join)) {
			const int ro = (int)((t - 1) % rounds);
			const float2* src = bufs[(t + 2) % 3];
			float2* dst = bufs[t % 3];
			// items handed out by the round's counter; the next index is fetched
			// while the current item is processed
			const int g = tid / kGT, lt = tid & (kGT - 1);
			int* ctr = p2ctr + ((t - 1) & 3);
			if (lt == 0) sh.next[g] = atomicAdd(ctr, 1);
			group_sync(g);
			int w = sh.next[g];
			while (w < nW) {
				int wn = 0;
				if (lt == 0) wn = atomicAdd(ctr, 1);
				phase2_item32(sh, g, w, ro, nb, np, kp, src, dst, V, Qbuf + ((t + 1) & 1) * qstride);
				if (lt == 0) sh.next[g] = wn;
				group_sync(g);
				w = sh.next[g];
			}
		}
		const bool sweep_end = do_p1 && (t % rounds == rounds - 1);
		if (sweep_end && tid == 0) {
			if (sh.cnt) atomicAdd(&counters[sweep], sh.cnt);
			if (sh.tmax) atomicMax(&tmaxg[sweep], sh.tmax);
			sh.cnt = 0;
			sh.tmax = 0ULL;
		}
		grid.sync();
		if (!do_p1) break;
		if (sweep_end) {
			const int cnt = *((volatile int*)&counters[sweep]);
			const double tm = __longlong_as_double((long long)*((volatile unsigned long long*)&tmaxg[sweep]));
			if (cnt == 0 || tm < tau_final) {
				converged = true;
				stop = true;
			}
			sweep++;
			if (sweep >= max_sweeps) stop = true;
		}
		t++;
	}
	if (blockIdx.x == 0 && tid == 0) {
		counters[max_sweeps] = converged ? sweep : -1;
		counters[max_sweeps + 1] = (int)(t % 3);
	}
}

// S (k x k, FP64) into the FP32 work matrix A (kp x kp, zero padded) and V = I.
__global__ void narrow_init_kernel(const double2* __restrict__ S, int k, int kp, float2* A, float2* V) {
	const long long n = (long long)kp * kp;
	for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
			idx += (long long)gridDim.x * blockDim.x) {
		const int i = (int)(idx / kp), j = (int)(idx % kp);
		const double2 s = (i < k && j < k) ? S[(long long)i * k + j] : make_double2(0.0, 0.0);
		A[idx] = make_float2((float)s.x, (float)s.y);
		V[idx] = make_float2(i == j ? 1.f : 0.f, 0.f);
	}
}

// The FP32 result widened into the FP64 work matrices the sort and the W build
// read: the diagonal of the final A (all of it with full set) into A0 (whose
// result index becomes 0) and V into the FP64 V.
__global__ void widen_result_kernel(const float2* A0f, const float2* A1f, const float2* A2f, const float2* Vf,
		int kp, int* counters, int max_sweeps, double2* A0, double2* V, int full) {
	const int which = counters[max_sweeps + 1];
	const float2* A = which == 0 ? A0f : (which == 1 ? A1f : A2f);
	const long long n = (long long)kp * kp;
	for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
			idx += (long long)gridDim.x * blockDim.x) {
		const float2 v = Vf[idx];
		V[idx] = make_double2(v.x, v.y);
		const int i = (int)(idx / kp), j = (int)(idx % kp);
		if (full) A0[idx] = make_double2(A[idx].x, i == j ? 0.0 : A[idx].y);
		else if (i == j) A0[idx] = make_double2(A[idx].x, 0.0);
	}
}

__global__ void set_result_index_kernel(int* counters, int max_sweeps) { counters[max_sweeps + 1] = 0; }

}  // namespace

cudaError_t launch_bjacobi32(const double2* S, int k, JacobiWork& w, int num_sms, cudaStream_t s) {
	const int kp = bjacobi_padded(k);
	const long long n = (long long)kp * kp;
	const unsigned gblocks = (unsigned)std::min<long long>((n + 255) / 256, 4096);
	narrow_init_kernel<<<gblocks, 256, 0, s>>>(S, k, kp, w.f32.A0, w.f32.V);
	const size_t smem = sizeof(Shared32);
	cudaError_t e = cudaFuncSetAttribute(bjacobi32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
	if (e != cudaSuccess) return e;
	int per_sm = 0;
	e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bjacobi32_kernel, kThreads, smem);
	if (e != cudaSuccess) return e;
	if (per_sm < 1) return cudaErrorLaunchOutOfResources;
	const int blocks = num_sms * std::min(per_sm, 1);
	int kpv = kp, ms = w.max_sweeps;
	double tau = w.tau_final > 0.0 ? w.tau_final : 1e-3;
	int* counters = w.counters;
	unsigned long long* tmax = reinterpret_cast<unsigned long long*>(counters + jacobi_tmax_offset(ms));
	float2 *a0 = w.f32.A0, *a1 = w.f32.A1, *a2 = w.f32.A2, *v = w.f32.V, *q = w.f32.Qbuf;
	int* p2ctr = counters + jacobi_p2ctr_offset(ms);
	void* args[] = {&a0, &a1, &a2, &v, &q, &kpv, &ms, &tau, &counters, &tmax, &p2ctr};
	e = cudaLaunchCooperativeKernel((void*)bjacobi32_kernel, dim3(blocks), dim3(kThreads), args, smem, s);
	if (e != cudaSuccess) return e;
	widen_result_kernel<<<gblocks, 256, 0, s>>>(w.f32.A0, w.f32.A1, w.f32.A2, w.f32.V, kp, w.counters, ms, w.A0,
			w.V, w.full_result ? 1 : 0);
	set_result_index_kernel<<<1, 1, 0, s>>>(w.counters, ms);
	return cudaGetLastError();
}

}  // namespace itp2d
