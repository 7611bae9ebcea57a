// Context and C ABI (include/itp2d_gpu.h) of the itp2d B200 hot path.
//
// Host-side plan building, table construction and the launch sequences of the
// three seams. Tables are computed on the host in double precision with the
// same formulas as the reference (ExpPotential exppotential.cpp:55-63,
// ExpKinetic expkinetic.cpp:65-136, Kinetic kinetic.cpp:25-83, Transformer
// k-tables and normalisations transformer.cpp:66-90) and uploaded once per
// time step.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <tuple>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/itp2d_gpu.h"
#include "common.cuh"
#include "contract.cuh"
#include "split.cuh"

using namespace itp2d;

namespace {

enum Phase { kPropagate = 0, kOverlap = 1, kEigen = 2, kRotate = 3, kEnergies = 4 };

struct DevBuf {
	void* p = nullptr;
	size_t n = 0;
};

struct MemberTables {
	double c = 1.0;        // multi-product coefficient c_t
	int t = 1;             // exponent (member index)
	void* vh = nullptr;    // exp(-eps_t V / 2)
	void* vp = nullptr;    // c_t exp(-eps_t V / 2)
	void* vsq = nullptr;   // exp(-eps_t V)
	void* kmul = nullptr;  // B = 0: 2-D kinetic multiplier
	void* kx = nullptr;    // B != 0: X(k_x, y) (Dirichlet: the cosh part)
	void* kx2 = nullptr;   // Dirichlet, B != 0: the sinh part of X
	void* ky = nullptr;    // B != 0: Y(k_y)
};

struct PlanStore {
	LinePlan lp{};
	void* tw = nullptr;
	void* ext = nullptr;
	bool ready = false;
};

}  // namespace

struct itp2d_ctx {
	std::mutex mu;
	int sx = 0, sy = 0, k = 0, boundary = 0, halforder = 1, m = 1, precision = 0;
	double dx = 0, B = 0, eps = 0;
	long long G = 0;
	size_t es = 16;  // bytes per complex element
	cudaStream_t stream = nullptr;
	bool own_stream = false;
	int num_sms = 148;
	void* psi = nullptr;
	void* acc = nullptr;
	void* work = nullptr;
	std::vector<double> V;
	bool null_pot = true;
	bool eps_set = false;
	PlanStore planstore[2][2][3];  // [precision][axis x=0/y=1][kind]
	std::vector<void*> table_allocs;  // tables (room for doubles; refilled in the working precision)
	std::vector<MemberTables> members;
	void* eV = nullptr;     // potential in working precision (energies)
	void* eT2 = nullptr;    // B = 0: 0.5 k^2 norm
	void* eTx = nullptr;    // B != 0: 0.5 (k_x - B y)^2 / sx
	void* eTy = nullptr;    // B != 0: 0.5 k_y^2 / sy
	void* eTx2 = nullptr;   // Dirichlet, B != 0: B y k_x normalisation (first-derivative part)
	// orthonormalisation
	double2* S = nullptr;
	double2* part = nullptr;
	double2* W = nullptr;
	int2* pairs = nullptr;
	int npairs = 0, nsplit = 1;
	JacobiWork jw{};
	EigStatus* dstat = nullptr;
	EigStatus* hstat = nullptr;
	double* dnorm = nullptr;
	int last_sweeps = 0;
	long long sweeps_total = 0;
	long long sweeps_p[2] = {0, 0};  // by precision: FP64, FP32
	int engine = ITP2D_CONTRACT_AUTO;
	unsigned char* tc_rows = nullptr;  // FP32 states pre-split for the overlap (allocated on first use)
	unsigned char* tc_cols = nullptr;  // and for the rotation's B operand
	bool tc_staged = false;            // pre-split scratch unavailable: split inside the contraction CTAs
	int tc_nsplit = 1;  // grid chunks of the tensor-core overlap
	int* dflag = nullptr;  // tensor-core wait time-outs (device)
	unsigned char* wsplit = nullptr;  // W^T in BF16 planes (tensor-core rotation)
	// FP64 overlap and rotation on the int8 tensor cores (scratch allocated on first use)
	int fp64_engine = ITP2D_FP64_DMMA;
	bool oz_failed = false;           // the scratch could not be allocated: DMMA
	unsigned char* oz_w = nullptr;    // W slices
	unsigned char* oz_scratch = nullptr;  // state slices
	int oz_nsplit = 1;                // grid splits of the int8 overlap
	int* oz_e = nullptr;              // row exponents
	long long oz_calls = 0;
	int* hflag = nullptr;  // pinned copy
	// energies
	double* sums = nullptr;
	double* sums2 = nullptr;  // Dirichlet, B != 0: tile sums of <psi|H H psi>
	double* dE = nullptr;
	double* dsig = nullptr;
	double* dres = nullptr;
	double* dEi = nullptr;
	double* dEshift = nullptr;
	double* hbuf = nullptr;  // pinned, 4k doubles
	long long launches = 0;
	bool timing = false;
	double phase_ms[5] = {0, 0, 0, 0, 0};
	double phase_ms_p[10] = {};     // [precision * 5 + phase]
	long long phase_calls_p[10] = {};
	std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
	std::vector<void*> allocs;
	// FP32 form: Lowdin or Cholesky steps between canonical ones
	int canonical_every = 0;     // 0 or 1: always canonical
	int between = ITP2D_BETWEEN_LOWDIN;
	double fp32_tau = 1e-3;      // FP32 eigensolve: largest rotation tangent at which it stops
	int fp32_sweep_cap = 0;      // FP32 canonical eigensolve: sweep cap with Cholesky finish (0: none)
	long long capped_calls = 0;  // canonical FP32 steps finished by the Cholesky step
	int since_canonical = 0;     // orthonormalisations since the last canonical one
	long long ortho_calls[3] = {0, 0, 0};  // canonical, Lowdin, Cholesky
	long long ritz_calls = 0;              // Rayleigh-Ritz steps
	long long tri_rot[2] = {0, 0};         // rotations by an upper-triangular W, per precision
	// register-FFT column pass variant per precision (kColRegSmem / kColTma):
	// -1 until tuned at the first time step of that precision
	int col_variant[2] = {-1, -1};
	int col_forced = -1;  // itp2d_set_column_variant
	double* lstat = nullptr;     // device: max |E|, |E|_F^2, bad diagonal
	double* hlstat = nullptr;    // pinned copy
	void* loop_buf = nullptr;    // device driver loop state (itp2d_run_device_loop)
	size_t device_bytes = 0;  // sum of this context's device allocations
	itp2d::CoopUser coop;     // counts toward the cooperative-eigensolve serialisation
};

namespace {

int cuda_status(cudaError_t e) {
	if (e == cudaSuccess) return ITP2D_OK;
	if (e == cudaErrorMemoryAllocation) return ITP2D_E_OOM;
	return ITP2D_E_CUDA;
}

#define ITP2D_TRY(expr)                          \
	do {                                         \
		cudaError_t e_ = (expr);                 \
		if (e_ != cudaSuccess) return cuda_status(e_); \
	} while (0)

bool smooth7(int n) {
	if (n < 1) return false;
	for (int p : {2, 3, 5, 7})
		while (n % p == 0) n /= p;
	return n == 1;
}

void factor(int n, FftPlan& p) {
	p.n = n;
	p.nstages = 0;
	while (n > 1) {
		int r;
		if (n % 8 == 0) r = 8;
		else if (n % 4 == 0) r = 4;
		else if (n % 2 == 0) r = 2;
		else if (n % 3 == 0) r = 3;
		else if (n % 5 == 0) r = 5;
		else r = 7;
		p.radix[p.nstages++] = r;
		n /= r;
	}
}

template <class R>
std::vector<c2<R>> make_twiddles(int n) {
	std::vector<c2<R>> tw(n);
	for (int t = 0; t < n; t++) {
		const long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)t / (long double)n;
		tw[t] = mk<R>((R)(double)cosl(a), (R)(double)(-sinl(a)));
	}
	return tw;
}

template <class R>
std::vector<c2<R>> make_ext(int N) {
	std::vector<c2<R>> e(2 * N + 1);
	for (int m = 0; m <= 2 * N; m++) {
		const long double a = 3.14159265358979323846264338327950288L * (long double)m / (long double)(2 * N);
		e[m] = mk<R>((R)(double)cosl(a), (R)(double)(-sinl(a)));
	}
	return e;
}

void* dalloc(itp2d_ctx* c, size_t bytes, cudaError_t* err) {
	void* p = nullptr;
	*err = cudaMalloc(&p, bytes ? bytes : 16);
	if (*err == cudaSuccess) {
		c->allocs.push_back(p);
		c->device_bytes += bytes ? bytes : 16;
	}
	return p;
}

template <class R>
int build_plan(itp2d_ctx* c, int axis, int kind) {
	PlanStore& ps = c->planstore[c->precision][axis][kind];
	if (ps.ready) return ITP2D_OK;
	const int N = axis == 0 ? c->sx : c->sy;
	const int n = kind == 0 ? N : 2 * N;
	ps.lp.N = N;
	ps.lp.kind = kind;
	factor(n, ps.lp.fft);
	cudaError_t e;
	auto tw = make_twiddles<R>(n);
	ps.tw = dalloc(c, tw.size() * sizeof(c2<R>), &e);
	if (e != cudaSuccess) return cuda_status(e);
	ITP2D_TRY(cudaMemcpy(ps.tw, tw.data(), tw.size() * sizeof(c2<R>), cudaMemcpyHostToDevice));
	ps.lp.fft.tw = ps.tw;
	if (kind != 0) {
		auto ex = make_ext<R>(N);
		ps.ext = dalloc(c, ex.size() * sizeof(c2<R>), &e);
		if (e != cudaSuccess) return cuda_status(e);
		ITP2D_TRY(cudaMemcpy(ps.ext, ex.data(), ex.size() * sizeof(c2<R>), cudaMemcpyHostToDevice));
	}
	ps.lp.ext = ps.ext;
	ps.ready = true;
	return ITP2D_OK;
}

int build_plans(itp2d_ctx* c, int axis, int kind) {
	int st = c->precision == ITP2D_FP64 ? build_plan<double>(c, axis, kind) : build_plan<float>(c, axis, kind);
	// Dirichlet with a magnetic field also needs the x-axis cosine lines
	if (!st && axis == 0 && kind == 1 && c->B != 0)
		st = c->precision == ITP2D_FP64 ? build_plan<double>(c, 0, 2) : build_plan<float>(c, 0, 2);
	return st;
}

const LinePlan& plan(const itp2d_ctx* c, int axis, int kind) { return c->planstore[c->precision][axis][kind].lp; }

// Uploads a double host table in the working precision into dst (allocating on
// first use, with room for doubles so that a precision switch reuses it).
int upload_table(itp2d_ctx* c, void** dst, const std::vector<double>& h) {
	const size_t n = h.size();
	if (!*dst) {
		const cudaError_t e = cudaMalloc(dst, n * sizeof(double));
		if (e != cudaSuccess) {
			*dst = nullptr;
			return cuda_status(e);
		}
		c->table_allocs.push_back(*dst);
		c->device_bytes += n * sizeof(double);
	}
	if (c->precision == ITP2D_FP64) {
		ITP2D_TRY(cudaMemcpy(*dst, h.data(), n * sizeof(double), cudaMemcpyHostToDevice));
	} else {
		std::vector<float> f(n);
		for (size_t i = 0; i < n; i++) f[i] = (float)h[i];
		ITP2D_TRY(cudaMemcpy(*dst, f.data(), n * sizeof(float), cudaMemcpyHostToDevice));
	}
	return ITP2D_OK;
}

// Transformer k-tables and normalisations (transformer.cpp:66-90).
struct KTables {
	std::vector<double> kx, ky, posy;
	double norm, normx, normy;
};

KTables ktables(const itp2d_ctx* c) {
	KTables t;
	const double lenx = (double)c->sx * c->dx, leny = (double)c->sy * c->dx;
	const double mx = M_PI / lenx, my = M_PI / leny;
	t.kx.resize(c->sx);
	t.ky.resize(c->sy);
	t.posy.resize(c->sy);
	const bool per = c->boundary == ITP2D_PERIODIC;
	for (int x = 0; x < c->sx; x++)
		t.kx[x] = per ? (double)((x < c->sx / 2) ? x : x - c->sx) * 2 * mx : (double)(x + 1) * mx;
	for (int y = 0; y < c->sy; y++) {
		t.ky[y] = per ? (double)((y < c->sy / 2) ? y : y - c->sy) * 2 * my : (double)(y + 1) * my;
		t.posy[y] = (double)(2 * y + 1 - c->sy) * 0.5 * c->dx;
	}
	if (per) {
		t.norm = 1.0 / (double)(c->sx * c->sy);
		t.normx = 1.0 / (double)c->sx;
		t.normy = 1.0 / (double)c->sy;
	} else {
		t.norm = 1.0 / (double)(4 * c->sx * c->sy);
		t.normx = 1.0 / (double)(2 * c->sx);
		t.normy = 1.0 / (double)(2 * c->sy);
	}
	return t;
}

// Multi-product coefficients c_t = t^{2(m-1)} / prod_{n != t}(t^2 - n^2)
// (multiproductsplit.cpp:49-59).
std::vector<double> mp_coefficients(int m) {
	std::vector<double> c(m);
	for (int t = 1; t <= m; t++) {
		int denom = 1;
		for (int n = 1; n <= m; n++)
			if (n != t) denom *= (t * t - n * n);
		c[t - 1] = std::pow((double)t, 2 * (m - 1)) / denom;
	}
	return c;
}

// Exponential kinetic tables of ExpKinetic::calculate_multipliers
// (expkinetic.cpp:65-136) for time step e, coefficient coeff, prefactor p.
int kinetic_exp_tables(itp2d_ctx* c, MemberTables& mt, double e, double coeff, double prefactor) {
	const KTables kt = ktables(c);
	const int sx = c->sx, sy = c->sy;
	if (c->B == 0) {
		std::vector<double> mul((size_t)sx * sy);
		const double A = coeff * e * 0.5;
		const double p = prefactor * kt.norm;
		for (int y = 0; y < sy; y++)
			for (int x = 0; x < sx; x++)
				mul[(size_t)y * sx + x] = p * std::exp(A * (kt.kx[x] * kt.kx[x] + kt.ky[y] * kt.ky[y]));
		return upload_table(c, &mt.kmul, mul);
	}
	// periodic: X is applied twice around one FFTx/iFFTx pair; Dirichlet: once
	// per DSTx / (iDSTx, iDCTx) round trip (expkinetic.cpp:83-85)
	const bool per = c->boundary == ITP2D_PERIODIC;
	const double normfacx = per ? std::sqrt(kt.normx) : kt.normx;
	const double z = c->B * e;
	const double Cy = (std::fabs(z) < 1e-6) ? 1 + std::pow(z, 2) / 6 + std::pow(z, 4) / 120 : std::sinh(z) / z;
	const double Cx = (std::fabs(z) < 1e-6) ? 0.5 - std::pow(z, 2) / 24 + std::pow(z, 4) / 240 : std::tanh(z / 2) / z;
	const double Ax = coeff * e * 0.5 * Cx;
	const double Ay = coeff * e * 0.5 * Cy;
	const double px = normfacx;
	const double py = prefactor * kt.normy;
	std::vector<double> X((size_t)sx * sy), Y(sy), X2;
	if (!per) X2.resize((size_t)sx * sy);
	for (int y = 0; y < sy; y++) {
		const double dy = kt.posy[y];
		Y[y] = py * std::exp(Ay * kt.ky[y] * kt.ky[y]);
		for (int x = 0; x < sx; x++) {
			if (per) {
				const double q = kt.kx[x] - c->B * dy;
				X[(size_t)y * sx + x] = px * std::exp(Ax * q * q);
			} else {
				// sine and cosine parts of exp(c P^2) on a sine series
				// (expkinetic.cpp:108-133)
				const double By = c->B * dy;
				const double common = px * std::exp(Ax * (kt.kx[x] * kt.kx[x] + By * By));
				const double arg = 2 * Ax * kt.kx[x] * By;
				X[(size_t)y * sx + x] = common * std::cosh(arg);
				X2[(size_t)y * sx + x] = common * std::sinh(arg);
			}
		}
	}
	int st = upload_table(c, &mt.kx, X);
	if (st) return st;
	if (!per) {
		st = upload_table(c, &mt.kx2, X2);
		if (st) return st;
	}
	return upload_table(c, &mt.ky, Y);
}

int potential_table(itp2d_ctx* c, void** dst, double e, double coeff, double prefactor) {
	std::vector<double> v(c->V.size());
	for (size_t i = 0; i < v.size(); i++) v[i] = prefactor * std::exp(e * coeff * c->V[i]);
	return upload_table(c, dst, v);
}

// Rebuilds every table for the current eps (SecondOrderSplit members of
// secondordersplit.cpp:21-49 inside MultiProductSplit).
int rebuild_tables(itp2d_ctx* c) {
	c->m = c->null_pot ? 1 : c->halforder;
	const std::vector<double> coef = mp_coefficients(c->m);
	if ((int)c->members.size() < c->m) c->members.resize(c->m);
	for (int t = 1; t <= c->m; t++) {
		MemberTables& mt = c->members[t - 1];
		mt.t = t;
		mt.c = coef[t - 1];
		const double et = c->eps / (double)t;
		int st;
		if (c->null_pot) {
			st = kinetic_exp_tables(c, mt, et, -1.0 * t, mt.c);
			if (st) return st;
			continue;
		}
		st = kinetic_exp_tables(c, mt, et, -1.0, 1.0);
		if (st) return st;
		st = potential_table(c, &mt.vh, et, -0.5, 1.0);
		if (st) return st;
		st = potential_table(c, &mt.vp, et, -0.5, mt.c);
		if (st) return st;
		if (t >= 2) {
			st = potential_table(c, &mt.vsq, et, -1.0, 1.0);
			if (st) return st;
		}
	}
	return ITP2D_OK;
}

// Kinetic (Hamiltonian) tables of kinetic.cpp:25-83 and the potential.
int rebuild_energy_tables(itp2d_ctx* c) {
	const KTables kt = ktables(c);
	const int sx = c->sx, sy = c->sy;
	int st;
	if (c->B == 0) {
		std::vector<double> t2((size_t)sx * sy);
		for (int y = 0; y < sy; y++)
			for (int x = 0; x < sx; x++)
				t2[(size_t)y * sx + x] = 0.5 * (kt.kx[x] * kt.kx[x] + kt.ky[y] * kt.ky[y]) * kt.norm;
		st = upload_table(c, &c->eT2, t2);
		if (st) return st;
	} else {
		const bool per = c->boundary == ITP2D_PERIODIC;
		std::vector<double> tx((size_t)sx * sy), ty(sy), tx2;
		if (!per) tx2.resize((size_t)sx * sy);
		for (int y = 0; y < sy; y++) {
			ty[y] = 0.5 * kt.ky[y] * kt.ky[y] * kt.normy;
			const double By = c->B * kt.posy[y];
			for (int x = 0; x < sx; x++) {
				if (per) {
					const double q = kt.kx[x] - By;
					tx[(size_t)y * sx + x] = 0.5 * q * q * kt.normx;
				} else {
					// kinetic.cpp:66-80: the first derivative gives a cosine series
					tx[(size_t)y * sx + x] = 0.5 * (kt.kx[x] * kt.kx[x] + By * By) * kt.normx;
					tx2[(size_t)y * sx + x] = By * kt.kx[x] * kt.normx;
				}
			}
		}
		st = upload_table(c, &c->eTx, tx);
		if (st) return st;
		if (!per) {
			st = upload_table(c, &c->eTx2, tx2);
			if (st) return st;
		}
		st = upload_table(c, &c->eTy, ty);
		if (st) return st;
	}
	if (!c->null_pot) {
		st = upload_table(c, &c->eV, c->V);
		if (st) return st;
	}
	return ITP2D_OK;
}

struct PhaseTimer {
	itp2d_ctx* c;
	int phase;
	cudaEvent_t a = nullptr, b = nullptr;
	PhaseTimer(itp2d_ctx* c_, int ph) : c(c_), phase(ph + 5 * c_->precision) {
		if (c->timing) {
			cudaEventCreate(&a);
			cudaEventCreate(&b);
			cudaEventRecord(a, c->stream);
		}
	}
	~PhaseTimer() {
		if (c->timing) {
			cudaEventRecord(b, c->stream);
			c->pending.push_back({phase, {a, b}});
		}
	}
};

void flush_timers(itp2d_ctx* c) {
	for (auto& p : c->pending) {
		cudaEventSynchronize(p.second.second);
		float ms = 0.f;
		cudaEventElapsedTime(&ms, p.second.first, p.second.second);
		c->phase_ms[p.first % 5] += ms;
		c->phase_ms_p[p.first] += ms;
		c->phase_calls_p[p.first]++;
		cudaEventDestroy(p.second.first);
		cudaEventDestroy(p.second.second);
	}
	c->pending.clear();
}

int line_len(const LinePlan& lp) { return lp.kind == 0 ? lp.N : 2 * lp.N; }

template <class R>
void row_pass(itp2d_ctx* c, const LinePlan& lp, const void* in, void* out, const void* acc, const void* pre,
		const void* mid, const void* post, int do_inv, int do_fwd) {
	RowPassArgs a;
	a.in = in; a.out = out; a.acc = acc;
	a.mul_pre = pre; a.mul_mid = mid; a.mul_post = post;
	a.do_inv = do_inv; a.do_fwd = do_fwd;
	a.sx = c->sx; a.sy = c->sy; a.G = c->G;
	a.rows_per_tile = row_tile_rows(line_len(lp), sizeof(c2<R>), c->sy);
	a.lp = lp;
	launch_row_pass<R>(a, c->k, nullptr, c->stream);
	c->launches++;
}

template <class R>
void col_pass(itp2d_ctx* c, const LinePlan& lp, void* data, const void* mul2d, const void* mul1d, int mode) {
	ColPassArgs a;
	a.data = data; a.mul2d = mul2d; a.mul1d = mul1d; a.mode = mode;
	a.sx = c->sx; a.sy = c->sy; a.G = c->G;
	a.cols_per_tile = col_tile_cols(line_len(lp), sizeof(c2<R>), c->sx);
	a.lp = lp;
	const int v = c->col_forced >= 0 ? c->col_forced : c->col_variant[c->precision];
	a.variant = v >= 0 ? v : kColRegSmem;
	a.err = c->dflag;
	launch_col_pass<R>(a, c->k, nullptr, c->stream);
	c->launches++;
}

// Times the column pass variants on the spare state buffer (its contents are
// scratch between calls) with the first member's kinetic table, on up to 1024
// states, and keeps the fastest for this precision.
template <class R>
int tune_columns(itp2d_ctx* c) {
	if (c->boundary != ITP2D_PERIODIC || c->members.empty()) return ITP2D_OK;
	const MemberTables& mt = c->members[0];
	ColPassArgs a;
	a.data = c->acc;
	a.mul2d = c->B == 0 ? mt.kmul : nullptr;
	a.mul1d = c->B == 0 ? nullptr : mt.ky;
	a.mode = 0;
	a.sx = c->sx; a.sy = c->sy; a.G = c->G;
	const LinePlan& ly = plan(c, 1, 0);
	a.cols_per_tile = col_tile_cols(line_len(ly), sizeof(c2<R>), c->sx);
	a.lp = ly;
	a.err = c->dflag;
	// up to 1024 states: enough tiles (32 per state at 512 points) for the
	// occupancy and tail of a full pass
	const int v = tune_col_pass_reg<R>(a, std::min(c->k, 1024), c->stream);
	c->col_variant[c->precision] = v >= 0 ? v : kColRegSmem;
	ITP2D_TRY(cudaGetLastError());
	ITP2D_TRY(cudaStreamSynchronize(c->stream));
	// a time-out of the TMA variant during tuning is reported, not hidden
	ITP2D_TRY(cudaMemcpy(c->hflag, c->dflag, sizeof(int), cudaMemcpyDeviceToHost));
	if (*c->hflag != ITP2D_OK) {
		const int f = *c->hflag;
		ITP2D_TRY(cudaMemset(c->dflag, 0, sizeof(int)));
		return f;
	}
	return ITP2D_OK;
}

// One SecondOrderSplit member t applied to `src`, result in `dst`, optionally
// added to `acc` (dst may equal src or acc). Pass structure: the first row pass
// applies V/2 and the forward x transform, each column pass the y transform
// pair with the kinetic multiplier, each interior row pass the inverse x
// transform, V and the forward x transform, and the last row pass the inverse
// x transform and c_t V/2.
bool dirichlet_magnetic(const itp2d_ctx* c) { return c->boundary == ITP2D_DIRICHLET && c->B != 0; }

// Row pass of a kinetic factor: do_inv ends the previous factor (X table and
// inverse x-transform), mid multiplies, do_fwd starts the next one (forward
// x-transform and X table). With Dirichlet boundaries and a magnetic field the
// x-part acts through the sine/cosine split of the Dirichlet magnetic row pass.
template <class R>
void kinetic_row(itp2d_ctx* c, const MemberTables& mt, const void* in, void* out, const void* acc,
		const void* mid, int do_inv, int do_fwd) {
	if (dirichlet_magnetic(c)) {
		DmRowArgs a;
		a.in = in; a.out = out; a.acc = acc;
		a.x1 = mt.kx; a.x2 = mt.kx2; a.mul_mid = mid; a.vadd = nullptr;
		a.lead_fwd = 0; a.do_inv = do_inv; a.do_fwd = do_fwd;
		a.sx = c->sx; a.sy = c->sy; a.G = c->G;
		a.rows_per_tile = dm_row_tile_rows(c->sx, sizeof(c2<R>), c->sy);
		a.lp_dst = plan(c, 0, 1);
		a.lp_dct = plan(c, 0, 2);
		launch_dm_row_pass<R>(a, c->k, c->stream);
		c->launches++;
		return;
	}
	const int kind = c->boundary == ITP2D_PERIODIC ? 0 : 1;
	row_pass<R>(c, plan(c, 0, kind), in, out, acc, do_inv ? mt.kx : nullptr, mid, do_fwd ? mt.kx : nullptr, do_inv,
			do_fwd);
}

template <class R>
void apply_member(itp2d_ctx* c, const MemberTables& mt, const void* src, void* dst, const void* acc) {
	const int kind = c->boundary == ITP2D_PERIODIC ? 0 : 1;
	const LinePlan& ly = plan(c, 1, kind);
	const void* vfirst = c->null_pot ? nullptr : mt.vh;
	const void* vlast = c->null_pot ? nullptr : mt.vp;
	kinetic_row<R>(c, mt, src, dst, nullptr, vfirst, 0, 1);
	for (int r = 1; r <= mt.t; r++) {
		col_pass<R>(c, ly, dst, c->B == 0 ? mt.kmul : nullptr, c->B == 0 ? nullptr : mt.ky, 0);
		if (r < mt.t) kinetic_row<R>(c, mt, dst, dst, nullptr, mt.vsq, 1, 1);
	}
	kinetic_row<R>(c, mt, dst, dst, acc, vlast, 1, 0);
}

// Multi-product propagation (MultiProductSplit over OperatorSum,
// operatorsum.cpp:61-86): member 1 goes out of place into acc; each later
// member reads the original psi and its last row pass adds into acc, so the
// sum is formed in the reference order (m1 + m2) + m3. The last member may work
// in place on psi because nothing reads the original afterwards.
template <class R>
int propagate_fused(itp2d_ctx* c) {
	const int kind = c->boundary == ITP2D_PERIODIC ? 0 : 1;
	const LinePlan& ly = plan(c, 1, kind);
	if (c->m == 1) {
		apply_member<R>(c, c->members[0], c->psi, c->psi, nullptr);
		return ITP2D_OK;
	}
	apply_member<R>(c, c->members[0], c->psi, c->acc, nullptr);
	for (int t = 2; t <= c->m; t++) {
		const MemberTables& mt = c->members[t - 1];
		void* buf = (t == c->m) ? c->psi : c->work;
		kinetic_row<R>(c, mt, c->psi, buf, nullptr, mt.vh, 0, 1);
		for (int r = 1; r <= mt.t; r++) {
			col_pass<R>(c, ly, buf, c->B == 0 ? mt.kmul : nullptr, c->B == 0 ? nullptr : mt.ky, 0);
			if (r < mt.t) kinetic_row<R>(c, mt, buf, buf, nullptr, mt.vsq, 1, 1);
		}
		// acc = member_t + acc
		kinetic_row<R>(c, mt, buf, c->acc, c->acc, mt.vp, 1, 0);
	}
	void* t = c->psi;
	c->psi = c->acc;
	c->acc = t;
	return ITP2D_OK;
}

// Row / column tile of the energy passes: the register-FFT tile where that
// path applies, else the shared-memory tile.
int energy_rows(const LinePlan& lp, int elem, int sy) {
	const int r = energy_row_tile_reg(lp, sy);
	return r ? r : row_tile_rows(line_len(lp), elem, sy);
}
int energy_cols(const LinePlan& lp, int elem, int sx) {
	const int c = energy_col_tile_reg(lp, sx);
	return c ? c : col_tile_cols(line_len(lp), elem, sx);
}

template <class R>
int energies_impl(itp2d_ctx* c, void* h_out, bool want_sums) {
	const int kind = c->boundary == ITP2D_PERIODIC ? 0 : 1;
	const LinePlan& lx = plan(c, 0, kind);
	const LinePlan& ly = plan(c, 1, kind);
	const void* V = c->null_pot ? nullptr : c->eV;
	if (c->B == 0) {
		// acc = F_x psi; acc = F_y^-1 T F_y acc; h = F_x^-1 acc + V psi
		row_pass<R>(c, lx, c->psi, c->acc, nullptr, nullptr, nullptr, nullptr, 0, 1);
		col_pass<R>(c, ly, c->acc, c->eT2, nullptr, 0);
		EnergyRowArgs a;
		a.src_t = c->acc; a.psi = c->psi; a.tmul = nullptr; a.V = V;
		a.h_out = h_out; a.sums = want_sums ? c->sums : nullptr; a.Eshift = c->dEshift;
		a.do_fwd = 0; a.sx = c->sx; a.sy = c->sy; a.G = c->G;
		a.rows_per_tile = energy_rows(lx, sizeof(c2<R>), c->sy);
		a.lp = lx;
		launch_energy_row<R>(a, c->k, nullptr, c->stream);
		c->launches++;
		if (want_sums) {
			const int nt = (c->sy + a.rows_per_tile - 1) / a.rows_per_tile;
			launch_energy_finish(c->sums, nullptr, c->k, nt, c->dx * c->dx, c->dEshift, c->precision == ITP2D_FP32,
					c->dE, c->dsig, c->dres, c->dEi, c->stream);
			c->launches++;
		}
		return ITP2D_OK;
	}
	// magnetic field: acc = T_x src + V src (row pass), h = T_y src + acc
	// (column pass, sums against psi)
	auto hpass = [&](const void* src, void* hout, double* sums) -> int {
		if (dirichlet_magnetic(c)) {
			// the x-part through the sine/cosine split (kinetic.cpp:126-138)
			DmRowArgs d;
			d.in = src; d.out = c->acc; d.acc = nullptr;
			d.x1 = c->eTx; d.x2 = c->eTx2; d.mul_mid = nullptr; d.vadd = V;
			d.lead_fwd = 1; d.do_inv = 1; d.do_fwd = 0;
			d.sx = c->sx; d.sy = c->sy; d.G = c->G;
			d.rows_per_tile = dm_row_tile_rows(c->sx, sizeof(c2<R>), c->sy);
			d.lp_dst = plan(c, 0, 1);
			d.lp_dct = plan(c, 0, 2);
			launch_dm_row_pass<R>(d, c->k, c->stream);
		} else {
			EnergyRowArgs a;
			a.src_t = src; a.psi = src; a.tmul = c->eTx; a.V = V;
			a.h_out = c->acc; a.sums = nullptr; a.Eshift = nullptr;
			a.do_fwd = 1; a.sx = c->sx; a.sy = c->sy; a.G = c->G;
			a.rows_per_tile = energy_rows(lx, sizeof(c2<R>), c->sy);
			a.lp = lx;
			launch_energy_row<R>(a, c->k, nullptr, c->stream);
		}
		c->launches++;
		EnergyColArgs b;
		b.src = src; b.psi = c->psi; b.add_in = c->acc; b.ty = c->eTy;
		b.h_out = hout; b.sums = sums; b.Eshift = c->dEshift;
		b.sx = c->sx; b.sy = c->sy; b.G = c->G;
		b.cols_per_tile = energy_cols(ly, sizeof(c2<R>), c->sx);
		b.lp = ly;
		launch_energy_col<R>(b, c->k, nullptr, c->stream);
		c->launches++;
		return (c->sx + b.cols_per_tile - 1) / b.cols_per_tile;
	};
	// The Dirichlet magnetic H is not Hermitian in its discrete form, so
	// <H^2> = <psi|H (H psi)> needs the second application the reference makes
	// (operators.cpp:40-50); elsewhere |H psi|^2 equals it.
	const bool second = want_sums && dirichlet_magnetic(c);
	const int nt = hpass(c->psi, second ? c->work : h_out, want_sums ? c->sums : nullptr);
	if (second) hpass(c->work, nullptr, c->sums2);
	if (want_sums) {
		launch_energy_finish(c->sums, second ? c->sums2 : nullptr, c->k, nt, c->dx * c->dx, c->dEshift,
				c->precision == ITP2D_FP32, c->dE, c->dsig, c->dres, c->dEi, c->stream);
		c->launches++;
	}
	return ITP2D_OK;
}

template <class R>
int transform_impl(itp2d_ctx* c, int kind_code) {
	// axis selection and direction per enum Transform (transformer.hpp:32-34)
	const int family = kind_code / 6;  // 0 FFT, 1 DST, 2 DCT
	const int sub = kind_code % 6;     // 0 2-D, 1 inv 2-D, 2 x, 3 inv x, 4 y, 5 inv y
	const bool inv = (sub & 1) != 0;
	const bool dox = sub <= 3;
	const bool doy = sub <= 1 || sub >= 4;
	int st = build_plans(c, 0, family);
	if (st) return st;
	st = build_plans(c, 1, family);
	if (st) return st;
	const LinePlan& lx = plan(c, 0, family);
	const LinePlan& ly = plan(c, 1, family);
	if (dox) row_pass<R>(c, lx, c->psi, c->psi, nullptr, nullptr, nullptr, nullptr, inv ? 1 : 0, inv ? 0 : 1);
	if (doy) col_pass<R>(c, ly, c->psi, nullptr, nullptr, inv ? 2 : 1);
	return ITP2D_OK;
}

}  // namespace

extern "C" {

const char* itp2d_status_string(int s) {
	switch (s) {
		case ITP2D_OK: return "ok";
		case ITP2D_E_INVALID: return "invalid argument";
		case ITP2D_E_CUDA: return "CUDA error";
		case ITP2D_E_OOM: return "device out of memory";
		case ITP2D_E_NONPOSITIVE_EIGENVALUE: return "non-positive overlap eigenvalue";
		case ITP2D_E_NONNORMAL_EIGENVALUE: return "non-normal overlap eigenvalue";
		case ITP2D_E_EIGENSOLVER: return "eigensolver did not converge";
		case ITP2D_E_TIMEOUT: return "device wait timed out";
		case ITP2D_E_UNSUPPORTED: return "unsupported configuration";
		default: return "unknown status";
	}
}

int itp2d_ctx_destroy(itp2d_ctx* c) {
	if (!c) return ITP2D_E_INVALID;
	if (c->stream) cudaStreamSynchronize(c->stream);
	flush_timers(c);
	for (void* p : c->allocs) cudaFree(p);
	for (void* p : c->table_allocs) cudaFree(p);
	if (c->hstat) cudaFreeHost(c->hstat);
	if (c->hbuf) cudaFreeHost(c->hbuf);
	if (c->hflag) cudaFreeHost(c->hflag);
	if (c->hlstat) cudaFreeHost(c->hlstat);
	if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
	delete c;
	return ITP2D_OK;
}

long long itp2d_ctx_footprint(int sx, int sy, int num_states, int boundary, double B, int halforder) {
	if (sx < 2 || sy < 2 || num_states < 1 || halforder < 1) return -1;
	int dev = 0, sms = 148;
	if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	const long long G = (long long)sx * sy, k = num_states;
	const bool dm = boundary == ITP2D_DIRICHLET && B != 0;
	// the allocations of itp2d_ctx_create, term by term
	long long b = (2 + ((halforder >= 3 || dm) ? 1 : 0)) * G * k * 16;  // psi, acc, work
	const int nt = overlap_tiles(num_states);
	const int npairs = nt * (nt + 1) / 2;
	const int nsplit = overlap_splits(num_states, G, sms);
	const int parts = std::max(nsplit, tc_overlap_splits(num_states, G, sms));
	const long long kp = std::max(bjacobi_padded(num_states), (num_states + 1) & ~1);
	// tensor-core scratch of the FP32 form: W^T planes, pre-split states for
	// the overlap and the rotation (counted whenever the size can use them)
	b += (2 + parts) * k * k * 16 + (tc_supported(num_states, G) ? (long long)(tc_wsplit_bytes(num_states) +
	                                                                           tc_rows_bytes(num_states, G) +
	                                                                           tc_cols_bytes(num_states, G))
	                                                             : 0);
	b += (num_states >= kBlockJacobiMinK ? 4 : 3) * kp * kp * 16 + npairs * 8;
	if (num_states >= kBlockJacobiMinK) b += (long long)bjacobi_qbuf_elems(num_states) * 16;
	b += k * std::max(sx, sy) * 5 * 8 * (dm ? 2 : 1) + 5 * k * 8 + 16 * k;
	// tables: three potential exponentials and a kinetic table per member, the
	// energy tables, and the line plans (twiddles)
	b += (4LL * halforder + 4) * G * 8 + 4LL * (sx + sy) * 16 * 4;
	return b + (64 << 10);
}

long long itp2d_ctx_device_bytes(itp2d_ctx* c) { return c ? (long long)c->device_bytes : -1; }

int itp2d_ctx_create(int sx, int sy, double dx, int num_states, int boundary, double B, int halforder,
		int precision, void* cuda_stream, itp2d_ctx** out) {
	if (!out || sx < 2 || sy < 2 || num_states < 1 || !(dx > 0) || halforder < 1 || halforder > 8)
		return ITP2D_E_INVALID;
	if (boundary != ITP2D_PERIODIC && boundary != ITP2D_DIRICHLET) return ITP2D_E_INVALID;
	if (precision != ITP2D_FP64 && precision != ITP2D_FP32) return ITP2D_E_INVALID;
	if (!smooth7(sx) || !smooth7(sy) || sx > 4096 || sy > 4096) return ITP2D_E_UNSUPPORTED;
	*out = nullptr;
	itp2d_ctx* c = new (std::nothrow) itp2d_ctx();
	if (!c) return ITP2D_E_OOM;
	c->sx = sx; c->sy = sy; c->dx = dx; c->k = num_states; c->boundary = boundary; c->B = B;
	c->halforder = halforder; c->precision = precision;
	c->G = (long long)sx * sy;
	c->es = precision == ITP2D_FP64 ? 16 : 8;
	c->V.assign((size_t)c->G, 0.0);
	int dev = 0;
	cudaError_t e = cudaGetDevice(&dev);
	if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, dev);
	if (e != cudaSuccess) { delete c; return cuda_status(e); }
	if (cuda_stream) {
		c->stream = (cudaStream_t)cuda_stream;
	} else {
		e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
		if (e != cudaSuccess) { delete c; return cuda_status(e); }
		c->own_stream = true;
	}
	// state buffers sized for FP64 whatever the starting precision, so that a
	// precision switch converts into the spare buffer without allocating
	const size_t sbytes = (size_t)c->G * c->k * 16;
	const int k = c->k;
	c->psi = dalloc(c, sbytes, &e);
	if (e == cudaSuccess) c->acc = dalloc(c, sbytes, &e);
	// work: third member buffer (halforder >= 3) or H psi for the second H
	// application of the Dirichlet magnetic energies
	if (e == cudaSuccess && (halforder >= 3 || (boundary == ITP2D_DIRICHLET && B != 0)))
		c->work = dalloc(c, sbytes, &e);
	// overlap / eigensolver buffers
	const int nt = overlap_tiles(k);
	c->npairs = nt * (nt + 1) / 2;
	c->nsplit = overlap_splits(k, c->G, c->num_sms);
	const int kp = std::max(bjacobi_padded(k), (k + 1) & ~1);  // covers the scalar and block layouts
	if (e == cudaSuccess) c->S = (double2*)dalloc(c, (size_t)k * k * sizeof(double2), &e);
	c->tc_nsplit = tc_overlap_splits(k, c->G, c->num_sms);
	const int parts = std::max(c->nsplit, c->tc_nsplit);
	if (e == cudaSuccess) c->part = (double2*)dalloc(c, (size_t)parts * k * k * sizeof(double2), &e);
	if (e == cudaSuccess) c->dflag = (int*)dalloc(c, sizeof(int), &e);
	if (e == cudaSuccess) e = cudaMemset(c->dflag, 0, sizeof(int));
	if (e == cudaSuccess && tc_supported(k, c->G)) c->wsplit = (unsigned char*)dalloc(c, tc_wsplit_bytes(k), &e);
	if (e == cudaSuccess) c->W = (double2*)dalloc(c, (size_t)k * k * sizeof(double2), &e);
	if (e == cudaSuccess) c->pairs = (int2*)dalloc(c, (size_t)c->npairs * sizeof(int2), &e);
	c->jw.max_sweeps = 60;
	if (e == cudaSuccess) c->jw.A0 = (double2*)dalloc(c, (size_t)kp * kp * sizeof(double2), &e);
	if (e == cudaSuccess) c->jw.A1 = (double2*)dalloc(c, (size_t)kp * kp * sizeof(double2), &e);
	if (e == cudaSuccess) c->jw.V = (double2*)dalloc(c, (size_t)kp * kp * sizeof(double2), &e);
	if (e == cudaSuccess && k >= kBlockJacobiMinK)
		c->jw.Qbuf = (double2*)dalloc(c, bjacobi_qbuf_elems(k) * sizeof(double2), &e);
	if (e == cudaSuccess && k >= kBlockJacobiMinK)
		c->jw.A2 = (double2*)dalloc(c, (size_t)kp * kp * sizeof(double2), &e);
	if (e == cudaSuccess) c->jw.evals = (double*)dalloc(c, (size_t)k * sizeof(double), &e);
	if (e == cudaSuccess) c->jw.perm = (int*)dalloc(c, (size_t)k * sizeof(int), &e);
	if (e == cudaSuccess) c->jw.counters = (int*)dalloc(c, jacobi_counters(c->jw.max_sweeps) * sizeof(int), &e);
	if (e == cudaSuccess) c->dstat = (EigStatus*)dalloc(c, sizeof(EigStatus), &e);
	if (e == cudaSuccess) c->dnorm = (double*)dalloc(c, sizeof(double), &e);
	if (e == cudaSuccess) c->lstat = (double*)dalloc(c, 4 * sizeof(double), &e);
	// energies
	const int ntiles = std::max(sx, sy);  // upper bound of row or column tiles
	if (e == cudaSuccess) c->sums = (double*)dalloc(c, (size_t)k * ntiles * 5 * sizeof(double), &e);
	if (e == cudaSuccess && boundary == ITP2D_DIRICHLET && B != 0)
		c->sums2 = (double*)dalloc(c, (size_t)k * ntiles * 5 * sizeof(double), &e);
	if (e == cudaSuccess) c->dE = (double*)dalloc(c, (size_t)5 * k * sizeof(double), &e);
	if (e == cudaSuccess) {
		c->dsig = c->dE + k;
		c->dres = c->dE + 2 * k;
		c->dEi = c->dE + 3 * k;
		c->dEshift = c->dE + 4 * k;
		e = cudaMemset(c->dE, 0, (size_t)5 * k * sizeof(double));
	}
	if (e == cudaSuccess) e = cudaMallocHost((void**)&c->hstat, sizeof(EigStatus));
	if (e == cudaSuccess) e = cudaMallocHost((void**)&c->hflag, sizeof(int));
	if (e == cudaSuccess) e = cudaMallocHost((void**)&c->hlstat, 4 * sizeof(double));
	if (e == cudaSuccess) e = cudaMallocHost((void**)&c->hbuf, (size_t)4 * k * sizeof(double));
	if (e == cudaSuccess) {
		std::vector<int2> pr;
		for (int i = 0; i < nt; i++)
			for (int j = i; j < nt; j++) pr.push_back(make_int2(i, j));
		e = cudaMemcpy(c->pairs, pr.data(), pr.size() * sizeof(int2), cudaMemcpyHostToDevice);
	}
	if (e != cudaSuccess) {
		const int st = cuda_status(e);
		itp2d_ctx_destroy(c);
		return st;
	}
	const int kind = boundary == ITP2D_PERIODIC ? 0 : 1;
	int st = build_plans(c, 0, kind);
	if (!st) st = build_plans(c, 1, kind);
	if (!st) st = rebuild_energy_tables(c);  // null potential until set
	if (st) {
		itp2d_ctx_destroy(c);
		return st;
	}
	*out = c;
	return ITP2D_OK;
}

int itp2d_set_potential(itp2d_ctx* c, const double* V) {
	if (!c) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	if (V) {
		std::memcpy(c->V.data(), V, (size_t)c->G * sizeof(double));
		c->null_pot = false;
	} else {
		std::fill(c->V.begin(), c->V.end(), 0.0);
		c->null_pot = true;
	}
	int st = rebuild_energy_tables(c);
	if (st) return st;
	if (c->eps_set) return rebuild_tables(c);
	return ITP2D_OK;
}

int itp2d_set_time_step(itp2d_ctx* c, double eps) {
	if (!c || !(eps > 0)) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	c->eps = eps;
	c->eps_set = true;
	const int st = rebuild_tables(c);
	if (st || c->col_variant[c->precision] >= 0) return st;
	// one tuning per device, precision and grid for the process: contexts of
	// the same size (a serving loop, a batch) reuse the choice
	static std::mutex mu;
	static std::map<std::tuple<int, int, int, int, int>, int> tuned;
	int dev = 0;
	cudaGetDevice(&dev);
	const auto key = std::make_tuple(dev, c->precision, c->sx, c->sy, c->boundary);
	{
		std::lock_guard<std::mutex> lk(mu);
		const auto it = tuned.find(key);
		if (it != tuned.end()) {
			c->col_variant[c->precision] = it->second;
			return ITP2D_OK;
		}
	}
	const int r = c->precision == ITP2D_FP64 ? tune_columns<double>(c) : tune_columns<float>(c);
	if (r == ITP2D_OK && c->col_variant[c->precision] >= 0) {
		std::lock_guard<std::mutex> lk(mu);
		tuned[key] = c->col_variant[c->precision];
	}
	return r;
}

int itp2d_set_column_variant(itp2d_ctx* c, int variant) {
	if (!c || variant < -1 || variant >= kColVariants) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	c->col_forced = variant;
	return ITP2D_OK;
}

int itp2d_column_variant(itp2d_ctx* c) {
	if (!c) return -1;
	std::lock_guard<std::mutex> g(c->mu);
	const int v = c->col_forced >= 0 ? c->col_forced : c->col_variant[c->precision];
	return v >= 0 ? v : kColRegSmem;
}

int itp2d_upload_states(itp2d_ctx* c, const double* h) {
	if (!c || !h) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	const size_t n = (size_t)c->G * c->k;
	if (c->precision == ITP2D_FP64) {
		ITP2D_TRY(cudaMemcpyAsync(c->psi, h, n * 16, cudaMemcpyHostToDevice, c->stream));
	} else {
		// FP64 values into the spare state buffer, converted on the device
		ITP2D_TRY(cudaMemcpyAsync(c->acc, h, n * 16, cudaMemcpyHostToDevice, c->stream));
		launch_convert(c->acc, 1, c->psi, (long long)n, c->stream);
		c->launches++;
		ITP2D_TRY(cudaGetLastError());
	}
	ITP2D_TRY(cudaStreamSynchronize(c->stream));
	return ITP2D_OK;
}

int itp2d_download_states(itp2d_ctx* c, double* h) {
	if (!c || !h) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	const size_t n = (size_t)c->G * c->k;
	if (c->precision == ITP2D_FP64) {
		ITP2D_TRY(cudaMemcpyAsync(h, c->psi, n * 16, cudaMemcpyDeviceToHost, c->stream));
		ITP2D_TRY(cudaStreamSynchronize(c->stream));
	} else {
		// widened on the device into the spare state buffer
		launch_convert(c->psi, 0, c->acc, (long long)n, c->stream);
		c->launches++;
		ITP2D_TRY(cudaGetLastError());
		ITP2D_TRY(cudaMemcpyAsync(h, c->acc, n * 16, cudaMemcpyDeviceToHost, c->stream));
		ITP2D_TRY(cudaStreamSynchronize(c->stream));
	}
	return ITP2D_OK;
}

int itp2d_device_states(itp2d_ctx* c, void** p) {
	if (!c || !p) return ITP2D_E_INVALID;
	*p = c->psi;
	return ITP2D_OK;
}

int itp2d_propagate(itp2d_ctx* c) {
	if (!c) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	if (!c->eps_set) return ITP2D_E_INVALID;
	PhaseTimer t(c, kPropagate);
	if (c->precision == ITP2D_FP64) propagate_fused<double>(c);
	else propagate_fused<float>(c);
	return cuda_status(cudaGetLastError());
}

int itp2d_energies(itp2d_ctx* c, double* E, double* sigma, double* sres, double* Eimag) {
	if (!c || !E || !sigma) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	{
		PhaseTimer t(c, kEnergies);
		if (c->precision == ITP2D_FP64) energies_impl<double>(c, nullptr, true);
		else energies_impl<float>(c, nullptr, true);
		ITP2D_TRY(cudaGetLastError());
		ITP2D_TRY(cudaMemcpyAsync(c->hbuf, c->dE, (size_t)4 * c->k * sizeof(double), cudaMemcpyDeviceToHost,
				c->stream));
		// the current energies are the shift of the next residual evaluation
		ITP2D_TRY(cudaMemcpyAsync(c->dEshift, c->dE, (size_t)c->k * sizeof(double), cudaMemcpyDeviceToDevice,
				c->stream));
		// status of the bounded waits of the passes since the last check
		ITP2D_TRY(cudaMemcpyAsync(c->hflag, c->dflag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
	}
	ITP2D_TRY(cudaStreamSynchronize(c->stream));
	if (*c->hflag != ITP2D_OK) {
		const int f = *c->hflag;
		ITP2D_TRY(cudaMemset(c->dflag, 0, sizeof(int)));
		return f;
	}
	const int k = c->k;
	std::memcpy(E, c->hbuf, k * sizeof(double));
	std::memcpy(sigma, c->hbuf + k, k * sizeof(double));
	if (sres) std::memcpy(sres, c->hbuf + 2 * k, k * sizeof(double));
	if (Eimag) std::memcpy(Eimag, c->hbuf + 3 * k, k * sizeof(double));
	return ITP2D_OK;
}

int itp2d_apply_hamiltonian(itp2d_ctx* c) {
	if (!c) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	// h is written into the second buffer, which then becomes the state array
	// (the field path reuses acc as its intermediate; every kernel reads an
	// element of acc before the same thread overwrites it)
	void* h = c->acc;
	if (c->precision == ITP2D_FP64) energies_impl<double>(c, h, false);
	else energies_impl<float>(c, h, false);
	void* t = c->psi;
	c->psi = c->acc;
	c->acc = t;
	return cuda_status(cudaGetLastError());
}

int itp2d_transform(itp2d_ctx* c, int kind) {
	if (!c || kind < 0 || kind > ITP2D_IDCTY) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	int st = c->precision == ITP2D_FP64 ? transform_impl<double>(c, kind) : transform_impl<float>(c, kind);
	if (st) return st;
	return cuda_status(cudaGetLastError());
}

static bool oz_ready(itp2d_ctx* c);

namespace {

bool use_tensor_cores(const itp2d_ctx* c) {
	return c->precision == ITP2D_FP32 && (c->engine == ITP2D_CONTRACT_AUTO || c->engine == ITP2D_CONTRACT_TC_STAGED) &&
	       tc_supported(c->k, c->G);
}

// The pre-split scratch of the tensor-core contractions, allocated on first
// use (FP32 form only); on failure the contractions split inside their CTAs.
bool presplit_ready(itp2d_ctx* c) {
	if (c->engine != ITP2D_CONTRACT_AUTO || c->tc_staged) return false;
	if (c->tc_rows && c->tc_cols) return true;
	cudaError_t e = cudaSuccess;
	if (!c->tc_rows) c->tc_rows = (unsigned char*)dalloc(c, tc_rows_bytes(c->k, c->G), &e);
	if (e == cudaSuccess && !c->tc_cols) c->tc_cols = (unsigned char*)dalloc(c, tc_cols_bytes(c->k, c->G), &e);
	if (e != cudaSuccess) {
		cudaGetLastError();  // an allocation failure is not sticky
		c->tc_staged = true;
		return false;
	}
	return true;
}

// psi W on the tensor cores into acc (W upper triangular: triangular K range).
void tc_rotate(itp2d_ctx* c, bool upper) {
	if (presplit_ready(c))
		launch_rotate_tc_presplit(c->W, (const float2*)c->psi, c->k, c->G, c->wsplit, c->tc_cols, (float2*)c->acc,
				c->dflag, c->stream, upper);
	else
		launch_rotate_tc(c->W, (const float2*)c->psi, c->k, c->G, c->wsplit, (float2*)c->acc, c->dflag, c->stream,
				upper);
}

// S = Psi^H Psi dx^2 (full Hermitian, row-major) by the selected engine.
// int8: the FP64 int8 engine may run (itp2d_overlap_matrix and
// itp2d_orthonormalize; the batched form and the captured device loop keep
// DMMA: they read no timeout flag, and the loop allocates nothing).
void launch_overlap_any(itp2d_ctx* c, bool tc, bool int8 = true) {
	if (int8 && !tc && c->precision == ITP2D_FP64 && oz_ready(c)) {
		launch_overlap_oz((const double2*)c->psi, c->k, c->G, c->oz_nsplit, c->oz_scratch, c->oz_e, c->part,
				c->dx * c->dx, c->S, c->dflag, c->stream);
		c->launches += oz_launches();
		c->oz_calls++;
		return;
	}
	if (tc)
		if (presplit_ready(c))
			launch_overlap_tc_presplit((const float2*)c->psi, c->k, c->G, c->tc_nsplit, c->tc_rows, c->part,
					c->dx * c->dx, c->S, c->dflag, c->stream);
		else
			launch_overlap_tc((const float2*)c->psi, c->k, c->G, c->tc_nsplit, c->part, c->dx * c->dx, c->S, c->dflag,
					c->stream);
	else if (c->precision == ITP2D_FP64)
		launch_overlap((const double2*)c->psi, c->k, c->G, c->pairs, c->npairs, c->nsplit, c->part, c->dx * c->dx,
				c->S, c->stream);
	else
		launch_overlap((const float2*)c->psi, c->k, c->G, c->pairs, c->npairs, c->nsplit, c->part, c->dx * c->dx,
				c->S, c->stream);
	c->launches += 2;
}

}  // namespace

int itp2d_set_contraction(itp2d_ctx* c, int engine) {
	if (!c || (engine != ITP2D_CONTRACT_AUTO && engine != ITP2D_CONTRACT_FP64 && engine != ITP2D_CONTRACT_TC_STAGED))
		return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	c->engine = engine;
	return ITP2D_OK;
}

int itp2d_set_fp32_orthonormalization(itp2d_ctx* c, int canonical_every) {
	if (!c || canonical_every < 0) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	c->canonical_every = canonical_every;
	c->since_canonical = 0;
	return ITP2D_OK;
}

int itp2d_set_fp32_canonical_delay(itp2d_ctx* c, int calls) {
	if (!c || calls < 0) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	c->since_canonical = -calls;
	return ITP2D_OK;
}

int itp2d_set_fp32_eig_tolerance(itp2d_ctx* c, double tau) {
	if (!c || !(tau > 0.0) || tau > 1.0) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	c->fp32_tau = tau;
	return ITP2D_OK;
}

int itp2d_set_fp64_engine(itp2d_ctx* c, int engine) {
	if (!c || (engine != ITP2D_FP64_DMMA && engine != ITP2D_FP64_INT8)) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	c->fp64_engine = engine;
	return ITP2D_OK;
}

long long itp2d_int8_contractions(itp2d_ctx* c) {
	if (!c) return -1;
	std::lock_guard<std::mutex> g(c->mu);
	return c->oz_calls;
}

int itp2d_set_fp32_eig_sweeps(itp2d_ctx* c, int max_sweeps) {
	if (!c || max_sweeps < 0 || max_sweeps > 60) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	c->fp32_sweep_cap = max_sweeps;
	return ITP2D_OK;
}

long long itp2d_fp32_capped_eigensolves(itp2d_ctx* c) {
	if (!c) return -1;
	std::lock_guard<std::mutex> g(c->mu);
	return c->capped_calls;
}

int itp2d_triangular_rotations(itp2d_ctx* c, long long* fp64, long long* fp32) {
	if (!c) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	if (fp64) *fp64 = c->tri_rot[ITP2D_FP64];
	if (fp32) *fp32 = c->tri_rot[ITP2D_FP32];
	return ITP2D_OK;
}

int itp2d_set_fp32_between(itp2d_ctx* c, int method) {
	if (!c || (method != ITP2D_BETWEEN_LOWDIN && method != ITP2D_BETWEEN_CHOLESKY)) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	c->between = method;
	return ITP2D_OK;
}

int itp2d_orthonormalization_counts(itp2d_ctx* c, long long* canonical, long long* lowdin, long long* cholesky) {
	if (!c) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	if (canonical) *canonical = c->ortho_calls[0];
	if (lowdin) *lowdin = c->ortho_calls[1];
	if (cholesky) *cholesky = c->ortho_calls[2];
	return ITP2D_OK;
}

int itp2d_overlap_matrix(itp2d_ctx* c, double* S) {
	if (!c || !S) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	const bool tc = use_tensor_cores(c);
	launch_overlap_any(c, tc);
	ITP2D_TRY(cudaGetLastError());
	ITP2D_TRY(cudaMemcpyAsync(S, c->S, (size_t)c->k * c->k * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
	// the tensor-core overlaps (BF16 planes, int8 slices) flag a bounded wait that gave up
	ITP2D_TRY(cudaMemcpyAsync(c->hflag, c->dflag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
	ITP2D_TRY(cudaStreamSynchronize(c->stream));
	if (*c->hflag != ITP2D_OK) {
		const int f = *c->hflag;
		ITP2D_TRY(cudaMemset(c->dflag, 0, sizeof(int)));
		return f;
	}
	return ITP2D_OK;
}

// psi <- psi W by the rotation engine of the precision (into acc, swapped on
// success); the tensor-core rotation's status when it fails. upper: W is
// upper triangular (Cholesky), each output tile reads only the states up to
// its own last one (about half the products).
// Scratch of the int8 FP64 contractions, allocated at the first use; false
// (and the DMMA contractions from then on) when it does not fit.
static bool oz_ready(itp2d_ctx* c) {
	if (c->fp64_engine != ITP2D_FP64_INT8 || c->oz_failed || !oz_supported(c->k, c->G)) return false;
	if (c->oz_w && c->oz_scratch && c->oz_e) return true;
	c->oz_nsplit = oz_overlap_splits(c->k, c->G, c->num_sms, std::max(c->nsplit, c->tc_nsplit));
	cudaError_t e = cudaSuccess;
	if (!c->oz_w) c->oz_w = (unsigned char*)dalloc(c, oz_w_bytes(c->k), &e);
	if (e == cudaSuccess && !c->oz_scratch) c->oz_scratch = (unsigned char*)dalloc(c, oz_scratch_bytes(c->k, c->G), &e);
	if (e == cudaSuccess && !c->oz_e) c->oz_e = (int*)dalloc(c, oz_exp_ints(c->k, c->G) * sizeof(int), &e);
	if (e != cudaSuccess) {
		cudaGetLastError();  // an allocation failure is not sticky
		c->oz_failed = true;
		return false;
	}
	return true;
}

static int rotate_states(itp2d_ctx* c, bool tc, bool upper = false) {
	const bool f64 = c->precision == ITP2D_FP64;
	if (upper) c->tri_rot[c->precision]++;
	const bool oz = !tc && f64 && oz_ready(c);
	{
		PhaseTimer t(c, kRotate);
		if (tc)
			tc_rotate(c, upper);
		else if (oz)
			launch_rotate_oz(c->W, (const double2*)c->psi, c->k, c->G, c->oz_w, c->oz_scratch, c->oz_e,
					(double2*)c->acc, c->dflag, c->stream, upper);
		else if (f64) launch_rotate(c->W, (const double2*)c->psi, c->k, c->G, (double2*)c->acc, c->stream, upper);
		else launch_rotate(c->W, (const float2*)c->psi, c->k, c->G, (float2*)c->acc, c->stream, upper);
		c->launches += tc ? 2 : (oz ? oz_launches() : 1);
	}
	if (oz) c->oz_calls++;
	const bool flagged = tc || oz;
	if (flagged) ITP2D_TRY(cudaMemcpyAsync(c->hflag, c->dflag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
	ITP2D_TRY(cudaGetLastError());
	ITP2D_TRY(cudaStreamSynchronize(c->stream));
	if (flagged && *c->hflag != ITP2D_OK) {
		const int f = *c->hflag;
		ITP2D_TRY(cudaMemset(c->dflag, 0, sizeof(int)));
		return f;
	}
	void* sw = c->psi;
	c->psi = c->acc;
	c->acc = sw;
	return ITP2D_OK;
}

// W = L^{-H} from the overlap in c->S (cholesky.cu). ITP2D_OK, or the
// failing pivot in *bad_index / *bad_value with the states unchanged.
static int cholesky_w(itp2d_ctx* c, int* bad_index, double* bad_value) {
	{
		PhaseTimer t(c, kEigen);
		const int st = launch_cholesky_w(c->S, c->k, c->jw.A0, c->jw.A1, c->jw.V, c->W, c->dstat, c->stream);
		if (st != ITP2D_OK) return st;
		c->launches += cholesky_launches(c->k);
	}
	ITP2D_TRY(cudaMemcpyAsync(c->hstat, c->dstat, sizeof(EigStatus), cudaMemcpyDeviceToHost, c->stream));
	ITP2D_TRY(cudaStreamSynchronize(c->stream));
	const EigStatus s = *c->hstat;
	c->last_sweeps = 0;
	if (s.status != ITP2D_OK) {
		if (bad_index) *bad_index = s.bad_index;
		if (bad_value) *bad_value = s.bad_value;
	}
	return s.status;
}

// Canonical step of FP32 states with a capped eigensolve (fp32_sweep_cap
// sweeps of the FP32 block Jacobi, then W = V_p L^{-H} from the Cholesky
// factorisation of the rotated overlap). Runs inside the eigensolve phase
// timer. *done is false when the path does not apply or the factorisation
// failed (c->S is intact: the caller runs the full eigensolve); a failed
// eigenvalue check of the capped solve is returned as its status.
static int capped_w(itp2d_ctx* c, bool* done, int* sweeps, int* bad_index, double* bad_value) {
	*done = false;
	JacobiWork& w = c->jw;
	if (!w.f32.A0 || c->k < kBlockJacobiMinK) return ITP2D_OK;
	const int ms = w.max_sweeps;
	w.max_sweeps = c->fp32_sweep_cap;
	w.full_result = true;
	cudaError_t e = launch_eigh(c->S, c->k, w, c->dstat, c->num_sms, c->stream, 2);
	w.full_result = false;
	// the rotated overlap into part, V_p^T into A2 (free once the FP32 solve
	// has widened its result)
	if (e == cudaSuccess) e = launch_eig_cholesky_prep(w, c->k, c->part, w.A2, c->stream);
	w.max_sweeps = ms;
	ITP2D_TRY(e);
	c->launches += 6;
	ITP2D_TRY(cudaMemcpyAsync(c->hstat, c->dstat, sizeof(EigStatus), cudaMemcpyDeviceToHost, c->stream));
	ITP2D_TRY(cudaStreamSynchronize(c->stream));
	const EigStatus es = *c->hstat;
	if (es.status != ITP2D_OK) {
		if (bad_index) *bad_index = es.bad_index;
		if (bad_value) *bad_value = es.bad_value;
		return es.status;
	}
	*sweeps = es.sweeps;
	const int st = launch_cholesky_w(c->part, c->k, w.A0, w.A1, w.V, c->W, c->dstat, c->stream);
	if (st != ITP2D_OK) return st;
	c->launches += cholesky_launches(c->k);
	ITP2D_TRY(cudaMemcpyAsync(c->hstat, c->dstat, sizeof(EigStatus), cudaMemcpyDeviceToHost, c->stream));
	ITP2D_TRY(cudaStreamSynchronize(c->stream));
	if (c->hstat->status != ITP2D_OK) return ITP2D_OK;  // not positive definite: full eigensolve
	// W = V_p W': out[i][n] = sum_m VT[m][i] W'[m][n]
	launch_rotate(w.A2, c->W, c->k, (long long)c->k, w.A1, c->stream);
	ITP2D_TRY(cudaMemcpyAsync(c->W, w.A1, (size_t)c->k * c->k * sizeof(double2), cudaMemcpyDeviceToDevice,
			c->stream));
	c->launches += 1;
	*done = true;
	return ITP2D_OK;
}

int itp2d_orthonormalize(itp2d_ctx* c, int algo, int* bad_index, double* bad_value) {
	if (!c || (algo != ITP2D_ORTHO_DEFAULT && algo != ITP2D_ORTHO_HIGHMEM && algo != ITP2D_ORTHO_CHOLESKY))
		return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	if (bad_index) *bad_index = -1;
	if (bad_value) *bad_value = 0.0;
	const bool f64 = c->precision == ITP2D_FP64;
	if (c->k == 1) {
		if (f64) launch_normalize1((double2*)c->psi, c->G, c->dx, c->dnorm, c->stream);
		else launch_normalize1((float2*)c->psi, c->G, c->dx, c->dnorm, c->stream);
		c->launches += 2;
		ITP2D_TRY(cudaGetLastError());
		ITP2D_TRY(cudaStreamSynchronize(c->stream));
		return ITP2D_OK;
	}
	const bool tc = use_tensor_cores(c);
	{
		PhaseTimer t(c, kOverlap);
		launch_overlap_any(c, tc);
	}
	if (algo == ITP2D_ORTHO_CHOLESKY) {
		const int st = cholesky_w(c, bad_index, bad_value);
		if (st != ITP2D_OK) return st;
		c->ortho_calls[2]++;
		return rotate_states(c, tc, true);
	}
	const bool between = !f64 && c->canonical_every > 1 && c->since_canonical + 1 < c->canonical_every;
	// FP32 form between canonical steps, Gram-Schmidt order: taken whenever
	// the factorisation succeeds (canonical below otherwise)
	if (between && c->between == ITP2D_BETWEEN_CHOLESKY && cholesky_w(c, nullptr, nullptr) == ITP2D_OK) {
		c->since_canonical++;
		c->ortho_calls[2]++;
		return rotate_states(c, tc, true);
	}
	// FP32 form between canonical steps: W = D (I + E)^{-1/2} to second order
	// when the normalised overlap is close enough to the identity
	bool lowdin = false;
	if (between && c->between == ITP2D_BETWEEN_LOWDIN) {
		PhaseTimer t(c, kEigen);
		launch_lowdin_prep(c->S, c->k, c->jw.evals, c->jw.A0, c->jw.A1, c->lstat, c->stream);
		ITP2D_TRY(cudaGetLastError());
		ITP2D_TRY(cudaMemcpyAsync(c->hlstat, c->lstat, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
		ITP2D_TRY(cudaStreamSynchronize(c->stream));
		const double emax = c->hlstat[0], efro = std::sqrt(c->hlstat[1]);
		if (c->hlstat[2] == 0.0 && emax < kLowdinMaxElement && efro < kLowdinMaxFrobenius) {
			launch_lowdin_w(c->jw.evals, c->jw.A0, c->jw.A1, c->jw.V, c->k, c->W, c->stream);
			c->launches += 3;
			lowdin = true;
		}
		c->launches += 1;
	}
	if (lowdin) {
		c->since_canonical++;
		c->ortho_calls[1]++;
		c->last_sweeps = 0;
		return rotate_states(c, tc);
	}
	c->since_canonical = 0;
	c->ortho_calls[0]++;
	bool capped = false;
	int capped_sweeps = 0;
	{
		PhaseTimer t(c, kEigen);
		// FP32 states: the overlap is accurate to about 1e-5; a final tangent of
		// 1e-3 leaves off-diagonal elements of about 1e-6, below that (measured
		// on the magnetic dot: one more FP32 iteration, 3% less solve time)
		c->jw.tau_final = f64 ? 0.0 : c->fp32_tau;
		// FP32 states also solve in FP32, on views of the FP64 buffers the block
		// path leaves free (A1 holds two FP32 matrices, A2 two more)
		c->jw.f32 = {};
		if (!f64 && c->jw.Qbuf && c->jw.A2) {
			const size_t kp2 = (size_t)bjacobi_padded(c->k) * bjacobi_padded(c->k);
			c->jw.f32.A0 = (float2*)c->jw.A1;
			c->jw.f32.A1 = c->jw.f32.A0 + kp2;
			c->jw.f32.A2 = (float2*)c->jw.A2;
			c->jw.f32.V = c->jw.f32.A2 + kp2;
			c->jw.f32.Qbuf = (float2*)c->jw.Qbuf;
		}
		if (!f64 && c->fp32_sweep_cap > 0) {
			const int st = capped_w(c, &capped, &capped_sweeps, bad_index, bad_value);
			if (st != ITP2D_OK) return st;
		}
		if (!capped) {
			ITP2D_TRY(launch_eigensolve(c->S, c->k, c->jw, c->W, c->dstat, c->num_sms, c->stream));
			c->launches += 6;
		}
	}
	const bool oz = !tc && f64 && oz_ready(c);
	{
		PhaseTimer t(c, kRotate);
		if (tc)
			tc_rotate(c, false);
		else if (oz)
			launch_rotate_oz(c->W, (const double2*)c->psi, c->k, c->G, c->oz_w, c->oz_scratch, c->oz_e,
					(double2*)c->acc, c->dflag, c->stream, false);
		else if (f64) launch_rotate(c->W, (const double2*)c->psi, c->k, c->G, (double2*)c->acc, c->stream);
		else launch_rotate(c->W, (const float2*)c->psi, c->k, c->G, (float2*)c->acc, c->stream);
		c->launches += tc ? 2 : (oz ? oz_launches() : 1);
	}
	if (oz) c->oz_calls++;
	const bool flagged = tc || oz;
	if (flagged) ITP2D_TRY(cudaMemcpyAsync(c->hflag, c->dflag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
	ITP2D_TRY(cudaGetLastError());
	ITP2D_TRY(cudaMemcpyAsync(c->hstat, c->dstat, sizeof(EigStatus), cudaMemcpyDeviceToHost, c->stream));
	ITP2D_TRY(cudaStreamSynchronize(c->stream));
	EigStatus s = *c->hstat;
	if (capped) {
		s.sweeps = capped_sweeps;  // the status read is the factorisation's
		c->capped_calls++;
	}
	c->last_sweeps = s.sweeps;
	if (s.sweeps > 0) {
		c->sweeps_total += s.sweeps;
		c->sweeps_p[f64 ? 0 : 1] += s.sweeps;
	}
	if (flagged && *c->hflag != ITP2D_OK) {
		const int f = *c->hflag;
		ITP2D_TRY(cudaMemset(c->dflag, 0, sizeof(int)));
		return f;
	}
	if (s.status != ITP2D_OK) {
		if (bad_index) *bad_index = s.bad_index;
		if (bad_value) *bad_value = s.bad_value;
		return s.status;
	}
	void* t = c->psi;
	c->psi = c->acc;
	c->acc = t;
	return ITP2D_OK;
}

int itp2d_rayleigh_ritz(itp2d_ctx* c, double* ritz_values) {
	if (!c) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	if (c->k < 2) return ITP2D_E_INVALID;
	const bool f64 = c->precision == ITP2D_FP64;
	// H psi into the second buffer (psi is not changed)
	int st = f64 ? energies_impl<double>(c, c->acc, false) : energies_impl<float>(c, c->acc, false);
	if (st) return st;
	{
		PhaseTimer t(c, kOverlap);
		// projected Hamiltonian psi^H (H psi) dx^2, FP64 products for either precision
		if (f64)
			launch_overlap((const double2*)c->psi, c->k, c->G, c->pairs, c->npairs, c->nsplit, c->part,
					c->dx * c->dx, c->S, c->stream, (const double2*)c->acc);
		else
			launch_overlap((const float2*)c->psi, c->k, c->G, c->pairs, c->npairs, c->nsplit, c->part,
					c->dx * c->dx, c->S, c->stream, (const float2*)c->acc);
		c->launches += 2;
	}
	{
		PhaseTimer t(c, kEigen);
		c->jw.tau_final = 0.0;
		c->jw.f32 = {};
		ITP2D_TRY(launch_ritz(c->S, c->k, c->jw, c->W, c->dstat, c->num_sms, c->stream));
		c->launches += 6;
	}
	ITP2D_TRY(cudaMemcpyAsync(c->hstat, c->dstat, sizeof(EigStatus), cudaMemcpyDeviceToHost, c->stream));
	ITP2D_TRY(cudaStreamSynchronize(c->stream));
	const EigStatus es = *c->hstat;
	if (es.status != ITP2D_OK) return es.status;
	if (ritz_values)
		ITP2D_TRY(cudaMemcpy(ritz_values, c->jw.evals, (size_t)c->k * sizeof(double), cudaMemcpyDeviceToHost));
	st = rotate_states(c, use_tensor_cores(c));
	if (st == ITP2D_OK) c->ritz_calls++;
	return st;
}

int itp2d_set_precision(itp2d_ctx* c, int precision) {
	if (!c || (precision != ITP2D_FP64 && precision != ITP2D_FP32)) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	if (precision == c->precision) return ITP2D_OK;
	const size_t n = (size_t)c->G * c->k;
	const size_t es_new = precision == ITP2D_FP64 ? 16 : 8;
	// the state buffers hold FP64 states: convert into the spare one and swap
	launch_convert(c->psi, c->precision == ITP2D_FP64 ? 1 : 0, c->acc, (long long)n, c->stream);
	c->launches++;
	ITP2D_TRY(cudaGetLastError());
	ITP2D_TRY(cudaStreamSynchronize(c->stream));
	void* t = c->psi;
	c->psi = c->acc;
	c->acc = t;
	// tables in the new precision, uploaded into the existing allocations
	c->precision = precision;
	c->es = es_new;
	const int kind = c->boundary == ITP2D_PERIODIC ? 0 : 1;
	int st = build_plans(c, 0, kind);
	if (!st) st = build_plans(c, 1, kind);
	if (!st) st = rebuild_energy_tables(c);
	if (!st && c->eps_set) st = rebuild_tables(c);
	return st;
}

int itp2d_synchronize(itp2d_ctx* c) {
	if (!c) return ITP2D_E_INVALID;
	return cuda_status(cudaStreamSynchronize(c->stream));
}

long long itp2d_launch_count(itp2d_ctx* c) { return c ? c->launches : -1; }

int itp2d_set_timing(itp2d_ctx* c, int enable) {
	if (!c) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	c->timing = enable != 0;
	return ITP2D_OK;
}

int itp2d_phase_times(itp2d_ctx* c, double* ms5) {
	if (!c || !ms5) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	flush_timers(c);
	for (int i = 0; i < 5; i++) ms5[i] = c->phase_ms[i];
	return ITP2D_OK;
}

int itp2d_phase_stats(itp2d_ctx* c, double* ms10, long long* calls10) {
	if (!c || !ms10 || !calls10) return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	flush_timers(c);
	for (int i = 0; i < 10; i++) {
		ms10[i] = c->phase_ms_p[i];
		calls10[i] = c->phase_calls_p[i];
	}
	return ITP2D_OK;
}

int itp2d_last_sweeps(itp2d_ctx* c) { return c ? c->last_sweeps : -1; }

long long itp2d_total_sweeps(itp2d_ctx* c) { return c ? c->sweeps_total : -1; }
long long itp2d_precision_sweeps(itp2d_ctx* c, int precision) {
	if (!c || (precision != ITP2D_FP64 && precision != ITP2D_FP32)) return -1;
	return c->sweeps_p[precision == ITP2D_FP64 ? 0 : 1];
}

int itp2d_hermitian_eigensolve(int n, const double* A, double* evals, double* evecs) {
	if (n < 1 || !A || !evals || !evecs) return ITP2D_E_INVALID;
	CoopUser user;
	const int kp = std::max(bjacobi_padded(n), (n + 1) & ~1);
	std::vector<double2> S((size_t)n * n);
	for (int i = 0; i < n; i++)
		for (int j = i; j < n; j++) {
			const double re = A[2 * ((size_t)j * n + i)], im = A[2 * ((size_t)j * n + i) + 1];
			S[(size_t)i * n + j] = make_double2(re, i == j ? 0.0 : im);
			S[(size_t)j * n + i] = make_double2(re, i == j ? 0.0 : -im);
		}
	int dev = 0, sms = 148;
	ITP2D_TRY(cudaGetDevice(&dev));
	ITP2D_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
	JacobiWork w{};
	w.max_sweeps = 60;
	std::vector<void*> bufs;
	auto al = [&](size_t b) -> void* {
		void* p = nullptr;
		if (cudaMalloc(&p, b) != cudaSuccess) return nullptr;
		bufs.push_back(p);
		return p;
	};
	double2* dS = (double2*)al(S.size() * sizeof(double2));
	w.A0 = (double2*)al((size_t)kp * kp * sizeof(double2));
	w.A1 = (double2*)al((size_t)kp * kp * sizeof(double2));
	w.V = (double2*)al((size_t)kp * kp * sizeof(double2));
	if (n >= kBlockJacobiMinK) w.Qbuf = (double2*)al(bjacobi_qbuf_elems(n) * sizeof(double2));
	if (n >= kBlockJacobiMinK) w.A2 = (double2*)al((size_t)kp * kp * sizeof(double2));
	w.evals = (double*)al((size_t)n * sizeof(double));
	w.perm = (int*)al((size_t)n * sizeof(int));
	w.counters = (int*)al(jacobi_counters(w.max_sweeps) * sizeof(int));
	EigStatus* dst = (EigStatus*)al(sizeof(EigStatus));
	int status = ITP2D_OK;
	if (!dS || !w.A0 || !w.A1 || !w.V || !w.evals || !w.perm || !w.counters || !dst ||
			(n >= kBlockJacobiMinK && (!w.Qbuf || !w.A2)))
		status = ITP2D_E_OOM;
	std::vector<double2> V;
	std::vector<int> perm(n);
	EigStatus hs{};
	if (status == ITP2D_OK) {
		cudaError_t e = cudaMemcpy(dS, S.data(), S.size() * sizeof(double2), cudaMemcpyHostToDevice);
		if (e == cudaSuccess) e = launch_eigh(dS, n, w, dst, sms, 0, 0);
		if (e == cudaSuccess) e = cudaDeviceSynchronize();
		V.resize((size_t)kp * kp);
		if (e == cudaSuccess) e = cudaMemcpy(V.data(), w.V, V.size() * sizeof(double2), cudaMemcpyDeviceToHost);
		if (e == cudaSuccess) e = cudaMemcpy(evals, w.evals, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
		if (e == cudaSuccess) e = cudaMemcpy(perm.data(), w.perm, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost);
		if (e == cudaSuccess) e = cudaMemcpy(&hs, dst, sizeof(EigStatus), cudaMemcpyDeviceToHost);
		status = cuda_status(e);
		if (status == ITP2D_OK && hs.status != ITP2D_OK) status = hs.status;
	}
	if (status == ITP2D_OK) {
		const int jkp = jacobi_kp(w, n);
		for (int m = 0; m < n; m++)
			for (int i = 0; i < n; i++) {
				const double2 v = V[(size_t)i * jkp + perm[m]];
				evecs[2 * ((size_t)m * n + i)] = v.x;
				evecs[2 * ((size_t)m * n + i) + 1] = v.y;
			}
	}
	for (void* p : bufs) cudaFree(p);
	return status;
}

}  // extern "C"

// ---- Batched calls over many contexts (the batched form) ----

namespace {

// Locks the contexts' mutexes in address order (no lock-order inversion
// between concurrent batches).
struct BatchLock {
	std::vector<std::unique_lock<std::mutex>> locks;
	explicit BatchLock(std::vector<itp2d_ctx*> cs) {
		std::sort(cs.begin(), cs.end());
		cs.erase(std::unique(cs.begin(), cs.end()), cs.end());
		for (itp2d_ctx* c : cs) locks.emplace_back(c->mu);
	}
};

std::mutex g_batch_mu;               // the process-wide batch stream and staging buffers
cudaStream_t g_batch_stream = nullptr;
BatchEigItem* g_items_host = nullptr;  // pinned
BatchEigItem* g_items_dev = nullptr;
int g_items_cap = 0;
int* g_queue_dev = nullptr;  // the batched eigensolver's work-queue position

int batch_resources(int n) {
	if (!g_batch_stream) ITP2D_TRY(cudaStreamCreateWithFlags(&g_batch_stream, cudaStreamNonBlocking));
	if (!g_queue_dev) ITP2D_TRY(cudaMalloc((void**)&g_queue_dev, sizeof(int)));
	if (n > g_items_cap) {
		if (g_items_host) cudaFreeHost(g_items_host);
		if (g_items_dev) cudaFree(g_items_dev);
		g_items_host = nullptr;
		g_items_dev = nullptr;
		g_items_cap = 0;
		const int cap = std::max(n, 256);
		ITP2D_TRY(cudaMallocHost((void**)&g_items_host, cap * sizeof(BatchEigItem)));
		ITP2D_TRY(cudaMalloc((void**)&g_items_dev, cap * sizeof(BatchEigItem)));
		g_items_cap = cap;
	}
	return ITP2D_OK;
}

}  // namespace

int itp2d_batch_orthonormalize(int n, itp2d_ctx* const* ctxs, int* status, int* bad_index, double* bad_value) {
	if (n < 0 || (n > 0 && (!ctxs || !status))) return ITP2D_E_INVALID;
	if (n == 0) return ITP2D_OK;
	for (int i = 0; i < n; i++)
		if (!ctxs[i] || ctxs[i]->k < 2 || ctxs[i]->k > batched_eigensolve_max_k()) return ITP2D_E_INVALID;
	BatchLock lk(std::vector<itp2d_ctx*>(ctxs, ctxs + n));
	std::lock_guard<std::mutex> gb(g_batch_mu);
	int st = batch_resources(n);
	if (st) return st;
	std::vector<cudaEvent_t> ev(n + 1, nullptr);
	auto cleanup = [&]() {
		for (cudaEvent_t e : ev)
			if (e) cudaEventDestroy(e);
	};
	for (int i = 0; i <= n; i++) {
		const cudaError_t e = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming);
		if (e != cudaSuccess) {
			cleanup();
			return cuda_status(e);
		}
	}
	// overlaps, each on its context's stream
	for (int i = 0; i < n; i++) {
		itp2d_ctx* c = ctxs[i];
		c->since_canonical = 0;
		c->ortho_calls[0]++;
		{
			PhaseTimer t(c, kOverlap);
			launch_overlap_any(c, use_tensor_cores(c), false);
		}
		cudaEventRecord(ev[i], c->stream);
		cudaStreamWaitEvent(g_batch_stream, ev[i], 0);
		BatchEigItem& it = g_items_host[i];
		it.S = c->S;
		it.A = c->jw.A0;
		it.V = c->jw.V;
		it.W = c->W;
		it.evals = c->jw.evals;
		it.perm = c->jw.perm;
		it.st = c->dstat;
		it.k = c->k;
		it.pad = 0;
		it.tau = c->precision == ITP2D_FP64 ? 3e-9 : 1e-3;
	}
	// every eigenproblem in one launch, the largest first (the work queue hands
	// them out in this order)
	std::stable_sort(g_items_host, g_items_host + n,
			[](const BatchEigItem& a, const BatchEigItem& b) { return a.k > b.k; });
	cudaError_t e = cudaMemcpyAsync(g_items_dev, g_items_host, n * sizeof(BatchEigItem), cudaMemcpyHostToDevice,
			g_batch_stream);
	int max_k = 2;
	for (int i = 0; i < n; i++) max_k = std::max(max_k, ctxs[i]->k);
	if (e == cudaSuccess) e = launch_batched_eigensolve(g_items_dev, n, 60, max_k, g_queue_dev, g_batch_stream);
	if (e == cudaSuccess) e = cudaEventRecord(ev[n], g_batch_stream);
	if (e != cudaSuccess) {
		cleanup();
		return cuda_status(e);
	}
	// rotations, each on its context's stream after the eigensolve
	for (int i = 0; i < n; i++) {
		itp2d_ctx* c = ctxs[i];
		cudaStreamWaitEvent(c->stream, ev[n], 0);
		const bool tc = use_tensor_cores(c);
		{
			PhaseTimer t(c, kRotate);
			if (tc)
				tc_rotate(c, false);
			else if (c->precision == ITP2D_FP64)
				launch_rotate(c->W, (const double2*)c->psi, c->k, c->G, (double2*)c->acc, c->stream);
			else launch_rotate(c->W, (const float2*)c->psi, c->k, c->G, (float2*)c->acc, c->stream);
		}
		c->launches += (tc ? 2 : 1) + 3;
		if (tc) cudaMemcpyAsync(c->hflag, c->dflag, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
		cudaMemcpyAsync(c->hstat, c->dstat, sizeof(EigStatus), cudaMemcpyDeviceToHost, c->stream);
	}
	for (int i = 0; i < n; i++) {
		itp2d_ctx* c = ctxs[i];
		e = cudaStreamSynchronize(c->stream);
		if (e != cudaSuccess) {
			cleanup();
			return cuda_status(e);
		}
		const EigStatus hs = *c->hstat;
		int si = hs.status;
		if (si == ITP2D_OK && use_tensor_cores(c) && *c->hflag != ITP2D_OK) {
			si = *c->hflag;
			cudaMemset(c->dflag, 0, sizeof(int));
		}
		status[i] = si;
		if (bad_index) bad_index[i] = hs.bad_index;
		if (bad_value) bad_value[i] = hs.bad_value;
		c->last_sweeps = hs.sweeps;
		if (hs.sweeps > 0) {
			c->sweeps_total += hs.sweeps;
			c->sweeps_p[c->precision == ITP2D_FP64 ? 0 : 1] += hs.sweeps;
		}
		if (si == ITP2D_OK) {
			void* t = c->psi;
			c->psi = c->acc;
			c->acc = t;
		}
	}
	cleanup();
	return ITP2D_OK;
}

int itp2d_batch_energies(int n, itp2d_ctx* const* ctxs, double* const* E, double* const* sigma,
		double* const* sigma_residual) {
	if (n < 0 || (n > 0 && (!ctxs || !E || !sigma))) return ITP2D_E_INVALID;
	for (int i = 0; i < n; i++)
		if (!ctxs[i] || !E[i] || !sigma[i]) return ITP2D_E_INVALID;
	BatchLock lk(std::vector<itp2d_ctx*>(ctxs, ctxs + n));
	for (int i = 0; i < n; i++) {
		itp2d_ctx* c = ctxs[i];
		PhaseTimer t(c, kEnergies);
		if (c->precision == ITP2D_FP64) energies_impl<double>(c, nullptr, true);
		else energies_impl<float>(c, nullptr, true);
		ITP2D_TRY(cudaGetLastError());
		ITP2D_TRY(cudaMemcpyAsync(c->hbuf, c->dE, (size_t)4 * c->k * sizeof(double), cudaMemcpyDeviceToHost,
				c->stream));
		ITP2D_TRY(cudaMemcpyAsync(c->dEshift, c->dE, (size_t)c->k * sizeof(double), cudaMemcpyDeviceToDevice,
				c->stream));
	}
	for (int i = 0; i < n; i++) {
		itp2d_ctx* c = ctxs[i];
		ITP2D_TRY(cudaStreamSynchronize(c->stream));
		const int k = c->k;
		std::memcpy(E[i], c->hbuf, k * sizeof(double));
		std::memcpy(sigma[i], c->hbuf + k, k * sizeof(double));
		if (sigma_residual && sigma_residual[i]) std::memcpy(sigma_residual[i], c->hbuf + 2 * k, k * sizeof(double));
	}
	return ITP2D_OK;
}

int itp2d_batch_propagate(int n, itp2d_ctx* const* ctxs) {
	if (n < 0 || (n > 0 && !ctxs)) return ITP2D_E_INVALID;
	for (int i = 0; i < n; i++) {
		const int st = itp2d_propagate(ctxs[i]);
		if (st) return st;
	}
	return ITP2D_OK;
}

// ---- Device-resident driver loop ----
//
// ITP iterations that never return to the host until the time-step test
// holds: one CUDA graph whose conditional WHILE node runs the body
//   propagate -> overlap -> eigensolve (batch.cu, one CTA; no cooperative
//   grid barrier inside a graph) -> rotation -> energies -> sort + test
// and whose last kernel sets the loop condition on the device. The test
// kernel restates the host driver's step logic for the time-step test
// (itpsystem.cpp:291-330, convergence.cpp:75-199): the (E, sigma, n) tuples
// sorted by energy, the test applied at every sorted position against the
// previous iteration's sorted values, a passing state's flag kept by its
// storage index, and the loop ending once every wanted position's state is
// flagged (or on an eigensolver failure, or after max_iterations).

namespace {

constexpr int kLoopThreads = 1024;

// loop[0] iterations done, loop[1] done, loop[2] status, loop[3] history length,
// loop[7] the batched eigensolver's work-queue position
__global__ void __launch_bounds__(kLoopThreads) loop_test_kernel(const double* __restrict__ E,
		const double* __restrict__ S, int k, int first, int count, int test, double limit, double diff_limit,
		int max_iterations, double* curE, double* curS, double* prevE, double* prevS, int* idx, int* flags,
		int* loop, const EigStatus* eig, cudaGraphConditionalHandle h) {
	__shared__ int s_fail;
	const int tid = threadIdx.x;
	if (tid == 0) s_fail = 0;
	// the previous sorted values become history
	for (int n = tid; n < k; n += blockDim.x) {
		prevE[n] = curE[n];
		prevS[n] = curS[n];
	}
	__syncthreads();
	for (int i = tid; i < k; i += blockDim.x) {
		const double ei = E[i];
		int r = 0;
		for (int j = 0; j < k; j++) {
			const double ej = E[j];
			r += (ej < ei || (ej == ei && (S[j] < S[i] || (S[j] == S[i] && j < i)))) ? 1 : 0;
		}
		curE[r] = ei;
		curS[r] = S[i];
		idx[r] = i;
	}
	__syncthreads();
	const int hist = loop[3] + 1;  // history entries including this iteration
	for (int n = tid; n < k; n += blockDim.x) {
		bool pass = false;
		if (test == 0 || test == 1) {  // abschange, relchange: need two entries
			if (hist >= 2) {
				const double d = fabs(curE[n] - prevE[n]);
				pass = test == 0 ? d < limit : fabs((curE[n] - prevE[n]) / prevE[n]) < limit;
			}
		} else if (hist >= 2) {  // absstdev, relstdev (deviation tests need two entries too)
			const double t = test == 2 ? curS[n] : curS[n] / curE[n];
			const double p = test == 2 ? prevS[n] : prevS[n] / prevE[n];
			pass = t < limit || fabs(t - p) < diff_limit;
		}
		if (pass) flags[idx[n]] = 1;
	}
	__syncthreads();
	for (int n = first + tid; n < first + count; n += blockDim.x)
		if (!flags[idx[n]]) atomicOr(&s_fail, 1);
	__syncthreads();
	if (tid == 0) {
		const int it = loop[0] + 1;
		loop[0] = it;
		loop[3] = hist;
		int done = !s_fail;
		if (eig->status != ITP2D_OK) {
			loop[2] = eig->status;
			done = 1;
		}
		if (it >= max_iterations) done = 1;
		loop[1] = done;
		cudaGraphSetConditional(h, done ? 0u : 1u);
	}
}

}  // namespace

int itp2d_run_device_loop(itp2d_ctx* c, int max_iterations, int test, double limit, double diff_limit, int first,
		int count, const double* prev_sorted_E, const double* prev_sorted_sigma, int* flags, int* iterations,
		int* status, double* sorted_E, double* sorted_sigma, int* sorted_index, double* prev_E_out,
		double* prev_sigma_out) {
	if (!c || max_iterations < 1 || test < 0 || test > 3 || first < 0 || count < 1 || !flags || !iterations ||
			!status || !sorted_E || !sorted_sigma)
		return ITP2D_E_INVALID;
	std::lock_guard<std::mutex> g(c->mu);
	const int k = c->k;
	if (first + count > k || k < 2 || k > batched_eigensolve_max_k() || !c->eps_set) return ITP2D_E_INVALID;
	// device loop state: sorted E, sigma (current and previous), sorted index,
	// flags, loop counters, one eigensolver item
	if (!c->loop_buf) {
		const size_t bytes = (size_t)4 * k * sizeof(double) + 2 * (size_t)k * sizeof(int) + 8 * sizeof(int) +
				sizeof(BatchEigItem) + 64;
		cudaError_t e = cudaSuccess;
		c->loop_buf = dalloc(c, bytes, &e);
		ITP2D_TRY(e);
	}
	double* curE = (double*)c->loop_buf;
	double* curS = curE + k;
	double* prevE = curS + k;
	double* prevS = prevE + k;
	int* idx = (int*)(prevS + k);
	int* dflags = idx + k;
	int* loop = dflags + k;
	BatchEigItem* item = (BatchEigItem*)(((uintptr_t)(loop + 8) + 15) & ~(uintptr_t)15);
	const bool have_prev = prev_sorted_E && prev_sorted_sigma;
	std::vector<int> hl = {0, 0, ITP2D_OK, have_prev ? 1 : 0, 0, 0, 0, 0};
	ITP2D_TRY(cudaMemcpyAsync(loop, hl.data(), 8 * sizeof(int), cudaMemcpyHostToDevice, c->stream));
	ITP2D_TRY(cudaMemcpyAsync(dflags, flags, k * sizeof(int), cudaMemcpyHostToDevice, c->stream));
	if (have_prev) {
		ITP2D_TRY(cudaMemcpyAsync(curE, prev_sorted_E, k * sizeof(double), cudaMemcpyHostToDevice, c->stream));
		ITP2D_TRY(cudaMemcpyAsync(curS, prev_sorted_sigma, k * sizeof(double), cudaMemcpyHostToDevice, c->stream));
	}
	BatchEigItem it;
	it.S = c->S;
	it.A = c->jw.A0;
	it.V = c->jw.V;
	it.W = c->W;
	it.evals = c->jw.evals;
	it.perm = c->jw.perm;
	it.st = c->dstat;
	it.k = k;
	it.pad = 0;
	it.tau = c->precision == ITP2D_FP64 ? 3e-9 : 1e-3;
	ITP2D_TRY(cudaMemcpyAsync(item, &it, sizeof(it), cudaMemcpyHostToDevice, c->stream));
	ITP2D_TRY(cudaStreamSynchronize(c->stream));

	// the graph: a WHILE node whose body is one iteration
	cudaGraph_t graph = nullptr;
	cudaGraphExec_t exec = nullptr;
	ITP2D_TRY(cudaGraphCreate(&graph, 0));
	auto fail = [&](cudaError_t e) {
		if (exec) cudaGraphExecDestroy(exec);
		if (graph) cudaGraphDestroy(graph);
		return cuda_status(e);
	};
	cudaGraphConditionalHandle h;
	cudaError_t e = cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault);
	if (e != cudaSuccess) return fail(e);
	cudaGraphNodeParams np = {};
	np.type = cudaGraphNodeTypeConditional;
	np.conditional.handle = h;
	np.conditional.type = cudaGraphCondTypeWhile;
	np.conditional.size = 1;
	cudaGraphNode_t node;
	e = cudaGraphAddNode(&node, graph, nullptr, 0, &np);
	if (e != cudaSuccess) return fail(e);
	cudaGraph_t body = np.conditional.phGraph_out[0];
	const bool timing = c->timing;
	c->timing = false;  // event records are not allowed in a conditional body
	void* const psi0 = c->psi;
	void* const acc0 = c->acc;
	const long long launches0 = c->launches;
	if (use_tensor_cores(c)) presplit_ready(c);  // allocations happen before the capture
	e = cudaStreamBeginCaptureToGraph(c->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
	if (e == cudaSuccess) {
		const bool tc = use_tensor_cores(c);
		if (c->precision == ITP2D_FP64) propagate_fused<double>(c);
		else propagate_fused<float>(c);
		launch_overlap_any(c, tc, false);
		launch_batched_eigensolve(item, 1, 60, k, loop + 7, c->stream);
		if (tc)
			tc_rotate(c, false);
		else if (c->precision == ITP2D_FP64)
			launch_rotate(c->W, (const double2*)c->psi, k, c->G, (double2*)c->acc, c->stream);
		else launch_rotate(c->W, (const float2*)c->psi, k, c->G, (float2*)c->acc, c->stream);
		std::swap(c->psi, c->acc);
		if (c->precision == ITP2D_FP64) energies_impl<double>(c, nullptr, true);
		else energies_impl<float>(c, nullptr, true);
		cudaMemcpyAsync(c->dEshift, c->dE, (size_t)k * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
		// the body starts and ends on the same state buffer
		if (c->psi != psi0)
			cudaMemcpyAsync(psi0, c->psi, (size_t)c->G * k * c->es, cudaMemcpyDeviceToDevice, c->stream);
		loop_test_kernel<<<1, kLoopThreads, 0, c->stream>>>(c->dE, c->dsig, k, first, count, test, limit,
				diff_limit, max_iterations, curE, curS, prevE, prevS, idx, dflags, loop, c->dstat, h);
		cudaGraph_t out = nullptr;
		const cudaError_t e2 = cudaStreamEndCapture(c->stream, &out);
		e = cudaGetLastError();
		if (e == cudaSuccess) e = e2;
	}
	c->psi = psi0;
	c->acc = acc0;
	c->timing = timing;
	const long long per_iteration = c->launches - launches0 + 1;
	c->launches = launches0;
	if (e != cudaSuccess) return fail(e);
	e = cudaGraphInstantiate(&exec, graph, 0);
	if (e == cudaSuccess) e = cudaGraphLaunch(exec, c->stream);
	std::vector<int> out(8);
	if (e == cudaSuccess) e = cudaMemcpyAsync(out.data(), loop, 8 * sizeof(int), cudaMemcpyDeviceToHost, c->stream);
	if (e == cudaSuccess) e = cudaMemcpyAsync(flags, dflags, k * sizeof(int), cudaMemcpyDeviceToHost, c->stream);
	if (e == cudaSuccess) e = cudaMemcpyAsync(sorted_E, curE, k * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
	if (e == cudaSuccess)
		e = cudaMemcpyAsync(sorted_sigma, curS, k * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
	if (e == cudaSuccess && sorted_index)
		e = cudaMemcpyAsync(sorted_index, idx, k * sizeof(int), cudaMemcpyDeviceToHost, c->stream);
	if (e == cudaSuccess && prev_E_out)
		e = cudaMemcpyAsync(prev_E_out, prevE, k * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
	if (e == cudaSuccess && prev_sigma_out)
		e = cudaMemcpyAsync(prev_sigma_out, prevS, k * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
	if (e == cudaSuccess) e = cudaMemcpyAsync(c->hflag, c->dflag, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
	if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
	if (e != cudaSuccess) return fail(e);
	cudaGraphExecDestroy(exec);
	cudaGraphDestroy(graph);
	*iterations = out[0];
	*status = out[2];
	if (*c->hflag != ITP2D_OK) {
		// a bounded wait of a pass inside the loop ran out
		*status = *c->hflag;
		ITP2D_TRY(cudaMemset(c->dflag, 0, sizeof(int)));
	}
	c->launches += per_iteration * out[0];
	// the current energies are the shift of the next residual evaluation
	return ITP2D_OK;
}
