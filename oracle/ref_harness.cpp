/*
 * Test-infrastructure harness around the itp2d reference sources, compiled
 * unmodified into oracle/_ref/libitp2d_ref.so by oracle/Makefile. It exposes
 * the reference's own objects through a small extern "C" surface so the
 * Python tests and the CPU baseline can drive them:
 *
 *  - "kit" mode builds the hot-path operators exactly like ITPSystem does
 *    (itpsystem.cpp:23-139): DataLayout, Transformer, Potential (+ an array
 *    added through the Noise hook, itpsystem.cpp:63-64), Kinetic, H = T+V
 *    (itpsystem.cpp:116-119), MultiProductSplit (itpsystem.cpp:121) and a
 *    StateSet, and applies them one seam at a time: propagate
 *    (itpsystem.cpp:243-256), StateSet::orthonormalize (stateset.cpp:136-232),
 *    H.mean_and_standard_deviation (operators.cpp:40-50).
 *  - "sys" mode runs the reference ITPSystem::step loop (itpsystem.cpp:407-470).
 *
 * Nothing here is part of the product.
 */
#include <cstring>
#include <string>
#include <vector>
#include <omp.h>

#include "itpsystem.hpp"

namespace {

// Adds a caller-supplied array to the potential through the reference's
// Noise interface (noise.hpp:34-44), which is how a precomputed potential
// (for example a bumpy dot) enters an unmodified ITPSystem.
class ArrayNoise : public Noise {
	public:
		ArrayNoise(const double* v, size_t n) : values(v, v + n), desc("array") {}
		void add_noise(DataLayout const& dl, double* pot_values) const {
			for (size_t i = 0; i < dl.N; i++) pot_values[i] += values[i];
		}
		std::string const& get_description() const { return desc; }
		std::string const& get_distribution_description() const { return desc; }
		std::string const& get_constraint_description() const { return desc; }
		void write_realization_data(std::vector<double>& vec) const { vec = values; }
	private:
		std::vector<double> values;
		std::string desc;
};

struct Kit {
	DataLayout dl;
	Transformer tr;
	BoundaryType bt;
	double B;
	PotentialType const* ptype;
	Noise* noise;
	Potential* pot;
	Kinetic* kin;
	OperatorSum H;
	MultiProductSplit* T;
	StateSet* states;
	std::vector<StateArray*> work;
	Kit(size_t sx, size_t sy, double dx, BoundaryType b, double B_)
		: dl(sx, sy, dx), tr(dl, FFTW_ESTIMATE), bt(b), B(B_), ptype(NULL), noise(NULL),
		  pot(NULL), kin(NULL), T(NULL), states(NULL) {}
	~Kit() {
		for (size_t i = 0; i < work.size(); i++) delete work[i];
		delete states;
		delete T;
		delete kin;
		delete pot;
		delete noise;
		delete ptype;
	}
};

struct Sys {
	Parameters params;
	ArrayNoise* noise;
	ITPSystem* sys;
	Sys() : noise(NULL), sys(NULL) {}
	~Sys() {
		delete sys;
		delete noise;
	}
};

void copy_in(StateSet const& s, size_t k, size_t G, const double* in) {
	for (size_t n = 0; n < k; n++) {
		comp* p = const_cast<comp*>(s[n].data_ptr());
		std::memcpy(p, in + 2 * n * G, G * sizeof(comp));
	}
}

void copy_out(StateSet const& s, size_t k, size_t G, double* out) {
	for (size_t n = 0; n < k; n++)
		std::memcpy(out + 2 * n * G, s[n].data_ptr(), G * sizeof(comp));
}

} // namespace

extern "C" {

/* Layout of the system parameters passed from Python (ctypes mirror). */
struct RefSysParams {
	int sx, sy;
	double len;
	int boundary;          /* 0 periodic, 1 Dirichlet */
	double B;
	int halforder;
	int num_states;
	int wanted;
	int ignore_lowest;
	int num_eps;
	double eps[8];
	double eps_divisor;
	int max_steps;
	double min_eps;
	unsigned long seed;
	int ortho_highmem;
	int threads;
	int recover;
	char potential[128];
	char timestep_test[128];
	char final_test[128];
};

void* refkit_create(int sx, int sy, double len, int boundary, double B, int halforder,
		double eps, int num_states, int ortho_highmem, const char* potential,
		const double* extra_potential, int threads) {
	const double dx = len / static_cast<double>(sx);
	Kit* k = new Kit(static_cast<size_t>(sx), static_cast<size_t>(sy), dx,
			boundary ? Dirichlet : Periodic, B);
	k->ptype = parse_potential_description(potential);
	if (extra_potential)
		k->noise = new ArrayNoise(extra_potential, k->dl.N);
	else
		k->noise = new NoNoise();
	k->pot = new Potential(k->dl, *k->ptype, *k->noise);
	k->kin = new Kinetic(B, k->tr, k->bt);
	k->H += *k->kin;
	if (!k->pot->is_null()) k->H += *k->pot;
	k->T = new MultiProductSplit(halforder, *k->pot, eps, k->tr, k->bt, B);
	k->states = new StateSet(static_cast<size_t>(num_states), k->dl, ortho_highmem ? HighMem : Default);
	const size_t ws = std::max(k->T->required_workspace(), k->H.required_workspace() + 1);
	if (threads < 1) threads = 1;
	omp_set_num_threads(threads);
	oracle_set_blas_threads(threads);
	for (int i = 0; i < threads; i++) k->work.push_back(new StateArray(ws, k->dl));
	return k;
}

void refkit_destroy(void* h) { delete static_cast<Kit*>(h); }

void refkit_get_potential(void* h, double* out) {
	Kit* k = static_cast<Kit*>(h);
	for (size_t y = 0; y < k->dl.sizey; y++)
		for (size_t x = 0; x < k->dl.sizex; x++)
			out[y * k->dl.sizex + x] = k->pot->get_value(x, y);
}

void refkit_kvalues(void* h, double* fkx, double* fky, double* dkx, double* dky) {
	Kit* k = static_cast<Kit*>(h);
	for (size_t x = 0; x < k->dl.sizex; x++) { fkx[x] = k->tr.fft_kx(x); dkx[x] = k->tr.dsct_kx(x); }
	for (size_t y = 0; y < k->dl.sizey; y++) { fky[y] = k->tr.fft_ky(y); dky[y] = k->tr.dsct_ky(y); }
}

void refkit_set_states(void* h, const double* in) {
	Kit* k = static_cast<Kit*>(h);
	copy_in(*k->states, k->states->get_num_states(), k->dl.N, in);
}

void refkit_get_states(void* h, double* out) {
	Kit* k = static_cast<Kit*>(h);
	copy_out(*k->states, k->states->get_num_states(), k->dl.N, out);
}

void refkit_init_gaussian(void* h, unsigned long seed) {
	Kit* k = static_cast<Kit*>(h);
	RNG rng(seed);
	k->states->init_to_gaussian_noise(rng);
}

void refkit_set_time_step(void* h, double eps) { static_cast<Kit*>(h)->T->set_time_step(eps); }

void refkit_propagate(void* h) {
	Kit* k = static_cast<Kit*>(h);
	const long n = static_cast<long>(k->states->get_num_states());
	#pragma omp parallel for
	for (long i = 0; i < n; i++)
		(*k->T)((*k->states)[static_cast<size_t>(i)], *k->work[static_cast<size_t>(omp_get_thread_num())]);
}

/* Returns 0 on success, 1 NonPositiveEigenvalue, 2 NonNormalEigenvalue,
 * 3 EigensolverError, 4 other exception. */
int refkit_orthonormalize(void* h) {
	Kit* k = static_cast<Kit*>(h);
	try {
		k->states->orthonormalize();
	}
	catch (NonPositiveEigenvalue&) { return 1; }
	catch (NonNormalEigenvalue&) { return 2; }
	catch (EigensolverError&) { return 3; }
	catch (std::exception&) { return 4; }
	return 0;
}

double refkit_how_orthonormal(void* h) { return static_cast<Kit*>(h)->states->how_orthonormal(); }

/* Per-state (E, sigma, Im E) in storage order, from H.mean_and_standard_deviation. */
void refkit_energies(void* h, double* E, double* sigma, double* E_imag) {
	Kit* k = static_cast<Kit*>(h);
	const long n = static_cast<long>(k->states->get_num_states());
	#pragma omp parallel for
	for (long i = 0; i < n; i++) {
		std::pair<comp, comp> r = k->H.mean_and_standard_deviation((*k->states)[static_cast<size_t>(i)],
				*k->work[static_cast<size_t>(omp_get_thread_num())]);
		E[i] = std::real(r.first);
		E_imag[i] = std::imag(r.first);
		sigma[i] = std::real(r.second);
	}
}

/* states <- H states (operator application through the reference OperatorSum). */
void refkit_apply_hamiltonian(void* h) {
	Kit* k = static_cast<Kit*>(h);
	const long n = static_cast<long>(k->states->get_num_states());
	#pragma omp parallel for
	for (long i = 0; i < n; i++) {
		StateArray& ws = *k->work[static_cast<size_t>(omp_get_thread_num())];
		k->H((*k->states)[static_cast<size_t>(i)], ws);
	}
}

/* Apply one Transformer transform (enum Transform, transformer.hpp:32-34) to every state. */
void refkit_transform(void* h, int kind) {
	Kit* k = static_cast<Kit*>(h);
	for (size_t i = 0; i < k->states->get_num_states(); i++)
		(*k->states)[i].transform(static_cast<Transform>(kind), k->tr);
}

/* Accumulated seconds of the last orthonormalisations of the kit's StateSet:
 * [0] overlap dots, [1] eigensolve, [2] lincomb, [3] total
 * (StateSet timers, stateset.hpp:77-80). */
void refkit_ortho_times(void* h, double* t4) {
	StateSet& st = *static_cast<Kit*>(h)->states;
	t4[0] = st.get_dot_time();
	t4[1] = st.get_eigensolve_time();
	t4[2] = st.get_lincomb_time();
	t4[3] = st.get_ortho_time();
}

double refkit_normalization_factor(void* h, int kind) {
	return static_cast<Kit*>(h)->tr.normalization_factor(static_cast<Transform>(kind));
}

/* ---- full ITPSystem ---- */

void* refsys_create(const RefSysParams* p, const double* extra_potential, const double* init_states) {
	Sys* s = new Sys();
	Parameters& P = s->params;
	P.set_verbosity(0);
	P.set_fftw_flags(FFTW_ESTIMATE);
	P.define_data_storage("", Parameters::Nothing);
	P.set_random_seed(p->seed);
	P.define_grid(static_cast<size_t>(p->sx), static_cast<size_t>(p->sy), p->len,
			p->boundary ? Dirichlet : Periodic);
	P.define_external_field(p->potential, p->B);
	P.set_num_states(static_cast<size_t>(p->num_states), static_cast<size_t>(p->wanted),
			static_cast<size_t>(p->ignore_lowest));
	P.set_operator_splitting_halforder(p->halforder);
	for (int i = 0; i < p->num_eps && i < 8; i++) P.add_eps_value(p->eps[i]);
	P.set_time_step_divisor(p->eps_divisor);
	P.set_bailout_limits(p->max_steps, p->min_eps);
	P.set_ortho_algorithm(p->ortho_highmem ? HighMem : Default);
	P.set_num_threads(p->threads > 0 ? p->threads : 1);
	P.set_recover(p->recover != 0);
	P.set_timestep_convergence_test(std::string(p->timestep_test));
	P.set_final_convergence_test(std::string(p->final_test));
	if (extra_potential) {
		const size_t G = static_cast<size_t>(p->sx) * static_cast<size_t>(p->sy);
		s->noise = new ArrayNoise(extra_potential, G);
		P.set_user_noise(*s->noise);
	}
	oracle_set_blas_threads(p->threads > 0 ? p->threads : 1);
	s->sys = new ITPSystem(P);
	if (init_states) {
		const size_t G = static_cast<size_t>(p->sx) * static_cast<size_t>(p->sy);
		copy_in(s->sys->get_states(), static_cast<size_t>(p->num_states), G, init_states);
	}
	return s;
}

void refsys_destroy(void* h) { delete static_cast<Sys*>(h); }

void refsys_step(void* h) { static_cast<Sys*>(h)->sys->step(); }

int refsys_is_finished(void* h) { return static_cast<Sys*>(h)->sys->is_finished() ? 1 : 0; }
int refsys_error_flag(void* h) { return static_cast<Sys*>(h)->sys->get_error_flag() ? 1 : 0; }
int refsys_total_steps(void* h) { return static_cast<Sys*>(h)->sys->get_total_step_counter(); }
double refsys_eps(void* h) { return static_cast<Sys*>(h)->sys->get_eps(); }
int refsys_num_finally_converged(void* h) { return static_cast<int>(static_cast<Sys*>(h)->sys->how_many_finally_converged()); }

/* Latest sorted energies and deviations (ascending energy). Returns count, 0 if none yet. */
int refsys_last_energies(void* h, double* E, double* sigma) {
	ITPSystem* sys = static_cast<Sys*>(h)->sys;
	std::vector<std::vector<double> > const& e = sys->get_energies();
	std::vector<std::vector<double> > const& sd = sys->get_standard_deviations();
	if (e.empty()) return 0;
	const std::vector<double>& le = e.back();
	const std::vector<double>& ls = sd.back();
	for (size_t i = 0; i < le.size(); i++) { E[i] = le[i]; sigma[i] = ls[i]; }
	return static_cast<int>(le.size());
}

void refsys_get_states(void* h, double* out) {
	Sys* s = static_cast<Sys*>(h);
	copy_out(s->sys->get_states(), s->params.get_N(), s->sys->datalayout.N, out);
}

/* Phase seconds: total, propagation, ortho, dot, eigensolve, lincomb, convtest. */
void refsys_times(void* h, double* t) {
	ITPSystem* sys = static_cast<Sys*>(h)->sys;
	try {
		t[0] = sys->get_total_time();
	} catch (std::exception&) {
		t[0] = -1.0;  // Timer::get_time throws while the total timer still runs
	}
	t[1] = sys->get_prop_time();
	t[2] = sys->get_ortho_time();
	t[3] = sys->get_dot_time();
	t[4] = sys->get_eigensolve_time();
	t[5] = sys->get_lincomb_time();
	t[6] = sys->get_convtest_time();
}

/* V += the impurities of imp (rows x, y, A, w), one GaussianImpurities::add_noise
 * call each in list order (noise.cpp:24-40) on a DataLayout(sx, sy, dx); the RNG
 * only satisfies the constructor and is never drawn from. */
void ref_add_gaussian_impurities(int sx, int sy, double dx, int n, const double* imp, double* V) {
	DataLayout dl(static_cast<size_t>(sx), static_cast<size_t>(sy), dx);
	RNG rng(1UL);
	GaussianImpurities g(0.0, 0.0, 0.0, 0.0, rng);
	std::vector<double> params(2);
	for (int j = 0; j < n; j++) {
		params[0] = imp[4 * j + 2];
		params[1] = imp[4 * j + 3];
		g.add_noise(imp[4 * j], imp[4 * j + 1], params, dl, V);
	}
}

/* V += n impurities of one shape through the reference's add_noise, in list
 * order (noise.cpp:42-87): shape 1 CoulombImpurities(p0 = exponent,
 * p1 = prefactor), rows (x, y); 2 HemisphereImpurities(p0 = amplitude,
 * p1 = radius), rows (x, y); 3 DeltaImpurities, rows (x, y, A). The RNG only
 * satisfies the constructors and is never drawn from. */
void ref_add_impurities(int shape, int sx, int sy, double dx, int n, const double* rows, double p0, double p1,
		double* V) {
	DataLayout dl(static_cast<size_t>(sx), static_cast<size_t>(sy), dx);
	RNG rng(1UL);
	CoulombImpurities coulomb(p0, p1, rng);
	HemisphereImpurities hemi(p0, p1, rng);
	DeltaImpurities delta(0.0, 0.0, dl, rng);
	std::vector<double> none, amp(1);
	for (int j = 0; j < n; j++) {
		if (shape == 1) coulomb.add_noise(rows[2 * j], rows[2 * j + 1], none, dl, V);
		else if (shape == 2) hemi.add_noise(rows[2 * j], rows[2 * j + 1], none, dl, V);
		else {
			amp[0] = rows[3 * j + 2];
			delta.add_noise(rows[3 * j], rows[3 * j + 1], amp, dl, V);
		}
	}
}

} // extern "C"
