// Native host layer: Parameters, ConvergenceTest, ITPSystem over the device
// C ABI, plus the extern "C" surface of include/itp2d_host.h.
#include "itp2d_host.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <ctime>
#include <sstream>
#include <thread>

#include <unistd.h>

#include "../../include/itp2d_datafile.h"

namespace itp2d {

namespace {

double now_s() {
	return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

std::string status_text(const std::string& where, int st) {
	return where + ": " + itp2d_status_string(st);
}

std::string num(double v) {
	std::ostringstream o;
	o << v;
	return o.str();
}

const char* kWhitespace = " \t\n";
// Largest device-loop chunk while abort or save flags are registered.
const int kFlagChunk = 32;
// FP32 noise floor of the per-step energy change, in single-precision
// roundings of the largest wanted energy.
const double kFp32FloorUlps = 64.0;
// The FP32 switch rule reads the energy change over this many iterations
// (per iteration): below the visible FP32 floor the subspace keeps converging,
// and the longer span delays the switch by the iterations that the FP64
// refinement would otherwise spend at several times the cost.
const size_t kFp32Span = 3;

}  // namespace

NonPositiveEigenvalue::NonPositiveEigenvalue(int n, double v)
	: std::runtime_error("non-positive eigenvalue " + num(v) + " of the overlap matrix at index " + num(n)),
	  index(n), value(v) {}

NonNormalEigenvalue::NonNormalEigenvalue(int n, double v)
	: std::runtime_error("non-normal eigenvalue " + num(v) + " of the overlap matrix at index " + num(n)),
	  index(n), value(v) {}

EigensolverError::EigensolverError(int status) : std::runtime_error(status_text("eigensolver", status)) {}

DeviceError::DeviceError(const std::string& where, int st) : std::runtime_error(status_text(where, st)), status(st) {}

std::pair<std::string, std::vector<double>> parse_parameter_string(const std::string& s) {
	const size_t start = s.find_first_not_of(kWhitespace);
	if (start == std::string::npos) throw ParseError(s);
	const size_t last = s.find_last_not_of(kWhitespace);
	size_t name_end = s.find_first_of(" \t\n(", start);
	if (name_end == std::string::npos || name_end > last) name_end = last + 1;
	std::pair<std::string, std::vector<double>> out(s.substr(start, name_end - start), std::vector<double>());
	const size_t rest = s.find_first_not_of(kWhitespace, name_end);
	if (rest == std::string::npos) return out;
	if (s[rest] != '(' || s[last] != ')') throw ParseError(s);
	std::string inner = s.substr(rest + 1, last - rest - 1);
	if (inner.find_first_not_of(kWhitespace) == std::string::npos) return out;
	std::istringstream in(inner);
	while (true) {
		double v;
		in >> v;
		if (in.fail()) throw ParseError(s);
		out.second.push_back(v);
		in >> std::ws;
		if (in.eof()) break;
		if (in.peek() != ',') throw ParseError(s);
		in.get();
	}
	return out;
}

// ---------------- convergence tests (convergence.cpp) ----------------

NoConvergenceTest::NoConvergenceTest(const std::vector<double>& params) {
	if (!params.empty()) throw GeneralError("convergence test 'none' takes no parameters");
	description = "none";
}

OneStepConvergenceTest::OneStepConvergenceTest(const std::vector<double>& params) {
	if (!params.empty()) throw GeneralError("convergence test 'onestep' takes no parameters");
	description = "one-step convergence";
}

bool OneStepConvergenceTest::test(const ITPSystem& sys, size_t n) const {
	return sys.get_step_counter() == 1 && sys.is_timestep_converged(sys.get_sorted_index(n));
}

RelativeEnergyChangeTest::RelativeEnergyChangeTest(const std::vector<double>& params) {
	if (params.size() != 1) throw GeneralError("relative energy change test takes exactly one parameter");
	limit = params[0];
	description = "relative energy change < " + num(limit);
}

bool RelativeEnergyChangeTest::test(const ITPSystem& sys, size_t n) const {
	const auto& e = sys.get_energies();
	if (e.size() < 2) return false;
	const double a = e[e.size() - 1][n], b = e[e.size() - 2][n];
	return std::fabs((a - b) / b) < limit;
}

AbsoluteEnergyChangeTest::AbsoluteEnergyChangeTest(const std::vector<double>& params) {
	if (params.size() != 1) throw GeneralError("absolute energy change test takes exactly one parameter");
	limit = params[0];
	description = "absolute energy change < " + num(limit);
}

bool AbsoluteEnergyChangeTest::test(const ITPSystem& sys, size_t n) const {
	const auto& e = sys.get_energies();
	if (e.size() < 2) return false;
	return std::fabs(e[e.size() - 1][n] - e[e.size() - 2][n]) < limit;
}

AbsoluteEnergyDeviationTest::AbsoluteEnergyDeviationTest(const std::vector<double>& params) {
	if (params.size() != 1 && params.size() != 2)
		throw GeneralError("absolute deviation test takes one or two parameters");
	dev_limit = params[0];
	diff_limit = params.size() == 2 ? params[1] : 0.0;
	description = "absolute energy deviation < " + num(dev_limit) + " or absolute energy deviation change < " +
	              num(diff_limit);
}

bool AbsoluteEnergyDeviationTest::test(const ITPSystem& sys, size_t n) const {
	const auto& s = sys.get_standard_deviations();
	if (s.size() < 2) return false;
	const double a = s[s.size() - 1][n], b = s[s.size() - 2][n];
	return a < dev_limit || std::fabs(a - b) < diff_limit;
}

RelativeEnergyDeviationTest::RelativeEnergyDeviationTest(const std::vector<double>& params) {
	if (params.size() != 1 && params.size() != 2)
		throw GeneralError("relative deviation test takes one or two parameters");
	dev_limit = params[0];
	diff_limit = params.size() == 2 ? params[1] : 0.0;
	description = "relative energy deviation < " + num(dev_limit) + " or relative energy deviation change < " +
	              num(diff_limit);
}

bool RelativeEnergyDeviationTest::test(const ITPSystem& sys, size_t n) const {
	const auto& e = sys.get_energies();
	const auto& s = sys.get_standard_deviations();
	if (e.size() < 2) return false;
	const size_t l = s.size() - 1;
	const double a = s[l][n] / e[l][n], b = s[l - 1][n] / e[l - 1][n];
	return a < dev_limit || std::fabs(a - b) < diff_limit;
}

std::unique_ptr<ConvergenceTest> parse_convergence_description(const std::string& str) {
	const auto p = parse_parameter_string(str);
	const std::string& n = p.first;
	if (n == "none" || n == "no" || n == "null") return std::unique_ptr<ConvergenceTest>(new NoConvergenceTest(p.second));
	if (n == "onestep" || n == "one-step")
		return std::unique_ptr<ConvergenceTest>(new OneStepConvergenceTest(p.second));
	if (n == "abschange" || n == "absEdelta")
		return std::unique_ptr<ConvergenceTest>(new AbsoluteEnergyChangeTest(p.second));
	if (n == "relchange" || n == "relEdelta")
		return std::unique_ptr<ConvergenceTest>(new RelativeEnergyChangeTest(p.second));
	if (n == "absstdev" || n == "absresidual")
		return std::unique_ptr<ConvergenceTest>(new AbsoluteEnergyDeviationTest(p.second));
	if (n == "relstdev" || n == "relresidual")
		return std::unique_ptr<ConvergenceTest>(new RelativeEnergyDeviationTest(p.second));
	throw GeneralError("unknown convergence test: " + str);
}

// ---------------- grid, potentials, parameters ----------------

DataLayout::DataLayout(size_t sx, size_t sy, double d)
	: sizex(sx), sizey(sy), N(sx * sy), dx(d), lenx((double)sx * d), leny((double)sy * d), posx(sx), posy(sy) {
	for (size_t x = 0; x < sx; x++) posx[x] = (double)(2 * (long)x + 1 - (long)sx) * 0.5 * dx;
	for (size_t y = 0; y < sy; y++) posy[y] = (double)(2 * (long)y + 1 - (long)sy) * 0.5 * dx;
}

// The potential of a description (potentialtypes.hpp:96-380), evaluated by
// the device kernel of itp2d_evaluate_potential_host. Returns false for the
// null potential.
bool evaluate_potential(const std::string& desc, const DataLayout& dl, std::vector<double>& out) {
	int is_null = 0;
	if (itp2d_potential_check(desc.c_str(), &is_null) != ITP2D_OK)
		throw GeneralError("invalid potential description: " + desc);
	out.assign(dl.N, 0.0);
	if (is_null) return false;
	const int st = itp2d_evaluate_potential_host(desc.c_str(), (int)dl.sizex, (int)dl.sizey, dl.dx, out.data());
	if (st != ITP2D_OK) throw DeviceError("itp2d_evaluate_potential_host", st);
	return true;
}

Parameters::Parameters() { itp2d_parameters_default(&p); }

void Parameters::define_grid(size_t sx, size_t sy, double lenx, int boundary) {
	p.sx = (int)sx;
	p.sy = (int)sy;
	p.length = lenx;
	p.boundary = boundary;
}

void Parameters::define_external_field(const std::string& ptype, double B) {
	if (ptype.size() >= sizeof(p.potential)) throw GeneralError("potential description too long");
	std::strcpy(p.potential, ptype.c_str());
	p.B = B;
}

void Parameters::set_num_states(size_t N, size_t wanted, size_t ignore_lowest) {
	if (ignore_lowest + wanted > N) throw GeneralError("wanted + ignored states exceed the number of states");
	p.num_states = (int)N;
	p.wanted = (int)wanted;
	p.ignore_lowest = (int)ignore_lowest;
}

void Parameters::add_eps_value(double e) {
	if (p.num_eps >= 16) throw GeneralError("at most 16 explicit time steps");
	p.eps[p.num_eps++] = e;
}

void Parameters::set_bailout_limits(int max_steps, double min_time_step) {
	p.max_steps = max_steps;
	p.min_eps = min_time_step;
}

void Parameters::set_timestep_convergence_test(const std::string& s) {
	parse_convergence_description(s);  // validate
	std::strncpy(p.timestep_test, s.c_str(), sizeof(p.timestep_test) - 1);
}

void Parameters::set_final_convergence_test(const std::string& s) {
	parse_convergence_description(s);
	std::strncpy(p.final_test, s.c_str(), sizeof(p.final_test) - 1);
}

void Parameters::set_precision(int prec, double fp32_switch) {
	p.precision = prec;
	p.fp32_switch = fp32_switch;
}

// ---------------- ITPSystem ----------------

ITPSystem::ITPSystem(const Parameters& params, void* stream)
	: p(params.raw()), dl((size_t)p.sx, (size_t)p.sy, p.length / (double)p.sx), exhausting(p.exhaust_eps != 0) {
	if (p.ignore_lowest + p.wanted > p.num_states) throw GeneralError("wanted + ignored states exceed N");
	ts_test = parse_convergence_description(p.timestep_test);
	final_test = parse_convergence_description(p.final_test);
	null_potential = !evaluate_potential(p.potential, dl, V);
	if (!params.user_potential.empty()) {
		if (params.user_potential.size() != dl.N) throw GeneralError("user potential has the wrong size");
		for (size_t i = 0; i < dl.N; i++) V[i] += params.user_potential[i];
		null_potential = false;
		user_noise = true;
	}
	for (int i = 0; i < p.num_eps; i++) eps_values.push_back(p.eps[i]);
	if (!eps_values.empty()) {
		eps = eps_values.front();
		eps_values.pop_front();
	} else {
		eps = 0.5;  // Parameters::default_initial_eps
	}
	eps_history.assign(1, std::make_pair(1, eps));
	precision = p.precision;
	check(itp2d_ctx_create(p.sx, p.sy, dl.dx, p.num_states, p.boundary, p.B, p.halforder, precision, stream, &ctx),
			"itp2d_ctx_create");
	check(itp2d_set_timing(ctx, 1), "itp2d_set_timing");
	check(itp2d_set_fp32_orthonormalization(ctx, p.fp32_canonical_every), "itp2d_set_fp32_orthonormalization");
	check(itp2d_set_fp32_canonical_delay(ctx, p.fp32_canonical_delay), "itp2d_set_fp32_canonical_delay");
	check(itp2d_set_fp32_between(ctx, p.fp32_between), "itp2d_set_fp32_between");
	check(itp2d_set_fp32_eig_sweeps(ctx, p.fp32_eig_sweeps), "itp2d_set_fp32_eig_sweeps");
	check(itp2d_set_fp64_engine(ctx, p.fp64_engine), "itp2d_set_fp64_engine");
	check(itp2d_set_potential(ctx, null_potential ? nullptr : V.data()), "itp2d_set_potential");
	check(itp2d_set_time_step(ctx, eps), "itp2d_set_time_step");
	initial_states = params.initial_states;
	if (!initial_states.empty() && initial_states.size() != 2 * dl.N * (size_t)p.num_states)
		throw GeneralError("initial states have the wrong size");
	rng_state = p.seed;
	timestep_converged.assign(p.num_states, false);
	finally_converged.assign(p.num_states, false);
	init_states();
}

ITPSystem::~ITPSystem() {
	if (ctx) itp2d_ctx_destroy(ctx);
}

void ITPSystem::check(int st, const char* where) {
	if (st != ITP2D_OK) throw DeviceError(where, st);
}

// Complex standard-normal noise per grid point, normalised per state
// (StateSet::init_to_gaussian_noise, stateset.cpp:124-131). The stream is a
// counter-based hash (splitmix64) with Box-Muller, so it does not depend on
// the number of host threads. Re-initialisation after a failed
// orthonormalisation draws a fresh stream.
void ITPSystem::init_states() {
	if (!initial_states.empty()) {
		check(itp2d_upload_states(ctx, initial_states.data()), "itp2d_upload_states");
		initial_states.clear();  // a recovery re-randomises like the reference
		return;
	}
	const size_t k = (size_t)p.num_states, G = dl.N;
	std::vector<double> psi(2 * k * G);
	const unsigned long base = rng_state;
	rng_state = rng_state * 6364136223846793005ULL + 1442695040888963407ULL;
	auto mix = [](unsigned long long z) {
		z += 0x9E3779B97F4A7C15ULL;
		z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
		z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
		return z ^ (z >> 31);
	};
	const unsigned nth = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
	std::vector<std::thread> th;
	for (unsigned t = 0; t < nth; t++)
		th.emplace_back([&, t]() {
			for (size_t n = t; n < k; n += nth) {
				double* s = psi.data() + 2 * n * G;
				double nrm = 0.0;
				for (size_t i = 0; i < G; i++) {
					const unsigned long long c = ((unsigned long long)base << 20) ^ (n * G + i);
					const unsigned long long a = mix(2 * c), b = mix(2 * c + 1);
					const double u1 = ((a >> 11) + 0.5) * (1.0 / 9007199254740992.0);
					const double u2 = (b >> 11) * (1.0 / 9007199254740992.0);
					const double r = std::sqrt(-2.0 * std::log(u1));
					s[2 * i] = r * std::cos(2 * M_PI * u2);
					s[2 * i + 1] = r * std::sin(2 * M_PI * u2);
					nrm += s[2 * i] * s[2 * i] + s[2 * i + 1] * s[2 * i + 1];
				}
				const double f = 1.0 / (std::sqrt(nrm) * dl.dx);
				for (size_t i = 0; i < 2 * G; i++) s[i] *= f;
			}
		});
	for (auto& x : th) x.join();
	check(itp2d_upload_states(ctx, psi.data()), "itp2d_upload_states");
}

void ITPSystem::propagate() {
	const double t0 = now_s();
	check(itp2d_propagate(ctx), "itp2d_propagate");
	t_prop += now_s() - t0;
}

void ITPSystem::orthonormalize() {
	const double t0 = now_s();
	int bi = -1;
	double bv = 0;
	long long c0 = 0, c1 = 0;
	const bool cholesky_between = p.fp32_canonical_every > 1 && p.fp32_between == ITP2D_BETWEEN_CHOLESKY;
	if (precision == ITP2D_FP32) {
		bool early;
		if (cholesky_between)
			early = canonical_prev.empty() ||
					!(wanted_change(canonical_last, canonical_prev, canonical_step_last - canonical_step_prev) < 1e-2);
		else
			early = energies.size() < 2 ||
					!(wanted_change(energies[energies.size() - 1], energies[energies.size() - 2], 1) < 1e-2);
		check(itp2d_set_fp32_eig_tolerance(ctx, early ? 0.05 : 1e-3), "itp2d_set_fp32_eig_tolerance");
	}
	int algo = p.ortho_algorithm;
	if (cholesky_pending && precision == ITP2D_FP64) {
		// the first FP64 iteration after the FP32 form's switch: its task is to
		// make the FP32-accurate states orthonormal in FP64, which a canonical
		// step would do by rotating close pairs (a spurious energy change
		// that the next step undoes); the canonical steps that follow decide
		// convergence
		algo = ITP2D_ORTHO_CHOLESKY;
		cholesky_pending = false;
	}
	itp2d_orthonormalization_counts(ctx, &c0, nullptr, nullptr);
	int st = itp2d_orthonormalize(ctx, algo, &bi, &bv);
	itp2d_orthonormalization_counts(ctx, &c1, nullptr, nullptr);
	last_ortho_canonical = c1 > c0;
	if (st == ITP2D_OK && ritz_pending && precision == ITP2D_FP64) {
		ritz_pending = false;
		st = itp2d_rayleigh_ritz(ctx, nullptr);
		if (st == ITP2D_OK) ritz_steps++;
	}
	t_ortho += now_s() - t0;
	orthonormalized(st, bi, bv);
}

// The outcome of an orthonormalisation: itpsystem.cpp:258-289.
void ITPSystem::orthonormalized(int st, int bi, double bv) {
	if (st == ITP2D_OK) return;
	if (st == ITP2D_E_NONPOSITIVE_EIGENVALUE) {
		// itpsystem.cpp:264-281: shrink eps and restart from noise, or stop.
		error_text = NonPositiveEigenvalue(bi, bv).what();
		if (p.recover) {
			change_time_step();
			init_states();
		} else {
			error_flag = true;
			finish();
		}
		return;
	}
	if (st == ITP2D_E_NONNORMAL_EIGENVALUE) error_text = NonNormalEigenvalue(bi, bv).what();
	else if (st == ITP2D_E_EIGENSOLVER) error_text = EigensolverError(st).what();
	else error_text = status_text("itp2d_orthonormalize", st);
	error_flag = true;
	finish();
}

void ITPSystem::calculate_energies() {
	if (total_step_counter == 0) return;
	const size_t k = (size_t)p.num_states;
	// FP32 form with Cholesky steps: nothing reads the energies of a Cholesky
	// iteration (the switch rule and the eigensolve tolerance compare
	// canonical iterations, the convergence tests run in FP64), so they are
	// not computed; the history repeats the previous iteration's entry
	if (precision == ITP2D_FP32 && p.fp32_canonical_every > 1 && p.fp32_between == ITP2D_BETWEEN_CHOLESKY &&
			!last_ortho_canonical && total_step_counter >= 2 && energies.size() >= (size_t)total_step_counter - 1 &&
			energies[total_step_counter - 2].size() == k) {
		energies.resize(total_step_counter);
		deviations.resize(total_step_counter);
		energies[total_step_counter - 1] = energies[total_step_counter - 2];
		deviations[total_step_counter - 1] = deviations[total_step_counter - 2];
		return;
	}
	std::vector<double> E(k), s(k), r(k);
	const double t0 = now_s();
	check(itp2d_energies(ctx, E.data(), s.data(), r.data(), nullptr), "itp2d_energies");
	t_conv += now_s() - t0;
	store_energies(E.data(), s.data(), r.data());
}

// Sorted (E, sigma, n) tuples and the histories (itpsystem.cpp:473-511).
void ITPSystem::store_energies(const double* E, const double* s, const double* r) {
	const double t0 = now_s();
	const size_t k = (size_t)p.num_states;
	sorted.resize(k);
	for (size_t n = 0; n < k; n++) sorted[n] = Esn(std::make_pair(E[n], s[n]), n);
	std::sort(sorted.begin(), sorted.end());
	if (energies.size() < (size_t)total_step_counter) {
		energies.resize(total_step_counter);
		deviations.resize(total_step_counter);
	}
	std::vector<double>& ne = energies[total_step_counter - 1];
	std::vector<double>& nd = deviations[total_step_counter - 1];
	ne.resize(k);
	nd.resize(k);
	residuals.resize(k);
	for (size_t n = 0; n < k; n++) {
		ne[n] = sorted[n].first.first;
		nd[n] = sorted[n].first.second;
		residuals[n] = r[sorted[n].second];
	}
	if (precision == ITP2D_FP32 && last_ortho_canonical) {
		canonical_prev.swap(canonical_last);
		canonical_last = ne;
		canonical_step_prev = canonical_step_last;
		canonical_step_last = total_step_counter;
	}
	t_conv += now_s() - t0;
}

void ITPSystem::check_timestep_convergence() {
	const double t0 = now_s();
	for (size_t n = 0; n < (size_t)p.num_states; n++)
		if (ts_test->test(*this, n)) timestep_converged[sorted[n].second] = true;
	bool flag = true;
	for (int n = p.ignore_lowest; n < p.ignore_lowest + p.wanted; n++)
		if (!timestep_converged[sorted[n].second]) flag = false;
	all_timestep_converged = flag;
	t_conv += now_s() - t0;
}

void ITPSystem::check_final_convergence() {
	const double t0 = now_s();
	for (size_t n = 0; n < (size_t)p.num_states; n++) finally_converged[sorted[n].second] = final_test->test(*this, n);
	bool flag = true;
	for (int n = p.ignore_lowest; n < p.ignore_lowest + p.wanted; n++)
		if (!finally_converged[sorted[n].second]) flag = false;
	all_finally_converged = flag;
	t_conv += now_s() - t0;
}

size_t ITPSystem::how_many_finally_converged() const {
	return (size_t)std::count(finally_converged.begin(), finally_converged.end(), true);
}

size_t ITPSystem::how_many_timestep_converged() const {
	return (size_t)std::count(timestep_converged.begin(), timestep_converged.end(), true);
}

// itpsystem.cpp:202-233
void ITPSystem::change_time_step() {
	if (!eps_values.empty()) {
		eps = eps_values.front();
		eps_values.pop_front();
		if (eps_values.empty()) exhausting = false;
	} else {
		eps /= p.eps_divisor;
	}
	if (eps < p.min_eps) {
		error_text = "minimum time step reached";
		error_flag = true;
		finish();
		return;
	}
	check(itp2d_set_time_step(ctx, eps), "itp2d_set_time_step");
	eps_history.emplace_back(total_step_counter + 1, eps);
	step_counter = 0;
	all_timestep_converged = false;
	std::fill(timestep_converged.begin(), timestep_converged.end(), false);
}

// FP32 form: once every wanted state's energy changes by less than the switch
// threshold per step (the FP32 sweep floor), continue in FP64, which refines
// the eigenpairs to the FP64 fixed point.
// The FP32 form switches to FP64 once every wanted energy changes by less than
// fp32_switch per step, once the largest change is within kFp32FloorUlps
// single-precision roundings of the largest wanted energy and has stopped
// decreasing since the previous comparison, or once it has not decreased for
// a few comparisons (the FP32 noise floor lies above fp32_switch).
// With Lowdin steps between canonical ones (fp32_canonical_every > 1) the
// rule skips the Lowdin iterations (a Lowdin step does not rotate within the
// subspace, so its per-state energy changes understate the subspace's
// progress and would end the phase early) and two stalled canonical
// iterations end the FP32 phase.
//
// The eigensolve tolerance of the FP32 canonical steps is loose (largest
// rotation tangent 0.05) while the energies still move by more than 1e-2 per
// step: the basis those steps produce is replaced on the next step anyway.
//
// The change is taken over kFp32Span iterations. With Cholesky steps between
// canonical ones the per-state energies of a Cholesky step are those of a
// Gram-Schmidt basis of the subspace, not of its Ritz-like canonical basis,
// so the rule compares each canonical iteration with the previous canonical
// one (the change divided by the iterations between them).
void ITPSystem::maybe_switch_precision() {
	if (precision != ITP2D_FP32 || !(p.fp32_switch > 0) || energies.size() < 2) return;
	const bool between = p.fp32_canonical_every > 1;
	if (between && !last_ortho_canonical) return;
	if (between && p.fp32_between == ITP2D_BETWEEN_CHOLESKY) {
		if (canonical_prev.empty()) return;
		fp32_compare_with(canonical_last, canonical_prev, 2, canonical_step_last - canonical_step_prev);
		return;
	}
	const size_t n = energies.size();
	const size_t want = p.fp32_switch_span > 0 ? (size_t)p.fp32_switch_span : kFp32Span;
	const int span = (int)std::min<size_t>(want, n - 1);
	fp32_compare_with(energies[n - 1], energies[n - 1 - span], between ? 2 : 3, span);
}

// Largest change per iteration of the wanted sorted energies between a and b,
// taken `steps` iterations apart (infinite if any is NaN).
double ITPSystem::wanted_change(const std::vector<double>& a, const std::vector<double>& b, int steps) const {
	double worst = 0.0;
	for (int n = p.ignore_lowest; n < p.ignore_lowest + p.wanted; n++) {
		const double d = std::fabs(a[n] - b[n]);
		worst = (d >= 0.0) ? std::max(worst, d) : INFINITY;  // NaN never counts as converged
	}
	return worst / std::max(steps, 1);
}

void ITPSystem::fp32_compare_with(const std::vector<double>& a, const std::vector<double>& b, int stall_limit,
		int steps) {
	const double worst = wanted_change(a, b, steps);
	const double prev = fp32_last;
	fp32_last = worst;
	// near the FP32 noise floor (kFp32FloorUlps single-precision roundings of
	// the largest wanted energy) a change that has stopped decreasing (within
	// 10 %) means the FP32 phase has reached that floor; a slowly converging
	// change still decreases
	double emax = 0.0;
	for (int n = p.ignore_lowest; n < p.ignore_lowest + p.wanted; n++) emax = std::max(emax, std::fabs(a[n]));
	// (a span of 1, the consecutive-iteration rule, relies on the stall test alone)
	const bool at_floor = p.fp32_switch_span != 1 && worst < kFp32FloorUlps * 0x1p-24 * emax && worst > 0.9 * prev;
	if (!(worst < p.fp32_switch) && !at_floor) {
		if (worst < fp32_best) {
			fp32_best = worst;
			fp32_stall = 0;
			return;
		}
		if (++fp32_stall < stall_limit) return;
	}
	check(itp2d_set_precision(ctx, ITP2D_FP64), "itp2d_set_precision");
	precision = ITP2D_FP64;
	check(itp2d_set_time_step(ctx, eps), "itp2d_set_time_step");
	step_counter = 0;
	all_timestep_converged = false;
	ritz_pending = p.switch_rayleigh_ritz != 0;
	cholesky_pending = p.fp32_canonical_every > 1 && p.fp32_between == ITP2D_BETWEEN_CHOLESKY;
	std::fill(timestep_converged.begin(), timestep_converged.end(), false);
}

// itpsystem.cpp:407-470
void ITPSystem::step() {
	if (!step_begin()) return;
	propagate();
	check_save_flag();
	orthonormalize();
	check_save_flag();
	calculate_energies();
	check_save_flag();
	step_end();
	check_save_flag();
}

// The abort flag raised by a signal handler ends the solve with the error
// flag set (itpsystem.cpp:409-415).
bool ITPSystem::check_abort_flag() {
	if (abort_flag == nullptr || !*abort_flag) return false;
	if (!finished) {
		error_text = "aborted: the abort flag was raised";
		error_flag = true;
		finish();
	}
	return true;
}

// itpsystem.cpp:236-241
void ITPSystem::check_save_flag() {
	if (save_flag != nullptr && *save_flag) {
		save_states();
		*save_flag = 0;
	}
}

// ITPSystem::save_states(sort = true) (itpsystem.cpp:374-389): the states in
// storage order with the storage indices in ascending energy (nullptr before
// the first energies), handed to the save callback.
void ITPSystem::save_states() {
	saves++;
	if (save_fn == nullptr) return;
	const size_t k = (size_t)p.num_states, n = (size_t)p.sx * p.sy;
	std::vector<double> host(2 * k * n);
	download_states(host.data());
	std::vector<int> order;
	if (sorted.size() == k)
		for (size_t i = 0; i < k; i++) order.push_back((int)sorted[i].second);
	save_fn(save_user, host.data(), order.empty() ? nullptr : order.data(), p.num_states, p.sx, p.sy,
			total_step_counter);
}

// Iterations on the device until the time-step test holds
// (itp2d_run_device_loop), then the host's final test and time-step
// schedule exactly as after a step() (itpsystem.cpp:454-466). Only for the
// FP64 sweeps, a time-step test of the four single-limit kinds and without
// eps exhaustion (which changes eps every step); otherwise one step().
void ITPSystem::run_device_phase() {
	if (finished || check_abort_flag()) return;
	check_save_flag();
	const auto spec = parse_parameter_string(p.timestep_test);
	static const char* names[] = {"abschange", "relchange", "absstdev", "relstdev"};
	int test = -1;
	for (int i = 0; i < 4; i++)
		if (spec.first == names[i]) test = i;
	const size_t npar = spec.second.size();
	const bool ok_params = (test < 2 && npar == 1) || (test >= 2 && (npar == 1 || npar == 2));
	int remaining = p.max_steps - total_step_counter;
	if (precision != ITP2D_FP64 || test < 0 || !ok_params || exhausting || remaining < 1) {
		step();
		return;
	}
	const double limit = spec.second[0], diff = npar == 2 ? spec.second[1] : 0.0;
	// The device loop sees no host flag: with flags registered it runs in
	// chunks of at most kFlagChunk iterations and the flags are read between.
	if ((abort_flag != nullptr || save_flag != nullptr) && remaining > kFlagChunk) remaining = kFlagChunk;
	const size_t k = (size_t)p.num_states;
	std::vector<int> flags(k);
	for (size_t i = 0; i < k; i++) flags[i] = timestep_converged[i] ? 1 : 0;
	const double* pe = energies.empty() || energies.back().empty() ? nullptr : energies.back().data();
	const double* ps = pe ? deviations.back().data() : nullptr;
	std::vector<double> E(k), S(k), E0(k), S0(k);
	std::vector<int> idx(k);
	int iters = 0, st = ITP2D_OK;
	if (total_step_counter == 0) t_start = now_s();
	const double t0 = now_s();
	check(itp2d_run_device_loop(ctx, remaining, test, limit, diff, p.ignore_lowest, p.wanted, pe, ps, flags.data(),
				  &iters, &st, E.data(), S.data(), idx.data(), E0.data(), S0.data()),
			"itp2d_run_device_loop");
	t_prop += now_s() - t0;
	device_iterations += iters;
	if (iters == 0) return;
	total_step_counter += iters;
	step_counter += iters;
	// history: the last two iterations (the ones the tests read); the
	// intermediate iterations' energies stayed on the device
	energies.resize(total_step_counter);
	deviations.resize(total_step_counter);
	if (iters >= 2 || !pe) {
		energies[total_step_counter - 2 >= 0 ? total_step_counter - 2 : 0] = E0;
		deviations[total_step_counter - 2 >= 0 ? total_step_counter - 2 : 0] = S0;
	}
	energies.back() = E;
	deviations.back() = S;
	sorted.resize(k);
	for (size_t n = 0; n < k; n++) sorted[n] = Esn(std::make_pair(E[n], S[n]), (size_t)idx[n]);
	residuals.assign(k, 0.0);
	for (size_t i = 0; i < k; i++) timestep_converged[i] = flags[i] != 0;
	if (st != ITP2D_OK) {
		orthonormalized(st, -1, 0.0);
		return;
	}
	bool all = true;
	for (int n = p.ignore_lowest; n < p.ignore_lowest + p.wanted; n++)
		if (!timestep_converged[sorted[n].second]) all = false;
	all_timestep_converged = all;
	if (all_timestep_converged) {
		check_final_convergence();
		if (all_finally_converged) {
			finish();
			return;
		}
		change_time_step();
	}
}

bool ITPSystem::step_begin() {
	if (finished || check_abort_flag()) return false;
	if (total_step_counter == 0) t_start = now_s();
	if (total_step_counter >= p.max_steps) {
		error_text = "maximum number of total steps reached";
		error_flag = true;
		finish();
		return false;
	}
	step_counter++;
	total_step_counter++;
	return true;
}

void ITPSystem::energies_computed(const double* E, const double* sigma, const double* residual) {
	store_energies(E, sigma, residual);
	step_end();
}

// The convergence tests and time-step schedule after the energies.
void ITPSystem::step_end() {
	if (finished) return;
	const bool was_fp32 = precision == ITP2D_FP32;
	maybe_switch_precision();
	if (was_fp32) return;  // convergence tests run on the FP64 refinement
	check_timestep_convergence();
	if (all_timestep_converged) {
		check_final_convergence();
		if (all_finally_converged) {
			finish();
			return;
		}
		change_time_step();
	} else if (exhausting) {
		change_time_step();
	}
}

void ITPSystem::finish() {
	if (finished) return;
	finished = true;
	if (total_step_counter > 0) t_total = now_s() - t_start;
}

void ITPSystem::reset(const double* init) {
	finished = error_flag = false;
	all_timestep_converged = all_finally_converged = false;
	exhausting = p.exhaust_eps != 0;
	total_step_counter = step_counter = 0;
	fp32_best = INFINITY;
	fp32_last = INFINITY;
	ritz_pending = false;
	cholesky_pending = false;
	ritz_steps = 0;
	fp32_stall = 0;
	canonical_last.clear();
	canonical_prev.clear();
	canonical_step_last = canonical_step_prev = 0;
	t_total = t_prop = t_ortho = t_conv = 0;
	energies.clear();
	deviations.clear();
	sorted.clear();
	residuals.clear();
	error_text.clear();
	std::fill(timestep_converged.begin(), timestep_converged.end(), false);
	std::fill(finally_converged.begin(), finally_converged.end(), false);
	eps_values.clear();
	for (int i = 0; i < p.num_eps; i++) eps_values.push_back(p.eps[i]);
	if (!eps_values.empty()) {
		eps = eps_values.front();
		eps_values.pop_front();
	} else {
		eps = 0.5;
	}
	eps_history.assign(1, std::make_pair(1, eps));
	if (precision != p.precision) {
		check(itp2d_set_precision(ctx, p.precision), "itp2d_set_precision");
		precision = p.precision;
	}
	check(itp2d_set_time_step(ctx, eps), "itp2d_set_time_step");
	// the FP32 form's canonical schedule restarts with the solve
	check(itp2d_set_fp32_orthonormalization(ctx, p.fp32_canonical_every), "itp2d_set_fp32_orthonormalization");
	check(itp2d_set_fp32_canonical_delay(ctx, p.fp32_canonical_delay), "itp2d_set_fp32_canonical_delay");
	if (init) {
		initial_states.clear();  // a later recovery re-randomises like the reference
		check(itp2d_upload_states(ctx, init), "itp2d_upload_states");
		return;
	}
	init_states();
}

void ITPSystem::download_states(double* out) { check(itp2d_download_states(ctx, out), "itp2d_download_states"); }

void ITPSystem::times(double* t) {
	double ms[5];
	check(itp2d_phase_times(ctx, ms), "itp2d_phase_times");
	t[0] = finished ? t_total : (total_step_counter > 0 ? now_s() - t_start : 0.0);
	t[1] = t_prop;
	t[2] = t_ortho;
	t[3] = ms[1] * 1e-3;
	t[4] = ms[2] * 1e-3;
	t[5] = ms[3] * 1e-3;
	t[6] = t_conv;
}

}  // namespace itp2d

// ---------------- C ABI (include/itp2d_host.h) ----------------

struct itp2d_system {
	itp2d::ITPSystem* sys = nullptr;
	std::string err;
};

extern "C" {

void itp2d_parameters_default(itp2d_parameters* p) {
	std::memset(p, 0, sizeof(*p));
	p->sx = p->sy = 64;
	p->length = 12;
	p->boundary = ITP2D_PERIODIC;
	p->B = 0;
	p->halforder = 5;
	p->num_states = 25;
	p->wanted = 16;
	p->ignore_lowest = 0;
	p->num_eps = 0;
	p->eps_divisor = 5.0;
	p->exhaust_eps = 0;
	p->max_steps = 50;
	p->min_eps = 1e-9;
	p->seed = 0x20120131UL;
	p->ortho_algorithm = ITP2D_ORTHO_DEFAULT;
	p->recover = 0;
	p->precision = ITP2D_FP64;
	p->fp32_switch = 0.0;
	p->fp32_canonical_every = 0;
	p->fp32_between = ITP2D_BETWEEN_LOWDIN;
	p->switch_rayleigh_ritz = 0;
	p->fp32_switch_span = 0;
	p->fp32_eig_sweeps = 0;
	p->fp32_canonical_delay = 0;
	p->fp64_engine = ITP2D_FP64_DMMA;
	std::strcpy(p->potential, "harmonic");
	std::strcpy(p->timestep_test, "relstdev(1e-3,1e-4)");
	std::strcpy(p->final_test, "relstdev(1e-3,0)");
}

int itp2d_system_create(const itp2d_parameters* p, const double* extra, const double* init, void* stream,
		itp2d_system** out) {
	if (!p || !out) return ITP2D_E_INVALID;
	*out = nullptr;
	itp2d_system* s = new itp2d_system();
	try {
		itp2d::Parameters P;
		P.raw() = *p;
		const size_t G = (size_t)p->sx * (size_t)p->sy;
		if (extra) P.user_potential.assign(extra, extra + G);
		if (init) P.initial_states.assign(init, init + 2 * G * (size_t)p->num_states);
		s->sys = new itp2d::ITPSystem(P, stream);
	} catch (itp2d::DeviceError& e) {
		const int st = e.status;
		delete s;
		return st;
	} catch (std::exception&) {
		delete s;
		return ITP2D_E_INVALID;
	}
	*out = s;
	return ITP2D_OK;
}

int itp2d_system_destroy(itp2d_system* s) {
	if (!s) return ITP2D_E_INVALID;
	delete s->sys;
	delete s;
	return ITP2D_OK;
}

int itp2d_system_reset(itp2d_system* s, const double* init) {
	if (!s || !s->sys) return ITP2D_E_INVALID;
	try {
		s->sys->reset(init);
	} catch (itp2d::DeviceError& e) {
		s->err = e.what();
		return e.status;
	} catch (std::exception& e) {
		s->err = e.what();
		return ITP2D_E_INVALID;
	}
	return ITP2D_OK;
}

int itp2d_system_step(itp2d_system* s) {
	if (!s || !s->sys) return ITP2D_E_INVALID;
	try {
		s->sys->step();
	} catch (itp2d::DeviceError& e) {
		s->err = e.what();
		return e.status;
	} catch (std::exception& e) {
		s->err = e.what();
		return ITP2D_E_INVALID;
	}
	return ITP2D_OK;
}

int itp2d_system_run(itp2d_system* s, int max_iterations) {
	if (!s || !s->sys) return ITP2D_E_INVALID;
	for (int i = 0; i < max_iterations && !s->sys->is_finished(); i++) {
		const int st = itp2d_system_step(s);
		if (st != ITP2D_OK) return st;
	}
	return ITP2D_OK;
}

int itp2d_system_run_device(itp2d_system* s, int max_phases) {
	if (!s || !s->sys) return ITP2D_E_INVALID;
	try {
		for (int i = 0; i < max_phases && !s->sys->is_finished(); i++) s->sys->run_device_phase();
	} catch (itp2d::DeviceError& e) {
		s->err = e.what();
		return e.status;
	} catch (std::exception& e) {
		s->err = e.what();
		return ITP2D_E_INVALID;
	}
	return ITP2D_OK;
}

int itp2d_system_device_iterations(const itp2d_system* s) { return s && s->sys ? s->sys->device_iterations : -1; }

int itp2d_system_is_finished(const itp2d_system* s) { return s && s->sys && s->sys->is_finished() ? 1 : 0; }
int itp2d_system_error_flag(const itp2d_system* s) { return s && s->sys && s->sys->get_error_flag() ? 1 : 0; }
int itp2d_system_total_steps(const itp2d_system* s) { return s && s->sys ? s->sys->get_total_step_counter() : -1; }
int itp2d_system_num_converged(const itp2d_system* s) {
	return s && s->sys ? (int)s->sys->how_many_finally_converged() : -1;
}
double itp2d_system_eps(const itp2d_system* s) { return s && s->sys ? s->sys->get_eps() : 0.0; }
int itp2d_system_in_fp32(const itp2d_system* s) { return s && s->sys && s->sys->in_fp32() ? 1 : 0; }

int itp2d_system_energies(const itp2d_system* s, double* E, double* sigma, double* residual, int* index) {
	if (!s || !s->sys) return -1;
	const auto& e = s->sys->get_energies();
	if (e.empty()) return 0;
	const auto& d = s->sys->get_standard_deviations();
	const size_t k = e.back().size();
	for (size_t n = 0; n < k; n++) {
		if (E) E[n] = e.back()[n];
		if (sigma) sigma[n] = d.back()[n];
		if (residual) residual[n] = s->sys->get_residuals()[n];
		if (index) index[n] = (int)s->sys->get_sorted_index(n);
	}
	return (int)k;
}

int itp2d_system_energy_history(const itp2d_system* s, int step, double* E) {
	if (!s || !s->sys) return -1;
	const auto& e = s->sys->get_energies();
	if (step < 0 || (size_t)step >= e.size()) return 0;
	std::copy(e[step].begin(), e[step].end(), E);
	return (int)e[step].size();
}

int itp2d_system_download_states(itp2d_system* s, double* out) {
	if (!s || !s->sys || !out) return ITP2D_E_INVALID;
	try {
		s->sys->download_states(out);
	} catch (itp2d::DeviceError& e) {
		return e.status;
	}
	return ITP2D_OK;
}

int itp2d_system_times(itp2d_system* s, double* t7) {
	if (!s || !s->sys || !t7) return ITP2D_E_INVALID;
	try {
		s->sys->times(t7);
	} catch (itp2d::DeviceError& e) {
		return e.status;
	}
	return ITP2D_OK;
}

// The reference ITPSystem's datafile with --save final states, written at the
// end of a solve from the driver's records (itpsystem.cpp:69-116 attributes,
// potential and noise; 113-114, 220-226 time steps; 399-402 histories;
// 513-531 final states, energies and run attributes).
static int write_datafile(itp2d_system* s, const char* filename, int clobber, int save_states);

int itp2d_system_write_datafile(itp2d_system* s, const char* filename, int clobber, int save_states) {
	if (!s || !s->sys || !filename) return ITP2D_E_INVALID;
	try {
		return write_datafile(s, filename, clobber, save_states);
	} catch (std::bad_alloc&) {
		s->err = "out of host memory";
		return ITP2D_E_OOM;
	} catch (std::exception& e) {
		s->err = e.what();
		return ITP2D_E_INVALID;
	}
}

static int write_datafile(itp2d_system* s, const char* filename, int clobber, int save_states) {
	itp2d::ITPSystem& sys = *s->sys;
	const itp2d_parameters& p = sys.p;
	const itp2d::DataLayout& dl = sys.datalayout();
	const double t0 = itp2d::now_s();
	itp2d_datafile* f = nullptr;
	int st = itp2d_datafile_create(filename, (int)dl.sizex, (int)dl.sizey, dl.dx, clobber, &f);
	auto ok = [&](int status) {
		if (st == ITP2D_OK && status != ITP2D_OK) {
			st = status;
			s->err = itp2d_datafile_last_error();
		}
	};
	if (st != ITP2D_OK) {
		s->err = itp2d_datafile_last_error();
		return st;
	}
	char timestring[32] = "";
	const std::time_t now = std::time(nullptr);
	std::tm utc;
	if (gmtime_r(&now, &utc)) std::strftime(timestring, sizeof timestring, "%Y-%m-%d %H:%M:%SZ", &utc);
	ok(itp2d_datafile_add_attribute_string(f, "program_version", "itp2d_b200"));
	ok(itp2d_datafile_add_attribute_ulong(f, "random_seed", p.seed));
	ok(itp2d_datafile_add_attribute_string(f, "start_time", timestring));
	ok(itp2d_datafile_add_attribute_ulong(f, "num_threads", 1));
	ok(itp2d_datafile_add_attribute_int(f, "num_states", p.num_states));
	ok(itp2d_datafile_add_attribute_int(f, "num_wanted_to_converge", p.wanted));
	ok(itp2d_datafile_add_attribute_int(f, "ignore_lowest", p.ignore_lowest));
	ok(itp2d_datafile_add_attribute_double(f, "grid_length", dl.lenx));
	ok(itp2d_datafile_add_attribute_string(f, "grid_boundary_type",
			p.boundary == ITP2D_DIRICHLET ? "dirichlet" : "periodic"));
	ok(itp2d_datafile_add_attribute_int(f, "operator_splitting_order", 2 * p.halforder));
	ok(itp2d_datafile_add_attribute_string(f, "potential", p.potential));
	ok(itp2d_datafile_add_attribute_string(f, "noise", sys.has_user_noise() ? "user" : "none"));
	ok(itp2d_datafile_add_attribute_string(f, "impurity_type", "N/A"));
	ok(itp2d_datafile_add_attribute_string(f, "impurity_distribution", "N/A"));
	ok(itp2d_datafile_add_attribute_string(f, "impurity_constraint", "none"));
	ok(itp2d_datafile_add_attribute_string(f, "timestep_convergence_test",
			sys.timestep_test().get_description().c_str()));
	ok(itp2d_datafile_add_attribute_string(f, "final_convergence_test",
			sys.final_convergence_test().get_description().c_str()));
	ok(itp2d_datafile_add_attribute_double(f, "magnetic_field_strength", p.B));
	if (!sys.is_null_potential() && sys.get_potential().size() == dl.N)
		ok(itp2d_datafile_write_potential(f, sys.get_potential().data()));
	ok(itp2d_datafile_write_noise_realization(f, nullptr, 0));
	if (!sys.eps_history.empty()) ok(itp2d_datafile_add_attribute_double(f, "initial_time_step", sys.eps_history[0].second));
	for (const auto& e : sys.eps_history) ok(itp2d_datafile_write_time_step_history(f, e.first, e.second));
	const auto& E = sys.get_energies();
	const auto& D = sys.get_standard_deviations();
	for (size_t i = 0; i < E.size(); i++) ok(itp2d_datafile_write_energy_history(f, E[i].data(), (int)E[i].size(), (int)i));
	for (size_t i = 0; i < D.size(); i++)
		ok(itp2d_datafile_write_deviation_history(f, D[i].data(), (int)D[i].size(), (int)i));
	if (save_states && st == ITP2D_OK) {
		const size_t k = (size_t)p.num_states;
		const bool sorted = !E.empty();
		try {
			std::vector<double> states(2 * dl.N * k);
			std::vector<int> order(k);
			for (size_t n = 0; sorted && n < k; n++) order[n] = (int)sys.get_sorted_index(n);
			sys.download_states(states.data());
			ok(itp2d_datafile_write_stateset(f, states.data(), (int)k, sys.get_total_step_counter(),
					sorted ? order.data() : nullptr));
		} catch (itp2d::DeviceError& e) {
			ok(e.status);
			s->err = e.what();
		} catch (std::bad_alloc&) {
			ok(ITP2D_E_OOM);
			s->err = "out of host memory for the states";
		}
	}
	if (!E.empty()) ok(itp2d_datafile_write_energies(f, E.back().data(), (int)E.back().size()));
	if (!D.empty()) ok(itp2d_datafile_write_energy_standard_deviations(f, D.back().data(), (int)D.back().size()));
	ok(itp2d_datafile_add_attribute_int(f, "num_converged", (int)sys.how_many_finally_converged()));
	ok(itp2d_datafile_add_attribute_int(f, "error_flag", sys.get_error_flag() ? 1 : 0));
	ok(itp2d_datafile_add_attribute_int(f, "total_steps_done", sys.get_total_step_counter()));
	double t[7] = {0, 0, 0, 0, 0, 0, 0};
	try {
		sys.times(t);
	} catch (itp2d::DeviceError& e) {
		ok(e.status);
		s->err = e.what();
	}
	ok(itp2d_datafile_add_attribute_double(f, "propagation_time", t[1]));
	ok(itp2d_datafile_add_attribute_double(f, "orthonormalization_time", t[2]));
	ok(itp2d_datafile_add_attribute_double(f, "dotproduct_time", t[3]));
	ok(itp2d_datafile_add_attribute_double(f, "eigensolve_time", t[4]));
	ok(itp2d_datafile_add_attribute_double(f, "lincomb_time", t[5]));
	ok(itp2d_datafile_add_attribute_double(f, "convtest_time", t[6]));
	ok(itp2d_datafile_add_attribute_double(f, "io_time", itp2d::now_s() - t0));
	ok(itp2d_datafile_close(f));
	return st;
}

// Process-wide flags and the handlers that raise them, as the reference's
// program installs them (itp2d.cpp:40-66): the first SIGINT raises the abort
// flag, a second one ends the process at once with status 1; SIGUSR1 raises
// the save flag. Only async-signal-safe calls (write, _exit) in the handlers.
static volatile sig_atomic_t g_abort_flag = 0;
static volatile sig_atomic_t g_save_flag = 0;

static void on_sigint(int) {
	static const char note[] =
			"\nSIGINT: the solve ends at its next step (states saved first if a save callback is set); "
			"a second SIGINT exits at once.\n";
	if (g_abort_flag) _exit(1);
	if (write(STDERR_FILENO, note, sizeof(note) - 1) < 0) {
	}
	g_abort_flag = 1;
}

static void on_sigusr1(int) {
	static const char note[] = "\nSIGUSR1: the states are saved at the next check point; the solve continues.\n";
	if (write(STDERR_FILENO, note, sizeof(note) - 1) < 0) {
	}
	g_save_flag = 1;
}

volatile sig_atomic_t* itp2d_abort_flag(void) { return &g_abort_flag; }
volatile sig_atomic_t* itp2d_save_flag(void) { return &g_save_flag; }

int itp2d_install_signal_handlers(void) {
	struct sigaction a;
	std::memset(&a, 0, sizeof(a));
	sigemptyset(&a.sa_mask);
	a.sa_flags = SA_RESTART;
	a.sa_handler = on_sigint;
	if (sigaction(SIGINT, &a, nullptr) != 0) return ITP2D_E_INVALID;
	a.sa_handler = on_sigusr1;
	if (sigaction(SIGUSR1, &a, nullptr) != 0) return ITP2D_E_INVALID;
	return ITP2D_OK;
}

int itp2d_system_set_flags(itp2d_system* s, volatile sig_atomic_t* abort_flag, volatile sig_atomic_t* save_flag) {
	if (!s || !s->sys) return ITP2D_E_INVALID;
	s->sys->set_flags(abort_flag, save_flag);
	return ITP2D_OK;
}

int itp2d_system_set_save_callback(itp2d_system* s, itp2d_save_states_fn fn, void* user) {
	if (!s || !s->sys) return ITP2D_E_INVALID;
	s->sys->set_save_callback(fn, user);
	return ITP2D_OK;
}

int itp2d_system_saves(const itp2d_system* s) { return s && s->sys ? s->sys->saves : -1; }

const char* itp2d_system_last_error(const itp2d_system* s) {
	if (!s) return "";
	if (!s->err.empty()) return s->err.c_str();
	return s->sys ? s->sys->last_error().c_str() : "";
}

itp2d_ctx* itp2d_system_context(itp2d_system* s) { return s && s->sys ? s->sys->context() : nullptr; }

}  // extern "C"
