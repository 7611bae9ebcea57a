// Native host layer of the itp2d B200 hot path: the reference's driver-level
// API (Parameters, ConvergenceTest, ITPSystem) over the device C ABI
// (include/itp2d_gpu.h). Only the three seams run on the device; the step
// logic, time-step schedule, sorting and convergence tests stay on the host
// exactly as in itpsystem.cpp:202-511 and convergence.cpp:28-199.
#pragma once

#include <csignal>
#include <cmath>
#include <list>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/itp2d_gpu.h"
#include "../../include/itp2d_host.h"

namespace itp2d {

// Exceptions carrying the reference's meaning (exceptions.hpp:37-254).
class GeneralError : public std::runtime_error {
  public:
	explicit GeneralError(const std::string& w) : std::runtime_error(w) {}
};
class ParseError : public std::runtime_error {
  public:
	explicit ParseError(const std::string& s) : std::runtime_error("could not parse parameter string: " + s) {}
};
class NonPositiveEigenvalue : public std::runtime_error {
  public:
	NonPositiveEigenvalue(int n, double v);
	int index;
	double value;
};
class NonNormalEigenvalue : public std::runtime_error {
  public:
	NonNormalEigenvalue(int n, double v);
	int index;
	double value;
};
class EigensolverError : public std::runtime_error {
  public:
	explicit EigensolverError(int status);
};
class DeviceError : public std::runtime_error {
  public:
	DeviceError(const std::string& where, int status);
	int status;
};

// name(v1,v2,...) mini-language of parser.cpp:26-60.
std::pair<std::string, std::vector<double>> parse_parameter_string(const std::string& s);

class ITPSystem;

// convergence.hpp:32-130
class ConvergenceTest {
  public:
	virtual ~ConvergenceTest() {}
	virtual bool test(const ITPSystem& sys, size_t n) const = 0;
	const std::string& get_description() const { return description; }

  protected:
	std::string description;
};

class NoConvergenceTest : public ConvergenceTest {
  public:
	explicit NoConvergenceTest(const std::vector<double>& params);
	bool test(const ITPSystem&, size_t) const override { return false; }
};

class OneStepConvergenceTest : public ConvergenceTest {
  public:
	explicit OneStepConvergenceTest(const std::vector<double>& params);
	bool test(const ITPSystem& sys, size_t n) const override;
};

class RelativeEnergyChangeTest : public ConvergenceTest {
  public:
	explicit RelativeEnergyChangeTest(const std::vector<double>& params);
	bool test(const ITPSystem& sys, size_t n) const override;

  private:
	double limit;
};

class AbsoluteEnergyChangeTest : public ConvergenceTest {
  public:
	explicit AbsoluteEnergyChangeTest(const std::vector<double>& params);
	bool test(const ITPSystem& sys, size_t n) const override;

  private:
	double limit;
};

class AbsoluteEnergyDeviationTest : public ConvergenceTest {
  public:
	explicit AbsoluteEnergyDeviationTest(const std::vector<double>& params);
	bool test(const ITPSystem& sys, size_t n) const override;

  private:
	double dev_limit, diff_limit;
};

class RelativeEnergyDeviationTest : public ConvergenceTest {
  public:
	explicit RelativeEnergyDeviationTest(const std::vector<double>& params);
	bool test(const ITPSystem& sys, size_t n) const override;

  private:
	double dev_limit, diff_limit;
};

std::unique_ptr<ConvergenceTest> parse_convergence_description(const std::string& s);

// The cell-centred grid of datalayout.cpp:21-36.
struct DataLayout {
	DataLayout(size_t sx, size_t sy, double dx);
	size_t sizex, sizey, N;
	double dx, lenx, leny;
	std::vector<double> posx, posy;
};

// The potential library of potentialtypes.hpp:96-380 (all 14 types, the
// reference's names, defaults and checks), evaluated on the device.
// Returns false for the null potential.
bool evaluate_potential(const std::string& desc, const DataLayout& dl, std::vector<double>& out);

class Parameters {
  public:
	Parameters();
	void set_recover(bool v) { p.recover = v; }
	void set_random_seed(unsigned long s) { p.seed = s; }
	void define_grid(size_t sx, size_t sy, double lenx, int boundary = ITP2D_PERIODIC);
	void define_external_field(const std::string& ptype, double B = 0);
	void set_num_states(size_t N, size_t wanted, size_t ignore_lowest = 0);
	void set_operator_splitting_halforder(int h) { p.halforder = h; }
	void add_eps_value(double e);
	void set_time_step_divisor(double d) { p.eps_divisor = d; }
	void set_exhaust_eps(bool v) { p.exhaust_eps = v; }
	void set_bailout_limits(int max_steps, double min_time_step);
	void set_ortho_algorithm(int a) { p.ortho_algorithm = a; }
	void set_timestep_convergence_test(const std::string& s);
	void set_final_convergence_test(const std::string& s);
	void set_precision(int prec, double fp32_switch = 1e-7);
	void set_user_potential(const std::vector<double>& v) { user_potential = v; }
	void set_initial_states(const std::vector<double>& v) { initial_states = v; }
	const itp2d_parameters& raw() const { return p; }
	itp2d_parameters& raw() { return p; }
	std::vector<double> user_potential;   // added to the potential (the user noise hook)
	std::vector<double> initial_states;   // k*sy*sx interleaved complex, empty = random

  private:
	itp2d_parameters p;
};

class ITPSystem {
  public:
	typedef std::pair<std::pair<double, double>, size_t> Esn;  // ((E, sigma), storage index)
	ITPSystem(const Parameters& params, void* cuda_stream = nullptr);
	~ITPSystem();
	ITPSystem(const ITPSystem&) = delete;
	ITPSystem& operator=(const ITPSystem&) = delete;

	void step();
	// step() in pieces, for a driver that runs many systems through the
	// batched device calls (itp2d_batch_*): step_begin() (false: finished),
	// the device work of propagate / orthonormalize / energies done by the
	// caller, then orthonormalized() with the orthonormalisation's status and
	// energies_computed() with the per-state energies in storage order.
	bool step_begin();
	// Iterations on the device until the time-step test holds, then the
	// host's final test and time-step schedule (FP64 sweeps; otherwise one
	// step()).
	void run_device_phase();
	int device_iterations = 0;  // iterations run by run_device_phase
	void orthonormalized(int status, int bad_index, double bad_value);
	void energies_computed(const double* E, const double* sigma, const double* residual);
	void finish();
	void reset(const double* init_states);
	bool is_finished() const { return finished; }
	bool get_error_flag() const { return error_flag; }
	int get_total_step_counter() const { return total_step_counter; }
	int get_step_counter() const { return step_counter; }
	double get_eps() const { return eps; }
	bool in_fp32() const { return precision == ITP2D_FP32; }
	size_t how_many_finally_converged() const;
	size_t how_many_timestep_converged() const;
	bool is_timestep_converged(size_t index) const { return timestep_converged[index]; }
	const std::vector<std::vector<double>>& get_energies() const { return energies; }
	const std::vector<std::vector<double>>& get_standard_deviations() const { return deviations; }
	double get_sorted_energy(size_t n) const { return sorted[n].first.first; }
	double get_sorted_deviation(size_t n) const { return sorted[n].first.second; }
	size_t get_sorted_index(size_t n) const { return sorted[n].second; }
	const std::vector<double>& get_residuals() const { return residuals; }
	const std::vector<double>& get_potential() const { return V; }
	bool is_null_potential() const { return null_potential; }
	bool has_user_noise() const { return user_noise; }  // an extra potential was added
	const ConvergenceTest& timestep_test() const { return *ts_test; }
	const ConvergenceTest& final_convergence_test() const { return *final_test; }
	const DataLayout& datalayout() const { return dl; }
	const std::string& last_error() const { return error_text; }
	itp2d_ctx* context() { return ctx; }
	void download_states(double* out);
	void times(double* t7);
	// The flags a signal handler raises (ITPSystem's abort_flagptr and
	// save_flagptr, itpsystem.hpp:59-62); nullptr disables each.
	void set_flags(volatile sig_atomic_t* abort, volatile sig_atomic_t* save) {
		abort_flag = abort;
		save_flag = save;
	}
	// Where save_states writes (the reference's datafile, itpsystem.cpp:374-389).
	void set_save_callback(itp2d_save_states_fn fn, void* user) {
		save_fn = fn;
		save_user = user;
	}
	int saves = 0;       // save_states calls made
	// (first step with the value, time step) at the start and at every change
	// of the time step: the datafile's time_step_history (itpsystem.cpp:113-114,
	// 220-226)
	std::vector<std::pair<int, double>> eps_history;
	int ritz_steps = 0;  // Rayleigh-Ritz steps taken (switch_rayleigh_ritz)
	const itp2d_parameters p;

  private:
	void propagate();
	void orthonormalize();
	void calculate_energies();
	void store_energies(const double* E, const double* sigma, const double* residual);
	void step_end();
	void check_timestep_convergence();
	void check_final_convergence();
	void change_time_step();
	void init_states();
	void maybe_switch_precision();
	void fp32_compare_with(const std::vector<double>& a, const std::vector<double>& b, int stall_limit, int steps);
	double wanted_change(const std::vector<double>& a, const std::vector<double>& b, int steps) const;
	void check(int status, const char* where);
	bool check_abort_flag();
	void check_save_flag();
	void save_states();

	DataLayout dl;
	volatile sig_atomic_t* abort_flag = nullptr;
	volatile sig_atomic_t* save_flag = nullptr;
	itp2d_save_states_fn save_fn = nullptr;
	void* save_user = nullptr;
	std::unique_ptr<ConvergenceTest> ts_test, final_test;
	std::vector<double> V;
	bool null_potential = true;
	bool user_noise = false;
	std::vector<double> initial_states;
	itp2d_ctx* ctx = nullptr;
	int precision = ITP2D_FP64;
	bool finished = false, error_flag = false;
	bool all_timestep_converged = false, all_finally_converged = false;
	bool exhausting;
	int total_step_counter = 0, step_counter = 0;
	double fp32_best = INFINITY;  // smallest per-step energy change seen in the FP32 form
	int fp32_stall = 0;           // FP32 steps since that change last decreased
	double fp32_last = INFINITY;  // the previous comparison's change
	bool ritz_pending = false;    // a Rayleigh-Ritz step after the next FP64 orthonormalisation
	bool cholesky_pending = false;  // the next FP64 orthonormalisation by Cholesky (after the switch)
	bool last_ortho_canonical = true;               // the last orthonormalisation's form
	// sorted energies of the last two canonical FP32 iterations and their steps
	std::vector<double> canonical_last, canonical_prev;
	int canonical_step_last = 0, canonical_step_prev = 0;
	double eps = 0;
	std::list<double> eps_values;
	std::vector<Esn> sorted;
	std::vector<std::vector<double>> energies, deviations;
	std::vector<double> residuals;
	std::vector<bool> timestep_converged, finally_converged;
	unsigned long rng_state;
	double t_total = 0, t_prop = 0, t_ortho = 0, t_conv = 0;
	double t_start = 0;
	std::string error_text;
};

}  // namespace itp2d
