/*
 * itp2d_host.h -- C ABI of the native ITP driver that runs on top of
 * itp2d_gpu.h. It mirrors the reference ITPSystem (itpsystem.hpp:55-156):
 * Parameters in, step() until finished, sorted energies and deviations out.
 * The C++ classes behind it (itp2d_b200/host/itp2d_host.hpp) keep the
 * reference names: Parameters, ConvergenceTest and its six tests, ITPSystem.
 */
#ifndef ITP2D_HOST_H
#define ITP2D_HOST_H

#include <signal.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Mirrors the Parameters setters of parameters.hpp:37-211 that the hot path
 * reads. Strings use the reference's mini-language, for example
 * "harmonic(1)", "abschange(1e-10)", "relstdev(1e-3,1e-4)" (parser.cpp:26-60,
 * convergence.cpp:28-55). */
typedef struct {
	int sx, sy;
	double length;          /* lenx; dx = length / sx (parameters.hpp:97) */
	int boundary;           /* ITP2D_PERIODIC or ITP2D_DIRICHLET */
	double B;
	int halforder;          /* order = 2 * halforder */
	int num_states;         /* N */
	int wanted;             /* needed_to_converge */
	int ignore_lowest;
	int num_eps;            /* leading time steps (add_eps_value) */
	double eps[16];
	double eps_divisor;
	int exhaust_eps;
	int max_steps;
	double min_eps;
	unsigned long seed;
	int ortho_algorithm;    /* ITP2D_ORTHO_DEFAULT / ITP2D_ORTHO_HIGHMEM */
	int recover;
	int precision;          /* ITP2D_FP64 or ITP2D_FP32 (sweeps; FP64 refinement, see below) */
	double fp32_switch;     /* FP32 form: switch sweeps to FP64 once every wanted state has
	                           |dE| per step below this (0: never switch) */
	char potential[128];
	char timestep_test[128];
	char final_test[128];
	int fp32_canonical_every; /* FP32 form: canonical orthonormalisation on every n-th
	                             step, fp32_between steps in between
	                             (itp2d_set_fp32_orthonormalization); 0: always canonical */
	int fp32_between;         /* ITP2D_BETWEEN_LOWDIN (0) or ITP2D_BETWEEN_CHOLESKY
	                             (itp2d_set_fp32_between); with Cholesky the energies of the
	                             Cholesky iterations are not computed (their history entries
	                             repeat the previous ones) and the first FP64 iteration after
	                             the switch is a Cholesky step too */
	int switch_rayleigh_ritz; /* FP32 form: 1 = one Rayleigh-Ritz step (itp2d_rayleigh_ritz)
	                             after the first FP64 orthonormalisation of the refinement */
	int fp32_switch_span;     /* FP32 form: iterations over which the switch rule reads the
	                             energy change (0: 3; 1: consecutive iterations with the
	                             stall test alone) */
	int fp32_eig_sweeps;      /* FP32 form: at most this many Jacobi sweeps in a canonical
	                             step, finished by a Cholesky step
	                             (itp2d_set_fp32_eig_sweeps); 0: full eigensolve */
	int fp32_canonical_delay; /* FP32 form: the first canonical step comes this many
	                             iterations later than fp32_canonical_every puts it
	                             (itp2d_set_fp32_canonical_delay) */
	int fp64_engine;        /* ITP2D_FP64_DMMA (0) or ITP2D_FP64_INT8 for the
	                             rotations of FP64 states (itp2d_set_fp64_engine) */
} itp2d_parameters;

typedef struct itp2d_system itp2d_system;

/* Reference defaults (parameters.cpp:25-55). */
void itp2d_parameters_default(itp2d_parameters* p);

/* Builds the system: grid, potential (+ optional extra_potential array added
 * like the reference's user noise hook, itpsystem.cpp:63-64), evolution
 * operator tables, and initial states (init_states: num_states*sy*sx
 * interleaved complex doubles, or NULL for seeded complex Gaussian noise
 * normalised per state, stateset.cpp:124-131). cuda_stream may be NULL. */
int itp2d_system_create(const itp2d_parameters* p, const double* extra_potential, const double* init_states,
		void* cuda_stream, itp2d_system** out);
int itp2d_system_destroy(itp2d_system* s);

/* Restarts the solve from new initial states (NULL: fresh seeded noise) with
 * the parameters' first time step, precision and empty histories, reusing
 * every device allocation. */
int itp2d_system_reset(itp2d_system* s, const double* init_states);

/* One ITP iteration, ITPSystem::step (itpsystem.cpp:407-470). */
int itp2d_system_step(itp2d_system* s);
/* step() until finished or max_iterations more iterations were taken;
 * returns ITP2D_OK (check itp2d_system_error_flag). */
int itp2d_system_run(itp2d_system* s, int max_iterations);

/* Like itp2d_system_run, with the FP64 iterations run on the device: each
 * phase is one itp2d_run_device_loop (iterations without host round trips
 * until the time-step test holds) followed by the driver's final test and
 * time-step schedule; the FP32 phase of the mixed form and time-step tests
 * other than abschange, relchange, absstdev and relstdev take step() instead.
 * The energy history keeps only the last two iterations of each device phase.
 * Runs at most max_phases phases. No reference counterpart. */
int itp2d_system_run_device(itp2d_system* s, int max_phases);
/* Iterations taken inside device phases. */
int itp2d_system_device_iterations(const itp2d_system* s);

int itp2d_system_is_finished(const itp2d_system* s);
int itp2d_system_error_flag(const itp2d_system* s);
int itp2d_system_total_steps(const itp2d_system* s);
int itp2d_system_num_converged(const itp2d_system* s);
double itp2d_system_eps(const itp2d_system* s);
/* 1 while the sweeps run in FP32 (FP32 form before its switch to FP64). */
int itp2d_system_in_fp32(const itp2d_system* s);

/* Latest energies sorted ascending with their deviations and storage
 * indices (ITPSystem::calculate_energies, itpsystem.cpp:473-511). Returns the
 * count (0 before the first step). residual may be NULL. */
int itp2d_system_energies(const itp2d_system* s, double* E, double* sigma, double* residual, int* index);
/* Energies of step `step` (0-based) of the history, sorted. */
int itp2d_system_energy_history(const itp2d_system* s, int step, double* E);

int itp2d_system_download_states(itp2d_system* s, double* states);

/* Seconds: [0] total, [1] propagation, [2] orthonormalisation, [3] overlap
 * (dot), [4] eigensolve, [5] lincomb, [6] energies + convergence tests. The
 * device phases [3..5] come from CUDA events. */
int itp2d_system_times(itp2d_system* s, double* t7);

/* ---- Signals (itp2d.cpp:40-66; itpsystem.cpp:236-241,407-415) ----
 * The reference's program traps SIGINT and SIGUSR1 into two process-wide
 * flags that its ITPSystem reads: a raised abort flag ends the solve at the
 * top of the next step with the error flag set; a raised save flag has the
 * states saved at the next check point (after propagation, after the
 * orthonormalisation, after the energies, at the end of a step) and is
 * lowered again. itp2d_install_signal_handlers installs those handlers over
 * this library's own pair of flags (a second SIGINT exits with status 1). */
int itp2d_install_signal_handlers(void);
volatile sig_atomic_t* itp2d_abort_flag(void);
volatile sig_atomic_t* itp2d_save_flag(void);

/* The flags this system reads (ITPSystem's abort_flagptr / save_flagptr,
 * itpsystem.hpp:59-62): any sig_atomic_t the caller owns, or the two above;
 * NULL disables either (the default). While either is set the device
 * phases of itp2d_system_run_device run in chunks of at most 32 iterations
 * and the flags are read between chunks. */
int itp2d_system_set_flags(itp2d_system* s, volatile sig_atomic_t* abort_flag, volatile sig_atomic_t* save_flag);

/* save_states (itpsystem.cpp:374-389) with the datafile replaced by a
 * callback: states in storage order (num_states*sy*sx interleaved complex
 * doubles, valid during the call), order = storage indices by ascending
 * energy (NULL before the first energies), step = iterations taken. */
typedef void (*itp2d_save_states_fn)(void* user, const double* states, const int* order, int num_states, int sx,
		int sy, int step);
int itp2d_system_set_save_callback(itp2d_system* s, itp2d_save_states_fn fn, void* user);
/* save_states calls made so far (with or without a callback). */
int itp2d_system_saves(const itp2d_system* s);

/* Last error message of the driver (exception text), or "". */
const char* itp2d_system_last_error(const itp2d_system* s);

/* The device context owned by the system (for itp2d_gpu.h calls). */
struct itp2d_ctx* itp2d_system_context(itp2d_system* s);

/* ---- Serving loop (no reference counterpart; the reference runs one
 * ITPSystem per process, itp2d.cpp:62-135) ----
 *
 * Solve requests (one itp2d_parameters each, plus optional extra potential and
 * initial states as for itp2d_system_create) are queued as they arrive. Up to
 * max_active of them run at once, each an ITPSystem on its own CUDA stream,
 * so their kernels overlap on the device; a request is admitted when its
 * device footprint (itp2d_ctx_footprint) fits in the part of
 * memory_budget_bytes that the running ones leave free, oldest first among
 * those that fit. A finished request frees its slot and memory at once.
 * Requests larger than the whole budget are refused (ITP2D_E_OOM). */
typedef struct itp2d_server itp2d_server;

typedef struct {
	int status;          /* ITP2D_OK, or the status that ended the solve */
	int error_flag;      /* the driver's error flag (e.g. maximum steps reached) */
	int iterations;      /* ITP iterations taken */
	int converged;       /* states passing the final convergence test */
	int num_energies;    /* entries written to E and sigma (num_states) */
	double t_submit;     /* seconds on a monotonic clock: submission, */
	double t_start;      /* start of the solve (admission), */
	double t_finish;     /* and end of the solve */
	double footprint_bytes;
} itp2d_request_info;

typedef struct {
	int queued, running, peak_running, completed;
	double bytes_in_use, peak_bytes_in_use, budget_bytes;
	double busy_seconds;     /* time with at least one solve running */
	double overlap_seconds;  /* time with two or more solves running at once */
} itp2d_server_stats;

int itp2d_server_create(int max_active, double memory_budget_bytes, itp2d_server** out);
/* Queues a request; *id names it in itp2d_server_wait. The arrays are copied. */
int itp2d_server_submit(itp2d_server* s, const itp2d_parameters* p, const double* extra_potential,
		const double* init_states, long long* id);
/* Waits up to timeout_s seconds for request id; ITP2D_E_TIMEOUT if it has not
 * finished. On success fills info and the sorted energies and deviations
 * (num_states doubles each; either array may be NULL). */
int itp2d_server_wait(itp2d_server* s, long long id, double timeout_s, itp2d_request_info* info, double* E,
		double* sigma);
/* Drops a finished request's record. */
int itp2d_server_forget(itp2d_server* s, long long id);
int itp2d_server_get_stats(itp2d_server* s, itp2d_server_stats* stats);
const char* itp2d_server_last_error(itp2d_server* s);
/* Runs the queued and running requests to the end, then frees the server. */
int itp2d_server_destroy(itp2d_server* s);

/* ---- Batched form (no reference counterpart) ----
 *
 * count independent solves (one itp2d_parameters each, any grid size and
 * state count >= 2; extra_potentials / init_states may be NULL or hold NULL
 * entries) stepped together: every iteration runs the unfinished instances'
 * propagations, overlaps, ONE batched eigensolve launch for all of them, the
 * rotations and the energies (itp2d_batch_* of itp2d_gpu.h), then each
 * instance's own convergence tests and time-step schedule. Instances leave
 * the batch as they finish. */
typedef struct itp2d_batch itp2d_batch;
int itp2d_batch_create(int count, const itp2d_parameters* params, const double* const* extra_potentials,
		const double* const* init_states, itp2d_batch** out);
/* Up to max_iterations batch iterations, fewer when every instance finishes. */
int itp2d_batch_run(itp2d_batch* b, int max_iterations);
/* Instance i: iterations, converged count, error flag, seconds from the
 * batch's start to the instance's finish (t_finish), sorted energies and
 * deviations (num_states doubles each; either array may be NULL). */
int itp2d_batch_result(itp2d_batch* b, int i, itp2d_request_info* info, double* E, double* sigma);
int itp2d_batch_size(const itp2d_batch* b);
int itp2d_batch_finished(const itp2d_batch* b);
int itp2d_batch_stats(const itp2d_batch* b, long long* iterations, double* seconds);
const char* itp2d_batch_last_error(const itp2d_batch* b);
int itp2d_batch_destroy(itp2d_batch* b);

#ifdef __cplusplus
}
#endif

#endif /* ITP2D_HOST_H */
