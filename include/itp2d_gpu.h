/*
 * itp2d_gpu.h -- C ABI of the B200 (sm_100a) implementation of the itp2d
 * imaginary-time-propagation hot path.
 *
 * One context holds one set of k states of an sx*sy grid resident in device
 * memory (state n at offset n*sx*sy, x fastest, complex values), the
 * potential, and the split-operator tables for the current time step. The
 * three seams of the reference driver map to one call each:
 *
 *   ITPSystem::propagate          (itpsystem.cpp:243-256)  -> itp2d_propagate
 *   StateSet::orthonormalize      (stateset.cpp:136-232)   -> itp2d_orthonormalize
 *   ITPSystem::calculate_energies (itpsystem.cpp:473-511)  -> itp2d_energies
 *
 * Conventions: every function returns an int status (ITP2D_OK = 0); no C++
 * exception crosses this boundary. A context is bound to one CUDA stream and
 * is not re-entrant: calls on one context must not overlap (the library
 * serialises them with a per-context mutex). Host arrays are plain doubles:
 * complex values are interleaved (re, im).
 */
#ifndef ITP2D_GPU_H
#define ITP2D_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. The C++ host layer maps them to the reference exceptions
 * (exceptions.hpp:37-254): NONPOSITIVE -> NonPositiveEigenvalue,
 * NONNORMAL -> NonNormalEigenvalue, EIGENSOLVER -> EigensolverError. */
enum {
	ITP2D_OK = 0,
	ITP2D_E_INVALID = 1,                /* bad argument or unsupported size */
	ITP2D_E_CUDA = 2,                   /* a CUDA runtime call failed */
	ITP2D_E_OOM = 3,                    /* device allocation failed */
	ITP2D_E_NONPOSITIVE_EIGENVALUE = 4, /* overlap eigenvalue <= 0 (stateset.cpp:163-167) */
	ITP2D_E_NONNORMAL_EIGENVALUE = 5,   /* overlap eigenvalue not FP_NORMAL (stateset.cpp:168-172) */
	ITP2D_E_EIGENSOLVER = 6,            /* eigensolver did not converge (eigensolver.hpp:80-84) */
	ITP2D_E_TIMEOUT = 7,                /* a bounded device wait ran out */
	ITP2D_E_UNSUPPORTED = 8             /* combination not built (for example a grid size) */
};

/* Boundary conditions, enum BoundaryType of itp2d_common.hpp:50. */
enum { ITP2D_PERIODIC = 0, ITP2D_DIRICHLET = 1 };

/* Arithmetic of the propagation sweeps and energies. */
enum { ITP2D_FP64 = 0, ITP2D_FP32 = 1 };

/* Orthonormalisation algorithm, enum OrthoAlgorithm of itp2d_common.hpp:53.
 * DEFAULT and HIGHMEM select the same out-of-place canonical device path; the
 * argument is accepted for interface compatibility. CHOLESKY (no reference
 * counterpart) orthonormalises in Gram-Schmidt order instead: S = L L^H,
 * psi'_n = sum_{i <= n} conj((L^{-1})_{n,i}) psi_i; the state order is kept and
 * a non-positive pivot of L is reported as ITP2D_E_NONPOSITIVE_EIGENVALUE with
 * the pivot's index and value. */
enum { ITP2D_ORTHO_DEFAULT = 0, ITP2D_ORTHO_HIGHMEM = 1, ITP2D_ORTHO_CHOLESKY = 2 };

/* Transform kinds in the order of enum Transform (transformer.hpp:32-34). */
enum {
	ITP2D_FFT = 0, ITP2D_IFFT, ITP2D_FFTX, ITP2D_IFFTX, ITP2D_FFTY, ITP2D_IFFTY,
	ITP2D_DST, ITP2D_IDST, ITP2D_DSTX, ITP2D_IDSTX, ITP2D_DSTY, ITP2D_IDSTY,
	ITP2D_DCT, ITP2D_IDCT, ITP2D_DCTX, ITP2D_IDCTX, ITP2D_DCTY, ITP2D_IDCTY
};

typedef struct itp2d_ctx itp2d_ctx;

/* Creates a context for num_states states on an sx*sy grid with spacing dx
 * (DataLayout, datalayout.cpp:21-36; Parameters::get_grid_delta,
 * parameters.hpp:97). B is the magnetic field (linear gauge, kinetic.hpp:24-29),
 * halforder the multi-product half order m (MultiProductSplit,
 * multiproductsplit.cpp:23-41; forced to 1 when the potential is null).
 * cuda_stream is a cudaStream_t or NULL for a stream owned by the context.
 * Replaces the allocation part of the ITPSystem constructor
 * (itpsystem.cpp:23-139) and StateSet::StateSet (stateset.cpp:23-44). */
int itp2d_ctx_create(int sx, int sy, double dx, int num_states, int boundary,
		double B, int halforder, int precision, void* cuda_stream,
		itp2d_ctx** out);

/* Frees every device allocation of the context. */
int itp2d_ctx_destroy(itp2d_ctx* ctx);

/* Device bytes a context of these arguments allocates (states, matrices,
 * tables), an upper bound computed without allocating: the admission figure
 * of the serving loop (itp2d_host.h). -1 for invalid arguments. No reference
 * counterpart (the reference allocates host memory in StateSet::StateSet,
 * stateset.cpp:23-44). */
long long itp2d_ctx_footprint(int sx, int sy, int num_states, int boundary, double B, int halforder);

/* Device bytes the context holds (-1 for NULL). */
long long itp2d_ctx_device_bytes(itp2d_ctx* ctx);

/* Sets the potential V (sx*sy doubles, y-major) or the null potential when
 * V is NULL. Replaces Potential (potential.cpp:21-63) as seen by
 * ExpPotential and the Hamiltonian. Tables are rebuilt for the current time
 * step. */
int itp2d_set_potential(itp2d_ctx* ctx, const double* V);

/* Sets the imaginary time step eps and rebuilds every exponential table:
 * MultiProductSplit::set_time_step (multiproductsplit.cpp:43-47). */
int itp2d_set_time_step(itp2d_ctx* ctx, double eps);

/* Copies all states host -> device / device -> host
 * (k*sy*sx interleaved complex doubles, StateArray layout statearray.cpp:21-75). */
int itp2d_upload_states(itp2d_ctx* ctx, const double* states);
int itp2d_download_states(itp2d_ctx* ctx, double* states);

/* Device pointer to the state array (double2 or float2 per element,
 * depending on the precision), valid until the next orthonormalisation,
 * which swaps buffers. */
int itp2d_device_states(itp2d_ctx* ctx, void** dev_ptr);

/* Applies the multi-product split evolution operator to every state:
 * ITPSystem::propagate (itpsystem.cpp:243-256) with MultiProductSplit
 * (multiproductsplit.cpp:23-41), SecondOrderSplit (secondordersplit.cpp:21-49),
 * ExpKinetic (expkinetic.cpp:138-197), ExpPotential (exppotential.hpp:56-65). */
int itp2d_propagate(itp2d_ctx* ctx);

/* Canonical subspace orthonormalisation of the state set,
 * StateSet::orthonormalize (stateset.cpp:136-232): S = Psi^H Psi dx^2,
 * S = U diag(l) U^H with ascending l, psi'_n = sum_i U_{i,n} l_n^{-1/2} psi_i.
 * On ITP2D_E_NONPOSITIVE_EIGENVALUE / ITP2D_E_NONNORMAL_EIGENVALUE the
 * states are left unchanged and (*bad_index, *bad_value) name the first
 * offending eigenvalue in ascending order. algo: ITP2D_ORTHO_*. Either out
 * pointer may be NULL. */
int itp2d_orthonormalize(itp2d_ctx* ctx, int algo, int* bad_index, double* bad_value);

/* Per-state energy and deviation in storage order:
 * Operator::mean_and_standard_deviation (operators.cpp:40-50) for H = T + V
 * (itpsystem.cpp:116-119): E = Re<psi|H psi>, sigma = Re sqrt(<H^2> - <H>^2)
 * with <H^2> = <H psi|H psi>. sigma_residual = ||H psi - E psi|| (no
 * cancellation floor). Arrays hold num_states doubles; sigma_residual and
 * E_imag may be NULL. In the FP32 form every expectation value is divided by
 * <psi|psi> (Rayleigh quotients), so that the FP32 accuracy of the state norms
 * does not enter E at first order; the FP64 form follows the reference
 * (states taken as normalised). */
int itp2d_energies(itp2d_ctx* ctx, double* E, double* sigma, double* sigma_residual, double* E_imag);

/* states <- H states (Hamiltonian OperatorSum of itpsystem.cpp:116-119),
 * the operator application tested by test_hamiltonian.cpp:40-106. */
int itp2d_apply_hamiltonian(itp2d_ctx* ctx);

/* states <- Transformer::transform(states, kind), unnormalised
 * (transformer.hpp:132-158). kind: ITP2D_FFT ... ITP2D_IDCTY. */
int itp2d_transform(itp2d_ctx* ctx, int kind);

/* Switches the arithmetic of the sweeps and energies (ITP2D_FP64 or
 * ITP2D_FP32), converting the resident states on the device and rebuilding
 * the tables. The FP32 form switches to FP64 at its accuracy floor to refine
 * the eigenpairs; no reference counterpart (the reference is FP64 only). */
int itp2d_set_precision(itp2d_ctx* ctx, int precision);

/* Contraction engine of the orthonormalisation (overlap S = Psi^H Psi and
 * rotation Psi W) for FP32 states. ITP2D_CONTRACT_AUTO uses the tensor cores
 * (tcgen05, each FP32 value split into three BF16 parts, FP32 accumulation
 * over grid chunks of at most 2048 points, chunks summed in FP64) when the
 * grid has an even number of points, else the FP64 path.
 * ITP2D_CONTRACT_FP64 always uses FP64 arithmetic (DMMA). FP64 states always
 * use FP64 arithmetic. No reference counterpart (the reference is FP64 only;
 * stateset.cpp:146-154 and 214-228 compute these products with ZHERK/ZGEMM). */
/* Rayleigh-Ritz step on orthonormal states (no reference counterpart; the
 * reference's energies are per-state expectation values, itpsystem.cpp:483-494):
 * the projected Hamiltonian H_ij = <psi_i|H psi_j> dx^2 (Hamiltonian passes
 * of itp2d_energies, FP64 contraction), its eigendecomposition
 * H = U diag(theta) U^H by the Jacobi eigensolver, and psi'_n =
 * sum_i U_{i,n} psi_i. ritz_values (k doubles, ascending, may be NULL)
 * receives theta. The states must be orthonormal (after
 * itp2d_orthonormalize); the result is orthonormal to the rotation's
 * accuracy and its energies are the Ritz values. */
int itp2d_rayleigh_ritz(itp2d_ctx* ctx, double* ritz_values);

/* Column passes of periodic 256- and 512-point lines: tiles staged through
 * registers and shared memory (0) or moved by TMA with a three-slot ring (1).
 * The first itp2d_set_time_step of each precision times both on the spare
 * state buffer and keeps the faster; the choice is kept for the process per
 * device, precision and grid, so later contexts of the same size reuse it.
 * variant >= 0 forces one, -1 restores the tuned choice.
 * itp2d_column_variant returns the variant in use. */
int itp2d_set_column_variant(itp2d_ctx* ctx, int variant);
int itp2d_column_variant(itp2d_ctx* ctx);

/* Contraction engine: AUTO (FP64 states: DMMA; FP32 states: tensor cores on
 * operands split into BF16 planes once per contraction), FP64 (DMMA for
 * either precision), TC_STAGED (tensor cores, operands split inside each CTA;
 * the same results as AUTO, bit for bit). */
enum { ITP2D_CONTRACT_AUTO = 0, ITP2D_CONTRACT_FP64 = 1, ITP2D_CONTRACT_TC_STAGED = 2 };
int itp2d_set_contraction(itp2d_ctx* ctx, int engine);

/* Engine of the overlap S = Psi^H Psi dx^2 and the rotation psi' = psi W of
 * itp2d_orthonormalize on FP64 states: ITP2D_FP64_DMMA (the default: FP64
 * tensor-core products) or ITP2D_FP64_INT8 (the int8 tensor cores: both
 * operands split into eight int8 slices under per-row power-of-two scales,
 * the slice products summed exactly in 32-bit integers and combined in FP64;
 * the results agree with FP64 products to about 1e-15 of the largest output
 * of each row; k < 8300). INT8 takes about 48 bytes per state and grid point
 * of scratch at its first use; where that cannot be allocated the DMMA
 * contractions run. FP32 states, the Rayleigh-Ritz step and the batched and
 * device-loop forms are not affected. */
enum { ITP2D_FP64_DMMA = 0, ITP2D_FP64_INT8 = 1 };
int itp2d_set_fp64_engine(itp2d_ctx* ctx, int engine);
/* Overlaps and rotations of FP64 states run on the int8 tensor cores since
 * creation. */
long long itp2d_int8_contractions(itp2d_ctx* ctx);

/* FP32 states: orthonormalise canonically only on every canonical_every-th
 * call and by a second-order Lowdin step in between, W = D (I + E)^{-1/2} with
 * D = diag(S)^{-1/2} and D S D = I + E, the series cut after E^2 (one k x k
 * product instead of the k x k eigendecomposition). A step whose E is not
 * small (largest element 0.05, Frobenius norm 0.25) is canonical anyway. The
 * Lowdin step keeps the state order (no sort by overlap eigenvalue) and does
 * not check the overlap eigenvalues. 0 or 1: always canonical (the default).
 * FP64 states are always orthonormalised canonically. No reference
 * counterpart (stateset.cpp:136-232 is the canonical form). */
int itp2d_set_fp32_orthonormalization(itp2d_ctx* ctx, int canonical_every);
/* Moves the next canonical step of that schedule `calls` orthonormalisations
 * later (the schedule then continues every canonical_every-th call). Called
 * after itp2d_set_fp32_orthonormalization, which restarts the schedule. */
int itp2d_set_fp32_canonical_delay(itp2d_ctx* ctx, int calls);
/* The orthonormalisation between the canonical calls of
 * itp2d_set_fp32_orthonormalization: ITP2D_BETWEEN_LOWDIN (the default, taken
 * only while the overlap is close to the identity) or ITP2D_BETWEEN_CHOLESKY
 * (Gram-Schmidt order, ITP2D_ORTHO_CHOLESKY; taken whenever the overlap's
 * Cholesky factorisation succeeds, canonical otherwise). */
enum { ITP2D_BETWEEN_LOWDIN = 0, ITP2D_BETWEEN_CHOLESKY = 1 };
int itp2d_set_fp32_between(itp2d_ctx* ctx, int method);
/* FP32 states: the canonical orthonormalisation's eigensolve stops at a
 * largest rotation tangent of tau (default 1e-3; off-diagonal elements of
 * about tau^2 remain). A looser tau suits the first iterations of a solve,
 * whose basis the next step replaces. FP64 states are not affected. */
int itp2d_set_fp32_eig_tolerance(itp2d_ctx* ctx, double tau);
/* FP32 states: the canonical orthonormalisation's eigensolve runs at most
 * max_sweeps Jacobi sweeps (0, the default: until the tolerance above); a
 * capped solve is finished by a Cholesky factorisation S' = L L^H of the
 * overlap of the states rotated onto its approximate eigenvectors V, in
 * descending eigenvalue order (lowest energy first): W = V L^{-H}. The states
 * are then orthonormal whatever the remaining off-diagonal elements, and the
 * rotation is the canonical one up to them. A factorisation that fails
 * falls back to the full eigensolve. FP64 states are not affected. */
int itp2d_set_fp32_eig_sweeps(itp2d_ctx* ctx, int max_sweeps);
/* Canonical orthonormalisations of FP32 states finished by the Cholesky step
 * (itp2d_set_fp32_eig_sweeps) since creation. */
long long itp2d_fp32_capped_eigensolves(itp2d_ctx* ctx);
/* Rotations by an upper-triangular W (Cholesky steps, about half the
 * products of a dense rotation) since creation, per precision. */
int itp2d_triangular_rotations(itp2d_ctx* ctx, long long* fp64, long long* fp32);
/* Number of canonical, Lowdin and Cholesky orthonormalisations since
 * creation; any pointer may be NULL. */
int itp2d_orthonormalization_counts(itp2d_ctx* ctx, long long* canonical, long long* lowdin, long long* cholesky);

/* Overlap matrix of the resident states, S_ij = <psi_i|psi_j> dx^2
 * (row-major, num_states^2 interleaved complex doubles), computed by the
 * engine itp2d_orthonormalize would use; the states are not changed.
 * The product of stateset.cpp:146-154. */
int itp2d_overlap_matrix(itp2d_ctx* ctx, double* S);

/* Waits for the context's stream. */
int itp2d_synchronize(itp2d_ctx* ctx);

/* Number of kernel launches issued by this context since creation. */
long long itp2d_launch_count(itp2d_ctx* ctx);

/* Accumulated device milliseconds per phase, measured with CUDA events on
 * the context's stream: [0] propagate, [1] overlap, [2] eigensolve,
 * [3] rotation, [4] energies. Timing is enabled by itp2d_set_timing(ctx, 1)
 * and costs one event pair per phase. */
int itp2d_set_timing(itp2d_ctx* ctx, int enable);
int itp2d_phase_times(itp2d_ctx* ctx, double* ms5);

/* The same phase times split by the precision the phase ran in, with the
 * number of timed calls: ms10[p * 5 + phase] and calls10[p * 5 + phase] for
 * p = ITP2D_FP64 (0) or ITP2D_FP32 (1), phases in the order above. */
int itp2d_phase_stats(itp2d_ctx* ctx, double* ms10, long long* calls10);

/* Jacobi sweeps used by the last orthonormalisation, and by all of them
 * since the context was created. */
int itp2d_last_sweeps(itp2d_ctx* ctx);
long long itp2d_total_sweeps(itp2d_ctx* ctx);
/* Jacobi sweeps of the orthonormalisations run on states of one precision
 * (ITP2D_FP64 or ITP2D_FP32); -1 for another value. */
long long itp2d_precision_sweeps(itp2d_ctx* ctx, int precision);

/* Eigen-decomposition of an n x n complex Hermitian matrix on the device,
 * the drop-in for EigenSolver::solve (ZHEEV("V","U"), eigensolver.hpp:80-84).
 * A is column-major interleaved complex (A[j*n+i] = element (i, j)); only
 * the upper triangle i <= j is read. On return evals holds the eigenvalues in
 * ascending order and evecs[m*n+i] element i of eigenvector m (the layout of
 * EigenSolver::eigenvector, eigensolver.hpp:60). Eigenvector phases are
 * those of the Jacobi method, not LAPACK's. Allocates temporary device
 * memory; runs on the default stream. */
int itp2d_hermitian_eigensolve(int n, const double* A, double* evals, double* evecs);

/* Largest n accepted by itp2d_hermitian_eigensolve_noalloc. */
#define ITP2D_NOALLOC_MAX_N 128

/* The same eigen-decomposition as itp2d_hermitian_eigensolve (same
 * arguments, layouts and results), for callers that cannot allocate memory:
 * applications whose memory manager owns the whole device, or loops that
 * cannot afford the synchronisation of cudaMalloc/cudaFree. It allocates
 * nothing; its temporaries live in one fixed device array of this library
 * (about 1.6 MB, resident on every GPU that loads the library until exit).
 * n above ITP2D_NOALLOC_MAX_N returns ITP2D_E_INVALID. All calls share that
 * array, so calls that overlap on the GPU race: serialise them. Every call
 * looks up the array's address on the current device (a device reset leaves
 * no stale address); the first call on a device loads the library's device
 * code there, so make it before any stream capture begins. Runs on the default stream.
 * No counterpart in the reference. */
int itp2d_hermitian_eigensolve_noalloc(int n, const double* A, double* evals, double* evecs);

/* Adds Gaussian impurities to a potential on the device:
 * V[y][x] += sum_j A_j exp(-r_j^2 / (2 w_j^2)), with r_j the distance of the
 * cell-centred grid point (x_i = (2i + 1 - sx) dx / 2) from impurity j, in
 * list order at every point — GaussianImpurities::add_noise (noise.cpp:24-40)
 * for a whole impurity list. impurities holds n rows (x, y, A, w) and V holds
 * sx * sy doubles; both must be device (or managed) memory, otherwise
 * ITP2D_E_INVALID. Asynchronous on cuda_stream (NULL: the default stream). */
int itp2d_add_gaussian_impurities(int sx, int sy, double dx, int n, const double* impurities, double* V,
		void* cuda_stream);

/* Potential of a description in the reference's mini-language, evaluated on
 * the device at the cell-centred grid points into V (sx * sy doubles, device
 * or managed memory, y-major): the 14 types of the reference's potential
 * library with their names, parameter counts, defaults and checks
 * (parse_potential_description, potentialtypes.cpp:56-100, and the
 * constructors after it): zero, harmonic, elliptic, prettyhardsquare,
 * softpentagon, henonheiles/henon, gaussian/gaussianblob,
 * quartic/quarticoscillator, squareoscillator, power/poweroscillator,
 * ring/ringpotential, cosh/coshpotential, softstadium, powerstadium.
 * Formulas follow the reference's operation order without fused
 * multiply-adds. ITP2D_E_INVALID for an unknown type, a wrong parameter count
 * or a value the reference rejects. Asynchronous on cuda_stream. */
int itp2d_evaluate_potential(const char* description, int sx, int sy, double dx, double* V, void* cuda_stream);
/* The same into a host array V (sx * sy doubles), through temporary device
 * memory; synchronous. */
int itp2d_evaluate_potential_host(const char* description, int sx, int sy, double dx, double* V);
/* Validates a description like itp2d_evaluate_potential (no device call);
 * *is_null (may be NULL) is 1 for the zero potential. */
int itp2d_potential_check(const char* description, int* is_null);

/* Impurity shapes of noise.cpp:42-87 added to a potential on the device, for
 * n impurities in list order at every grid point (rows and V in device or
 * managed memory):
 *   ITP2D_IMPURITY_COULOMB:    rows (x, y); V += param1 * (r^2)^(-param0 / 2)
 *                              (CoulombImpurities: exponent, prefactor)
 *   ITP2D_IMPURITY_HEMISPHERE: rows (x, y); V += param0 sqrt(1 - d^2 / param1^2)
 *                              inside radius param1 (HemisphereImpurities)
 *   ITP2D_IMPURITY_DELTA:      rows (x, y, A); V += A at the nearest grid point
 *                              (DeltaImpurities, DataLayout::nearest_index)
 * Gaussian impurities: itp2d_add_gaussian_impurities. */
enum { ITP2D_IMPURITY_COULOMB = 1, ITP2D_IMPURITY_HEMISPHERE = 2, ITP2D_IMPURITY_DELTA = 3 };
int itp2d_add_impurities(int shape, int sx, int sy, double dx, int n, const double* rows, double param0,
		double param1, double* V, void* cuda_stream);

/* Measures the FP64 tensor-core (DMMA) throughput of the current device in
 * TFLOP/s with a register-only kernel: the roofline denominator of the FP64
 * contractions. Diagnostic; no reference counterpart. */
int itp2d_device_fp64_peak(double* tflops);
/* The same for FP32 FFMA throughput (CUDA cores): the roofline denominator of
 * the single-precision eigensolver. Diagnostic; no reference counterpart. */
int itp2d_device_fp32_peak(double* tflops);

/* ---- Batched form: one call over many contexts (independent state sets of
 * any grid size and state count; no reference counterpart, the reference
 * runs one state set per process) ----
 *
 * itp2d_batch_propagate: itp2d_propagate on every context (each on its own
 * stream, so the instances' passes overlap on the device).
 * itp2d_batch_orthonormalize: the canonical orthonormalisation of every
 * context (StateSet::orthonormalize, stateset.cpp:136-232): the overlaps on
 * the contexts' streams, then ALL k x k eigenproblems in one launch (one CTA
 * per instance, cyclic Jacobi; 2 <= k <= 4096), then the rotations. status[i]
 * (and bad_index[i], bad_value[i] when not NULL) report each instance like
 * itp2d_orthonormalize; an instance that fails keeps its states.
 * itp2d_batch_energies: itp2d_energies of every context into E[i], sigma[i]
 * (and sigma_residual[i] when that array and entry are not NULL).
 * Contexts must be distinct. */
int itp2d_batch_propagate(int n, itp2d_ctx* const* ctxs);
int itp2d_batch_orthonormalize(int n, itp2d_ctx* const* ctxs, int* status, int* bad_index, double* bad_value);
int itp2d_batch_energies(int n, itp2d_ctx* const* ctxs, double* const* E, double* const* sigma,
		double* const* sigma_residual);

/* ---- Device-resident driver loop (no reference counterpart) ----
 *
 * Runs ITP iterations of the context without returning to the host until the
 * time-step test of the driver holds: one CUDA graph launch whose conditional
 * WHILE node repeats propagate, canonical orthonormalisation (the batched
 * eigensolver's one-CTA Jacobi), energies, and a device kernel that sorts the
 * (E, sigma, n) tuples and applies the test at every sorted position against
 * the previous iteration (itpsystem.cpp:291-330 with the tests of
 * convergence.cpp:75-199): test 0 abschange(limit), 1 relchange(limit),
 * 2 absstdev(limit, diff_limit), 3 relstdev(limit, diff_limit). A passing
 * state's flag is kept by its storage index (flags: k ints, in and out); the
 * loop ends once the states at sorted positions first .. first + count - 1
 * are all flagged, on an orthonormalisation failure (*status; the failed
 * iteration's rotation has then been applied with the previous W), or after
 * max_iterations. prev_sorted_E / prev_sorted_sigma (may be NULL) are the
 * previous iteration's sorted values. On return: iterations taken, the last
 * sorted energies, deviations and storage indices, and the sorted values of
 * the iteration before it (k each; sorted_index and the prev outputs may be
 * NULL). The time step does not change inside the loop. */
int itp2d_run_device_loop(itp2d_ctx* ctx, int max_iterations, int test, double limit, double diff_limit, int first,
		int count, const double* prev_sorted_E, const double* prev_sorted_sigma, int* flags, int* iterations,
		int* status, double* sorted_E, double* sorted_sigma, int* sorted_index, double* prev_E_out,
		double* prev_sigma_out);

/* Diagnostic of the bounded device waits: one CTA of the tensor-core kernels'
 * set-up (tensor memory and mbarriers) waits on a barrier that nothing
 * completes. Returns ITP2D_E_TIMEOUT when the wait gives up after its limit
 * (about a second) and the kernel frees its tensor memory and returns, as the
 * overlap and rotation kernels do on a stalled pipeline; the context stays
 * usable. No reference counterpart. */
int itp2d_tc_wait_probe(void);

/* Short description of a status code. */
const char* itp2d_status_string(int status);

#ifdef __cplusplus
}
#endif

#endif /* ITP2D_GPU_H */
