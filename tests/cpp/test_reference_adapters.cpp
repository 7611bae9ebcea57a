/*
 * Drives the device library from the itp2d reference's own C++ API
 * (include/itp2d_reference.hpp) next to the reference's CPU classes, compiled
 * from the reference sources (oracle/Makefile target `adapters`). Each check
 * prints one line "ok <name> <figure>" or "FAIL <name> <figure>"; the exit
 * code is the number of failures.
 *
 *  1. DeviceTransformer vs Transformer::transform, all 18 kinds.
 *  2. DeviceMultiProductSplit vs MultiProductSplit, through the reference's
 *     EvolutionOperator interface (per state) and operate_all (whole set).
 *  3. DeviceEnergies vs OperatorSum H = T + V, mean_and_standard_deviation.
 *  4. DeviceOrthonormalizer vs StateSet::orthonormalize: same subspace.
 *  5. DeviceEigenSolver vs EigenSolver (ZHEEV): eigenvalues.
 *  6. The harmonic-oscillator case of test_itp.cpp:56-91 (40 x 40 grid, L = 12,
 *     harmonic(1), 14 states, 8 wanted): the reference ITPSystem::step loop
 *     (itpsystem.cpp:407-470) with its three seams swapped for the device
 *     classes, against the same loop on the reference's CPU classes from the
 *     same initial states (energies per iteration) and against the analytic
 *     spectrum n_x + n_y + 1 (1e-4, the reference test's tolerance).
 */
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "eigensolver.hpp"
#include "kinetic.hpp"
#include "multiproductsplit.hpp"
#include "noise.hpp"
#include "operatorsum.hpp"
#include "potential.hpp"
#include "potentialtypes.hpp"
#include "rng.hpp"
#include "stateset.hpp"
#include "transformer.hpp"

#include "itp2d_reference.hpp"

namespace {

int failures = 0;

void report(const char* name, double figure, bool ok) {
	std::printf("%s %s %.3e\n", ok ? "ok" : "FAIL", name, figure);
	if (!ok) failures++;
}

std::vector<comp> snapshot(StateSet const& s, size_t k, size_t G) {
	std::vector<comp> out(k * G);
	for (size_t n = 0; n < k; n++) std::copy(s[n].data_ptr(), s[n].data_ptr() + G, &out[n * G]);
	return out;
}

void restore(StateSet& s, std::vector<comp> const& in, size_t k, size_t G) {
	for (size_t n = 0; n < k; n++) std::copy(&in[n * G], &in[n * G] + G, const_cast<comp*>(s[n].data_ptr()));
}

// max over states of max|a - b| / max|b|
double per_state_rel(std::vector<comp> const& a, std::vector<comp> const& b, size_t k, size_t G) {
	double worst = 0;
	for (size_t n = 0; n < k; n++) {
		double d = 0, m = 0;
		for (size_t i = 0; i < G; i++) {
			d = std::max(d, std::abs(a[n * G + i] - b[n * G + i]));
			m = std::max(m, std::abs(b[n * G + i]));
		}
		worst = std::max(worst, d / m);
	}
	return worst;
}

// Smallest singular value of A^H B dx^2 (both orthonormal sets): 1 when they
// span the same subspace. Computed as the smallest eigenvalue of M^H M.
double subspace_cosine(std::vector<comp> const& a, std::vector<comp> const& b, size_t k, size_t G, double dx) {
	std::vector<comp> M(k * k);
	for (size_t i = 0; i < k; i++)
		for (size_t j = 0; j < k; j++) {
			comp s = 0;
			for (size_t t = 0; t < G; t++) s += std::conj(a[i * G + t]) * b[j * G + t];
			M[i * k + j] = s * dx * dx;
		}
	std::vector<comp> MM(k * k);  // column-major M^H M
	for (size_t i = 0; i < k; i++)
		for (size_t j = 0; j < k; j++) {
			comp s = 0;
			for (size_t t = 0; t < k; t++) s += std::conj(M[t * k + i]) * M[t * k + j];
			MM[j * k + i] = s;
		}
	EigenSolver es(k);
	es.solve(&MM[0]);
	return std::sqrt(std::max(0.0, es.eigenvalue(0)));
}

struct Problem {
	DataLayout dl;
	Transformer tr;
	BoundaryType bt;
	double B;
	PotentialType const* ptype;
	NoNoise noise;
	Potential pot;
	Kinetic kin;
	OperatorSum H;
	Problem(size_t s, double L, BoundaryType bt_, double B_, std::string const& potential)
		: dl(s, s, L / static_cast<double>(s)), tr(dl, FFTW_ESTIMATE), bt(bt_), B(B_),
		  ptype(parse_potential_description(potential)), pot(dl, *ptype, noise), kin(B_, tr, bt_) {
		H += kin;
		H += pot;
	}
	~Problem() { delete ptype; }
};

void check_operators() {
	const size_t s = 48, k = 6, G = s * s;
	Problem P(s, 14.0, Periodic, 0.5, "harmonic(1)");
	RNG rng(7);
	StateSet set(k, P.dl);
	set.init_to_gaussian_noise(rng);
	const std::vector<comp> psi = snapshot(set, k, G);

	// 1. transforms
	{
		itp2d_b200::DeviceTransformer dt(P.dl);
		double worst = 0;
		for (int kind = 0; kind <= 17; kind++) {
			std::vector<comp> a(psi.begin(), psi.begin() + G), b(a);
			P.tr.transform(&a[0], static_cast<Transform>(kind));
			dt.transform(&b[0], static_cast<Transform>(kind));
			worst = std::max(worst, per_state_rel(b, a, 1, G));
		}
		report("transformer_18_kinds", worst, worst < 1e-14);
	}
	// 2. propagation through the EvolutionOperator interface
	{
		MultiProductSplit T(2, P.pot, 0.05, P.tr, P.bt, P.B);
		itp2d_b200::DeviceMultiProductSplit D(2, P.pot, 0.05, P.tr, P.bt, P.B);
		StateArray ws(T.required_workspace(), P.dl);
		EvolutionOperator& cpu = T;
		EvolutionOperator& dev = D;
		restore(set, psi, k, G);
		for (size_t n = 0; n < k; n++) cpu(set[n], ws);
		const std::vector<comp> ref = snapshot(set, k, G);
		restore(set, psi, k, G);
		for (size_t n = 0; n < k; n++) dev(set[n], ws);
		const double e1 = per_state_rel(snapshot(set, k, G), ref, k, G);
		report("evolution_operator_per_state", e1, e1 < 1e-12);
		restore(set, psi, k, G);
		D.operate_all(set, k);
		const double e2 = per_state_rel(snapshot(set, k, G), ref, k, G);
		report("evolution_operator_batched", e2, e2 < 1e-12);
		// a time-step change rebuilds the device tables like set_time_step
		T.set_time_step(0.02);
		D.set_time_step(0.02);
		restore(set, psi, k, G);
		for (size_t n = 0; n < k; n++) cpu(set[n], ws);
		const std::vector<comp> ref2 = snapshot(set, k, G);
		restore(set, psi, k, G);
		D.operate_all(set, k);
		const double e3 = per_state_rel(snapshot(set, k, G), ref2, k, G);
		report("evolution_operator_new_time_step", e3, e3 < 1e-12);
	}
	// 3. energies
	{
		restore(set, psi, k, G);
		StateArray ws(P.H.required_workspace() + 1, P.dl);
		itp2d_b200::DeviceEnergies de(P.pot, P.dl, k, P.bt, P.B);
		std::vector<double> E, sd;
		de.mean_and_standard_deviation(set, E, sd);
		double worst = 0, worst_sd = 0, Emax = 0;
		for (size_t n = 0; n < k; n++) {
			const std::pair<comp, comp> r = P.H.mean_and_standard_deviation(set[n], ws);
			worst = std::max(worst, std::abs(E[n] - r.first.real()) / std::abs(r.first.real()));
			worst_sd = std::max(worst_sd, std::abs(sd[n] - r.second.real()));
			Emax = std::max(Emax, std::abs(r.first.real()));
		}
		report("hamiltonian_energies", worst, worst < 1e-12);
		report("hamiltonian_deviations", worst_sd / Emax, worst_sd < 1e-10 * Emax);
	}
	// 4. orthonormalisation
	{
		StateSet cpu(k, P.dl), dev(k, P.dl);
		restore(cpu, psi, k, G);
		restore(dev, psi, k, G);
		cpu.orthonormalize();
		itp2d_b200::DeviceOrthonormalizer o(P.dl, k);
		o.orthonormalize(dev);
		const double c = subspace_cosine(snapshot(dev, k, G), snapshot(cpu, k, G), k, G, P.dl.dx);
		report("orthonormalize_subspace", 1 - c, 1 - c < 1e-10);
		report("orthonormalize_orthonormal", dev.how_orthonormal(), dev.how_orthonormal() < 64 * 2.2e-16);
		// a rank-deficient set raises the reference's exception
		StateSet bad(k, P.dl);
		restore(bad, psi, k, G);
		std::fill(const_cast<comp*>(bad[2].data_ptr()), const_cast<comp*>(bad[2].data_ptr()) + G, comp(0));
		bool thrown = false;
		try {
			o.orthonormalize(bad);
		} catch (NonPositiveEigenvalue&) {
			thrown = true;
		}
		report("orthonormalize_nonpositive_throws", thrown ? 0.0 : 1.0, thrown);
	}
	// 5. eigensolver
	{
		const int n = 40;
		std::vector<comp> A(n * n);
		for (int i = 0; i < n; i++)
			for (int j = i; j < n; j++) {
				const comp v = i == j ? comp(2.0 + i, 0) : comp(std::sin(i + 2.0 * j), std::cos(3.0 * i - j)) / 10.0;
				A[j * n + i] = v;
				A[i * n + j] = std::conj(v);
			}
		std::vector<comp> B(A);
		EigenSolver cpu(n);
		itp2d_b200::DeviceEigenSolver dev(n);
		cpu.solve(&A[0]);
		dev.solve(&B[0]);
		double worst = 0;
		for (int i = 0; i < n; i++) worst = std::max(worst, std::abs(cpu.eigenvalue(i) - dev.eigenvalue(i)));
		report("eigensolver_values", worst, worst < 1e-12 * (n + 2));
		// eigenvectors agree up to phase
		double wv = 0;
		for (int m = 0; m < n; m++) {
			comp d = 0;
			for (int i = 0; i < n; i++) d += std::conj(cpu.eigenvector(&A[0], m, i)) * dev.eigenvector(&B[0], m, i);
			wv = std::max(wv, std::abs(1.0 - std::abs(d)));
		}
		report("eigensolver_vectors", wv, wv < 1e-10);
	}
}

// 6. The reference step loop with its three seams on the device.
void check_harmonic_oscillator() {
	const size_t s = 40, k = 14, wanted = 8, G = s * s;
	Problem P(s, 12.0, Periodic, 0.0, "harmonic(1)");
	RNG rng(20120131UL);
	StateSet cpu(k, P.dl), dev(k, P.dl);
	cpu.init_to_gaussian_noise(rng);
	restore(dev, snapshot(cpu, k, G), k, G);
	const int halforder = 5;  // the reference default (parameters.cpp:48)
	MultiProductSplit T(halforder, P.pot, 0.25, P.tr, P.bt, P.B);
	StateArray ws(std::max(T.required_workspace(), P.H.required_workspace() + 1), P.dl);
	itp2d_b200::DeviceMultiProductSplit DT(halforder, P.pot, 0.25, P.tr, P.bt, P.B);
	itp2d_b200::DeviceOrthonormalizer DO(P.dl, k);
	itp2d_b200::DeviceEnergies DE(P.pot, P.dl, k, P.bt, P.B);
	std::vector<double> Ec(k), Ed, sd;
	double worst_step = 0;
	for (int it = 0; it < 120; it++) {
		// ITPSystem::propagate (itpsystem.cpp:243-256)
		for (size_t n = 0; n < k; n++) T(cpu[n], ws);
		DT.operate_all(dev, k);
		// ITPSystem::orthonormalize -> StateSet::orthonormalize
		cpu.orthonormalize();
		DO.orthonormalize(dev);
		// ITPSystem::calculate_energies: per-state mean, then sorted
		for (size_t n = 0; n < k; n++) Ec[n] = P.H.mean_and_standard_deviation(cpu[n], ws).first.real();
		DE.mean_and_standard_deviation(dev, Ed, sd);
		std::vector<double> a(Ec), b(Ed);
		std::sort(a.begin(), a.end());
		std::sort(b.begin(), b.end());
		for (size_t n = 0; n < k; n++) worst_step = std::max(worst_step, std::abs(a[n] - b[n]) / std::abs(a[n]));
		if (it == 60) {
			// the reference's time-step change (itpsystem.cpp:202-233)
			T.set_time_step(0.05);
			DT.set_time_step(0.05);
		}
	}
	report("ho_loop_energies_vs_cpu_loop", worst_step, worst_step < 1e-10);
	std::sort(Ed.begin(), Ed.end());
	double worst = 0;
	int E = 1, deg = 1;
	for (size_t n = 0; n < wanted; n++) {
		worst = std::max(worst, std::abs(Ed[n] - E));
		if (deg++ >= E) {
			E++;
			deg = 1;
		}
	}
	report("ho_loop_analytic_spectrum", worst, worst < 1e-4);
}

}  // namespace

int main() {
	try {
		check_operators();
		check_harmonic_oscillator();
	} catch (std::exception& e) {
		std::printf("FAIL exception %s\n", e.what());
		failures++;
	}
	std::printf("%d failures\n", failures);
	return failures;
}
