/*
 * itp2d_reference.hpp -- the device library behind the itp2d reference's own
 * C++ operator API, for code compiled inside the reference (C++98, the
 * reference's headers on the include path: operators.hpp, potential.hpp,
 * transformer.hpp, statearray.hpp, exceptions.hpp).
 *
 * Each class keeps the interface of the reference class it replaces, so a
 * maintainer swaps a type, not the code around it:
 *
 *   DeviceMultiProductSplit  -- MultiProductSplit (multiproductsplit.hpp:31-44):
 *                               an EvolutionOperator (operators.hpp:33-69) with
 *                               the same constructor; operate() is the
 *                               batch-of-1 compatibility path, operate_all()
 *                               propagates a whole StateSet or StateArray in
 *                               one call.
 *   DeviceOrthonormalizer    -- StateSet::orthonormalize (stateset.cpp:136-232)
 *                               for a StateSet or StateArray, with the
 *                               reference's exceptions on failure.
 *   DeviceEnergies           -- Operator::mean_and_standard_deviation of the
 *                               Hamiltonian (operators.cpp:40-50) for every
 *                               state of a StateSet or StateArray.
 *   DeviceEigenSolver        -- EigenSolver (eigensolver.hpp:57-84): solve(),
 *                               eigenvalue(), eigenvector(), scale_eigenvector().
 *   DeviceTransformer        -- Transformer::transform (transformer.hpp:132-158)
 *                               on one state's data.
 *
 * Status codes of itp2d_gpu.h become the reference's exceptions
 * (exceptions.hpp): NonPositiveEigenvalue, NonNormalEigenvalue,
 * EigensolverError, GeneralError. Link with -litp2d_b200.
 */
#ifndef ITP2D_REFERENCE_HPP
#define ITP2D_REFERENCE_HPP

#include <cstring>
#include <ostream>
#include <sstream>
#include <string>
#include <vector>

#include "exceptions.hpp"
#include "itp2d_common.hpp"
#include "operators.hpp"
#include "potential.hpp"
#include "statearray.hpp"
#include "transformer.hpp"

#include "itp2d_gpu.h"

namespace itp2d_b200 {

// Throws the reference exception that matches a status code.
inline void check_status(int status, const char* what, int bad_index = -1, double bad_value = 0.0) {
	switch (status) {
		case ITP2D_OK:
			return;
		case ITP2D_E_NONPOSITIVE_EIGENVALUE:
			throw NonPositiveEigenvalue(static_cast<size_t>(bad_index < 0 ? 0 : bad_index), bad_value, NULL, 0);
		case ITP2D_E_NONNORMAL_EIGENVALUE:
			throw NonNormalEigenvalue(static_cast<size_t>(bad_index < 0 ? 0 : bad_index), bad_value, NULL, 0);
		case ITP2D_E_EIGENSOLVER:
			throw EigensolverError(-1);
		default: {
			std::stringstream ss;
			ss << what << ": " << itp2d_status_string(status);
			throw GeneralError(ss.str());
		}
	}
}

inline int boundary_code(BoundaryType bt) { return bt == Dirichlet ? ITP2D_DIRICHLET : ITP2D_PERIODIC; }

inline comp const* first(State const& s) { return s.data_ptr(); }
template <class States> inline comp const* first(States const& states) { return states[0].data_ptr(); }

// One device context for k states of a DataLayout (owned, not copyable).
class DeviceContext {
	public:
		DeviceContext(DataLayout const& dl, size_t k, BoundaryType bt = Periodic, double B = 0, int halforder = 1)
				: ctx(NULL), num_states(k) {
			check_status(itp2d_ctx_create(static_cast<int>(dl.sizex), static_cast<int>(dl.sizey), dl.dx,
					static_cast<int>(k), boundary_code(bt), B, halforder, ITP2D_FP64, NULL, &ctx),
					"itp2d_ctx_create");
		}
		~DeviceContext() { itp2d_ctx_destroy(ctx); }
		itp2d_ctx* get() const { return ctx; }
		size_t size() const { return num_states; }
		// k states stored contiguously from the first one: a State (k = 1), a
		// StateArray (statearray.cpp:21-75) or a StateSet's current array
		// (stateset.cpp:23-44). State exposes its storage read-only; the
		// values written back are its own.
		template <class States> void upload(States const& states) const {
			check_status(itp2d_upload_states(ctx, reinterpret_cast<const double*>(first(states))),
					"itp2d_upload_states");
		}
		template <class States> void download(States& states) const {
			check_status(itp2d_download_states(ctx, reinterpret_cast<double*>(const_cast<comp*>(first(states)))),
					"itp2d_download_states");
		}
	private:
		DeviceContext(DeviceContext const&);
		DeviceContext& operator=(DeviceContext const&);
		itp2d_ctx* ctx;
		const size_t num_states;
};

// MultiProductSplit (multiproductsplit.cpp:23-59) on the device. The
// constructor takes the reference's arguments; the potential table is read
// through Potential::get_valueptr (NULL for the null potential).
class DeviceMultiProductSplit : public EvolutionOperator {
	public:
		DeviceMultiProductSplit(int halforder, Potential const& pot, double time_step, Transformer const& tr,
				BoundaryType bt, double B = 0)
				: halforder(halforder), dl(tr.datalayout), bt(bt), B(B), eps(time_step), potential(NULL),
				  single(tr.datalayout, 1, bt, B, halforder), batch(NULL) {
			if (pot.get_valueptr() != NULL) {
				potential = new std::vector<double>(pot.get_valueptr(), pot.get_valueptr() + dl.N);
			}
			setup(single.get());
		}
		~DeviceMultiProductSplit() {
			delete batch;
			delete potential;
		}
		void set_time_step(double time_step) {
			eps = time_step;
			check_status(itp2d_set_time_step(single.get(), eps), "itp2d_set_time_step");
			if (batch) check_status(itp2d_set_time_step(batch->get(), eps), "itp2d_set_time_step");
		}
		// Operator interface: one state per call (the reference's per-state
		// OpenMP loop, itpsystem.cpp:243-256, calls this from several threads;
		// the context serialises them).
		void operate(State& state, __attribute__((unused)) StateArray& workspace) const {
			single.upload(state);
			check_status(itp2d_propagate(single.get()), "itp2d_propagate");
			single.download(state);
		}
		size_t required_workspace() const { return 0; }
		std::ostream& print(std::ostream& out) const {
			return out << "DeviceMultiProductSplit(order " << 2 * halforder << ")";
		}
		// The first `count` states of a StateArray or StateSet in one device
		// call: the batched seam that replaces ITPSystem::propagate's loop.
		template <class States> void operate_all(States& states, size_t count) const {
			if (batch == NULL || batch->size() != count) {
				delete batch;
				batch = NULL;
				batch = new DeviceContext(dl, count, bt, B, halforder);
				setup(batch->get());
			}
			batch->upload(states);
			check_status(itp2d_propagate(batch->get()), "itp2d_propagate");
			batch->download(states);
		}
		const int halforder;
	private:
		void setup(itp2d_ctx* c) const {
			check_status(itp2d_set_potential(c, potential ? &(*potential)[0] : NULL), "itp2d_set_potential");
			check_status(itp2d_set_time_step(c, eps), "itp2d_set_time_step");
		}
		DataLayout const& dl;
		const BoundaryType bt;
		const double B;
		double eps;
		std::vector<double>* potential;
		DeviceContext single;
		mutable DeviceContext* batch;
};

// StateSet::orthonormalize (stateset.cpp:136-232) for a StateSet or StateArray
// of N states, in place:
// canonical orthonormalisation, output state n belonging to the n-th smallest
// overlap eigenvalue. Throws NonPositiveEigenvalue / NonNormalEigenvalue like
// the reference (states unchanged then).
class DeviceOrthonormalizer {
	public:
		DeviceOrthonormalizer(DataLayout const& dl, size_t N) : dev(dl, N) {}
		template <class States> void orthonormalize(States& states, int algo = ITP2D_ORTHO_DEFAULT) {
			dev.upload(states);
			int bad = -1;
			double val = 0.0;
			check_status(itp2d_orthonormalize(dev.get(), algo, &bad, &val), "itp2d_orthonormalize", bad, val);
			dev.download(states);
		}
	private:
		DeviceContext dev;
};

// Energies and deviations of the N states of a StateSet or StateArray for H = T + V
// (itpsystem.cpp:116-119, operators.cpp:40-50), in storage order: the
// batched seam of ITPSystem::calculate_energies (itpsystem.cpp:473-511).
class DeviceEnergies {
	public:
		DeviceEnergies(Potential const& pot, DataLayout const& dl, size_t N, BoundaryType bt, double B)
				: dev(dl, N, bt, B) {
			std::vector<double> v;
			if (pot.get_valueptr() != NULL) v.assign(pot.get_valueptr(), pot.get_valueptr() + dl.N);
			check_status(itp2d_set_potential(dev.get(), v.empty() ? NULL : &v[0]), "itp2d_set_potential");
		}
		template <class States> void mean_and_standard_deviation(States const& states, std::vector<double>& E,
				std::vector<double>& sigma) {
			E.resize(dev.size());
			sigma.resize(dev.size());
			dev.upload(states);
			check_status(itp2d_energies(dev.get(), &E[0], &sigma[0], NULL, NULL), "itp2d_energies");
		}
	private:
		DeviceContext dev;
};

// EigenSolver (eigensolver.hpp:57-84): the same calls, ZHEEV("V","U")
// semantics, on the device. solve() overwrites the column-major input with
// the eigenvectors (eigenvector n in column n) like ZHEEV.
class DeviceEigenSolver {
	public:
		explicit DeviceEigenSolver(size_t N) : size(static_cast<int>(N)), evals(N) {}
		inline comp const& eigenvector(comp const* input_matrix, size_t n, size_t i) const {
			return input_matrix[n * size + i];
		}
		inline void scale_eigenvector(comp* input_matrix, size_t n, double value) const {
			for (int i = 0; i < size; i++) input_matrix[n * size + i] *= value;
		}
		inline double const& eigenvalue(size_t n) const { return evals[n]; }
		void solve(comp* input_matrix) {
			std::vector<comp> vecs(static_cast<size_t>(size) * size);
			const int st = itp2d_hermitian_eigensolve(size, reinterpret_cast<const double*>(input_matrix), &evals[0],
					reinterpret_cast<double*>(&vecs[0]));
			if (st == ITP2D_E_EIGENSOLVER) throw EigensolverError(-1);
			check_status(st, "itp2d_hermitian_eigensolve");
			std::memcpy(input_matrix, &vecs[0], vecs.size() * sizeof(comp));
		}
	private:
		const int size;
		std::vector<double> evals;
};

// Transformer::transform (transformer.hpp:132-158) on one state's data:
// unnormalised, the 18 kinds of enum Transform (transformer.hpp:32-34).
class DeviceTransformer {
	public:
		explicit DeviceTransformer(DataLayout const& dl) : dl(dl), dev(dl, 1) {}
		void transform(comp* data, Transform trans) const {
			check_status(itp2d_upload_states(dev.get(), reinterpret_cast<const double*>(data)), "itp2d_upload_states");
			check_status(itp2d_transform(dev.get(), static_cast<int>(trans)), "itp2d_transform");
			check_status(itp2d_download_states(dev.get(), reinterpret_cast<double*>(data)), "itp2d_download_states");
		}
		DataLayout const& dl;
	private:
		DeviceContext dev;
};

}  // namespace itp2d_b200

#endif  // ITP2D_REFERENCE_HPP
