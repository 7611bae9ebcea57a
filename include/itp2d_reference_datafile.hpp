/*
 * itp2d_reference_datafile.hpp -- the reference's Datafile class
 * (datafile.hpp:39-75) over include/itp2d_datafile.h, for code compiled
 * inside the reference (C++98, the reference's headers on the include path)
 * on a machine without the HDF5 library. A maintainer replaces
 * `#include "datafile.hpp"` by this header and `Datafile` by
 * `itp2d_b200::Datafile`; the body of StateSet::init_from_datafile
 * (stateset.cpp:86-109) becomes itp2d_b200::init_from_datafile(*this, name).
 * Same constructor, methods, arguments and storage (one element per chunk,
 * deflate 9); a failure throws the reference's
 * GeneralError with the library's message (the reference rethrows HDF5's
 * exceptions). Link with -litp2d_b200.
 */
#ifndef ITP2D_REFERENCE_DATAFILE_HPP
#define ITP2D_REFERENCE_DATAFILE_HPP

#include <list>
#include <string>
#include <vector>

#include "datalayout.hpp"
#include "exceptions.hpp"
#include "noise.hpp"
#include "potential.hpp"
#include "state.hpp"
#include "stateset.hpp"

#include "itp2d_datafile.h"

namespace itp2d_b200 {

inline void check_datafile(int status, const char* what) {
	if (status != 0) throw GeneralError(std::string(what) + ": " + itp2d_datafile_last_error());
}

class Datafile {
  public:
	struct state_history_pair { int step; int index; };
	struct time_step_history_pair { int step; double time_step; };
	Datafile(std::string filename, DataLayout const& dl, bool clobber = false) : f(NULL), sx(dl.sizex), sy(dl.sizey) {
		check_datafile(itp2d_datafile_create(filename.c_str(), static_cast<int>(dl.sizex), static_cast<int>(dl.sizey),
				dl.dx, clobber ? 1 : 0, &f), "Datafile");
		// the reference's storage: one element per chunk, deflate 9 (datafile.cpp:76-88)
		check_datafile(itp2d_datafile_set_chunking(f, 9), "Datafile");
	}
	~Datafile() { itp2d_datafile_close(f); }

	void write_state(size_t n, size_t m, State const& state) {
		check_datafile(itp2d_datafile_write_state(f, static_cast<long long>(n), static_cast<long long>(m),
				reinterpret_cast<const double*>(state.data_ptr())), "write_state");
	}
	void write_stateset(StateSet const& stateset, int step, std::list<size_t> const* sort_order = NULL) {
		const size_t N = stateset.get_num_states();
		const size_t G = sx * sy;
		// one contiguous block (stateset.cpp:23-44), else a gathered copy
		const comp* first = stateset[0].data_ptr();
		bool contiguous = true;
		for (size_t m = 0; m < N; m++) contiguous = contiguous && stateset[m].data_ptr() == first + m * G;
		std::vector<comp> copy;
		if (!contiguous) {
			copy.resize(N * G);
			for (size_t m = 0; m < N; m++)
				for (size_t i = 0; i < G; i++) copy[m * G + i] = stateset[m].data_ptr()[i];
			first = &copy[0];
		}
		std::vector<int> order;
		if (sort_order != NULL)
			for (std::list<size_t>::const_iterator it = sort_order->begin(); it != sort_order->end(); ++it)
				order.push_back(static_cast<int>(*it));
		if (sort_order != NULL && order.size() != N) throw GeneralError("write_stateset: sort order of another length");
		check_datafile(itp2d_datafile_write_stateset(f, reinterpret_cast<const double*>(first), static_cast<int>(N),
				step, sort_order != NULL ? &order[0] : NULL), "write_stateset");
	}
	void write_time_step_history(size_t index, double eps) {
		check_datafile(itp2d_datafile_write_time_step_history(f, static_cast<int>(index), eps),
				"write_time_step_history");
	}
	void write_energy_history(std::vector<double> energy_history, size_t index) {
		check_datafile(itp2d_datafile_write_energy_history(f, data(energy_history),
				static_cast<int>(energy_history.size()), static_cast<int>(index)), "write_energy_history");
	}
	void write_energy_history(std::vector<std::vector<double> > energy_history) {
		for (size_t n = 0; n < energy_history.size(); n++) write_energy_history(energy_history[n], n);
	}
	void write_deviation_history(std::vector<double> deviation_history, size_t index) {
		check_datafile(itp2d_datafile_write_deviation_history(f, data(deviation_history),
				static_cast<int>(deviation_history.size()), static_cast<int>(index)), "write_deviation_history");
	}
	void write_deviation_history(std::vector<std::vector<double> > deviation_history) {
		for (size_t n = 0; n < deviation_history.size(); n++) write_deviation_history(deviation_history[n], n);
	}
	void write_energies(std::vector<double> energies) {
		check_datafile(itp2d_datafile_write_energies(f, data(energies), static_cast<int>(energies.size())),
				"write_energies");
	}
	void write_energy_standard_deviations(std::vector<double> standard_deviations) {
		check_datafile(itp2d_datafile_write_energy_standard_deviations(f, data(standard_deviations),
				static_cast<int>(standard_deviations.size())), "write_energy_standard_deviations");
	}
	void write_potential(Potential const& pot) {
		if (pot.is_null()) return;  // nothing to write, as datafile.cpp:382-383
		check_datafile(itp2d_datafile_write_potential(f, pot.get_valueptr()), "write_potential");
	}
	void write_noise_realization(Noise const& noise) {
		std::vector<double> vec;
		noise.write_realization_data(vec);
		check_datafile(itp2d_datafile_write_noise_realization(f, data(vec), static_cast<int>(vec.size())),
				"write_noise_realization");
	}
	void add_attribute(const char* name, int value) {
		check_datafile(itp2d_datafile_add_attribute_int(f, name, value), "add_attribute");
	}
	void add_attribute(const char* name, unsigned long int value) {
		check_datafile(itp2d_datafile_add_attribute_ulong(f, name, value), "add_attribute");
	}
	void add_attribute(const char* name, double value) {
		check_datafile(itp2d_datafile_add_attribute_double(f, name, value), "add_attribute");
	}
	void add_attribute(const char* name, const char* value) {
		check_datafile(itp2d_datafile_add_attribute_string(f, name, value), "add_attribute");
	}
	void add_attribute(const char* name, std::string const& value) { add_attribute(name, value.c_str()); }
	void flush() { check_datafile(itp2d_datafile_flush(f), "flush"); }
	bool is_open() const { return f != NULL; }

  private:
	Datafile(Datafile const&);
	Datafile& operator=(Datafile const&);
	static const double* data(std::vector<double> const& v) { return v.empty() ? NULL : &v[0]; }
	itp2d_datafile* f;
	size_t sx, sy;
};

// StateSet::init_from_datafile (stateset.cpp:86-109): the last state set saved
// in the file, after the file's num_states, grid_sizex, grid_sizey and
// grid_delta are checked against the StateSet.
inline void init_from_datafile(StateSet& stateset, std::string filename) {
	const size_t N = stateset.get_num_states();
	DataLayout const& dl = stateset[0].datalayout;
	std::vector<comp> buf(N * dl.sizex * dl.sizey);
	const int st = itp2d_datafile_init_states(filename.c_str(), static_cast<int>(N), static_cast<int>(dl.sizex),
			static_cast<int>(dl.sizey), dl.dx, reinterpret_cast<double*>(&buf[0]));
	if (st != 0) throw GeneralError(itp2d_datafile_last_error());
	for (size_t m = 0; m < N; m++)
		for (size_t y = 0; y < dl.sizey; y++)
			for (size_t x = 0; x < dl.sizex; x++) stateset[m](x, y) = buf[(m * dl.sizey + y) * dl.sizex + x];
}

}  // namespace itp2d_b200

#endif
