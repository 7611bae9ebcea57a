/*
 * Oracle-only definitions for the Datafile interface declared by the itp2d
 * reference (datafile.hpp:38-120). Test infrastructure: the oracle runs every
 * ITPSystem with Parameters::Nothing (itpsystem.cpp:70,101-102), so no
 * datafile is ever opened; each entry point throws to make accidental use
 * loud. Replaces datafile.cpp, which needs the HDF5 C++ library.
 */
#include "datafile.hpp"

const H5::PredType H5::PredType::C_S1;
const H5::PredType H5::PredType::NATIVE_INT;
const H5::PredType H5::PredType::NATIVE_ULONG;
const H5::PredType H5::PredType::NATIVE_DOUBLE;

namespace {
void no_hdf5() { throw GeneralError("HDF5 output is not available in the itp2d oracle build"); }
}

Datafile::Datafile(std::string, DataLayout const& dl, bool) :
		datalayout(dl),
		double_type(H5::PredType::NATIVE_DOUBLE),
		int_type(H5::PredType::NATIVE_INT),
		state_type(NULL),
		potential_type(NULL) {
	no_hdf5();
}

Datafile::~Datafile() {}

void Datafile::write_state(size_t, size_t, State const&) { no_hdf5(); }
void Datafile::write_stateset(StateSet const&, int, std::list<size_t> const*) { no_hdf5(); }
void Datafile::write_time_step_history(size_t, double) { no_hdf5(); }
void Datafile::write_energy_history(std::vector<double>, size_t) { no_hdf5(); }
void Datafile::write_energy_history(std::vector<std::vector<double> >) { no_hdf5(); }
void Datafile::write_deviation_history(std::vector<double>, size_t) { no_hdf5(); }
void Datafile::write_deviation_history(std::vector<std::vector<double> >) { no_hdf5(); }
void Datafile::write_energies(std::vector<double>) { no_hdf5(); }
void Datafile::write_energy_standard_deviations(std::vector<double>) { no_hdf5(); }
void Datafile::write_potential(Potential const&) { no_hdf5(); }
void Datafile::write_noise_realization(Noise const&) { no_hdf5(); }
void Datafile::add_attribute(const char*, int) { no_hdf5(); }
void Datafile::add_attribute(const char*, unsigned long int) { no_hdf5(); }
void Datafile::add_attribute(const char*, double) { no_hdf5(); }
void Datafile::add_attribute(const char*, const char*) { no_hdf5(); }
void Datafile::add_attribute(const char*, std::string const&) { no_hdf5(); }
bool Datafile::is_open() const { return false; }
