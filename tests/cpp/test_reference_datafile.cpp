// The reference-API Datafile (include/itp2d_reference_datafile.hpp) driven
// with the reference's own StateSet, Potential and Noise objects, compiled
// against the reference sources (make -C oracle datafile-adapter): the writes
// that ITPSystem makes (itpsystem.cpp:69-116, 220-226, 374-402, 513-531), the
// file read back through the library's reader and compared bit for bit, then
// itp2d_b200::init_from_datafile (StateSet::init_from_datafile,
// stateset.cpp:86-109) into a second StateSet. Host only: no GPU is touched.
#include <cstdio>
#include <cstring>
#include <list>
#include <string>
#include <vector>

#include "datalayout.hpp"
#include "noise.hpp"
#include "potential.hpp"
#include "potentialtypes.hpp"
#include "rng.hpp"
#include "stateset.hpp"

#include "itp2d_reference_datafile.hpp"

static int failures = 0;

static void expect(bool ok, const char* what) {
	if (!ok) {
		std::printf("FAIL: %s\n", what);
		failures++;
	}
}

static std::vector<double> read_all(const char* path, const char* name) {
	long long n = 0;
	itp2d_datafile_read_values(path, name, NULL, 0, &n);
	std::vector<double> v(n > 0 ? n : 1);
	if (itp2d_datafile_read_values(path, name, &v[0], n, &n) != 0) {
		std::printf("FAIL: reading %s: %s\n", name, itp2d_datafile_last_error());
		failures++;
	}
	v.resize(n);
	return v;
}

static bool same_state(const double* file, State const& s, size_t G) {
	return std::memcmp(file, s.data_ptr(), G * 2 * sizeof(double)) == 0;
}

int main(int argc, char** argv) {
	const char* path = argc > 1 ? argv[1] : "reference_datafile.h5";
	const size_t sx = 24, sy = 16, N = 5, G = sx * sy;
	DataLayout dl(sx, sy, 0.5);
	StateSet states(N, dl);
	RNG rng(12345);
	states.init_to_gaussian_noise(rng);
	HarmonicOscillator ho(1.0);
	NoNoise noise;
	Potential pot(dl, ho, noise);
	size_t order_arr[N] = {4, 2, 0, 1, 3};
	std::list<size_t> order(order_arr, order_arr + N);
	std::vector<std::vector<double> > E(3, std::vector<double>(N)), D(3, std::vector<double>(N));
	for (size_t i = 0; i < 3; i++)
		for (size_t n = 0; n < N; n++) {
			E[i][n] = 1.0 + n + 0.5 / (i + 1);
			D[i][n] = 1e-3 / (i + 1) / (n + 1);
		}
	{
		// ITPSystem's sequence: run attributes, potential, noise, time steps,
		// per-step histories, saved states, final energies
		itp2d_b200::Datafile df(path, dl, true);
		df.add_attribute("program_version", "test");
		df.add_attribute("random_seed", 12345UL);
		df.add_attribute("num_states", static_cast<int>(N));
		df.add_attribute("grid_length", 12.0);
		df.add_attribute("grid_boundary_type", std::string("periodic"));
		df.write_potential(pot);
		df.write_noise_realization(noise);
		df.add_attribute("initial_time_step", 0.5);
		df.write_time_step_history(1, 0.5);
		df.write_energy_history(E);
		df.write_deviation_history(D);
		df.write_stateset(states, 3, NULL);
		df.write_time_step_history(4, 0.1);
		df.write_stateset(states, 7, &order);
		df.write_energies(E.back());
		df.write_energy_standard_deviations(D.back());
		df.add_attribute("total_steps_done", 7);
		df.flush();
		expect(df.is_open(), "is_open");
		bool threw = false;
		try {
			df.add_attribute("num_states", 1);  // createAttribute on an existing name
		} catch (GeneralError&) {
			threw = true;
		}
		expect(threw, "a second attribute of the same name throws GeneralError");
	}
	// read back through the library's reader
	std::vector<double> s = read_all(path, "states");
	expect(s.size() == 2 * N * G * 2, "states: 2 slots of N states");
	for (size_t m = 0; m < N && s.size() == 2 * N * G * 2; m++) {
		expect(same_state(&s[m * G * 2], states[m], G), "slot 0 in storage order");
		expect(same_state(&s[(N + m) * G * 2], states[order_arr[m]], G), "slot 1 in the given order");
	}
	std::vector<double> V = read_all(path, "potential_values");
	expect(V.size() == G && std::memcmp(&V[0], pot.get_valueptr(), G * sizeof(double)) == 0, "potential values");
	std::vector<double> h = read_all(path, "state_history");
	expect(h.size() == 4 && h[0] == 3 && h[1] == 0 && h[2] == 7 && h[3] == 1, "state_history");
	std::vector<double> t = read_all(path, "time_step_history");
	expect(t.size() == 4 && t[0] == 1 && t[1] == 0.5 && t[2] == 4 && t[3] == 0.1, "time_step_history");
	std::vector<double> eh = read_all(path, "energy_history");
	expect(eh.size() == 3 * N && std::memcmp(&eh[2 * N], &E[2][0], N * sizeof(double)) == 0, "energy_history");
	std::vector<double> fe = read_all(path, "final_energies");
	expect(fe.size() == N && std::memcmp(&fe[0], &E.back()[0], N * sizeof(double)) == 0, "final_energies");
	expect(read_all(path, "noise_data").empty(), "noise_data of NoNoise is empty");
	unsigned char lay[64];
	int lay_size = 0;
	itp2d_datafile_header_message(path, "energy_history", 8, 0, lay, sizeof lay, &lay_size);
	expect(lay_size >= 3 && lay[0] == 3 && lay[1] == 2, "stored chunked, as the reference's datasets");
	double seed = 0;
	itp2d_datafile_read_attribute(path, "/", "random_seed", &seed);
	expect(seed == 12345.0, "random_seed attribute");
	// --copy-states into a second StateSet: the last slot
	StateSet copy(N, dl);
	itp2d_b200::init_from_datafile(copy, path);
	for (size_t m = 0; m < N; m++)
		expect(std::memcmp(copy[m].data_ptr(), states[order_arr[m]].data_ptr(), G * 2 * sizeof(double)) == 0,
				"init_from_datafile copies the last slot");
	bool threw = false;
	try {
		StateSet other(N - 1, dl);
		itp2d_b200::init_from_datafile(other, path);
	} catch (GeneralError& e) {
		threw = std::strstr(e.what(), "num_states does not match") != NULL;
	}
	expect(threw, "a StateSet of another size is refused with the reference's message");
	std::printf("%s: %d failure(s)\n", failures ? "FAILED" : "ok", failures);
	return failures;
}
