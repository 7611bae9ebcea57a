/*
 * itp2d_datafile.h -- the reference's HDF5 datafile (Datafile,
 * datafile.hpp:38-147 / datafile.cpp:32-467) and its --copy-states reader
 * (StateSet::init_from_datafile, stateset.cpp:86-109), written and read by
 * this library's own code: no HDF5 library is linked.
 *
 * The files follow the HDF5 file-format specification in its oldest layout
 * (version 0 superblock, version 1 object headers, the root group indexed by
 * a version 1 B-tree, one symbol-table node and a local heap), which every
 * HDF5 release reads. Dataset names, element types, shapes and attribute
 * names and types are those of the reference: "/states" (slots x states of
 * complex[sizey][sizex] arrays), "/state_history" {step, index},
 * "/time_step_history" {step, time_step}, "/energy_history" and
 * "/deviation_history" (steps x states), "/final_energies",
 * "/final_energy_standard_deviations", "/potential_values" (scalar of
 * double[sizey][sizex]), "/noise_data"; complex values are the compound
 * {r, i} of two doubles. Datasets are stored contiguous and uncompressed at
 * their current size unless itp2d_datafile_set_chunking selects the
 * reference's storage (1 x 1 chunks, deflate, unlimited maximum sizes); the
 * file is rewritten as a whole on every flush, and the "description" texts
 * are this library's own. The readers also read chunked, deflated datasets,
 * so files written by the reference itself can seed --copy-states.
 *
 * All functions return ITP2D_OK or an error status (ITP2D_E_INVALID for bad
 * arguments or a mismatching file, ITP2D_E_IO for file-system or format
 * errors); itp2d_datafile_last_error() gives the message of the calling
 * thread's last failure. Host code only: no device memory is touched.
 */
#ifndef ITP2D_DATAFILE_H
#define ITP2D_DATAFILE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status of a failed read or write of a datafile. */
#define ITP2D_E_IO 9

typedef struct itp2d_datafile itp2d_datafile;
struct itp2d_system;

/* Datafile::Datafile (datafile.cpp:32-93): creates the file (clobber = 0
 * fails on an existing file, like H5F_ACC_EXCL), writes the root
 * "description" and the attributes grid_sizex, grid_sizey, grid_delta. */
int itp2d_datafile_create(const char* filename, int sizex, int sizey, double dx, int clobber,
		itp2d_datafile** out);
/* Storage of the datasets written from now on (every flush rewrites them
 * all): deflate_level 0-9 stores them as the reference does (one element per
 * chunk, deflated at that level, unlimited maximum sizes; the reference uses
 * 9, datafile.cpp:76-88); a negative level (the default) stores them
 * contiguous and uncompressed, which is faster to write and read. The scalar
 * "/potential_values" stays contiguous, as in the reference. */
int itp2d_datafile_set_chunking(itp2d_datafile* f, int deflate_level);
/* Writes the whole file as it stands (Datafile::flush, datafile.hpp). */
int itp2d_datafile_flush(itp2d_datafile* f);
/* Flushes and frees (Datafile::~Datafile). */
int itp2d_datafile_close(itp2d_datafile* f);

/* Datafile::add_attribute overloads (datafile.cpp:416-466): scalar root
 * attributes of NATIVE_INT, NATIVE_DOUBLE, NATIVE_ULONG and fixed-length
 * C strings (size = length, at least 1). A name used twice is an error. */
int itp2d_datafile_add_attribute_int(itp2d_datafile* f, const char* name, int value);
int itp2d_datafile_add_attribute_double(itp2d_datafile* f, const char* name, double value);
int itp2d_datafile_add_attribute_ulong(itp2d_datafile* f, const char* name, unsigned long value);
int itp2d_datafile_add_attribute_string(itp2d_datafile* f, const char* name, const char* value);

/* Datafile::write_state (datafile.cpp:207-225): state (sizey*sizex
 * interleaved complex doubles) at slot n, index m; "/states" grows to at
 * least (n+1, m+1), new places zero. */
int itp2d_datafile_write_state(itp2d_datafile* f, long long n, long long m, const double* state);
/* Datafile::write_stateset (datafile.cpp:230-269): the next slot of
 * "/states" receives the num_states states (storage order, or sort_order[m]
 * at index m when sort_order is not NULL) and "/state_history" gets
 * (step, slot). */
int itp2d_datafile_write_stateset(itp2d_datafile* f, const double* states, int num_states, int step,
		const int* sort_order);
/* Datafile::write_time_step_history (datafile.cpp:271-293): appends
 * (step, eps). */
int itp2d_datafile_write_time_step_history(itp2d_datafile* f, int step, double eps);
/* Datafile::write_energy_history / write_deviation_history
 * (datafile.cpp:295-364): row `index` of n values; the dataset grows to at
 * least (index+1, n). */
int itp2d_datafile_write_energy_history(itp2d_datafile* f, const double* values, int n, int index);
int itp2d_datafile_write_deviation_history(itp2d_datafile* f, const double* values, int n, int index);
/* Datafile::write_energies / write_energy_standard_deviations
 * (datafile.cpp:323-336, 366-379). */
int itp2d_datafile_write_energies(itp2d_datafile* f, const double* values, int n);
int itp2d_datafile_write_energy_standard_deviations(itp2d_datafile* f, const double* values, int n);
/* Datafile::write_potential (datafile.cpp:381-392): sizey*sizex doubles. */
int itp2d_datafile_write_potential(itp2d_datafile* f, const double* V);
/* Datafile::write_noise_realization (datafile.cpp:394-410). */
int itp2d_datafile_write_noise_realization(itp2d_datafile* f, const double* values, int n);

/* An itp2d_save_states_fn (itp2d_host.h) that writes the states it is given
 * as a new slot of the datafile passed as `user` (in energy order when
 * `order` is given) and flushes: ITPSystem::save_states
 * (itpsystem.cpp:374-389) with this datafile behind the save callback. */
void itp2d_datafile_save_states(void* user, const double* states, const int* order, int num_states, int sx,
		int sy, int step);

/* The datafile of a solve, as the reference's ITPSystem writes it with
 * --save final states (itpsystem.cpp:69-116, 220-226, 390-402, 440-453, 513-531): the run
 * attributes, "/potential_values" (when the potential is not zero),
 * "/noise_data" (empty: impurities are passed in explicitly),
 * "/time_step_history", "/energy_history", "/deviation_history", the final
 * energies and deviations, and, when save_states is 1, the states in energy
 * order as one slot. */
int itp2d_system_write_datafile(struct itp2d_system* s, const char* filename, int clobber, int save_states);

/* StateSet::init_from_datafile (stateset.cpp:86-109): checks the file's
 * num_states, grid_sizex, grid_sizey and grid_delta against the arguments
 * (ITP2D_E_INVALID with the reference's message on a mismatch; grid_sizey
 * is read from grid_sizey, where the reference reads grid_sizex twice) and
 * copies the states of the last slot of "/states" into `states`
 * (num_states*sizey*sizex interleaved complex doubles). */
int itp2d_datafile_init_states(const char* filename, int num_states, int sizex, int sizey, double dx,
		double* states);

/* Generic readers, for HDF5 files in the layouts above (version 0 or 1
 * superblock after an optional user block, version 1 object headers with
 * continuation blocks, symbol-table groups, contiguous or compact storage;
 * integer, IEEE float, string, compound and array element types).
 * Shape of a dataset: rank (0 for a scalar), dims[0..rank-1] (at most 8)
 * and the number of numeric values in one element. */
int itp2d_datafile_dataset_shape(const char* filename, const char* dataset, int* rank, long long* dims,
		long long* values_per_element);
/* Every numeric value of the dataset in storage order (compound members in
 * their order, array elements row-major) converted to double; at most
 * max_values are written, *n_values receives the total. */
int itp2d_datafile_read_values(const char* filename, const char* dataset, double* out, long long max_values,
		long long* n_values);
/* A scalar numeric attribute of the root group (object "/" or NULL) or of a
 * dataset, converted to double. */
int itp2d_datafile_read_attribute(const char* filename, const char* object, const char* name, double* value);
/* A string attribute, NUL-terminated into buf (at most buflen-1 bytes). */
int itp2d_datafile_read_string_attribute(const char* filename, const char* object, const char* name, char* buf,
		int buflen);
/* The encoded body of the index-th header message of the given message type
 * of an object, for format checks: bytes copied to buf (at most buflen),
 * *size receives the body's size. */
int itp2d_datafile_header_message(const char* filename, const char* object, int type, int index,
		unsigned char* buf, int buflen, int* size);

/* Message of the calling thread's last failed datafile call, or "". */
const char* itp2d_datafile_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
