/*
 * Oracle-only stand-in for the HDF5 C++ API names used by the itp2d reference
 * headers (datafile.hpp:32-145) and StateSet::init_from_datafile
 * (stateset.cpp:86-109). Test infrastructure: the oracle never writes or reads
 * datafiles (it runs with Parameters::Nothing), so every operation here throws
 * H5::Exception. Only enough surface exists for the reference sources to
 * compile unmodified.
 */
#ifndef ITP2D_ORACLE_H5CPP_STUB_H
#define ITP2D_ORACLE_H5CPP_STUB_H

#include <string>

typedef unsigned long long hsize_t;
typedef int hid_t;

enum H5F_scope_t { H5F_SCOPE_LOCAL = 0, H5F_SCOPE_GLOBAL = 1 };
enum H5S_class_t { H5S_SCALAR = 0, H5S_SIMPLE = 1, H5S_NULL = 2 };
enum H5S_seloper_t { H5S_SELECT_SET = 0 };
#define H5F_ACC_RDONLY 0u
#define H5F_ACC_RDWR 1u
#define H5F_ACC_TRUNC 2u
#define H5F_ACC_EXCL 4u
#define H5S_UNLIMITED ((hsize_t)(-1))
#define H5I_INVALID_HID (-1)

namespace H5 {

class Exception {
	public:
		Exception() : msg("HDF5 is not available in the itp2d oracle build") {}
		explicit Exception(std::string const& m) : msg(m) {}
		virtual ~Exception() {}
		void printError() const {}
		std::string getDetailMsg() const { return msg; }
		static void dontPrint() {}
	private:
		std::string msg;
};

class GroupIException : public Exception {};

inline void unavailable() { throw Exception(); }

class DataType {
	public:
		DataType() {}
		virtual ~DataType() {}
		void setSize(size_t) { unavailable(); }
};

class AtomType : public DataType {
	public:
		AtomType() {}
		AtomType(DataType const&) {}
};

class PredType : public AtomType {
	public:
		static const PredType C_S1;
		static const PredType NATIVE_INT;
		static const PredType NATIVE_ULONG;
		static const PredType NATIVE_DOUBLE;
};

class CompType : public DataType {
	public:
		CompType() {}
		explicit CompType(size_t) {}
		void insertMember(std::string const&, size_t, DataType const&) { unavailable(); }
};

class ArrayType : public DataType {
	public:
		ArrayType(DataType const&, int, hsize_t const*) {}
};

class DataSpace {
	public:
		DataSpace() {}
		DataSpace(H5S_class_t) {}
		DataSpace(int, hsize_t const*, hsize_t const* = 0) {}
		bool selectValid() const { unavailable(); return false; }
		void getSelectBounds(hsize_t*, hsize_t*) const { unavailable(); }
		void selectHyperslab(H5S_seloper_t, hsize_t const*, hsize_t const*) const { unavailable(); }
};

class DSetCreatPropList {
	public:
		DSetCreatPropList() {}
		void setChunk(int, hsize_t const*) const { unavailable(); }
};

class Attribute {
	public:
		void read(DataType const&, void*) const { unavailable(); }
		void write(DataType const&, void const*) const { unavailable(); }
};

class DataSet {
	public:
		DataType getArrayType() const { unavailable(); return DataType(); }
		DataSpace getSpace() const { unavailable(); return DataSpace(); }
		void read(void*, DataType const&) const { unavailable(); }
		void write(void const*, DataType const&) const { unavailable(); }
		Attribute createAttribute(const char*, DataType const&, DataSpace const&) const { unavailable(); return Attribute(); }
};

class Group {
	public:
		Attribute openAttribute(const char*) const { unavailable(); return Attribute(); }
		Attribute createAttribute(const char*, DataType const&, DataSpace const&) const { unavailable(); return Attribute(); }
};

class H5File {
	public:
		H5File() {}
		void openFile(std::string const&, unsigned) { unavailable(); }
		Group openGroup(const char*) const { unavailable(); return Group(); }
		DataSet openDataSet(const char*) const { unavailable(); return DataSet(); }
		void flush(H5F_scope_t) const { unavailable(); }
};

} // namespace H5

#endif /* ITP2D_ORACLE_H5CPP_STUB_H */
