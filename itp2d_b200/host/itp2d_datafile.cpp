// The reference's HDF5 datafile (Datafile, datafile.cpp:32-467) and the
// --copy-states reader (StateSet::init_from_datafile, stateset.cpp:86-109),
// written and read here without an HDF5 library (none is installed).
//
// Writer. The file is built in memory and written as a whole on every flush,
// in the HDF5 format's oldest layout, which every HDF5 release reads:
//   superblock version 0 (offsets and lengths of 8 bytes, no user block)
//   root group object header (version 1): symbol-table message + attributes
//   local heap ("HEAP") holding the link names, "" at offset 0
//   one version 1 B-tree leaf ("TREE", group type) with one child, the
//   symbol-table node ("SNOD") listing the datasets sorted by name
//   one version 1 object header per dataset: fill value, datatype, dataspace,
//   layout (version 3, contiguous), attributes
//   the raw data of every dataset, 8-byte aligned.
// The encodings of the superblock, heap, B-tree and symbol-table node, the
// version 1 object header, the IEEE double and C-string datatypes, the
// version 1 dataspace, the fill-value message and the version 1 attribute
// message follow the HDF5 file-format specification and match, field for
// field, a file written by the HDF5 library itself (the tests compare them).
// Compound (version 1) and array (version 2) datatypes follow the
// specification.
//
// Reader. Parses the same layouts (superblock version 0 or 1 after an
// optional user block, version 1 object headers with continuation blocks,
// multi-level group B-trees, layout messages version 1-3 with contiguous or
// compact storage, attribute messages version 1-3, datatype classes integer,
// float, string, compound and array). Chunked storage and version 2 object
// headers are reported as unsupported.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <zlib.h>

#include "../../include/itp2d_datafile.h"
#include "../../include/itp2d_gpu.h"

namespace {

thread_local std::string g_error;

struct Failure : std::runtime_error {
	int status;
	Failure(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

[[noreturn]] void io_fail(const std::string& m) { throw Failure(ITP2D_E_IO, m); }
[[noreturn]] void bad_arg(const std::string& m) { throw Failure(ITP2D_E_INVALID, m); }

template <typename F>
int guarded(F&& f) {
	try {
		f();
		g_error.clear();
		return ITP2D_OK;
	} catch (Failure& e) {
		g_error = e.what();
		return e.status;
	} catch (std::bad_alloc&) {
		g_error = "out of host memory";
		return ITP2D_E_OOM;
	} catch (std::exception& e) {  // nothing else may cross the C ABI
		g_error = e.what();
		return ITP2D_E_IO;
	}
}

constexpr uint64_t kUndef = ~0ull;
constexpr int kLeafK = 16;      // a symbol-table node holds up to 2K entries
constexpr int kInternalK = 16;  // a group B-tree node holds up to 2K children
constexpr size_t kSuperblockBytes = 96;
constexpr size_t kBtreeBytes = 24 + 2 * kInternalK * 8 + (2 * kInternalK + 1) * 8;
constexpr size_t kSnodBytes = 8 + 2 * kLeafK * 40;
constexpr size_t kHeapHeaderBytes = 32;
constexpr uint64_t kHeapFreeNull = 1;  // "no free block" in a local heap's free list

size_t round8(size_t n) { return (n + 7) & ~size_t(7); }

// ---------------------------------------------------------------- datatypes

struct Type;
using TypeP = std::shared_ptr<const Type>;
struct Member {
	std::string name;
	uint32_t offset;
	TypeP type;
};
struct Type {
	enum Class { kInt = 0, kFloat = 1, kString = 3, kCompound = 6, kArray = 10 };
	Class cls = kInt;
	uint32_t size = 0;
	bool is_signed = true;        // kInt
	std::vector<Member> members;  // kCompound
	std::vector<uint32_t> dims;   // kArray
	TypeP base;                   // kArray
};

TypeP int_type(uint32_t size, bool sign) {
	auto t = std::make_shared<Type>();
	t->cls = Type::kInt;
	t->size = size;
	t->is_signed = sign;
	return t;
}
TypeP double_type() {
	auto t = std::make_shared<Type>();
	t->cls = Type::kFloat;
	t->size = 8;
	return t;
}
TypeP string_type(uint32_t n) {
	auto t = std::make_shared<Type>();
	t->cls = Type::kString;
	t->size = n;
	return t;
}
TypeP compound_type(uint32_t size, std::vector<Member> m) {
	auto t = std::make_shared<Type>();
	t->cls = Type::kCompound;
	t->size = size;
	t->members = std::move(m);
	return t;
}
TypeP array_type(TypeP base, std::vector<uint32_t> dims) {
	auto t = std::make_shared<Type>();
	t->cls = Type::kArray;
	uint64_t n = base->size;
	for (uint32_t d : dims) n *= d;
	if (n > 0xffffffffull) bad_arg("array element too large for a datatype");
	t->size = (uint32_t)n;
	t->dims = std::move(dims);
	t->base = std::move(base);
	return t;
}

// The reference's element types (datafile.cpp:56-70).
TypeP complex_type() { return compound_type(16, {{"r", 0, double_type()}, {"i", 8, double_type()}}); }
TypeP state_history_type() { return compound_type(8, {{"step", 0, int_type(4, true)}, {"index", 4, int_type(4, true)}}); }
TypeP time_step_history_type() {
	return compound_type(16, {{"step", 0, int_type(4, true)}, {"time_step", 8, double_type()}});
}

// ---------------------------------------------------------------- encoding

struct Out {
	std::vector<uint8_t> b;
	void u8(unsigned v) { b.push_back((uint8_t)v); }
	void u16(unsigned v) {
		u8(v & 0xff);
		u8((v >> 8) & 0xff);
	}
	void u32(uint32_t v) {
		for (int i = 0; i < 4; i++) u8((v >> (8 * i)) & 0xff);
	}
	void u64(uint64_t v) {
		for (int i = 0; i < 8; i++) u8((v >> (8 * i)) & 0xff);
	}
	void raw(const void* p, size_t n) {
		const uint8_t* c = static_cast<const uint8_t*>(p);
		b.insert(b.end(), c, c + n);
	}
	void zeros(size_t n) { b.insert(b.end(), n, 0); }
	// a NUL-terminated name padded with NULs to a multiple of 8 bytes
	void name8(const std::string& s) {
		raw(s.c_str(), s.size() + 1);
		zeros(round8(s.size() + 1) - (s.size() + 1));
	}
	void pad_to(size_t n) {
		if (b.size() < n) zeros(n - b.size());
	}
	size_t size() const { return b.size(); }
};

void encode_type(Out& o, const Type& t) {
	switch (t.cls) {
	case Type::kInt:  // version 1, little-endian two's complement or unsigned
		o.u8(0x10);
		o.u8(t.is_signed ? 0x08 : 0x00);
		o.u8(0);
		o.u8(0);
		o.u32(t.size);
		o.u16(0);           // bit offset
		o.u16(8 * t.size);  // bit precision
		break;
	case Type::kFloat:  // version 1, IEEE 754 binary64, little-endian
		o.u8(0x11);
		o.u8(0x20);  // mantissa normalisation: implied leading bit
		o.u8(63);    // sign bit position
		o.u8(0);
		o.u32(8);
		o.u16(0);   // bit offset
		o.u16(64);  // bit precision
		o.u8(52);   // exponent position
		o.u8(11);   // exponent size
		o.u8(0);    // mantissa position
		o.u8(52);   // mantissa size
		o.u32(1023);
		break;
	case Type::kString:  // version 1, NUL-terminated ASCII
		o.u8(0x13);
		o.u8(0);
		o.u8(0);
		o.u8(0);
		o.u32(t.size);
		break;
	case Type::kCompound:  // version 1: every member with the (unused) array-dimension fields
		o.u8(0x16);
		o.u16((unsigned)t.members.size());
		o.u8(0);
		o.u32(t.size);
		for (const Member& m : t.members) {
			o.name8(m.name);
			o.u32(m.offset);
			o.u8(0);  // dimensionality
			o.zeros(3);
			o.u32(0);  // dimension permutation
			o.u32(0);
			o.zeros(16);  // four dimension sizes
			encode_type(o, *m.type);
		}
		break;
	case Type::kArray:  // version 2 (the first version with the array class)
		o.u8(0x2a);
		o.u8(0);
		o.u8(0);
		o.u8(0);
		o.u32(t.size);
		o.u8((unsigned)t.dims.size());
		o.zeros(3);
		for (uint32_t d : t.dims) o.u32(d);
		for (size_t i = 0; i < t.dims.size(); i++) o.u32((uint32_t)i);  // permutation: identity
		encode_type(o, *t.base);
		break;
	}
}

// Version 1 dataspace; no dims = scalar. The maximum sizes equal the sizes,
// or are unlimited (extendible, as the reference creates its datasets).
void encode_space(Out& o, const std::vector<uint64_t>& dims, bool unlimited = false) {
	o.u8(1);
	o.u8((unsigned)dims.size());
	o.u8(unlimited ? 1 : 0);
	o.u8(0);
	o.u32(0);
	for (uint64_t d : dims) o.u64(d);
	if (unlimited)
		for (size_t i = 0; i < dims.size(); i++) o.u64(kUndef);
}

struct Attr {
	std::string name;
	TypeP type;
	std::vector<uint8_t> data;  // one element (scalar dataspace)
};

// Version 1 attribute message: sizes unpadded, fields padded to 8 bytes.
void encode_attr(Out& o, const Attr& a) {
	Out t, s;
	encode_type(t, *a.type);
	encode_space(s, {});
	o.u8(1);
	o.u8(0);
	o.u16((unsigned)a.name.size() + 1);
	o.u16((unsigned)t.size());
	o.u16((unsigned)s.size());
	o.name8(a.name);
	o.raw(t.b.data(), t.size());
	o.zeros(round8(t.size()) - t.size());
	o.raw(s.b.data(), s.size());
	o.zeros(round8(s.size()) - s.size());
	o.raw(a.data.data(), a.data.size());
}

struct Msg {
	uint16_t type;
	uint8_t flags;
	std::vector<uint8_t> data;
};

// Version 1 object header: 16-byte prefix, then 8-byte-aligned messages.
std::vector<uint8_t> object_header(const std::vector<Msg>& msgs) {
	size_t body = 0;
	for (const Msg& m : msgs) {
		if (round8(m.data.size()) > 0xffff) bad_arg("header message larger than 64 KiB (attribute too long)");
		body += 8 + round8(m.data.size());
	}
	Out o;
	o.u8(1);
	o.u8(0);
	o.u16((unsigned)msgs.size());
	o.u32(1);  // reference count
	o.u32((uint32_t)body);
	o.u32(0);
	for (const Msg& m : msgs) {
		o.u16(m.type);
		o.u16((unsigned)round8(m.data.size()));
		o.u8(m.flags);
		o.zeros(3);
		o.raw(m.data.data(), m.data.size());
		o.zeros(round8(m.data.size()) - m.data.size());
	}
	return o.b;
}

constexpr uint16_t kMsgNil = 0x0000, kMsgSpace = 0x0001, kMsgType = 0x0003, kMsgFill = 0x0005,
		kMsgLayout = 0x0008, kMsgFilters = 0x000b, kMsgAttr = 0x000c, kMsgCont = 0x0010, kMsgSymtab = 0x0011;
constexpr uint8_t kConstant = 0x01;

Msg attr_msg(const Attr& a) {
	Out o;
	encode_attr(o, a);
	return {kMsgAttr, 0, o.b};
}

// ---------------------------------------------------------------- the file in memory

struct Dataset {
	TypeP type;
	std::vector<uint64_t> dims;  // empty: scalar
	std::vector<uint8_t> data;   // row-major elements
	std::vector<Attr> attrs;
	uint64_t elements() const {
		uint64_t n = 1;
		for (uint64_t d : dims) n *= d;
		return n;
	}
};

Attr string_attr(const std::string& name, const std::string& value) {
	// C_S1 sized to the string (datafile.cpp:453-466); an empty string keeps size 1
	Attr a;
	a.name = name;
	const size_t n = std::max<size_t>(1, value.size());
	a.type = string_type((uint32_t)n);
	a.data.assign(n, 0);
	std::memcpy(a.data.data(), value.data(), value.size());
	return a;
}

template <typename T>
Attr value_attr(const std::string& name, TypeP type, T v) {
	Attr a;
	a.name = name;
	a.type = std::move(type);
	a.data.resize(sizeof(T));
	std::memcpy(a.data.data(), &v, sizeof(T));
	return a;
}

// Grows a dataset to at least new_dims (same rank), keeping every element at
// its index and zero-filling the new ones (H5Dextend, then the fill value).
void grow(Dataset& d, const std::vector<uint64_t>& want) {
	std::vector<uint64_t> nd = d.dims;
	bool changed = false;
	for (size_t i = 0; i < nd.size(); i++)
		if (want[i] > nd[i]) {
			nd[i] = want[i];
			changed = true;
		}
	if (!changed) return;
	const size_t es = d.type->size;
	uint64_t n = 1;
	for (uint64_t x : nd) n *= x;
	std::vector<uint8_t> out(n * es, 0);
	if (nd.size() == 1) {
		if (!d.data.empty()) std::memcpy(out.data(), d.data.data(), d.data.size());
	} else if (d.dims[1] > 0) {  // rank 2
		for (uint64_t r = 0; r < d.dims[0]; r++)
			std::memcpy(out.data() + r * nd[1] * es, d.data.data() + r * d.dims[1] * es, d.dims[1] * es);
	}
	d.dims = nd;
	d.data.swap(out);
}

}  // namespace

struct itp2d_datafile {
	std::string path;
	int sx = 0, sy = 0;
	double dx = 0;
	std::vector<Attr> root_attrs;
	std::map<std::string, Dataset> sets;  // by name without '/', sorted like the symbol-table node
	int deflate = -1;                     // < 0: contiguous datasets; 0-9: chunked, deflated at this level

	void add_root_attr(Attr a) {
		for (const Attr& b : root_attrs)
			if (b.name == a.name) bad_arg("attribute '" + a.name + "' already exists");
		root_attrs.push_back(std::move(a));
	}

	// the reference's lazily created datasets (datafile.cpp:130-200), with a
	// description of their own
	Dataset& ensure(const std::string& name) {
		auto it = sets.find(name);
		if (it != sets.end()) return it->second;
		Dataset d;
		std::string text;
		if (name == "states") {
			d.type = array_type(complex_type(), {(uint32_t)sy, (uint32_t)sx});
			d.dims = {0, 0};
			text = "Saved state sets: index 0 is the save slot (see state_history), index 1 the state within the "
			       "set; each element is one wave function on the sizey x sizex grid as complex {r, i} values.";
		} else if (name == "state_history") {
			d.type = state_history_type();
			d.dims = {0};
			text = "One (step, index) pair per saved state set: the iteration after which it was saved and its "
			       "slot (first index) in states.";
		} else if (name == "final_energies") {
			d.type = double_type();
			d.dims = {0};
			text = "The last energy of every state, in ascending order.";
		} else if (name == "time_step_history") {
			d.type = time_step_history_type();
			d.dims = {0};
			text = "One (step, time_step) pair per time-step value: the first iteration that used it and the value.";
		} else if (name == "energy_history") {
			d.type = double_type();
			d.dims = {0, 0};
			text = "Energies of all states after every iteration: index 0 is the iteration, index 1 the state in "
			       "ascending order of energy.";
		} else if (name == "final_energy_standard_deviations") {
			d.type = double_type();
			d.dims = {0};
			text = "The last energy standard deviation of every state, in the order of final_energies.";
		} else if (name == "deviation_history") {
			d.type = double_type();
			d.dims = {0, 0};
			text = "Energy standard deviations of all states after every iteration, indexed like energy_history.";
		} else if (name == "potential_values") {
			d.type = array_type(double_type(), {(uint32_t)sy, (uint32_t)sx});
			d.dims = {};
			d.data.assign(d.type->size, 0);
			text = "The external potential at every grid point (sizey x sizex).";
		} else if (name == "noise_data") {
			d.type = double_type();
			d.dims = {0};
			text = "The data that reproduces the potential's random part (empty when there is none).";
		} else {
			bad_arg("unknown dataset " + name);
		}
		d.attrs.push_back(string_attr("description", text));
		return sets.emplace(name, std::move(d)).first->second;
	}

	std::vector<uint8_t> serialise() const;
	void write() const;
};

namespace {

std::vector<uint8_t> layout_msg(uint64_t addr, uint64_t size) {
	Out o;
	o.u8(3);  // version 3
	o.u8(1);  // contiguous
	o.u64(addr);
	o.u64(size);
	return o.b;
}

// K of the chunk-index B-trees: a version 0 superblock has no field for it,
// so readers take the format's default.
constexpr int kChunkK = 32;

// Chunked storage as the reference's datasets have it (datafile.cpp:76-88):
// one element per chunk, each deflated, indexed by a version 1 B-tree (type 1)
// whose nodes hold up to 2K chunks. Returns the bytes to place at `start`;
// *root receives the B-tree's address (undefined for an empty dataset).
std::vector<uint8_t> chunk_storage(const Dataset& d, uint64_t start, int level, uint64_t* root) {
	const size_t rank = d.dims.size();
	const uint64_t es = d.type->size, n = d.elements();
	*root = kUndef;
	Out o;
	if (n == 0) return o.b;
	struct Key {
		uint32_t size;
		std::vector<uint64_t> off;  // rank offsets, then the element's byte offset
	};
	std::vector<Key> keys(n);
	std::vector<uint64_t> addr(n);
	std::vector<uint8_t> z(compressBound((uLong)es));
	std::vector<uint64_t> idx(rank, 0);
	for (uint64_t e = 0; e < n; e++) {
		uLongf len = (uLongf)z.size();
		if (compress2(z.data(), &len, d.data.data() + e * es, (uLong)es, level) != Z_OK) io_fail("deflate failed");
		addr[e] = start + o.size();
		o.raw(z.data(), len);
		keys[e].size = (uint32_t)len;
		keys[e].off = idx;
		keys[e].off.push_back(0);
		for (size_t i = rank; i-- > 0;) {
			if (++idx[i] < d.dims[i]) break;
			idx[i] = 0;
		}
	}
	// the right boundary of the last chunk: its offsets plus the chunk dimensions
	Key right = {0, keys.back().off};
	for (size_t i = 0; i < rank; i++) right.off[i] += 1;
	right.off[rank] = es;
	const size_t ks = 8 + 8 * (rank + 1);
	const size_t node_bytes = 24 + 2 * kChunkK * 8 + (2 * kChunkK + 1) * ks;
	auto put_key = [](Out& w, const Key& k) {
		w.u32(k.size);
		w.u32(0);  // filter mask: every filter applied
		for (uint64_t x : k.off) w.u64(x);
	};
	o.pad_to(round8(o.size()));
	// level by level: the children (addresses and left keys) grouped into nodes
	std::vector<uint64_t> child_addr = addr;
	std::vector<Key> child_key = keys;
	for (int lvl = 0;; lvl++) {
		const size_t per = 2 * kChunkK, nn = (child_addr.size() + per - 1) / per;
		const uint64_t first = start + o.size();
		std::vector<uint64_t> node_addr(nn);
		std::vector<Key> node_key(nn);
		for (size_t j = 0; j < nn; j++) {
			node_addr[j] = first + j * node_bytes;
			const size_t b = j * per, e = std::min(child_addr.size(), b + per);
			node_key[j] = child_key[b];
			Out w;
			w.raw("TREE", 4);
			w.u8(1);  // chunk index
			w.u8((unsigned)lvl);
			w.u16((unsigned)(e - b));
			w.u64(j > 0 ? first + (j - 1) * node_bytes : kUndef);
			w.u64(j + 1 < nn ? first + (j + 1) * node_bytes : kUndef);
			for (size_t c = b; c < e; c++) {
				put_key(w, child_key[c]);
				w.u64(child_addr[c]);
			}
			put_key(w, e < child_addr.size() ? child_key[e] : right);
			w.pad_to(node_bytes);
			o.raw(w.b.data(), w.size());
		}
		if (nn == 1) {
			*root = node_addr[0];
			break;
		}
		child_addr.swap(node_addr);
		child_key.swap(node_key);
	}
	return o.b;
}

bool is_chunked(const Dataset& d, int level) { return level >= 0 && !d.dims.empty(); }

std::vector<Msg> dataset_msgs(const Dataset& d, uint64_t addr, int level) {
	const bool chunked = is_chunked(d, level);
	std::vector<Msg> m;
	// fill value message version 1: allocation late (incremental when chunked),
	// fill written if set, default (zero) fill
	m.push_back({kMsgFill, kConstant, {1, (uint8_t)(chunked ? 3 : 2), 2, 1, 0, 0, 0, 0}});
	Out t, s;
	encode_type(t, *d.type);
	encode_space(s, d.dims, chunked);
	m.push_back({kMsgType, kConstant, t.b});
	m.push_back({kMsgSpace, 0, s.b});
	if (chunked) {
		Out l;
		l.u8(3);  // version 3
		l.u8(2);  // chunked
		l.u8((unsigned)d.dims.size() + 1);
		l.u64(addr);
		for (size_t i = 0; i < d.dims.size(); i++) l.u32(1);
		l.u32(d.type->size);
		m.push_back({kMsgLayout, kConstant, l.b});
		Out f;  // filter pipeline version 1: deflate at `level`
		f.u8(1);
		f.u8(1);
		f.zeros(6);
		f.u16(1);  // deflate
		f.u16(8);  // name length, padded
		f.u16(0);  // mandatory
		f.u16(1);  // one client value
		f.name8("deflate");
		f.u32((uint32_t)level);
		f.u32(0);  // padding after an odd number of values
		m.push_back({kMsgFilters, kConstant, f.b});
	} else {
		m.push_back({kMsgLayout, kConstant, layout_msg(d.data.empty() ? kUndef : addr, d.data.size())});
	}
	for (const Attr& a : d.attrs) m.push_back(attr_msg(a));
	return m;
}

}  // namespace

std::vector<uint8_t> itp2d_datafile::serialise() const {
	if (sets.size() > 2 * kLeafK) bad_arg("too many datasets for one symbol-table node");
	// local heap data: "" at 0, then every name padded to 8 bytes
	Out heap;
	heap.zeros(8);
	std::vector<uint64_t> name_off;
	for (const auto& kv : sets) {
		name_off.push_back(heap.size());
		heap.name8(kv.first);
	}
	// root object header: symbol-table message + root attributes
	std::vector<Msg> root_msgs;
	root_msgs.push_back({kMsgSymtab, kConstant, std::vector<uint8_t>(16, 0)});
	for (const Attr& a : root_attrs) root_msgs.push_back(attr_msg(a));
	const size_t root_bytes = object_header(root_msgs).size();
	// addresses
	const uint64_t a_root = kSuperblockBytes;
	const uint64_t a_heap = round8(a_root + root_bytes);
	const uint64_t a_heap_data = a_heap + kHeapHeaderBytes;
	const uint64_t a_btree = round8(a_heap_data + heap.size());
	const uint64_t a_snod = a_btree + kBtreeBytes;
	uint64_t at = sets.empty() ? a_snod : a_snod + kSnodBytes;
	std::vector<uint64_t> a_hdr, a_raw;
	std::vector<size_t> hdr_bytes;
	for (const auto& kv : sets) {
		a_hdr.push_back(at);
		hdr_bytes.push_back(object_header(dataset_msgs(kv.second, 0, deflate)).size());
		at = round8(at + hdr_bytes.back());
	}
	std::vector<std::vector<uint8_t>> chunks;  // chunked storage of each dataset
	std::vector<uint64_t> a_layout;
	for (const auto& kv : sets) {
		a_raw.push_back(at);
		uint64_t la = kv.second.data.empty() ? kUndef : at;
		chunks.emplace_back();
		if (is_chunked(kv.second, deflate)) chunks.back() = chunk_storage(kv.second, at, deflate, &la);
		a_layout.push_back(la);
		at = round8(at + (is_chunked(kv.second, deflate) ? chunks.back().size() : kv.second.data.size()));
	}
	const uint64_t eof = at;

	Out f;
	// superblock version 0
	const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
	f.raw(sig, 8);
	f.u8(0);  // superblock version
	f.u8(0);  // free-space storage version
	f.u8(0);  // root group symbol-table entry version
	f.u8(0);
	f.u8(0);  // shared header message format version
	f.u8(8);  // size of offsets
	f.u8(8);  // size of lengths
	f.u8(0);
	f.u16(kLeafK);
	f.u16(kInternalK);
	f.u32(0);  // file consistency flags
	f.u64(0);  // base address
	f.u64(kUndef);  // free-space info
	f.u64(eof);
	f.u64(kUndef);  // driver information block
	// root group symbol-table entry, with the B-tree and heap addresses cached
	f.u64(0);
	f.u64(a_root);
	f.u32(1);
	f.u32(0);
	f.u64(a_btree);
	f.u64(a_heap);
	// root object header
	{
		Out st;
		st.u64(a_btree);
		st.u64(a_heap);
		root_msgs[0].data = st.b;
		const auto h = object_header(root_msgs);
		f.raw(h.data(), h.size());
	}
	f.pad_to(a_heap);
	// local heap
	f.raw("HEAP", 4);
	f.u8(0);
	f.zeros(3);
	f.u64(heap.size());
	f.u64(kHeapFreeNull);
	f.u64(a_heap_data);
	f.raw(heap.b.data(), heap.size());
	f.pad_to(a_btree);
	// group B-tree: one leaf whose only child is the symbol-table node
	f.raw("TREE", 4);
	f.u8(0);  // group node
	f.u8(0);  // leaf
	f.u16(sets.empty() ? 0 : 1);
	f.u64(kUndef);
	f.u64(kUndef);
	f.u64(0);  // key 0: the empty name
	if (!sets.empty()) {
		f.u64(a_snod);
		f.u64(name_off.back());  // key 1: the last name of the child
	}
	f.pad_to(a_btree + kBtreeBytes);
	if (!sets.empty()) {
		f.raw("SNOD", 4);
		f.u8(1);
		f.u8(0);
		f.u16((unsigned)sets.size());
		for (size_t i = 0; i < sets.size(); i++) {
			f.u64(name_off[i]);
			f.u64(a_hdr[i]);
			f.u32(0);  // nothing cached
			f.u32(0);
			f.zeros(16);
		}
		f.pad_to(a_snod + kSnodBytes);
	}
	size_t i = 0;
	for (const auto& kv : sets) {
		f.pad_to(a_hdr[i]);
		const auto h = object_header(dataset_msgs(kv.second, a_layout[i], deflate));
		if (h.size() != hdr_bytes[i]) io_fail("internal: header size changed");
		f.raw(h.data(), h.size());
		i++;
	}
	i = 0;
	for (const auto& kv : sets) {
		f.pad_to(a_raw[i]);
		if (is_chunked(kv.second, deflate))
			f.raw(chunks[i].data(), chunks[i].size());
		else
			f.raw(kv.second.data.data(), kv.second.data.size());
		i++;
	}
	f.pad_to(eof);
	return f.b;
}

void itp2d_datafile::write() const {
	const std::vector<uint8_t> bytes = serialise();
	FILE* fp = std::fopen(path.c_str(), "wb");
	if (!fp) io_fail("cannot write datafile '" + path + "': " + std::strerror(errno));
	const size_t n = std::fwrite(bytes.data(), 1, bytes.size(), fp);
	const int c = std::fclose(fp);
	if (n != bytes.size() || c != 0) io_fail("short write to datafile '" + path + "'");
}

// ---------------------------------------------------------------- reader

namespace {

struct Reader {
	std::vector<uint8_t> d;
	uint64_t base = 0;      // absolute position of the superblock's base address
	uint64_t root_hdr = 0;  // relative
	uint8_t so = 8, sl = 8;

	explicit Reader(const char* path) {
		if (!path) bad_arg("filename is NULL");
		struct stat sb;
		if (::stat(path, &sb) == 0 && !S_ISREG(sb.st_mode))
			io_fail(std::string("datafile '") + path + "' is not a regular file");
		FILE* fp = std::fopen(path, "rb");
		if (!fp) io_fail(std::string("cannot open datafile '") + path + "': " + std::strerror(errno));
		std::fseek(fp, 0, SEEK_END);
		const long n = std::ftell(fp);
		std::fseek(fp, 0, SEEK_SET);
		if (n < 0) {
			std::fclose(fp);
			io_fail(std::string("cannot size datafile '") + path + "'");
		}
		d.resize(n > 0 ? (size_t)n : 0);
		const size_t got = d.empty() ? 0 : std::fread(d.data(), 1, d.size(), fp);
		std::fclose(fp);
		if (got != d.size()) io_fail(std::string("cannot read datafile '") + path + "'");
		parse_superblock();
	}

	void need(uint64_t at, uint64_t n) const {
		if (at > d.size() || n > d.size() - at) io_fail("datafile truncated or corrupt (read past the end)");
	}
	uint64_t uint(uint64_t at, int n) const {
		need(at, n);
		uint64_t v = 0;
		for (int i = 0; i < n; i++) v |= (uint64_t)d[at + i] << (8 * i);
		return v;
	}
	uint64_t abs(uint64_t rel) const { return base + rel; }
	void expect(uint64_t at, const char* sig) const {
		need(at, 4);
		if (std::memcmp(&d[at], sig, 4) != 0) io_fail(std::string("datafile corrupt: no ") + sig + " signature");
	}

	void parse_superblock() {
		static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
		uint64_t at = 0;
		for (;;) {  // at 0, 512, 1024, 2048, ...
			if (at + 8 > d.size()) io_fail("not an HDF5 file (no superblock signature)");
			if (std::memcmp(&d[at], sig, 8) == 0) break;
			at = at ? 2 * at : 512;
		}
		const int version = (int)uint(at + 8, 1);
		if (version > 1) io_fail("superblock version " + std::to_string(version) + " is not supported");
		so = (uint8_t)uint(at + 13, 1);
		sl = (uint8_t)uint(at + 14, 1);
		if (so != 8 || sl != 8) io_fail("only 8-byte offsets and lengths are supported");
		uint64_t p = at + 24 + (version == 1 ? 4 : 0);
		base = uint(p, 8);
		p += 32;  // base, free space, end of file, driver block
		// root group symbol-table entry: link name offset, object header address
		root_hdr = uint(p + 8, 8);
	}

	struct RawMsg {
		uint16_t type;
		uint64_t at;  // absolute position of the body
		uint64_t size;
	};

	std::vector<RawMsg> messages(uint64_t rel) const {
		const uint64_t at = abs(rel);
		need(at, 16);
		if (d[at] != 1) {
			if (d[at] == 'O') io_fail("version 2 object headers are not supported");
			io_fail("unsupported object header version " + std::to_string(d[at]));
		}
		const uint64_t nmsgs = uint(at + 2, 2);
		std::vector<std::pair<uint64_t, uint64_t>> blocks{{at + 16, uint(at + 8, 4)}};
		std::vector<RawMsg> out;
		for (size_t b = 0; b < blocks.size() && out.size() < nmsgs; b++) {
			uint64_t p = blocks[b].first;
			const uint64_t end = p + blocks[b].second;
			need(blocks[b].first, blocks[b].second);
			while (p + 8 <= end && out.size() < nmsgs) {
				const uint16_t type = (uint16_t)uint(p, 2);
				const uint64_t size = uint(p + 2, 2);
				need(p + 8, size);
				if (type == kMsgCont) blocks.push_back({abs(uint(p + 8, 8)), uint(p + 16, 8)});
				out.push_back({type, p + 8, size});
				p += 8 + size;
			}
			if (blocks.size() > 4096) io_fail("datafile corrupt: too many header continuation blocks");
		}
		return out;
	}

	const RawMsg* find(const std::vector<RawMsg>& m, uint16_t type) const {
		for (const RawMsg& x : m)
			if (x.type == type) return &x;
		return nullptr;
	}

	std::string heap_string(uint64_t data_at, uint64_t data_size, uint64_t off) const {
		if (off >= data_size) io_fail("datafile corrupt: name outside the local heap");
		std::string s;
		for (uint64_t p = data_at + off; p < data_at + data_size; p++) {
			need(p, 1);
			if (!d[p]) return s;
			s.push_back((char)d[p]);
		}
		io_fail("datafile corrupt: unterminated name");
	}

	void btree_entries(uint64_t rel, uint64_t heap_at, uint64_t heap_size,
			std::vector<std::pair<std::string, uint64_t>>& out, int depth) const {
		if (depth > 64) io_fail("datafile corrupt: group B-tree too deep");
		const uint64_t at = abs(rel);
		expect(at, "TREE");
		if (uint(at + 4, 1) != 0) io_fail("datafile corrupt: not a group B-tree");
		const int level = (int)uint(at + 5, 1);
		const uint64_t n = uint(at + 6, 2);
		for (uint64_t i = 0; i < n; i++) {
			const uint64_t child = uint(at + 24 + 8 + 16 * i, 8);
			if (level > 0) {
				btree_entries(child, heap_at, heap_size, out, depth + 1);
				continue;
			}
			const uint64_t s = abs(child);
			expect(s, "SNOD");
			const uint64_t nsym = uint(s + 6, 2);
			for (uint64_t j = 0; j < nsym; j++) {
				const uint64_t e = s + 8 + 40 * j;
				out.push_back({heap_string(heap_at, heap_size, uint(e, 8)), uint(e + 8, 8)});
			}
		}
	}

	// address (relative) of an object named "/name", "name" or "/" (the root)
	uint64_t lookup(const char* name) const {
		std::string n = name ? name : "/";
		while (!n.empty() && n[0] == '/') n.erase(0, 1);
		if (n.empty()) return root_hdr;
		if (n.find('/') != std::string::npos) bad_arg("only objects in the root group are supported: " + n);
		const auto m = messages(root_hdr);
		const RawMsg* st = find(m, kMsgSymtab);
		if (!st) io_fail("the root group has no symbol table (new-style groups are not supported)");
		const uint64_t bt = uint(st->at, 8), heap = abs(uint(st->at + 8, 8));
		expect(heap, "HEAP");
		const uint64_t heap_size = uint(heap + 8, 8), heap_data = abs(uint(heap + 24, 8));
		std::vector<std::pair<std::string, uint64_t>> entries;
		btree_entries(bt, heap_data, heap_size, entries, 0);
		for (const auto& e : entries)
			if (e.first == n) return e.second;
		bad_arg("no dataset '" + n + "' in the datafile");
	}

	// datatype at absolute position p; returns the type and advances p
	TypeP decode_type(uint64_t& p, int depth = 0) const {
		if (depth > 32) io_fail("datatype nested too deeply");
		need(p, 8);
		const int cls = d[p] & 0x0f, version = d[p] >> 4;
		const uint8_t b0 = d[p + 1], b1 = d[p + 2];
		const uint32_t size = (uint32_t)uint(p + 4, 4);
		p += 8;
		auto t = std::make_shared<Type>();
		t->size = size;
		switch (cls) {
		case 0:
			if (b0 & 1) io_fail("big-endian integers are not supported");
			t->cls = Type::kInt;
			t->is_signed = (b0 & 0x08) != 0;
			if (size != 1 && size != 2 && size != 4 && size != 8) io_fail("unsupported integer size");
			p += 4;
			break;
		case 1:
			if (b0 & 1) io_fail("big-endian floats are not supported");
			if (size != 4 && size != 8) io_fail("unsupported float size");
			t->cls = Type::kFloat;
			p += 12;
			break;
		case 3:
			t->cls = Type::kString;
			break;
		case 6: {
			t->cls = Type::kCompound;
			const unsigned nm = b0 | (b1 << 8);
			for (unsigned i = 0; i < nm; i++) {
				Member m;
				const uint64_t s = p;
				while (true) {
					need(p, 1);
					if (!d[p]) break;
					m.name.push_back((char)d[p++]);
				}
				if (version < 3) {
					p = s + round8(m.name.size() + 1);
					m.offset = (uint32_t)uint(p, 4);
					p += 4;
					if (version == 1) {
						if (uint(p, 1) != 0) io_fail("compound members with array dimensions are not supported");
						p += 28;
					}
				} else {
					p++;
					int nb = 1;
					while (nb < 4 && (uint64_t(1) << (8 * nb)) <= size) nb++;
					m.offset = (uint32_t)uint(p, nb);
					p += nb;
				}
				m.type = decode_type(p, depth + 1);
				if ((uint64_t)m.offset + m.type->size > size) io_fail("datafile corrupt: compound member outside");
				t->members.push_back(std::move(m));
			}
			break;
		}
		case 10: {
			t->cls = Type::kArray;
			const int nd = (int)uint(p, 1);
			p += version < 3 ? 4 : 1;
			for (int i = 0; i < nd; i++) t->dims.push_back((uint32_t)uint(p + 4 * i, 4));
			p += 4 * nd;
			if (version < 3) p += 4 * nd;  // permutation indices
			t->base = decode_type(p, depth + 1);
			uint64_t cnt = 1;
			for (uint32_t x : t->dims) {
				cnt *= x;
				if (cnt > 0xffffffffull) io_fail("datafile corrupt: array datatype too large");
			}
			if (t->base->size == 0 || cnt * t->base->size != size) io_fail("datafile corrupt: array datatype size");
			break;
		}
		default:
			io_fail("datatype class " + std::to_string(cls) + " is not supported");
		}
		return t;
	}

	// dataspace at absolute p: dims (empty for scalar); false for a null space
	bool decode_space(uint64_t p, std::vector<uint64_t>& dims) const {
		const int version = (int)uint(p, 1);
		const int rank = (int)uint(p + 1, 1);
		dims.clear();
		uint64_t q;
		if (version == 1) {
			q = p + 8;
		} else if (version == 2) {
			if (uint(p + 3, 1) == 2) return false;
			q = p + 4;
		} else {
			io_fail("dataspace version " + std::to_string(version) + " is not supported");
		}
		for (int i = 0; i < rank; i++) dims.push_back(uint(q + 8 * i, 8));
		return true;
	}

	struct Data {
		TypeP type;
		std::vector<uint64_t> dims;
		uint64_t at = 0;  // absolute; raw data of every element
		bool present = false;
	};

	// Deflate (filter 1) is the one filter read; the pipeline's filter ids in order.
	std::vector<unsigned> filters(const std::vector<RawMsg>& m) const {
		std::vector<unsigned> ids;
		const RawMsg* f = find(m, kMsgFilters);
		if (!f) return ids;
		const int v = (int)uint(f->at, 1), nf = (int)uint(f->at + 1, 1);
		uint64_t p = f->at + (v == 1 ? 8 : 2);
		for (int i = 0; i < nf; i++) {
			const unsigned id = (unsigned)uint(p, 2);
			uint64_t name_len = 0;
			p += 2;
			if (v == 1 || id >= 256) {
				name_len = uint(p, 2);
				p += 2;
			}
			const uint64_t nvals = uint(p + 2, 2);
			p += 4;
			p += v == 1 ? round8(name_len) : name_len;
			p += 4 * nvals + (v == 1 && (nvals & 1) ? 4 : 0);
			ids.push_back(id);
		}
		return ids;
	}

	// Chunks of a version 1 B-tree (type 1): offsets (rank + 1 values, the
	// last the element's byte offset), stored size, filter mask, address.
	struct Chunk {
		std::vector<uint64_t> off;
		uint64_t size, mask, addr;
	};
	void chunk_tree(uint64_t rel, int nd, std::vector<Chunk>& out, int depth) const {
		if (depth > 64) io_fail("datafile corrupt: chunk B-tree too deep");
		const uint64_t at = abs(rel);
		expect(at, "TREE");
		if (uint(at + 4, 1) != 1) io_fail("datafile corrupt: not a chunk B-tree");
		const int level = (int)uint(at + 5, 1);
		const uint64_t n = uint(at + 6, 2);
		const uint64_t ks = 8 + 8 * (uint64_t)nd;
		for (uint64_t i = 0; i < n; i++) {
			const uint64_t key = at + 24 + i * (ks + 8);
			const uint64_t child = uint(key + ks, 8);
			if (level > 0) {
				chunk_tree(child, nd, out, depth + 1);
				continue;
			}
			Chunk c;
			c.size = uint(key, 4);
			c.mask = uint(key + 4, 4);
			for (int j = 0; j < nd; j++) c.off.push_back(uint(key + 8 + 8 * j, 8));
			c.addr = child;
			out.push_back(c);
			if (out.size() > (uint64_t)1 << 32) io_fail("datafile corrupt: too many chunks");
		}
	}

	// Number of elements of a dataspace, refusing products that overflow or
	// exceed what one read can hold (2^40 bytes at the given element size).
	static uint64_t element_count(const std::vector<uint64_t>& dims, uint64_t es) {
		uint64_t n = 1;
		for (uint64_t x : dims) {
			if (x != 0 && n > ((uint64_t)1 << 40) / x) io_fail("dataset too large to read");
			n *= x;
		}
		if (es != 0 && n > ((uint64_t)1 << 40) / es) io_fail("dataset too large to read");
		return n;
	}

	// The elements of a chunked dataset, decompressed and placed row-major
	// into one buffer (unwritten chunks read as zero, the default fill).
	std::vector<uint8_t> gather_chunks(const std::vector<RawMsg>& m, uint64_t tree, const std::vector<uint32_t>& cdims,
			const std::vector<uint64_t>& dims, uint64_t es) const {
		const size_t rank = dims.size();
		if (cdims.size() != rank + 1) io_fail("chunk dimensions do not match the dataspace");
		const uint64_t n = element_count(dims, es);
		uint64_t cn = 1;
		for (size_t i = 0; i < rank; i++) {
			cn *= cdims[i];
			if (cn * es > ((uint64_t)1 << 32)) io_fail("chunk too large");
		}
		std::vector<uint8_t> out(n * es, 0);
		if (tree == kUndef || n == 0) return out;
		const std::vector<unsigned> ids = filters(m);
		for (unsigned id : ids)
			if (id != 1) io_fail("filter " + std::to_string(id) + " is not supported (deflate only)");
		std::vector<Chunk> chunks;
		chunk_tree(tree, (int)rank + 1, chunks, 0);
		std::vector<uint8_t> raw(cn * es);
		for (const Chunk& c : chunks) {
			const uint64_t at = abs(c.addr);
			need(at, c.size);
			const bool deflated = !ids.empty() && !(c.mask & 1);
			if (deflated) {
				uLongf len = (uLongf)raw.size();
				if (uncompress(raw.data(), &len, &d[at], (uLong)c.size) != Z_OK || len != raw.size())
					io_fail("datafile corrupt: a chunk does not inflate to its size");
			} else {
				if (c.size != raw.size()) io_fail("datafile corrupt: chunk of the wrong size");
				std::memcpy(raw.data(), &d[at], raw.size());
			}
			// copy the chunk's part inside the dataset, element by element
			std::vector<uint64_t> idx(rank, 0);
			for (uint64_t e = 0; e < cn; e++) {
				uint64_t lin = 0;
				bool inside = true;
				for (size_t i = 0; i < rank; i++) {
					const uint64_t g = c.off[i] + idx[i];
					if (g >= dims[i]) inside = false;
					lin = lin * dims[i] + g;
				}
				if (inside) std::memcpy(&out[lin * es], &raw[e * es], es);
				for (size_t i = rank; i-- > 0;) {
					if (++idx[i] < cdims[i]) break;
					idx[i] = 0;
				}
			}
		}
		return out;
	}

	Data dataset(const char* name) {
		const auto m = messages(lookup(name));
		const RawMsg *t = find(m, kMsgType), *s = find(m, kMsgSpace), *l = find(m, kMsgLayout);
		if (!t || !s || !l) bad_arg(std::string("'") + (name ? name : "/") + "' is not a dataset");
		Data out;
		uint64_t p = t->at;
		out.type = decode_type(p);
		const bool nonnull = decode_space(s->at, out.dims);
		uint64_t n = element_count(out.dims, out.type->size);
		if (!nonnull) n = 0;
		const int lv = (int)uint(l->at, 1);
		int cls;
		uint64_t addr = kUndef;
		uint64_t tree = kUndef;
		std::vector<uint32_t> cdims;
		if (lv == 3) {
			cls = (int)uint(l->at + 1, 1);
			if (cls == 1) addr = uint(l->at + 2, 8);
			if (cls == 0) addr = l->at + 4 - base;  // compact: data inside the message
			if (cls == 2) {
				const int nd = (int)uint(l->at + 2, 1);
				tree = uint(l->at + 3, 8);
				for (int i = 0; i < nd; i++) cdims.push_back((uint32_t)uint(l->at + 11 + 4 * i, 4));
			}
		} else if (lv == 1 || lv == 2) {
			const int nd = (int)uint(l->at + 1, 1);
			cls = (int)uint(l->at + 2, 1);
			if (cls == 1) addr = uint(l->at + 8, 8);
			if (cls == 0) addr = l->at + 8 + 4 * nd + 4 - base;
			if (cls == 2) {
				tree = uint(l->at + 8, 8);
				for (int i = 0; i < nd; i++) cdims.push_back((uint32_t)uint(l->at + 16 + 4 * i, 4));
			}
		} else {
			io_fail("layout message version " + std::to_string(lv) + " is not supported");
		}
		if (cls == 2) {
			if (!cdims.empty() && cdims.back() != out.type->size) io_fail("chunk element size differs from the type");
			for (size_t i = 0; i + 1 < cdims.size(); i++)
				if (cdims[i] == 0) io_fail("datafile corrupt: zero chunk dimension");
			std::vector<uint8_t> all = gather_chunks(m, tree, cdims, out.dims, out.type->size);
			// the gathered elements are read like contiguous storage placed after the file
			out.at = d.size();
			d.insert(d.end(), all.begin(), all.end());
			out.present = n > 0;
			return out;
		}
		if (n > 0) {
			if (addr == kUndef) io_fail("dataset has no storage");
			out.at = abs(addr);
			need(out.at, n * out.type->size);
			out.present = true;
		}
		return out;
	}

	// scalar attribute body of an object (absolute position of the data and its type)
	std::pair<TypeP, uint64_t> attribute(const char* object, const char* name) const {
		if (!name) bad_arg("attribute name is NULL");
		const auto m = messages(lookup(object));
		for (const RawMsg& x : m) {
			if (x.type != kMsgAttr) continue;
			const int v = (int)uint(x.at, 1);
			const uint64_t nlen = uint(x.at + 2, 2), tlen = uint(x.at + 4, 2), slen = uint(x.at + 6, 2);
			uint64_t p = x.at + (v == 3 ? 9 : 8);
			need(p, nlen);
			const std::string an(reinterpret_cast<const char*>(&d[p]), nlen ? nlen - 1 : 0);
			const bool padded = v == 1;
			p += padded ? round8(nlen) : nlen;
			uint64_t tp = p;
			TypeP t = decode_type(tp);
			p += padded ? round8(tlen) : tlen;
			std::vector<uint64_t> dims;
			if (!decode_space(p, dims)) continue;
			p += padded ? round8(slen) : slen;
			if (an != name) continue;
			uint64_t n = 1;
			for (uint64_t x2 : dims) n *= x2;
			if (n != 1) bad_arg(std::string("attribute '") + name + "' is not a scalar");
			need(p, t->size);
			return {t, p};
		}
		bad_arg(std::string("no attribute '") + name + "'");
	}

	// every numeric leaf of the element at p, in order
	void values(const Type& t, uint64_t p, std::vector<double>& out) const {
		switch (t.cls) {
		case Type::kInt: {
			const uint64_t u = uint(p, (int)t.size);
			if (t.is_signed) {
				const int sh = 64 - 8 * (int)t.size;
				out.push_back((double)((int64_t)(u << sh) >> sh));
			} else {
				out.push_back((double)u);
			}
			break;
		}
		case Type::kFloat:
			need(p, t.size);
			if (t.size == 8) {
				double v;
				std::memcpy(&v, &d[p], 8);
				out.push_back(v);
			} else {
				float v;
				std::memcpy(&v, &d[p], 4);
				out.push_back(v);
			}
			break;
		case Type::kCompound:
			for (const Member& m : t.members) values(*m.type, p + m.offset, out);
			break;
		case Type::kArray: {
			uint64_t n = 1;
			for (uint32_t x : t.dims) n *= x;
			for (uint64_t i = 0; i < n; i++) values(*t.base, p + i * t.base->size, out);
			break;
		}
		case Type::kString:
			bad_arg("string values are not numeric");
		}
	}
};

uint64_t count_values(const Type& t) {
	switch (t.cls) {
	case Type::kCompound: {
		uint64_t n = 0;
		for (const Member& m : t.members) n += count_values(*m.type);
		return n;
	}
	case Type::kArray: {
		uint64_t n = count_values(*t.base);
		for (uint32_t x : t.dims) n *= x;
		return n;
	}
	case Type::kString:
		return 0;
	default:
		return 1;
	}
}

itp2d_datafile* checked(itp2d_datafile* f) {
	if (!f) bad_arg("datafile is NULL");
	return f;
}

void check_name(const char* name) {
	if (!name || !*name) bad_arg("attribute name is empty");
}

template <typename T>
void put(std::vector<uint8_t>& data, uint64_t at, T v) {
	std::memcpy(data.data() + at, &v, sizeof(T));
}

void write_history_row(itp2d_datafile* f, const char* name, const double* v, int n, int index) {
	// an empty row (n = 0) only extends the dataset: the device loop keeps no
	// energies for the iterations between its last two
	if ((!v && n > 0) || n < 0 || index < 0) bad_arg("bad history row");
	Dataset& d = f->ensure(name);
	grow(d, {(uint64_t)index + 1, (uint64_t)n});
	if (n) std::memcpy(d.data.data() + (uint64_t)index * d.dims[1] * 8, v, (size_t)n * 8);
}

void write_vector(itp2d_datafile* f, const char* name, const double* v, int n) {
	if ((!v && n > 0) || n < 0) bad_arg("bad vector");
	Dataset& d = f->ensure(name);
	grow(d, {(uint64_t)n});
	if (n) std::memcpy(d.data.data(), v, (size_t)n * 8);
}

void append_pair(itp2d_datafile* f, const char* name, int step, const void* second, size_t second_at,
		size_t second_bytes) {
	Dataset& d = f->ensure(name);
	const uint64_t i = d.dims[0];
	grow(d, {i + 1});
	const uint64_t at = i * d.type->size;
	put<int32_t>(d.data, at, step);
	std::memcpy(d.data.data() + at + second_at, second, second_bytes);
}

}  // namespace

extern "C" {

const char* itp2d_datafile_last_error(void) { return g_error.c_str(); }

int itp2d_datafile_create(const char* filename, int sizex, int sizey, double dx, int clobber,
		itp2d_datafile** out) {
	return guarded([&] {
		if (!filename || !out || sizex < 1 || sizey < 1 || !(dx > 0)) bad_arg("bad datafile arguments");
		*out = nullptr;
		// H5F_ACC_EXCL without clobber, H5F_ACC_TRUNC with it
		const int fd = ::open(filename, O_WRONLY | O_CREAT | (clobber ? O_TRUNC : O_EXCL), 0644);
		if (fd < 0)
			io_fail(std::string("cannot create datafile '") + filename + "': " + std::strerror(errno) +
					(clobber ? "" : " (an existing file is only overwritten with clobber)"));
		::close(fd);
		std::unique_ptr<itp2d_datafile> f(new itp2d_datafile);
		f->path = filename;
		f->sx = sizex;
		f->sy = sizey;
		f->dx = dx;
		f->add_root_attr(string_attr("description",
				"A datafile of an itp2d imaginary-time propagation run. Values are in Hartree atomic units "
				"(the magnetic field in the SI-based atomic unit), program timings in seconds; every dataset "
				"carries a description of its own."));
		f->add_root_attr(value_attr<int32_t>("grid_sizex", int_type(4, true), sizex));
		f->add_root_attr(value_attr<int32_t>("grid_sizey", int_type(4, true), sizey));
		f->add_root_attr(value_attr<double>("grid_delta", double_type(), dx));
		f->write();
		*out = f.release();
	});
}

int itp2d_datafile_flush(itp2d_datafile* f) { return guarded([&] { checked(f)->write(); }); }

int itp2d_datafile_set_chunking(itp2d_datafile* f, int deflate_level) {
	return guarded([&] {
		if (deflate_level > 9) bad_arg("deflate level above 9");
		checked(f)->deflate = deflate_level < 0 ? -1 : deflate_level;
	});
}

int itp2d_datafile_close(itp2d_datafile* f) {
	if (!f) return ITP2D_OK;
	const int st = itp2d_datafile_flush(f);
	delete f;
	return st;
}

int itp2d_datafile_add_attribute_int(itp2d_datafile* f, const char* name, int value) {
	return guarded([&] {
		check_name(name);
		checked(f)->add_root_attr(value_attr<int32_t>(name, int_type(4, true), value));
	});
}

int itp2d_datafile_add_attribute_double(itp2d_datafile* f, const char* name, double value) {
	return guarded([&] {
		check_name(name);
		checked(f)->add_root_attr(value_attr<double>(name, double_type(), value));
	});
}

int itp2d_datafile_add_attribute_ulong(itp2d_datafile* f, const char* name, unsigned long value) {
	return guarded([&] {
		check_name(name);
		checked(f)->add_root_attr(value_attr<uint64_t>(name, int_type(8, false), value));
	});
}

int itp2d_datafile_add_attribute_string(itp2d_datafile* f, const char* name, const char* value) {
	return guarded([&] {
		check_name(name);
		if (!value) bad_arg("string value is NULL");
		checked(f)->add_root_attr(string_attr(name, value));
	});
}

int itp2d_datafile_write_state(itp2d_datafile* f, long long n, long long m, const double* state) {
	return guarded([&] {
		checked(f);
		if (!state || n < 0 || m < 0) bad_arg("bad state arguments");
		Dataset& d = f->ensure("states");
		grow(d, {(uint64_t)n + 1, (uint64_t)m + 1});
		const uint64_t es = d.type->size;
		std::memcpy(d.data.data() + ((uint64_t)n * d.dims[1] + (uint64_t)m) * es, state, es);
	});
}

int itp2d_datafile_write_stateset(itp2d_datafile* f, const double* states, int num_states, int step,
		const int* sort_order) {
	return guarded([&] {
		checked(f);
		if (!states || num_states < 1) bad_arg("bad state set");
		Dataset& d = f->ensure("states");
		const uint64_t slot = d.dims[0];
		const int32_t pair_index = (int32_t)slot;
		append_pair(f, "state_history", step, &pair_index, 4, 4);
		const uint64_t G = (uint64_t)f->sx * f->sy;
		Dataset& s = f->ensure("states");
		grow(s, {slot + 1, (uint64_t)num_states});
		for (int m = 0; m < num_states; m++) {
			const int src = sort_order ? sort_order[m] : m;
			if (src < 0 || src >= num_states) bad_arg("sort order index out of range");
			std::memcpy(s.data.data() + (slot * s.dims[1] + m) * s.type->size, states + 2 * G * src,
					s.type->size);
		}
	});
}

int itp2d_datafile_write_time_step_history(itp2d_datafile* f, int step, double eps) {
	return guarded([&] { append_pair(checked(f), "time_step_history", step, &eps, 8, 8); });
}

int itp2d_datafile_write_energy_history(itp2d_datafile* f, const double* values, int n, int index) {
	return guarded([&] { write_history_row(checked(f), "energy_history", values, n, index); });
}

int itp2d_datafile_write_deviation_history(itp2d_datafile* f, const double* values, int n, int index) {
	return guarded([&] { write_history_row(checked(f), "deviation_history", values, n, index); });
}

int itp2d_datafile_write_energies(itp2d_datafile* f, const double* values, int n) {
	return guarded([&] { write_vector(checked(f), "final_energies", values, n); });
}

int itp2d_datafile_write_energy_standard_deviations(itp2d_datafile* f, const double* values, int n) {
	return guarded([&] { write_vector(checked(f), "final_energy_standard_deviations", values, n); });
}

int itp2d_datafile_write_potential(itp2d_datafile* f, const double* V) {
	return guarded([&] {
		checked(f);
		if (!V) bad_arg("potential is NULL");
		Dataset& d = f->ensure("potential_values");
		std::memcpy(d.data.data(), V, d.data.size());
	});
}

int itp2d_datafile_write_noise_realization(itp2d_datafile* f, const double* values, int n) {
	return guarded([&] { write_vector(checked(f), "noise_data", values, n); });
}

void itp2d_datafile_save_states(void* user, const double* states, const int* order, int num_states, int sx,
		int sy, int step) {
	itp2d_datafile* f = static_cast<itp2d_datafile*>(user);
	if (!f || sx != f->sx || sy != f->sy) {
		g_error = "save callback: datafile missing or of another grid";
		return;
	}
	if (itp2d_datafile_write_stateset(f, states, num_states, step, order) == ITP2D_OK) itp2d_datafile_flush(f);
}

int itp2d_datafile_init_states(const char* filename, int num_states, int sizex, int sizey, double dx,
		double* states) {
	return guarded([&] {
		if (!states || num_states < 1 || sizex < 1 || sizey < 1) bad_arg("bad arguments");
		Reader r(filename);
		auto num = [&](const char* n) {
			const auto a = r.attribute("/", n);
			std::vector<double> v;
			r.values(*a.first, a.second, v);
			if (v.size() != 1) bad_arg(std::string("attribute '") + n + "' is not a number");
			return v[0];
		};
		const char* msg = "Cannot copy state data from datafile: value for ";
		if ((int)num("num_states") != num_states) bad_arg(std::string(msg) + "num_states does not match.");
		if ((int)num("grid_sizex") != sizex) bad_arg(std::string(msg) + "grid_sizex does not match.");
		if ((int)num("grid_sizey") != sizey) bad_arg(std::string(msg) + "grid_sizey does not match.");
		if (num("grid_delta") != dx) bad_arg(std::string(msg) + "grid_delta does not match.");
		const auto ds = r.dataset("states");
		const uint64_t es = (uint64_t)sizex * sizey * 16;
		if (ds.dims.size() != 2 || ds.type->size != es || count_values(*ds.type) != es / 8)
			bad_arg("states dataset has another shape or element type");
		if (ds.dims[1] != (uint64_t)num_states || ds.dims[0] == 0)
			bad_arg("states dataset holds no complete state set");
		// the last slot, the latest states
		const uint64_t at = ds.at + (ds.dims[0] - 1) * ds.dims[1] * es;
		std::vector<double> v;
		v.reserve(es / 8 * num_states);
		for (int m = 0; m < num_states; m++) r.values(*ds.type, at + m * es, v);
		std::memcpy(states, v.data(), v.size() * 8);
	});
}

int itp2d_datafile_dataset_shape(const char* filename, const char* dataset, int* rank, long long* dims,
		long long* values_per_element) {
	return guarded([&] {
		Reader r(filename);
		const auto ds = r.dataset(dataset);
		if (ds.dims.size() > 8) io_fail("rank above 8");
		if (rank) *rank = (int)ds.dims.size();
		if (dims)
			for (size_t i = 0; i < ds.dims.size(); i++) dims[i] = (long long)ds.dims[i];
		if (values_per_element) *values_per_element = (long long)count_values(*ds.type);
	});
}

int itp2d_datafile_read_values(const char* filename, const char* dataset, double* out, long long max_values,
		long long* n_values) {
	return guarded([&] {
		Reader r(filename);
		const auto ds = r.dataset(dataset);
		uint64_t n = 1;
		for (uint64_t x : ds.dims) n *= x;
		std::vector<double> v;
		if (ds.present)
			for (uint64_t i = 0; i < n; i++) r.values(*ds.type, ds.at + i * ds.type->size, v);
		if (n_values) *n_values = (long long)v.size();
		const uint64_t nv = std::min<uint64_t>(v.size(), (uint64_t)std::max(0ll, max_values));
		if (out && nv) std::memcpy(out, v.data(), nv * 8);
	});
}

int itp2d_datafile_read_attribute(const char* filename, const char* object, const char* name, double* value) {
	return guarded([&] {
		if (!value) bad_arg("value is NULL");
		Reader r(filename);
		const auto a = r.attribute(object, name);
		std::vector<double> v;
		r.values(*a.first, a.second, v);
		if (v.size() != 1) bad_arg(std::string("attribute '") + name + "' is not a single number");
		*value = v[0];
	});
}

int itp2d_datafile_read_string_attribute(const char* filename, const char* object, const char* name, char* buf,
		int buflen) {
	return guarded([&] {
		if (!buf || buflen < 1) bad_arg("no buffer");
		Reader r(filename);
		const auto a = r.attribute(object, name);
		if (a.first->cls != Type::kString) bad_arg(std::string("attribute '") + name + "' is not a string");
		std::string s(reinterpret_cast<const char*>(&r.d[a.second]), a.first->size);
		s = s.substr(0, s.find('\0'));
		const size_t n = std::min<size_t>(s.size(), (size_t)buflen - 1);
		std::memcpy(buf, s.data(), n);
		buf[n] = 0;
	});
}

int itp2d_datafile_header_message(const char* filename, const char* object, int type, int index,
		unsigned char* buf, int buflen, int* size) {
	return guarded([&] {
		Reader r(filename);
		int seen = 0;
		for (const auto& m : r.messages(r.lookup(object))) {
			if (m.type != type || seen++ != index) continue;
			if (size) *size = (int)m.size;
			if (buf && buflen > 0) std::memcpy(buf, &r.d[m.at], std::min<uint64_t>(m.size, (uint64_t)buflen));
			return;
		}
		bad_arg("no such header message");
	});
}

}  // extern "C"
