// Gaussian impurity potentials built on the device (V and the impurity list in
// device memory; host pointers are rejected before any launch).
//
// V(x, y) += sum_j A_j exp(-r_j^2 / (2 w_j^2)), r_j the distance of the grid
// point from impurity j: GaussianImpurities::add_noise (noise.cpp:24-40)
// applied to a whole impurity list, in list order at every grid point as the
// reference's loop over impurities does. Grid positions are cell-centred,
// x_i = (2i + 1 - sx) dx / 2 (DataLayout, datalayout.cpp:21-35); V is stored
// [y][x] like the potential arrays of the path. The products and sums are
// rounded one at a time (no fused multiply-add), so the result differs from
// the reference's host loop only through exp().
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/itp2d_gpu.h"

namespace {

constexpr int kThreads = 256;  // also the impurities staged in shared memory per pass

__global__ void __launch_bounds__(kThreads) gaussian_impurities_kernel(int sx, int sy, double dx, int n,
		const double* __restrict__ imp, double* __restrict__ V) {
	__shared__ double4 st[kThreads];  // (x, y, A, w)
	const long long G = (long long)sx * sy;
	const long long idx = (long long)blockIdx.x * kThreads + threadIdx.x;
	const bool in = idx < G;
	const int x = in ? (int)(idx % sx) : 0, y = in ? (int)(idx / sx) : 0;
	const double px = (2.0 * x + 1.0 - sx) * 0.5 * dx;
	const double py = (2.0 * y + 1.0 - sy) * 0.5 * dx;
	double v = in ? V[idx] : 0.0;
	for (int c0 = 0; c0 < n; c0 += kThreads) {
		const int m = min(kThreads, n - c0);
		__syncthreads();  // the previous chunk has been read
		if ((int)threadIdx.x < m) {
			const double* p = imp + 4LL * (c0 + threadIdx.x);
			st[threadIdx.x] = make_double4(p[0], p[1], p[2], p[3]);
		}
		__syncthreads();
		for (int j = 0; j < m; j++) {
			const double4 p = st[j];
			const double rx = __dsub_rn(p.x, px), ry = __dsub_rn(p.y, py);
			const double r2 = __dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry));
			const double w2 = __dmul_rn(p.w, p.w);
			v = __dadd_rn(v, __dmul_rn(p.z, exp(__dmul_rn(-0.5, __ddiv_rn(r2, w2)))));
		}
	}
	if (in) V[idx] = v;
}

// True when p is device (or managed) memory the kernel can dereference.
bool device_pointer(const void* p) {
	cudaPointerAttributes a;
	if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
		cudaGetLastError();  // clear the error an unknown pointer leaves behind
		return false;
	}
	return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" int itp2d_add_gaussian_impurities(int sx, int sy, double dx, int n, const double* impurities, double* V,
		void* cuda_stream) {
	if (sx < 1 || sy < 1 || !(dx > 0.0) || n < 0 || !V || (n > 0 && !impurities)) return ITP2D_E_INVALID;
	if (n == 0) return ITP2D_OK;
	if (!device_pointer(V) || !device_pointer(impurities)) return ITP2D_E_INVALID;
	const long long G = (long long)sx * sy;
	const unsigned blocks = (unsigned)((G + kThreads - 1) / kThreads);
	gaussian_impurities_kernel<<<blocks, kThreads, 0, (cudaStream_t)cuda_stream>>>(sx, sy, dx, n, impurities, V);
	return cudaGetLastError() == cudaSuccess ? ITP2D_OK : ITP2D_E_CUDA;
}

// ---- The potential-type library (potentialtypes.hpp:96-380) on the device ----
//
// itp2d_evaluate_potential writes V(x, y) of a potential description in the
// reference's mini-language ("harmonic(1)", "ring(3,1,2)", ...) at the
// cell-centred grid points. The description is parsed on the host with the
// reference's names, parameter counts, defaults and checks
// (potentialtypes.cpp:56-500); every formula is evaluated in the reference's
// operation order with each product, quotient and sum rounded on its own (no
// fused multiply-add), so a value differs from the reference's host loop only
// through the library functions (exp, pow, sin, cos, atan2, cosh, hypot).

namespace {

enum PotKind {
	kZero, kHarmonic, kElliptic, kPrettyHardSquare, kSoftPentagon, kHenonHeiles, kGaussian, kQuartic,
	kSquareOscillator, kPower, kRing, kCosh, kSoftStadium, kPowerStadium
};

struct PotSpec {
	int kind;
	double p[6];
};

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }

// The stadium coordinate q of softstadium / powerstadium (potentialtypes.hpp:330-376).
__device__ double stadium_q(double x, double y, double R, double halfL, bool absolute) {
	if (fabs(x) <= halfL) return absolute ? fabs(dvd(y, R)) : dvd(y, R);
	if (x < -halfL) return dvd(hypot(add(x, halfL), y), R);
	return dvd(hypot(sub(x, halfL), y), R);
}

__device__ double eval_potential(const PotSpec& s, double x, double y) {
	const double* p = s.p;
	switch (s.kind) {
		case kHarmonic: {
			const double px = sub(x, p[1]), py = sub(y, p[2]);
			return mul(mul(0.5, p[0]), add(mul(px, px), mul(py, py)));
		}
		case kElliptic:
			return mul(0.5, add(mul(mul(p[0], x), x), mul(mul(p[1], y), y)));
		case kPrettyHardSquare: {
			const double ax = fabs(dvd(mul(2.0, x), M_PI)), ay = fabs(dvd(mul(2.0, y), M_PI));
			return pow(ax > ay ? ax : ay, p[0]);
		}
		case kSoftPentagon: {
			const double r2 = add(mul(x, x), mul(y, y));
			const double t = atan2(y, x);
			return mul(mul(0.5, r2), add(1.0, mul(0.5, sin(mul(5.0, t)))));
		}
		case kHenonHeiles: {
			const double r2 = add(mul(x, x), mul(y, y));
			const double r3 = pow(r2, 3.0 / 2.0);
			const double r4 = mul(r2, r2);
			const double t = atan2(y, x);
			return add(add(r4, mul(p[0], r2)), mul(mul(p[1], r3), cos(mul(3.0, t))));
		}
		case kGaussian: {
			const double xp = sub(x, p[2]), yp = sub(y, p[3]);
			const double e = dvd(-add(mul(xp, xp), mul(yp, yp)), mul(mul(2.0, p[1]), p[1]));
			return mul(p[0], exp(e));
		}
		case kQuartic: {
			const double s2 = sqrt(2.0);
			const double qx = dvd(sub(x, y), s2), qy = dvd(add(x, y), s2);
			const double x2 = mul(qx, qx), y2 = mul(qy, qy);
			const double x4 = mul(x2, x2), y4 = mul(y2, y2);
			return add(dvd(mul(x2, y2), 2.0), dvd(mul(p[0], add(x4, y4)), 4.0));
		}
		case kSquareOscillator:
			return mul(0.5, add(pow(fabs(x), p[0]), pow(fabs(y), p[0])));
		case kPower:
			return mul(mul(0.5, p[1]), pow(hypot(x, y), p[0]));
		case kRing: {
			const double z = dvd(fabs(sub(hypot(x, y), p[0])), p[1]);
			const double xp = sub(x, p[0]);
			const double ge = dvd(-add(mul(xp, xp), mul(y, y)), mul(mul(2.0, p[4]), p[4]));
			return add(mul(0.5, pow(z, p[2])), mul(p[3], exp(ge)));
		}
		case kCosh:
			return mul(p[0], sub(cosh(dvd(hypot(x, y), p[1])), 1.0));
		case kSoftStadium: {
			const double q = stadium_q(x, y, p[0], p[1], false);
			return dvd(p[2], add(1.0, mul(p[3], exp(mul(p[4], sub(1.0, mul(q, q)))))));
		}
		case kPowerStadium:
			return mul(0.5, pow(stadium_q(x, y, p[0], p[1], true), p[2]));
		default:
			return 0.0;
	}
}

__global__ void potential_kernel(int sx, int sy, double dx, PotSpec s, double* __restrict__ V) {
	const long long G = (long long)sx * sy;
	for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < G;
			idx += (long long)gridDim.x * blockDim.x) {
		const int x = (int)(idx % sx), y = (int)(idx / sx);
		const double px = (2.0 * x + 1.0 - sx) * 0.5 * dx;
		const double py = (2.0 * y + 1.0 - sy) * 0.5 * dx;
		V[idx] = eval_potential(s, px, py);
	}
}

// name(v1,v2,...) (parser.cpp:26-60): false when the string is malformed.
bool parse_description(const char* str, std::string& name, std::vector<double>& params) {
	std::string s(str);
	s.erase(std::remove_if(s.begin(), s.end(), [](char c) { return std::isspace((unsigned char)c); }), s.end());
	const size_t open = s.find('(');
	if (open == std::string::npos) {
		name = s;
		return !name.empty();
	}
	if (s.back() != ')') return false;
	name = s.substr(0, open);
	const std::string inner = s.substr(open + 1, s.size() - open - 2);
	size_t pos = 0;
	while (pos < inner.size()) {
		const size_t comma = inner.find(',', pos);
		const std::string tok = inner.substr(pos, comma == std::string::npos ? std::string::npos : comma - pos);
		char* end = nullptr;
		const double v = std::strtod(tok.c_str(), &end);
		if (tok.empty() || *end != '\0') return false;
		params.push_back(v);
		if (comma == std::string::npos) break;
		pos = comma + 1;
	}
	return !name.empty();
}

// The reference constructor's parameters, defaults and checks: false for an
// unknown name, a wrong parameter count or a rejected value.
bool make_spec(const std::string& name, const std::vector<double>& a, PotSpec& s) {
	const size_t n = a.size();
	for (double& v : s.p) v = 0.0;
	auto set = [&](std::initializer_list<double> v) {
		int i = 0;
		for (double x : v) s.p[i++] = x;
	};
	if (name == "zero") {
		s.kind = kZero;
		return n == 0;
	}
	if (name == "harmonic") {  // potentialtypes.cpp:120-145
		s.kind = kHarmonic;
		if (n == 0) set({1, 0, 0});
		else if (n == 1) set({a[0], 0, 0});
		else if (n == 3) set({a[0], a[1], a[2]});
		else return false;
		return s.p[0] >= 0;
	}
	if (name == "elliptic") {
		s.kind = kElliptic;
		if (n == 0) set({1, 1.6180339887498948482});
		else if (n == 2) set({a[0], a[1]});
		else return false;
		return s.p[0] >= 0 && s.p[1] >= 0;
	}
	if (name == "prettyhardsquare") {
		s.kind = kPrettyHardSquare;
		if (n == 0) set({8});
		else if (n == 1) set({a[0]});
		else return false;
		return true;
	}
	if (name == "softpentagon") {
		s.kind = kSoftPentagon;
		return n == 0;
	}
	if (name == "henonheiles" || name == "henon") {
		s.kind = kHenonHeiles;
		if (n == 0) set({205.0 / 42.0, -13.0 / 3.0});
		else if (n == 2) set({a[0], a[1]});
		else return false;
		return true;
	}
	if (name == "gaussian" || name == "gaussianblob") {
		s.kind = kGaussian;
		if (n == 0) set({1, 1, 0, 0});
		else if (n == 2) set({a[0], a[1], 0, 0});
		else if (n == 4) set({a[0], a[1], a[2], a[3]});
		else return false;
		return s.p[0] >= 0 && s.p[1] != 0;
	}
	if (name == "quartic" || name == "quarticoscillator") {
		s.kind = kQuartic;
		if (n == 0) set({0.01});
		else if (n == 1) set({a[0]});
		else return false;
		return s.p[0] >= 0;
	}
	if (name == "squareoscillator") {
		s.kind = kSquareOscillator;
		if (n == 0) set({8});
		else if (n == 1) set({a[0]});
		else return false;
		return true;
	}
	if (name == "power" || name == "poweroscillator") {  // (exponent, prefactor)
		s.kind = kPower;
		if (n == 0) set({4, 1});
		else if (n == 1) set({a[0], 1});
		else if (n == 2) set({a[0], a[1]});
		else return false;
		return s.p[1] >= 0;
	}
	if (name == "ring" || name == "ringpotential") {  // (r, w, e, asymm A, asymm w)
		s.kind = kRing;
		if (n == 0) set({3, 1, 2, 0, 1});
		else if (n == 3) set({a[0], a[1], a[2], 0, 1});
		else if (n == 5) set({a[0], a[1], a[2], a[3], a[4]});
		else return false;
		return s.p[0] >= 0 && s.p[1] > 0;
	}
	if (name == "cosh" || name == "coshpotential") {
		s.kind = kCosh;
		if (n == 0) set({1, 1});
		else if (n == 2) set({a[0], a[1]});
		else return false;
		return s.p[0] > 0 && s.p[1] > 0;
	}
	if (name == "softstadium") {  // (R, L, V[, a, b]); halfL = L / 2
		s.kind = kSoftStadium;
		if (n == 0) set({1, 1, 100, 1, 10});
		else if (n == 3) set({a[0], a[1] / 2, a[2], 1, 10});
		else if (n == 5) set({a[0], a[1] / 2, a[2], a[3], a[4]});
		else return false;
		return s.p[0] > 0 && s.p[1] > 0 && s.p[2] > 0 && s.p[3] > 0 && s.p[4] > 0;
	}
	if (name == "powerstadium") {  // (R, L, power) or (power)
		s.kind = kPowerStadium;
		if (n == 0) set({1, 1, 4});
		else if (n == 1) set({1, 1, a[0]});
		else if (n == 3) set({a[0], a[1] / 2, a[2]});
		else return false;
		return s.p[0] > 0 && s.p[1] > 0;
	}
	return false;
}

}  // namespace

extern "C" int itp2d_potential_check(const char* description, int* is_null) {
	if (!description) return ITP2D_E_INVALID;
	std::string name;
	std::vector<double> params;
	PotSpec s;
	if (!parse_description(description, name, params) || !make_spec(name, params, s)) return ITP2D_E_INVALID;
	if (is_null) *is_null = s.kind == kZero ? 1 : 0;
	return ITP2D_OK;
}

extern "C" int itp2d_evaluate_potential(const char* description, int sx, int sy, double dx, double* V,
		void* cuda_stream) {
	if (!description || sx < 1 || sy < 1 || !(dx > 0.0) || !V) return ITP2D_E_INVALID;
	std::string name;
	std::vector<double> params;
	PotSpec s;
	if (!parse_description(description, name, params) || !make_spec(name, params, s)) return ITP2D_E_INVALID;
	if (!device_pointer(V)) return ITP2D_E_INVALID;
	const long long G = (long long)sx * sy;
	const unsigned blocks = (unsigned)std::min<long long>((G + kThreads - 1) / kThreads, 148LL * 16);
	potential_kernel<<<blocks, kThreads, 0, (cudaStream_t)cuda_stream>>>(sx, sy, dx, s, V);
	return cudaGetLastError() == cudaSuccess ? ITP2D_OK : ITP2D_E_CUDA;
}

// ---- The other impurity shapes of noise.cpp:42-87 ----
//
// For a list of n impurities, in list order at every grid point:
//   Coulomb    (rows x, y; params e, alpha):  V += alpha * (r^2)^(-e/2)
//   hemisphere (rows x, y; params A, radius): V += A sqrt(1 - d^2 / radius^2) for d < radius
//   delta      (rows x, y, A):                V += A at the grid point nearest to (x, y)
// (CoulombImpurities, HemisphereImpurities, DeltaImpurities::add_noise).

namespace {

// DataLayout::nearest_index (datalayout.hpp:79-88) with round_to_int
// (itp2d_common.hpp:69-71); -1 when the index falls outside the grid.
__device__ int nearest_index(double x, int s, double d) {
	const double r = __dadd_rn(__ddiv_rn(x, d), (s - 1.0) / 2.0);
	const int i = (int)(r > 0 ? floor(r + 0.5) : ceil(r - 0.5));
	return (i < 0 || i >= s) ? -1 : i;
}

__global__ void __launch_bounds__(kThreads) impurities_kernel(int shape, int sx, int sy, double dx, int n,
		const double* __restrict__ rows, double p0, double p1, double* __restrict__ V) {
	const int width = shape == ITP2D_IMPURITY_DELTA ? 3 : 2;
	const long long G = (long long)sx * sy;
	const long long idx = (long long)blockIdx.x * kThreads + threadIdx.x;
	if (idx >= G) return;
	const int x = (int)(idx % sx), y = (int)(idx / sx);
	const double px = (2.0 * x + 1.0 - sx) * 0.5 * dx;
	const double py = (2.0 * y + 1.0 - sy) * 0.5 * dx;
	double v = V[idx];
	const double r2lim = __dmul_rn(p1, p1);
	for (int j = 0; j < n; j++) {
		const double* r = rows + (long long)width * j;
		if (shape == ITP2D_IMPURITY_DELTA) {
			if (nearest_index(r[0], sx, dx) == x && nearest_index(r[1], sy, dx) == y) v = __dadd_rn(v, r[2]);
			continue;
		}
		const double rx = __dsub_rn(r[0], px), ry = __dsub_rn(r[1], py);
		const double d2 = __dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry));
		if (shape == ITP2D_IMPURITY_COULOMB) {
			v = __dadd_rn(v, __dmul_rn(p1, pow(d2, -(p0 / 2))));
		} else if (d2 < r2lim) {
			v = __dadd_rn(v, __dmul_rn(p0, sqrt(__dsub_rn(1.0, __ddiv_rn(d2, r2lim)))));
		}
	}
	V[idx] = v;
}

}  // namespace

extern "C" int itp2d_add_impurities(int shape, int sx, int sy, double dx, int n, const double* rows,
		double param0, double param1, double* V, void* cuda_stream) {
	if (shape != ITP2D_IMPURITY_COULOMB && shape != ITP2D_IMPURITY_HEMISPHERE && shape != ITP2D_IMPURITY_DELTA)
		return ITP2D_E_INVALID;
	if (sx < 1 || sy < 1 || !(dx > 0.0) || n < 0 || !V || (n > 0 && !rows)) return ITP2D_E_INVALID;
	if (n == 0) return ITP2D_OK;
	if (!device_pointer(V) || !device_pointer(rows)) return ITP2D_E_INVALID;
	const long long G = (long long)sx * sy;
	const unsigned blocks = (unsigned)((G + kThreads - 1) / kThreads);
	impurities_kernel<<<blocks, kThreads, 0, (cudaStream_t)cuda_stream>>>(shape, sx, sy, dx, n, rows, param0, param1,
			V);
	return cudaGetLastError() == cudaSuccess ? ITP2D_OK : ITP2D_E_CUDA;
}

extern "C" int itp2d_evaluate_potential_host(const char* description, int sx, int sy, double dx, double* V) {
	if (!description || sx < 1 || sy < 1 || !(dx > 0.0) || !V) return ITP2D_E_INVALID;
	int is_null = 0;
	int st = itp2d_potential_check(description, &is_null);
	if (st) return st;
	const size_t bytes = (size_t)sx * sy * sizeof(double);
	double* d = nullptr;
	if (cudaMalloc(&d, bytes) != cudaSuccess) return ITP2D_E_OOM;
	st = itp2d_evaluate_potential(description, sx, sy, dx, d, nullptr);
	if (st == ITP2D_OK && cudaMemcpy(V, d, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) st = ITP2D_E_CUDA;
	cudaFree(d);
	return st;
}
