"""CPU restatement (numpy/scipy) of the itp2d hot path. TEST INFRASTRUCTURE ONLY.

This module is the checker that the CUDA product is compared against; it is
imported only by tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py``. The product never imports it.

Parity is pinned two ways (see tests/test_oracle.py): against the itp2d
reference sources compiled unmodified into ``oracle/_ref/libitp2d_ref.so``
(elementwise agreement of every seam on identical inputs), and against the
known-answer vectors of the reference's own unit tests
(test_transformer.cpp:59-149, test_laplacian.cpp:38-58,
test_eigensolver.cpp:25-74, test_stateset.cpp:26-42).

Array convention: a state set is a complex128 array of shape (k, sy, sx),
state n at offset n*G, x fastest -- the reference's StateArray layout
(statearray.cpp:21-75, datalayout.hpp:69-77).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import scipy.fft as sfft

PERIODIC = 0
DIRICHLET = 1

# Transform enum order of transformer.hpp:32-34.
TRANSFORMS = ["FFT", "iFFT", "FFTx", "iFFTx", "FFTy", "iFFTy", "DST", "iDST", "DSTx", "iDSTx",
              "DSTy", "iDSTy", "DCT", "iDCT", "DCTx", "iDCTx", "DCTy", "iDCTy"]


@dataclass
class Grid:
    """Cell-centred grid of datalayout.cpp:21-36: dx = len/sx, x_j = (2j+1-sx)*dx/2."""

    sx: int
    sy: int
    dx: float

    @classmethod
    def from_length(cls, sx: int, sy: int, length: float) -> "Grid":
        # Parameters::get_grid_delta, parameters.hpp:97
        return cls(sx, sy, length / float(sx))

    @property
    def lenx(self) -> float:
        return float(self.sx) * self.dx

    @property
    def leny(self) -> float:
        return float(self.sy) * self.dx

    @property
    def G(self) -> int:
        return self.sx * self.sy

    @property
    def posx(self) -> np.ndarray:
        return np.array([float(2 * x + 1 - self.sx) * 0.5 * self.dx for x in range(self.sx)])

    @property
    def posy(self) -> np.ndarray:
        return np.array([float(2 * y + 1 - self.sy) * 0.5 * self.dx for y in range(self.sy)])


def fft_k(n: int, length: float) -> np.ndarray:
    """FFT wavenumbers, transformer.cpp:83-90."""
    m = math.pi / length
    return np.array([float(j if j < n // 2 else j - n) * 2 * m for j in range(n)])


def dsct_k(n: int, length: float) -> np.ndarray:
    """DST/DCT wavenumbers, transformer.cpp:85,89."""
    m = math.pi / length
    return np.array([float(j + 1) * m for j in range(n)])


def norm_factors(g: Grid) -> dict:
    """Normalisations of transformer.cpp:66-73."""
    return {
        "FFT": 1.0 / float(g.sx * g.sy),
        "FFTx": 1.0 / float(g.sx),
        "FFTy": 1.0 / float(g.sy),
        "DSCT": 1.0 / float(4 * g.sx * g.sy),
        "DSCTx": 1.0 / float(2 * g.sx),
        "DSCTy": 1.0 / float(2 * g.sy),
    }


def _r2r(a: np.ndarray, kind: str, axis: int) -> np.ndarray:
    # scipy's unnormalised type-2/3 DST/DCT equal FFTW's RODFT10/01 and
    # REDFT10/01; applied to Re and Im separately like transformer.cpp:112-151.
    f = {"DST2": (sfft.dst, 2), "DST3": (sfft.dst, 3), "DCT2": (sfft.dct, 2), "DCT3": (sfft.dct, 3)}[kind]
    fn, t = f
    return fn(a.real, type=t, axis=axis) + 1j * fn(a.imag, type=t, axis=axis)


def transform(a: np.ndarray, kind: str) -> np.ndarray:
    """Unnormalised transforms of Transformer::transform (transformer.hpp:132-158)
    on arrays of shape (..., sy, sx). Forward DFT uses exp(-2 pi i jk/n)."""
    X, Y = -1, -2
    if kind == "FFT":
        return np.fft.fft2(a, axes=(Y, X))
    if kind == "iFFT":
        return np.fft.ifft2(a, axes=(Y, X), norm="forward")
    if kind == "FFTx":
        return np.fft.fft(a, axis=X)
    if kind == "iFFTx":
        return np.fft.ifft(a, axis=X, norm="forward")
    if kind == "FFTy":
        return np.fft.fft(a, axis=Y)
    if kind == "iFFTy":
        return np.fft.ifft(a, axis=Y, norm="forward")
    table = {
        "DST": [("DST2", X), ("DST2", Y)], "iDST": [("DST3", X), ("DST3", Y)],
        "DSTx": [("DST2", X)], "iDSTx": [("DST3", X)],
        "DSTy": [("DST2", Y)], "iDSTy": [("DST3", Y)],
        "DCT": [("DCT2", X), ("DCT2", Y)], "iDCT": [("DCT3", X), ("DCT3", Y)],
        "DCTx": [("DCT2", X)], "iDCTx": [("DCT3", X)],
        "DCTy": [("DCT2", Y)], "iDCTy": [("DCT3", Y)],
    }
    out = a
    for k, ax in table[kind]:
        out = _r2r(out, k, ax)
    return out


def multiproduct_coefficients(m: int) -> list:
    """c_t = t^{2(m-1)} / prod_{n != t} (t^2 - n^2), multiproductsplit.cpp:49-59
    (integer denominator as in the reference)."""
    out = []
    for t in range(1, m + 1):
        denom = 1
        for n in range(1, m + 1):
            if n != t:
                denom *= t * t - n * n
        out.append(math.pow(t, 2 * (m - 1)) / denom)
    return out


def shift_x_imag(a: np.ndarray, values: np.ndarray) -> np.ndarray:
    """State::pointwise_multiply_imaginary_shiftx (state.hpp:192-201):
    out(x,y) = a(x-1,y) * i*values(x-1,y) for x >= 1, out(0,y) = 0."""
    out = np.zeros_like(a)
    out[..., 1:] = a[..., :-1] * (1j * values[:, :-1])
    return out


class ExpKinetic:
    """p*exp(-e*c*T) of expkinetic.cpp:65-197 (linear gauge A = (-By, 0, 0))."""

    def __init__(self, g: Grid, bt: int, B: float, eps: float, coeff: float = -1.0, prefactor: float = 1.0):
        self.g, self.bt, self.B, self.coeff, self.prefactor = g, bt, B, coeff, prefactor
        self.set_time_step(eps)

    def set_time_step(self, eps: float) -> None:
        g, bt, B = self.g, self.bt, self.B
        self.eps = eps
        nf = norm_factors(g)
        kx = fft_k(g.sx, g.lenx) if bt == PERIODIC else dsct_k(g.sx, g.lenx)
        ky = fft_k(g.sy, g.leny) if bt == PERIODIC else dsct_k(g.sy, g.leny)
        posy = g.posy
        if B == 0:
            normfac = nf["FFT"] if bt == PERIODIC else nf["DSCT"]
            A = self.coeff * eps * 0.5
            p = self.prefactor * normfac
            self.mult = np.array([[p * math.exp(A * (kx[x] * kx[x] + ky[y] * ky[y])) for x in range(g.sx)]
                                  for y in range(g.sy)])
            return
        normfacx = math.sqrt(nf["FFTx"]) if bt == PERIODIC else nf["DSCTx"]
        normfacy = nf["FFTy"] if bt == PERIODIC else nf["DSCTy"]
        z = B * eps
        if abs(z) < 1e-6:
            Cy = 1 + math.pow(z, 2) / 6 + math.pow(z, 4) / 120
            Cx = 0.5 - math.pow(z, 2) / 24 + math.pow(z, 4) / 240
        else:
            Cy = math.sinh(z) / z
            Cx = math.tanh(z / 2) / z
        Ax = self.coeff * eps * 0.5 * Cx
        Ay = self.coeff * eps * 0.5 * Cy
        px = normfacx
        py = self.prefactor * normfacy
        self.ymult = np.array([py * math.exp(Ay * ky[y] * ky[y]) for y in range(g.sy)])
        if bt == PERIODIC:
            self.xmult = np.array([[px * math.exp(Ax * (kx[x] - B * posy[y]) * (kx[x] - B * posy[y]))
                                    for x in range(g.sx)] for y in range(g.sy)])
        else:
            xm = np.empty((g.sy, g.sx))
            xm2 = np.empty((g.sy, g.sx))
            for y in range(g.sy):
                By = B * posy[y]
                for x in range(g.sx):
                    common = px * math.exp(Ax * (kx[x] * kx[x] + By * By))
                    arg = 2 * Ax * kx[x] * By
                    xm[y, x] = common * math.cosh(arg)
                    xm2[y, x] = common * math.sinh(arg)
            self.xmult, self.xmult2 = xm, xm2

    def apply(self, a: np.ndarray) -> np.ndarray:
        """ExpKinetic::operate, expkinetic.cpp:138-197."""
        if self.B == 0:
            f, fi = ("FFT", "iFFT") if self.bt == PERIODIC else ("DST", "iDST")
            return transform(transform(a, f) * self.mult, fi)
        if self.bt == PERIODIC:
            s = transform(a, "FFTx") * self.xmult
            s = transform(s, "FFTy") * self.ymult[:, None]
            s = transform(s, "iFFTy") * self.xmult
            return transform(s, "iFFTx")
        s = transform(a, "DSTx")
        temp = shift_x_imag(s, self.xmult2)
        s = transform(s * self.xmult, "iDSTx") + transform(temp, "iDCTx")
        s = transform(s, "DST") * self.ymult[:, None]
        s = transform(s, "iDSTy")
        temp = shift_x_imag(s, self.xmult2)
        return transform(s * self.xmult, "iDSTx") + transform(temp, "iDCTx")


def exp_potential(V: np.ndarray, eps: float, coeff: float, prefactor: float) -> np.ndarray:
    """ExpPotential table prefactor*exp(eps*coeff*V), exppotential.cpp:55-63."""
    return prefactor * np.exp(eps * coeff * V)


class MultiProductSplit:
    """T_{2m}(eps) = sum_t c_t [T_2(eps/t)]^t (multiproductsplit.cpp:23-59) with the
    members of secondordersplit.cpp:21-49 applied right-to-left
    (operatorproduct.cpp:48-52) and summed like OperatorSum::operate
    (operatorsum.cpp:61-86)."""

    def __init__(self, g: Grid, V, bt: int, B: float, halforder: int, eps: float):
        self.g, self.V, self.bt, self.B = g, V, bt, B
        self.null = V is None
        self.m = 1 if self.null else halforder
        self.coeffs = multiproduct_coefficients(self.m)
        self.set_time_step(eps)

    def set_time_step(self, eps: float) -> None:
        self.eps = eps
        self.members = []
        for t in range(1, self.m + 1):
            et = eps / t
            c = self.coeffs[t - 1]
            if self.null:
                K = ExpKinetic(self.g, self.bt, self.B, et, -1.0 * t, c)
                self.members.append((t, K, None, None, None))
            else:
                K = ExpKinetic(self.g, self.bt, self.B, et, -1.0)
                vh = exp_potential(self.V, et, -0.5, 1.0)
                vp = exp_potential(self.V, et, -0.5, c) if c != 1.0 else vh
                vsq = exp_potential(self.V, et, -1.0, 1.0) if t >= 2 else None
                self.members.append((t, K, vh, vp, vsq))

    def _member(self, t, K, vh, vp, vsq, a):
        if vh is None:
            return K.apply(a)
        s = a * vh
        s = K.apply(s)
        for _ in range(2, t + 1):
            s = K.apply(s * vsq)
        return s * vp

    def apply(self, a: np.ndarray) -> np.ndarray:
        if len(self.members) == 1:
            return self._member(*self.members[0], a)
        out = self._member(*self.members[0], a)
        for mem in self.members[1:]:
            out = out + self._member(*mem, a)
        return out


class Kinetic:
    """T of kinetic.cpp:25-142 (linear gauge)."""

    def __init__(self, g: Grid, bt: int, B: float):
        self.g, self.bt, self.B = g, bt, B
        nf = norm_factors(g)
        kx = fft_k(g.sx, g.lenx) if bt == PERIODIC else dsct_k(g.sx, g.lenx)
        ky = fft_k(g.sy, g.leny) if bt == PERIODIC else dsct_k(g.sy, g.leny)
        posy = g.posy
        nfac = nf["FFT"] if bt == PERIODIC else nf["DSCT"]
        nfx = nf["FFTx"] if bt == PERIODIC else nf["DSCTx"]
        nfy = nf["FFTy"] if bt == PERIODIC else nf["DSCTy"]
        if B == 0:
            self.mxy = np.array([[0.5 * (kx[x] * kx[x] + ky[y] * ky[y]) * nfac for x in range(g.sx)]
                                 for y in range(g.sy)])
            return
        self.my = np.array([0.5 * ky[y] * ky[y] * nfy for y in range(g.sy)])
        if bt == PERIODIC:
            self.mx = np.array([[0.5 * (kx[x] - B * posy[y]) * (kx[x] - B * posy[y]) * nfx for x in range(g.sx)]
                                for y in range(g.sy)])
        else:
            self.mx = np.array([[0.5 * (kx[x] * kx[x] + B * B * posy[y] * posy[y]) * nfx for x in range(g.sx)]
                                for y in range(g.sy)])
            self.mx2 = np.array([[B * posy[y] * kx[x] * nfx for x in range(g.sx)] for y in range(g.sy)])

    def apply(self, a: np.ndarray) -> np.ndarray:
        if self.B == 0:
            f, fi = ("FFT", "iFFT") if self.bt == PERIODIC else ("DST", "iDST")
            return transform(transform(a, f) * self.mxy, fi)
        if self.bt == PERIODIC:
            s = transform(transform(a, "FFTx") * self.mx, "iFFTx")
            t = transform(transform(a, "FFTy") * self.my[:, None], "iFFTy")
            return s + t
        s = transform(a, "DSTx")
        t2 = shift_x_imag(s, self.mx2)
        s = transform(s * self.mx, "iDSTx") + transform(t2, "iDCTx")
        t = transform(transform(a, "DSTy") * self.my[:, None], "iDSTy")
        return s + t


class Hamiltonian:
    """H = T + V as the OperatorSum of itpsystem.cpp:116-119 (potential term only
    when V is not null)."""

    def __init__(self, g: Grid, V, bt: int, B: float):
        self.g, self.V = g, V
        self.T = Kinetic(g, bt, B)

    def apply(self, a: np.ndarray) -> np.ndarray:
        out = self.T.apply(a)
        if self.V is not None:
            out = out + a * self.V
        return out


def dot(g: Grid, a: np.ndarray, b: np.ndarray):
    """State::dot, state.hpp:227-240: sum conj(a)*b * dx^2 over the last two axes."""
    return np.sum(np.conj(a) * b, axis=(-2, -1)) * g.dx * g.dx


def energies(H: Hamiltonian, psi: np.ndarray):
    """Operator::mean_and_standard_deviation (operators.cpp:40-50) per state:
    mean = <psi|H psi>, sd = sqrt(<psi|H(H psi)> - mean^2) (complex sqrt)."""
    g = H.g
    t = H.apply(psi)
    mean = dot(g, psi, t)
    t2 = H.apply(t)
    meansqr = dot(g, psi, t2)
    sd = np.sqrt((meansqr - mean * mean).astype(np.complex128))
    return mean, sd


class NonPositiveEigenvalue(Exception):
    def __init__(self, n, value):
        super().__init__(f"non-positive overlap eigenvalue {value} at index {n}")
        self.n, self.value = n, value


class NonNormalEigenvalue(Exception):
    def __init__(self, n, value):
        super().__init__(f"non-normal overlap eigenvalue {value} at index {n}")
        self.n, self.value = n, value


def overlap(g: Grid, psi: np.ndarray) -> np.ndarray:
    """S_ij = <psi_i|psi_j> (stateset.cpp:146-154), full Hermitian k x k."""
    k = psi.shape[0]
    A = psi.reshape(k, -1)
    return (np.conj(A) @ A.T) * (g.dx * g.dx)


def orthonormalize(g: Grid, psi: np.ndarray):
    """Canonical subspace orthonormalisation, StateSet::orthonormalize
    (stateset.cpp:136-232): S = U diag(l) U^H with ascending l, checks of
    stateset.cpp:158-173, psi'_n = sum_i U_{i,n} l_n^{-1/2} psi_i. Returns
    (new states, eigenvalues)."""
    k = psi.shape[0]
    if k == 1:
        nrm = math.sqrt(float(np.sum(np.abs(psi) ** 2))) * g.dx
        return psi * (1.0 / nrm), np.array([nrm * nrm])
    S = overlap(g, psi)
    lam, U = np.linalg.eigh(S, UPLO="U")
    for n in range(k):
        if lam[n] <= 0:
            raise NonPositiveEigenvalue(n, lam[n])
        if not np.isfinite(lam[n]) or (lam[n] != 0 and abs(lam[n]) < np.finfo(float).tiny):
            raise NonNormalEigenvalue(n, lam[n])
    W = U / np.sqrt(lam)[None, :]
    out = (W.T @ psi.reshape(k, -1)).reshape(psi.shape)
    return out, lam


def how_orthonormal(g: Grid, psi: np.ndarray) -> float:
    """StateSet::how_orthonormal (stateset.cpp:251-269): max deviation of the
    overlap matrix from the identity."""
    S = overlap(g, psi)
    return float(np.max(np.abs(S - np.eye(S.shape[0]))))


def subspace_cosines(g: Grid, a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Singular values of A^H B dx^2 for orthonormal sets A, B: all equal 1 when
    the two sets span the same subspace."""
    k = a.shape[0]
    M = (np.conj(a.reshape(k, -1)) @ b.reshape(b.shape[0], -1).T) * (g.dx * g.dx)
    return np.linalg.svd(M, compute_uv=False)


def gaussian_states(g: Grid, k: int, seed: int) -> np.ndarray:
    """Complex standard-normal states normalised like init_to_gaussian_noise
    (stateset.cpp:124-131). Uses numpy's generator, so values differ from the
    reference's TR1 stream; states are passed to both codes explicitly."""
    rng = np.random.default_rng(seed)
    psi = rng.standard_normal((k, g.sy, g.sx)) + 1j * rng.standard_normal((k, g.sy, g.sx))
    nrm = np.sqrt(np.sum(np.abs(psi) ** 2, axis=(1, 2))) * g.dx
    return psi / nrm[:, None, None]


def harmonic(g: Grid, A: float = 1.0) -> np.ndarray:
    """harmonic(A): 0.5*A*(x^2+y^2), potentialtypes.hpp:103-107."""
    x, y = g.posx[None, :], g.posy[:, None]
    return 0.5 * A * (x * x + y * y)


def fock_darwin(n: int, m: int, B: float) -> float:
    """Fock-Darwin level E(n, m) for V = r^2/2, test_itp.cpp:28-31."""
    U = math.sqrt(1 + 0.25 * B * B)
    return (2 * n + abs(m) + 1) * U - 0.5 * m * B


def fock_darwin_spectrum(count: int, B: float) -> np.ndarray:
    vals = []
    lim = int(2 * math.sqrt(count)) + 8
    for n in range(lim):
        for m in range(-4 * lim, 4 * lim + 1):
            vals.append(fock_darwin(n, m, B))
    return np.sort(np.array(vals))[:count]


def bumpy_potential(g: Grid, nbumps: int, seed: int, amp=(0.8, 1.2), width=0.1, extent=6.0) -> np.ndarray:
    """Harmonic dot plus seeded Gaussian bumps A*exp(-|r-c|^2/(2 w^2)) (the
    Gaussian-impurity form of noise.cpp:38), amplitudes U[amp], centres
    uniform in |x|,|y| < extent. Returns only the bump part."""
    rng = np.random.default_rng(seed)
    A = rng.uniform(amp[0], amp[1], nbumps)
    c = rng.uniform(-extent, extent, (nbumps, 2))
    x, y = g.posx[None, :], g.posy[:, None]
    out = np.zeros((g.sy, g.sx))
    for j in range(nbumps):
        out += A[j] * np.exp(-((x - c[j, 0]) ** 2 + (y - c[j, 1]) ** 2) / (2 * width * width))
    return out


def gaussian_impurities(g: Grid, impurities: np.ndarray, V: np.ndarray) -> np.ndarray:
    """V plus the impurities (rows x, y, A, w) added one at a time in list order,
    each as A*exp(-0.5*(r2/w2)) with r = impurity - grid point
    (GaussianImpurities::add_noise, noise.cpp:24-40, on the grid of
    datalayout.cpp:21-36). V is [sy][sx]; returns a new array."""
    out = np.array(V, dtype=np.float64, copy=True)
    px, py = g.posx[None, :], g.posy[:, None]
    for cx, cy, A, w in np.asarray(impurities, dtype=np.float64):
        rx = cx - px
        ry = cy - py
        out += A * np.exp(-0.5 * ((rx * rx + ry * ry) / (w * w)))
    return out
