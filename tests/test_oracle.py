"""CPU tests of the oracle: the numpy restatement against the reference's own
known-answer tests, and against the reference sources compiled into
oracle/_ref (when built). No GPU needed."""
import glob
import math
import os

import numpy as np
import pytest

from oracle import itp_oracle as O
from oracle import refkit as R

EPS = np.finfo(float).eps


def rms(a, b):
    return math.sqrt(float(np.mean(np.abs(a - b) ** 2)))


# ---- test_transformer.cpp:25-149 known answers (16x16, dx = 0.5) ----

TSX, TSY, TDX = 16, 16, 0.5


def _tgrid():
    return O.Grid(TSX, TSY, TDX)


def _field(g, f):
    X, Y = np.meshgrid(g.posx, g.posy)
    return f(X, Y)


def _initfunc(x, y):
    v = np.exp(-(x * x + y * y))
    return v - 1j * v


def _sine_blob(x, y):
    v = 4 * np.cos(x * math.pi / (TSX * TDX)) * np.cos(y * math.pi / (TSY * TDX))
    return v - 1j * v


def _unit_wave(x, y):
    px = 2 * math.pi * x / (TSX * TDX) - math.pi / TSX
    py = 2 * math.pi * y / (TSY * TDX) - math.pi / TSY
    return np.exp(1j * px) * np.exp(1j * py)


def test_kvalues():
    g = _tgrid()
    kx = O.fft_k(g.sx, g.lenx)
    for x in range(g.sx):
        assert kx[x] == (2 * math.pi / g.lenx) * float(x if x < g.sx // 2 else x - g.sx)
        assert O.dsct_k(g.sx, g.lenx)[x] == (math.pi / g.lenx) * float(x + 1)


@pytest.mark.parametrize("kind", ["FFT", "FFTx", "FFTy", "DST", "DSTx", "DSTy", "DCT", "DCTx", "DCTy"])
def test_inverse_transform_roundtrip(kind):
    g = _tgrid()
    A = _field(g, _initfunc)
    inv = {"FFT": "iFFT", "FFTx": "iFFTx", "FFTy": "iFFTy", "DST": "iDST", "DSTx": "iDSTx",
           "DSTy": "iDSTy", "DCT": "iDCT", "DCTx": "iDCTx", "DCTy": "iDCTy"}[kind]
    nf = O.norm_factors(g)
    fac = {"FFT": nf["FFT"], "FFTx": nf["FFTx"], "FFTy": nf["FFTy"], "DST": nf["DSCT"], "DSTx": nf["DSCTx"],
           "DSTy": nf["DSCTy"], "DCT": nf["DSCT"], "DCTx": nf["DSCTx"], "DCTy": nf["DSCTy"]}[kind]
    T = O.transform(O.transform(A, kind), inv) * fac
    assert rms(A, T) < EPS


def test_dirac_delta_idst():
    g = _tgrid()
    T = np.zeros((g.sy, g.sx), complex)
    T[0, 0] = 1 - 1j
    assert rms(O.transform(T, "iDST"), _field(g, _sine_blob)) < 10 * EPS


def test_dirac_delta_ifft():
    g = _tgrid()
    T = np.zeros((g.sy, g.sx), complex)
    T[1, 1] = 1.0
    assert rms(O.transform(T, "iFFT"), _field(g, _unit_wave)) < 10 * EPS


def test_sine_blob_dst():
    g = _tgrid()
    T = O.transform(_field(g, _sine_blob), "DST") * O.norm_factors(g)["DSCT"]
    D = np.zeros_like(T)
    D[0, 0] = 1 - 1j
    assert rms(T, D) < 10 * EPS


def test_unit_wave_fft():
    g = _tgrid()
    T = O.transform(_field(g, _unit_wave), "FFT") * O.norm_factors(g)["FFT"]
    D = np.zeros_like(T)
    D[1, 1] = 1.0
    assert rms(T, D) < 10 * EPS


# ---- test_laplacian.cpp:38-58 ----

def test_laplacian_of_gaussian():
    N, L = 42, 12.0
    g = O.Grid(N, N, L / N)
    G = _field(g, lambda x, y: np.exp(-(x * x + y * y)) + 0j)
    kx, ky = O.fft_k(N, g.lenx), O.fft_k(N, g.leny)
    mult = (-(kx[None, :] ** 2) - ky[:, None] ** 2) * O.norm_factors(g)["FFT"]
    out = O.transform(O.transform(G, "FFT") * mult, "iFFT")
    ref = _field(g, lambda x, y: 4 * (x * x + y * y - 1) * np.exp(-(x * x + y * y)) + 0j)
    assert rms(out, ref) < 100 * EPS
    assert np.max(np.abs(out - ref)) < 1000 * EPS


# ---- test_eigensolver.cpp:25-74 and test_stateset.cpp:26-42 ----

def test_eigen_2x2_known():
    M = np.array([[1, 2], [2, 4]], dtype=complex)
    lam, U = np.linalg.eigh(M, UPLO="U")
    assert abs(lam[0] - 0) < 4 * EPS and abs(lam[1] - 5) < 8 * EPS
    # eigenvectors up to a phase: (-2, 1)/sqrt5 and (1, 2)/sqrt5
    for n, ref in [(0, np.array([-2, 1]) / math.sqrt(5)), (1, np.array([1, 2]) / math.sqrt(5))]:
        assert abs(abs(np.vdot(ref, U[:, n])) - 1) < 4 * EPS


def test_eigen_spectral_decomposition():
    N = 8
    M = np.zeros((N, N), complex)
    for i in range(N):
        for j in range(N):
            M[i, j] = 1 if i == j else (1j * abs(i - j) if j > i else -1j * abs(i - j))
    lam, U = np.linalg.eigh(M, UPLO="U")
    R = (U * lam[None, :]) @ U.conj().T
    assert np.linalg.norm(M - R) < 300 * EPS


def test_stateset_orthonormalization():
    g = O.Grid(16, 16, 1.0)
    psi = O.gaussian_states(g, 8, 3)
    out, _ = O.orthonormalize(g, psi)
    assert O.how_orthonormal(g, out) < 16 * EPS


def test_orthonormalize_rejects_dependent_states():
    g = O.Grid(12, 12, 1.0)
    psi = O.gaussian_states(g, 4, 3)
    psi[3] = 0.0
    with pytest.raises(O.NonPositiveEigenvalue):
        O.orthonormalize(g, psi)
    psi = O.gaussian_states(g, 4, 3)
    psi[1, 2, 2] = np.nan
    with pytest.raises((O.NonNormalEigenvalue, np.linalg.LinAlgError)):
        O.orthonormalize(g, psi)


def test_multiproduct_coefficients():
    assert O.multiproduct_coefficients(1) == [1.0]
    c2 = O.multiproduct_coefficients(2)
    assert abs(c2[0] + 1 / 3) < EPS and abs(c2[1] - 4 / 3) < 2 * EPS
    c3 = O.multiproduct_coefficients(3)
    for a, b in zip(c3, [1 / 24, -16 / 15, 81 / 40]):
        assert abs(a - b) < 4 * EPS
    for m in range(1, 6):
        assert abs(sum(O.multiproduct_coefficients(m)) - 1) < 1e-13


# ---- the restatement against the compiled reference, seam by seam ----

CONFIGS = [
    # sx, sy, L, boundary, B, halforder, eps
    (24, 20, 12.0, O.PERIODIC, 0.0, 1, 0.1),
    (24, 20, 12.0, O.DIRICHLET, 0.0, 2, 0.1),
    (24, 20, 12.0, O.PERIODIC, 1.0, 2, 0.05),
    (24, 20, 12.0, O.DIRICHLET, 0.7, 3, 0.05),
    (16, 16, 12.0, O.PERIODIC, 0.5, 3, 0.05),
    (40, 42, 12.0, O.PERIODIC, 0.0, 2, 0.2),
]


@pytest.mark.parametrize("cfg", CONFIGS)
def test_restatement_matches_reference(cfg, refkit_available):
    if not refkit_available:
        pytest.skip("oracle/_ref not built")
    sx, sy, L, bt, B, m, eps = cfg
    g = O.Grid.from_length(sx, sy, L)
    k = 5
    psi = O.gaussian_states(g, k, 7)
    kit = R.RefKit(sx, sy, L, bt, B, m, eps, k, threads=2)
    V = kit.potential()
    assert np.allclose(V, O.harmonic(g), rtol=0, atol=1e-14)
    fkx, fky, dkx, dky = kit.kvalues()
    assert np.array_equal(fkx, O.fft_k(sx, g.lenx)) and np.array_equal(dky, O.dsct_k(sy, g.leny))
    # one propagation step, elementwise per state relative to max|psi|
    kit.set_states(psi)
    kit.propagate()
    a = kit.states()
    b = O.MultiProductSplit(g, V, bt, B, m, eps).apply(psi)
    err = np.max(np.abs(a - b), axis=(1, 2)) / np.max(np.abs(b), axis=(1, 2))
    assert err.max() < 1e-13
    # Hamiltonian application and energies
    H = O.Hamiltonian(g, V, bt, B)
    kit.set_states(psi)
    kit.apply_hamiltonian()
    assert np.max(np.abs(kit.states() - H.apply(psi))) < 1e-13 * np.max(np.abs(H.apply(psi)))
    kit.set_states(b)
    E, s, Ei = kit.energies()
    mean, sd = O.energies(H, b)
    assert np.max(np.abs(E - mean.real) / np.abs(E)) < 1e-13
    # orthonormalisation: same subspace, orthonormal to 16 eps
    kit.set_states(b)
    assert kit.orthonormalize() == 0
    oa = kit.states()
    ob, _ = O.orthonormalize(g, b)
    assert kit.how_orthonormal() < 16 * EPS
    assert O.how_orthonormal(g, ob) < 16 * EPS
    assert 1 - O.subspace_cosines(g, oa, ob).min() < 1e-12


def test_reference_rejects_dependent_states(refkit_available):
    if not refkit_available:
        pytest.skip("oracle/_ref not built")
    g = O.Grid.from_length(12, 12, 12.0)
    psi = O.gaussian_states(g, 4, 3)
    psi[3] = 0.0
    kit = R.RefKit(12, 12, 12.0, 0, 0.0, 1, 0.1, 4)
    kit.set_states(psi)
    assert kit.orthonormalize() == 1


@pytest.mark.slow
def test_reference_harmonic_oscillator_spectrum(refkit_available):
    """test_itp.cpp:56-91 with a fixed seed: HO 40x40, L=12, N=14, wanted 8."""
    if not refkit_available:
        pytest.skip("oracle/_ref not built")
    tol = 1e-4
    sysm = R.RefSystem(40, 40, 12.0, 0, 0.0, 5, 14, 8, [1.0], eps_divisor=5.0,
                       timestep_test=f"relstdev({tol},{0.1 * tol})", final_test=f"relstdev({tol})",
                       max_steps=50, seed=20120131, threads=2)
    while not sysm.finished:
        sysm.step()
    assert not sysm.error_flag
    E, _ = sysm.energies()
    ref = [1, 2, 2, 3, 3, 3, 4, 4]
    assert np.max(np.abs(E[:8] - ref)) < tol


# ---- the restatement against the golden fixtures (outputs of the compiled reference) ----

GOLDEN_SEAMS = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "seam_*.npz")))


@pytest.mark.parametrize("path", GOLDEN_SEAMS, ids=[p.rsplit("seam_", 1)[1][:-4] for p in GOLDEN_SEAMS])
def test_restatement_matches_golden_fixtures(path):
    """tests/golden/seam_*.npz hold the compiled reference's propagation step,
    H psi, energies and orthonormalised states on seeded inputs
    (tests/golden/make_golden.py); the numpy restatement reproduces them."""
    z = np.load(path)
    sx, sy, L, bt, B, m, eps = z["cfg"]
    g = O.Grid.from_length(int(sx), int(sy), float(L))
    V = None if bool(z["potential_null"]) else z["V"]
    bt, B, m, eps = int(bt), float(B), int(m), float(eps)
    psi = z["psi"]
    prop = O.MultiProductSplit(g, V, bt, B, m, eps).apply(psi)
    rel = np.max(np.abs(prop - z["prop"]), axis=(1, 2)) / np.max(np.abs(z["prop"]), axis=(1, 2))
    assert rel.max() < 1e-13
    H = O.Hamiltonian(g, V, bt, B)
    hpsi = H.apply(psi)
    assert np.max(np.abs(hpsi - z["hpsi"])) < 1e-13 * np.max(np.abs(z["hpsi"]))
    mean, _ = O.energies(H, z["prop"])
    assert np.max(np.abs(mean.real - z["E"]) / np.abs(z["E"])) < 1e-13
    ortho, _ = O.orthonormalize(g, z["prop"])
    assert 1 - O.subspace_cosines(g, ortho, z["ortho"]).min() < 1e-12


def test_gaussian_impurities_restatement_matches_reference(refkit_available):
    """The numpy restatement of GaussianImpurities::add_noise (noise.cpp:24-40)
    against the compiled reference on the same impurity list: bit-identical
    (same operations in the same order, glibc exp on both sides)."""
    if not refkit_available:
        pytest.skip("oracle/_ref not built")
    g = O.Grid.from_length(40, 28, 12.0)
    rng = np.random.default_rng(7)
    n = 60
    imp = np.column_stack([rng.uniform(-6, 6, n), rng.uniform(-4, 4, n), rng.uniform(0.5, 1.5, n),
                           rng.uniform(0.1, 0.3, n)])
    V0 = O.harmonic(g)
    ours = O.gaussian_impurities(g, imp, V0)
    ref = R.add_gaussian_impurities(g.sx, g.sy, g.dx, imp, V0)
    assert np.max(np.abs(ours - ref)) <= 1e-15 * np.max(np.abs(ref))
    assert np.max(np.abs(ours - V0)) > 0.5  # the impurities are there
