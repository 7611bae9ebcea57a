"""GPU parity tests: the CUDA path through the C ABI against the reference's
outputs (golden fixtures from the compiled reference), the numpy restatement,
and the known answers of the reference's unit tests."""
import glob
import math
import os

import numpy as np
import pytest

from oracle import itp_oracle as O

pytestmark = pytest.mark.gpu

EPS = np.finfo(float).eps
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def capi():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from itp2d_b200 import capi as C
    C.lib()
    return C


def rms(a, b):
    return math.sqrt(float(np.mean(np.abs(a - b) ** 2)))


def per_state_rel(a, b):
    return float(np.max(np.max(np.abs(a - b), axis=(-2, -1)) / np.max(np.abs(b), axis=(-2, -1))))


def make_ctx(capi, g, k, bt, B, m, V, eps=None, precision=0):
    c = capi.Context(g.sx, g.sy, g.dx, k, bt, B, m, precision)
    c.set_potential(V)
    if eps is not None:
        c.set_time_step(eps)
    return c


# ---------------- transforms (test_transformer.cpp) ----------------

def _field(g, f):
    X, Y = np.meshgrid(g.posx, g.posy)
    return f(X, Y)


TG = O.Grid(16, 16, 0.5)


def _one(capi, a, kind):
    c = capi.Context(a.shape[-1], a.shape[-2], TG.dx, 1)
    c.upload(a[None])
    c.transform(kind)
    return c.download()[0]


def test_transform_known_answers(capi):
    sine_blob = _field(TG, lambda x, y: (4 * np.cos(x * math.pi / 8) * np.cos(y * math.pi / 8)) * (1 - 1j))
    unit_wave = _field(TG, lambda x, y: np.exp(1j * (2 * math.pi * x / 8 - math.pi / 16))
                       * np.exp(1j * (2 * math.pi * y / 8 - math.pi / 16)))
    nf = O.norm_factors(TG)
    d = np.zeros((16, 16), complex)
    d[0, 0] = 1 - 1j
    assert rms(_one(capi, d, "iDST"), sine_blob) < 10 * EPS
    d1 = np.zeros((16, 16), complex)
    d1[1, 1] = 1.0
    assert rms(_one(capi, d1, "iFFT"), unit_wave) < 10 * EPS
    assert rms(_one(capi, sine_blob, "DST") * nf["DSCT"], d) < 10 * EPS
    assert rms(_one(capi, unit_wave, "FFT") * nf["FFT"], d1) < 10 * EPS


@pytest.mark.parametrize("kind", ["FFT", "FFTx", "FFTy", "DST", "DSTx", "DSTy", "DCT", "DCTx", "DCTy"])
def test_transform_roundtrip(capi, kind):
    A = _field(TG, lambda x, y: np.exp(-(x * x + y * y)) * (1 - 1j))
    nf = O.norm_factors(TG)
    fac = {"FFT": nf["FFT"], "FFTx": nf["FFTx"], "FFTy": nf["FFTy"]}.get(
        kind, nf["DSCT"] if kind in ("DST", "DCT") else (nf["DSCTx"] if kind.endswith("x") else nf["DSCTy"]))
    inv = "i" + kind
    c = capi.Context(16, 16, TG.dx, 1)
    c.upload(A[None])
    c.transform(kind)
    c.transform(inv)
    T = c.download()[0] * fac
    assert rms(A, T) < 2 * EPS


@pytest.mark.parametrize("shape", [(24, 20), (40, 42), (96, 40), (56, 40)])
def test_all_transforms_match_oracle(capi, shape):
    sx, sy = shape
    g = O.Grid(sx, sy, 0.3)
    psi = O.gaussian_states(g, 3, 11)
    for kind in capi.TRANSFORMS:
        c = capi.Context(sx, sy, g.dx, 3)
        c.upload(psi)
        c.transform(kind)
        out = c.download()
        ref = O.transform(psi, kind)
        err = np.max(np.abs(out - ref)) / np.max(np.abs(ref))
        assert err < 1e-14, (kind, err)


# ---------------- the three seams against the compiled reference ----------------

SEAMS = sorted(glob.glob(os.path.join(GOLDEN, "seam_*.npz")))


def _seam(path):
    z = np.load(path)
    sx, sy, L, bt, B, m, eps = z["cfg"]
    g = O.Grid.from_length(int(sx), int(sy), float(L))
    V = None if bool(z["potential_null"]) else z["V"]
    return z, g, int(bt), float(B), int(m), float(eps), V


@pytest.mark.parametrize("path", SEAMS, ids=[os.path.basename(p)[5:-4] for p in SEAMS])
def test_seams_match_reference(capi, path):
    z, g, bt, B, m, eps, V = _seam(path)
    psi = z["psi"]
    k = psi.shape[0]
    c = make_ctx(capi, g, k, bt, B, m, V, eps)
    c.upload(psi)
    c.propagate()
    prop = c.download()
    # one FP64 propagation step elementwise within 1e-12 of the reference
    assert per_state_rel(prop, z["prop"]) < 1e-12
    # Hamiltonian application
    c.upload(psi)
    c.apply_hamiltonian()
    assert per_state_rel(c.download(), z["hpsi"]) < 1e-12
    # energies of the propagated states
    c.upload(z["prop"])
    E, sig, res, Ei = c.energies()
    assert np.max(np.abs(E - z["E"]) / np.abs(z["E"])) < 1e-12
    assert np.max(np.abs(sig - z["sigma"])) < 1e-10 * np.max(np.abs(z["E"]))
    # orthonormalisation: same subspace, orthonormal
    c.upload(z["prop"])
    c.orthonormalize()
    ortho = c.download()
    assert O.how_orthonormal(g, ortho) < 64 * EPS
    assert 1 - O.subspace_cosines(g, ortho, z["ortho"]).min() < 1e-10


CONFIGS = [
    # sx, sy, L, boundary, B, m, eps
    (64, 64, 12.0, O.PERIODIC, 0.0, 1, 0.1),
    (64, 48, 12.0, O.DIRICHLET, 0.0, 2, 0.05),
    (64, 64, 14.0, O.PERIODIC, 1.0, 2, 0.05),
    (64, 64, 16.0, O.PERIODIC, 0.5, 3, 0.05),
    (96, 40, 12.0, O.PERIODIC, 0.3, 2, 0.05),
    (42, 42, 12.0, O.DIRICHLET, 0.0, 3, 0.1),
    (64, 48, 12.0, O.DIRICHLET, 0.7, 2, 0.05),
    (40, 40, 10.0, O.DIRICHLET, 1.5, 3, 0.05),
]


@pytest.mark.parametrize("cfg", CONFIGS)
def test_propagate_energies_match_oracle(capi, cfg):
    sx, sy, L, bt, B, m, eps = cfg
    g = O.Grid.from_length(sx, sy, L)
    V = O.harmonic(g) + O.bumpy_potential(g, 10, 3, extent=L / 3)
    k = 6
    psi = O.gaussian_states(g, k, 5)
    c = make_ctx(capi, g, k, bt, B, m, V, eps)
    c.upload(psi)
    c.propagate()
    prop = c.download()
    ref = O.MultiProductSplit(g, V, bt, B, m, eps).apply(psi)
    assert per_state_rel(prop, ref) < 1e-12
    H = O.Hamiltonian(g, V, bt, B)
    E, sig, res, Ei = c.energies()
    mean, sd = O.energies(H, ref)
    assert np.max(np.abs(E - mean.real) / np.abs(mean.real)) < 1e-12
    # residual deviation ||H psi - E psi|| of normalised states (the FP64 form
    # takes states as normalised, like the reference): the second evaluation
    # shifts by the first one's energies and has no cancellation
    pn = ref / (np.sqrt(np.sum(np.abs(ref) ** 2, axis=(1, 2))) * g.dx)[:, None, None]
    c.upload(pn)
    c.energies()
    E2, _, res2, _ = c.energies()
    hp = H.apply(pn)
    r_ref = np.sqrt(np.sum(np.abs(hp - E2[:, None, None] * pn) ** 2, axis=(1, 2))) * g.dx
    assert np.max(np.abs(res2 - r_ref) / r_ref) < 1e-10


def test_timestep_change_rebuilds_tables(capi):
    g = O.Grid.from_length(32, 32, 12.0)
    V = O.harmonic(g)
    psi = O.gaussian_states(g, 2, 1)
    c = make_ctx(capi, g, 2, O.PERIODIC, 0.5, 2, V, 0.2)
    c.set_time_step(0.05)
    c.upload(psi)
    c.propagate()
    ref = O.MultiProductSplit(g, V, O.PERIODIC, 0.5, 2, 0.05).apply(psi)
    assert per_state_rel(c.download(), ref) < 1e-12


# ---------------- orthonormalisation and eigensolver ----------------

def test_stateset_orthonormalization(capi):
    """test_stateset.cpp:26-42: 16x16 grid, dx = 1, 8 random states -> 16 eps."""
    g = O.Grid(16, 16, 1.0)
    psi = O.gaussian_states(g, 8, 3)
    c = capi.Context(16, 16, 1.0, 8)
    c.set_potential(None)
    c.upload(psi)
    c.orthonormalize(capi.ORTHO_DEFAULT)
    out = c.download()
    assert O.how_orthonormal(g, out) < 16 * EPS
    c.upload(psi)
    c.orthonormalize(capi.ORTHO_HIGHMEM)
    assert O.how_orthonormal(g, c.download()) < 16 * EPS


@pytest.mark.parametrize("k", [2, 7, 33, 130, 300])
def test_orthonormalize_subspace_and_order(capi, k):
    g = O.Grid.from_length(32, 24, 12.0)
    V = O.harmonic(g)
    psi = O.MultiProductSplit(g, V, O.PERIODIC, 0.0, 1, 0.3).apply(O.gaussian_states(g, k, k))
    c = capi.Context(32, 24, g.dx, k)
    c.set_potential(V)
    c.upload(psi)
    c.orthonormalize()
    out = c.download()
    ref, lam = O.orthonormalize(g, psi)
    # the achievable orthonormality scales with the overlap's condition
    # number; bound the GPU by the oracle's own result on the same input
    bound = max(64 * EPS, 4 * O.how_orthonormal(g, ref))
    assert O.how_orthonormal(g, out) < bound
    # both sets span the input's subspace; the cosines can only be as close to 1
    # as the two sets are orthonormal
    assert 1 - O.subspace_cosines(g, out, ref).min() < max(1e-10, 2 * bound)
    # state n belongs to the n-th smallest overlap eigenvalue: compare norms of
    # projections onto the oracle's state n (phases are arbitrary)
    ov = np.abs(np.sum(np.conj(ref) * out, axis=(1, 2)) * g.dx * g.dx)
    gaps = np.diff(lam) / lam[1:]
    isolated = [n for n in range(k) if (n == 0 or gaps[n - 1] > 1e-6) and (n == k - 1 or gaps[n] > 1e-6)]
    assert np.all(ov[isolated] > 1 - 1e-8)


def test_orthonormalize_errors(capi):
    g = O.Grid(12, 12, 1.0)
    psi = O.gaussian_states(g, 4, 3)
    psi[2] = 0.0
    c = capi.Context(12, 12, 1.0, 4)
    c.set_potential(None)
    c.upload(psi)
    with pytest.raises(capi.ITP2DError) as e:
        c.orthonormalize()
    assert e.value.status == capi.E_NONPOSITIVE_EIGENVALUE and e.value.bad_index == 0
    assert np.array_equal(c.download(), psi)  # states unchanged on failure
    psi = O.gaussian_states(g, 4, 3)
    psi[1, 3, 3] = np.nan
    c.upload(psi)
    with pytest.raises(capi.ITP2DError) as e:
        c.orthonormalize()
    assert e.value.status == capi.E_NONNORMAL_EIGENVALUE


def test_single_state_normalises(capi):
    g = O.Grid(16, 16, 0.5)
    psi = O.gaussian_states(g, 1, 1) * 3.0
    c = capi.Context(16, 16, 0.5, 1)
    c.set_potential(None)
    c.upload(psi)
    c.orthonormalize()
    out = c.download()
    assert abs(np.sqrt(np.sum(np.abs(out) ** 2)) * g.dx - 1) < 4 * EPS


def test_eigensolver_2x2_known(capi):
    """test_eigensolver.cpp:25-41 (eigenvectors up to phase)."""
    ev, U = capi.hermitian_eigensolve(np.array([[1, 2], [2, 4]], dtype=complex))
    assert abs(ev[0]) < 4 * EPS and abs(ev[1] - 5) < 8 * EPS
    for n, ref in [(0, np.array([-2, 1]) / math.sqrt(5)), (1, np.array([1, 2]) / math.sqrt(5))]:
        assert abs(abs(np.vdot(ref, U[:, n])) - 1) < 8 * EPS


def test_eigensolver_spectral_decomposition(capi):
    """test_eigensolver.cpp:43-74: reconstruction within 300 eps."""
    N = 8
    M = np.zeros((N, N), complex)
    for i in range(N):
        for j in range(N):
            M[i, j] = 1 if i == j else (1j * abs(i - j) if j > i else -1j * abs(i - j))
    ev, U = capi.hermitian_eigensolve(M)
    R = (U * ev[None, :]) @ U.conj().T
    assert np.linalg.norm(M - R) < 300 * EPS


@pytest.mark.parametrize("n", [3, 64, 255, 256, 600, 1000, 2000])
def test_eigensolver_random(capi, n):
    rng = np.random.default_rng(n)
    X = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    M = X @ X.conj().T / n + np.eye(n)
    ev, U = capi.hermitian_eigensolve(M)
    ref = np.linalg.eigvalsh(M)
    assert np.max(np.abs(ev - ref)) < 1e-13 * np.max(np.abs(ref))
    # rounding of the accumulated rotations grows like sqrt(n) eps
    assert np.max(np.abs(U.conj().T @ U - np.eye(n))) < max(2e-14, 1e-15 * math.sqrt(n))
    assert np.max(np.abs(M @ U - U * ev[None, :])) < 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("n", [300, 520, 2000])
def test_eigensolver_graded_spectrum(capi, n):
    """Overlap-like matrix: eigenvalues exp(-2 eps E) spread over three decades,
    near-degenerate pairs included; absolute accuracy eps-scale, eigenvectors
    orthonormal."""
    rng = np.random.default_rng(n)
    E = np.sort(rng.uniform(1, 70, n))
    E[1::7] = E[0::7][: len(E[1::7])] + 1e-9  # near-degenerate pairs
    lam = np.exp(-0.1 * E)
    X = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))[0]
    M = (X * lam[None, :]) @ X.conj().T
    M = 0.5 * (M + M.conj().T)
    ev, U = capi.hermitian_eigensolve(M)
    assert np.max(np.abs(ev - np.sort(lam))) < 1e-13 * lam.max()
    assert np.max(np.abs(U.conj().T @ U - np.eye(n))) < 1e-13
    assert np.max(np.abs(M @ U - U * ev[None, :])) < 1e-13 * lam.max()
