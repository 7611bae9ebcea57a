"""FP64 overlap and rotation on the int8 tensor cores (ITP2D_FP64_INT8,
csrc/oz.cu) against the FP64 (DMMA) contractions of the same states: the
overlap matrix, canonical and Cholesky orthonormalisations
(stateset.cpp:136-232) and a whole FP64 solve.

The int8 engine splits both operands into eight int8 slices under per-row
power-of-two scales and sums the slice products exactly; its results agree
with FP64 products to about 1e-15 of the largest output of a row, so the two
engines agree to 1e-13 of the largest value here.
"""
import numpy as np
import pytest

from itp2d_b200 import capi

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")


def _states(sx, sy, k, seed, L=10.0):
    dx = L / sx
    rng = np.random.default_rng(seed)
    x = (np.arange(sx) - sx / 2) * dx
    y = (np.arange(sy) - sy / 2) * dx
    env = np.exp(-0.5 * (y[:, None] ** 2 + x[None, :] ** 2) / 6.0)
    return (rng.standard_normal((k, sy, sx)) + 1j * rng.standard_normal((k, sy, sx))) * env, dx


def _orthonormalized(psi, dx, sx, sy, engine, algo):
    k = psi.shape[0]
    c = capi.Context(sx, sy, dx, k)
    c.set_fp64_engine(engine)
    c.upload(psi)
    c.orthonormalize(algo)
    out = c.download()
    n = c.int8_contractions()
    c.close()
    return out, n


def _gram(out, dx):
    X = out.reshape(out.shape[0], -1)
    return (X.conj() @ X.T) * dx * dx


# 48 x 42: 2016 grid points (31.5 tiles of 64); k = 70, 130: ragged state
# tiles and K steps; 300: three state tiles
@pytest.mark.parametrize("sx,sy,k", [(48, 42, 70), (64, 64, 130), (64, 64, 300)])
@pytest.mark.parametrize("algo", [capi.ORTHO_DEFAULT, capi.ORTHO_CHOLESKY])
def test_int8_orthonormalisation_matches_dmma(sx, sy, k, algo):
    """Orthonormalised states from the int8 engine (overlap and rotation)
    against the DMMA engine's. The Cholesky factor depends smoothly on the
    overlap (condition numbers 3 to 6 here): agreement to 1e-13. The canonical
    eigenvectors of two overlaps that differ by their rounding (about 1e-14)
    differ by that over the eigenvalue gaps, so the canonical states are
    checked by their defining property instead: P = <out|psi> dx^2 gives
    P P^H = diag(ascending eigenvalues of the overlap)."""
    psi, dx = _states(sx, sy, k, seed=k + sx)
    ref, n0 = _orthonormalized(psi, dx, sx, sy, capi.FP64_DMMA, algo)
    out, n1 = _orthonormalized(psi, dx, sx, sy, capi.FP64_INT8, algo)
    assert n0 == 0 and n1 == 2  # the overlap and the rotation
    P = psi.reshape(k, -1)
    S = (P.conj() @ P.T) * dx * dx
    lam = np.linalg.eigvalsh(S)
    gap = np.min(np.diff(lam)) / lam[-1]
    err = np.max(np.abs(out - ref)) / np.max(np.abs(ref))
    orth = np.max(np.abs(_gram(out, dx) - np.eye(k)))
    print(f"int8 orthonormalisation {sx}x{sy} k={k} algo={algo}: max |int8 - dmma| / max |dmma| {err:.1e} "
          f"(smallest relative gap {gap:.1e}), orthonormality {orth:.1e}")
    assert orth < 1e-12
    if algo == capi.ORTHO_CHOLESKY:
        assert err < 1e-13
    else:
        Pn = (out.reshape(k, -1).conj() @ P.T) * dx * dx
        M = Pn @ Pn.conj().T
        assert np.max(np.abs(M - np.diag(np.diag(M)))) < 1e-13 * lam[-1]
        assert np.max(np.abs(np.diag(M).real - lam)) < 1e-13 * lam[-1]


# 48 x 42: grid steps of 16 points with a ragged end; 64 x 64 with k = 300:
# three state tiles; 512 x 256 with k = 1024: about 9 grid splits of 900
# steps, each summed in two chunks of at most 512 steps (the S32 bound)
@pytest.mark.parametrize("sx,sy,k", [(48, 42, 70), (64, 64, 300), (512, 256, 1024)])
def test_int8_overlap_matches_dmma(sx, sy, k):
    psi, dx = _states(sx, sy, k, seed=3 * k + sy, L=16.0)
    S = {}
    for engine in (capi.FP64_DMMA, capi.FP64_INT8):
        c = capi.Context(sx, sy, dx, k)
        c.set_fp64_engine(engine)
        c.upload(psi)
        S[engine] = c.overlap_matrix()
        assert c.int8_contractions() == (1 if engine == capi.FP64_INT8 else 0)
        c.close()
    scale = np.max(np.abs(S[capi.FP64_DMMA]))
    err = np.max(np.abs(S[capi.FP64_INT8] - S[capi.FP64_DMMA])) / scale
    msg = f"int8 overlap {sx}x{sy} k={k}: vs DMMA {err:.1e}"
    if k * sx * sy <= 2e7:
        # the split's error bound per element: each of the 2 G real products
        # x y is off by at most about 9.1 x 2^-56 x 2^(e_x + e_y) (the dropped
        # slice pairs and the remainders below the eighth slice), e the
        # states' scale exponents (max |component| < 2^e)
        P = psi.reshape(k, -1)
        e = np.frexp(np.maximum(np.abs(P.real), np.abs(P.imag)).max(axis=1))[1].astype(float)
        bound = 10.0 * 2.0 ** -56 * 2 * P.shape[1] * 2.0 ** (e[:, None] + e[None, :]) * dx * dx
        diff = np.abs(S[capi.FP64_INT8] - (P.conj() @ P.T) * dx * dx)
        msg += f", vs numpy {np.max(diff) / scale:.1e} (largest share of the bound {np.max(diff / bound):.2f})"
        assert np.all(diff <= bound)
    print(msg)
    # the two engines' own roundings (each about 1e-14 of max |S| here)
    assert err < 1e-13
    assert np.array_equal(S[capi.FP64_INT8], S[capi.FP64_INT8].conj().T)


def test_fp64_solve_with_int8_contractions_matches_dmma():
    """A whole FP64 solve (harmonic oscillator in a field, 64 x 64, 40 states)
    with every overlap and rotation on the int8 tensor cores: the same
    iterations and the same energies as the DMMA solve to 1e-11."""
    from itp2d_b200 import system
    common = dict(sx=64, sy=64, length=10.0, boundary=capi.PERIODIC, B=0.5, halforder=2, num_states=40,
                  wanted=20, eps=[0.05], timestep_test="abschange(1e-9)", final_test="abschange(1e-9)",
                  potential="harmonic(1)", max_steps=3000)
    psi, _ = _states(64, 64, 40, seed=5)
    runs = {}
    for engine in (capi.FP64_DMMA, capi.FP64_INT8):
        s = system.ITPSystem(system.Parameters(fp64_engine=engine, **common), init_states=psi)
        s.run()
        assert s.finished and not s.error_flag
        runs[engine] = (s.total_steps, s.energies()[0][:20].copy(),
                        capi.lib().itp2d_int8_contractions(s.context_handle()))
        s.close()
    (n0, E0, c0), (n1, E1, c1) = runs[capi.FP64_DMMA], runs[capi.FP64_INT8]
    print(f"FP64 solve: DMMA {n0} iterations, int8 {n1} ({c1} int8 contractions); "
          f"max |dE| {np.max(np.abs(E0 - E1)):.1e}")
    assert c0 == 0 and c1 >= 2 * n1
    assert abs(n0 - n1) <= 1
    assert np.max(np.abs(E0 - E1)) < 1e-11
