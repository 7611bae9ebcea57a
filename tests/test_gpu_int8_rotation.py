"""FP64 rotation on the int8 tensor cores (ITP2D_ROTATION_INT8, csrc/oz.cu)
against the FP64 (DMMA) rotation of the same states: canonical and Cholesky
orthonormalisations (stateset.cpp:136-232) and a whole FP64 solve.

The int8 rotation splits W and the states into eight int8 slices under
per-row power-of-two scales and sums the slice products exactly; its result
agrees with FP64 products to about 1e-15 of the largest output of a row, so
the two rotations agree to 1e-13 of the largest state value here.
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
    c.set_fp64_rotation(engine)
    c.upload(psi)
    c.orthonormalize(algo)
    out = c.download()
    n = c.int8_rotations()
    c.close()
    return out, n


def _gram(out, dx):
    X = out.reshape(out.shape[0], -1)
    return (X.conj() @ X.T) * dx * dx


# 48 x 42: 2016 grid points (31.5 tiles of 64); k = 70, 130: ragged state
# tiles and K steps; 300: three state tiles
@pytest.mark.parametrize("sx,sy,k", [(48, 42, 70), (64, 64, 130), (64, 64, 300)])
@pytest.mark.parametrize("algo", [capi.ORTHO_DEFAULT, capi.ORTHO_CHOLESKY])
def test_int8_rotation_matches_dmma(sx, sy, k, algo):
    psi, dx = _states(sx, sy, k, seed=k + sx)
    ref, n0 = _orthonormalized(psi, dx, sx, sy, capi.ROTATION_DMMA, algo)
    out, n1 = _orthonormalized(psi, dx, sx, sy, capi.ROTATION_INT8, algo)
    assert n0 == 0 and n1 == 1
    err = np.max(np.abs(out - ref)) / np.max(np.abs(ref))
    orth = np.max(np.abs(_gram(out, dx) - np.eye(k)))
    print(f"int8 rotation {sx}x{sy} k={k} algo={algo}: max |int8 - dmma| / max |dmma| {err:.1e}, "
          f"orthonormality {orth:.1e}")
    assert err < 1e-13
    assert orth < 1e-12


def test_fp64_solve_with_int8_rotations_matches_dmma():
    """A whole FP64 solve (harmonic oscillator in a field, 64 x 64, 40 states)
    with every rotation on the int8 tensor cores: the same iterations and the
    same energies as the DMMA solve to 1e-11."""
    from itp2d_b200 import system
    common = dict(sx=64, sy=64, length=10.0, boundary=capi.PERIODIC, B=0.5, halforder=2, num_states=40,
                  wanted=20, eps=[0.05], timestep_test="abschange(1e-9)", final_test="abschange(1e-9)",
                  potential="harmonic(1)", max_steps=3000)
    psi, _ = _states(64, 64, 40, seed=5)
    runs = {}
    for engine in (capi.ROTATION_DMMA, capi.ROTATION_INT8):
        s = system.ITPSystem(system.Parameters(fp64_rotation=engine, **common), init_states=psi)
        s.run()
        assert s.finished and not s.error_flag
        runs[engine] = (s.total_steps, s.energies()[0][:20].copy(),
                        capi.lib().itp2d_int8_rotations(s.context_handle()))
        s.close()
    (n0, E0, c0), (n1, E1, c1) = runs[capi.ROTATION_DMMA], runs[capi.ROTATION_INT8]
    print(f"FP64 solve: DMMA {n0} iterations, int8 {n1} ({c1} int8 rotations); "
          f"max |dE| {np.max(np.abs(E0 - E1)):.1e}")
    assert c0 == 0 and c1 >= n1
    assert abs(n0 - n1) <= 1
    assert np.max(np.abs(E0 - E1)) < 1e-11
