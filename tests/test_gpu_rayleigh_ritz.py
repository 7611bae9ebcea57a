"""Rayleigh-Ritz step on the device (itp2d_rayleigh_ritz): the projected
Hamiltonian <psi_i|H psi_j> dx^2, its eigendecomposition and the rotation of
the states onto the Ritz vectors.

No reference counterpart (the reference's energies are per-state expectation
values, itpsystem.cpp:483-494); checked against the numpy oracle's
Hamiltonian (Kinetic kinetic.cpp:99-142 plus the potential) projected on the
same states and diagonalised by numpy.
"""
import numpy as np
import pytest

from oracle import itp_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def capi():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from itp2d_b200 import capi as C
    C.lib()
    return C


def _setup(sx, sy, L, bt, B, k, seed):
    g = O.Grid.from_length(sx, sy, L)
    V = O.harmonic(g) + O.bumpy_potential(g, 6, seed, extent=L / 3)
    psi, _ = O.orthonormalize(g, O.gaussian_states(g, k, seed))
    H = O.Hamiltonian(g, V, bt, B)
    P = psi.reshape(k, -1)
    Hs = (np.conj(P) @ H.apply(psi).reshape(k, -1).T) * g.dx * g.dx
    theta = np.linalg.eigvalsh(0.5 * (Hs + Hs.conj().T))
    return g, V, psi, H, theta


# (periodic, B = 0.5): complex projected matrix; (Dirichlet, B = 0): the
# DST-II/III lines; k = 300 takes the block Jacobi eigensolver
@pytest.mark.parametrize("sx,sy,bt,B,k", [(64, 64, 0, 0.5, 24), (48, 40, 1, 0.0, 17), (96, 96, 0, 1.0, 300)])
def test_rayleigh_ritz_fp64_matches_numpy(capi, sx, sy, bt, B, k):
    g, V, psi, H, theta_ref = _setup(sx, sy, 10.0, bt, B, k, seed=sx + k)
    c = capi.Context(sx, sy, g.dx, k, bt, B, 2)
    c.set_potential(V)
    c.set_time_step(0.05)
    c.upload(psi)
    theta = c.rayleigh_ritz()
    out = c.download()
    scale = np.max(np.abs(theta_ref))
    err = np.max(np.abs(theta - theta_ref)) / scale
    orth = O.how_orthonormal(g, out)
    # the Ritz vectors diagonalise the projected Hamiltonian: their energies
    # are the Ritz values and the off-diagonal elements vanish
    X = out.reshape(k, -1)
    Hout = (np.conj(X) @ H.apply(out).reshape(k, -1).T) * g.dx * g.dx
    off = np.max(np.abs(Hout - np.diag(np.diag(Hout)))) / scale
    print(f"Rayleigh-Ritz FP64 {sx}x{sy} k={k}: Ritz values {err:.1e}, orthonormality {orth:.1e}, "
          f"off-diagonal {off:.1e}")
    assert err < 1e-12
    assert orth < 1e-12
    assert off < 1e-11
    assert np.max(np.abs(np.diag(Hout).real - theta_ref)) / scale < 1e-11
    # the states span the same subspace as the input
    Pin = psi.reshape(k, -1)
    proj = (np.conj(Pin) @ X.T) * g.dx * g.dx
    assert np.max(np.abs(np.linalg.svd(proj, compute_uv=False) - 1.0)) < 1e-11


def test_rayleigh_ritz_fp32_states(capi):
    """FP32 states: H psi in single precision, the projection and the
    eigensolve in FP64: Ritz values to the FP32 Hamiltonian's accuracy."""
    g, V, psi, H, theta_ref = _setup(128, 128, 12.0, 0, 0.5, 64, seed=3)
    c = capi.Context(128, 128, g.dx, 64, 0, 0.5, 2, capi.FP32)
    c.set_potential(V)
    c.set_time_step(0.05)
    c.upload(psi)
    theta = c.rayleigh_ritz()
    err = np.max(np.abs(theta - theta_ref)) / np.max(np.abs(theta_ref))
    print(f"Rayleigh-Ritz FP32 states: Ritz values {err:.1e}")
    assert err < 2e-6
    assert O.how_orthonormal(g, c.download()) < 2e-5
