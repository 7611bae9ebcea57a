"""Cholesky (Gram-Schmidt order) orthonormalisation, ITP2D_ORTHO_CHOLESKY and
the FP32 form's Cholesky steps between canonical ones (csrc/cholesky.cu).

No reference counterpart (the reference orthonormalises canonically,
stateset.cpp:136-232), so the checks are against numpy's Cholesky
factorisation of the same overlap: psi'_n = sum_{i <= n} conj((L^-1)_{n,i})
psi_i with S = L L^H, S = Psi^H Psi dx^2.
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


def _states(sx, sy, k, seed, L=10.0, width2=8.0):
    """Seeded complex Gaussian noise under a Gaussian envelope of variance
    width2 (None: flat, for k close to the number of grid points)."""
    dx = L / sx
    rng = np.random.default_rng(seed)
    x = (np.arange(sx) - sx / 2) * dx
    y = (np.arange(sy) - sy / 2) * dx
    env = 1.0 if width2 is None else np.exp(-0.5 * (y[:, None] ** 2 + x[None, :] ** 2) / width2)
    psi = (rng.standard_normal((k, sy, sx)) + 1j * rng.standard_normal((k, sy, sx))) * env
    return psi, dx


def _gram_schmidt(psi, dx):
    k = psi.shape[0]
    P = psi.reshape(k, -1)
    S = (P.conj() @ P.T) * dx * dx  # S_ij = <psi_i|psi_j>
    Linv = np.linalg.inv(np.linalg.cholesky(S))
    # psi'_n = sum_i W_in psi_i with W = L^{-H}: row n of conj(L^{-1}) P
    return (np.conj(Linv) @ P).reshape(psi.shape)


def _gram(out, dx):
    X = out.reshape(out.shape[0], -1)
    return (X.conj() @ X.T) * dx * dx


# k = 5: one partial panel; 70, 130: ragged last panels; 1000, 2000: many
# panels (2000 = the bumpy dot's state count). Flat noise on 4096 grid points
# keeps the overlap's condition number near ((1 + r) / (1 - r))^2 with
# r = sqrt(k / 4096), about 32 at k = 2000.
@pytest.mark.parametrize("sx,sy,k", [(16, 16, 5), (48, 40, 70), (64, 64, 130), (64, 64, 1000), (64, 64, 2000)])
def test_cholesky_fp64_matches_numpy(sx, sy, k):
    psi, dx = _states(sx, sy, k, seed=k, width2=None)
    c = capi.Context(sx, sy, dx, k)
    c.upload(psi)
    c.orthonormalize(capi.ORTHO_CHOLESKY)
    assert c.orthonormalization_counts() == (0, 0, 1)
    out = c.download()
    ref = _gram_schmidt(psi, dx)
    err = np.max(np.abs(out - ref)) / np.max(np.abs(ref))
    orth = np.max(np.abs(_gram(out, dx) - np.eye(k)))
    print(f"Cholesky FP64 {sx}x{sy} k={k}: max |out - numpy| / max |numpy| {err:.2e}, orthonormality {orth:.2e}")
    assert err < 1e-10
    assert orth < 1e-11
    # the state order is kept: output n has no component along inputs > n
    # (the first output is the first input, normalised)
    n0 = np.sqrt(np.sum(np.abs(psi[0]) ** 2)) * dx
    assert np.max(np.abs(out[0] - psi[0] / n0)) < 1e-12 * np.max(np.abs(psi[0] / n0))


def test_cholesky_zero_state_reports_pivot_and_keeps_states():
    psi, dx = _states(32, 32, 40, seed=3)
    psi[37] = 0.0  # S is singular at row 37: pivot exactly 0
    c = capi.Context(32, 32, dx, 40)
    c.upload(psi)
    with pytest.raises(capi.ITP2DError) as e:
        c.orthonormalize(capi.ORTHO_CHOLESKY)
    assert e.value.status == capi.E_NONPOSITIVE_EIGENVALUE
    assert e.value.bad_index == 37 and e.value.bad_value == 0.0
    assert np.array_equal(c.download(), psi)
    # the context stays usable: with an independent state in its place it succeeds
    psi[37] = _states(32, 32, 1, seed=99)[0][0]
    c.upload(psi)
    c.orthonormalize(capi.ORTHO_CHOLESKY)
    assert np.max(np.abs(_gram(c.download(), dx) - np.eye(40))) < 1e-11


def test_fp32_form_cholesky_between_canonical_steps():
    """FP32 states with canonical_every = 3 and Cholesky in between: every
    third call is canonical, the two before it Cholesky (the Cholesky step
    needs no guard: it applies to any positive definite overlap, random
    states included); the Cholesky steps give states orthonormal to the FP32
    contraction accuracy that agree with numpy's Gram-Schmidt of the same
    FP32 states."""
    sx = sy = 64
    k = 96
    psi, dx = _states(sx, sy, k, seed=11)
    c = capi.Context(sx, sy, dx, k, precision=capi.FP32)
    c.set_fp32_orthonormalization(3)
    c.set_fp32_between(capi.BETWEEN_CHOLESKY)
    c.upload(psi)
    for n in range(2):
        before = c.download()  # the FP32 values, widened exactly
        c.orthonormalize()
        assert c.orthonormalization_counts() == (0, 0, n + 1)
        out = c.download()
        assert np.max(np.abs(_gram(out, dx) - np.eye(k))) < 2e-5
        ref = _gram_schmidt(before, dx)
        assert np.max(np.abs(out - ref)) / np.max(np.abs(ref)) < 1e-4
    c.orthonormalize()
    assert c.orthonormalization_counts() == (1, 0, 2)
    c.orthonormalize()
    assert c.orthonormalization_counts() == (1, 0, 3)
    with pytest.raises(capi.ITP2DError):
        c.set_fp32_between(7)


def test_mixed_solve_with_cholesky_steps_matches_fp64():
    """A whole FP32-form solve with Cholesky steps between canonical ones
    (every third canonical) reaches the FP64 form's energies: the FP64
    refinement ends the solve with the reference's canonical steps."""
    from itp2d_b200 import system
    common = dict(sx=64, sy=64, length=10.0, boundary=capi.PERIODIC, B=0.5, halforder=2, num_states=40,
                  wanted=20, eps=[0.05], timestep_test="abschange(1e-9)", final_test="abschange(1e-9)",
                  potential="harmonic(1)", max_steps=3000)
    psi, _ = _states(64, 64, 40, seed=5)
    ref = system.ITPSystem(system.Parameters(**common), init_states=psi)
    ref.run()
    mixed = system.ITPSystem(system.Parameters(precision=capi.FP32, fp32_switch=1e-7, fp32_canonical_every=3,
                                               fp32_between=capi.BETWEEN_CHOLESKY, **common), init_states=psi)
    mixed.run()
    assert ref.finished and not ref.error_flag and mixed.finished and not mixed.error_flag
    import ctypes as C
    n = [C.c_longlong(0) for _ in range(3)]
    assert capi.lib().itp2d_orthonormalization_counts(C.c_void_p(mixed.context_handle()),
                                                     *[C.byref(v) for v in n]) == capi.OK
    c0, c1, c2 = (v.value for v in n)
    print(f"mixed with Cholesky: {mixed.total_steps} iterations (canonical {c0}, Cholesky {c2}); "
          f"FP64 form {ref.total_steps}")
    assert c2 > 0 and c1 == 0
    E64, Em = ref.energies()[0][:20], mixed.energies()[0][:20]
    assert np.max(np.abs(E64 - Em)) < 1e-8
    ref.close()
    mixed.close()


def _span_distance(a, b, dx):
    """Largest norm of a state of a outside the span of b (b orthonormal in FP64)."""
    k = a.shape[0]
    A, B = a.reshape(k, -1), b.reshape(k, -1)
    C = (B.conj() @ A.T) * dx * dx          # C[j, n] = <b_j|a_n>
    R = A - C.T @ B
    return float(np.max(np.sqrt(np.sum(np.abs(R) ** 2, axis=1)) * dx))


@pytest.mark.parametrize("cap", [1, 2, 60])
def test_fp32_capped_eigensolve_is_finished_by_cholesky(cap):
    """FP32 canonical step with the eigensolve capped at `cap` sweeps (k = 300:
    the block Jacobi path): the states come out orthonormal to the FP32
    contraction accuracy, span the input's space, and the solve reports at most
    `cap` sweeps. Rotated states of a nearly diagonal overlap (propagated
    eigenstate-like inputs) agree with the uncapped canonical step's."""
    sx = sy = 64
    k = 300
    psi, dx = _states(sx, sy, k, seed=21, width2=None)
    c = capi.Context(sx, sy, dx, k, precision=capi.FP32)
    c.set_fp32_eig_sweeps(cap)
    c.upload(psi)
    before = c.download()
    c.orthonormalize()
    out = c.download()
    assert c.orthonormalization_counts() == (1, 0, 0)
    assert c.capped_eigensolves() == 1
    assert 1 <= c.last_sweeps <= cap
    orth = np.max(np.abs(_gram(out, dx) - np.eye(k)))
    ref = _gram_schmidt(before, dx)
    span = _span_distance(out, ref, dx)
    print(f"capped FP32 eigensolve, {cap} sweeps max ({c.last_sweeps} run): orthonormality {orth:.1e}, "
          f"span distance {span:.1e}")
    assert orth < 2e-5
    assert span < 1e-4
    # a second step on orthonormal states (overlap I plus FP32 noise, whose
    # eigenvectors are arbitrary): still orthonormal, same span
    c.orthonormalize()
    again = c.download()
    assert c.capped_eigensolves() == 2
    assert np.max(np.abs(_gram(again, dx) - np.eye(k))) < 2e-5
    assert _span_distance(again, ref, dx) < 1e-4


def test_fp32_capped_eigensolve_matches_canonical_on_a_near_diagonal_overlap():
    """States that are nearly orthogonal with distinct norms (the overlap of
    propagated, almost converged states: diagonal plus small couplings): the
    capped step's states equal the canonical ones up to phase, to the FP32
    accuracy, in the same (descending-norm) order."""
    sx = sy = 64
    k = 300
    basis, dx = _states(sx, sy, k, seed=5, width2=None)
    basis = _gram_schmidt(basis, dx)
    rng = np.random.default_rng(9)
    scale = np.exp(-0.05 * np.arange(k))                 # e^{-eps E_n}: distinct, well separated
    mix = np.eye(k) + 1e-3 * (rng.standard_normal((k, k)) + 1j * rng.standard_normal((k, k)))
    psi = (scale[:, None] * mix) @ basis.reshape(k, -1)
    psi = psi.reshape(basis.shape)
    outs = {}
    for cap in (0, 2):
        c = capi.Context(sx, sy, dx, k, precision=capi.FP32)
        c.set_fp32_eig_sweeps(cap)
        c.upload(psi)
        c.orthonormalize()
        outs[cap] = c.download()
        assert c.capped_eigensolves() == (1 if cap else 0)
    A, B = outs[0].reshape(k, -1), outs[2].reshape(k, -1)
    # canonical: ascending eigenvalue order; capped: descending
    X = (A[::-1].conj() @ B.T) * dx * dx
    d = np.abs(np.diag(X))
    print(f"near-diagonal overlap: min |<canonical_n|capped_n>| {d.min():.7f}")
    assert np.min(d) > 1 - 1e-4


def test_mixed_solve_with_capped_eigensolves_matches_fp64():
    """A whole FP32-form solve whose canonical steps cap the eigensolve at two
    sweeps (k = 260: the block Jacobi path) reaches the FP64 form's energies."""
    from itp2d_b200 import system
    common = dict(sx=64, sy=64, length=10.0, boundary=capi.PERIODIC, B=0.5, halforder=2, num_states=260,
                  wanted=60, eps=[0.05], timestep_test="abschange(1e-9)", final_test="abschange(1e-9)",
                  potential="harmonic(1)", max_steps=3000)
    psi, _ = _states(64, 64, 260, seed=8)
    ref = system.ITPSystem(system.Parameters(**common), init_states=psi)
    ref.run()
    mixed = system.ITPSystem(system.Parameters(precision=capi.FP32, fp32_switch=1e-7, fp32_canonical_every=3,
                                               fp32_between=capi.BETWEEN_CHOLESKY, fp32_eig_sweeps=2, **common),
                             init_states=psi)
    mixed.run()
    assert ref.finished and not ref.error_flag and mixed.finished and not mixed.error_flag
    capped = capi.lib().itp2d_fp32_capped_eigensolves(mixed.context_handle())
    print(f"mixed with capped eigensolves: {mixed.total_steps} iterations ({capped} capped); "
          f"FP64 form {ref.total_steps}")
    assert capped > 0
    E64, Em = ref.energies()[0][:60], mixed.energies()[0][:60]
    assert np.max(np.abs(E64 - Em)) < 1e-8
    ref.close()
    mixed.close()
