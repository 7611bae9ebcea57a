"""Tensor-core contractions of the FP32 form (tcgen05, split-BF16 operands,
FP32 accumulation over bounded grid chunks) against FP64 products of the same
FP32 states: the overlap S = Psi^H Psi dx^2 of stateset.cpp:146-154 and the
rotation Psi W of stateset.cpp:214-228."""
import numpy as np
import pytest

from itp2d_b200 import capi

pytestmark = pytest.mark.gpu

# Norm-relative error bound of the split-BF16 products with FP32 accumulation
# over grid chunks of at most 2048 points: |S_ij - S_ij(FP64)| <= TOL_S
# sqrt(S_ii S_jj). Each MMA rounds the FP32 accumulator once; the error grows
# about linearly with the chunk length (about 1e-5 at 2048 points).
TOL_S = 2e-5
# Orthonormality of the rotated FP32 states: |<psi_i|psi_j> - delta_ij| <= TOL_ORTHO.
TOL_ORTHO = 2e-5


def _ctx(sx, sy, k, seed, L=10.0):
    dx = L / sx
    c = capi.Context(sx, sy, dx, k, precision=capi.FP32)
    rng = np.random.default_rng(seed)
    x = (np.arange(sx) - sx / 2) * dx
    y = (np.arange(sy) - sy / 2) * dx
    env = np.exp(-0.5 * (y[:, None] ** 2 + x[None, :] ** 2) / 4.0)
    psi = (rng.standard_normal((k, sy, sx)) + 1j * rng.standard_normal((k, sy, sx))) * env
    c.upload(psi)
    return c, dx


def _exact_overlap(c, dx):
    psi = c.download().reshape(c.k, -1)  # the FP32 values, widened exactly
    return (psi.conj() @ psi.T) * dx * dx


def _rel(S, ref):
    d = np.sqrt(np.abs(np.diag(ref)))
    return np.max(np.abs(S - ref) / np.outer(d, d))


@pytest.mark.parametrize("sx,sy,k", [(32, 32, 5), (64, 48, 130), (128, 128, 300), (256, 256, 64)])
def test_overlap_tensor_cores(sx, sy, k):
    c, dx = _ctx(sx, sy, k, seed=sx + k)
    ref = _exact_overlap(c, dx)
    S_tc = c.overlap_matrix()
    c.set_contraction(capi.CONTRACT_FP64)
    S_64 = c.overlap_matrix()
    assert _rel(S_64, ref) < 1e-12
    err = _rel(S_tc, ref)
    print(f"overlap {sx}x{sy} k={k}: split-BF16 norm-relative error {err:.2e}")
    assert err < TOL_S
    assert np.array_equal(S_tc, S_tc.conj().T)
    assert np.all(np.diag(S_tc).imag == 0)


def test_overlap_odd_grid_uses_fp64():
    # an odd number of grid points leaves the tensor-core path (paired loads)
    c, dx = _ctx(35, 45, 20, seed=3)
    assert _rel(c.overlap_matrix(), _exact_overlap(c, dx)) < 1e-12


@pytest.mark.parametrize("sx,sy,k", [(64, 64, 40), (128, 96, 200)])
def test_rotation_tensor_cores(sx, sy, k):
    c, dx = _ctx(sx, sy, k, seed=7 * k)
    psi0 = c.download().reshape(k, -1)
    c.orthonormalize()
    out = c.download().reshape(k, -1)
    O = (out.conj() @ out.T) * dx * dx
    dev = np.max(np.abs(O - np.eye(k)))
    print(f"rotation {sx}x{sy} k={k}: orthonormality {dev:.2e}")
    assert dev < TOL_ORTHO
    # same span as the input states: the projection of psi0 on the new set
    # reproduces psi0
    coef = (out.conj() @ psi0.T) * dx * dx
    resid = psi0 - coef.T @ out
    rel = np.linalg.norm(resid, axis=1) / np.linalg.norm(psi0, axis=1)
    assert np.max(rel) < 1e-4
    # the same states as the FP64 engine (distinct overlap eigenvalues here)
    c2, _ = _ctx(sx, sy, k, seed=7 * k)
    c2.set_contraction(capi.CONTRACT_FP64)
    c2.orthonormalize()
    ref = c2.download().reshape(k, -1)
    phase = np.sum(ref.conj() * out, axis=1)
    phase /= np.abs(phase)
    diff = np.linalg.norm(out - phase[:, None] * ref, axis=1) / np.linalg.norm(ref, axis=1)
    print(f"rotation {sx}x{sy} k={k}: max state difference to FP64 engine {np.max(diff):.2e}")
    assert np.median(diff) < 1e-4


# k = 5 and 130: ragged state tiles; 48 x 40 and 56 x 24: a grid that is not
# a multiple of the 128-point tile; 128 x 128, k = 300: several tile pairs
@pytest.mark.parametrize("sx,sy,k", [(32, 32, 5), (48, 40, 130), (56, 24, 64), (128, 128, 300)])
def test_presplit_contractions_match_staged(sx, sy, k):
    """The tensor-core overlap and rotation from operands split once per call
    (BF16 planes in global memory, copied block by block by cp.async.bulk)
    issue the same MMAs in the same order as the kernels that split inside
    each CTA: the overlap, the canonical orthonormalisation and a Cholesky
    step (triangular rotation) are bit-identical."""
    out = {}
    for engine in (capi.CONTRACT_AUTO, capi.CONTRACT_TC_STAGED):
        c, dx = _ctx(sx, sy, k, seed=sx + sy + k)
        c.set_contraction(engine)
        S = c.overlap_matrix()
        c.orthonormalize()
        canon = c.download()
        c.orthonormalize(capi.ORTHO_CHOLESKY)
        out[engine] = (S, canon, c.download())
        c.close()
    for a, b in zip(out[capi.CONTRACT_AUTO], out[capi.CONTRACT_TC_STAGED]):
        assert np.array_equal(a, b)
    # and the pre-split overlap against FP64 products of the same FP32 states
    c, dx = _ctx(sx, sy, k, seed=sx + sy + k)
    assert _rel(c.overlap_matrix(), _exact_overlap(c, dx)) < TOL_S


@pytest.mark.parametrize("sx,k", [(128, 320), (128, 1024)])
def test_fp32_block_jacobi_canonical(sx, k):
    """k >= 256: the FP32 form solves the overlap eigenproblem by block Jacobi
    in single precision (stopping at a rotation tangent of 1e-3). The result is
    the canonical orthonormalisation Psi' = Psi V L^{-1/2} of stateset.cpp:136-232
    up to the FP32 accuracy: with M = Psi'^H Psi dx^2 = L^{1/2} V^H, M M^H is
    diagonal and its diagonal holds the eigenvalues of S. These checks do not
    depend on the gaps between eigenvalues (the eigenvectors themselves do).
    k = 1024 has more block products per round than the phase-2 CTAs take in
    eight turns, so the phase-1 CTAs take products as well."""
    sy = sx
    c, dx = _ctx(sx, sy, k, seed=11 + k)
    psi0 = c.download().reshape(k, -1)
    S = (psi0.conj() @ psi0.T) * dx * dx
    S0 = np.abs(S - np.diag(np.diag(S))) / np.sqrt(np.outer(np.diag(S).real, np.diag(S).real))
    c.orthonormalize()
    out = c.download().reshape(k, -1)
    O = (out.conj() @ out.T) * dx * dx
    dev = np.max(np.abs(O - np.eye(k)))
    M = (out.conj() @ psi0.T) * dx * dx
    MM = M @ M.conj().T
    lam = np.diag(MM).real
    off = np.max(np.abs(MM - np.diag(lam)) / np.sqrt(np.outer(lam, lam)))
    ev = np.linalg.eigvalsh(S)
    lam_err = np.max(np.abs(lam - ev) / ev)
    # the overlap's split-BF16 error (TOL_S relative to the diagonal) reaches
    # the output's Gram matrix scaled by 1 / lambda_min through W = V L^{-1/2}
    tol_dev = 2 * TOL_S * np.max(np.diag(S).real) / ev.min()
    print(f"FP32 block Jacobi k={k}: orthonormality {dev:.2e} (bound {tol_dev:.1e}), off-diagonal "
          f"{np.max(S0):.1e} -> {off:.2e}, eigenvalues {lam_err:.2e}")
    assert dev < tol_dev
    assert np.all(np.diff(lam) > -1e-4 * lam[1:])  # ascending, as the sort leaves them
    assert off < 1e-4
    assert lam_err < 1e-4


def test_tensor_core_solve_matches_fp64_engine():
    """The mixed form (FP32 sweeps, FP64 refinement) reaches the same
    energies with tensor-core contractions as with FP64 contractions."""
    from itp2d_b200.system import ITPSystem, Parameters

    kw = dict(sx=48, sy=48, length=12.0, B=1.0, halforder=2, num_states=12, wanted=6, eps=[0.1],
              potential="harmonic(1)", timestep_test="abschange(1e-10)", final_test="abschange(1e-10)",
              max_steps=600, seed=5, precision=capi.FP32, fp32_switch=1e-6)
    res = {}
    for engine in (capi.CONTRACT_AUTO, capi.CONTRACT_FP64):
        s = ITPSystem(Parameters(**kw))
        assert capi.lib().itp2d_set_contraction(s.context_handle(), engine) == capi.OK
        s.run()
        assert not s.error_flag, s.last_error
        assert not s.in_fp32
        print(f"engine {engine}: {s.total_steps} steps")
        res[engine] = s.energies()[0][:6]
    assert np.max(np.abs(res[capi.CONTRACT_AUTO] - res[capi.CONTRACT_FP64])) < 1e-9


def _near_orthonormal(sx, sy, k, seed, delta, L=10.0):
    """FP32 context holding k states that are orthonormal up to perturbations
    of relative size delta (the situation after one propagation step), with
    the FP64 states they came from."""
    from oracle import itp_oracle as O
    g = O.Grid(sx, sy, L / sx)
    psi = O.gaussian_states(g, k, seed)
    q, _ = np.linalg.qr(psi.reshape(k, -1).T)
    base = (q.T / g.dx).reshape(k, sy, sx)
    rng = np.random.default_rng(seed + 1)
    pert = rng.standard_normal((k, sy, sx)) + 1j * rng.standard_normal((k, sy, sx))
    pert *= delta / (np.sqrt(np.sum(np.abs(pert) ** 2, axis=(1, 2)))[:, None, None] * g.dx)
    scale = np.exp(-6.0 * np.arange(k) / k)[:, None, None]  # graded norms, like exp(-eps E)
    psi = (base + pert) * scale
    c = capi.Context(sx, sy, g.dx, k, precision=capi.FP32)
    c.upload(psi)
    return c, g, psi


@pytest.mark.parametrize("k,delta", [(64, 1e-3), (300, 3e-4)])
def test_lowdin_step_orthonormalises(k, delta):
    """Between canonical steps the FP32 form orthonormalises with
    W = D (I + E)^{-1/2} cut after E^2: the states come out orthonormal to the
    FP32 contraction accuracy, span the input's subspace, and each output state
    stays within O(delta) of its (normalised) input state: no reordering."""
    from oracle import itp_oracle as O
    c, g, psi = _near_orthonormal(128, 128, k, 7, delta)
    c.set_fp32_orthonormalization(4)
    c.orthonormalize()
    assert c.orthonormalization_counts() == (0, 1, 0)
    out = c.download()
    assert O.how_orthonormal(g, out) < TOL_ORTHO
    # every output state lies in the input's span: its residual outside an
    # FP64 orthonormal basis of that span is at the FP32 / split-BF16 level
    ref, _ = O.orthonormalize(g, psi)
    R = ref.reshape(k, -1)
    X = out.reshape(k, -1)
    P = (np.conj(R) @ X.T) * g.dx * g.dx
    res = X - P.T @ R
    assert np.max(np.sqrt(np.sum(np.abs(res) ** 2, axis=1)) * g.dx) < 5 * TOL_ORTHO
    nrm = np.sqrt(np.sum(np.abs(psi) ** 2, axis=(1, 2))) * g.dx
    move = np.sqrt(np.sum(np.abs(out - psi / nrm[:, None, None]) ** 2, axis=(1, 2))) * g.dx
    assert np.max(move) < 10 * delta


def test_lowdin_guard_falls_back_to_canonical():
    """A set far from orthonormal (random states) is orthonormalised
    canonically even between canonical steps; every canonical_every-th call is
    canonical; FP64 states are always canonical."""
    c, dx = _ctx(64, 64, 40, seed=5)
    c.set_fp32_orthonormalization(3)
    c.orthonormalize()  # random states: the guard refuses the Lowdin step
    assert c.orthonormalization_counts() == (1, 0, 0)
    c.orthonormalize()  # now near orthonormal: Lowdin
    c.orthonormalize()  # Lowdin (second since the canonical one)
    c.orthonormalize()  # third: canonical by the schedule
    assert c.orthonormalization_counts() == (2, 2, 0)
    c.set_precision(capi.FP64)
    c.orthonormalize()
    c.orthonormalize()
    assert c.orthonormalization_counts() == (4, 2, 0)


def test_bounded_wait_gives_up_and_device_stays_usable():
    """The tensor-core kernels' mbarrier waits are bounded: a CTA set up like
    them that waits on a barrier nothing completes returns ITP2D_E_TIMEOUT
    after about a second, having freed its tensor memory; the tensor-core
    overlap then runs normally on the same device."""
    import time
    L = capi.lib()
    L.itp2d_tc_wait_probe.argtypes = []
    t0 = time.perf_counter()
    assert L.itp2d_tc_wait_probe() == capi.E_TIMEOUT
    waited = time.perf_counter() - t0
    print(f"wait gave up after {waited:.2f} s")
    # the wait is bounded by the global timer (1 s), not by a poll count
    assert 0.9 < waited < 10.0
    c, dx = _ctx(64, 64, 20, seed=9)
    assert _rel(c.overlap_matrix(), _exact_overlap(c, dx)) < TOL_S
