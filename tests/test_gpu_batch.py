"""The batched form (itp2d_batch_* in include/itp2d_gpu.h and itp2d_host.h)
on the GPU: many independent solves of uneven grid size and state count
stepped together, with every instance's overlap eigenproblem in one launch.

* the batched eigensolver reproduces the single-instance orthonormalisation
  (same subspace, orthonormal, ascending-eigenvalue order) for uneven k;
* a batch of instances drawn like the batched configuration (N in
  {64, 96, 128, 160, 192}, L = 12, k in 16..128, omega^2 r^2 / 2 plus
  Gaussian bumps, B in [0, 2], 4th-order split) gives every instance the
  energies of the same solve run alone, within 1e-9 (both solves stop at
  abschange(1e-10) on the lower half of the states);
* an instance that fails (rank-deficient states) reports its status without
  disturbing the others.
"""
import numpy as np
import pytest

from oracle import itp_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from itp2d_b200 import capi, system
    capi.lib()
    return capi, system


def _batch_ortho(capi, ctxs):
    import ctypes as C
    L = capi.lib()
    n = len(ctxs)
    L.itp2d_batch_orthonormalize.argtypes = [C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_int),
                                             C.POINTER(C.c_int), C.POINTER(C.c_double)]
    arr = (C.c_void_p * n)(*[c.h.value for c in ctxs])
    st, bi, bv = (C.c_int * n)(), (C.c_int * n)(), (C.c_double * n)()
    assert L.itp2d_batch_orthonormalize(n, arr, st, bi, bv) == capi.OK
    return list(st), list(bi), list(bv)


def test_batched_orthonormalize_matches_single(mods):
    capi, _ = mods
    shapes = [(32, 24, 5), (48, 48, 33), (40, 32, 64), (64, 64, 128), (24, 24, 2)]
    ctxs, refs = [], []
    for i, (sx, sy, k) in enumerate(shapes):
        g = O.Grid.from_length(sx, sy, 12.0)
        V = O.harmonic(g)
        psi = O.MultiProductSplit(g, V, O.PERIODIC, 0.0, 1, 0.3).apply(O.gaussian_states(g, k, 10 + i))
        c = capi.Context(sx, sy, g.dx, k)
        c.set_potential(V)
        c.upload(psi)
        ctxs.append(c)
        ref, lam = O.orthonormalize(g, psi)
        refs.append((g, k, ref, lam))
    st, _, _ = _batch_ortho(capi, ctxs)
    assert st == [0] * len(ctxs)
    for c, (g, k, ref, lam) in zip(ctxs, refs):
        out = c.download()
        bound = max(64 * np.finfo(float).eps, 4 * O.how_orthonormal(g, ref))
        assert O.how_orthonormal(g, out) < bound
        assert 1 - O.subspace_cosines(g, out, ref).min() < max(1e-10, 2 * bound)
        # output n belongs to the n-th smallest overlap eigenvalue (phases free)
        ov = np.abs(np.sum(np.conj(ref) * out, axis=(1, 2)) * g.dx * g.dx)
        gaps = np.diff(lam) / lam[1:]
        isolated = [n for n in range(k) if (n == 0 or gaps[n - 1] > 1e-6) and (n == k - 1 or gaps[n] > 1e-6)]
        assert np.all(ov[isolated] > 1 - 1e-8)
        assert c.last_sweeps > 0


def test_batched_failure_is_per_instance(mods):
    capi, _ = mods
    g = O.Grid(16, 16, 1.0)
    good = capi.Context(16, 16, 1.0, 4)
    bad = capi.Context(16, 16, 1.0, 4)
    psi = O.gaussian_states(g, 4, 3)
    good.upload(psi)
    broken = psi.copy()
    broken[2] = 0.0
    bad.upload(broken)
    st, bi, _ = _batch_ortho(capi, [good, bad])
    assert st[0] == capi.OK and st[1] == capi.E_NONPOSITIVE_EIGENVALUE and bi[1] == 0
    assert np.array_equal(bad.download(), broken)
    assert O.how_orthonormal(g, good.download()) < 64 * np.finfo(float).eps


def instances(system, capi, count, seed, precision):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        N = int(rng.choice([64, 96, 128, 160, 192]))
        k = int(rng.integers(16, 129))
        om = float(rng.uniform(0.5, 2.0))
        g = O.Grid.from_length(N, N, 12.0)
        bumps = O.bumpy_potential(g, int(rng.integers(0, 51)), int(rng.integers(1 << 30)), amp=(0.5, 1.5),
                                  width=float(rng.uniform(0.1, 0.3)), extent=4.0)
        p = system.Parameters(sx=N, sy=N, length=12.0, B=float(rng.uniform(0, 2)), halforder=2, num_states=k,
                              wanted=k // 2, eps=[0.05], timestep_test="abschange(1e-10)",
                              final_test="abschange(1e-10)", max_steps=4000, potential=f"harmonic({om * om})",
                              precision=precision, fp32_switch=1e-7 if precision == capi.FP32 else 0.0)
        out.append((p, bumps, O.gaussian_states(g, k, 500 + i)))
    return out


@pytest.mark.parametrize("form", ["fp64", "mixed"])
def test_batch_matches_instances_alone(mods, form):
    capi, system = mods
    prec = capi.FP64 if form == "fp64" else capi.FP32
    inst = instances(system, capi, 32 if form == "fp64" else 12, 4 if form == "fp64" else 5, prec)
    with system.Batch([p for p, _, _ in inst], [b for _, b, _ in inst], [s for _, _, s in inst]) as b:
        b.run()
        assert b.finished
        res = [b.result(i) for i in range(len(inst))]
    for (p, bumps, psi), r in zip(inst, res):
        s = system.ITPSystem(p, extra_potential=bumps, init_states=psi)
        s.run()
        assert s.finished and not s.error_flag and not r["error_flag"]
        E = s.energies()[0]
        n = p.wanted
        assert np.max(np.abs(E[:n] - r["E"][:n])) < 1e-9, (p.sx, p.num_states)
        assert r["converged"] >= n
        s.close()
