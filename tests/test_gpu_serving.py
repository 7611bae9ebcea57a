"""The serving loop (itp2d_server_* in include/itp2d_host.h) on the GPU.

A request is one whole solve (the reference's ITPSystem run to is_finished(),
itpsystem.cpp:407-470). The server runs several at once on their own streams,
admitted by device footprint. The tests check that

* each request's energies are the same alone (one solve at a time) and in the
  mix (several running at once): a request's kernels are its own, so the
  bound is the one the benchmark counts converged states with, 1e-9;
* the mix really overlapped (two or more solves running at once) and never
  held more than the memory budget;
* a request larger than the whole budget is refused.
"""
import numpy as np
import pytest

from oracle import itp_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def system():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from itp2d_b200 import system as S
    return S


def requests(system, count, seed):
    """Requests drawn like the serving configuration, at small sizes: grid
    N in {32, 48, 64} (L = 12), k in {8, 12, 16}, B ~ U[0, 2], harmonic
    confinement with omega^2 ~ U[0.5, 2] plus 0-5 Gaussian bumps, 4th-order
    split, FP64 or mixed form, abschange(1e-9)."""
    from itp2d_b200 import capi
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        N = int(rng.choice([32, 48, 64]))
        k = int(rng.choice([8, 12, 16]))
        B = float(rng.uniform(0, 2))
        w2 = float(rng.uniform(0.5, 2.0))
        g = O.Grid.from_length(N, N, 12.0)
        bumps = O.bumpy_potential(g, int(rng.integers(0, 6)), int(rng.integers(1 << 30)), amp=(0.5, 1.5),
                                  width=0.2, extent=4.0)
        mixed = bool(i % 2)
        p = system.Parameters(sx=N, sy=N, length=12.0, B=B, halforder=2, num_states=k, wanted=k // 2,
                              eps=[0.05], timestep_test="abschange(1e-9)", final_test="abschange(1e-9)",
                              max_steps=3000, potential=f"harmonic({w2})", seed=1000 + i,
                              precision=capi.FP32 if mixed else capi.FP64, fp32_switch=1e-7 if mixed else 0.0)
        out.append((p, bumps, O.gaussian_states(g, k, 77 + i)))
    return out


def run_all(system, reqs, max_active, budget):
    with system.Server(max_active, budget) as srv:
        ids = [srv.submit(p, bumps, psi) for p, bumps, psi in reqs]
        res = [srv.wait(i, timeout=600) for i in ids]
        stats = srv.stats()
    return res, stats


def test_alone_and_in_the_mix_agree(system):
    reqs = requests(system, 8, 1)
    alone, s1 = run_all(system, reqs, 1, 64e9)
    mix, s2 = run_all(system, reqs, 4, 64e9)
    assert s1["peak_running"] == 1 and s2["peak_running"] >= 2
    assert s2["overlap_seconds"] > 0
    for (p, _, _), a, m in zip(reqs, alone, mix):
        assert a["status"] == 0 and m["status"] == 0 and not a["error_flag"] and not m["error_flag"]
        n = p.wanted
        assert np.max(np.abs(a["E"][:n] - m["E"][:n])) <= 1e-9
        assert a["converged"] >= n and m["converged"] >= n
        assert m["t_submit"] <= m["t_start"] <= m["t_finish"]


def test_admission_by_footprint(system):
    from itp2d_b200 import capi
    reqs = requests(system, 6, 2)
    fps = [system.footprint(p) for p, _, _ in reqs]
    budget = 2.2 * max(fps)  # room for two of the largest at a time
    res, st = run_all(system, reqs, 6, budget)
    assert st["peak_bytes_in_use"] <= budget and st["completed"] == len(reqs)
    assert all(r["status"] == 0 for r in res)
    with system.Server(2, 0.5 * min(fps)) as srv:
        with pytest.raises(capi.ITP2DError) as e:
            srv.submit(reqs[0][0], reqs[0][1], reqs[0][2])
        assert e.value.status == capi.E_OOM
