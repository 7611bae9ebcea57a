"""Whole solves on the GPU against the reference's own solve of the same
workload: the magnetic dot (V = r^2/2, B = 1, periodic 256 x 256, L = 14,
k = 500, 4th-order split, eps = 0.05, abschange(1e-9) on the 250 lowest states,
the benchmark's seeded initial states). The fixture
golden/solve_magnetic_dot_256_k500.json holds the reference ITPSystem's sorted
converged energies (itpsystem.cpp:407-470, compiled from its sources, HighMem
orthonormalisation), written by golden/make_solve_golden.py.

Both GPU forms must reproduce the reference's 250 wanted energies: the plain
FP64 form and the mixed form (FP32 sweeps, FP64 refinement). Each energy
passed abschange(1e-9) in both runs, so two solves that stop one iteration
apart can differ by up to about 1e-9 besides rounding; the bound is 2e-9.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "solve_magnetic_dot_256_k500.json")


@pytest.fixture(scope="module")
def setup():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    import bench
    bench.WORKLOAD = bench.WORKLOADS["dot"]
    psi, _ = bench.initial_states(pinned=False)
    ref = json.load(open(GOLDEN))
    return bench, psi, ref


@pytest.mark.parametrize("form", ["fp64", "mixed", "fp64_device"])
def test_solve_matches_reference_solve(setup, form):
    """fp64_device: the same FP64 solve with its iterations in a device-side
    loop (itp2d_system_run_device), the time-step test evaluated on the GPU."""
    bench, psi, ref = setup
    from itp2d_b200 import system
    w = bench.WORKLOAD
    s = system.ITPSystem(bench.params("fp64" if form == "fp64_device" else form), init_states=psi)
    if form == "fp64_device":
        s.run_device()
        assert s.device_iterations == s.total_steps
    else:
        s.run()
    assert s.finished and not s.error_flag, s.last_error
    E = s.energies()[0]
    Eref = np.array(ref["energies"])
    n = w["wanted"]
    dE = np.abs(E[:n] - Eref[:n])
    print(f"{form}: {s.total_steps} iterations (reference {ref['iterations']}), {s.num_converged} converged "
          f"(reference {ref['converged']}), max |dE| over the {n} wanted states {dE.max():.3e}")
    assert dE.max() < 2e-9
    if form.startswith("fp64"):
        # the same algorithm from the same states: the solve length can differ
        # only where an energy change sits at the 1e-9 threshold
        assert abs(s.total_steps - ref["iterations"]) <= 1
        assert abs(s.num_converged - ref["converged"]) <= 10
    s.close()
