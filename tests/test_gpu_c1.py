"""Configuration C1 on the GPU: V = r^2/2, B = 0, Dirichlet box of side 12 on
128 x 128 (DST-II/III lines), k = 64, 2nd-order split at eps = 0.02,
abschange(1e-10) as time-step and final test (the deviation the deviation
tests read has an FP64 cancellation floor of about 5e-5 on this grid),
the 55 states of the levels E = 1..10 wanted (the 64 states end inside the
11-fold level E = 11).

Checked against the reference's own whole solve of the same initial states
(golden/solve_harmonic_dirichlet_128_k64.json, written by
golden/make_solve_golden.py --workload c1) and against the analytic spectrum
E = n_x + n_y + 1 of test_itp.cpp:56-91 within that test's 1e-4 (the box and
the grid move the upper levels by up to about 5e-5).
"""
import importlib.util
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "solve_harmonic_dirichlet_128_k64.json")


def _golden_module():
    spec = importlib.util.spec_from_file_location("make_solve_golden",
                                                  os.path.join(HERE, "golden", "make_solve_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def analytic(n):
    out, E = [], 1
    while len(out) < n:
        out += [float(E)] * E
        E += 1
    return np.array(out[:n])


@pytest.mark.parametrize("form", ["fp64", "mixed", "fp64_device"])
def test_c1_solve(form):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from itp2d_b200 import capi, system
    g = _golden_module()
    w = g.C1
    ref = json.load(open(GOLDEN))
    p = system.Parameters(sx=w["sx"], sy=w["sy"], length=w["length"], boundary=capi.DIRICHLET, B=w["B"],
                          halforder=w["halforder"], num_states=w["num_states"], wanted=w["wanted"], eps=[w["eps"]],
                          eps_divisor=w["eps_divisor"], timestep_test=w["timestep_test"],
                          final_test=w["final_test"], max_steps=20000, potential=w["potential"],
                          precision=capi.FP32 if form == "mixed" else capi.FP64,
                          fp32_switch=1e-7 if form == "mixed" else 0.0)
    s = system.ITPSystem(p, init_states=g.c1_states())
    if form == "fp64_device":
        # iterations on the device until the time-step test holds (one CUDA
        # graph with a conditional loop), the final test on the host
        s.run_device()
        assert s.device_iterations == s.total_steps
    else:
        s.run()
    assert s.finished and not s.error_flag, s.last_error
    E = s.energies()[0]
    n = w["wanted"]
    Eref = np.array(ref["energies"])
    d_ref = np.max(np.abs(E[:n] - Eref[:n]))
    d_ana = np.max(np.abs(E[:n] - analytic(n)))
    print(f"C1 {form}: {s.total_steps} iterations (reference {ref['iterations']}), final eps {s.eps:g}, "
          f"max |E - E_ref| {d_ref:.2e}, max |E - analytic| {d_ana:.2e}")
    assert d_ref < 1e-9
    assert d_ana < 1e-4
    s.close()
