"""Whole imaginary-time solves through the native driver on the GPU: the
reference's integration tests (test_itp.cpp, test_hamiltonian.cpp) with fixed
seeds, whole-solve parity with the compiled reference, and the FP32 form."""
import math

import numpy as np
import pytest

from oracle import itp_oracle as O
from oracle import refkit as R

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def itp():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from itp2d_b200 import capi, system
    capi.lib()
    return system


def _solve(itp, **kw):
    p = itp.Parameters(**kw)
    s = itp.ITPSystem(p)
    s.run()
    assert not s.error_flag, s.last_error
    return s


def _ho_reference(n):
    out, E, deg = [], 1, 1
    for _ in range(n):
        out.append(E)
        if deg >= E:
            E, deg = E + 1, 1
        else:
            deg += 1
    return np.array(out, float)


TOL = 1e-4
HO = dict(sx=40, sy=40, length=12.0, num_states=14, wanted=8, eps=[1.0], potential="harmonic(1)",
          timestep_test=f"relstdev({TOL},{0.1 * TOL})", final_test=f"relstdev({TOL})", seed=12345)


def test_harmonic_oscillator(itp):
    """test_itp.cpp:56-91"""
    s = _solve(itp, **HO)
    E = s.energies()[0]
    assert np.max(np.abs(E[:8] - _ho_reference(8))) < TOL


def test_harmonic_oscillator_dirichlet(itp):
    """test_itp.cpp:93-128"""
    s = _solve(itp, **{**HO, "boundary": 1})
    assert np.max(np.abs(s.energies()[0][:8] - _ho_reference(8))) < TOL


def test_harmonic_oscillator_nonsquare(itp):
    """test_itp.cpp:130-165"""
    s = _solve(itp, **{**HO, "sy": 56})
    assert np.max(np.abs(s.energies()[0][:8] - _ho_reference(8))) < TOL


def test_particle_in_a_box(itp):
    """test_itp.cpp:167-198: zero potential, pi x pi Dirichlet box, E = (nx^2 + ny^2)/2."""
    s = _solve(itp, sx=40, sy=40, length=math.pi, boundary=1, num_states=16, wanted=12, eps=[0.5],
               potential="zero", timestep_test=f"relstdev({TOL},{0.1 * TOL})", final_test=f"relstdev({TOL})",
               seed=7)
    ref = sorted(0.5 * (x * x + y * y) for x in range(1, 16) for y in range(1, 16))[:12]
    assert np.max(np.abs(s.energies()[0][:12] - np.array(ref))) < TOL


def test_harmonic_oscillator_magnetic(itp):
    """test_itp.cpp:266-300: B = 10 periodic, Fock-Darwin energies within 1e-3."""
    tol = 1e-3
    s = _solve(itp, sx=40, sy=40, length=7.0, num_states=14, wanted=8, eps=[1.0], potential="harmonic(1)", B=10.0,
               timestep_test=f"relstdev({tol},{0.1 * tol})", final_test=f"relstdev({tol})", seed=3)
    assert np.max(np.abs(s.energies()[0][:8] - O.fock_darwin_spectrum(8, 10.0))) < tol


@pytest.mark.parametrize("case", ["harmonic", "harmonic_magnetic", "box"])
def test_hamiltonian_ground_state_stable(itp, case):
    """test_hamiltonian.cpp:40-106: H applied to the converged ground state
    (divided by its energy) changes it by less than 5e-3 rms."""
    from itp2d_b200 import capi
    kw = dict(sx=40, sy=40, num_states=1, wanted=1, eps=[1.0], halforder=5, seed=1)
    if case == "box":
        kw.update(length=math.pi, boundary=1, potential="zero")
    else:
        kw.update(length=10.0, potential="harmonic(1)", B=1.0 if case == "harmonic_magnetic" else 0.0)
    s = _solve(itp, **kw)
    E0 = s.energies()[0][0]
    gs = s.states()[0]
    g = O.Grid.from_length(40, 40, kw["length"])
    V = None if case == "box" else O.harmonic(g)
    c = capi.Context(40, 40, g.dx, 1, kw.get("boundary", 0), kw.get("B", 0.0), 1)
    c.set_potential(V)
    c.upload(gs[None])
    t = gs.copy()
    for _ in range(3):
        c.apply_hamiltonian()
        t = c.download()[0] / E0
        c.upload(t[None])
        assert math.sqrt(np.mean(np.abs(t - gs) ** 2)) < 5e-3


def test_particle_in_a_box_magnetic(itp):
    """test_itp.cpp:412-443: Dirichlet box 64x64, L = pi, B = 1, no potential;
    the lowest 8 converged energies equal the reference's known-good values
    (tests/golden/magnetic_box_energies.json) within twice the test tolerance."""
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "magnetic_box_energies.json")) as f:
        ref = json.load(f)
    s = _solve(itp, sx=64, sy=64, length=math.pi, boundary=1, B=1.0, num_states=16, wanted=8,
               eps=[0.3], potential="zero", timestep_test="abschange(1e-3)", final_test="onestep",
               max_steps=2000)
    E = s.energies()[0]
    assert np.max(np.abs(E[:8] - np.array(ref["energies"]))) < 2e-3


def test_dirichlet_magnetic_whole_solve_matches_reference(itp):
    """Dirichlet boundaries with a magnetic field through the reference
    ITPSystem (compiled oracle) and the GPU driver, same initial states."""
    if not R.available():
        pytest.skip("oracle/_ref not built")
    g = O.Grid.from_length(32, 32, 10.0)
    psi = O.gaussian_states(g, 8, 17)
    kw = dict(num_states=8, wanted=5, eps_values=[0.1], eps_divisor=2.0, timestep_test="abschange(1e-11)",
              final_test="abschange(1e-11)", max_steps=600)
    ref = R.RefSystem(32, 32, 10.0, 1, 1.0, 2, potential="harmonic(1)", init_states=psi, threads=4, **kw)
    while not ref.finished:
        ref.step()
    assert not ref.error_flag
    Er, _ = ref.energies()
    s = itp.ITPSystem(itp.Parameters(sx=32, sy=32, length=10.0, boundary=1, B=1.0, halforder=2, num_states=8,
                                     wanted=5, eps=[0.1], eps_divisor=2.0, timestep_test="abschange(1e-11)",
                                     final_test="abschange(1e-11)", max_steps=600, potential="harmonic(1)"),
                      init_states=psi)
    s.run()
    assert not s.error_flag, s.last_error
    assert np.max(np.abs(s.energies()[0][:5] - Er[:5])) < 1e-9


def test_whole_solve_matches_reference(itp):
    """Same parameters and initial states through the reference ITPSystem
    (compiled oracle) and the GPU driver: sorted converged energies agree."""
    if not R.available():
        pytest.skip("oracle/_ref not built")
    g = O.Grid.from_length(32, 32, 12.0)
    psi = O.gaussian_states(g, 10, 99)
    kw = dict(num_states=10, wanted=6, eps_values=[0.2], eps_divisor=2.0, timestep_test="abschange(1e-11)",
              final_test="abschange(1e-11)", max_steps=400)
    ref = R.RefSystem(32, 32, 12.0, 0, 0.5, 2, potential="harmonic(1)", init_states=psi, threads=4, **kw)
    while not ref.finished:
        ref.step()
    assert not ref.error_flag
    Er, _ = ref.energies()
    s = itp.ITPSystem(itp.Parameters(sx=32, sy=32, length=12.0, B=0.5, halforder=2, num_states=10, wanted=6,
                                     eps=[0.2], eps_divisor=2.0, timestep_test="abschange(1e-11)",
                                     final_test="abschange(1e-11)", max_steps=400, potential="harmonic(1)"),
                      init_states=psi)
    s.run()
    assert not s.error_flag, s.last_error
    Eg = s.energies()[0]
    assert np.max(np.abs(Eg[:6] - Er[:6])) < 1e-9
    assert abs(s.eps - ref.eps) < 1e-15


def test_fp32_form_refines_to_fp64(itp):
    """FP32 sweeps until the energies stall at the FP32 floor, then FP64
    refinement: the converged energies equal the plain FP64 solve's."""
    kw = dict(sx=48, sy=48, length=12.0, B=1.0, halforder=2, num_states=12, wanted=6, eps=[0.1],
              potential="harmonic(1)", timestep_test="abschange(1e-10)", final_test="abschange(1e-10)",
              max_steps=600, seed=5)
    s64 = _solve(itp, **kw)
    s32 = _solve(itp, **kw, precision=1, fp32_switch=1e-6)
    assert not s32.in_fp32
    E64, E32 = s64.energies()[0], s32.energies()[0]
    assert np.max(np.abs(E32[:6] - E64[:6])) < 1e-9
    assert np.max(np.abs(E64[:6] - O.fock_darwin_spectrum(6, 1.0))) < 1e-3


@pytest.mark.parametrize("span", [1, 3])
def test_fp32_switch_rule_spans_reach_fp64_energies(itp, span):
    """Either switch rule (consecutive iterations with the stall test, or the
    change over three iterations with the floor test) ends the FP32 phase and
    the FP64 refinement reaches the plain FP64 energies."""
    kw = dict(sx=48, sy=48, length=12.0, B=1.0, halforder=2, num_states=12, wanted=6, eps=[0.1],
              potential="harmonic(1)", timestep_test="abschange(1e-10)", final_test="abschange(1e-10)",
              max_steps=600, seed=5)
    s64 = _solve(itp, **kw)
    s32 = _solve(itp, **kw, precision=1, fp32_switch=1e-7, fp32_switch_span=span)
    assert s32.finished and not s32.in_fp32
    assert np.max(np.abs(s32.energies()[0][:6] - s64.energies()[0][:6])) < 1e-9


def test_recovery_from_dependent_states(itp):
    """A rank-deficient start makes the overlap singular; with recover the
    driver shrinks eps and restarts from noise (itpsystem.cpp:264-281)."""
    g = O.Grid.from_length(24, 24, 12.0)
    psi = O.gaussian_states(g, 6, 1)
    psi[5] = 0.0
    p = itp.Parameters(sx=24, sy=24, length=12.0, num_states=6, wanted=3, eps=[0.5], eps_divisor=2.0,
                       potential="harmonic(1)", timestep_test="abschange(1e-8)", final_test="abschange(1e-8)",
                       max_steps=300, recover=True)
    s = itp.ITPSystem(p, init_states=psi)
    s.step()
    assert abs(s.eps - 0.25) < 1e-15  # shrunk once by the divisor
    s.run()
    assert not s.error_flag
    assert np.max(np.abs(s.energies()[0][:3] - np.array([1, 2, 2]))) < 1e-3
    p.recover = False
    s2 = itp.ITPSystem(p, init_states=psi)
    s2.step()
    assert s2.error_flag and s2.finished
