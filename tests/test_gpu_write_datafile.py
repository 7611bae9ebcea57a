"""The datafile of a whole solve (itp2d_system_write_datafile, the reference
ITPSystem's --save final states: itpsystem.cpp:69-116, 390-402, 513-531)
read back with the library's reader, and a --copy-states restart from it
(StateSet::init_from_datafile, stateset.cpp:86-109)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def itp():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from itp2d_b200 import capi, system
    capi.lib()
    return system


TOL = 1e-4
HO = dict(sx=40, sy=40, length=12.0, num_states=14, wanted=8, eps=[1.0], potential="harmonic(1)",
          timestep_test=f"relstdev({TOL},{0.1 * TOL})", final_test=f"relstdev({TOL})", seed=12345)


def test_solve_datafile_and_copy_states_restart(itp, tmp_path):
    from itp2d_b200 import datafile as D
    p = itp.Parameters(**HO)
    s = itp.ITPSystem(p)
    s.run()
    assert not s.error_flag, s.last_error
    path = str(tmp_path / "solve.h5")
    s.write_datafile(path, clobber=True)
    E, sig, _, idx = s.energies()
    steps, k = s.total_steps, HO["num_states"]
    assert np.array_equal(D.read(path, "final_energies"), E)
    assert np.array_equal(D.read(path, "final_energy_standard_deviations"), sig)
    hist = D.read(path, "energy_history")
    assert hist.shape == (steps, k)
    assert np.array_equal(hist[-1], E) and np.array_equal(hist[0], s.energy_history(0))
    assert D.read(path, "deviation_history").shape == (steps, k)
    ts = D.read(path, "time_step_history")
    assert tuple(ts[0]) == (1.0, 1.0)  # the first step ran with the first listed time step
    assert D.attribute(path, "num_states") == k
    assert D.attribute(path, "total_steps_done") == steps
    assert D.attribute(path, "num_converged") == s.num_converged
    assert D.attribute(path, "error_flag") == 0
    assert D.string_attribute(path, "grid_boundary_type") == "periodic"
    assert D.string_attribute(path, "potential") == "harmonic(1)"
    dx = HO["length"] / HO["sx"]
    x = (2 * np.arange(HO["sx"]) + 1 - HO["sx"]) * dx / 2
    V = D.read(path, "potential_values").reshape(HO["sy"], HO["sx"])
    assert np.allclose(V, 0.5 * (x[None, :] ** 2 + x[:, None] ** 2), rtol=1e-12, atol=1e-12)
    # the saved slot holds the states in energy order
    saved = D.init_states(path, k, HO["sx"], HO["sy"], dx)
    assert np.array_equal(saved, s.states()[idx])
    # --copy-states: a solve started from the saved states ends at the same energies
    s2 = itp.ITPSystem(p, init_states=saved)
    s2.run()
    assert not s2.error_flag, s2.last_error
    assert np.max(np.abs(s2.energies()[0][:8] - E[:8])) < TOL
