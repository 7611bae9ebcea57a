"""Abort and save flags of the native driver, and the SIGINT / SIGUSR1
handlers that raise them (itp2d.cpp:40-66; ITPSystem::step and
check_save_flag, itpsystem.cpp:236-241,407-470).

The handler tests run in a child process (the handlers replace Python's own
SIGINT handler) and need no GPU: the child only loads the library, installs
the handlers and signals itself. The system tests run a small solve on the
GPU with flags the test owns.
"""
import ctypes as C
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = textwrap.dedent("""
    import os, signal, sys
    sys.path.insert(0, {root!r})
    from itp2d_b200 import system
    system.install_signal_handlers()
    a, s = system.abort_flag(), system.save_flag()
    assert a[0] == 0 and s[0] == 0
    os.kill(os.getpid(), signal.SIGUSR1)
    assert s[0] == 1 and a[0] == 0, (a[0], s[0])
    s[0] = 0
    os.kill(os.getpid(), signal.SIGINT)
    assert a[0] == 1 and s[0] == 0, (a[0], s[0])
    print("first SIGINT survived", flush=True)
    os.kill(os.getpid(), signal.SIGINT)
    print("second SIGINT survived", flush=True)
""")


def test_signal_handlers_raise_flags_and_second_sigint_exits():
    r = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT)], capture_output=True, text=True, timeout=120)
    assert "first SIGINT survived" in r.stdout, r.stderr
    assert "second SIGINT survived" not in r.stdout
    assert r.returncode == 1, (r.returncode, r.stderr)
    assert "SIGUSR1" in r.stderr and "SIGINT" in r.stderr


def _small_system(system, capi):
    p = system.Parameters(sx=64, sy=64, length=10.0, boundary=capi.PERIODIC, B=0.0, halforder=1, num_states=8,
                          wanted=4, eps=[0.05], timestep_test="abschange(1e-9)", final_test="abschange(1e-9)",
                          potential="harmonic(1)", max_steps=5000)
    return system.ITPSystem(p)


@pytest.mark.gpu
def test_save_flag_saves_then_abort_flag_ends_solve():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from itp2d_b200 import capi, system
    s = _small_system(system, capi)
    abort, save = C.c_int(0), C.c_int(0)
    s.set_flags(abort, save)
    saved = []
    s.set_save_callback(lambda st, order, step: saved.append((st, order, step)))
    s.step()
    assert not saved and s.saves == 0
    save.value = 1
    s.step()
    # saved at the first check point of the step (after propagation), once
    assert len(saved) == 1 and s.saves == 1 and save.value == 0
    st, order, step = saved[0]
    assert step == 2 and st.shape == (8, 64, 64) and np.all(np.isfinite(st))
    assert order is not None and sorted(order.tolist()) == list(range(8))
    # the order is the previous step's energy order: its first state is the
    # lowest of step 1's energies
    E1 = s.energy_history(0)
    assert np.all(np.diff(E1) >= 0)
    steps = s.total_steps
    abort.value = 1
    s.step()
    assert s.finished and s.error_flag and s.total_steps == steps
    assert "abort" in s.last_error
    s.close()


@pytest.mark.gpu
def test_flags_between_device_loop_chunks():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    from itp2d_b200 import capi, system
    s = _small_system(system, capi)
    abort, save = C.c_int(0), C.c_int(0)
    s.set_flags(abort, save)
    count = []
    s.set_save_callback(lambda st, order, step: count.append(step))
    save.value = 1
    s.run_device(max_phases=1)
    # the save flag is read before the phase; with flags registered a phase
    # runs at most 32 iterations on the device
    assert count == [0] and save.value == 0
    assert 1 <= s.device_iterations <= 32
    abort.value = 1
    s.run_device()
    assert s.finished and s.error_flag
    assert s.device_iterations <= 32
    s.close()
