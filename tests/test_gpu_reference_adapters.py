"""The device library driven from the reference's own C++ operator API
(include/itp2d_reference.hpp): tests/cpp/test_reference_adapters.cpp, built
against the reference sources by ``make -C oracle adapters``, runs the
device classes beside the reference's CPU classes (transforms, the
EvolutionOperator MultiProductSplit per state and batched, energies,
StateSet::orthonormalize, EigenSolver) and the reference step loop on the
harmonic-oscillator case of test_itp.cpp:56-91 with its three seams on the
device. Each check prints "ok <name> <figure>"; the exit code counts failures."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "test_reference_adapters")


def test_reference_api_adapters():
    if not os.path.exists(BIN):
        pytest.fail(f"{BIN} missing: build it with make -C oracle adapters")
    r = subprocess.run([BIN], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, timeout=600,
                       env=dict(os.environ, OPENBLAS_NUM_THREADS="1"))
    print(r.stdout)
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith(("ok ", "FAIL "))]
    assert len(lines) >= 13, r.stdout
    assert r.returncode == 0 and not any(ln.startswith("FAIL") for ln in lines), r.stdout
