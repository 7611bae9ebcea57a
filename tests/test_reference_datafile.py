"""The reference-API Datafile (include/itp2d_reference_datafile.hpp) beside
the reference's own StateSet, Potential and Noise classes:
tests/cpp/test_reference_datafile.cpp, built against the reference sources by
``make -C oracle datafile-adapter`` (part of the build where the reference
sources are present). Host only."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "test_reference_datafile")


@pytest.mark.skipif(not os.path.exists(BIN), reason="built only where the reference sources are present")
def test_reference_datafile_adapter(tmp_path):
    r = subprocess.run([BIN, str(tmp_path / "reference.h5")], capture_output=True, text=True, timeout=120)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ok: 0 failure(s)" in r.stdout
