"""Host-side checks of the benchmark workloads (no GPU): the bumpy-dot
potential is the seeded sum of Gaussian bumps the workload describes, added
to the analytic r^2/2 through the extra-potential hook; the magnetic dot has
none."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import bench  # noqa: E402


def _with(name):
    bench.WORKLOAD = bench.WORKLOADS[name]


def test_dot_has_no_extra_potential():
    _with("dot")
    assert bench.extra_potential() is None
    assert bench.config_block("mixed")["workload"].startswith("magnetic dot")


def test_bumpy_potential_is_seeded_gaussian_sum():
    _with("bumpy")
    try:
        w = bench.WORKLOAD
        b = w["bumps"]
        V = bench.extra_potential()
        assert V.shape == (w["sy"], w["sx"])
        assert np.array_equal(V, bench.extra_potential())  # deterministic
        # restated independently: the same draws, one bump at a time
        rng = np.random.default_rng(b["seed"])
        amp = rng.uniform(*b["amp"], size=b["n"])
        cen = rng.uniform(-b["box"], b["box"], size=(b["n"], 2))
        assert amp.min() >= 0.8 and amp.max() <= 1.2 and np.abs(cen).max() <= 6.0
        dx = w["length"] / w["sx"]
        x = (2 * np.arange(w["sx"]) + 1 - w["sx"]) * dx / 2  # cell-centred, datalayout.cpp:21-35
        j = int(np.argmax(amp))
        ix = int(np.argmin(np.abs(x - cen[j, 0])))
        iy = int(np.argmin(np.abs(x - cen[j, 1])))
        r2 = (x[ix] - cen[j, 0]) ** 2 + (x[iy] - cen[j, 1]) ** 2
        assert V[iy, ix] >= amp[j] * np.exp(-r2 / (2 * b["width"] ** 2)) - 1e-12
        assert V.min() >= 0.0 and V.max() < 1.2 * 4  # a few overlapping bumps at most
        cfg = bench.config_block("mixed")
        assert cfg["grid"] == [512, 512] and cfg["global_batch"] == 2000
        assert "6th-order" in cfg["workload"]
    finally:
        _with("dot")
