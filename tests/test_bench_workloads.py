"""Host-side checks of the benchmark workloads (no GPU): the bumpy-dot
potential is the seeded sum of Gaussian bumps the workload describes, added
to the analytic r^2/2 through the extra-potential hook; the magnetic dot has
none."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import bench  # noqa: E402
from itp2d_b200 import capi  # noqa: E402


def _with(name):
    bench.WORKLOAD = bench.WORKLOADS[name]


def test_default_workload_is_the_bumpy_dot():
    import importlib
    b = importlib.reload(bench)
    assert b.WORKLOAD is b.WORKLOADS["bumpy"]
    assert b.WORKLOAD["num_states"] == 2000 and b.WORKLOAD["halforder"] == 3


def test_reference_solve_figures():
    """The magnetic dot extrapolates with the reference's own solve (golden
    fixture); the bumpy dot with the FP64 form's, which every run checks."""
    _with("dot")
    it, conv, src = bench.reference_solve()
    assert (it, conv) == (32, 288) and "reference's own solve" in src
    _with("bumpy")
    try:
        it, conv, src = bench.reference_solve()
        assert (it, conv) == bench.WORKLOADS["bumpy"]["fp64_solve"] and "fp64_solve_check" in src
        r64 = {"steps": [it], "conv": [conv]}
        assert bench.fp64_solve_check(r64)["ok"]
        assert not bench.fp64_solve_check({"steps": [it + 1], "conv": [conv]})["ok"]
    finally:
        _with("dot")


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


def test_phase_rooflines_arithmetic():
    """Per-phase rooflines from synthetic per-solve stats: algorithmic bytes and
    flops over the phase time, split by precision, eigensolve flops scaled by
    the sweeps of that precision."""
    import json
    import os
    _with("dot")
    w = bench.WORKLOAD
    k, G, m = w["num_states"], w["sx"] * w["sy"], w["halforder"]
    stats = {(p, ph): (0.0, 0) for p in ("fp64", "fp32") for ph in capi.PHASES}
    stats[("fp64", "propagate")] = (10.0, 5)
    stats[("fp64", "overlap")] = (4.0, 5)
    stats[("fp32", "eigensolve")] = (20.0, 10)
    r = {"stats": stats, "sweeps": {"fp64": 0.0, "fp32": 40.0}}
    roof = bench.phase_rooflines(r, fp64_peak=40.0, fp32_peak=80.0)
    assert set(roof) == {"propagate_fp64", "overlap_fp64", "eigensolve_fp32"}  # phases with calls only
    try:  # the measured copy bandwidth, else the benchmark's stated fallback
        hbm = json.load(open(os.path.join(bench.ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
    except (OSError, KeyError, ValueError):
        hbm = 6650.0
    p = roof["propagate_fp64"]
    assert abs(p["achieved"] - k * G * 16 * (2 * m * (m + 2) + (m - 1)) * 5 / 10e-3 / 1e9) < 1e-6 * p["achieved"]
    assert abs(p["frac"] - p["achieved"] / hbm) < 1e-12 and p["unit"] == "GB/s"
    o = roof["overlap_fp64"]
    assert abs(o["achieved"] - 4 * k * k * G * 5 / 4e-3 / 1e12) < 1e-9 * o["achieved"]
    assert o["peak"] == 40.0 and o["bound"] == "tensor"
    e = roof["eigensolve_fp32"]
    # algorithmic: 10 k^3 flops per eigensolve call
    assert abs(e["achieved"] - 10.0 * k ** 3 * 10 / 20e-3 / 1e12) < 1e-9 * e["achieved"]
    kp = (k + 31) // 32 * 32
    flops = (kp // 16 - 1) * 3 * 8 * 32 * kp * kp * 40.0
    assert abs(e["method_tflops"] - flops / 20e-3 / 1e12) < 1e-9 * e["method_tflops"]
    assert e["peak"] == 80.0 and e["bound"] == "fp32" and e["sweeps_per_solve"] == 40.0
