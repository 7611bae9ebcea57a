"""Runs the compiled itp2d reference (oracle/_ref, ``make -C oracle`` first)
through a whole solve of a benchmark workload and stores its converged
energies as a golden fixture.

    python tests/golden/make_solve_golden.py [--workload dot|bumpy] [--threads T]

Workloads (bench.py's WORKLOADS, same seeded initial states and potential):

* dot: V = r^2/2, B = 1 (linear gauge), periodic 256 x 256 grid of side 14,
  k = 500, 4th-order multi-product split at eps = 0.05, abschange(1e-9) as
  time-step and final test on the 250 lowest states
  -> solve_magnetic_dot_256_k500.json (a few minutes on 8 cores);
* bumpy: V = r^2/2 + 400 seeded Gaussian bumps, B = 0.5, periodic 512 x 512
  grid of side 16, k = 2000, 6th-order split, the 1000 lowest states
  -> solve_bumpy_dot_512_k2000.json (out of reach: the reference's pairwise
  overlap dots stream terabytes per iteration at this size);
* c1: configuration C1 (C1 below) -> solve_harmonic_dirichlet_128_k64.json.

The eps divisor is 5 (the reference default) and the orthonormalisation is
HighMem (one ZGEMM, stateset.cpp:214-228). The reference's ITPSystem::step
(itpsystem.cpp:407-470) runs until is_finished(); the sorted energies,
deviations, iteration count, converged count and the reference's own phase
times (itpsystem.cpp:551-567) are written after every iteration, so an
interrupted run leaves its progress behind (``finished`` false).
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from oracle import refkit as R  # noqa: E402

OUT = {"dot": "solve_magnetic_dot_256_k500.json", "bumpy": "solve_bumpy_dot_512_k2000.json",
       "c1": "solve_harmonic_dirichlet_128_k64.json"}

# Configuration C1: V = r^2/2, B = 0, Dirichlet box of side 12 on 128 x 128,
# k = 64 states from seeded complex Gaussian noise, 2nd-order split at
# eps = 0.02 (divisor 2), abschange(1e-10) as time-step and final test. The
# deviation sqrt(<H^2> - <H>^2) that the deviation tests read sits at a floor
# of about 5e-5 for every state on this grid (FP64 cancellation of <H^2> and
# <H>^2 with the large kinetic eigenvalues of 128 DST-II points), so
# absstdev(1e-8) never passes; with an energy-change time-step test and a
# deviation final test the reference's schedule then halves eps every step
# down to its bail-out limit. The same test for both ends the solve once every
# wanted energy moves by less than 1e-10 per step. The 64 states end
# inside the 11-fold degenerate level E = 11, which cannot converge, so the 55
# states of the levels E = 1..10 are the wanted ones.
C1 = dict(sx=128, sy=128, length=12.0, boundary=1, B=0.0, halforder=1, num_states=64, wanted=55, eps=0.02,
          eps_divisor=2.0, timestep_test="abschange(1e-10)", final_test="abschange(1e-10)",
          potential="harmonic(1)", seed=20240607)


def c1_states():
    w = C1
    rng = np.random.default_rng(w["seed"])
    dx = w["length"] / w["sx"]
    psi = rng.standard_normal((w["num_states"], w["sy"], w["sx"])) + 1j * rng.standard_normal(
        (w["num_states"], w["sy"], w["sx"]))
    return psi / (np.sqrt(np.sum(np.abs(psi) ** 2, axis=(1, 2))) * dx)[:, None, None]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="dot", choices=sorted(OUT))
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    a = ap.parse_args()
    if a.workload == "c1":
        w = C1
        psi = c1_states()
        ref = R.RefSystem(w["sx"], w["sy"], w["length"], w["boundary"], w["B"], w["halforder"], w["num_states"],
                          w["wanted"], [w["eps"]], eps_divisor=w["eps_divisor"], timestep_test=w["timestep_test"],
                          final_test=w["final_test"], potential=w["potential"], init_states=psi,
                          threads=a.threads, highmem=True, max_steps=20000, min_eps=1e-9)
        label = ("C1: harmonic(1), Dirichlet 128x128, L=12, k=64 (55 wanted), halforder 1, eps 0.02 / 2, "
                 "abschange(1e-10) as time-step and final test")
    else:
        w = bench.WORKLOADS[a.workload]
        bench.WORKLOAD = w
        psi, _ = bench.initial_states(pinned=False)
        ref = R.RefSystem(w["sx"], w["sy"], w["length"], 0, w["B"], w["halforder"], w["num_states"], w["wanted"],
                          [w["eps"]], eps_divisor=5.0, timestep_test=w["test"], final_test=w["test"],
                          potential=w["potential"], extra_potential=bench.extra_potential(), init_states=psi,
                          threads=a.threads, highmem=True, max_steps=5000, min_eps=1e-9)
        label = bench.config_block("reference")["workload"]
    del psi
    path = os.path.join(HERE, OUT[a.workload])
    t0 = time.perf_counter()
    iter_s = []
    while not ref.finished:
        t1 = time.perf_counter()
        ref.step()
        iter_s.append(time.perf_counter() - t1)
        assert not ref.error_flag
        E, sig = ref.energies()
        out = {"workload": label, "seed": w["seed"],
               "finished": ref.finished, "iterations": ref.total_steps, "converged": ref.num_converged,
               "final_eps": ref.eps, "threads": a.threads, "seconds": time.perf_counter() - t0,
               "seconds_per_iteration": iter_s, "energies": E.tolist(), "sigma": sig.tolist(),
               "phase_seconds": ref.times()}
        with open(path, "w") as f:
            json.dump(out, f)
        if ref.total_steps % 50 == 0 or ref.finished:
            print(f"iteration {ref.total_steps}: eps {ref.eps:.4g}, {iter_s[-1]:.2f} s", flush=True)
    print(f"wrote {path}: {ref.total_steps} iterations, {ref.num_converged} converged, "
          f"{time.perf_counter() - t0:.0f} s")


if __name__ == "__main__":
    main()
