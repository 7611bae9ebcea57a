"""Generates the golden fixtures in this directory from the itp2d reference
sources compiled into oracle/_ref (``make -C oracle`` first).

    python tests/golden/make_golden.py

Each seam_*.npz holds, for one operator configuration, the seeded input
states and potential and the reference's outputs of one MultiProductSplit
application, one Hamiltonian application, the energies/deviations of
Operator::mean_and_standard_deviation, and the canonically orthonormalised
states of StateSet::orthonormalize.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import itp_oracle as O  # noqa: E402
from oracle import refkit as R  # noqa: E402

# name: sx, sy, L, boundary, B, halforder, eps, potential
SEAMS = {
    "periodic_b0_m1": (16, 12, 12.0, O.PERIODIC, 0.0, 1, 0.1, "harmonic(1)"),
    "dirichlet_b0_m2": (20, 16, 12.0, O.DIRICHLET, 0.0, 2, 0.1, "harmonic(1)"),
    "periodic_b1_m2": (16, 12, 14.0, O.PERIODIC, 1.0, 2, 0.05, "harmonic(1)"),
    "periodic_b05_m3": (16, 16, 16.0, O.PERIODIC, 0.5, 3, 0.05, "harmonic(1)"),
    "periodic_b0_null": (16, 12, 6.0, O.PERIODIC, 0.0, 2, 0.1, "zero"),
    "dirichlet_b07_m2": (20, 16, 12.0, O.DIRICHLET, 0.7, 2, 0.1, "harmonic(1)"),
}
K = 3


def make_seam(name, cfg):
    sx, sy, L, bt, B, m, eps, pot = cfg
    g = O.Grid.from_length(sx, sy, L)
    psi = O.gaussian_states(g, K, 1234)
    kit = R.RefKit(sx, sy, L, bt, B, m, eps, K, potential=pot, threads=1)
    V = kit.potential()
    kit.set_states(psi)
    kit.propagate()
    prop = kit.states()
    kit.set_states(psi)
    kit.apply_hamiltonian()
    hpsi = kit.states()
    kit.set_states(prop)
    E, sig, Ei = kit.energies()
    kit.set_states(prop)
    assert kit.orthonormalize() == 0
    ortho = kit.states()
    np.savez_compressed(os.path.join(HERE, f"seam_{name}.npz"), cfg=np.array([sx, sy, L, bt, B, m, eps]),
                        potential_null=np.array(pot == "zero"), psi=psi, V=V, prop=prop, hpsi=hpsi, E=E,
                        sigma=sig, ortho=ortho)


def main():
    if not R.available():
        raise SystemExit("build oracle/_ref first: make -C oracle")
    for name, cfg in SEAMS.items():
        make_seam(name, cfg)
    # Known-good energies of the magnetic particle in a box, as hard-coded in
    # the reference test test_itp.cpp:433-436 (64x64, L=pi, Dirichlet, B=1).
    with open(os.path.join(HERE, "magnetic_box_energies.json"), "w") as f:
        json.dump({"source": "test_itp.cpp:433-436", "grid": [64, 64], "length": 3.141592653589793,
                   "B": 1.0, "tolerance": 2e-3,
                   "energies": [1.077814, 2.134673, 3.089442, 3.551456, 5.075289, 5.499240, 5.729555,
                                7.042548]}, f, indent=1)
    print("ok")


if __name__ == "__main__":
    main()
