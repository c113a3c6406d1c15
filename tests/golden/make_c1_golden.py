"""Golden trajectory of the plain-FP64 two-bubble configuration (the reference's main.cpp set-up),
100 RK4 steps, produced by the REFERENCE's own code.

Two icospheres nu=7 (492 vertices, 980 triangles each, N = 984), radius 1, centres (2.5,0,0) and
(5.5,0,0) (3.0 apart, in x > 0 so test_negative never fires), phi = -R*Rdot with Rdot = +0.5 / -0.5,
p_inf = 1, epsilon = 0, sigma = 0, no wall image, 100 RK4 steps (evolve_system_RK4,
LinLinSim.cpp:194-257) at dt = 1e-3 with the PartialPivLU solve, the loop shape of main.cpp:61-73.
The reference build (oracle/_ref/ref_harness_free) runs on one thread so its assembly sums in a fixed
order.  Stored: x, phi, psi and time after steps 25, 50, 75 and 100.

Run in the build container (needs `make -C oracle ref`):
    python tests/golden/make_c1_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "bem-bubbles_b200"))

import oracle as O  # noqa: E402
from bem_b200 import mesh  # noqa: E402

STEPS, KEEP = 100, (25, 50, 75, 100)


def config1():
    a = mesh.bubble(7, 1.0, (2.5, 0.0, 0.0))
    b = mesh.bubble(7, 1.0, (5.5, 0.0, 0.0))
    v, f = mesh.join([a, b])
    n = len(a[0])
    phi = np.r_[np.full(n, -0.5), np.full(n, 0.5)]
    return v, f, phi


def main():
    if not O.ref_available(False):
        raise SystemExit("build the reference first: make -C oracle ref")
    v, f, phi = config1()
    N = len(v)
    recs = O.ref_run("rk4", v, f, phi, steps=STEPS, dt=1e-3, p_inf=1.0, epsilon=0.0, sigma=0.0, gamma=1.0,
                     lu=1, threads=1).reshape(STEPS, 5 * N + 1)
    keep = np.array(KEEP)
    np.savez_compressed(os.path.join(HERE, "c1_100.npz"), steps=keep, records=recs[keep - 1])
    print("wrote", os.path.join(HERE, "c1_100.npz"))


if __name__ == "__main__":
    main()
