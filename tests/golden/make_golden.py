"""Generate the golden vectors that pin the oracle (and, through it, the CUDA path).

Every array here is produced by the REFERENCE's own code: the bem-bubbles sources
(Bem/Integration, Bem/Simulation, Bem/Mesh) compiled against the oracle's Eigen-API shim
into oracle/_ref/ref_harness_{free,mirror} (recipe: oracle/Makefile).  The reference
ships no tests, fixtures or golden vectors, so these outputs are the pins.

Also stores SHA-256 digests of the reference's icosphere generator output
(python_utils/icosphere/icosphere.py, imported from the reference checkout) so that the
project's own mesh generator can be checked without the reference present.

Run in the build container (needs the reference checkout and `make -C oracle ref`):
    python tests/golden/make_golden.py [path/to/reference]
(default: the checkout oracle/Makefile compiles from, BEM_REFERENCE).
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "bem-bubbles_b200"))

import oracle as O  # noqa: E402
from bem_b200 import mesh  # noqa: E402


def two_bubbles(nu, r1=1.0, r2=0.7, c1=2.5, c2=4.5):
    a = mesh.bubble(nu, r1, (c1, 0, 0))
    b = mesh.bubble(nu, r2, (c2, 0, 0))
    v, f = mesh.join([a, b])
    phi = np.r_[np.full(len(a[0]), -0.5 * r1), np.full(len(b[0]), 0.2 * r2)]
    return v, f, phi


def main(ref_root=None):
    ref_root = ref_root or O.reference_dir()
    if not (O.ref_available(False) and O.ref_available(True)):
        raise SystemExit("build the reference first: make -C oracle ref")
    out = {}
    field = dict(p_inf=1.0, epsilon=1.0, sigma=0.0, gamma=1.4, amp=-0.8, omega=2 * np.pi / 5, phase=0.0)
    out["field"] = np.array([field[k] for k in ("p_inf", "epsilon", "sigma", "gamma", "amp", "omega", "phase")])

    # 1) assembly, single bubble nu=2 and two bubbles nu=2, wall image off and on
    cases = {
        "one": (*mesh.bubble(2, 1.0, (2.0, 0.0, 0.0)), None),
        "two": two_bubbles(2),
    }
    for name, (v, f, phi) in cases.items():
        N = len(v)
        if phi is None:
            phi = np.linspace(-1.0, 1.0, N)
        out[f"{name}_verts"], out[f"{name}_trigs"], out[f"{name}_phi"] = v, f, phi
        for mir in (0, 1):
            r = O.ref_run("assemble", v, f, phi, mirror=bool(mir))
            out[f"{name}_G_m{mir}"] = r[: N * N].reshape(N, N, order="F")
            out[f"{name}_H_m{mir}"] = r[N * N:].reshape(N, N, order="F")
            out[f"{name}_psiLU_m{mir}"] = O.ref_run("solve", v, f, phi, mirror=bool(mir), lu=1)
            out[f"{name}_psiBiCG_m{mir}"] = O.ref_run("solve", v, f, phi, mirror=bool(mir), lu=0)

    v, f, phi = cases["two"]
    V0 = O.volume(v, f)
    out["two_V0"] = np.array([V0])
    out["two_vel"] = O.ref_run("position_t", v, f, phi, V0=V0, **field).reshape(-1, 3)
    out["two_pot_t"] = O.ref_run("pot_t", v, f, phi, t=0.3, V0=V0, **field)
    out["two_pot_t_sigma"] = O.ref_run("pot_t", v, f, phi, t=0.3, V0=V0, **dict(field, sigma=0.3))

    # 2) trajectories: 3 fixed RK4 steps (LU), 2 adaptive RK4 steps (BiCGSTAB), 2 Euler steps
    out["two_rk4"] = O.ref_run("rk4", v, f, phi, steps=3, dt=1e-2, V0=V0, lu=1, **field).reshape(3, -1)
    out["two_rk4_adapt"] = O.ref_run("rk4", v, f, phi, steps=2, dt=0.05, fixdt=0, lu=0, V0=V0,
                                     **field).reshape(2, -1)
    out["two_euler"] = O.ref_run("euler", v, f, phi, steps=2, dt=1e-2, V0=V0, lu=1, **field).reshape(2, -1)

    # exterior potential at points off the surface (outside both bubbles, between them, inside one):
    # compute_exterior_pot with a given psi, and exterior_pot (assemble, LU solve, then the same)
    pts = np.array([[0.5, 0.3, 0.1], [2.5, 1.8, 0.0], [3.5, 0.0, 0.2], [6.0, -1.0, 2.0], [2.5, 0.0, 0.0],
                    [4.5, 0.2, -0.1], [3.6, 0.5, 0.4]])
    psi_x = 0.2 * np.cos(v[:, 2]) - 0.1 * v[:, 1]
    out["ext_points"], out["ext_psi"] = pts, psi_x
    out["ext_direct"] = O.ref_run("exterior_direct", v, f, phi, points=pts, psi=psi_x)
    out["ext_solve"] = O.ref_run("exterior", v, f, phi, points=pts, lu=1)

    # 3) wall: bubble touching the x=eps line, image kernel on, collapsing -> nopenetration
    vw, fw = mesh.bubble(2, 1.0, (1.004, 0.0, 0.0))
    out["wall_verts"], out["wall_trigs"] = vw, fw
    out["wall_rk4"] = O.ref_run("rk4", vw, fw, np.full(len(vw), 0.6), mirror=True, steps=2, dt=2e-2,
                                p_inf=1.0, epsilon=0.0, sigma=0.0, gamma=1.0, lu=1).reshape(2, -1)

    # 4) config-1 shape: two nu=7 bubbles (N=984), 2 RK4 steps at dt=1e-3, LU, eps=0
    v7, f7, _ = two_bubbles(7, 1.0, 1.0, 2.5, 5.5)
    n7 = len(v7) // 2
    phi7 = np.r_[np.full(n7, -0.5), np.full(n7, 0.5)]
    out["c1_rk4"] = O.ref_run("rk4", v7, f7, phi7, steps=2, dt=1e-3, p_inf=1.0, epsilon=0.0, sigma=0.0,
                              gamma=1.0, lu=1, threads=1).reshape(2, -1)

    # 5) icosphere digests from the reference's generator
    sys.path.insert(0, os.path.join(ref_root, "python_utils", "icosphere"))
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        import icosphere as ref_ico
    nus = np.array([1, 2, 3, 4, 7, 10, 16, 20])
    digests = []
    for nu in nus:
        rv, rf = ref_ico.icosphere(int(nu))
        h = hashlib.sha256(np.ascontiguousarray(rv, dtype=np.float64).tobytes()
                           + np.ascontiguousarray(rf, dtype=np.int64).tobytes()).hexdigest()
        digests.append(h)
    out["ico_nus"] = nus
    out["ico_sha256"] = np.array(digests)

    np.savez_compressed(os.path.join(HERE, "ref_cases.npz"), **out)
    print("wrote", os.path.join(HERE, "ref_cases.npz"))


if __name__ == "__main__":
    main(*sys.argv[1:])
