"""ctypes front-end of the oracle (liboracle.so, the CPU restatement in bem_oracle.c)
and of the reference harness binaries in oracle/_ref/.

Test infrastructure: imported only by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg, as the checker.  The product path never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_P = C.POINTER(C.c_double)
_PI = C.POINTER(C.c_int64)


class Params(C.Structure):
    _fields_ = [("p_inf", C.c_double), ("epsilon", C.c_double), ("sigma", C.c_double),
                ("gamma", C.c_double), ("V0", C.c_double), ("field_amp", C.c_double),
                ("field_omega", C.c_double), ("field_phase", C.c_double), ("min_dt", C.c_double),
                ("dp_balance", C.c_double), ("nopen_eps", C.c_double), ("mirror", C.c_int32),
                ("use_lu", C.c_int32)]


def make_params(p_inf=1.0, epsilon=1.0, sigma=0.0, gamma=1.0, V0=1.0, amp=0.0, omega=0.0, phase=0.0,
                min_dt=-1.0, dp_balance=3.0, nopen_eps=1e-2, mirror=False, use_lu=True) -> Params:
    return Params(p_inf, epsilon, sigma, gamma, V0, amp, omega, phase, min_dt, dp_balance, nopen_eps,
                  int(bool(mirror)), int(bool(use_lu)))


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True, stdout=subprocess.DEVNULL)
        L = C.CDLL(LIB_PATH)
        L.orc_assemble.argtypes = [C.c_int64, C.c_int64, _P, _PI, C.c_int32, _P, _P]
        L.orc_gemv.argtypes = [C.c_int64, _P, _P, _P]
        L.orc_solve_lu.argtypes = [C.c_int64, _P, _P, _P]
        L.orc_solve_bicgstab.argtypes = [C.c_int64, _P, _P, _P, _PI, _P]
        L.orc_vertex_normals.argtypes = [C.c_int64, C.c_int64, _P, _PI, _P]
        L.orc_volume.argtypes = [C.c_int64, C.c_int64, _P, _PI]
        L.orc_volume.restype = C.c_double
        L.orc_position_t.argtypes = [C.c_int64, C.c_int64, _P, _PI, _P, C.POINTER(Params), _P, _P]
        L.orc_pot_t_multi.argtypes = [C.c_int64, C.c_int64, _P, _PI, _P, C.c_double, C.POINTER(Params), _P]
        L.orc_rk4_step.argtypes = [C.c_int64, C.c_int64, _P, _PI, _P, _P, _P, C.c_double, C.c_int32,
                                   C.POINTER(Params), _P]
        L.orc_euler_step.argtypes = [C.c_int64, C.c_int64, _P, _PI, _P, _P, C.c_double, C.c_int32,
                                     C.POINTER(Params), _P]
        L.orc_exterior_pot.argtypes = [C.c_int64, C.c_int64, _P, _PI, _P, _P, C.c_int64, _P, _P]
        L.orc_exterior_pot.restype = None
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_P)


def _i(a):
    return a.ctypes.data_as(_PI)


def _prep(verts, tris):
    v = np.ascontiguousarray(verts, dtype=np.float64)
    t = np.ascontiguousarray(tris, dtype=np.int64)
    return v, t


def assemble(verts, tris, mirror=False):
    v, t = _prep(verts, tris)
    N = len(v)
    G = np.empty((N, N), dtype=np.float64, order="F")
    H = np.empty((N, N), dtype=np.float64, order="F")
    lib().orc_assemble(N, len(t), _d(v), _i(t), int(mirror), _d(G), _d(H))
    return G, H


def gemv(A, x):
    A = np.asfortranarray(A, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty(A.shape[0])
    lib().orc_gemv(A.shape[0], _d(A), _d(x), _d(y))
    return y


def solve(G, b, use_lu=True):
    G = np.asfortranarray(G, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.empty_like(b)
    if use_lu:
        rc = lib().orc_solve_lu(len(b), _d(G), _d(b), _d(x))
        return x, {"rc": rc}
    it = np.zeros(1, dtype=np.int64)
    err = np.zeros(1)
    rc = lib().orc_solve_bicgstab(len(b), _d(G), _d(b), _d(x), _i(it), _d(err))
    return x, {"rc": rc, "iters": int(it[0]), "error": float(err[0])}


def vertex_normals(verts, tris):
    v, t = _prep(verts, tris)
    out = np.empty_like(v)
    lib().orc_vertex_normals(len(v), len(t), _d(v), _i(t), _d(out))
    return out


def exterior_pot(verts, tris, phi, psi, points):
    """compute_exterior_pot (LinLinSim.cpp:440-477) restated in C."""
    v, t = _prep(verts, tris)
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
    out = np.empty(len(pts))
    lib().orc_exterior_pot(len(v), len(t), _d(v), _i(t), _d(np.ascontiguousarray(phi, dtype=np.float64)),
                           _d(np.ascontiguousarray(psi, dtype=np.float64)), len(pts), _d(pts), _d(out))
    return out


def volume(verts, tris):
    v, t = _prep(verts, tris)
    return lib().orc_volume(len(v), len(t), _d(v), _i(t))


def position_t(verts, tris, pot, params: Params):
    v, t = _prep(verts, tris)
    pot = np.ascontiguousarray(pot, dtype=np.float64)
    vel = np.empty_like(v)
    psi = np.empty(len(v))
    rc = lib().orc_position_t(len(v), len(t), _d(v), _i(t), _d(pot), C.byref(params), _d(vel), _d(psi))
    if rc not in (0,):
        raise RuntimeError(f"orc_position_t failed ({rc})")
    return vel, psi


def pot_t_multi(verts, tris, grads, t, params: Params):
    v, tr = _prep(verts, tris)
    g = np.ascontiguousarray(grads, dtype=np.float64)
    out = np.empty(len(v))
    lib().orc_pot_t_multi(len(v), len(tr), _d(v), _i(tr), _d(g), float(t), C.byref(params), _d(out))
    return out


class State:
    """Simulation state (mesh.verts, phi, psi, time) stepped by the oracle."""

    def __init__(self, verts, tris, phi, psi=None, time=0.0):
        self.x, self.tri = _prep(verts, tris)
        self.x = self.x.copy()
        self.phi = np.array(phi, dtype=np.float64)
        self.psi = np.zeros(len(self.x)) if psi is None else np.array(psi, dtype=np.float64)
        self.time = np.array([time], dtype=np.float64)

    def rk4(self, dp, params: Params, fixdt=True):
        dt = np.zeros(1)
        rc = lib().orc_rk4_step(len(self.x), len(self.tri), _d(self.x), _i(self.tri), _d(self.phi),
                                _d(self.psi), _d(self.time), float(dp), int(fixdt), C.byref(params), _d(dt))
        if rc == -2:
            raise IndexError("negative values")  # the reference throws std::out_of_range
        if rc != 0:
            raise RuntimeError(f"orc_rk4_step failed ({rc})")
        return float(dt[0])

    def euler(self, dp, params: Params, fixdt=True):
        dt = np.zeros(1)
        rc = lib().orc_euler_step(len(self.x), len(self.tri), _d(self.x), _i(self.tri), _d(self.phi),
                                  _d(self.time), float(dp), int(fixdt), C.byref(params), _d(dt))
        if rc != 0:
            raise RuntimeError(f"orc_euler_step failed ({rc})")
        return float(dt[0])


# ---------------------------------------------------------------- reference harness
def reference_dir() -> str:
    """The reference checkout the oracle's recipe compiles from (oracle/Makefile's BEM_REFERENCE: the
    environment variable of that name, else its default)."""
    out = subprocess.run(["make", "-s", "--no-print-directory", "-C", HERE, "refdir"], check=True,
                         capture_output=True, text=True)
    return out.stdout.strip()


def ref_available(mirror=False) -> bool:
    return os.path.exists(os.path.join(REF_DIR, "ref_harness_" + ("mirror" if mirror else "free")))


def ref_run(action, verts, tris, phi, mirror=False, timing=False, points=None, psi=None, **kw):
    """Run the reference's own code (oracle/_ref/ref_harness_*) and return its float64 output.
    points (P x 3) and psi (N) are the extra inputs of the exterior actions."""
    v, t = _prep(verts, tris)
    exe = os.path.join(REF_DIR, "ref_harness_" + ("mirror" if mirror else "free"))
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(fin, "wb") as fh:
            np.array([len(v), len(t)], dtype=np.int64).tofile(fh)
            v.tofile(fh)
            t.tofile(fh)
            np.ascontiguousarray(phi, dtype=np.float64).tofile(fh)
            if points is not None:
                pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
                np.array([len(pts)], dtype=np.int64).tofile(fh)
                pts.tofile(fh)
                if psi is not None:
                    np.ascontiguousarray(psi, dtype=np.float64).tofile(fh)
        args = [exe, action, fin, fout] + [f"{k}={float(val)!r}" for k, val in kw.items()]
        if timing:
            args.append("timing=1")
        env = dict(os.environ)
        env.setdefault("OMP_NUM_THREADS", str(int(kw.get("threads", 1))))
        r = subprocess.run(args, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, env=env)
        out = np.fromfile(fout, dtype=np.float64)
    if timing:
        return out, r.stderr.decode()
    return out


def ref_rk4_timed(verts, tris, phi, warm, steps, budget=0.0, **kw):
    """Real RK4 steps of the reference's own code (evolve_system_RK4, LinLinSim.cpp:194-257):
    `warm` untimed steps from (verts, phi), then up to `steps` timed ones, stopping once `budget`
    seconds of timed steps are spent (0: no limit).  Returns a dict with per-step seconds, BiCGSTAB
    solves and iterations, and the final state (x, phi, psi, time)."""
    out = ref_run("rk4_timed", verts, tris, phi, warm=warm, steps=steps, budget=budget, **kw)
    n = len(verts)
    k = int(out[0])
    rec = out[1:1 + 3 * k].reshape(k, 3)
    st = out[1 + 3 * k:]
    return {"seconds": rec[:, 0].copy(), "solves": rec[:, 1].astype(int), "iters": rec[:, 2].astype(int),
            "x": st[:3 * n].reshape(n, 3), "phi": st[3 * n:4 * n], "psi": st[4 * n:5 * n], "time": float(st[5 * n])}
