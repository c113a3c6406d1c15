"""Host-side mirror of the reference's simulation interface, over the C ABI.

``ColocSim`` follows Bem::ColocSim / Bem::LinLinSim / Bem::Simulation
(Bem/Simulation/ColocSim.hpp:13-28, LinLinSim.hpp:19-90, Simulation.hpp:26-210): same method
names, argument meaning and error behaviour (a vertex with x < 0 at an RK4 step raises, as the
reference's ``std::out_of_range`` from ``test_negative`` does).  The state lives in GPU memory;
every call crosses the C ABI with host arrays.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib as L


def _d(a):
    return a.ctypes.data_as(L._D)


class ColocSim:
    """Collocation BEM simulation of gas/vapour bubbles on one GPU.

    verts: (N,3) float64, trigs: (M,3) int; p_inf, epsilon, sigma, gamma as in the reference
    constructor (Simulation.hpp:29).  ``pressurefield`` is either None (the reference's
    default_field, 0), a tuple ``(amp, omega, phase[, kx])`` for amp*sin(kx*x + omega*t + phase)
    evaluated on the device, or a Python callable f(x: ndarray(3), t: float) -> float evaluated
    on the host for every vertex at every stage.
    """

    def __init__(self, verts, trigs, p_inf=1.0, epsilon=1.0, sigma=0.0, gamma=1.0, pressurefield=None,
                 device=0, solver="bicgstab", mirror=False):
        self._L = L.load()
        self._h = C.c_void_p()
        p = L.Params()
        self._L.bem_default_params(C.byref(p))
        p.p_inf, p.epsilon, p.sigma, p.gamma = float(p_inf), float(epsilon), float(sigma), float(gamma)
        p.mirror = int(bool(mirror))
        p.solver = {"bicgstab": L.SOLVER_BICGSTAB, "lu": L.SOLVER_LU, "mixed": L.SOLVER_MIXED}[solver]
        self._cb = None
        if pressurefield is not None and not callable(pressurefield):
            amp, omega, phase = pressurefield[:3]
            kx = pressurefield[3] if len(pressurefield) > 3 else 0.0
            p.field_amp, p.field_omega, p.field_phase, p.field_kx = float(amp), float(omega), float(phase), float(kx)
        rc = self._L.bem_create(C.byref(self._h), int(device), C.byref(p))
        if rc != L.BEM_OK:
            raise L.BemError(rc, "bem_create failed (no CUDA device?)")
        v = np.ascontiguousarray(verts, dtype=np.float64)
        t = np.ascontiguousarray(trigs, dtype=np.int64)
        self.N, self.M = len(v), len(t)
        self._check(self._L.bem_set_mesh(self._h, self.N, _d(v), self.M, t.ctypes.data_as(L._I64)))
        if callable(pressurefield):
            fn = pressurefield

            def _cb(xp, tt, user):
                return float(fn(np.array([xp[0], xp[1], xp[2]]), tt))

            self._cb = L.FIELD_FN(_cb)
            self._check(self._L.bem_set_field_callback(self._h, self._cb, None))

    # -------------------------------------------------------------- plumbing
    def _check(self, rc):
        if rc == L.BEM_OK:
            return
        msg = self._L.bem_last_error(self._h).decode() if self._h else ""
        if rc == L.BEM_ERR_NEGATIVE_X:
            raise IndexError(msg or "negative values")
        raise L.BemError(rc, msg)

    def close(self):
        if self._h:
            self._L.bem_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> L.Params:
        p = L.Params()
        self._check(self._L.bem_get_params(self._h, C.byref(p)))
        return p

    def _update(self, **kw):
        p = self.params()
        for k, v in kw.items():
            setattr(p, k, v)
        self._check(self._L.bem_set_params(self._h, C.byref(p)))

    # -------------------------------------------------------------- setters (Simulation.hpp:92-167)
    def set_phi(self, value):
        a = np.full(self.N, float(value)) if np.isscalar(value) else np.ascontiguousarray(value, dtype=np.float64)
        self._check(self._L.bem_set_phi(self._h, _d(a)))

    def set_psi(self, value):
        a = np.ascontiguousarray(value, dtype=np.float64)
        self._check(self._L.bem_set_psi(self._h, _d(a)))

    def get_phi(self):
        a = np.empty(self.N)
        self._check(self._L.bem_get_phi(self._h, _d(a)))
        return a

    def get_psi(self):
        a = np.empty(self.N)
        self._check(self._L.bem_get_psi(self._h, _d(a)))
        return a

    def get_vertices(self):
        a = np.empty((self.N, 3))
        self._check(self._L.bem_get_vertices(self._h, _d(a)))
        return a

    def set_vertices(self, v):
        a = np.ascontiguousarray(v, dtype=np.float64)
        self._check(self._L.bem_set_vertices(self._h, _d(a)))

    def set_state(self, verts=None, phi=None, psi=None, time=None):
        """Vertices, phi, psi and time in one call (None skips a part); the arrays are copied before
        the call returns and the device copies are queued without a wait."""
        arrs = []
        for a, shape in ((verts, (self.N, 3)), (phi, (self.N,)), (psi, (self.N,))):
            arrs.append(None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(shape))
        t = None if time is None else np.array([float(time)])
        self._check(self._L.bem_set_state(self._h, *[None if a is None else _d(a) for a in arrs],
                                          None if t is None else _d(t)))

    def get_state(self, out=None):
        """(vertices, phi, psi, time) with one wait; `out` = (verts, phi, psi) arrays to fill."""
        if out is None:
            out = (np.empty((self.N, 3)), np.empty(self.N), np.empty(self.N))
        t = np.zeros(1)
        self._check(self._L.bem_get_state(self._h, _d(out[0]), _d(out[1]), _d(out[2]), _d(t)))
        return out[0], out[1], out[2], float(t[0])

    def set_V_0(self, v):
        self._check(self._L.bem_set_V0(self._h, float(v)))

    def get_V_0(self):
        a = np.zeros(1)
        self._check(self._L.bem_get_V0(self._h, _d(a)))
        return float(a[0])

    def set_time(self, t):
        self._check(self._L.bem_set_time(self._h, float(t)))

    def get_time(self):
        a = np.zeros(1)
        self._check(self._L.bem_get_time(self._h, _d(a)))
        return float(a[0])

    def get_volume(self):
        a = np.zeros(1)
        self._check(self._L.bem_get_volume(self._h, _d(a)))
        return float(a[0])

    def set_min_dt(self, v):
        self._update(min_dt=float(v))

    def set_dp_balance(self, v):
        self._update(dp_balance=float(v))

    def set_bcgstab(self, on: bool):
        self._update(solver=L.SOLVER_BICGSTAB if on else L.SOLVER_LU)

    def set_solver(self, name: str):
        self._update(solver={"bicgstab": L.SOLVER_BICGSTAB, "lu": L.SOLVER_LU, "mixed": L.SOLVER_MIXED}[name])

    def set_mirror(self, on: bool):
        self._update(mirror=int(bool(on)))

    def stats(self) -> L.Stats:
        s = L.Stats()
        self._check(self._L.bem_get_stats(self._h, C.byref(s)))
        return s

    # -------------------------------------------------------------- hot path
    def assemble_matrices(self, verts=None):
        """ColocSim::assemble_matrices -> (G, H), column-major N x N float64."""
        G = np.empty((self.N, self.N), order="F")
        H = np.empty((self.N, self.N), order="F")
        v = None if verts is None else np.ascontiguousarray(verts, dtype=np.float64)
        self._check(self._L.bem_assemble(self._h, _d(v) if v is not None else None, _d(G), _d(H)))
        return G, H

    def assemble_rhs(self, pot, verts=None):
        """(G, b): G and b = H*pot after the 4 pi rule as the step path forms them (position_t,
        LinLinSim.cpp:26-83), without materialising H."""
        p = np.ascontiguousarray(pot, dtype=np.float64)
        G = np.empty((self.N, self.N), order="F")
        b = np.empty(self.N)
        v = None if verts is None else np.ascontiguousarray(verts, dtype=np.float64)
        self._check(self._L.bem_assemble_rhs(self._h, _d(v) if v is not None else None, _d(p), _d(G), _d(b)))
        return G, b

    def solve_system(self, G, b):
        G = np.asfortranarray(G, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.empty(self.N)
        self._check(self._L.bem_solve_system(self._h, _d(G), _d(b), _d(x)))
        return x

    def position_t(self, pot, verts=None, return_psi=False):
        pot = np.ascontiguousarray(pot, dtype=np.float64)
        vel = np.empty((self.N, 3))
        psi = np.empty(self.N)
        v = None if verts is None else np.ascontiguousarray(verts, dtype=np.float64)
        self._check(self._L.bem_position_t(self._h, _d(v) if v is not None else None, _d(pot), _d(vel), _d(psi)))
        return (vel, psi) if return_psi else vel

    def pot_t_multi(self, grads, t, verts=None):
        g = np.ascontiguousarray(grads, dtype=np.float64)
        out = np.empty(self.N)
        v = None if verts is None else np.ascontiguousarray(verts, dtype=np.float64)
        self._check(self._L.bem_pot_t_multi(self._h, _d(v) if v is not None else None, _d(g), float(t), _d(out)))
        return out

    def export_ply_async(self, path):
        """Simulation::export_mesh of the current state, written in the background (see export_wait)."""
        self._check(self._L.bem_export_ply_async(self._h, str(path).encode()))

    def export_wait(self):
        self._check(self._L.bem_export_wait(self._h))

    def exterior_potential(self, points, phi=None, psi=None):
        """compute_exterior_pot (LinLinSim.cpp:440-477) at points (P x 3) off the surface; with psi None,
        LinLinSim::exterior_pot: psi is solved first at the current positions."""
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        out = np.empty(len(pts))
        ph = None if phi is None else np.ascontiguousarray(phi, dtype=np.float64)
        ps = None if psi is None else np.ascontiguousarray(psi, dtype=np.float64)
        self._check(self._L.bem_exterior_potential(self._h, len(pts), _d(pts), None if ph is None else _d(ph),
                                                   None if ps is None else _d(ps), _d(out)))
        return out

    def evolve_system_RK4(self, dp, fixdt=False):
        dt = np.zeros(1)
        self._check(self._L.bem_evolve_rk4(self._h, float(dp), int(bool(fixdt)), _d(dt)))
        return float(dt[0])

    def evolve_system(self, dp, fixdt=False):
        dt = np.zeros(1)
        self._check(self._L.bem_evolve_euler(self._h, float(dp), int(bool(fixdt)), _d(dt)))
        return float(dt[0])

    def evolve_rk4_steps(self, dt, steps):
        """`steps` fixed-dt RK4 steps with no host round trip in between."""
        self._check(self._L.bem_evolve_rk4_n(self._h, float(dt), int(steps)))

    def sync(self):
        self._check(self._L.bem_sync(self._h))

    def stream_handle(self) -> int:
        h = C.c_void_p()
        self._check(self._L.bem_get_stream(self._h, C.byref(h)))
        return h.value or 0

    def set_profiling(self, on: bool):
        self._check(self._L.bem_set_profiling(self._h, int(bool(on))))

    def reset_profile(self):
        self._check(self._L.bem_reset_profile(self._h))

    def profile(self) -> L.Profile:
        p = L.Profile()
        self._check(self._L.bem_get_profile(self._h, C.byref(p)))
        return p


WALL_THRESHOLD = 1e-5  # |x| below which a vertex is on the wall (ColocSimPin.cpp:230, 264)
# the reference's contact-angle drift law (ColocSimPin.cpp:126-136): beta, cos(theta_eq), c_nonlinear
DRIFT_LAW = (0.2, math.cos(130.0 / 180.0 * math.pi), 0.01)


def move_flagged_to_end(verts, trigs, flagged, *per_vertex):
    """The reference's scan that moves flagged vertices to the end of the vertex list
    (ColocSimPin::set_x_boundary / rearrange_boundary, ColocSimPin.cpp:196-287): over the unsettled
    range [0, k) a flagged vertex trades places with vertex k-1, the range shrinks and the vertex
    that came in is examined next.  ``flagged(verts, i)`` may edit verts[i] (set_x_boundary puts the
    wall vertices exactly on x = 0).  ``per_vertex`` arrays are permuted along.
    Returns (verts, trigs, origin, count, *per_vertex): origin[p] = old index of the vertex now at p."""
    v = np.array(verts, dtype=np.float64, copy=True)
    t = np.array(trigs, dtype=np.int64, copy=True)
    extra = [np.array(a, copy=True) for a in per_vertex]
    n = len(v)
    origin = np.arange(n)
    k, i, moved = n, 0, 0
    while i < k:
        if not flagged(v, i):
            i += 1
            continue
        j = k - 1
        for arr in (v, origin, *extra):
            arr[[i, j]] = arr[[j, i]]
        k -= 1
        moved += 1
    where = np.empty(n, dtype=np.int64)
    where[origin] = np.arange(n)
    return (v, where[t], origin, moved, *extra)


def _on_wall(v, i):
    if abs(v[i, 0]) >= WALL_THRESHOLD:
        return False
    v[i, 0] = 0.0
    return True


class ColocSimPin(ColocSim):
    """A bubble on the wall x = 0 with its contact line pinned to the wall: Bem::ColocSimPin
    (Bem/Simulation/ColocSimPin.hpp:13-66, ColocSimPin.cpp:25-194).

    The constructor moves the vertices with |x| < 1e-5 to the end of the vertex list and puts them on
    x = 0 (set_x_boundary); ``perm`` holds the old index of each vertex, ``N_pin`` their number.
    ``phi_init`` / ``psi_init`` (old order) become the initial state, as in the reference's second
    constructor.  Every assembly exchanges the pinned columns of G and H after the 4 pi rule, the
    stages use the stored psi in place of the potential at the pinned vertices, and the pinned
    vertices slide along the wall with the drift velocity ``drift`` = (beta, cos theta_eq, c_nl).
    The wall image is on by default (the reference's MIRROR_MESH build, the setting of its
    pinned-bubble drivers).
    """

    def __init__(self, verts, trigs, p_inf=1.0, epsilon=1.0, sigma=0.0, gamma=1.0, pressurefield=None,
                 device=0, solver="bicgstab", mirror=True, phi_init=None, psi_init=None, drift=DRIFT_LAW):
        n = len(verts)
        phi0 = np.zeros(n) if phi_init is None else np.asarray(phi_init, dtype=np.float64)
        psi0 = np.zeros(n) if psi_init is None else np.asarray(psi_init, dtype=np.float64)
        v, t, self.perm, self.N_pin, phi0, psi0 = move_flagged_to_end(verts, trigs, _on_wall, phi0, psi0)
        super().__init__(v, t, p_inf, epsilon, sigma, gamma, pressurefield, device, solver, mirror)
        self.drift = tuple(float(d) for d in drift)
        self._check(self._L.bem_set_pinned(self._h, int(self.N_pin), *self.drift))
        self.set_phi(phi0)
        self.set_psi(psi0)

    def position_t(self, pot, verts=None, return_psi=False):
        """ColocSimPin::position_t: vertex velocities; ``pot`` (float64, C-contiguous ndarray) receives
        the solved potential at the pinned vertices, as the reference's PotVec& argument does."""
        if not (isinstance(pot, np.ndarray) and pot.dtype == np.float64 and pot.flags.c_contiguous
                and pot.flags.writeable and pot.shape == (self.N,)):
            raise TypeError("pot must be a writable C-contiguous float64 array of N entries")
        vel = np.empty((self.N, 3))
        psi = np.empty(self.N)
        v = None if verts is None else np.ascontiguousarray(verts, dtype=np.float64)
        self._check(self._L.bem_position_t_inout(self._h, _d(v) if v is not None else None, _d(pot), _d(vel),
                                                 _d(psi)))
        return (vel, psi) if return_psi else vel


def measure_fma_peaks(device=0):
    """(FP64, FP32) FMA throughput of `device` in TFLOP/s from the library's FMA-loop kernels."""
    lib = L.load()
    a, b = np.zeros(1), np.zeros(1)
    rc = lib.bem_measure_fma_peaks(int(device), _d(a), _d(b))
    if rc != L.BEM_OK:
        raise L.BemError(rc, "bem_measure_fma_peaks failed")
    return float(a[0]), float(b[0])
