"""Batches of independent bubbles on one GPU (a radius x pressure sweep).

The reference runs a sweep as one process per point (``oscillations-array.sh`` driving
``oscillations.cpp``, each an independent ``ColocSim``).  ``BubbleBatch`` steps all points as one
simulation whose boundary-element systems do not couple: the meshes are concatenated, every
per-vertex and per-triangle kernel of a stage runs once over all bubbles, the influence matrices are
block-diagonal (one persistent assembly launch per stage over every bubble's tiles) and the
mixed-precision solve is batched over the blocks without host synchronisation, so that a whole RK4
step is one CUDA graph.  Each bubble keeps its own V_0 (its initial volume) and its own far-field
pressure ``amp * sin(kx*x + omega*t + phase)``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from . import mesh as _mesh
from .sim import ColocSim, _d


class BubbleBatch(ColocSim):
    """``meshes``: list of (verts (n_b,3), trigs (m_b,3)) pairs, one per bubble.  Physics constants
    as in ColocSim; ``mixed_tol``: relative residual of the batched refinement."""

    def __init__(self, meshes, p_inf=1.0, epsilon=1.0, sigma=0.0, gamma=1.0, device=0, mixed_tol=1e-12):
        self._L = L.load()
        self._h = C.c_void_p()
        self._cb = None
        p = L.Params()
        self._L.bem_default_params(C.byref(p))
        p.p_inf, p.epsilon, p.sigma, p.gamma = float(p_inf), float(epsilon), float(sigma), float(gamma)
        p.mirror = 0
        p.solver = L.SOLVER_MIXED
        p.mixed_tol = float(mixed_tol)
        rc = self._L.bem_create(C.byref(self._h), int(device), C.byref(p))
        if rc != L.BEM_OK:
            raise L.BemError(rc, "bem_create failed (no CUDA device?)")
        v, f = _mesh.join([(np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.int64)) for a, b in meshes])
        sizes = [len(a) for a, _ in meshes]
        self.offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        self.nblocks = len(meshes)
        v = np.ascontiguousarray(v, dtype=np.float64)
        t = np.ascontiguousarray(f, dtype=np.int64)
        self.N, self.M = len(v), len(t)
        self._check(self._L.bem_set_mesh_blocks(self._h, self.N, _d(v), self.M, t.ctypes.data_as(L._I64),
                                                 self.nblocks, self.offsets.ctypes.data_as(L._I64)))

    def block(self, b):
        """Slice of bubble b in the per-vertex arrays."""
        return slice(int(self.offsets[b]), int(self.offsets[b + 1]))

    def set_block_params(self, V0=None, amp=None, kx=None, omega=None, phase=None):
        def arr(a):
            if a is None:
                return None, None
            a = np.ascontiguousarray(np.broadcast_to(np.asarray(a, dtype=np.float64), (self.nblocks,)))
            return a, _d(a)

        keep = [arr(a) for a in (V0, amp, kx, omega, phase)]
        self._check(self._L.bem_set_block_params(self._h, *[k[1] for k in keep]))

    def block_params(self):
        out = {k: np.empty(self.nblocks) for k in ("V0", "amp", "kx", "omega", "phase")}
        self._check(self._L.bem_get_block_params(self._h, *[_d(out[k]) for k in ("V0", "amp", "kx", "omega", "phase")]))
        return out

    def block_stats(self):
        """Per bubble: contraction per refinement step, final relative residual and refinement steps of
        the last batched solve."""
        rho, rel = np.empty(self.nblocks), np.empty(self.nblocks)
        steps = np.empty(self.nblocks, dtype=np.int32)
        self._check(self._L.bem_get_block_stats(self._h, _d(rho), _d(rel), steps.ctypes.data_as(C.POINTER(C.c_int32))))
        return rho, rel, steps

    def evolve_graph(self, dt, steps):
        """``steps`` fixed-dt RK4 steps, each one replay of a captured CUDA graph."""
        self._check(self._L.bem_evolve_rk4_graph(self._h, float(dt), int(steps)))

    def autotune(self):
        """Time the assembly tile shapes on this batch and keep the fastest; returns (width, ms) with ms the
        times of the widths 32, 48, 64 and 16."""
        cg = C.c_int32(0)
        ms = np.empty(4)
        self._check(self._L.bem_autotune_assembly(self._h, C.byref(cg), _d(ms)))
        return int(cg.value), ms

    def assemble_blocks(self, verts=None):
        """Packed G and H blocks: list of (G_b, H_b), each n_b x n_b."""
        tot = int(np.sum(np.diff(self.offsets) ** 2))
        G, H = np.empty(tot), np.empty(tot)
        v = None if verts is None else np.ascontiguousarray(verts, dtype=np.float64)
        self._check(self._L.bem_assemble(self._h, None if v is None else _d(v), _d(G), _d(H)))
        out, o = [], 0
        for b in range(self.nblocks):
            n = int(self.offsets[b + 1] - self.offsets[b])
            out.append((G[o:o + n * n].reshape(n, n, order="F"), H[o:o + n * n].reshape(n, n, order="F")))
            o += n * n
        return out

    def assemble_matrices(self, verts=None):
        """The block-diagonal G and H as their blocks (see assemble_blocks)."""
        return self.assemble_blocks(verts)

    # not offered on a batch
    def set_mirror(self, on):
        if on:
            raise ValueError("batches simulate free-space bubbles")

    def solve_system(self, G, b):
        raise NotImplementedError("a batch solves its blocks internally")

    def set_solver(self, name):
        if name != "mixed":
            raise ValueError("a batch always uses the mixed solver")

    def evolve_system(self, dp, fixdt=False):
        raise NotImplementedError("batches step with RK4 at a fixed dt")
