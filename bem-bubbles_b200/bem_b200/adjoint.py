"""Differentiable RK4 trajectories: a torch.autograd.Function over the C ABI's adjoint.

``rk4_flow(sim, x0, phi0, dt, steps)`` maps the initial state (positions N x 3, potential N; FP64
CUDA tensors on the simulation's device) to the state after ``steps`` fixed-dt RK4 steps
(LinLinSim::evolve_system_RK4, LinLinSim.cpp:194-257).  Its backward is the hand-written adjoint in
libbem_b200.so (transposed solves, the assembly's derivative with respect to the vertex positions,
per-step checkpoints with the stages recomputed).  ``volume`` is the enclosed volume of a mesh
(Mesh.cpp:206-218) in torch, so that ``volume(rk4_flow(...)[0], trigs)`` is differentiable end to end.
The tensors' data pointers are passed to the library; no host copies are made.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib as L


def _ptr(t: torch.Tensor):
    return C.c_void_p(t.data_ptr())


class RK4Flow(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x0, phi0, sim, dt, steps):
        if x0.dtype != torch.float64 or phi0.dtype != torch.float64 or not x0.is_cuda:
            raise TypeError("rk4_flow: FP64 CUDA tensors expected")
        x0, phi0 = x0.contiguous(), phi0.contiguous()
        torch.cuda.synchronize(x0.device)
        sim._check(sim._L.bem_set_state_device(sim._h, _ptr(x0), _ptr(phi0)))
        sim._check(sim._L.bem_adjoint_record(sim._h, float(dt), int(steps)))
        xK, phiK = torch.empty_like(x0), torch.empty_like(phi0)
        sim._check(sim._L.bem_get_state_device(sim._h, _ptr(xK), _ptr(phiK)))
        ctx.sim = sim
        return xK, phiK

    @staticmethod
    def backward(ctx, gx, gphi):
        sim = ctx.sim
        ref = gx if gx is not None else gphi
        xb = (gx if gx is not None else torch.zeros((sim.N, 3), dtype=torch.float64, device=ref.device)).contiguous().clone()
        pb = (gphi if gphi is not None else torch.zeros(sim.N, dtype=torch.float64, device=ref.device)).contiguous().clone()
        torch.cuda.synchronize(xb.device)
        sim._check(sim._L.bem_adjoint_backward_device(sim._h, _ptr(xb), _ptr(pb)))
        return xb, pb, None, None, None


def rk4_flow(sim, x0, phi0, dt, steps):
    """State after ``steps`` RK4 steps from (x0, phi0); differentiable with respect to both."""
    return RK4Flow.apply(x0, phi0, sim, dt, steps)


def volume(x: torch.Tensor, trigs: torch.Tensor) -> torch.Tensor:
    """Signed enclosed volume sum over triangles of (a x b).c / 6."""
    a, b, c = x[trigs[:, 0]], x[trigs[:, 1]], x[trigs[:, 2]]
    return (torch.linalg.cross(a, b) * c).sum() / 6.0
