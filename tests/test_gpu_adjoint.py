"""The adjoint of RK4 trajectories against central finite differences.

The gradient of an objective of the final state (enclosed volume plus a weighted sum of the final
potential) with respect to the initial positions and potential comes from the torch.autograd.Function
over the C ABI's adjoint.  Directional derivatives along seeded random directions are compared with
central differences (h = 1e-6) of the same objective computed by the FP64 paths: the GPU path with
the FP64 LU solver, and on the smallest case the oracle (the CPU restatement of the reference).
Tolerance: 1e-5 relative to the directional derivative.
"""
import ctypes

import numpy as np
import pytest
import torch

import oracle as O
from bem_b200 import mesh
from bem_b200.adjoint import rk4_flow, volume
from bem_b200.sim import ColocSim

pytestmark = pytest.mark.gpu

TOL = 1e-5
H = 1e-6


def setup(nu, seed=0, phi0=0.3):
    rng = np.random.default_rng(seed)
    v, f = mesh.bubble(nu, 1.0, (0.0, 0.0, 0.0))
    v = v * (1.0 + 0.01 * rng.standard_normal(len(v)))[:, None] + np.array([2.0, 0.0, 0.0])
    phi = phi0 + 0.02 * rng.standard_normal(len(v))
    w = rng.standard_normal(len(v))  # weights of the final potential in the objective
    return v, f, phi, w


def objective_np(x, f, phi, w):
    a, b, c = x[f[:, 0]], x[f[:, 1]], x[f[:, 2]]
    return float(np.sum(np.cross(a, b) * c) / 6.0 + 0.1 * np.dot(w, phi))


def adjoint_grad(v, f, phi, w, dt, steps, field=None, **phys):
    sim = ColocSim(v, f, pressurefield=field, solver="mixed", **phys)
    dev = torch.device("cuda:0")
    x0 = torch.tensor(v, dtype=torch.float64, device=dev, requires_grad=True)
    p0 = torch.tensor(phi, dtype=torch.float64, device=dev, requires_grad=True)
    tr = torch.tensor(f, dtype=torch.int64, device=dev)
    wt = torch.tensor(w, dtype=torch.float64, device=dev)
    xK, pK = rk4_flow(sim, x0, p0, dt, steps)
    J = volume(xK, tr) + 0.1 * (wt * pK).sum()
    J.backward()
    return float(J.item()), x0.grad.cpu().numpy(), p0.grad.cpu().numpy()


def fd_gpu(v, f, phi, w, dt, steps, dirs, field=None, **phys):
    sim = ColocSim(v, f, pressurefield=field, solver="lu", **phys)  # V0 = volume of v, held fixed

    def J(x, p):
        sim.set_vertices(x)
        sim.set_phi(p)
        sim.set_time(0.0)
        sim.evolve_rk4_steps(dt, steps)
        return objective_np(sim.get_vertices(), f, sim.get_phi(), w)

    return [(J(v + H * dx, phi + H * dp) - J(v - H * dx, phi - H * dp)) / (2 * H) for dx, dp in dirs]


def directions(n, k, seed=1):
    rng = np.random.default_rng(seed)
    return [(rng.standard_normal((n, 3)), rng.standard_normal(n)) for _ in range(k)]


def check(gx, gp, fd, dirs):
    for (dx, dp), d in zip(dirs, fd):
        ad = float(np.sum(gx * dx) + np.dot(gp, dp))
        assert abs(ad - d) <= TOL * abs(d), (ad, d)


PHYS = dict(p_inf=1.0, epsilon=1.0, sigma=0.0, gamma=1.4)


def test_volume_gradient_entry_point():
    v, f, _, _ = setup(4)
    sim = ColocSim(v, f)
    g = np.empty((len(v), 3))
    sim._check(sim._L.bem_volume_gradient(sim._h, g.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    x = torch.tensor(v, dtype=torch.float64, requires_grad=True)
    volume(x, torch.tensor(f, dtype=torch.int64)).backward()
    assert np.allclose(g, x.grad.numpy(), rtol=0, atol=1e-15)


def test_adjoint_matches_fd_with_field():
    # x-dependent field A sin(kx x + w t) exercises the field term of the Bernoulli equation
    v, f, phi, w = setup(3)
    field = (-0.5, 2 * np.pi / 3, 0.0, 0.3)
    dt, steps = 2e-3, 6
    _, gx, gp = adjoint_grad(v, f, phi, w, dt, steps, field=field, **PHYS)
    dirs = directions(len(v), 6)
    check(gx, gp, fd_gpu(v, f, phi, w, dt, steps, dirs, field=field, **PHYS), dirs)


def test_adjoint_matches_oracle_fd():
    # the FP64 reference gradient: central differences of the oracle (CPU restatement)
    v, f, phi, w = setup(2, seed=3)
    dt, steps = 2e-3, 3
    _, gx, gp = adjoint_grad(v, f, phi, w, dt, steps, **PHYS)
    prm = O.make_params(V0=O.volume(v, f), use_lu=True, **PHYS)

    def J(x, p):
        st = O.State(x, f, p)
        for _ in range(steps):
            st.rk4(dt, prm)
        return objective_np(st.x, f, st.phi, w)

    dirs = directions(len(v), 3, seed=5)
    fd = [(J(v + H * dx, phi + H * dp) - J(v - H * dx, phi - H * dp)) / (2 * H) for dx, dp in dirs]
    check(gx, gp, fd, dirs)


def test_adjoint_config4_mesh():
    # the adjoint configuration's mesh (nu = 10, N = 1002, phi = -R Rdot = 0.3), fewer steps
    v, f = mesh.bubble(10, 1.0, (2.0, 0.0, 0.0))
    phi = np.full(len(v), 0.3)
    w = np.zeros(len(v))
    dt, steps = 2e-3, 8
    _, gx, gp = adjoint_grad(v, f, phi, w, dt, steps, **PHYS)
    dirs = directions(len(v), 4, seed=7)
    check(gx, gp, fd_gpu(v, f, phi, w, dt, steps, dirs, **PHYS), dirs)


def test_adjoint_refuses_wall_treatment_range():
    v, f = mesh.bubble(2, 1.0, (1.005, 0.0, 0.0))  # leftmost vertex at x = 0.005 < 1e-2
    sim = ColocSim(v, f, solver="mixed", **PHYS)
    with pytest.raises(Exception):
        sim._check(sim._L.bem_adjoint_record(sim._h, 1e-3, 2))
