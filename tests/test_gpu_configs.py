"""Parity at the named workload sizes, through the C ABI.

* The headline bubble (icosphere nu=20, N = 4002, seeded 1% radial perturbation): G and H entry by
  entry against the oracle's C restatement of ColocSim::assemble_matrices (ColocSim.cpp:21-110),
  computed on the fly; and the mixed-precision RK4 trajectory against the FP64 BiCGSTAB trajectory
  (the reference's default solver, Simulation.cpp:49-53), two contexts from the same start, the
  dphi/dn error bounded at every step.
* The plain-FP64 two-bubble configuration (main.cpp's set-up, N = 984): all 100 RK4 steps of
  evolve_system_RK4 (LinLinSim.cpp:194-257) with LU against the reference's own trajectory
  (tests/golden/c1_100.npz, made by tests/golden/make_c1_golden.py from the reference build).
* The batched sweep: batched bubble-steps/s at least 3x the same bubbles stepped one after another.
* The large pair (N = 32004): a mixed-precision RK4 step, psi against the FP64 BiCGSTAB solve.
"""
import os

import numpy as np
import pytest

import bench
import oracle as O
from bem_b200.sim import ColocSim

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_headline_mesh_assembly_matches_oracle():
    # entry-wise G and H at N = 4002 against the oracle (the bit-exact C restatement), 1e-13 relative
    v, f = bench.workload()
    sim = ColocSim(v, f, **bench.PHYS)
    G, H = sim.assemble_matrices()
    sim.close()
    Go, Ho = O.assemble(v, f)
    assert rel(G, Go) <= 1e-13
    assert rel(H, Ho) <= 1e-13


def test_headline_mixed_trajectory_tracks_fp64_trajectory():
    # 20 RK4 steps of the headline workload (dt = 5e-3, oscillating far field) in two contexts, the
    # mixed-precision path and the FP64 BiCGSTAB path; dphi/dn (psi) within 1e-8 of the FP64 path at
    # every step, positions and potential within 1e-10
    v, f = bench.workload()
    mix = ColocSim(v, f, pressurefield=bench.FIELD, solver="mixed", **bench.PHYS)
    ref = ColocSim(v, f, pressurefield=bench.FIELD, solver="bicgstab", **bench.PHYS)
    worst = {"x": 0.0, "phi": 0.0, "psi": 0.0}
    for sim in (mix, ref):
        sim.set_phi(0.0)
    for step in range(20):
        for sim in (mix, ref):
            sim.evolve_system_RK4(bench.DT, fixdt=True)
        xm, pm, sm, tm = mix.get_state()
        x6, p6, s6, t6 = ref.get_state()
        assert tm == t6
        e = {"x": rel(xm, x6), "phi": rel(pm, p6), "psi": rel(sm, s6)}
        for k in worst:
            worst[k] = max(worst[k], e[k])
        assert e["psi"] <= 1e-8, (step, e)
        assert e["x"] <= 1e-10 and e["phi"] <= 1e-10, (step, e)
    mix.close()
    ref.close()


def test_config1_100_steps_match_reference():
    from bem_b200 import mesh

    gold = np.load(os.path.join(HERE, "golden", "c1_100.npz"))
    a = mesh.bubble(7, 1.0, (2.5, 0.0, 0.0))
    b = mesh.bubble(7, 1.0, (5.5, 0.0, 0.0))
    v, f = mesh.join([a, b])
    n = len(a[0])
    sim = ColocSim(v, f, p_inf=1.0, epsilon=0.0, sigma=0.0, gamma=1.0, solver="lu")
    sim.set_phi(np.r_[np.full(n, -0.5), np.full(n, 0.5)])
    keep = {int(s): r for s, r in zip(gold["steps"], gold["records"])}
    N = len(v)
    for step in range(1, 101):
        sim.evolve_system_RK4(1e-3, fixdt=True)
        if step in keep:
            x, phi, psi, t = sim.get_state()
            r = keep[step]
            assert rel(x, r[:3 * N].reshape(N, 3)) <= 1e-10, step
            assert rel(phi, r[3 * N:4 * N]) <= 1e-10, step
            assert rel(psi, r[4 * N:5 * N]) <= 1e-10, step
            assert abs(t - r[5 * N]) <= 1e-12, step
    assert sorted(keep) == [25, 50, 75, 100]
    sim.close()


def test_batched_sweep_at_least_3x_sequential():
    # 64 bubbles of the radius x pressure sweep (nu ~ U{4..16}, seed 0), 3 timed RK4 steps at dt = 2e-3:
    # the batch (one CUDA graph per step) against the same bubbles stepped one after another through
    # the single-bubble mixed path, both timed on the device after two warm-up steps
    import torch

    from bem_b200.batch import BubbleBatch

    dt, steps = 2e-3, 3
    meshes, _, _, amp, om = bench.sweep_workload(64)
    phys = dict(p_inf=1.0, epsilon=1.0, sigma=0.0, gamma=1.4)

    def timed(stream, fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b)

    bb = BubbleBatch(meshes, **phys)
    bb.set_block_params(amp=amp, omega=om)
    bb.evolve_graph(dt, 2)
    bb.sync()
    ext = torch.cuda.ExternalStream(bb.stream_handle())
    batched = len(meshes) * steps / timed(ext, lambda: bb.evolve_graph(dt, steps))
    bb.close()
    seq_ms = 0.0
    for b, (v, f) in enumerate(meshes):
        sim = ColocSim(v, f, pressurefield=(float(amp[b]), float(om[b]), 0.0), solver="mixed", **phys)
        sim.evolve_rk4_steps(dt, 2)
        sim.sync()
        sext = torch.cuda.ExternalStream(sim.stream_handle())
        seq_ms += timed(sext, lambda: [sim.evolve_system_RK4(dt, fixdt=True) for _ in range(steps)])
        sim.close()
    sequential = len(meshes) * steps / seq_ms
    assert batched >= 3.0 * sequential, (batched * 1e3, sequential * 1e3)


def test_large_pair_mixed_step_matches_fp64():
    # the two-bubble pair at N = 32004 (two icospheres nu=40): one mixed-precision RK4 step, then psi
    # of the mixed solve on the new state against the FP64 BiCGSTAB solve, <= 1e-8 relative
    v, f, phi = bench.pair_workload()
    sim = ColocSim(v, f, p_inf=1.0, epsilon=0.0, sigma=0.0, gamma=1.0, solver="mixed")
    sim.set_phi(phi)
    sim.evolve_system_RK4(1e-3, fixdt=True)
    ph = sim.get_phi()
    _, psi_mix = sim.position_t(ph, return_psi=True)
    sim.set_solver("bicgstab")
    _, psi64 = sim.position_t(ph, return_psi=True)
    st = sim.stats()
    sim.close()
    assert st.gj_inverses == 1  # the set-up of the inverse at this size: tensor-core Gauss-Jordan
    assert st.last_rel_residual <= 1e-14
    assert rel(psi_mix, psi64) <= 1e-8
