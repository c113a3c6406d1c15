"""Benchmark of the BEM hot path on B200: RK4 steps/s of one N=4002 bubble.

Workload (the headline configuration): one bubble, icosphere nu=20 (N=4002 vertices, M=8000
triangles), R0=1 centred at (2,0,0), 1% radial perturbation N(0, 0.01^2) per vertex (seed 0),
phi=0, p_inf=1, epsilon=1, gamma=1.4, sigma=0, far-field pressure -0.8*sin(2*pi*t/5), dt=5e-3,
fixed step, no wall image.  A "step" is one RK4 step (4 stages of assembly + solve + update).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--solver mixed|bicgstab|lu]
                  [--workload headline|pair|sweep|adjoint]

--workload pair runs the large two-bubble pair instead (two icospheres nu=40, N=32004 unknowns,
radii 1.0 and 0.7, centres (2,0,0) and (4.2,0,0), phi = +0.4 and -0.14, epsilon=0, no field,
dt=1e-3): mixed-precision RK4 steps/s, with the error of psi against the FP64 BiCGSTAB path on the
same GPU at the first and the last state, and the one-time set-up of the approximate inverse.

--workload sweep runs the batched parameter sweep: 256 independent bubbles, icosphere nu ~ U{4..16},
R0 log-uniform in [0.5, 2] centred at (R0 + 1, 0, 0), far field -A sin(2 pi t/T) with A ~ U[0.1, 1.5],
T ~ U[2, 10] (seed 0), phi = 0, epsilon = 1, gamma = 1.4, dt = 2e-3, mixed precision: bubble-steps/s of
the batch (one CUDA graph per RK4 step, tile shape from the autotuner) against the same bubbles
stepped one after another through the single-bubble path.

--workload adjoint: one bubble, icosphere nu=10 (N=1002) at (2,0,0), phi = -R Rdot = 0.3, epsilon=1,
gamma=1.4, p_inf=1, no field; objective the enclosed volume after 50 RK4 steps at dt=2e-3; gradient
with respect to the initial positions and potential through the torch.autograd.Function over the
adjoint, against central differences (h=1e-6) of the FP64 BiCGSTAB GPU path on 32 seeded directions.

ours: the mixed-precision path (FP64 assembly, FP64 GMRES, FP32 approximate-inverse preconditioner)
through libbem_b200.so.  value = device time of K steps with the state resident in HBM (CUDA events
on the library's stream, max over ranks); e2e = the same K steps through the C ABI with host
buffers, the step's state copied in from pinned memory and the result copied back every step.
Beside it: the all-FP64 GPU paths (BiCGSTAB, the reference's default, and LU) each in its own
context over the same warm-up and K-step window from the same initial state; the mixed trajectory
against the FP64 one step by step; the one-time set-up of the approximate inverse.
reference: the reference's own CPU code (oracle/_ref, built from the reference sources) on all host
cores: real RK4 steps (evolve_system_RK4 with its default BiCGSTAB solve) after untimed warm-up
steps, up to K timed steps within about two minutes; `steps` is the number actually timed.  With
--gpus N > 1 every rank runs an independent replica (the path does not shard: replicas only);
rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "bem-bubbles_b200"))

METRIC = "RK4 steps/s at N=4002: mixed-precision vs FP64 GPU at <=1e-8 rel dphi/dn error"
NU, DT = 20, 5e-3
PHYS = dict(p_inf=1.0, epsilon=1.0, sigma=0.0, gamma=1.4)
FIELD = (-0.8, 2.0 * np.pi / 5.0, 0.0)


def workload():
    from bem_b200 import mesh

    v, f = mesh.bubble(NU, 1.0, (0.0, 0.0, 0.0))
    rng = np.random.default_rng(0)
    v = v * (1.0 + 0.01 * rng.standard_normal(len(v)))[:, None] + np.array([2.0, 0.0, 0.0])
    return v, f


def pair_workload():
    from bem_b200 import mesh

    va, fa = mesh.bubble(40, 1.0, (2.0, 0.0, 0.0))
    vb, fb = mesh.bubble(40, 0.7, (4.2, 0.0, 0.0))
    v, f = mesh.join([(va, fa), (vb, fb)])
    phi = np.concatenate([np.full(len(va), 0.4), np.full(len(vb), -0.14)])
    return v, f, phi


def sweep_workload(nb=256, seed=0):
    from bem_b200 import mesh

    rng = np.random.default_rng(seed)
    nus = rng.integers(4, 17, size=nb)
    R0 = np.exp(rng.uniform(np.log(0.5), np.log(2.0), size=nb))
    A = rng.uniform(0.1, 1.5, size=nb)
    T = rng.uniform(2.0, 10.0, size=nb)
    meshes = [mesh.bubble(int(nu), float(r), (float(r) + 1.0, 0.0, 0.0)) for nu, r in zip(nus, R0)]
    return meshes, nus, R0, -A, 2.0 * np.pi / T


def max_over_ranks(x, dist, device=None):
    """Largest value of x over all ranks (the timing rule for replicas); x itself without a group."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(ws, steps, elapsed_ms):
    """Whole-job throughput of ws replicas, each taking `steps` steps, timed as the slowest rank."""
    return ws * steps / (elapsed_ms * 1e-3)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def read_traffic():
    """DRAM bytes per launch of the assembly tile kernel from the committed ncu summary (profiles/), or None."""
    p = os.path.join(ROOT, "profiles", "assemble_patch_nu20_ncu.md")
    try:
        for line in open(p):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region (every 20 ms;
    the sampler is running before the region starts, and only samples taken inside it count -- or,
    for a region shorter than one interval, the sample taken right before it)."""

    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.first = threading.Event()
        self.begin = self.end = 0

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            self.first.wait(3.0)
        except OSError:
            self.proc = None
        self.begin = len(self.lines)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())
            self.first.set()

    def __exit__(self, *a):
        self.end = len(self.lines)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def window(self):
        w = self.lines[self.begin:self.end]
        if not w and self.begin > 0:
            w = self.lines[self.begin - 1:self.begin]
        return w

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.window():
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 6:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[2:]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


class NvmlClockSampler:
    """NVML sampling of the SM clock and the clock-event reasons every 2 ms (read-only queries), for
    timed regions too short for nvidia-smi's interval; same summary as ClockSampler."""

    PERIOD_S = 0.002

    def __init__(self, index):
        import pynvml

        self.nv = pynvml
        pynvml.nvmlInit()
        self.h = pynvml.nvmlDeviceGetHandleByIndex(int(index))
        self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
        self.samples = []
        self.stop = threading.Event()
        self.begin = self.end = 0

    def _run(self):
        nv = self.nv
        while not self.stop.is_set():
            try:
                mhz = float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                mask = int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))
                self.samples.append((mhz, mask))
            except nv.NVMLError:
                pass
            time.sleep(self.PERIOD_S)

    def __enter__(self):
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()
        t0 = time.time()
        while not self.samples and time.time() - t0 < 3.0:
            time.sleep(0.001)
        self.begin = len(self.samples)
        return self

    def __exit__(self, *a):
        self.end = len(self.samples)
        self.stop.set()
        self.t.join(timeout=1.0)

    def summary(self):
        nv = self.nv
        w = self.samples[self.begin:self.end] or self.samples[max(0, self.begin - 1):self.begin]
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        reasons = sorted({k for _, m in w for k, b in bits.items() if m & b})
        sm = [mhz for mhz, _ in w]
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(sm), "source": "nvml"}


def clock_sampler(index):
    """NVML sampler when the bindings are present, else nvidia-smi."""
    try:
        return NvmlClockSampler(index)
    except Exception:
        return ClockSampler(index)


def headline_config(ws):
    """The workload description both arms report (the same dict, so the arms compare like for like)."""
    return {"workload": "single bubble icosphere nu=20 (N=4002, M=8000), R0=1 at (2,0,0), 1% radial perturbation "
                        "(seed 0), phi=0, p_inf=1, epsilon=1, gamma=1.4, RK4 dt=5e-3 fixed, "
                        "p(t)=1-0.8 sin(2 pi t/5)",
            "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
            "l2": "working set larger than L2 (G+H = 256 MB per stage)"}


REF_SOLVER = "BiCGSTAB (the reference default: Jacobi preconditioner, tolerance machine epsilon, <= 2N iterations)"


def cpu_reference_steps(warm, steps, threads, budget_s):
    """Real RK4 steps (evolve_system_RK4 with its default BiCGSTAB solve) of the reference's own code
    (oracle/_ref) on `threads` host threads: `warm` untimed steps from the workload's initial state
    (phi = 0, so the first stage's right-hand side is zero; later stages and steps solve in earnest),
    then up to `steps` timed ones, stopping once budget_s seconds of timed steps are spent.  None when
    the reference build is absent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    if not O.ref_available(False):
        return None
    v, f = workload()
    return O.ref_rk4_timed(v, f, np.zeros(len(v)), warm=warm, steps=steps, budget=budget_s, dt=DT, fixdt=1,
                           lu=0, V0=O.volume(v, f), amp=FIELD[0], omega=FIELD[1], phase=FIELD[2],
                           threads=threads, **PHYS)


def ref_sample_text(r, warm, threads):
    k = len(r["seconds"])
    return (f"{k} timed RK4 steps of the reference code (oracle/_ref: evolve_system_RK4, {REF_SOLVER}) after "
            f"{warm} untimed steps from the workload's initial state, {threads} OpenMP threads; "
            f"{int(r['solves'].sum())} BiCGSTAB solves, mean {float(r['iters'].sum()) / max(1, int(r['solves'].sum())):.1f} "
            f"iterations per solve")


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    # warm-up as in our arm (capped: a reference step takes seconds), then the K timed steps, bounded
    # to about two minutes of timed work
    warm = min(args.warmup, 5)
    r = cpu_reference_steps(warm, args.steps, threads, budget_s=120.0)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (reference checkout absent at build time)"}))
        return 0
    k = len(r["seconds"])
    total_s = float(r["seconds"].sum())
    value = k / total_s
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": args.gpus, "steps": k,
        "warmup": warm, "ms_per_step": total_s / k * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference", "solver": REF_SOLVER,
        "config": headline_config(1),
        "bicgstab": {"solves": int(r["solves"].sum()), "iterations": int(r["iters"].sum()),
                     "iters_per_solve": float(r["iters"].sum()) / max(1, int(r["solves"].sum()))},
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": threads, "kind": "reference",
                         "sample": ref_sample_text(r, warm, threads)},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def fp64_comparator(solver, device, warmup, steps):
    """Steps/s of an all-FP64 solver path on the GPU ("bicgstab": the reference's default solver, "lu":
    its PartialPivLU option) in a context of its own, from the workload's initial state, with the same
    warm-up and timed window as the mixed arm (CUDA events on the library's stream)."""
    import torch

    from bem_b200.sim import ColocSim

    v, f = workload()
    sim = ColocSim(v, f, pressurefield=FIELD, solver=solver, device=device, **PHYS)
    sim.set_phi(0.0)
    ext = torch.cuda.ExternalStream(sim.stream_handle(), device=device)
    for _ in range(warmup):
        sim.evolve_rk4_steps(DT, 1)
    sim.sync()
    st0 = sim.stats()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(ext)
    sim.evolve_rk4_steps(DT, steps)
    b.record(ext)
    b.synchronize()
    ms = a.elapsed_time(b) / steps
    st1 = sim.stats()
    sim.close()
    out = {"solver": solver, "ms_per_step": ms, "steps_per_s": 1e3 / ms, "steps": steps, "warmup": warmup}
    if solver == "bicgstab":
        solves = int(st1.solves - st0.solves)
        out["iters_per_solve"] = float(st1.total_iters - st0.total_iters) / max(1, solves)
    return out


def trajectory_error(device, steps):
    """Mixed-precision trajectory against the FP64 BiCGSTAB trajectory: two contexts from the workload's
    initial state, `steps` RK4 steps each, the state read after every step.  Returns the largest
    relative difference over the steps of psi (dphi/dn), of x and of phi (max-norm relative to the
    FP64 path's max |.|)."""
    from bem_b200.sim import ColocSim

    v, f = workload()
    sims = [ColocSim(v, f, pressurefield=FIELD, solver=s, device=device, **PHYS) for s in ("mixed", "bicgstab")]
    worst = {"psi": 0.0, "x": 0.0, "phi": 0.0}
    per_step_psi = []
    for sim in sims:
        sim.set_phi(0.0)
    for _ in range(steps):
        st = []
        for sim in sims:
            sim.evolve_system_RK4(DT, fixdt=True)
            st.append(sim.get_state())
        (xm, pm, sm, _), (x6, p6, s6, _) = st
        e = {"x": np.max(np.abs(xm - x6)) / np.max(np.abs(x6)),
             "phi": np.max(np.abs(pm - p6)) / max(np.max(np.abs(p6)), 1e-300),
             "psi": np.max(np.abs(sm - s6)) / max(np.max(np.abs(s6)), 1e-300)}
        per_step_psi.append(float(e["psi"]))
        for k in worst:
            worst[k] = max(worst[k], float(e[k]))
    for sim in sims:
        sim.close()
    return {"steps": steps, "max_rel_err": worst, "psi_last_step": per_step_psi[-1],
            "target_psi": 1e-8, "fp64_solver": "bicgstab"}


def run_ours(args):
    ws, rank, local = dist_env()
    import torch

    dist = None
    if ws > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta

        dist = dist_mod
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    device = local if ws > 1 else 0
    torch.cuda.set_device(device)

    from bem_b200.sim import ColocSim, measure_fma_peaks

    v, f = workload()
    N, M = len(v), len(f)
    sim = ColocSim(v, f, pressurefield=FIELD, solver=args.solver, device=device, **PHYS)
    if args.inverse != "auto":  # how the mixed solver builds its approximate inverse from scratch
        from bem_b200 import _lib as L

        sim._update(flags=L.FLAG_INVERSE_GJ if args.inverse == "gj" else L.FLAG_INVERSE_NS)
    sim.set_phi(0.0)
    ext = torch.cuda.ExternalStream(sim.stream_handle(), device=device)

    # warm-up; the first step also builds the approximate inverse (the mixed path's one-time set-up),
    # timed on its own
    ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sim.sync()
    ea.record(ext)
    sim.evolve_rk4_steps(DT, 1)
    eb.record(ext)
    eb.synchronize()
    first_step_ms = ea.elapsed_time(eb)
    for _ in range(args.warmup - 1):
        sim.evolve_rk4_steps(DT, 1)
    sim.sync()
    start_state = sim.get_state()  # the e2e leg below runs the same window of the trajectory

    # ---- timed region: K steps, state resident in HBM
    fp64_peak, fp32_peak = measure_fma_peaks(device)
    sim.set_profiling(True)
    sim.reset_profile()
    st0 = sim.stats()
    if dist:
        dist.barrier()
    torch.cuda.synchronize(device)
    sim.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with clock_sampler(device) as clk:
        torch.cuda.nvtx.range_push("timed_region")
        e0.record(ext)
        sim.evolve_rk4_steps(DT, args.steps)
        e1.record(ext)
        e1.synchronize()
        torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize(device)
    elapsed_ms = e0.elapsed_time(e1)
    prof = sim.profile()
    st1 = sim.stats()
    sim.set_profiling(False)
    if dist:
        elapsed_ms = max_over_ranks(elapsed_ms, dist, f"cuda:{device}")
        dist.barrier()
    value = replica_value(ws, args.steps, elapsed_ms)
    ms_per_step = elapsed_ms / args.steps

    # ---- end to end through the C ABI with host buffers (pinned), copies inside the timed region;
    # from the state the timed region started from (the same K steps of the trajectory)
    hx = torch.empty((N, 3), dtype=torch.float64, pin_memory=True).numpy()
    hphi = torch.empty(N, dtype=torch.float64, pin_memory=True).numpy()
    hpsi = torch.empty(N, dtype=torch.float64, pin_memory=True).numpy()
    hx[:], hphi[:], hpsi[:] = start_state[0], start_state[1], start_state[2]
    sim.set_state(hx, hphi, hpsi, start_state[3])
    e2e_steps = args.steps
    if dist:
        dist.barrier()
    tw0 = time.perf_counter()
    for _ in range(e2e_steps):
        sim.set_state(hx, hphi, hpsi)
        sim.evolve_system_RK4(DT, fixdt=True)
        sim.get_state(out=(hx, hphi, hpsi))
    e2e_s = time.perf_counter() - tw0
    if dist:
        e2e_s = max_over_ranks(e2e_s, dist, f"cuda:{device}")
    e2e_value = ws * e2e_steps / e2e_s
    h2d = N * 3 * 8 + 2 * N * 8
    d2h = N * 3 * 8 + 2 * N * 8

    # accuracy of one solve on the current state: the mixed solve first (warm-started from its own
    # previous stage, as in the timed steps), then the FP64 BiCGSTAB solve (zero start) of the same system
    phi_now = sim.get_phi()
    _, psimx = sim.position_t(phi_now, return_psi=True)
    sim.set_solver("bicgstab")
    _, psi64 = sim.position_t(phi_now, return_psi=True)
    psi_err = float(np.max(np.abs(psimx - psi64)) / max(np.max(np.abs(psi64)), 1e-300))
    sim.close()

    # the all-FP64 paths on the same GPU, each in its own context over the same window, and the
    # mixed trajectory against the FP64 one step by step
    fp64 = {s: fp64_comparator(s, device, args.warmup, args.steps) for s in ("bicgstab", "lu")}
    best64 = max(fp64.values(), key=lambda d: d["steps_per_s"])
    traj = trajectory_error(device, args.warmup + args.steps)

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0

    # roofline of the dominant kernel (the assembly tile kernel): algorithmic FLOPs per launch
    evals = (N * M - 3 * M) * 7
    flops = 32.0 * evals
    avg_asm_ms = prof.assemble_ms / max(prof.assemble_launches, 1)
    achieved = flops / (avg_asm_ms * 1e-3) / 1e12
    traffic = read_traffic()

    # CPU baseline: the reference's own RK4 steps on the host cores, a bounded sample
    cpu = None
    if ws == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        os.environ["OMP_NUM_THREADS"] = str(threads)
        r = cpu_reference_steps(1, 3, threads, budget_s=20.0)
        if r is not None:
            cpu = {"value": len(r["seconds"]) / float(r["seconds"].sum()), "unit": "steps/s", "cores": threads,
                   "kind": "reference", "sample": ref_sample_text(r, 1, threads)}

    setup_ms = max(first_step_ms - ms_per_step, 0.0)
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 (assembly, residual, state) + f32 (preconditioner)",
        "data": "synthetic", "solver": args.solver,
        "config": dict(headline_config(ws), **({"inverse": args.inverse} if args.inverse != "auto" else {})),
        "fp64_gpu": fp64["bicgstab"],
        "fp64_lu_gpu": fp64["lu"],
        "speedup_vs_fp64_gpu": value / ws / fp64["bicgstab"]["steps_per_s"],
        "speedup_vs_best_fp64_gpu": {"solver": best64["solver"], "ratio": value / ws / best64["steps_per_s"]},
        "psi_rel_err_vs_fp64": psi_err,
        "trajectory_vs_fp64": traj,
        "setup": {"first_step_ms": first_step_ms, "setup_ms": setup_ms,
                  "steps_per_s_incl_setup": args.steps / ((elapsed_ms / ws + setup_ms) * 1e-3),
                  "note": "setup_ms = first warm-up step (builds the approximate inverse) minus a timed step"},
        "during_timed_steps": {"solves": int(st1.solves - st0.solves),
                               "refinement_steps_per_solve": float(st1.total_iters - st0.total_iters) /
                               max(1, int(st1.solves - st0.solves)),
                               "newton_schulz_steps": int(st1.ns_steps - st0.ns_steps),
                               "refreshes": int(st1.precond_refresh - st0.precond_refresh)},
        "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(prof.kernel_launches),
        "roofline": {"bound": "fp64-fma", "kernel": "k_patch_records + k_assemble_patch + k_rhs_finish (G-only assembly: records with the singular pairs, triangle-patch tiles with the shared columns summed, row partials of b with the 4 pi term); traffic: the tile kernel", "achieved": achieved,
                     "peak": fp64_peak, "unit": "TFLOP/s", "frac": achieved / fp64_peak, "traffic": traffic,
                     "peak_source": "measured live: FP64 FMA-loop kernel (bem_measure_fma_peaks)",
                     "flops_per_launch": flops, "avg_launch_ms": avg_asm_ms,
                     "assemble_share_of_step": prof.assemble_ms / elapsed_ms},
        "fp32_fma_peak_tflops": fp32_peak,
        "clocks": clk.summary(),
    }
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()
    return 0


def run_pair(args):
    """Large two-bubble pair (N = 32004): replicas only, rank 0 reports."""
    ws, rank, local = dist_env()
    import torch

    device = local if ws > 1 else 0
    torch.cuda.set_device(device)
    from bem_b200.sim import ColocSim

    dt = 1e-3
    v, f, phi0 = pair_workload()
    N = len(v)
    sim = ColocSim(v, f, p_inf=1.0, epsilon=0.0, sigma=0.0, gamma=1.0, solver="mixed", device=device)
    sim.set_phi(phi0)
    ext = torch.cuda.ExternalStream(sim.stream_handle(), device=device)

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        sim.sync()
        a.record(ext)
        out = fn()
        b.record(ext)
        b.synchronize()
        return out, a.elapsed_time(b)

    # one-time set-up: the first mixed solve (zero start) builds the approximate inverse from scratch
    (_, psi_cold), setup_ms = timed(lambda: sim.position_t(phi0, return_psi=True))
    setup_ns = int(sim.stats().ns_steps)
    for _ in range(args.warmup):
        sim.evolve_rk4_steps(dt, 1)
    st0 = sim.stats()
    with clock_sampler(device) as clk:
        _, el = timed(lambda: sim.evolve_rk4_steps(dt, args.steps))
    st1 = sim.stats()

    def rel(a, b):
        return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))

    # end state: mixed solve (warm-started from its own last stage), then FP64 BiCGSTAB (zero start)
    ph = sim.get_phi()
    (_, pmx), stagemx_ms = timed(lambda: sim.position_t(ph, return_psi=True))
    sim.set_solver("bicgstab")
    (_, p64), stage64_ms = timed(lambda: sim.position_t(ph, return_psi=True))
    it64 = int(sim.stats().last_iters)
    err_end = rel(pmx, p64)
    # initial state: the cold first mixed solve against FP64 on the same state
    sim.set_vertices(v)
    (_, p64_0), _ = timed(lambda: sim.position_t(phi0, return_psi=True))
    err_init = rel(psi_cold, p64_0)
    if rank != 0:
        return 0
    value = ws * args.steps / (el * 1e-3)
    line = {
        "metric": "RK4 steps/s at N=32004 (two-bubble pair): mixed precision, psi error vs FP64 BiCGSTAB",
        "value": value, "unit": "steps/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": el / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 (assembly, residual, state) + f32 (preconditioner)", "data": "synthetic",
        "config": {"workload": "two icospheres nu=40 (N=32004, M=64000), radii 1.0/0.7, centres 2.2 apart, "
                               "phi=+0.4/-0.14, epsilon=0, RK4 dt=1e-3", "solver": "mixed",
                   "l2": "working set larger than L2 (G+H = 16.4 GB per stage)"},
        "psi_rel_err_vs_fp64": {"initial_state_cold_start": err_init, "after_timed_steps": err_end},
        "fp64_bicgstab": {"stage_ms": stage64_ms, "iters": it64, "steps_per_s_est": 1e3 / (4.0 * stage64_ms)},
        "mixed_stage_ms": stagemx_ms,
        "setup": {"first_solve_ms": setup_ms, "newton_schulz_steps": setup_ns},
        "during_timed_steps": {"ns_steps": int(st1.ns_steps - st0.ns_steps),
                               "refreshes": int(st1.precond_refresh - st0.precond_refresh),
                               "gmres_fallbacks": int(st1.gmres_fallbacks - st0.gmres_fallbacks)},
        "clocks": clk.summary(),
    }
    print(json.dumps(line))
    return 0


def run_lu(args):
    """FP64 LU solve (the reference's PartialPivLU option, Simulation.cpp:57-60) of the headline G."""
    ws, rank, local = dist_env()
    import torch

    device = local if ws > 1 else 0
    torch.cuda.set_device(device)
    from bem_b200.sim import ColocSim, measure_fma_peaks

    v, f = workload()
    N = len(v)
    sim = ColocSim(v, f, solver="lu", device=device, **PHYS)
    phi = np.cos(v[:, 0]) + 0.1 * v[:, 1]
    G, b = sim.assemble_rhs(phi)
    fp64_peak, _ = measure_fma_peaks(device)
    for _ in range(args.warmup):
        sim.solve_system(G, b)
    sim.set_profiling(True)
    sim.reset_profile()
    with clock_sampler(device) as clk:
        for _ in range(args.steps):
            x = sim.solve_system(G, b)
    prof = sim.profile()
    sim.set_profiling(False)
    ms = prof.solve_ms / max(1, prof.solve_calls)
    res = float(np.linalg.norm(G @ x - b) / (np.linalg.norm(G, 1) * np.linalg.norm(x)))
    if rank != 0:
        return 0
    flops = 2.0 / 3.0 * N ** 3 + 4.0 * N ** 2  # factorisation + the two triangular solves
    achieved = flops / (ms * 1e-3) / 1e12
    line = {
        "metric": "FP64 LU solve of G at N=4002 (PartialPivLU option): device time per solve",
        "value": ms, "unit": "ms", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "G of the headline mesh (icosphere nu=20, N=4002), b = H phi with phi = cos x + 0.1 y; "
                               "factorisation and triangular solves, device-resident G (the copy-in excluded)",
                   "solver": "lu"},
        "scaled_residual": res,
        "roofline": {"bound": "fp64-fma", "kernel": "k_lu_panel_cluster + k_lu_update + k_lu_trsm + k_trsv_*",
                     "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s", "frac": achieved / fp64_peak,
                     "flops_per_solve": flops},
        "gpu_launches": int(prof.kernel_launches / max(1, prof.solve_calls)),
        "clocks": clk.summary(),
    }
    print(json.dumps(line))
    return 0


def run_sweep(args):
    """Batched radius x pressure sweep (256 bubbles): replicas only, rank 0 reports."""
    ws, rank, local = dist_env()
    import torch

    device = local if ws > 1 else 0
    torch.cuda.set_device(device)
    from bem_b200.batch import BubbleBatch
    from bem_b200.sim import ColocSim

    dt = 2e-3
    phys = dict(p_inf=1.0, epsilon=1.0, sigma=0.0, gamma=1.4)
    meshes, nus, R0, amp, om = sweep_workload(args.bubbles)
    nb = len(meshes)
    bb = BubbleBatch(meshes, device=device, **phys)
    bb.set_block_params(amp=amp, omega=om)
    ext = torch.cuda.ExternalStream(bb.stream_handle(), device=device)

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        bb.sync()
        a.record(ext)
        fn()
        b.record(ext)
        b.synchronize()
        return a.elapsed_time(b)

    tw = time.perf_counter()
    cg, tune_ms = bb.autotune()
    tune_s = time.perf_counter() - tw
    tw = time.perf_counter()
    bb.evolve_graph(dt, 1)  # approximate inverses of every bubble + graph capture + one step
    bb.sync()
    setup_s = time.perf_counter() - tw
    for _ in range(args.warmup):
        bb.evolve_graph(dt, 1)
    st0 = bb.stats()
    bb.reset_profile()
    with clock_sampler(device) as clk:
        el = timed(lambda: bb.evolve_graph(dt, args.steps))
    launches = int(bb.profile().kernel_launches)
    st1 = bb.stats()
    value = ws * nb * args.steps / (el * 1e-3)

    # end to end through the public API with host buffers (pinned), copies inside the timed region
    N = bb.N
    hx = torch.empty((N, 3), dtype=torch.float64, pin_memory=True).numpy()
    hphi = torch.empty(N, dtype=torch.float64, pin_memory=True).numpy()
    hpsi = torch.empty(N, dtype=torch.float64, pin_memory=True).numpy()
    hx[:], hphi[:], hpsi[:] = bb.get_vertices(), bb.get_phi(), bb.get_psi()
    tw = time.perf_counter()
    for _ in range(args.steps):
        bb.set_vertices(hx)
        bb.set_phi(hphi)
        bb.set_psi(hpsi)
        bb.evolve_graph(dt, 1)
        hx[:], hphi[:], hpsi[:] = bb.get_vertices(), bb.get_phi(), bb.get_psi()
    e2e_value = ws * nb * args.steps / (time.perf_counter() - tw)

    # assembly kernel alone (one plain, profiled step), for the roofline
    bb.set_profiling(True)
    bb.reset_profile()
    bb.evolve_rk4_steps(dt, 1)
    prof = bb.profile()
    bb.set_profiling(False)
    avg_asm_ms = prof.assemble_ms / max(prof.assemble_launches, 1)
    flops = sum(32.0 * (len(v) * len(f) - 3 * len(f)) * 7 for v, f in meshes)
    from bem_b200.sim import measure_fma_peaks

    fp64_peak, _ = measure_fma_peaks(device)
    achieved = flops / (avg_asm_ms * 1e-3) / 1e12

    # accuracy: batched psi against the FP64 BiCGSTAB single-bubble path on the same state
    X, P = bb.get_vertices(), bb.get_phi()
    _, psib = bb.position_t(P, return_psi=True)
    errs = []
    for b in np.linspace(0, nb - 1, 8).astype(int):
        sl = bb.block(b)
        sim = ColocSim(X[sl], meshes[b][1], solver="bicgstab", device=device, **phys)
        _, p64 = sim.position_t(P[sl], return_psi=True)
        errs.append(float(np.max(np.abs(psib[sl] - p64)) / max(np.max(np.abs(p64)), 1e-300)))
        sim.close()

    # sequential baseline: every bubble on its own through the single-bubble mixed path
    seq_steps, seq_ms, seq_setup = 3, 0.0, 0.0
    if not args.no_seq:
        for b, (v, f) in enumerate(meshes):
            sim = ColocSim(v, f, pressurefield=(float(amp[b]), float(om[b]), 0.0), solver="mixed", device=device,
                           **phys)
            sext = torch.cuda.ExternalStream(sim.stream_handle(), device=device)
            tw = time.perf_counter()
            sim.evolve_rk4_steps(dt, 2)
            sim.sync()
            seq_setup += time.perf_counter() - tw
            a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(sext)
            for _ in range(seq_steps):
                sim.evolve_system_RK4(dt, fixdt=True)
            e.record(sext)
            e.synchronize()
            seq_ms += a.elapsed_time(e)
            sim.close()
    seq_value = nb * seq_steps / (seq_ms * 1e-3) if seq_ms > 0 else None
    if rank != 0:
        return 0
    Ns = np.array([len(v) for v, _ in meshes])
    line = {
        "metric": f"bubble RK4 steps/s, {nb}-bubble radius x pressure sweep: batched (CUDA graph) vs sequential GPU",
        "value": value, "unit": "bubble-steps/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": el / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 (assembly, residual, state) + f32 (preconditioner)", "data": "synthetic",
        "config": {"workload": f"{nb} bubbles, nu~U{{4..16}}, R0 log-U[0.5,2], A~U[0.1,1.5], T~U[2,10], seed 0, "
                               "phi=0, epsilon=1, gamma=1.4, RK4 dt=2e-3",
                   "total_unknowns": int(Ns.sum()), "solver": "batched mixed",
                   "l2": f"working set larger than L2 (G+H = {16 * float((Ns ** 2).sum()) / 1e9:.1f} GB per stage)"},
        "sequential_gpu": {"value": seq_value, "unit": "bubble-steps/s", "steps_per_bubble": seq_steps,
                           "solver": "mixed, one bubble at a time", "setup_s": seq_setup},
        "speedup_vs_sequential": (value / ws / seq_value) if seq_value else None,
        "autotune": {"chosen_column_group": cg, "ms_per_assembly": {"32x128": tune_ms[0], "48x64": tune_ms[1],
                                                                     "64x64": tune_ms[2], "16x256": tune_ms[3]},
                     "seconds": tune_s},
        "setup_s_first_step": setup_s,
        "during_timed_steps": {"ns_steps": int(st1.ns_steps - st0.ns_steps),
                               "refreshes": int(st1.precond_refresh - st0.precond_refresh),
                               "repeated_steps": int(st1.gmres_fallbacks - st0.gmres_fallbacks)},
        "psi_rel_err_vs_fp64": {"max_over_8_bubbles": max(errs)},
        "e2e": {"value": e2e_value, "unit": "bubble-steps/s", "h2d_bytes_per_step": 40 * N,
                "d2h_bytes_per_step": 40 * N},
        "gpu_launches": launches,
        "roofline": {"bound": "fp64-fma", "kernel": "k_patch_records + k_assemble_patch + k_rhs_finish_batch (G-only assembly of every bubble)",
                     "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s", "frac": achieved / fp64_peak,
                     "flops_per_launch": flops, "avg_launch_ms": avg_asm_ms,
                     "peak_source": "measured live: FP64 FMA-loop kernel (bem_measure_fma_peaks)"},
        "clocks": clk.summary(),
    }
    print(json.dumps(line))
    return 0


def run_adjoint(args):
    """Adjoint gradient of the volume after 50 RK4 steps (N = 1002) against central differences."""
    ws, rank, local = dist_env()
    import torch

    device = local if ws > 1 else 0
    torch.cuda.set_device(device)
    from bem_b200 import mesh
    from bem_b200.adjoint import rk4_flow, volume
    from bem_b200.sim import ColocSim

    dt, steps, ndir, h = 2e-3, 50, args.dirs, 1e-6
    phys = dict(p_inf=1.0, epsilon=1.0, sigma=0.0, gamma=1.4)
    v, f = mesh.bubble(10, 1.0, (2.0, 0.0, 0.0))
    phi = np.full(len(v), 0.3)
    N = len(v)
    sim = ColocSim(v, f, solver="mixed", device=device, **phys)
    dev = torch.device(f"cuda:{device}")
    tr = torch.tensor(f, dtype=torch.int64, device=dev)
    fw, bw = [], []
    for rep in range(args.warmup + 1):  # warm-up repetitions, then the timed one
        x0 = torch.tensor(v, dtype=torch.float64, device=dev, requires_grad=True)
        p0 = torch.tensor(phi, dtype=torch.float64, device=dev, requires_grad=True)
        sim.set_time(0.0)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        xK, pK = rk4_flow(sim, x0, p0, dt, steps)
        J = volume(xK, tr)
        torch.cuda.synchronize(dev)
        t1 = time.perf_counter()
        J.backward()
        torch.cuda.synchronize(dev)
        t2 = time.perf_counter()
        fw.append(t1 - t0)
        bw.append(t2 - t1)
    gx, gp = x0.grad.cpu().numpy(), p0.grad.cpu().numpy()
    J0 = float(J.item())

    fd_sim = ColocSim(v, f, solver="bicgstab", device=device, **phys)  # V0 = initial volume, held fixed

    def Jfd(x, p):
        fd_sim.set_vertices(x)
        fd_sim.set_phi(p)
        fd_sim.set_time(0.0)
        fd_sim.evolve_rk4_steps(dt, steps)
        xe = fd_sim.get_vertices()
        a, b, c = xe[f[:, 0]], xe[f[:, 1]], xe[f[:, 2]]
        return float(np.sum(np.cross(a, b) * c) / 6.0)

    rng = np.random.default_rng(0)
    errs, errs_n = [], []
    tw = time.perf_counter()
    for _ in range(ndir):
        dx, dp = rng.standard_normal((N, 3)), rng.standard_normal(N)
        fd = (Jfd(v + h * dx, phi + h * dp) - Jfd(v - h * dx, phi - h * dp)) / (2 * h)
        ad = float(np.sum(gx * dx) + np.dot(gp, dp))
        errs.append(abs(ad - fd) / abs(fd))
        errs_n.append(abs(ad - fd) / (np.sqrt(np.sum(gx ** 2) + np.sum(gp ** 2)) *
                                      np.sqrt(np.sum(dx ** 2) + np.sum(dp ** 2))))
    fd_s = time.perf_counter() - tw
    if rank != 0:
        return 0
    line = {
        "metric": "adjoint gradient of the volume after 50 RK4 steps (N=1002): max relative error vs central FD",
        "value": max(errs), "unit": "relative error", "n_gpus": ws, "steps": steps, "warmup": args.warmup,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 (adjoint, assembly derivative, residuals) + f32 (preconditioner)", "data": "synthetic",
        "config": {"workload": "one bubble nu=10 (N=1002, M=2000) at (2,0,0), phi=0.3, epsilon=1, gamma=1.4, "
                               "p_inf=1, RK4 dt=2e-3 x 50, objective V(x_50)",
                   "directions": ndir, "fd_step": h, "fd_solver": "FP64 BiCGSTAB GPU path"},
        "target": 1e-5,
        "rel_err": {"max": max(errs), "median": float(np.median(errs)),
                    "max_normalised_by_norms": max(errs_n)},
        "objective": J0,
        "grad_norm": {"x": float(np.sqrt(np.sum(gx ** 2))), "phi": float(np.sqrt(np.sum(gp ** 2)))},
        "time_s": {"forward_with_checkpoints": fw[-1], "backward": bw[-1], "fd_64_forward_runs": fd_s},
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--solver", default="mixed", choices=["mixed", "bicgstab", "lu"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--workload", default="headline", choices=["headline", "pair", "sweep", "adjoint", "lu"])
    ap.add_argument("--no-seq", action="store_true", help="sweep: skip the sequential baseline")
    ap.add_argument("--bubbles", type=int, default=256, help="sweep: number of bubbles")
    ap.add_argument("--dirs", type=int, default=32, help="adjoint: finite-difference directions")
    ap.add_argument("--inverse", default="auto", choices=["auto", "gj", "ns"],
                    help="headline, mixed solver: build the approximate inverse by Gauss-Jordan (gj) or "
                         "Newton-Schulz (ns); auto: Gauss-Jordan from N = 8192")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "pair":
        return run_pair(args)
    if args.workload == "sweep":
        return run_sweep(args)
    if args.workload == "adjoint":
        return run_adjoint(args)
    if args.workload == "lu":
        return run_lu(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
