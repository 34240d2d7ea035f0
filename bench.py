"""Throughput of the RHS + TVD-RK3 step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload wavy4|tgv32|tree24|ensemble64] [--precision f32|f64] [--n 128]
                    [--no-cpu] [--no-adjoint] [--no-error-table]
    python bench.py --adjoint-only [--adjoint-n 96] [--adjoint-steps 50] [--adjoint-every 10]
                    [--adjoint-precision both|f32|f64] [--adjoint-variant 0..4]

One "step" = one full TVD-RK3 time step (halo fill + boundary conditions +
three RHS/stage evaluations) over every block of the workload, replayed from a
captured CUDA graph.  The default workload is 4 curvilinear blocks of 128^3
cells (2 x 2 in i-j, periodic, Mach 0.5, Re 1e4, 1 % seeded noise; synthetic
data, inputs larger than L2).  Before timing, each plan's launch shape is
picked by the autotuner (fj_plan_autotune).

Printed on rank 0 as ONE JSON line:
  value        whole-job Mcell-stages/s of the selected precision (default the
               FP32-flux/FP64-state path): interior cells x 3 stages x steps /
               device time (CUDA events, max over ranks), state in HBM;
  variants     the same for both precisions, measured in the same run, and the
               relative L2 difference of the FP32-flux state from the FP64
               state after the same steps (the FP64 GPU path matches the CPU
               oracle to 1e-12 per step);
  e2e          the metric through the public ``step()`` API with the state
               copied host->device and the result device->host every step;
  roofline     the dominant kernel group -- one TVD-RK3 stage of all blocks
               (three launches: primitives, fluxes, assembly) -- timed live:
               algorithmic bytes (q, q0, metrics, vol read, stage result
               written: 164 B per padded cell with the FP32 metric copy, 200 B
               in FP64) / its CUDA-event duration, against the measured HBM
               copy bandwidth;
  cpu_baseline the NumPy FP64 oracle (1 core) on one block for one step;
  fp32_error_table  FP32-flux against FP64 per conserved variable, full and
               interior, at steps 1, 10, 100 (and 200 for tree24);
  workloads    (default workload only) the same record -- value, step time,
               stage-group roofline, end to end -- for the uneven 24-block
               tree, the 64-instance ensemble and the 32^3 Taylor-Green block,
               in both precisions;
  adjoint      adjoint/forward and gradient/forward time of the checkpointed
               trajectory adjoint on the 96^3 Taylor-Green case (50 steps, a
               checkpoint every 10), FP64 and FP32-flux, with dJ/dmu0, dJ/dM0
               and the FP64 gradient's central-difference check.

``--impl reference`` times the reference algorithm on the host cores (the
PyTorch-CPU FP64 port of the reference, all threads; the reference itself is
JAX, which is not installed in this image) on a bounded sample of the same
workload.  Multi-GPU (torchrun): each rank runs an independent replica of the
workload (weak scaling, no data-path collective); rank 0 reports the aggregate.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import threading
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Mcell-stages/s & HBM % (FP32 vs FP64, stated L2 err); adjoint/forward time"
UNIT = "Mcell-stages/s"
# algorithmic bytes per padded cell of one stage-2/3 evaluation: read q (40),
# q0 (40), metrics (72 FP64 or 36 as the FP32 copy), vol (8); write 40
STAGE_BYTES = {"f64": 200.0, "f32": 164.0}
STEP_BYTES = {"f64": 560.0, "f32": 452.0}
# DRAM bytes per padded cell of one stage-2 launch group (dram__bytes_read +
# dram__bytes_write summed over its kernels), measured by ncu on
# `bench.py --stage-only --n 96` (4 blocks of 100^3 padded cells, 4.0 M) and
# scaled per cell: split FP32 59 + 147 + 283 B (primitives, fluxes, assembly),
# split FP64 75 + 259 + 406 B; the fused tile kernel 220 B (its primitive
# launch not included)
STAGE_TRAFFIC = {("f32", "split"): 489.0, ("f64", "split"): 740.0, ("f32", "tile"): 220.0}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _dist():
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0"))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms around the
    timed region: entering waits for the first sample (so sampling is live
    when timing starts), leaving waits for one more sample taken after the
    region, then stops the sampler."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu, self.proc, self.lines = gpu_index, None, []
        self._cv = threading.Condition()
        self._reader = None

    def _read(self):
        for line in self.proc.stdout:
            if line.strip():
                with self._cv:
                    self.lines.append(line.strip())
                    self._cv.notify_all()

    def _wait_for(self, n, timeout):
        with self._cv:
            self._cv.wait_for(lambda: len(self.lines) >= n, timeout=timeout)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return self
        self._reader = threading.Thread(target=self._read, daemon=True)
        self._reader.start()
        self._wait_for(1, 10.0)
        return self

    def __exit__(self, *a):
        if self.proc is None:
            return
        with self._cv:
            n = len(self.lines)
        self._wait_for(n + 1, 2.0)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
            self.proc.wait()
        if self._reader is not None:
            self._reader.join(timeout=5)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            parts = [p.strip() for p in l.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _gpu_index(local_rank: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        try:
            return int(vis.split(",")[local_rank])
        except (ValueError, IndexError):
            return local_rank
    return local_rank


def build_case(args, metrics_fn=None):
    from famrdp_jax_b200 import cases
    if args.workload == "wavy4":
        return cases.wavy4(n=args.n, metrics_fn=metrics_fn, seed=args.seed)
    if args.workload == "tgv32":
        return cases.tgv(n=32)
    if args.workload == "tree24":
        return cases.tree24(seed=args.seed)
    if args.workload == "ensemble64":
        return cases.ensemble(ninst=64, n=64, seed=args.seed)
    raise SystemExit(f"unknown workload {args.workload}")


def workload_desc(case, args):
    desc = {"wavy4": f"{args.n}^3 cells each, 2x2 in i-j, periodic, curvilinear, M 0.5, Re 1e4, 1% noise",
            "tgv32": "32^3 Taylor-Green vortex, M0 0.1, Re 1600, constant viscosity, self-periodic",
            "tree24": "uneven blocks U[16,160]^3 on a random spanning tree, farfield/periodic faces, M 0.8, Re 5e4",
            "ensemble64": "64 independent self-periodic 64^3 Taylor-Green instances, M U[0.1,0.9], Re log-U[1e2,1e4], "
                          "0.5% noise, per-instance mu0 and dt, all instances per launch"}
    # per padded cell a step reads at least q, kxyz and vol and writes q: 160 B
    mb = 160.0 * case.padded_cells / 1e6
    l2 = (f"inputs larger than L2 (state + metrics {mb:.0f} MB per step >> 126 MB)" if mb > 2 * 126 else
          f"inputs of {mb:.0f} MB per step, not flushed from L2 between steps (a launch-bound case)")
    return {"workload": f"{case.name}: {len(case.qs)} blocks, {desc[args.workload]}",
            "blocks": len(case.qs), "cells_interior": case.interior_cells, "cells_padded": case.padded_cells,
            "precision": args.precision, "ghost": case.cfg.ghost, "seed": args.seed,
            "l2": l2,
            "cuda_graph": "each timed step is one replay of a captured step graph (halo, BCs, 3 stages)"}


def cpu_oracle_sample(case, dt):
    """NumPy oracle: one TVD-RK3 step of block 0 alone."""
    from oracle.ref import NP
    q = case.qs[0]
    kxyz, vol = case.metrics[0][1], case.metrics[0][2]
    t0 = time.perf_counter()
    NP.rk3_step(q, lambda x: NP.rhs_block(x, kxyz, vol, case.cfg), dt)
    el = time.perf_counter() - t0
    g = case.cfg.ghost
    cells = (q.shape[1] - 2 * g) * (q.shape[2] - 2 * g) * (q.shape[3] - 2 * g)
    return {"value": cells * 3 / el / 1e6, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"NumPy FP64 oracle, one TVD-RK3 step of block 0 ({q.shape[1]}x{q.shape[2]}x{q.shape[3]} "
                      f"padded), {el:.1f} s"}


def run_reference(args):
    """The reference algorithm on the host cores (PyTorch-CPU FP64 port)."""
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    import torch
    from famrdp_jax_b200 import cases
    from oracle.ref import NP, TORCH
    cores = len(os.sched_getaffinity(0))
    torch.set_num_threads(cores)
    if args.workload == "wavy4":
        c = cases.wavy4(n=args.n, metrics_fn=lambda x: NP.compute_metrics(x, ghost=2), seed=args.seed)
    else:
        c = build_case(args)
    c.qs, c.metrics = c.qs[:1], c.metrics[:1]
    q = torch.tensor(c.qs[0])
    kxyz = torch.tensor(c.metrics[0][1])
    vol = torch.tensor(c.metrics[0][2])
    dt = NP.cfl_dt(c.qs, [(c.metrics[0][1], c.metrics[0][2])], c.cfg.gas.gamma, c.cfl, c.cfg.ghost)

    def L(x):
        return TORCH.rhs_block(x, kxyz, vol, c.cfg)

    with torch.no_grad():
        for _ in range(args.warmup):
            q = TORCH.rk3_step(q, L, dt)
        times = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            q = TORCH.rk3_step(q, L, dt)
            times.append(time.perf_counter() - t0)
    ms = statistics.median(times) * 1e3
    value = c.interior_cells * 3 / (ms / 1e3) / 1e6
    sample = (f"PyTorch-CPU FP64 port of the reference algorithm, {cores} threads, one TVD-RK3 step of "
              f"block 0 ({c.qs[0].shape[1]}^3 padded) per step, median of {args.steps}")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {k: v for k, v in workload_desc(c, args).items() if k != "cuda_graph"}
                      | {"sample": "block 0 only", "precision": "f64"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference (JAX) not installable in this image: no jax/jaxlib wheel, no network"}
    print(json.dumps(line), flush=True)
    return 0


def adjoint_timing(device, n=96, nsteps=50, every=10, precisions=("f64", "f32"), fd=True):
    """Adjoint/forward time on the 96^3 Taylor-Green configuration (M0 0.3,
    Re 800, constant viscosity, 1 % noise, kinetic-energy objective after 50
    steps, a checkpoint every 10 steps), FP64 and FP32-flux, with the FP32-flux
    gradient's relative L2 distance from the FP64 gradient.  Device time by
    CUDA events on the stream the kernels run on; "adjoint_over_forward" is the
    reverse sweep (segment recompute + step adjoints) over the plain forward,
    "gradient_over_forward" the whole gradient (checkpointed forward + reverse
    sweep) over the plain forward.  With fd, the FP64 gradient is also checked
    against central differences of the forward (eps 1e-6, 16 directions)."""
    import dataclasses as dc

    import torch

    from famrdp_jax_b200 import cases
    from famrdp_jax_b200.solver import adjoint, diagnostics
    from famrdp_jax_b200.solver.step import StepPlan

    out = {"workload": f"tgv{n}: {n}^3 cells, M0 0.3, Re 800, 1% noise, J = kinetic energy after {nsteps} steps, "
                       f"checkpoint every {every} steps"}
    c = cases.tgv(n=n, M0=0.3, Re=800.0, noise=0.01, seed=0)
    dq_dM0 = cases.tgv_dq0_dM0(c)
    grads = {}
    stream = torch.cuda.current_stream(device)

    clocks = {}

    def timed(fn, clock_key=None):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        clk = ClockSampler(_gpu_index(device.index or 0)) if clock_key else None
        if clk:
            clk.__enter__()
        e0.record(stream)
        r = fn()
        e1.record(stream)
        torch.cuda.synchronize(device)
        if clk:
            clk.__exit__(None, None, None)
            clocks[clock_key] = clk.summary()
        return r, e0.elapsed_time(e1)

    for prec in precisions:
        cfg = dc.replace(c.cfg, precision=prec)
        st = cases.to_state(c, device)
        plan = StepPlan(st, cfg)
        dt = diagnostics.cfl_dt(st, cfg, c.cfl)
        qa = [st.blocks[0].q.clone()]
        qb = [torch.empty_like(qa[0])]
        for _ in range(4):  # also captures the two ping-pong step graphs
            plan.run(qa, qb, dt, graph=True)
            qa, qb = qb, qa

        def fwd():  # the plain forward, as graph replays (its fastest form)
            a, b = qa, qb
            for _ in range(nsteps):
                plan.run(a, b, dt, graph=True)
                a, b = b, a

        _, t_fwd = timed(fwd, "forward")
        adjoint.adjoint_kinetic_energy(st, cfg, dt, 2, checkpoint_every=1, plan=plan)  # warm-up
        run = adjoint._Run(cfg=cfg, metrics=st.metrics, dt=float(dt), nsteps=nsteps, every=every, plan=plan,
                           tables=adjoint._Tables(cfg), dmu=torch.zeros(1, dtype=torch.float64, device=device))
        run.buffers([st.blocks[0].q])  # the driver's reusable buffers, outside the timed region
        run.reverse_buffers([st.blocks[0].q])
        adjoint._forward_with_checkpoints(run, [st.blocks[0].q])  # warm-up: captures the step graphs
        (final, checkpoints), t_ckpt = timed(lambda: adjoint._forward_with_checkpoints(run, [st.blocks[0].q]))
        lams = adjoint.kinetic_energy_grad(final, st.metrics, cfg.ghost)
        g, t_rev = timed(lambda: adjoint._reverse_sweep(run, checkpoints, lams), "reverse")
        fstate = dc.replace(st, blocks=(dc.replace(st.blocks[0], q=final[0]),))
        J = diagnostics.kinetic_energy(fstate, cfg.ghost)
        grads[prec] = g[0]
        dmu = float(run.dmu.item())
        # M0 enters the initial state and mu0 = rho0 M0 / Re (dt held fixed)
        dJ_dM0 = float(torch.sum(g[0] * torch.as_tensor(dq_dM0, device=device))) + dmu * 1.0 / c.meta["Re"]
        out[prec] = {"forward_ms_per_step": t_fwd / nsteps, "checkpointed_forward_ms_per_step": t_ckpt / nsteps,
                     "reverse_sweep_ms_per_step": t_rev / nsteps, "adjoint_over_forward": t_rev / t_fwd,
                     "gradient_over_forward": (t_ckpt + t_rev) / t_fwd,
                     "J": J, "dJ_dmu0": dmu, "dJ_dM0": dJ_dM0,
                     # SM clocks during the timed forward and reverse sweeps: the
                     # issue-bound adjoint kernels run under the power cap
                     "clocks": dict(clocks)}
        del plan, run, final, checkpoints, lams, g, qa, qb
        torch.cuda.empty_cache()
    out["ratios_note"] = ("adjoint_over_forward = reverse sweep (segment recompute + step adjoints) / plain "
                          "forward; gradient_over_forward = (checkpointed forward + reverse sweep) / plain forward")
    if len(grads) == 2:
        out["f32_vs_f64_grad_rel_l2"] = float(torch.linalg.vector_norm(grads["f32"] - grads["f64"]) /
                                              torch.linalg.vector_norm(grads["f64"]))
    if fd:
        from famrdp_jax_b200.solver.gradcheck import fd_check_kinetic_energy
        st = cases.to_state(c, device)
        dt = diagnostics.cfl_dt(st, c.cfg, c.cfl)
        r = fd_check_kinetic_energy(st, dc.replace(c.cfg, precision="f64"), dt, nsteps, checkpoint_every=every,
                                    eps=1e-6, ndirs=16, seed=0)
        out["fd_check_f64"] = {k: v for k, v in r.items() if k != "per_direction"} | {
            "rel_direction": [row["rel_direction"] for row in r["per_direction"]],
            "rel_gradnorm": [row["rel_gradnorm"] for row in r["per_direction"]],
            "note": "central differences of the GPU forward, eps 1e-6, 16 seeded unit-L2 directions; "
                    "rel_direction = |fd-ad|/|ad|, rel_gradnorm = |fd-ad|/|grad J|"}
    return out


def error_table(case, dt, device, marks=(1, 10, 100), ens=None):
    """FP32-flux against FP64, both on this GPU from the same start, in
    lockstep: relative L2 per conserved variable over the full padded state
    and over the interior at the marked steps.  The FP64 GPU path matches the
    CPU oracle to <= 1e-12 per step (the parity tests), so it stands in for the
    oracle over runs the oracle cannot finish here."""
    import torch

    from famrdp_jax_b200 import cases
    from famrdp_jax_b200.solver.step import StepPlan

    runs = {}
    for prec in ("f64", "f32"):
        cfg = dataclasses.replace(case.cfg, precision=prec)
        st = cases.to_state(case, device)
        plan = StepPlan(st, cfg)
        if ens:
            plan.set_ensemble(*ens)
        runs[prec] = [plan, [b.q.clone() for b in st.blocks], [torch.empty_like(b.q) for b in st.blocks]]
    g = case.cfg.ghost
    names = ["rho", "rhou", "rhov", "rhow", "rhoE"]
    table = {}
    for n in range(1, max(marks) + 1):
        for prec, r in runs.items():
            r[0].run(r[1], r[2], dt, graph=True)
            r[1], r[2] = r[2], r[1]
        if n in marks:
            row = {}
            for part in ("full", "interior"):
                for v, nm in enumerate(names):
                    num = den = 0.0
                    for a, b in zip(runs["f32"][1], runs["f64"][1]):
                        x, y = a[v], b[v]
                        if part == "interior":
                            x, y = x[g:-g, g:-g, g:-g], y[g:-g, g:-g, g:-g]
                        num += float(torch.sum((x - y) ** 2))
                        den += float(torch.sum(y ** 2))
                    row[f"{part}_{nm}"] = (num / den) ** 0.5
            table[str(n)] = row
    return {"reference": "FP64 path on the GPU (<= 1e-12 per step against the oracle)", "rel_l2": table}


def _throughput(cells: int, steps: int, ms: float, ws: int) -> float:
    """Whole-job Mcell-stages/s of ws replicas that each advanced `cells`
    interior cells by `steps` steps (3 stages each) in `ms` (slowest rank)."""
    return ws * cells * 3 * steps / (ms / 1e3) / 1e6


def _max_over_ranks(x: float, ws: int, device) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _stage_roofline(plan, q0s, dt, prec, padded_cells):
    """The dominant kernel group, one stage-2 evaluation of all blocks, timed
    live (10 launches of the group after 3 warm-ups, CUDA events on the
    launching stream)."""
    import torch
    kern = plan.kernel
    # the persistent step has no stage-sized launch: its one launch is the
    # whole step (halo, boundary faces and three stages), timed as a graph
    # replay and counted as three stages' algorithmic bytes
    whole_step = kern == "persistent"
    qin = [q.clone() for q in q0s]  # the stage input, distinct from the step's start state q0
    outs = [torch.empty_like(q) for q in q0s]

    def launch():
        if whole_step:
            plan.run(qin, outs, dt, graph=True)
        else:
            plan.stage(qin, q0s, outs, dt, 2)

    for _ in range(3):
        launch()
    torch.cuda.synchronize()
    reps = 10
    s = torch.cuda.current_stream()
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a0.record(s)
    for _ in range(reps):
        launch()
    a1.record(s)
    torch.cuda.synchronize()
    stage_ms = a0.elapsed_time(a1) / reps
    alg = STAGE_BYTES[prec] * padded_cells * (3 if whole_step else 1)
    peak, peak_kind = _peaks()
    achieved = alg / (stage_ms / 1e3) / 1e9
    traffic = STAGE_TRAFFIC.get((prec, kern))
    del qin, outs
    what = ("one TVD-RK3 stage of all blocks (fused TMA-tile kernel: one persistent launch, plus the launch "
            "that fills the padded primitive planes)" if kern == "tile" else
            "one whole TVD-RK3 step of all blocks (persistent kernel: halo, boundary faces, primitives and the "
            "three stages in one launch after a counter reset; algorithmic bytes of three stages)" if whole_step
            else "one TVD-RK3 stage of all blocks (split pipeline: prims, fluxes, assembly; 3 launches)")
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic * padded_cells * (3 if whole_step else 1) if traffic else None,
            "traffic_note": f"{traffic:.0f} B per padded cell (ncu dram__bytes_read+write of the stage-2 group on "
                            f"4 x 100^3 padded cells) x the cells of one launch" if traffic else None,
            "kernel": what, "stage_kernel": kern,
            "alg_bytes_per_cell": STAGE_BYTES[prec], "alg_bytes_per_launch": alg, "launch_ms": stage_ms,
            "peak_kind": peak_kind}


def _end_to_end(plan, cfg, state, q0s, dt, cells, steps, ws, device, barrier):
    """The metric through the public API with host buffers: every step copies
    its input state from pinned host memory and its result back.  Two public
    paths: step() per call (copy in, step, copy out, one stream) and
    HostStepper, which overlaps step n's copy-in, step n-1 and the copy-out of
    step n-2 on three streams; the faster is reported."""
    import torch

    from famrdp_jax_b200.core.types import Block, State
    from famrdp_jax_b200.solver.step import step
    from famrdp_jax_b200.solver.stream import HostStepper
    s = torch.cuda.current_stream()
    host_in = [q.detach().cpu().pin_memory() for q in q0s]
    host_out = [torch.empty_like(h).pin_memory() for h in host_in]
    dev_in = [torch.empty_like(q) for q in q0s]
    e2e_steps = max(3, min(steps, 10))

    def e2e_step():
        for d, h in zip(dev_in, host_in):
            d.copy_(h, non_blocking=True)
        s_ = State(blocks=tuple(Block(q=d, xyz=b.xyz) for d, b in zip(dev_in, state.blocks)), metrics=state.metrics)
        s2 = step(s_, cfg, dt, plan=plan)
        for h, b in zip(host_out, s2.blocks):
            h.copy_(b.q, non_blocking=True)

    def timed_e2e(fn):
        fn()  # warm-up (graphs, buffers)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        x0, x1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        x0.record(s)
        fn()
        x1.record(s)
        torch.cuda.synchronize()
        return _max_over_ranks(x0.elapsed_time(x1), ws, device)

    serial_ms = timed_e2e(lambda: [e2e_step() for _ in range(e2e_steps)])
    stepper = HostStepper(plan)
    piped_ms = timed_e2e(lambda: stepper.run([host_in] * e2e_steps, [host_out] * e2e_steps, dt))
    bytes_io = sum(h.numel() * 8 for h in host_in)
    e2e_ms = min(serial_ms, piped_ms)
    del stepper, host_in, host_out, dev_in
    return {"value": _throughput(cells, e2e_steps, e2e_ms, ws), "unit": UNIT, "h2d_bytes_per_step": bytes_io,
            "d2h_bytes_per_step": bytes_io, "ms_per_step": e2e_ms / e2e_steps, "steps": e2e_steps,
            "path": "HostStepper (pipelined)" if piped_ms <= serial_ms else "step() per call",
            "serial_step_value": _throughput(cells, e2e_steps, serial_ms, ws),
            "pipelined_value": _throughput(cells, e2e_steps, piped_ms, ws)}


def measure_case(case, prec, steps, warm, device, ws, local, barrier, ens=None, sample_clocks=False, kernel="auto"):
    """Graph-replayed steps of one workload in one precision: throughput,
    launches, the autotuner's choice, the stage-group roofline and the
    end-to-end figure.  Returns (record, final state, clock summary)."""
    import torch

    from famrdp_jax_b200 import _capi, cases
    from famrdp_jax_b200.solver import diagnostics
    from famrdp_jax_b200.solver.step import StepPlan
    cells = case.interior_cells
    cfg = dataclasses.replace(case.cfg, precision=prec)
    state = cases.to_state(case, device)
    dt = diagnostics.cfl_dt(state, cfg, case.cfl)
    plan = StepPlan(state, cfg)
    if ens:
        plan.set_ensemble(*ens)
    qa = [b.q for b in state.blocks]
    qb = [torch.empty_like(q) for q in qa]
    tuned = plan.autotune(qa, qb, dt, reps=3)  # launch shape of the FP32 kernels (qb is scratch here)
    if prec == "f32" and kernel != "auto":
        plan.set_kernel(kernel)
    for _ in range(warm):  # also captures the two ping-pong step graphs
        plan.run(qa, qb, dt, graph=True)
        qa, qb = qb, qa
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n0 = _capi.launch_count(device)
    clk = ClockSampler(_gpu_index(local)) if sample_clocks else None
    if clk:
        clk.__enter__()
    e0.record(s)
    for _ in range(steps):
        plan.run(qa, qb, dt, graph=True)
        qa, qb = qb, qa
    e1.record(s)
    torch.cuda.synchronize()
    if clk:
        clk.__exit__(None, None, None)
    launches = _capi.launch_count(device) - n0
    barrier()
    ms = _max_over_ranks(e0.elapsed_time(e1), ws, device)
    rec = {"ms_per_step": ms / steps, "value": _throughput(cells, steps, ms, ws), "launches": launches,
           "launches_per_step": launches / steps,
           "autotune": {"chosen": tuned[0], "ms_per_step": tuned[1]},
           "step_hbm_gbs": STEP_BYTES[prec] * case.padded_cells * ws / (ms / steps / 1e3) / 1e9}
    rec["roofline"] = _stage_roofline(plan, qa, dt, prec, case.padded_cells)
    rec["e2e"] = _end_to_end(plan, cfg, state, qa, dt, cells, steps, ws, device, barrier)
    final = [q.clone() for q in qa]
    del plan, qa, qb, state
    torch.cuda.empty_cache()
    return rec, final, (clk.summary() if clk else None)


def run_ours(args):
    import torch
    import torch.distributed as dist

    from famrdp_jax_b200 import cases
    from famrdp_jax_b200.core.types import State
    from famrdp_jax_b200.mesh.metric import compute_metrics
    from famrdp_jax_b200.solver import diagnostics
    from famrdp_jax_b200.solver.step import StepPlan

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", device_id=device, timeout=datetime.timedelta(seconds=300))

    def metrics_fn(xyz):
        m = compute_metrics(torch.as_tensor(xyz, dtype=torch.float64, device=device), ghost=2)
        return m.jac.cpu().numpy(), m.kxyz.cpu().numpy(), m.vol.cpu().numpy()

    case = build_case(args, metrics_fn)
    warm = max(args.warmup, 3)
    st0 = cases.to_state(case, device)
    dt = diagnostics.cfl_dt(st0, case.cfg, case.cfl)
    if args.stage_only:
        # four standalone stage-2 evaluations of all blocks (the launch group
        # the roofline line times), for a profiler to capture: nothing else
        cfg = dataclasses.replace(case.cfg, precision=args.precision)
        plan = StepPlan(st0, cfg)
        if args.precision == "f32":
            plan.set_variant(args.shape)
            if args.kernel != "auto":
                plan.set_kernel(args.kernel)
            if args.kernel == "persistent":
                plan.set_persist_shape(args.persist_shape)
        q0s = [b.q for b in st0.blocks]
        qin = [q.clone() for q in q0s]  # the stage input, distinct from the step's start state
        outs = [torch.empty_like(q) for q in q0s]
        for _ in range(4):
            if plan.kernel == "persistent":  # its one launch is a whole step
                plan.run(qin, outs, dt)
            else:
                plan.stage(qin, q0s, outs, dt, 2)
        torch.cuda.synchronize()
        if rank == 0:
            print(json.dumps({"stage_only": True, "precision": args.precision, "shape": args.shape,
                              "kernel": plan.kernel,
                              "padded_cells": case.padded_cells}), flush=True)
        return 0

    def ensemble_of(c, st):
        if "mu0" in c.meta and isinstance(c.meta["mu0"], list):  # independent instances
            return (c.meta["mu0"], [diagnostics.cfl_dt(State(blocks=(b,), metrics=(m,)), c.cfg, c.cfl)
                                    for b, m in zip(st.blocks, st.metrics)])
        return None

    ens = ensemble_of(case, st0)
    del st0

    def barrier():
        if ws > 1:
            dist.barrier()

    order = [args.precision] + [p for p in ("f32", "f64") if p != args.precision]
    results, finals = {}, {}
    clk_summary = None
    for prec in order:
        rec, finals[prec], clk = measure_case(case, prec, args.steps, warm, device, ws, local, barrier, ens,
                                              sample_clocks=(prec == args.precision), kernel=args.kernel)
        results[prec] = rec
        if clk is not None:
            clk_summary = clk
    num = sum(float(torch.sum((finals["f32"][b] - finals["f64"][b]) ** 2)) for b in range(len(case.qs)))
    den = sum(float(torch.sum(finals["f64"][b] ** 2)) for b in range(len(case.qs)))
    err_f32 = (num / den) ** 0.5
    del finals

    # ---- the other configurations, each in both precisions -----------------
    others = {}
    if args.workload == "wavy4" and not args.no_workloads:
        for wl in ("tree24", "ensemble64", "tgv32"):
            sub = argparse.Namespace(**{**vars(args), "workload": wl})
            c2 = build_case(sub)
            st2 = cases.to_state(c2, device)
            ens2 = ensemble_of(c2, st2)
            del st2
            entry = {"config": workload_desc(c2, sub)}
            for prec in ("f32", "f64"):
                rec, _, _ = measure_case(c2, prec, args.steps, warm, device, ws, local, barrier, ens2,
                                         kernel=args.kernel)
                entry[prec] = rec
            entry["f32_over_f64"] = entry["f64"]["ms_per_step"] / entry["f32"]["ms_per_step"]
            others[wl] = entry
            del c2
            torch.cuda.empty_cache()

    cpu = cpu_oracle_sample(case, dt) if (rank == 0 and not args.no_cpu) else None
    marks = (1, 10, 100, 200) if args.workload == "tree24" else (1, 10, 100)
    errs = error_table(case, dt, device, marks, ens) if (rank == 0 and not args.no_error_table) else None
    adj = (adjoint_timing(device, args.adjoint_n, args.adjoint_steps, args.adjoint_every, fd=not args.no_fd)
           if (rank == 0 and not args.no_adjoint) else None)
    if rank == 0:
        r = results[args.precision]
        line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": warm, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64" if args.precision == "f64" else "f32-flux/f64-state",
                "data": "synthetic", "config": workload_desc(case, args) | {"parallelism": f"replicas x{ws}"},
                "roofline": r["roofline"], "cpu_baseline": cpu, "e2e": r["e2e"], "gpu_launches": r["launches"],
                "clocks": clk_summary,
                "variants": {p: results[p] for p in order} | {
                    "f32_over_f64": results["f64"]["ms_per_step"] / results["f32"]["ms_per_step"],
                    "f32_vs_f64_rel_l2": err_f32,
                    "f32_vs_f64_note": f"whole state after {warm + args.steps} steps from the same start"},
                "workloads": others or None,
                "adjoint": adj, "fp32_error_table": errs,
                "dt": dt if not ens else {"per_instance": True, "min": min(ens[1]), "max": max(ens[1])}}
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_sharded(args):
    """--shard: the workload's blocks partitioned over the ranks (one GPU
    each), every step exchanging the face slabs of links that cross ranks
    (famrdp_jax_b200.solver.sharded: one NCCL send and receive per peer and
    step).  Strong scaling: the whole topology's cells over the slowest rank's
    time.  With one rank the same path runs over a one-rank group."""
    import datetime
    import socket

    import torch
    import torch.distributed as dist

    from famrdp_jax_b200 import _topology, cases
    from famrdp_jax_b200.core.types import State
    from famrdp_jax_b200.mesh.metric import compute_metrics
    from famrdp_jax_b200.solver import diagnostics, sharded

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    timeout = datetime.timedelta(seconds=120)  # ranks that wait for one another end with an error
    if not dist.is_initialized():
        if ws > 1:
            dist.init_process_group("nccl", device_id=device, timeout=timeout)
        else:
            with socket.socket() as so:
                so.bind(("127.0.0.1", 0))
                port = so.getsockname()[1]
            dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                                    device_id=device, timeout=timeout)

    def metrics_fn(xyz):
        m = compute_metrics(torch.as_tensor(xyz, dtype=torch.float64, device=device), ghost=2)
        return m.jac.cpu().numpy(), m.kxyz.cpu().numpy(), m.vol.cpu().numpy()

    case = build_case(args, metrics_fn)
    cfg = dataclasses.replace(case.cfg, precision=args.precision)
    state = cases.to_state(case, device)
    shapes = [tuple(b.q.shape) for b in state.blocks]
    owner = sharded.partition(shapes, _topology.links(cfg.topology), ws)
    local_state = sharded.shard_state(state, owner, rank)
    del state
    torch.cuda.empty_cache()
    step = sharded.ShardedStep(shapes, owner, rank, local_state, cfg)
    dt = sharded.cfl_dt(local_state, cfg, case.cfl)
    if "mu0" in case.meta and isinstance(case.meta["mu0"], list):
        # independent instances (no links between blocks): each its own mu0 and
        # dt, every rank stepping its share of them
        dts = [0.0] * len(shapes)
        for b, blk, m in zip(step.ids, local_state.blocks, local_state.metrics):
            dts[b] = diagnostics.cfl_dt(State(blocks=(blk,), metrics=(m,)), cfg, case.cfl)
        t = torch.tensor(dts, dtype=torch.float64, device=device)
        dist.all_reduce(t)  # every block's dt comes from its owner, the others add 0
        step.set_ensemble(case.meta["mu0"], [float(x) for x in t.tolist()])
    step.share_p_ref()
    qa = [b.q.clone() for b in local_state.blocks]
    qb = [torch.empty_like(q) for q in qa]
    for _ in range(max(args.warmup, 3)):
        step.run(qa, qb, dt, graph=True)
        qa, qb = qb, qa
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step.run(qa, qb, dt, graph=True)
        qa, qb = qb, qa
    e1.record()
    torch.cuda.synchronize()
    dist.barrier()
    t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    cut = sum(1 for (tb, _tf, sb, _sf, _o) in step.links if owner[tb] != owner[sb])
    if rank == 0:
        line = {"metric": METRIC, "value": case.interior_cells * 3 * args.steps / (ms / 1e3) / 1e6, "unit": UNIT,
                "n_gpus": ws, "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                "dtype": "f64" if args.precision == "f64" else "f32-flux/f64-state", "data": "synthetic",
                "config": workload_desc(case, args) | {"parallelism": f"blocks over {ws} ranks",
                                                       "links_cut": cut, "links": len(step.links),
                                                       "blocks_per_rank": [owner.count(r) for r in range(ws)]}}
        print(json.dumps(line), flush=True)
    dist.barrier()
    del step
    dist.destroy_process_group()
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["wavy4", "tgv32", "tree24", "ensemble64"], default="wavy4")
    ap.add_argument("--precision", choices=["f32", "f64"], default="f32")
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--shard", action="store_true",
                    help="partition the workload's blocks over the ranks (halo slabs exchanged every step)")
    ap.add_argument("--stage-only", action="store_true",
                    help="only run four standalone stage-2 evaluations (four steps with --kernel persistent), "
                         "for a profiler")
    ap.add_argument("--shape", type=int, default=1, help="FP32 launch shape for --stage-only")
    ap.add_argument("--persist-shape", type=int, default=0,
                    help="launch shape of the persistent step for --stage-only --kernel persistent")
    ap.add_argument("--kernel", choices=["auto", "split", "tile", "persistent", "split_fill"], default="auto",
                    help="FP32 stage kernels: auto = the autotuner's choice (split shapes, the tile kernel and the "
                         "persistent step's shapes)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle sample")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint/forward timing")
    ap.add_argument("--no-error-table", action="store_true", help="skip the FP32-vs-FP64 error table")
    ap.add_argument("--no-workloads", action="store_true",
                    help="skip the sub-records of the other configurations (tree24, ensemble64, tgv32)")
    ap.add_argument("--no-fd", action="store_true", help="skip the adjoint's central-difference check")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="print only the adjoint/forward timing (one JSON line)")
    ap.add_argument("--adjoint-n", type=int, default=96)
    ap.add_argument("--adjoint-steps", type=int, default=50)
    ap.add_argument("--adjoint-every", type=int, default=10)
    ap.add_argument("--adjoint-precision", choices=["both", "f32", "f64"], default="both")
    ap.add_argument("--adjoint-variant", type=int, default=0, help="face-VJP launch shape (0..2)")
    args = ap.parse_args(argv)
    if args.adjoint_only:
        import torch

        from famrdp_jax_b200 import _capi
        _capi.set_adjoint_variant(args.adjoint_variant, torch.device("cuda:0"))
        precs = ("f64", "f32") if args.adjoint_precision == "both" else (args.adjoint_precision,)
        print(json.dumps(adjoint_timing(torch.device("cuda:0"), args.adjoint_n, args.adjoint_steps,
                                        args.adjoint_every, precs, fd=not args.no_fd)), flush=True)
        return 0
    if args.impl == "reference":
        return run_reference(args)
    if args.shard:
        return run_sharded(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
