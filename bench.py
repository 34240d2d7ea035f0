"""Throughput of the RHS + TVD-RK3 step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload wavy4|tgv32|tree24] [--precision f64|f32] [--n 128]

One "step" = one full TVD-RK3 time step (halo fill + boundary conditions +
three RHS/stage evaluations) over every block of the workload.  The default
workload is 4 curvilinear blocks of 128^3 cells (2 x 2 in i-j, periodic,
Mach 0.5, Re 1e4, 1 % seeded noise; synthetic data).

Printed on rank 0 as ONE JSON line:
  value        whole-job Mcell-stages/s (interior cells x 3 stages x steps /
               device time, max over ranks), inputs resident in HBM;
  e2e          the same metric through the public ``step()`` API with the
               state copied host->device and the result device->host every
               step (pinned host buffers);
  roofline     the dominant kernel group (one RK stage of one block) against
               the measured HBM copy bandwidth: algorithmic bytes per launch
               (200 B per padded cell: read q, q0, kxyz, vol; write out)
               over its CUDA-event duration;
  cpu_baseline the CPU oracle (NumPy FP64, 1 core) on one block, one step;
  clocks       nvidia-smi samples during the timed region.

``--impl reference`` times the reference algorithm's CPU port (the PyTorch-CPU
FP64 restatement, all host threads) on a bounded sample of the same workload,
since the reference (JAX) is not installable in this image.
Multi-GPU (torchrun): each rank runs an independent replica of the workload
(weak scaling, no data-path collective); rank 0 reports the aggregate.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Mcell-stages/s & HBM % (FP32 vs FP64, stated L2 err); adjoint/forward time"
UNIT = "Mcell-stages/s"
# algorithmic bytes per padded cell of one RK stage (stages 2 and 3): read q (40),
# q0 (40), kxyz (72), vol (8); write the stage result (40)
STAGE_BYTES_F64 = 200.0
STEP_BYTES_F64 = 560.0


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

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
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def _gpu_index(local_rank: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        try:
            return int(vis.split(",")[local_rank])
        except (ValueError, IndexError):
            return local_rank
    return local_rank


def build_case(args, device):
    from famrdp_jax_b200 import cases
    if args.workload == "wavy4":
        import torch
        from famrdp_jax_b200.mesh.metric import compute_metrics

        def metrics_fn(xyz):
            m = compute_metrics(torch.as_tensor(xyz, dtype=torch.float64, device=device), ghost=2)
            return m.jac.cpu().numpy(), m.kxyz.cpu().numpy(), m.vol.cpu().numpy()
        return cases.wavy4(n=args.n, metrics_fn=metrics_fn, precision=args.precision, seed=args.seed)
    if args.workload == "tgv32":
        return cases.tgv(n=32, precision=args.precision)
    if args.workload == "tree24":
        return cases.tree24(precision=args.precision, seed=args.seed)
    raise SystemExit(f"unknown workload {args.workload}")


def workload_desc(case, args):
    return {"workload": f"{case.name}: {len(case.qs)} blocks, " + (
        f"{args.n}^3 cells each, 2x2 in i-j, periodic, curvilinear, M 0.5, Re 1e4, 1% noise"
        if args.workload == "wavy4" else args.workload),
            "blocks": len(case.qs), "cells_interior": case.interior_cells, "cells_padded": case.padded_cells,
            "precision": args.precision, "ghost": case.cfg.ghost, "seed": args.seed,
            "l2": "inputs larger than L2 (state + metrics per step >> 126 MB)"}


def cpu_oracle_sample(case, dt):
    """NumPy oracle: one step of block 0 alone (its own self-contained stages)."""
    from oracle.ref import NP
    q = case.qs[0]
    kxyz, vol = case.metrics[0][1], case.metrics[0][2]
    cfg = case.cfg

    def L(x):
        return NP.rhs_block(x, kxyz, vol, cfg)

    t0 = time.perf_counter()
    NP.rk3_step(q, L, dt)
    el = time.perf_counter() - t0
    g = cfg.ghost
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
    # bounded sample of the workload: one block of the default case per step
    if args.workload == "wavy4":
        c = cases.wavy4(n=args.n, metrics_fn=lambda x: NP.compute_metrics(x, ghost=2), seed=args.seed)
        c.qs, c.metrics = c.qs[:1], c.metrics[:1]
    elif args.workload == "tgv32":
        c = cases.tgv(n=32)
    else:
        c = cases.tree24(seed=args.seed)
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
    g = c.cfg.ghost
    cells = c.interior_cells
    ms = statistics.median(times) * 1e3
    value = cells * 3 / (ms / 1e3) / 1e6
    sample = (f"PyTorch-CPU FP64 port of the reference algorithm, {cores} threads, one TVD-RK3 step of "
              f"block 0 ({c.qs[0].shape[1]}^3 padded) per step, median of {args.steps}")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_desc(c, args) | {"sample": "block 0 only"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference (JAX) not installable in this image: no jax/jaxlib wheel, no network"}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    import torch.distributed as dist

    from famrdp_jax_b200 import _capi, cases
    from famrdp_jax_b200.solver import diagnostics
    from famrdp_jax_b200.solver.step import StepPlan, rk_stage, step

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if ws > 1:
        dist.init_process_group("nccl", device_id=device, timeout=__import__("datetime").timedelta(seconds=300))

    case = build_case(args, device)
    state = cases.to_state(case, device)
    dt = diagnostics.cfl_dt(state, case.cfg, case.cfl)
    plan = StepPlan(state, case.cfg)
    qa = [b.q for b in state.blocks]
    qb = [torch.empty_like(q) for q in qa]

    def barrier():
        if ws > 1:
            dist.barrier()

    # ---- device-resident throughput -------------------------------------
    for _ in range(max(args.warmup, 3)):
        plan.run(qa, qb, dt)
        qa, qb = qb, qa
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n_launch0 = _capi.launch_count(device)
    with ClockSampler(_gpu_index(local)) as clk:
        e0.record(st)
        for _ in range(args.steps):
            plan.run(qa, qb, dt)
            qa, qb = qb, qa
        e1.record(st)
        torch.cuda.synchronize()
    launches = _capi.launch_count(device) - n_launch0
    barrier()
    ms_total = e0.elapsed_time(e1)
    if ws > 1:
        t = torch.tensor([ms_total], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_total = float(t.item())
    ms_step = ms_total / args.steps
    cells = case.interior_cells
    value = ws * cells * 3 * args.steps / (ms_total / 1e3) / 1e6

    # ---- dominant kernel group: one RK stage of block 0 ----------------------
    m0 = state.metrics[0]
    q0 = qa[0]
    out = torch.empty_like(q0)
    for _ in range(3):
        rk_stage(q0, q0, m0, case.cfg, dt, 2, out=out)
    torch.cuda.synchronize()
    reps = 10
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(st)
    for r in range(reps):
        rk_stage(q0, q0, m0, case.cfg, dt, 2, out=out)
    s1.record(st)
    torch.cuda.synchronize()
    stage_ms = s0.elapsed_time(s1) / reps
    padded0 = q0.shape[1] * q0.shape[2] * q0.shape[3]
    alg_bytes = STAGE_BYTES_F64 * padded0
    peak, peak_kind = _peaks()
    achieved = alg_bytes / (stage_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "kernel": "one TVD-RK3 stage of one block (staged pipeline)",
                "alg_bytes_per_launch": alg_bytes, "launch_ms": stage_ms, "peak_kind": peak_kind}

    # ---- end to end through step() with host buffers ---------------------
    host_in = [q.detach().cpu().pin_memory() for q in qa]
    host_out = [torch.empty_like(h).pin_memory() for h in host_in]
    dev_in = [torch.empty_like(q) for q in qa]
    e2e_steps = max(1, min(args.steps, 5))
    from famrdp_jax_b200.core.types import Block, State

    def e2e_step():
        for d, h in zip(dev_in, host_in):
            d.copy_(h, non_blocking=True)
        s = State(blocks=tuple(Block(q=d, xyz=b.xyz) for d, b in zip(dev_in, state.blocks)),
                  metrics=state.metrics)
        s2 = step(s, case.cfg, dt, plan=plan)
        for h, b in zip(host_out, s2.blocks):
            h.copy_(b.q, non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    x0, x1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    x0.record(st)
    for _ in range(e2e_steps):
        e2e_step()
    x1.record(st)
    torch.cuda.synchronize()
    e2e_ms = x0.elapsed_time(x1)
    if ws > 1:
        t = torch.tensor([e2e_ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    bytes_io = sum(h.numel() * 8 for h in host_in)
    e2e = {"value": ws * cells * 3 * e2e_steps / (e2e_ms / 1e3) / 1e6, "unit": UNIT,
           "h2d_bytes_per_step": bytes_io, "d2h_bytes_per_step": bytes_io,
           "ms_per_step": e2e_ms / e2e_steps, "steps": e2e_steps}

    cpu = None
    if rank == 0 and not args.no_cpu:
        cpu = cpu_oracle_sample(case, dt)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": max(args.warmup, 3), "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64" if args.precision == "f64" else "f32-flux/f64-state",
                "data": "synthetic", "config": workload_desc(case, args) | {"parallelism": f"replicas x{ws}"},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
                "clocks": clk.summary(), "step_hbm_gbs": STEP_BYTES_F64 * case.padded_cells * ws / (ms_step / 1e3) / 1e9,
                "dt": dt}
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["wavy4", "tgv32", "tree24"], default="wavy4")
    ap.add_argument("--precision", choices=["f64", "f32"], default="f64")
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle sample")
    args = ap.parse_args(argv)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
