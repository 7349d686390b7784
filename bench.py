#!/usr/bin/env python
"""Benchmark of the DC forward + adjoint hot path: eval+grad =
`eng.misfit(m, dobs, w).backward()` (dpred + the full adjoint gradient).

Default workload: the 3-D DC problem (TensorMesh 64x64x32 core cells of 5 m +
8 padding cells per face, 256,000 cells, 269,001 nodes; 10x10 surface grid,
200 pole-dipole sources, 6,000 data; layered model + 2 ellipsoids).
`value` is the float32 factor/solve + float64 iterative refinement eval+grad
time, accepted only at dpred rel-err <= 1e-6 and gradient rel-err <= 1e-5
against the float64 path of the same engine, whose time is reported beside it
(`fp64_ms`).  Inputs are resident in HBM for `value`; `e2e` repeats the step
through the public API from pinned host buffers (model, data, weights in;
misfit and gradient out).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
                    [--workload dc3d|dc2d_large|dc2d_small]

With N > 1 (torchrun, one process per GPU) every rank solves its own seeded
instance of the workload (independent replicas: the path has no exchange
step at one survey per GPU); the time is the max over ranks.

`--impl reference` times the reference algorithm on the host cores (the CPU
oracle, a float64 SuperLU restatement of the reference's CPU path) on a
bounded sample of the workload, rank 0 only.
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
sys.path.insert(0, ROOT)

METRIC = "eval+grad ms, FP32+IR vs plain FP64 on same B200, at dpred rel-err ≤1e-6"

WORKLOADS = {
    "dc3d": dict(desc="3-D DC, TensorMesh 64x64x32 core @5 m + 8 padding/face "
                      "(x1.3), 10x10 surface grid, 200 pole-dipole sources, "
                      "~30 receivers each"),
    "dc2d_large": dict(desc="2.5-D DC, TensorMesh 400x120 core @1 m + padding "
                            "(x1.3), 96 electrodes, dipole-dipole + Wenner, nky 12"),
    "dc2d_small": dict(desc="2.5-D DC, TensorMesh 100x50 core @2.5 m + 10 padding "
                            "(x1.3), 21 electrodes, dipole-dipole n=1..6, nky 11"),
    # a reduced 3-D case for profiler captures (a few GB on the device)
    "dc3d_mid": dict(desc="3-D DC, TensorMesh 40x40x20 core @8 m + 6 padding/face "
                          "(x1.3), same 200 sources and 6,000 data"),
}
# bounded CPU sample: the same workload family on a coarser grid
CPU_SAMPLE = {
    "dc3d": dict(kw=dict(ncore=(24, 24, 12), dx=13.0, npad=4),
                 desc="3-D workload family coarsened: 24x24x12 core cells of "
                      "13 m + 4 padding/face (18,513 nodes), same 200 sources "
                      "and 6,000 data; one full eval+grad per step"),
    "dc2d_large": dict(kw={}, desc="the full 2.5-D workload"),
    "dc2d_small": dict(kw={}, desc="the full 2.5-D workload"),
    "dc3d_mid": dict(kw=dict(ncore=(24, 24, 12), dx=13.0, npad=4),
                     desc="coarsened as for dc3d"),
}


def build_case(name, seed, sample=False):
    from simpeg_dc_torch_b200 import synthetic as syn
    if name in ("dc3d", "dc3d_mid"):
        kw = CPU_SAMPLE[name]["kw"] if sample else (
            {} if name == "dc3d" else dict(ncore=(40, 40, 20), dx=8.0, npad=6))
        return syn.dc3d(seed=seed, **kw)
    if name == "dc2d_large":
        return syn.dc2d_large(seed=seed)
    return syn.dc2d_small(seed=seed)


def make_engine(name, mesh, survey, device, dtype):
    from simpeg_dc_torch_b200 import TorchDC2D, TorchDC3D
    if name in ("dc3d", "dc3d_mid"):
        return TorchDC3D(mesh, survey, device=device, dtype=dtype)
    nky = 12 if name == "dc2d_large" else 11
    return TorchDC2D(mesh, survey, nky=nky, device=device, dtype=dtype)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,"
              "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# -------------------------------------------------------------- reference
def oracle_ops(name, mesh, survey):
    from oracle import dc_oracle as O  # noqa: F401
    from simpeg_dc_torch_b200.operators import nodal_operators
    from simpeg_dc_torch_b200.quadrature import (electrode_distance_range,
                                                 k0_quadrature)
    import scipy.sparse as sp
    ops = nodal_operators(mesh, survey)
    op = dict(crow=ops.crow, col=ops.col, nN=ops.nN, Q=ops.q.toarray(),
              Pd=ops.Pd, sidx=ops.sidx)
    if name.startswith("dc3d"):
        op["L3"] = ops.L3()
    else:
        nky = 12 if name == "dc2d_large" else 11
        kys, wq, _ = k0_quadrature(*electrode_distance_range(survey), nky)
        op["Lstack"] = sp.vstack([ops.L_ky(k) for k in kys]).tocsr()
        op["wq"] = wq
    return op


def cpu_eval_grad_timer(name, seed=0):
    """Returns (run_once, sample description): one oracle eval+grad."""
    from oracle import dc_oracle as O
    from simpeg_dc_torch_b200 import synthetic as syn
    mesh, survey, m = build_case(name, seed, sample=True)
    op = oracle_ops(name, mesh, survey)
    three_d = name.startswith("dc3d")
    d = O.dpred_3d(op, m) if three_d else O.dpred_2d(op, m)
    dobs, w = syn.observed(d, np.random.default_rng(seed + 1))

    def once():
        t = time.perf_counter()
        if three_d:
            O.misfit_grad_3d(op, m, dobs, w)
        else:
            O.misfit_grad_2d(op, m, dobs, w)
        return 1e3 * (time.perf_counter() - t)
    return once, CPU_SAMPLE[name]["desc"]


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    once, desc = cpu_eval_grad_timer(args.workload)
    for _ in range(args.warmup):
        once()
    ts = [once() for _ in range(args.steps)]
    ms = float(np.mean(ts))
    cores = os.cpu_count()
    line = {
        "impl": "reference", "metric": METRIC, "value": ms, "unit": "ms",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload,
                   "description": WORKLOADS[args.workload]["desc"],
                   "sample": desc},
        "cpu_baseline": {"value": ms, "unit": "ms", "cores": cores,
                         "kind": "port", "sample": desc,
                         "note": "float64 SuperLU (scipy splu, single-threaded "
                                 "factorization) restatement of the reference's "
                                 "CPU path"},
        "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------- ours
def count_launches(eng):
    """Kernels of libdct launched by one eval+grad (forward + adjoint),
    counted from the plan's launch schedules (the same lists the library
    walks) and the fixed launches of the fused path around them."""
    sym = eng.solver._sym
    code = eng.solver._code
    nl = {}
    for which in range(5):
        _, launches = sym.schedule(code, which)
        nl[which] = int((launches[:, 3] > 0).sum())
    # factor: schedule + panel inverses + supernode inverses, the lower-
    # triangle clearing launched with every large-front scatter, and the
    # float64 value copy of float32 plans
    _, fl = sym.schedule(code, 0)
    nscatter = int(((fl[:, 0] == 1) & (fl[:, 3] > 0)).sum())
    factor = nl[0] + nscatter + nl[3] + nl[4] + (1 if code == 1 else 0)
    passes = nl[1] + nl[2]
    if code == 0:
        solve = 1 + passes                       # rhs copy + substitution
    else:
        ir = eng.solver.refine
        solve = 1 + (1 + ir) * (passes + 1) + ir  # + updates and residuals
    # sigma/values (2), source scatter, projection, adjoint scatter,
    # gather-contract, values vjp
    return 7 + factor + 2 * solve


# launch kinds whose dominant cost is tensor-core arithmetic (float32 plans)
TENSOR_KINDS = {"trailing_update", "fwd_linv_tc", "fwd_bnd_tc", "bwd_gemm_tc",
                "bwd_linv_tc"}


def max_over_ranks(x, world, device):
    """The maximum of a per-rank value over all ranks of the job (every rank
    calls it, in the same order); with one rank, the value itself."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="dc3d", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    from simpeg_dc_torch_b200 import synthetic as syn

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def rank_max(x):
        return max_over_ranks(x, world, dev)

    mesh, survey, m_np = build_case(args.workload, seed=rank)
    e32 = make_engine(args.workload, mesh, survey, dev, torch.float32)
    e64 = make_engine(args.workload, mesh, survey, dev, torch.float64)
    m = torch.tensor(m_np, device=dev)
    with torch.no_grad():
        d64 = e64.dpred(m)
    dobs_np, w_np = syn.observed(d64.cpu().numpy(),
                                 np.random.default_rng(100 + rank))
    dobs = torch.tensor(dobs_np, device=dev)
    w = torch.tensor(w_np, device=dev)

    def eval_grad(eng, mm):
        x = mm.detach().requires_grad_(True)
        phi = eng.misfit(x, dobs, w)
        phi.backward()
        return phi.detach(), x.grad

    # accuracy of the float32 + refinement path against float64
    phi64, g64 = eval_grad(e64, m)
    phi32, g32 = eval_grad(e32, m)
    with torch.no_grad():
        d32 = e32.dpred(m)
    e32.check()
    e64.check()
    acc = {"dpred_rel": float(torch.linalg.norm(d32 - d64) / torch.linalg.norm(d64)),
           "grad_rel": float(torch.linalg.norm(g32 - g64) / torch.linalg.norm(g64)),
           "phi_rel": float(abs(phi32 - phi64) / abs(phi64))}

    def timed(eng, steps, warmup, sampler=None, tag=None):
        for _ in range(warmup):
            eval_grad(eng, m)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        if sampler:
            sampler.start()
        st = torch.cuda.current_stream()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        if tag:   # NVTX range: lets a profiler select the timed launches
            torch.cuda.nvtx.range_push(tag)
        a.record(st)
        for _ in range(steps):
            eval_grad(eng, m)
        b.record(st)
        if tag:
            torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        clocks = sampler.stop() if sampler else None
        barrier()
        return rank_max(a.elapsed_time(b) / steps), clocks

    sampler = ClockSampler(local)
    ms32, clocks = timed(e32, args.steps, args.warmup, sampler, tag="timed_fp32")
    ms64, _ = timed(e64, args.steps, args.warmup, tag="timed_fp64")

    # end to end through the public API, host buffers in and out
    e2e = None
    if not args.no_e2e:
        m_h = torch.tensor(m_np).pin_memory()
        dobs_h = torch.tensor(dobs_np).pin_memory()
        w_h = torch.tensor(w_np).pin_memory()
        g_h = torch.empty_like(m_h).pin_memory()
        phi_h = torch.empty((), dtype=torch.float64).pin_memory()

        def e2e_step():
            md = m_h.to(dev, non_blocking=True).requires_grad_(True)
            dd = dobs_h.to(dev, non_blocking=True)
            wd = w_h.to(dev, non_blocking=True)
            phi = e32.misfit(md, dd, wd)
            phi.backward()
            g_h.copy_(md.grad, non_blocking=True)
            phi_h.copy_(phi.detach(), non_blocking=True)

        for _ in range(args.warmup):
            e2e_step()
        torch.cuda.synchronize()
        barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.steps):
            e2e_step()
        b.record()
        torch.cuda.synchronize()
        barrier()
        e2e_ms = rank_max(a.elapsed_time(b) / args.steps)
        e2e = {"value": e2e_ms, "unit": "ms",
               "h2d_bytes_per_step": (m_h.numel() + dobs_h.numel()
                                      + w_h.numel()) * 8,
               "d2h_bytes_per_step": (g_h.numel() + 1) * 8}

    # per-kernel-kind device time of one profiled eval+grad (CUDA events)
    plan = e32.solver.plan
    plan.profile(True, reset=True)
    for _ in range(2):
        eval_grad(e32, m)
    torch.cuda.synchronize()
    prof = plan.profile_read()
    plan.profile(False, reset=True)
    tot = sum(v[0] for v in prof.values())
    dom = max(prof, key=lambda k: prof[k][0])
    dms, dn, dfl, dby = prof[dom]
    import json as _j
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = _j.load(open(pk))
    hbm = peaks.get("hbm_gbs", 6650.0)
    tc = peaks.get("bf16_tflops", 1590.0)
    traffic = None
    tj = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tj):
        traffic = _j.load(open(tj)).get(args.workload, {}).get(dom)
    if dom in TENSOR_KINDS:
        ach = dfl / (dms * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": ach, "peak": tc, "unit": "TFLOP/s",
                "frac": ach / tc,
                "note": "3xTF32: three TF32 MMAs per product; the TF32 rate is "
                        "half the bf16 rate, so this kernel's ceiling is "
                        "peak/6 (frac_of_3xtf32_ceiling)",
                "frac_of_3xtf32_ceiling": ach / (tc / 6.0)}
    else:
        ach = dby / (dms * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s",
                "frac": ach / hbm}
    roof.update({"kernel": dom, "launches_per_step": dn / 2,
                 "avg_launch_ms": dms / max(dn, 1),
                 "algorithmic_bytes_per_launch": dby / max(dn, 1),
                 "algorithmic_flops_per_launch": dfl / max(dn, 1),
                 "share_of_solver_time": dms / tot if tot else None,
                 "traffic": traffic,
                 "peak_source": ("MEASURED_PEAKS.json (burst)" if peaks
                                 else "fallback")})

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        once, desc = cpu_eval_grad_timer(args.workload)
        once()
        t0 = time.perf_counter()
        ts = []
        while len(ts) < 3 and time.perf_counter() - t0 < 20:
            ts.append(once())
        cpu = {"value": float(np.mean(ts)), "unit": "ms",
               "cores": os.cpu_count(), "kind": "port", "sample": desc,
               "note": "CPU oracle (float64 SuperLU restatement of the "
                       "reference's CPU path); SuperLU factorization is "
                       "single-threaded"}

    sinfo = e32.solver.analysis()
    if rank == 0:
        line = {
            "metric": METRIC, "value": ms32, "unit": "ms", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms32,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 factor/solve + f64 refinement, f64 data/misfit",
            "data": "synthetic (seeded)",
            "config": {"workload": args.workload,
                       "description": WORKLOADS[args.workload]["desc"],
                       "cells": int(e32.nC), "nodes": int(e32.nN),
                       "sources": int(e32.nS), "data": int(e32.nD),
                       "nsystems": int(e32.solver.nbatch),
                       "nnz_L": int(sinfo["nnz_L"]),
                       "factor_flops": float(sinfo["flops_factor"]),
                       "l2": "inputs larger than L2 (float32 fronts "
                             f"{4 * sinfo['front_total'] * e32.solver.nbatch / 1e9:.2f} GB)",
                       "parallelism": f"replicas x{world}"},
            "fp64_ms": ms64, "speedup_vs_fp64": ms64 / ms32,
            "accuracy_vs_fp64": acc,
            "e2e": e2e, "gpu_launches": count_launches(e32),
            "roofline": roof,
            "kernel_ms": {k: v[0] / 2 for k, v in prof.items()},
            "cpu_baseline": cpu, "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
