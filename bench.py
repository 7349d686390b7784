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
oracle, a float64 SuperLU restatement of the reference's CPU path), rank 0
only: the whole eval+grad per step on dc2d_small, an exactly scaled sample
of the same workload on dc2d_large (see ReferenceCpu); on the 3-D workloads
one eval+grad takes ~30 minutes on the CPU, and the arm prints an
`unavailable` line with the measured figures instead.
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

# l2: how the timed steps avoid reading a warm L2 (126 MB) -- inputs larger
# than L2, or an L2 flush (a 512 MB write) between timed steps
WORKLOADS = {
    "dc3d": dict(desc="3-D DC, TensorMesh 64x64x32 core @5 m + 8 padding/face "
                      "(x1.3), 10x10 surface grid, 200 pole-dipole sources, "
                      "~30 receivers each",
                 l2="inputs larger than L2 (float32 fronts 3.8 GB, fields 0.43 GB)",
                 flush=False),
    "dc2d_large": dict(desc="2.5-D DC, TensorMesh 400x120 core @1 m + padding "
                            "(x1.3), 96 electrodes, dipole-dipole + Wenner, nky 12",
                       l2="inputs larger than L2 (float32 fronts 0.56 GB, fields 1.0 GB)",
                       flush=False),
    "dc2d_small": dict(desc="2.5-D DC, TensorMesh 100x50 core @2.5 m + 10 padding "
                            "(x1.3), 21 electrodes, dipole-dipole n=1..6, nky 11",
                       l2="L2 flushed between timed steps (working set ~0.1 GB)",
                       flush=True),
    "dc2d_batch": dict(desc="64 independent 2.5-D DC surveys of uneven size (5k-40k "
                            "cells, 24-64 electrodes, dipole-dipole n=1..6, nky 12) "
                            "in the same launches; autotuned schedule shapes",
                       l2="inputs larger than L2 (float32 fronts of 64 surveys)",
                       flush=False),
    # a reduced 3-D case for profiler captures (a few GB on the device)
    "dc3d_tree": dict(desc="3-D DC, octree TreeMesh (2:1 balanced, 5 m finest cells "
                           "refined around a 21x21 surface grid at 10 m, 293,868 "
                           "cells, 286,960 free nodes), 400 gradient-array sources "
                           "x 40 dipoles (16,000 data), Gaussian random field "
                           "log-rho (50 m correlation, sigma 0.5)",
                      l2="inputs larger than L2 (fields 0.92 GB in float64)",
                      flush=False),
    "dc3d_mid": dict(desc="3-D DC, TensorMesh 40x40x20 core @8 m + 6 padding/face "
                          "(x1.3), same 200 sources and 6,000 data",
                     l2="inputs larger than L2 (float32 fronts 0.62 GB)",
                     flush=False),
}
# The reference's CPU path (float64 SuperLU, scipy splu with its default
# COLAMD ordering, single-threaded; dctorch/solver.py:314-374) cannot run
# every workload inside a bench run.  Measured in the build container (one
# core): the 269,001-node 3-D system takes 951.6 s to factor (nnz(L) =
# nnz(U) = 4.46e8) and 23.8 s per 10 right-hand sides to solve, so one
# eval+grad with 200 sources (factor + 2 x 200 right-hand sides) is ~1,900 s;
# the 75,843-node 3-D case did not finish its factorization in 7 minutes.
# The 2.5-D workloads factor in well under a second per wavenumber but solve
# slowly (56,525 nodes: 39 s per wavenumber for 186 right-hand sides).
REFERENCE_3D_UNAVAILABLE = (
    "the reference's CPU path (float64 SuperLU, COLAMD, single-threaded) takes "
    "~1,900 s per eval+grad on this 3-D workload (factorization of the 269,001-"
    "node system measured at 951.6 s, solves at 23.8 s per 10 right-hand sides, "
    "200 sources forward + 200 adjoint), so warm-up + timed steps cannot finish "
    "in a bench run; no smaller grid stands in for it")
REFERENCE_TREE_UNAVAILABLE = (
    "the reference builds TreeMesh operators through SimPEG/discretize, which "
    "are absent, and its CPU path (float64 SuperLU, single-threaded) on this "
    "286,960-node octree system with 400 sources (factor + 800 right-hand "
    "sides) exceeds the ~1,900 s measured for the 269,001-node tensor case")


def _unavailable_reason(name):
    return REFERENCE_TREE_UNAVAILABLE if name == "dc3d_tree" else REFERENCE_3D_UNAVAILABLE


def build_case(name, seed):
    from simpeg_dc_torch_b200 import synthetic as syn
    if name == "dc3d":
        return syn.dc3d(seed=seed)
    if name == "dc3d_mid":
        return syn.dc3d(seed=seed, ncore=(40, 40, 20), dx=8.0, npad=6)
    if name == "dc3d_tree":
        return syn.dc3d_tree(seed=seed)
    if name == "dc2d_large":
        return syn.dc2d_large(seed=seed)
    if name == "dc2d_batch":
        probs = syn.dc2d_batch(n_problems=64, seed=seed)
        return ([(mesh, survey) for mesh, survey, _ in probs], None,
                np.concatenate([m for *_, m in probs]))
    return syn.dc2d_small(seed=seed)


def workload_config(name):
    """The workload as both arms name it (identical dicts)."""
    return {"workload": name, "description": WORKLOADS[name]["desc"],
            "l2": WORKLOADS[name]["l2"]}


def make_engine(name, mesh, survey, device, dtype):
    """The engine of a workload; for dc2d_batch `mesh` is the list of
    (mesh, survey) problems."""
    from simpeg_dc_torch_b200 import TorchDC2D, TorchDC2DBatch, TorchDC3D
    if name == "dc2d_batch":
        import torch
        return TorchDC2DBatch(mesh, nky=12, device=device, dtype=dtype,
                              tune=dtype == torch.float32)
    if name in ("dc3d", "dc3d_mid", "dc3d_tree"):
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


class ReferenceCpu:
    """The reference's CPU eval+grad (the oracle's SuperLU restatement of
    dctorch/solver.py:314-374 with the engines' chain) on a 2.5-D workload.

    dc2d_small: one full eval+grad per step.  dc2d_large: each step is a
    bounded sample of the same workload -- the factorization of one of its
    wavenumber systems (cycling through them) and the forward and adjoint
    solves of all source columns on it, as the reference's batch solver
    does per system -- scaled exactly to one eval+grad: the wavenumber
    systems are independent, so eval+grad = nky (t_factor + t_solves) +
    t_rest, with the projection / contraction rest timed once on the full
    problem.  `cols` < the source count solves that many columns and scales
    the solve time linearly (SuperLU solves column by column)."""

    def __init__(self, name, seed=0, cols=None):
        from oracle import dc_oracle as O
        from simpeg_dc_torch_b200 import synthetic as syn
        self.name, self.O = name, O
        if name == "dc2d_batch":
            self._init_batch(seed)
            return
        mesh, survey, m = build_case(name, seed)
        self.op = op = oracle_ops(name, mesh, survey)
        self.m = m
        self.nky = len(op["wq"])
        self.nS = op["Q"].shape[1]
        self.cols = self.nS if cols is None else min(int(cols), self.nS)
        self.vals = O.vals_2d(op["Lstack"], m, self.nky)
        self.step_i = 0
        if name == "dc2d_small":
            d = O.dpred_2d(op, m)
            self.dobs, self.w = syn.observed(d, np.random.default_rng(seed + 1))
            self.desc = "the full workload: one eval+grad per step"
            return
        # the rest of the chain around the solves, on the full problem:
        # quadrature sum + projection, adjoint scatter, contraction, L^T
        rng = np.random.default_rng(seed + 1)
        U = rng.standard_normal((self.nky, op["nN"], self.nS))
        t = time.perf_counter()
        Ubar = np.tensordot(op["wq"], U, axes=(0, 0))
        PU = op["Pd"] @ Ubar
        d = PU[np.arange(PU.shape[0]), op["sidx"]]
        G = np.zeros((op["Pd"].shape[0], self.nS))
        G[np.arange(G.shape[0]), op["sidx"]] = d
        GU = op["Pd"].T @ G
        r = O.row_of(op["crow"])
        gv = np.empty((self.nky, len(op["col"])))
        for k in range(self.nky):
            gv[k] = -op["wq"][k] * np.einsum("es,es->e", U[k][r], U[k][op["col"]])
        _ = op["Lstack"].T @ gv.reshape(-1) + GU.sum()
        self.t_rest = 1e3 * (time.perf_counter() - t)
        self.desc = (f"each step: SuperLU factorization of one of the "
                     f"{self.nky} wavenumber systems and forward + adjoint "
                     f"solves of {self.cols} of its {self.nS} source columns, "
                     f"scaled exactly to one eval+grad ({self.nky} systems, "
                     f"{self.nS} columns each way) plus the projection / "
                     f"contraction rest timed once ({self.t_rest:.0f} ms)")

    def _init_batch(self, seed):
        """dc2d_batch: every survey with its own operators and quadrature;
        step k factors and solves wavenumber system k of every survey
        (forward and adjoint, all its sources) and scales by the number of
        systems: over a cycle of steps, exactly the factorizations and
        solves of one eval+grad of all 64 surveys (the projection /
        contraction rest is left out, so the CPU time is understated)."""
        import scipy.sparse as sp
        from simpeg_dc_torch_b200.quadrature import (electrode_distance_range,
                                                     k0_quadrature)
        from simpeg_dc_torch_b200.operators import nodal_operators
        problems, _, m = build_case("dc2d_batch", seed)
        self.surveys = []
        c0 = 0
        for mesh, survey in problems:
            o = nodal_operators(mesh, survey)
            kys, wq, _ = k0_quadrature(*electrode_distance_range(survey), 12)
            mb = m[c0:c0 + o.nC]
            c0 += o.nC
            sig = np.exp(-mb)
            vals = [o.L_ky(k) @ sig for k in kys]
            self.surveys.append((o, vals))
        self.nky = max(len(v) for _, v in self.surveys)
        self.step_i = 0
        self.desc = ("each step: SuperLU factorization of wavenumber system k of "
                     "all 64 surveys and their forward + adjoint solves (all "
                     "sources), scaled by the number of systems (projection / "
                     "contraction left out)")

    def step(self):
        O = self.O
        if self.name == "dc2d_batch":
            import scipy.sparse as sp
            import scipy.sparse.linalg as spla
            k = self.step_i % self.nky
            self.step_i += 1
            t = time.perf_counter()
            for o, vals in self.surveys:
                if k >= len(vals):
                    continue
                lu = spla.splu(sp.csr_matrix((vals[k], o.col, o.crow),
                                             shape=(o.nN, o.nN)).tocsc())
                x = lu.solve(o.q.toarray())
                lu.solve(np.ascontiguousarray(x[::-1]))
            return 1e3 * self.nky * (time.perf_counter() - t)
        op = self.op
        if self.name == "dc2d_small":
            t = time.perf_counter()
            O.misfit_grad_2d(op, self.m, self.dobs, self.w)
            return 1e3 * (time.perf_counter() - t)
        import scipy.sparse as sp
        import scipy.sparse.linalg as spla
        k = self.step_i % self.nky
        c0 = (self.step_i * self.cols) % self.nS
        self.step_i += 1
        cols = np.arange(c0, c0 + self.cols) % self.nS
        t = time.perf_counter()
        lu = spla.splu(sp.csr_matrix((self.vals[k], op["col"], op["crow"]),
                                     shape=(op["nN"], op["nN"])).tocsc())
        t_f = time.perf_counter() - t
        B = np.ascontiguousarray(op["Q"][:, cols])
        t = time.perf_counter()
        x = lu.solve(B)
        lu.solve(np.ascontiguousarray(x[::-1]))      # the adjoint solve
        t_s = time.perf_counter() - t
        return 1e3 * self.nky * (t_f + t_s * self.nS / self.cols) + self.t_rest


def reference_line(args, ms, desc, cores):
    return {
        "impl": "reference", "metric": METRIC, "value": ms, "unit": "ms",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": workload_config(args.workload),
        "cpu_baseline": {"value": ms, "unit": "ms", "cores": cores,
                         "kind": "port", "sample": desc,
                         "note": "float64 SuperLU (scipy splu, COLAMD, "
                                 "single-threaded) restatement of the "
                                 "reference's CPU path"},
        "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.workload.startswith("dc3d"):
        print(json.dumps({"impl": "reference", "metric": METRIC,
                          "config": workload_config(args.workload),
                          "unavailable": _unavailable_reason(args.workload)}), flush=True)
        return 0
    ref = ReferenceCpu(args.workload)
    for _ in range(args.warmup):
        ref.step()
    ts = [ref.step() for _ in range(args.steps)]
    ms = float(np.mean(ts))
    print(json.dumps(reference_line(args, ms, ref.desc, 1)), flush=True)
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
        # conversion, first solve and update, then per correction the
        # residual, the solve, the update and the stopping decision (the
        # launches of corrections not needed still run, and return at entry)
        ir = eng.solver.refine
        solve = 2 + passes + ir * (passes + 3)
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


def cpu_baseline_leg(name):
    """The reference's CPU path timed on the host cores beside the GPU line:
    a bounded run of `ReferenceCpu` steps (2.5-D workloads, ~20 s), or, for
    the 3-D workloads, the reason it cannot run with the full-size record."""
    if name.startswith("dc3d"):
        out = {"value": None, "unit": "ms", "cores": 1, "kind": "port",
               "sample": "none", "unavailable": _unavailable_reason(name)}
        if name == "dc3d":
            # 951.6 s factorization + 2 x 200 right-hand sides at 2.38 s each
            out["recorded_full_size_estimate_ms"] = 1e3 * (951.6 + 2 * 200 * 2.38)
        return out
    ref = ReferenceCpu(name)
    ref.step()
    t0 = time.perf_counter()
    ts = []
    while len(ts) < 3 or (len(ts) < 12 and time.perf_counter() - t0 < 30):
        ts.append(ref.step())
    return {"value": float(np.mean(ts)), "unit": "ms", "cores": 1,
            "kind": "port", "sample": ref.desc,
            "note": "float64 SuperLU (scipy splu, COLAMD, single-threaded) "
                    "restatement of the reference's CPU path"}


def factor_once(args, mesh, survey, m_np, dev):
    """One float32 factorization inside the NVTX range `fact_once`, after a
    warm eval+grad and a warm factorization: the launch list of one
    factorization for ncu (--nvtx --nvtx-include "fact_once/")."""
    import torch
    e32 = make_engine(args.workload, mesh, survey, dev, torch.float32)
    m = torch.tensor(m_np, device=dev, requires_grad=True)
    with torch.no_grad():
        d = e32.dpred(m)
    e32.misfit(m, d * 1.05, 1.0 / d.abs()).backward()
    _, vals = e32._path.values(m.detach())
    e32._path.factorize(vals)
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("fact_once")
    a.record()
    e32._path.factorize(vals)
    b.record()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    e32.check()
    print(json.dumps({"workload": args.workload, "factorization_ms": a.elapsed_time(b)}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="dc3d", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--side", action="store_true",
                    help="also time the complex-resistivity and DC-IP engines "
                         "(2.5-D workloads)")
    ap.add_argument("--factor-once", action="store_true",
                    help="profiling mode: one float32 eval+grad, then one "
                         "factorization inside the NVTX range fact_once (3-D "
                         "workloads); prints its time and no bench line")
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
    if args.factor_once:
        return factor_once(args, mesh, survey, m_np, dev)
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

    # accuracy of the float32 + refinement path against float64, and the
    # refinement record of the forward and adjoint solves of that step
    phi64, g64 = eval_grad(e64, m)
    e32._path.record_refinement = True
    phi32, g32 = eval_grad(e32, m)
    e32._path.record_refinement = False
    refinement = {k: {"corrections": v["iters"], "converged": v["converged"],
                      "est_error": v["est_error"], "rho": v["rho"]}
                  for k, v in e32._path.last_refinement.items()}
    with torch.no_grad():
        d32 = e32.dpred(m)
    e32.check()
    e64.check()
    acc = {"dpred_rel": float(torch.linalg.norm(d32 - d64) / torch.linalg.norm(d64)),
           "grad_rel": float(torch.linalg.norm(g32 - g64) / torch.linalg.norm(g64)),
           "phi_rel": float(abs(phi32 - phi64) / abs(phi64))}

    # working sets below L2: a 512 MB write between timed steps, outside
    # the timed events
    flush_buf = (torch.empty(512 << 20, dtype=torch.uint8, device=dev)
                 if WORKLOADS[args.workload]["flush"] else None)

    def timed_loop(step, steps, warmup, sampler=None, tag=None):
        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        if sampler:
            sampler.start()
        st = torch.cuda.current_stream()
        if tag:   # NVTX range: lets a profiler select the timed launches
            torch.cuda.nvtx.range_push(tag)
        pairs = []
        if flush_buf is None:
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(st)
            for _ in range(steps):
                step()
            b.record(st)
            pairs.append((a, b))
        else:
            for _ in range(steps):
                flush_buf.zero_()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(st)
                step()
                b.record(st)
                pairs.append((a, b))
        if tag:
            torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        clocks = sampler.stop() if sampler else None
        barrier()
        ms = sum(a.elapsed_time(b) for a, b in pairs) / steps
        return rank_max(ms), clocks

    sampler = ClockSampler(local)
    ms32, clocks = timed_loop(lambda: eval_grad(e32, m), args.steps, args.warmup,
                              sampler, tag="timed_fp32")
    ms64, _ = timed_loop(lambda: eval_grad(e64, m), args.steps, args.warmup,
                         tag="timed_fp64")

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

        e2e_ms, _ = timed_loop(e2e_step, args.steps, args.warmup)
        e2e = {"value": e2e_ms, "unit": "ms",
               "h2d_bytes_per_step": (m_h.numel() + dobs_h.numel()
                                      + w_h.numel()) * 8,
               "d2h_bytes_per_step": (g_h.numel() + 1) * 8}

    # the same eval+grad (misfit and gradient, no autograd) replayed from one
    # CUDA graph of the whole launch sequence
    graph = None
    if not args.no_graph:
        from simpeg_dc_torch_b200 import GraphedMisfitGrad
        gmg = GraphedMisfitGrad(e32, m, dobs, w)
        phi_g, g_g = gmg.replay(m)
        graph_rel = float(torch.linalg.norm(g_g - g32) / torch.linalg.norm(g32))
        graph_ms, _ = timed_loop(lambda: gmg.replay(m), args.steps, args.warmup)
        graph = {"value": graph_ms, "unit": "ms", "launches": 1,
                 "kernel_nodes": count_launches(e32),
                 "grad_rel_vs_autograd": graph_rel}
        del gmg

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
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    hbm = peaks.get("hbm_gbs", 6650.0)
    tc = peaks.get("bf16_tflops", 1590.0)
    traffic, traffic_launch = None, None
    tj = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tj):
        tw = json.load(open(tj)).get(args.workload, {})
        traffic, traffic_launch = tw.get(dom), tw.get(dom + "_launch")
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
                 "traffic": traffic, "traffic_launch": traffic_launch,
                 "peak_source": ("MEASURED_PEAKS.json (burst)" if peaks
                                 else "fallback")})

    # the side engines on the same 2.5-D mesh and survey: complex resistivity
    # (complex128 L L^T) and joint DC + IP (two float64 states), eval+grad
    side = None
    if args.side and args.workload in ("dc2d_small", "dc2d_large"):
        from simpeg_dc_torch_b200 import TorchCR2D, TorchDCIP2D
        nky = 12 if args.workload == "dc2d_large" else 11
        chg = torch.tensor(np.random.default_rng(5).uniform(0.01, 0.2, m.numel()),
                           device=dev)
        side = {}
        for name, eng, mm in (
                ("cr2d_complex128", TorchCR2D(mesh, survey, nky=nky, device=dev,
                                              ip_scale=1000.0), torch.cat([m, chg])),
                ("dcip2d_float64", TorchDCIP2D(mesh, survey, nky=nky, device=dev,
                                               eta_max=0.8, ip_scale=1000.0),
                 torch.cat([m, torch.logit(chg / 0.8)]))):
            with torch.no_grad():
                d_a, d_b = eng.dpred(mm)
            oa = d_a * 1.03
            ob = d_b + 2.0
            wa, wb = 1.0 / oa.abs(), torch.full_like(ob, 0.5)

            def side_step(eng=eng, mm=mm, oa=oa, ob=ob, wa=wa, wb=wb):
                x = mm.detach().requires_grad_(True)
                eng.misfit(x, oa, wa, ob, wb, lam=0.7).backward()

            ms_side, _ = timed_loop(side_step, args.steps, args.warmup)
            eng.check()
            side[name] = {"value": ms_side, "unit": "ms",
                          "model": int(mm.numel()), "data": 2 * int(d_a.numel())}
            del eng

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_leg(args.workload)

    sinfo = e32.solver.analysis()
    if rank == 0:
        line = {
            "metric": METRIC, "value": ms32, "unit": "ms", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms32,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 factor/solve + f64 refinement, f64 data/misfit",
            "data": "synthetic (seeded)",
            "config": workload_config(args.workload),
            "problem": {"cells": int(e32.nC), "nodes": int(e32.nN),
                        "sources": int(e32.nS), "data": int(e32.nD),
                        "nsystems": int(e32.solver.nbatch),
                        "nnz_L": int(sinfo["nnz_L"]),
                        "factor_flops": float(sinfo["flops_factor"]),
                        "parallelism": f"replicas x{world}"},
            "fp64_ms": ms64, "speedup_vs_fp64": ms64 / ms32,
            "accuracy_vs_fp64": acc, "refinement": refinement,
            "e2e": e2e, "graph": graph, "side_engines": side,
            "gpu_launches": count_launches(e32),
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
