"""Autotuner of the solver's schedule shapes (the front tiles of its launches).

A plan is built with a `dct_tuning` (include/dct.h): which fronts a single
CTA factors in shared memory (`small_front_max`), how many 64-column panels
a float32 trailing-update block holds (`update_block`, the K of the deferred
update), how the float32 substitution splits its K ranges over tasks
(`solve_target`, `solve_split_max`, `solve_split_min`) and whether
single-panel supernodes take the tensor-core products (`small_tc`).  The
best shapes depend on the pattern: a 3-D grid has a few fronts thousands of
rows wide, a batch of 2.5-D surveys thousands of narrow ones.

`tune_schedule` times one factorization plus one refined solve of the
actual pattern and right-hand-side width for candidate shapes, by
coordinate descent from the library's defaults (each field in turn, keeping
the fastest), and returns the best shapes with the timing table.  Results
are cached per pattern for the life of the process.  The reference has no
counterpart: cuDSS picks its own schedule (dctorch/solver.py:103-109).
"""
from __future__ import annotations

import hashlib

import numpy as np
import torch

from . import _native as nat

_CACHE = {}

# candidate values of each field, tried in this order (float32 / float64)
CANDIDATES = {
    nat.F32: [("small_front_max", (96, 128, 160, 192, 224)),
              ("update_block", (2, 3, 4)),
              ("solve_target", (296, 592, 1184)),
              ("small_tc", (1, 2))],
    nat.F64: [("small_front_max", (64, 96, 128, 160))],
}


def _key(crow, col, nbatch, n_rhs, code):
    h = hashlib.sha1()
    h.update(np.ascontiguousarray(crow, dtype=np.int32).tobytes())
    h.update(np.ascontiguousarray(col, dtype=np.int32).tobytes())
    return (h.hexdigest(), int(nbatch), int(n_rhs), int(code))


def _time_plan(sym, tuning, nbatch, n_rhs, code, device, vals, rhs, refine, reps):
    """Median device ms of factor + refined solve with one plan."""
    plan = nat.Plan(sym, nbatch, n_rhs, code, device.index, tuning)
    try:
        plan.set_refinement(refine)
        x = torch.empty((nbatch,) + tuple(rhs.shape), dtype=torch.float64, device=device)
        st = torch.cuda.current_stream(device)
        s = st.cuda_stream

        def step():
            plan.factorize(vals.data_ptr(), nat.F64, vals.shape[-1], s)
            plan.solve_permuted(rhs.data_ptr(), 0, rhs.shape[-1], x.data_ptr(), s)

        step()
        st.synchronize()
        out = []
        for _ in range(reps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(st)
            step()
            b.record(st)
            b.synchronize()
            out.append(a.elapsed_time(b))
        code_, _, _ = plan.status(s)
        if code_ != 0:
            return float("inf"), plan.tuning()
        return float(np.median(out)), plan.tuning()
    finally:
        plan.free()


def tune_schedule(crow, col, n, n_rhs, nbatch, device, dtype, vals, coords=None,
                  refine=2, reps=3):
    """(best tuning dict, [(tuning, ms), ...]) for nbatch systems on the
    pattern (crow, col) with values `vals` (nbatch, nnz) float64 on the
    device and n_rhs right-hand sides."""
    code = nat.F64 if dtype == torch.float64 else nat.F32
    key = _key(crow, col, nbatch, n_rhs, code)
    if key in _CACHE:
        return _CACHE[key]
    device = torch.device(device)
    sym = nat.Symbolic(np.asarray(crow, np.int32), np.asarray(col, np.int32), coords)
    vals = torch.as_tensor(vals, dtype=torch.float64, device=device).reshape(nbatch, -1)
    vals = vals.contiguous()
    rng = np.random.default_rng(0)
    rhs = torch.as_tensor(rng.standard_normal((n, n_rhs)), device=device)
    best = nat.default_tuning(code)
    table = []
    seen = {}

    def run(t):
        k = tuple(sorted(t.items()))
        if k not in seen:
            seen[k] = _time_plan(sym, t, nbatch, n_rhs, code, device, vals, rhs,
                                 refine, reps)[0]
            table.append((dict(t), seen[k]))
        return seen[k]

    best_ms = run(best)
    for field, values in CANDIDATES[code]:
        for v in values:
            t = dict(best)
            t[field] = v
            ms = run(t)
            if ms < best_ms:
                best, best_ms = t, ms
    _CACHE[key] = (best, table)
    return best, table
