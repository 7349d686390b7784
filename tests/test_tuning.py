"""The schedule tuner's search on the CPU, with the device timing replaced
by a cost function of the candidate shapes: coordinate descent from the
library's defaults (each field in turn, keeping the fastest), every shape
timed once, plans that report an error ranked last, results cached per
pattern."""
import numpy as np
import scipy.sparse as sp
import torch

from simpeg_dc_torch_b200 import _native as nat
from simpeg_dc_torch_b200 import tuning


def _pattern(n=200):
    A = sp.diags([np.full(n - 1, -1.0), np.full(n, 4.0), np.full(n - 1, -1.0)],
                 [-1, 0, 1], format="csr")
    A.sort_indices()
    return A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data


def test_coordinate_descent_and_cache(monkeypatch):
    calls = []

    def fake_time(sym, t, nbatch, n_rhs, code, device, vals, rhs, refine, reps):
        calls.append(dict(t))
        # fastest at small_front_max 160, update_block 3, solve_target 1184;
        # small_tc 2 fails (inf) and must not be chosen
        if t["small_tc"] == 2:
            return float("inf"), t
        cost = (abs(t["small_front_max"] - 160) / 32 + abs(t["update_block"] - 3)
                + (0 if t["solve_target"] == 1184 else 1))
        return 10.0 + cost, t

    monkeypatch.setattr(tuning, "_time_plan", fake_time)
    tuning._CACHE.clear()
    crow, col, vals = _pattern()
    best, table = tuning.tune_schedule(crow, col, 200, 8, 1, "cpu", torch.float32,
                                       vals[None, :])
    assert best["small_front_max"] == 160
    assert best["update_block"] == 3
    assert best["solve_target"] == 1184
    assert best["small_tc"] == nat.default_tuning(nat.F32)["small_tc"]
    keys = [tuple(sorted(t.items())) for t, _ in table]
    assert len(keys) == len(set(keys)) == len(calls)
    assert min(ms for _, ms in table) == 10.0
    # cached: a second call times nothing
    n = len(calls)
    again = tuning.tune_schedule(crow, col, 200, 8, 1, "cpu", torch.float32, vals[None, :])
    assert len(calls) == n and again[0] == best
    tuning._CACHE.clear()
