"""Parity at the benchmarked scales: the GPU engines against the CPU oracle on
the full 2.5-D configuration with 12 wavenumbers (56,525 nodes, 186 sources)
and on a 3-D grid of 75,843 nodes whose top fronts span several blocks of
the blocked float32 update and whose substitution launches split their K
ranges (the schedule features the 269,001-node benchmark exercises at more
depth).

The oracle solves exactly in float64 with the block-tridiagonal slab
Cholesky (`SlabCholeskyBatch`; SuperLU needs minutes per factorization at
these sizes); `tests/test_oracle.py` pins that solver against SuperLU and the
reference's golden vectors.

Tolerances: float64 < 1e-10 (data) and 1e-9 (gradients) relative, the
reference's parity level (dctorch/tests/test_suite.py:127-132); float32 +
refinement: data <= 1e-6 and gradients <= 1e-5 relative
(dctorch/tests/test_jtvec.py:37-64 asks 1e-5 of the gradients)."""
import numpy as np
import pytest
import torch

from oracle import dc_oracle as O
from simpeg_dc_torch_b200 import TorchDC2D, TorchDC3D
from simpeg_dc_torch_b200 import synthetic as syn
from simpeg_dc_torch_b200._native import F32

pytestmark = pytest.mark.gpu

TOL = {torch.float64: (1e-10, 1e-9), torch.float32: (1e-6, 1e-5)}


def rel(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _gpu_eval(eng, m, dobs, w, v, dev):
    mt = torch.tensor(m, device=dev, requires_grad=True)
    phi = eng.misfit(mt, torch.tensor(dobs, device=dev), torch.tensor(w, device=dev))
    phi.backward()
    with torch.no_grad():
        d = eng.dpred(torch.tensor(m, device=dev)).cpu().numpy()
    jt = eng.Jtvec(torch.tensor(m, device=dev), torch.tensor(v, device=dev)).cpu().numpy()
    eng.check()
    return d, float(phi), mt.grad.cpu().numpy(), jt


def _check(eng, dtype, m, dobs, w, v, ref, dev):
    d, phi, g, jt = _gpu_eval(eng, m, dobs, w, v, dev)
    td, tg = TOL[dtype]
    errs = {"dpred": rel(d, ref["d"]), "grad": rel(g, ref["g"]),
            "jtvec": rel(jt, ref["jt"]), "phi": abs(phi - ref["phi"]) / ref["phi"]}
    assert errs["dpred"] < td, errs
    assert errs["phi"] < 10 * td, errs
    assert errs["grad"] < tg, errs
    assert errs["jtvec"] < tg, errs
    return errs


def test_dc2d_large_workload_against_oracle(cuda):
    """The 2.5-D benchmark's large configuration at full size (400x120 core
    cells + padding, 96 electrodes, dipole-dipole + Wenner, nky 12)."""
    mesh, survey, m = syn.dc2d_large(seed=0)
    e64 = TorchDC2D(mesh, survey, nky=12, device=cuda)
    ops = e64._ops
    op = dict(Lstack=e64._L, crow=ops.crow, col=ops.col, nN=ops.nN,
              Q=ops.q.toarray(), Pd=ops.Pd, sidx=ops.sidx, wq=e64.wq_np,
              slab=O.grid_slabs(mesh.node_grid_index()))
    # 12 wavenumbers asked; the fit drops points it gives zero weight
    assert ops.nN > 50000 and e64.nky >= 10
    fields = O.dpred_2d(op, m, return_fields=True)
    dobs, w = syn.observed(fields[0], np.random.default_rng(7))
    r = w * (fields[0] - dobs)
    _, g_ref = O._adjoint_2d(op, m, 2.0 * w * r, fields)
    v = np.random.default_rng(8).standard_normal(e64.nD)
    _, jt_ref = O._adjoint_2d(op, m, v, fields)
    ref = dict(d=fields[0], g=g_ref, jt=jt_ref, phi=float((r ** 2).sum()))
    for dtype in (torch.float64, torch.float32):
        eng = e64 if dtype == torch.float64 else TorchDC2D(
            mesh, survey, nky=12, device=cuda, dtype=dtype)
        _check(eng, dtype, m, dobs, w, v, ref, cuda)
        del eng
    torch.cuda.empty_cache()


def _schedule_depth(eng):
    """(widest supernode in panels, largest K-split piece count of one output
    tile, most tasks of one substitution launch) of the float32 plan."""
    sym = eng.solver._sym
    sn = sym.array("sn_first")
    widest = int(np.max(np.diff(sn)))
    most_split, most_tasks = 0, 0
    for which in (1, 2):
        tasks, launches = sym.schedule(F32, which)
        for kind, lv, first, count, arg in launches:
            t = tasks[first:first + count]
            most_tasks = max(most_tasks, int(count))
            if count:
                _, cnt = np.unique(t[:, [0, 2]], axis=0, return_counts=True)
                most_split = max(most_split, int(cnt.max()))
    return widest, most_split, most_tasks


def test_dc3d_multiblock_case_against_oracle(cuda):
    """A 3-D grid (40x40x20 core cells of 8 m + 6 padding cells per face,
    75,843 nodes, 200 pole-dipole sources, 6,000 data) whose float32 plan
    has supernodes several update blocks wide and K-split substitution
    launches of hundreds of tasks, against the oracle."""
    mesh, survey, m = syn.dc3d(seed=0, ncore=(40, 40, 20), dx=8.0, npad=6)
    e32 = TorchDC3D(mesh, survey, device=cuda, dtype=torch.float32)
    widest, most_split, most_tasks = _schedule_depth(e32)
    # several blocks of four 64-column panels, split K ranges, big launches
    assert widest > 2 * 4 * 64, widest
    assert most_split >= 2, most_split
    assert most_tasks >= 592, most_tasks
    ops = e32._ops
    op = dict(L3=e32._L, crow=ops.crow, col=ops.col, nN=ops.nN,
              Q=ops.q.toarray(), Pd=ops.Pd, sidx=ops.sidx,
              slab=O.grid_slabs(mesh.node_grid_index()))
    fields = O.dpred_3d(op, m, return_fields=True)
    dobs, w = syn.observed(fields[0], np.random.default_rng(9))
    r = w * (fields[0] - dobs)
    _, g_ref = O._adjoint_3d(op, m, 2.0 * w * r, fields)
    v = np.random.default_rng(10).standard_normal(e32.nD)
    _, jt_ref = O._adjoint_3d(op, m, v, fields)
    ref = dict(d=fields[0], g=g_ref, jt=jt_ref, phi=float((r ** 2).sum()))
    _check(e32, torch.float32, m, dobs, w, v, ref, cuda)
    del e32
    torch.cuda.empty_cache()
    e64 = TorchDC3D(mesh, survey, device=cuda, dtype=torch.float64)
    _check(e64, torch.float64, m, dobs, w, v, ref, cuda)
