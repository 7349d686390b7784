"""A batch of uneven 2.5-D surveys factored and solved in the same launches
(TorchDC2DBatch) against each survey evaluated alone by the CPU oracle with
its own wavenumber quadrature: data and misfit gradient, float64 within
1e-10 / 1e-9 and float32 + refinement within 1e-6 / 1e-5 relative; and the
autotuned schedule gives the untuned results."""
import numpy as np
import pytest
import torch

from oracle import dc_oracle as O
from simpeg_dc_torch_b200 import TorchDC2DBatch
from simpeg_dc_torch_b200 import synthetic as syn
from test_batch import alone_ops, small_batch

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def _reference(problems, models, bo):
    rng = np.random.default_rng(21)
    d, g, dobs, w = [], [], [], []
    for b, (mesh, survey) in enumerate(problems):
        ob = alone_ops(bo.ops[b], survey)
        ob["slab"] = O.grid_slabs(mesh.node_grid_index())
        db = O.dpred_2d(ob, models[b])
        do, wo = syn.observed(db, rng)
        _, gb = O.misfit_grad_2d(ob, models[b], do, wo)
        d.append(db), g.append(gb), dobs.append(do), w.append(wo)
    return [np.concatenate(x) for x in (d, g, dobs, w)]


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_batch_of_uneven_surveys_matches_each_alone(cuda, dtype):
    problems, models = small_batch(n=6, seed=8, scale=0.5)
    eng = TorchDC2DBatch(problems, nky=12, device=cuda, dtype=dtype)
    d_ref, g_ref, dobs, w = _reference(problems, models, eng._bo)
    m = torch.tensor(np.concatenate(models), device=cuda, requires_grad=True)
    phi = eng.misfit(m, torch.tensor(dobs, device=cuda), torch.tensor(w, device=cuda))
    phi.backward()
    with torch.no_grad():
        d = eng.dpred(m.detach()).cpu().numpy()
    eng.check()
    td, tg = (1e-10, 1e-9) if dtype == torch.float64 else (1e-6, 1e-5)
    assert rel(d, d_ref) < td
    assert rel(m.grad.cpu().numpy(), g_ref) < tg
    # each survey's part on its own, too
    for db, dr in zip(eng.split_data(d), eng.split_data(d_ref)):
        assert rel(db, dr) < td


def test_autotuned_schedule_gives_the_same_results(cuda):
    problems, models = small_batch(n=4, seed=9, scale=0.5)
    m = torch.tensor(np.concatenate(models), device=cuda)
    e0 = TorchDC2DBatch(problems, device=cuda, dtype=torch.float32)
    e1 = TorchDC2DBatch(problems, device=cuda, dtype=torch.float32, tune=True)
    assert e1.tuning is not None and len(e1.tuning_table) >= 3
    assert all(np.isfinite(ms) for _, ms in e1.tuning_table)
    with torch.no_grad():
        d0 = e0.dpred(m).cpu().numpy()
        d1 = e1.dpred(m).cpu().numpy()
    e0.check(), e1.check()
    assert rel(d1, d0) < 1e-6
