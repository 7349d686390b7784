"""The block-diagonal operators of a batch of uneven 2.5-D surveys (host):
each survey's data and misfit gradient through the batch's scaled,
side-by-side systems equal the survey's own, evaluated alone with its own
wavenumber quadrature (the CPU oracle on both)."""
import numpy as np
import scipy.sparse as sp

from oracle import dc_oracle as O
from simpeg_dc_torch_b200 import synthetic as syn
from simpeg_dc_torch_b200.batch import _equalise, batch_operators
from simpeg_dc_torch_b200.quadrature import electrode_distance_range, k0_quadrature


def small_batch(n=3, seed=5, scale=0.25):
    probs = syn.dc2d_batch(n_problems=n, seed=seed, scale=scale)
    return [(mesh, survey) for mesh, survey, _ in probs], [m for *_, m in probs]


def alone_ops(o, survey, nky=12):
    """One survey's oracle operators with its own quadrature."""
    kys, wq, _ = k0_quadrature(*electrode_distance_range(survey), nky)
    return dict(Lstack=sp.vstack([o.L_ky(k) for k in kys]).tocsr(), crow=o.crow,
                col=o.col, nN=o.nN, Q=o.q.toarray(), Pd=o.Pd, sidx=o.sidx, wq=wq)


def batch_oracle_ops(bo):
    return dict(Lstack=bo.L, crow=bo.crow, col=bo.col, nN=int(bo.node_off[-1]),
                Q=bo.Q.toarray(), Pd=bo.Pd, sidx=bo.sidx, wq=np.ones(bo.nky))


def test_weight_splitting_keeps_the_quadrature_sum():
    k, w = _equalise([0.1, 0.5, 2.0], [0.2, 0.7, 0.1], 5)
    assert k.size == w.size == 5
    assert np.isclose(w.sum(), 1.0)
    assert np.isclose((w * np.cos(k)).sum(),
                      0.2 * np.cos(0.1) + 0.7 * np.cos(0.5) + 0.1 * np.cos(2.0))


def test_batch_matches_each_survey_alone():
    problems, models = small_batch()
    bo = batch_operators(problems, nky=12)
    assert len({o.nN for o in bo.ops}) == len(problems)        # uneven sizes
    op = batch_oracle_ops(bo)
    m = np.concatenate(models)
    rng = np.random.default_rng(2)
    alone, dobs, w = [], [], []
    d_all = O.dpred_2d(op, m)
    for b, (mesh, survey) in enumerate(problems):
        ob = alone_ops(bo.ops[b], survey)
        alone.append(ob)
        db = O.dpred_2d(ob, models[b])
        assert O.rel(d_all[bo.data_off[b]:bo.data_off[b + 1]], db) < 1e-11
        do, wo = syn.observed(db, rng)
        dobs.append(do)
        w.append(wo)
    _, g_all = O.misfit_grad_2d(op, m, np.concatenate(dobs), np.concatenate(w))
    for b in range(len(problems)):
        _, gb = O.misfit_grad_2d(alone[b], models[b], dobs[b], w[b])
        assert O.rel(g_all[bo.cell_off[b]:bo.cell_off[b + 1]], gb) < 1e-10
