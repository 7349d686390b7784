"""The 3-D engine on an octree (the refined 3-D workload's mesh type, at a small
size): float64 and float32 + refinement against the oracle (SuperLU on the
tree operators), the float64 adjoint gradient against central finite
differences on 20 random directions (that workload's check), and ten L-BFGS
iterations of the float32 engine (its optimizer contract)."""
import numpy as np
import pytest
import torch

from oracle import dc_oracle as O
from simpeg_dc_torch_b200 import TorchDC2D, TorchDC3D, TreeMesh
from simpeg_dc_torch_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

TOL = {torch.float64: (1e-10, 1e-9), torch.float32: (1e-6, 1e-5)}


def rel(a, b):
    a = np.asarray(a.detach().cpu() if torch.is_tensor(a) else a, float)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _case(cuda, dtype):
    mesh, survey, m = syn.tree_small(seed=0)
    assert mesh.n_hanging_nodes > 0
    eng = TorchDC3D(mesh, survey, device=cuda, dtype=dtype)
    o = eng._ops
    op = dict(L3=eng._L, crow=o.crow, col=o.col, nN=o.nN, Q=o.q.toarray(), Pd=o.Pd,
              sidx=o.sidx)
    return eng, op, m


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_tree_engine_against_oracle(cuda, dtype):
    eng, op, m = _case(cuda, dtype)
    d_ref = O.dpred_3d(op, m)
    dobs, w = syn.observed(d_ref, np.random.default_rng(3))
    phi_ref, g_ref = O.misfit_grad_3d(op, m, dobs, w)
    v = np.random.default_rng(4).standard_normal(d_ref.size)
    jt_ref = O.jtvec_3d(op, m, v)
    x = torch.tensor(m, device=cuda, requires_grad=True)
    phi = eng.misfit(x, torch.tensor(dobs, device=cuda), torch.tensor(w, device=cuda))
    phi.backward()
    with torch.no_grad():
        d = eng.dpred(torch.tensor(m, device=cuda))
    jt = eng.Jtvec(torch.tensor(m, device=cuda), torch.tensor(v, device=cuda))
    eng.check()
    td, tg = TOL[dtype]
    assert rel(d, d_ref) < td
    assert abs(float(phi.detach()) - phi_ref) <= 10 * td * phi_ref
    assert rel(x.grad, g_ref) < tg
    assert rel(jt, jt_ref) < tg


def test_tree_gradient_finite_differences(cuda):
    eng, op, m = _case(cuda, torch.float64)
    d0 = O.dpred_3d(op, m)
    dobs, w = syn.observed(d0 * 1.1, np.random.default_rng(5))
    dobs_t, w_t = torch.tensor(dobs, device=cuda), torch.tensor(w, device=cuda)
    x = torch.tensor(m, device=cuda, requires_grad=True)
    eng.misfit(x, dobs_t, w_t).backward()
    g = x.grad.cpu().numpy()
    rng = np.random.default_rng(6)
    eps = 1e-4
    worst = 0.0
    with torch.no_grad():
        for _ in range(20):
            u = rng.standard_normal(m.size)
            u /= np.linalg.norm(u)
            fp = float(eng.misfit(torch.tensor(m + eps * u, device=cuda), dobs_t, w_t))
            fm = float(eng.misfit(torch.tensor(m - eps * u, device=cuda), dobs_t, w_t))
            fd = (fp - fm) / (2 * eps)
            worst = max(worst, abs(fd - g @ u) / (abs(g @ u) + 1e-12 * np.abs(g).sum()))
    eng.check()
    assert worst < 1e-5, worst


def test_tree_lbfgs_ten_iterations(cuda):
    eng, op, m = _case(cuda, torch.float32)
    m_true = m
    d_true = O.dpred_3d(op, m_true)
    dobs, w = syn.observed(d_true, np.random.default_rng(7), rel_noise=0.01)
    dobs_t, w_t = torch.tensor(dobs, device=cuda), torch.tensor(w, device=cuda)
    x = torch.full((m.size,), float(np.log(100.0)), dtype=torch.float64, device=cuda,
                   requires_grad=True)
    opt = torch.optim.LBFGS([x], lr=1.0, max_iter=10, history_size=10,
                            line_search_fn="strong_wolfe")
    values = []

    def closure():
        opt.zero_grad()
        phi = eng.misfit(x, dobs_t, w_t)
        phi.backward()
        values.append(float(phi.detach()))
        return phi

    opt.step(closure)
    eng.check()
    assert len(values) >= 3
    assert min(values) < 0.5 * values[0]


def test_quadtree_2p5d_engine_against_oracle(cuda):
    """The 2.5-D engine on a quadtree refined along the electrode line
    (hanging nodes in every wavenumber system), float64 and float32 +
    refinement against the oracle."""
    tm = TreeMesh([(1.0, 128)] * 2, origin=[-64.0, -128.0])
    tm.refine(lambda lo, hi: np.full(lo.shape[0], 3))
    xe = np.linspace(-20.0, 20.0, 11)
    el = np.c_[xe, np.zeros_like(xe)]
    for level, pad in ((7, 4.0), (6, 12.0), (5, 30.0)):
        tm.refine_points(el, level, padding=pad)
    tm.finalize()
    assert tm.n_hanging_nodes > 0
    mesh_survey = syn.dipole_dipole_2d(xe, 4, a=1)
    from simpeg_dc_torch_b200.survey import Survey
    survey = Survey(mesh_survey)
    rng = np.random.default_rng(8)
    m = np.log(100.0) + 0.3 * rng.standard_normal(tm.nC)
    for dtype in (torch.float64, torch.float32):
        eng = TorchDC2D(tm, survey, nky=8, device=cuda, dtype=dtype)
        o = eng._ops
        op = dict(Lstack=eng._L, crow=o.crow, col=o.col, nN=o.nN, Q=o.q.toarray(), Pd=o.Pd,
                  sidx=o.sidx, wq=eng.wq_np)
        d_ref = O.dpred_2d(op, m)
        dobs, w = syn.observed(d_ref, np.random.default_rng(9))
        phi_ref, g_ref = O.misfit_grad_2d(op, m, dobs, w)
        x = torch.tensor(m, device=cuda, requires_grad=True)
        phi = eng.misfit(x, torch.tensor(dobs, device=cuda), torch.tensor(w, device=cuda))
        phi.backward()
        with torch.no_grad():
            d = eng.dpred(torch.tensor(m, device=cuda))
        eng.check()
        td, tg = TOL[dtype]
        assert rel(d, d_ref) < td
        assert rel(x.grad, g_ref) < tg
