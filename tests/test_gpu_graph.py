"""An engine's eval + gradient replayed from one CUDA graph
(GraphedMisfitGrad) against the same evaluation launched eagerly: float64
2.5-D with active cells and float32 + refinement 3-D, new models replayed
through the captured graph, and an autograd backward that outlives a replay
(the replay advances the solver's stamp, so the backward refactorizes)."""
import numpy as np
import pytest
import torch

from simpeg_dc_torch_b200 import GraphedMisfitGrad, TorchDC2D, TorchDC3D
from simpeg_dc_torch_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


def _data(eng, m, cuda, seed):
    with torch.no_grad():
        d = eng.dpred(m)
    dobs_np, w_np = syn.observed(d.cpu().numpy(), np.random.default_rng(seed))
    return torch.tensor(dobs_np, device=cuda), torch.tensor(w_np, device=cuda)


def test_graph_2d_fp64_active_cells(cuda):
    mesh, survey, m_np = syn.suite_case("2d-tensor")
    act = np.random.default_rng(3).uniform(size=mesh.nC) > 0.2
    eng = TorchDC2D(mesh, survey, nky=8, device=cuda, active_cells=act,
                    val_inactive=float(np.log(100.0)))
    m = torch.tensor(m_np[act], device=cuda)
    dobs, w = _data(eng, m, cuda, 1)
    gm = GraphedMisfitGrad(eng, m, dobs, w)
    rng = np.random.default_rng(4)
    for _ in range(3):
        mm = m + 0.1 * torch.tensor(rng.standard_normal(m.numel()), device=cuda)
        phi_g, g_g = gm(mm)
        phi_e, g_e = eng.misfit_and_grad(mm, dobs, w)
        assert abs(phi_g - phi_e) <= 1e-12 * abs(phi_e)
        assert rel(g_g, g_e) < 1e-12
    eng.check()


def test_graph_3d_fp32_refined(cuda):
    mesh, survey, m_np = syn.suite_case("3d-tensor")
    eng = TorchDC3D(mesh, survey, device=cuda, dtype=torch.float32)
    m = torch.tensor(m_np, device=cuda)
    dobs, w = _data(eng, m, cuda, 2)
    gm = GraphedMisfitGrad(eng, m, dobs, w)
    rng = np.random.default_rng(5)
    for _ in range(3):
        mm = m + 0.1 * torch.tensor(rng.standard_normal(m.numel()), device=cuda)
        phi_g, g_g = gm(mm)
        phi_e, g_e = eng.misfit_and_grad(mm, dobs, w)
        assert abs(phi_g - phi_e) <= 1e-10 * abs(phi_e)
        assert rel(g_g, g_e) < 1e-8
    eng.check()


def test_backward_after_a_replay_refactorizes(cuda):
    """dpred at m (eager, factors at m kept for the backward), then a graph
    replay at another model, then the backward: the gradient is that at m."""
    mesh, survey, m_np = syn.suite_case("2d-tensor")
    eng = TorchDC2D(mesh, survey, nky=8, device=cuda)
    m = torch.tensor(m_np, device=cuda)
    dobs, w = _data(eng, m, cuda, 6)
    _, g_ref = eng.misfit_and_grad(m, dobs, w)
    gm = GraphedMisfitGrad(eng, m, dobs, w)
    x = m.clone().requires_grad_(True)
    phi = eng.misfit(x, dobs, w)
    gm(m + 0.3)
    phi.backward()
    assert rel(x.grad, g_ref) < 1e-12
    eng.check()
