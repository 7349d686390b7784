"""The side engines at the large 2.5-D configuration (56,525 nodes, 10
wavenumbers, 186 sources) against the CPU oracle: the linearized IP engine
(dctorch/ip2d.py: data J(m_dc) eta and the misfit gradient in eta, with every
other receiver of apparent-chargeability type), its 3-D counterpart
(dctorch/ip3d.py) on a 75,843-node grid with 200 sources, and the joint
non-linear DC + IP engine (dctorch/dcip2d.py: both data kinds and the
gradient in (log-rho, logit-eta)).  The oracle solves exactly with the block-tridiagonal
slab Cholesky.  float64 is held to 1e-10 (data) / 1e-9 (gradients);
float32 + refinement to 1e-6 / 1e-5, the levels of the DC scale tests."""
import numpy as np
import pytest
import torch

from oracle import dc_oracle as O
from simpeg_dc_torch_b200 import TorchDCIP2D, TorchIP2D, TorchIP3D
from simpeg_dc_torch_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

TOL = {torch.float64: (1e-10, 1e-9), torch.float32: (1e-6, 1e-5)}


def rel(a, b):
    a = np.asarray(a.detach().cpu() if torch.is_tensor(a) else a, float)
    b = np.asarray(b, float)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _op(dc, mesh):
    ops = dc._ops
    return dict(Lstack=dc._L, crow=ops.crow, col=ops.col, nN=ops.nN, Q=ops.q.toarray(),
                Pd=ops.Pd, sidx=ops.sidx, wq=dc.wq_np,
                slab=O.grid_slabs(mesh.node_grid_index()))


def _mark_every_other(survey):
    flags = []
    i = 0
    for src in survey.source_list:
        for rx in src.receiver_list:
            if i % 2 == 1:
                rx.data_type = "apparent_chargeability"
            flags.append(i % 2 == 1)
            i += 1
    return flags


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_ip2d_large_against_oracle(cuda, dtype):
    mesh, survey, m = syn.dc2d_large(seed=0)
    flags = _mark_every_other(survey)
    ip = TorchIP2D(mesh, survey, m, nky=12, device=cuda, dtype=dtype)
    op = _op(ip.dc, mesh)
    nd = ip.dc.nD
    # receivers carry one datum each here: the per-receiver flags are the
    # per-datum flags
    charge = np.repeat(flags, [rx.nD for s in survey.source_list
                               for rx in s.receiver_list])
    assert charge.size == nd
    eta = np.random.default_rng(9).uniform(0.0, 0.2, ip.dc.nC)
    fields = O.dpred_2d(op, m, return_fields=True)
    scale = O.ip_scale(fields[0], charge)
    d_ref = scale * O.jvec_2d(op, m, eta, fields)
    dobs = d_ref * 1.05
    w = 1.0 / (np.abs(dobs) + 1e-3 * np.abs(dobs).max())
    g_ref = O._adjoint_2d(op, m, scale * 2.0 * w * w * (d_ref - dobs), fields)[1]
    td, tg = TOL[dtype]
    et = torch.tensor(eta, device=cuda, requires_grad=True)
    phi = ip.misfit(et, torch.tensor(dobs, device=cuda), torch.tensor(w, device=cuda))
    phi.backward()
    with torch.no_grad():
        d = ip.dpred(et)
    ip.check()
    assert rel(d, d_ref) < td
    assert rel(et.grad, g_ref) < tg


def test_dcip2d_large_against_oracle(cuda):
    mesh, survey, m = syn.dc2d_large(seed=0)
    eng = TorchDCIP2D(mesh, survey, nky=12, device=cuda, eta_max=0.8, ip_scale=1000.0)
    op = _op(eng.dc, mesh)
    eta = np.random.default_rng(10).uniform(0.02, 0.3, eng.dc.nC)
    mm = np.concatenate([m, eng.m_eta_of(eta)])
    d_dc, d_ip, _, _ = O.dcip_dpred_2d(op, m, eta, 1000.0, "total")
    dobs_dc = d_dc * 1.03
    w_dc = 1.0 / np.abs(dobs_dc)
    dobs_ip = d_ip + 2.0
    w_ip = np.full(d_ip.size, 0.5)
    phi_ref, g_ref = O.dcip_misfit_grad_2d(op, mm, 0.8, 1000.0, "total", dobs_dc, w_dc,
                                           dobs_ip, w_ip, 0.7)
    x = torch.tensor(mm, device=cuda, requires_grad=True)
    t = lambda a: torch.tensor(a, device=cuda)  # noqa: E731
    phi = eng.misfit(x, t(dobs_dc), t(w_dc), t(dobs_ip), t(w_ip), lam=0.7)
    phi.backward()
    with torch.no_grad():
        a, b = eng.dpred(x)
    eng.check()
    assert rel(a, d_dc) < 1e-10 and rel(b, d_ip) < 1e-10
    assert abs(float(phi.detach()) - phi_ref) <= 1e-9 * phi_ref
    assert rel(x.grad, g_ref) < 1e-9


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_ip3d_mid_against_oracle(cuda, dtype):
    mesh, survey, m = syn.dc3d(seed=0, ncore=(40, 40, 20), dx=8.0, npad=6)
    flags = _mark_every_other(survey)
    ip = TorchIP3D(mesh, survey, m, device=cuda, dtype=dtype)
    ops = ip.dc._ops
    op = dict(L3=ip.dc._L, crow=ops.crow, col=ops.col, nN=ops.nN, Q=ops.q.toarray(),
              Pd=ops.Pd, sidx=ops.sidx, slab=O.grid_slabs(mesh.node_grid_index()))
    charge = np.repeat(flags, [rx.nD for s in survey.source_list for rx in s.receiver_list])
    eta = np.random.default_rng(11).uniform(0.0, 0.2, ip.dc.nC)
    v_dc = O.dpred_3d(op, m)
    scale = O.ip_scale(v_dc, charge)
    d_ref = scale * O.jvec_3d(op, m, eta)
    dobs = d_ref * 1.05
    w = 1.0 / (np.abs(dobs) + 1e-3 * np.abs(dobs).max())
    g_ref = O.jtvec_3d(op, m, scale * 2.0 * w * w * (d_ref - dobs))
    et = torch.tensor(eta, device=cuda, requires_grad=True)
    phi = ip.misfit(et, torch.tensor(dobs, device=cuda), torch.tensor(w, device=cuda))
    phi.backward()
    with torch.no_grad():
        d = ip.dpred(et)
    ip.check()
    td, tg = TOL[dtype]
    assert rel(d, d_ref) < td
    assert rel(et.grad, g_ref) < tg
