"""IP engines on the GPU against the reference's own: the linearized
TorchIP2D / TorchIP3D (golden fixture ip_tiny, made by running
dctorch/ip2d.py and ip3d.py on the tiny problems with every other receiver
of apparent-chargeability type: background data V_dc, the per-datum scale,
the IP data and the misfit gradient with respect to eta) and the joint
non-linear TorchDCIP2D (dcip_tiny, dctorch/dcip2d.py, both DC states).
float64 is held to 1e-10, float32 + refinement to 1e-6 (data) / 1e-5
(gradient), the levels of the DC engine tests."""
import numpy as np
import pytest
import torch

from conftest import golden
from simpeg_dc_torch_b200 import TorchDCIP2D, TorchIP2D, TorchIP3D
from simpeg_dc_torch_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a.detach().cpu() if torch.is_tensor(a) else a, float)
    b = np.asarray(b, float)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _mark(survey, flags):
    i = 0
    for src in survey.source_list:
        for rx in src.receiver_list:
            if flags[i]:
                rx.data_type = "apparent_chargeability"
            i += 1


def _make(tag, cuda, dtype, **kw):
    g = golden("ip_tiny")
    if tag == "2d":
        mesh, survey, _ = syn.tiny_2d()
        _mark(survey, g["2d_flags"])
        ip = TorchIP2D(mesh, survey, g["2d_m"], nky=7, device=cuda, dtype=dtype,
                       quadrature=(g["kys"], g["wq"]), **kw)
    else:
        mesh, survey, _ = syn.tiny_3d()
        _mark(survey, g["3d_flags"])
        ip = TorchIP3D(mesh, survey, g["3d_m"], device=cuda, dtype=dtype, **kw)
    return ip, g


@pytest.mark.parametrize("tag", ["2d", "3d"])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_ip_matches_reference(cuda, tag, dtype):
    ip, g = _make(tag, cuda, dtype)
    tol_d, tol_g = (1e-10, 1e-10) if dtype == torch.float64 else (1e-6, 1e-5)
    assert rel(ip.v_dc, g[f"{tag}_vdc"]) < tol_d
    assert rel(ip._scale, g[f"{tag}_scale"]) < tol_d
    eta = torch.tensor(g[f"{tag}_eta"], device=cuda, requires_grad=True)
    phi = ip.misfit(eta, torch.tensor(g[f"{tag}_dobs"], device=cuda),
                    torch.tensor(g[f"{tag}_w"], device=cuda))
    phi.backward()
    with torch.no_grad():
        d = ip.dpred(eta)
    assert rel(d, g[f"{tag}_d"]) < tol_d
    assert abs(float(phi) - g[f"{tag}_phi"]) <= tol_g * abs(g[f"{tag}_phi"])
    assert rel(eta.grad, g[f"{tag}_grad"]) < tol_g
    ip.check()


def test_ip_background_survives_a_refactorization(cuda):
    """A DC evaluation at another model on the wrapped engine replaces its
    factors; the next IP product restores the background's."""
    ip, g = _make("2d", cuda, torch.float64)
    with torch.no_grad():
        ip.dc.dpred(torch.tensor(g["2d_m"] + 0.3, device=cuda))
        d = ip.dpred(torch.tensor(g["2d_eta"], device=cuda))
    assert rel(d, g["2d_d"]) < 1e-10


def test_ip_active_cells(cuda):
    """eta on the active cells equals the full-mesh eta with zeros on the
    inactive cells, data and gradient (dctorch/ip2d.py:73-80)."""
    g = golden("ip_tiny")
    rng = np.random.default_rng(4)
    act = rng.uniform(size=g["2d_eta"].size) > 0.3
    full, _ = _make("2d", cuda, torch.float64)
    part, _ = _make("2d", cuda, torch.float64, active_cells=act)
    eta = g["2d_eta"].copy()
    eta[~act] = 0.0
    ef = torch.tensor(eta, device=cuda, requires_grad=True)
    ea = torch.tensor(eta[act], device=cuda, requires_grad=True)
    w = torch.tensor(g["2d_w"], device=cuda)
    dobs = torch.tensor(g["2d_dobs"], device=cuda)
    full.misfit(ef, dobs, w).backward()
    part.misfit(ea, dobs, w).backward()
    assert rel(part.dpred(ea.detach()), full.dpred(ef.detach()).cpu()) < 1e-12
    assert rel(ea.grad, ef.grad[torch.tensor(act, device=cuda)].cpu()) < 1e-12


@pytest.mark.parametrize("state", ["total", "instantaneous"])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_dcip_matches_reference(cuda, state, dtype):
    J = golden("dcip_tiny")
    mesh, survey, _ = syn.tiny_2d()
    eng = TorchDCIP2D(mesh, survey, nky=7, device=cuda, dtype=dtype, eta_max=0.8,
                      ip_scale=1000.0, dc_state=state, quadrature=(J["kys"], J["wq"]))
    tol_d, tol_g = (1e-10, 1e-9) if dtype == torch.float64 else (1e-6, 1e-5)
    t = lambda k: torch.tensor(J[f"{state}_{k}"], device=cuda)  # noqa: E731
    mm = torch.tensor(J[f"{state}_m"], device=cuda, requires_grad=True)
    phi = eng.misfit(mm, t("dobs_dc"), t("w_dc"), t("dobs_ip"), t("w_ip"), lam=0.7)
    phi.backward()
    with torch.no_grad():
        d_dc, d_ip = eng.dpred(mm)
    assert rel(d_dc, J[f"{state}_d_dc"]) < tol_d
    assert rel(d_ip, J[f"{state}_d_ip"]) < tol_d
    assert abs(float(phi) - J[f"{state}_phi"]) <= tol_g * abs(J[f"{state}_phi"])
    assert rel(mm.grad, J[f"{state}_grad"]) < tol_g
    eng.check()


def test_dcip_active_cells(cuda):
    """On the active cells, with log-rho val_inactive and eta = 0 elsewhere,
    the joint data equal those of the full-mesh engine."""
    J = golden("dcip_tiny")
    mesh, survey, _ = syn.tiny_2d()
    n = J["m_rho"].size
    act = np.random.default_rng(6).uniform(size=n) > 0.3
    kw = dict(nky=7, device=cuda, eta_max=0.8, ip_scale=1000.0,
              quadrature=(J["kys"], J["wq"]))
    full = TorchDCIP2D(mesh, survey, **kw)
    part = TorchDCIP2D(mesh, survey, active_cells=act, val_inactive=4.0, **kw)
    m_rho = J["m_rho"].copy()
    m_rho[~act] = 4.0
    eta = np.where(act, 0.1, 0.0)
    df = full.dpred_from_fields(torch.tensor(m_rho, device=cuda), torch.tensor(eta, device=cuda))
    dp = part.dpred_from_fields(torch.tensor(m_rho[act], device=cuda),
                                torch.tensor(eta[act], device=cuda))
    assert rel(dp[0], df[0].cpu()) < 1e-12
    assert rel(dp[1], df[1].cpu()) < 1e-12

