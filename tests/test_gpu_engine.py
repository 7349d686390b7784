"""Engine-level parity on the GPU: TorchDC2D / TorchDC3D (fused CUDA path)
against the reference's own dpred / misfit gradient / Jtvec (golden fixtures)
and against the CPU oracle on the larger workloads.

Tolerances: float64 path < 1e-10 relative (the reference's parity specs are
1e-9..1e-12, dctorch/tests/test_suite.py:132, test_jtvec.py:64); float32 +
refinement: dpred <= 1e-6 and gradient <= 1e-5 relative."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

from conftest import golden
from oracle import dc_oracle as O
from simpeg_dc_torch_b200 import TorchDC2D, TorchDC3D
from simpeg_dc_torch_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _run(eng, m, dobs, w, v, dev):
    mt = torch.tensor(m, device=dev, requires_grad=True)
    phi = eng.misfit(mt, torch.tensor(dobs, device=dev),
                     torch.tensor(w, device=dev))
    phi.backward()
    with torch.no_grad():
        d = eng.dpred(torch.tensor(m, device=dev)).cpu().numpy()
    jt = eng.Jtvec(torch.tensor(m, device=dev),
                   torch.tensor(v, device=dev)).cpu().numpy()
    return d, float(phi), mt.grad.cpu().numpy(), jt


@pytest.mark.parametrize("name,case", [("dc2d_tiny", syn.tiny_2d),
                                       ("dc2d_suite",
                                        lambda: syn.suite_case("2d-tensor"))])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_dc2d_matches_reference(cuda, name, case, dtype):
    g = golden(name)
    mesh, survey, m = case()
    eng = TorchDC2D(mesh, survey, device=cuda, dtype=dtype,
                    quadrature=(g["kys"], g["wq"]))
    d, phi, grad, jt = _run(eng, g["m"], g["dobs"], g["w"], g["v"], cuda)
    tol_d, tol_g = (1e-10, 1e-9) if dtype == torch.float64 else (1e-6, 1e-5)
    assert rel(d, g["dpred"]) < tol_d
    assert abs(phi - g["phi"]) <= 10 * tol_d * abs(g["phi"])
    assert rel(grad, g["grad"]) < tol_g
    assert rel(jt, g["jtvec"]) < tol_g
    f, g2 = eng.misfit_and_grad(torch.tensor(g["m"], device=cuda),
                                torch.tensor(g["dobs"], device=cuda),
                                torch.tensor(g["w"], device=cuda))
    assert rel(g2.cpu().numpy(), g["mag_grad"]) < tol_g
    eng.check()


@pytest.mark.parametrize("name,case", [("dc3d_tiny", syn.tiny_3d),
                                       ("dc3d_suite",
                                        lambda: syn.suite_case("3d-tensor"))])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_dc3d_matches_reference(cuda, name, case, dtype):
    g = golden(name)
    mesh, survey, m = case()
    eng = TorchDC3D(mesh, survey, device=cuda, dtype=dtype)
    d, phi, grad, jt = _run(eng, g["m"], g["dobs"], g["w"], g["v"], cuda)
    tol_d, tol_g = (1e-10, 1e-9) if dtype == torch.float64 else (1e-6, 1e-5)
    assert rel(d, g["dpred"]) < tol_d
    assert rel(grad, g["grad"]) < tol_g
    assert rel(jt, g["jtvec"]) < tol_g
    eng.check()


def _oracle_ops_2d(eng):
    ops = eng._ops
    return dict(Lstack=eng._L, crow=ops.crow, col=ops.col, nN=ops.nN,
                Q=ops.q.toarray(), Pd=ops.Pd, sidx=ops.sidx, wq=eng.wq_np)


def test_dc2d_small_workload_against_oracle(cuda):
    """The 2.5-D benchmark's small configuration (100x50 core cells + padding,
    21 electrodes, nky 11): GPU float64 and float32+refinement vs the oracle."""
    mesh, survey, m = syn.dc2d_small()
    e64 = TorchDC2D(mesh, survey, nky=11, device=cuda)
    op = _oracle_ops_2d(e64)
    d_ref = O.dpred_2d(op, m)
    rng = np.random.default_rng(4)
    dobs, w = syn.observed(d_ref, rng)
    phi_ref, g_ref = O.misfit_grad_2d(op, m, dobs, w)
    for dtype, td, tg in [(torch.float64, 1e-10, 1e-9),
                          (torch.float32, 1e-6, 1e-5)]:
        eng = e64 if dtype == torch.float64 else TorchDC2D(
            mesh, survey, nky=11, device=cuda, dtype=dtype)
        phi, g = eng.misfit_and_grad(torch.tensor(m, device=cuda),
                                     torch.tensor(dobs, device=cuda),
                                     torch.tensor(w, device=cuda))
        with torch.no_grad():
            d = eng.dpred(torch.tensor(m, device=cuda)).cpu().numpy()
        assert rel(d, d_ref) < td
        assert rel(g.cpu().numpy(), g_ref) < tg
        assert abs(phi - phi_ref) <= 10 * td * phi_ref


def test_gradient_matches_central_differences(cuda):
    mesh, survey, m = syn.tiny_2d()
    eng = TorchDC2D(mesh, survey, nky=7, device=cuda)
    rng = np.random.default_rng(3)
    with torch.no_grad():
        d = eng.dpred(torch.tensor(m, device=cuda)).cpu().numpy()
    dobs, w = syn.observed(d, rng)
    dobs_t, w_t = torch.tensor(dobs, device=cuda), torch.tensor(w, device=cuda)
    mt = torch.tensor(m, device=cuda, requires_grad=True)
    eng.misfit(mt, dobs_t, w_t).backward()
    for _ in range(3):
        u = rng.standard_normal(m.size)
        u /= np.linalg.norm(u)
        h = 1e-4
        with torch.no_grad():
            fp = float(eng.misfit(torch.tensor(m + h * u, device=cuda), dobs_t, w_t))
            fm = float(eng.misfit(torch.tensor(m - h * u, device=cuda), dobs_t, w_t))
        fd = (fp - fm) / (2 * h)
        an = float(mt.grad.cpu().numpy() @ u)
        assert abs(fd - an) <= 1e-6 * abs(fd)


def test_active_cells_restrict_the_gradient(cuda):
    mesh, survey, m = syn.tiny_2d()
    act = mesh.cell_centers[:, 1] < -1.0
    val = float(np.log(100.0))
    m_full = m.copy()
    m_full[~act] = val
    ef = TorchDC2D(mesh, survey, nky=7, device=cuda)
    ea = TorchDC2D(mesh, survey, nky=7, device=cuda, active_cells=act,
                   val_inactive=val)
    v = torch.tensor(np.random.default_rng(0).standard_normal(ef.nD), device=cuda)
    jf = ef.Jtvec(torch.tensor(m_full, device=cuda), v).cpu().numpy()
    ja = ea.Jtvec(torch.tensor(m_full[act], device=cuda), v).cpu().numpy()
    assert ja.shape == (int(act.sum()),)
    assert rel(ja, jf[act]) < 1e-12
    # against the oracle: the model on the active cells injected into the
    # full mesh with the inactive value, the gradient restricted back
    # (dctorch/simulation2d.py:122-134, 299-304)
    op = _oracle_ops_2d(ea)
    d_ref = O.dpred_2d(op, m_full)
    dobs, w = syn.observed(d_ref, np.random.default_rng(6))
    _, g_ref = O.misfit_grad_2d(op, m_full, dobs, w)
    for dtype, td, tg in [(torch.float64, 1e-10, 1e-9), (torch.float32, 1e-6, 1e-5)]:
        eng = ea if dtype == torch.float64 else TorchDC2D(
            mesh, survey, nky=7, device=cuda, dtype=dtype, active_cells=act,
            val_inactive=val)
        ma = torch.tensor(m_full[act], device=cuda, requires_grad=True)
        eng.misfit(ma, torch.tensor(dobs, device=cuda),
                   torch.tensor(w, device=cuda)).backward()
        with torch.no_grad():
            d = eng.dpred(torch.tensor(m_full[act], device=cuda)).cpu().numpy()
        assert rel(d, d_ref) < td
        assert rel(ma.grad.cpu().numpy(), g_ref[act]) < tg


def test_adjoint_survives_a_clobbered_factorization(cuda):
    """A second forward between dpred and backward replaces the factors; the
    backward must refactorize at its own model (solver stamp)."""
    g = golden("dc2d_tiny")
    mesh, survey, _ = syn.tiny_2d()
    eng = TorchDC2D(mesh, survey, device=cuda, quadrature=(g["kys"], g["wq"]))
    mt = torch.tensor(g["m"], device=cuda, requires_grad=True)
    phi = eng.misfit(mt, torch.tensor(g["dobs"], device=cuda),
                     torch.tensor(g["w"], device=cuda))
    with torch.no_grad():
        eng.dpred(torch.tensor(g["m"] + 0.3, device=cuda))
    phi.backward()
    assert rel(mt.grad.cpu().numpy(), g["grad"]) < 1e-9


@pytest.mark.parametrize("tag,rho_p", [("model", None), ("fixed", 50.0)])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_dc2d_singularity_removal_matches_reference(cuda, tag, rho_p, dtype):
    """TorchDC2D(singularity_removal=True) against the reference's own
    (golden sr_tiny: dctorch/simulation2d.py:306-333 with
    dctorch/singularity.py), the primary's background from the model or
    fixed; the Jacobian products of the plain formulation refuse, as there."""
    g = golden("sr_tiny")
    mesh, survey, _ = syn.tiny_2d()
    eng = TorchDC2D(mesh, survey, nky=7, device=cuda, dtype=dtype,
                    quadrature=(g["kys"], g["wq"]), singularity_removal=True,
                    rho_primary=rho_p)
    d, phi, grad, jt = _run(eng, g["m"], g[f"{tag}_dobs"], g[f"{tag}_w"],
                            g[f"{tag}_v"], cuda)
    tol_d, tol_g = (1e-10, 1e-9) if dtype == torch.float64 else (1e-6, 1e-5)
    assert rel(d, g[f"{tag}_dpred"]) < tol_d
    assert abs(phi - g[f"{tag}_phi"]) <= tol_g * abs(g[f"{tag}_phi"])
    assert rel(grad, g[f"{tag}_grad"]) < tol_g
    assert rel(jt, g[f"{tag}_jtvec"]) < tol_g
    f, gm = eng.misfit_and_grad(torch.tensor(g["m"], device=cuda),
                                torch.tensor(g[f"{tag}_dobs"], device=cuda),
                                torch.tensor(g[f"{tag}_w"], device=cuda))
    assert abs(f - g[f"{tag}_mag_phi"]) <= tol_g * abs(g[f"{tag}_mag_phi"])
    assert rel(gm.cpu().numpy(), g[f"{tag}_mag_grad"]) < tol_g
    with pytest.raises(NotImplementedError):
        eng.Jmatrix(torch.tensor(g["m"], device=cuda))
    eng.check()
