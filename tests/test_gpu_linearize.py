"""Linearised products of the 2.5-D engine on the GPU: TorchDC2D.Jmatrix /
Jvec and Linearization2D (Jvec, Jtvec, diag_JtDJ, Jmatrix) against the
reference's own outputs (golden fixture dc2d_lin, made by running
dctorch/simulation2d.py:439-818) and against the CPU oracle on the small
2.5-D workload.  The reference's own spec for J is 1e-12 against its Jtvec
(dctorch/tests/test_jmatrix.py:77-79); float64 here is held to 1e-10,
float32 + refinement to 1e-6."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

from conftest import golden
from oracle import dc_oracle as O
from simpeg_dc_torch_b200 import TorchDC2D
from simpeg_dc_torch_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _tiny(cuda, dtype):
    g = golden("dc2d_tiny")
    mesh, survey, _ = syn.tiny_2d()
    return TorchDC2D(mesh, survey, device=cuda, dtype=dtype,
                     quadrature=(g["kys"], g["wq"]))


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_linearised_products_match_reference(cuda, dtype):
    L = golden("dc2d_lin")
    eng = _tiny(cuda, dtype)
    tol = 1e-10 if dtype == torch.float64 else 1e-6
    m = torch.tensor(L["m"], device=cuda)
    u = torch.tensor(L["u"], device=cuda)
    v = torch.tensor(L["v"], device=cuda)
    dw = torch.tensor(L["dw"], device=cuda)
    assert rel(eng.Jmatrix(m, block=5).cpu(), L["jmatrix"]) < tol
    assert rel(eng.Jvec(m, u).cpu(), L["jvec"]) < tol
    lin = eng.linearize(m)
    assert rel(lin.d.cpu(), L["lin_d"]) < tol
    assert rel(lin.Jvec(u).cpu(), L["lin_jvec"]) < tol
    assert rel(lin.Jtvec(v).cpu(), L["lin_jtvec"]) < tol
    assert rel(lin.diag_JtDJ(dw, sub=3).cpu(), L["lin_diag"]) < tol
    assert rel(lin.Jmatrix(sub=4).cpu(), L["lin_jmatrix"]) < tol
    eng.check()


def test_block_width_is_bookkeeping(cuda):
    """Blocks of 7 (padded tail), 1 and nD give the same matrix
    (dctorch/tests/test_jmatrix.py:68-79)."""
    mesh, survey, m = syn.dc2d_small()
    eng = TorchDC2D(mesh, survey, nky=11, device=cuda)
    mt = torch.tensor(m, device=cuda)
    J = eng.Jmatrix(mt).cpu().numpy()
    assert J.shape == (eng.nD, eng.nC)
    for blk in (7, 1, eng.nD):
        assert rel(eng.Jmatrix(mt, block=blk).cpu(), J) < 1e-12
    # rows of J are J^T e_i, columns J e_j
    e = torch.zeros(eng.nD, dtype=torch.float64, device=cuda)
    for i in (0, eng.nD // 2, eng.nD - 1):
        e.zero_()
        e[i] = 1.0
        assert rel(eng.Jtvec(mt, e).cpu(), J[i]) < 1e-10
    rng = np.random.default_rng(5)
    u = rng.standard_normal(eng.nC)
    assert rel(eng.Jvec(mt, torch.tensor(u, device=cuda)).cpu(), J @ u) < 1e-10
    eng.check()


def test_c1_products_against_oracle(cuda):
    mesh, survey, m = syn.dc2d_small()
    eng = TorchDC2D(mesh, survey, nky=11, device=cuda)
    op = dict(crow=eng._ops.crow, col=eng._ops.col, nN=eng.nN,
              Q=eng._ops.q.toarray(), Pd=sp.csr_matrix(eng._ops.Pd),
              sidx=eng._ops.sidx, Lstack=eng._L, wq=eng.wq_np)
    rng = np.random.default_rng(9)
    u = rng.standard_normal(eng.nC)
    dw = rng.uniform(0.5, 2.0, eng.nD)
    mt = torch.tensor(m, device=cuda)
    lin = eng.linearize(mt)
    assert rel(lin.Jvec(torch.tensor(u, device=cuda)).cpu(), O.jvec_2d(op, m, u)) < 1e-9
    assert rel(lin.diag_JtDJ(torch.tensor(dw, device=cuda)).cpu(),
               O.diag_jtdj_2d(op, m, dw)) < 1e-9


def test_active_cells_select_columns(cuda):
    """With active cells J has the active columns, equal to the full-mesh
    columns there (dctorch/tests/test_jmatrix.py:82-97)."""
    mesh, survey, m = syn.dc2d_small()
    rng = np.random.default_rng(2)
    act = rng.uniform(size=mesh.nC) > 0.3
    eng_f = TorchDC2D(mesh, survey, nky=11, device=cuda)
    eng_a = TorchDC2D(mesh, survey, nky=11, device=cuda, active_cells=act,
                      val_inactive=float(np.log(100.0)))
    m_full = m.copy()
    m_full[~act] = np.log(100.0)
    Jf = eng_f.Jmatrix(torch.tensor(m_full, device=cuda)).cpu().numpy()
    Ja = eng_a.Jmatrix(torch.tensor(m[act], device=cuda)).cpu().numpy()
    assert Ja.shape == (eng_a.nD, int(act.sum()))
    assert rel(Ja, Jf[:, act]) < 1e-12


def test_linearization_survives_a_refactorization(cuda):
    """A line-search dpred at another model replaces the factors; the next
    product restores this linearization's."""
    L = golden("dc2d_lin")
    eng = _tiny(cuda, torch.float64)
    m = torch.tensor(L["m"], device=cuda)
    lin = eng.linearize(m)
    with torch.no_grad():
        eng.dpred(m + 0.3)
    assert rel(lin.Jvec(torch.tensor(L["u"], device=cuda)).cpu(), L["lin_jvec"]) < 1e-10
    assert rel(lin.Jtvec(torch.tensor(L["v"], device=cuda)).cpu(), L["lin_jtvec"]) < 1e-10
