"""Complex-symmetric systems on the GPU: the solver's complex128 plans
(A^T = A, factored L L^T without conjugation) against complex SuperLU, the
complex-safe adjoint of the batched solve (dctorch/solver.py:236-281), and the
complex-resistivity engine TorchCR2D against the reference's own
(golden cr_tiny, made by running dctorch/cr2d.py on the tiny 2-D problem on
its complex SciPyBatchSolver), and at the large 2.5-D configuration (56,525
nodes, 10 wavenumbers, 186 sources) against the oracle on the block LU slab
solver.  Complex128 is held to 1e-10 on data and 1e-9 on gradients, the
levels of the float64 engine tests.""" 
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

from conftest import golden
from simpeg_dc_torch_b200 import TorchCR2D, make_batch_solver, sparse_solve_batch
from simpeg_dc_torch_b200 import synthetic as syn
from simpeg_dc_torch_b200.operators import nodal_operators

import oracle.dc_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a.detach().cpu() if torch.is_tensor(a) else a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _complex_systems(kind, nbatch, seed):
    """nbatch complex-symmetric systems A(sigma*), sigma* = sigma (1 - i m)
    with sigma and m random per system, on the pattern of a 2.5-D (one
    wavenumber) or 3-D nodal operator.  Returns (crow, col, n, vals)."""
    if kind == "2d":
        mesh, survey, _ = syn.suite_case("2d-tensor")
        ops = nodal_operators(mesh, survey)
        L = ops.L_ky(0.1)
    else:
        mesh, survey, _ = syn.tiny_3d() if kind == "3d-tiny" else syn.suite_case("3d-tensor")
        ops = nodal_operators(mesh, survey)
        L = ops.L3()
    rng = np.random.default_rng(seed)
    vals = []
    for _ in range(nbatch):
        sig = np.exp(rng.uniform(-3, 1, ops.nC))
        chg = rng.uniform(0.0, 0.3, ops.nC)
        vals.append(L @ sig - 1j * (L @ (sig * chg)))
    return ops.crow, ops.col, ops.nN, np.stack(vals)


@pytest.mark.parametrize("kind", ["2d", "3d-tiny", "3d"])
def test_complex_solve_matches_superlu(cuda, kind):
    """Forward solves of shared and per-system right-hand sides, against
    complex SuperLU; the 3-D patterns carry fronts wider than one CTA's
    shared-memory factorization, so the large-front kernels run too."""
    crow, col, n, vals = _complex_systems(kind, 3, 1)
    rng = np.random.default_rng(2)
    k = 5
    B = rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k))
    Bb = rng.standard_normal((3, n, k)) + 1j * rng.standard_normal((3, n, k))
    s = make_batch_solver(torch.tensor(crow), torch.tensor(col), n, k, 3,
                          device=cuda, dtype=torch.complex128)
    s.factorize(torch.tensor(vals, device=cuda))
    X = s.solve(torch.tensor(B, device=cuda)).cpu().numpy()
    Xb = s.solve(torch.tensor(Bb, device=cuda)).cpu().numpy()
    s.check()
    for b in range(3):
        A = sp.csr_matrix((vals[b], col, crow), shape=(n, n)).tocsc()
        lu = spla.splu(A)
        assert rel(X[b], lu.solve(B)) < 1e-11
        assert rel(Xb[b], lu.solve(Bb[b])) < 1e-11
    s.free()


def test_complex_solve_adjoint(cuda):
    """The backward of sparse_solve_batch on complex values: for the real loss
    sum |x - t|^2 torch hands the solve G = 2 (x - t); the adjoint
    adj = A^{-1} conj(G) gives grad_vals = conj(-sum_s adj[row_e] x[col_e])
    and grad_b = conj(sum_b adj) (dctorch/solver.py:261-281)."""
    crow, col, n, vals = _complex_systems("2d", 2, 3)
    rng = np.random.default_rng(4)
    k = 3
    B = rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k))
    T = rng.standard_normal((2, n, k)) + 1j * rng.standard_normal((2, n, k))
    s = make_batch_solver(torch.tensor(crow), torch.tensor(col), n, k, 2,
                          device=cuda, dtype=torch.complex128, matrix_type="symmetric")
    v = torch.tensor(vals, device=cuda, requires_grad=True)
    b = torch.tensor(B, device=cuda, requires_grad=True)
    x = sparse_solve_batch(v, b, s)
    loss = ((x - torch.tensor(T, device=cuda)).abs() ** 2).sum()
    loss.backward()
    s.check()
    r = O.row_of(crow)
    X, ADJ = [], []
    for i in range(2):
        A = sp.csr_matrix((vals[i], col, crow), shape=(n, n)).tocsc()
        lu = spla.splu(A)
        xi = lu.solve(B)
        X.append(xi)
        ADJ.append(lu.solve(np.conj(2.0 * (xi - T[i]))))
    X, ADJ = np.stack(X), np.stack(ADJ)
    gv = np.conj(-np.einsum("bes,bes->be", ADJ[:, r], X[:, col]))
    gb = np.conj(ADJ.sum(0))
    assert rel(x, X) < 1e-11
    assert rel(v.grad, gv) < 1e-10
    assert rel(b.grad, gb) < 1e-10
    s.free()


def test_complex_plan_rejects_real_values(cuda):
    crow, col, n, vals = _complex_systems("2d", 1, 5)
    s = make_batch_solver(torch.tensor(crow), torch.tensor(col), n, 1, 1,
                          device=cuda, dtype=torch.complex128)
    with pytest.raises(Exception):
        s._plan.factorize(torch.tensor(vals.real, device=cuda).data_ptr(), 0,
                          vals.shape[1], torch.cuda.current_stream(cuda).cuda_stream)
    with pytest.raises(NotImplementedError):
        make_batch_solver(torch.tensor(crow), torch.tensor(col), n, 1, 1,
                          device=cuda, dtype=torch.complex128, matrix_type="spd")
    s.free()


@pytest.mark.parametrize("datum", ["magnitude", "real"])
def test_cr_matches_reference(cuda, datum):
    J = golden("cr_tiny")
    mesh, survey, _ = syn.tiny_2d()
    eng = TorchCR2D(mesh, survey, nky=7, device=cuda, ip_scale=1000.0,
                    dc_datum=datum, quadrature=(J["kys"], J["wq"]))
    t = lambda k: torch.tensor(J[f"{datum}_{k}"], device=cuda)  # noqa: E731
    mm = torch.tensor(J[f"{datum}_m"], device=cuda, requires_grad=True)
    phi = eng.misfit(mm, t("dobs_rho"), t("w_rho"), t("dobs_ip"), t("w_ip"), lam=0.7)
    phi.backward()
    with torch.no_grad():
        d_rho, d_ip = eng.dpred(mm)
    eng.check()
    assert rel(d_rho, J[f"{datum}_d_rho"]) < 1e-10
    assert rel(d_ip, J[f"{datum}_d_ip"]) < 1e-10
    assert abs(float(phi.detach()) - J[f"{datum}_phi"]) <= 1e-9 * abs(J[f"{datum}_phi"])
    assert rel(mm.grad, J[f"{datum}_grad"]) < 1e-9


def test_cr_active_cells_and_complex64(cuda):
    """On active cells (log-rho val_inactive and m = 0 elsewhere) the data and
    the gradient equal the full-mesh oracle's restricted to the active cells;
    a complex64 engine (solved in complex128) returns the model's dtype."""
    g = golden("dc2d_tiny")
    J = golden("cr_tiny")
    mesh, survey, _ = syn.tiny_2d()
    n = J["m_rho"].size
    act = np.random.default_rng(6).uniform(size=n) > 0.3
    eng = TorchCR2D(mesh, survey, nky=7, device=cuda, ip_scale=1000.0,
                    active_cells=act, val_inactive=4.0, quadrature=(J["kys"], J["wq"]))
    m_rho = J["m_rho"].copy()
    m_rho[~act] = 4.0
    chg = np.where(act, J["magnitude_m"][n:], 0.0)
    op = dict(crow=g["crow"], col=g["col"], nN=g["crow"].size - 1, Q=g["Q"],
              Pd=sp.csr_matrix((g["Pd_data"], g["Pd_indices"], g["Pd_indptr"]),
                               shape=(g["sidx"].size, g["crow"].size - 1)),
              sidx=g["sidx"], wq=g["wq"],
              Lstack=sp.csr_matrix((g["L_data"], g["L_indices"], g["L_indptr"])))
    dr, di = O.cr_dpred_2d(op, m_rho, chg, 1000.0, "magnitude")
    mm = torch.tensor(np.concatenate([m_rho[act], chg[act]]), device=cuda,
                      requires_grad=True)
    d_rho, d_ip = eng.dpred(mm)
    assert rel(d_rho, dr) < 1e-10 and rel(d_ip, di) < 1e-10
    dobs_r, dobs_i = dr * 1.05, di + 3.0
    w_r, w_i = 1.0 / np.abs(dr), np.full(di.size, 0.5)
    phi = eng.misfit(mm, *(torch.tensor(a, device=cuda) for a in
                           (dobs_r, w_r, dobs_i, w_i)), lam=0.7)
    phi.backward()
    phi_o, grad_o = O.cr_misfit_grad_2d(op, np.concatenate([m_rho, chg]), 1000.0,
                                        "magnitude", dobs_r, w_r, dobs_i, w_i, 0.7)
    assert abs(float(phi.detach()) - phi_o) <= 1e-9 * phi_o
    want = np.concatenate([grad_o[:n][act], grad_o[n:][act]])
    assert rel(mm.grad, want) < 1e-9
    e64 = TorchCR2D(mesh, survey, nky=7, device=cuda, dtype=torch.complex64,
                    ip_scale=1000.0, quadrature=(J["kys"], J["wq"]))
    d32 = e64.dpred(torch.tensor(J["magnitude_m"], dtype=torch.float32, device=cuda))
    assert d32[0].dtype == torch.float32
    assert rel(d32[0], J["magnitude_d_rho"]) < 1e-6
    assert rel(d32[1], J["magnitude_d_ip"]) < 1e-5
    eng.check()


def test_cr_large_2d_against_oracle(cuda):
    """TorchCR2D on the large 2.5-D workload against the oracle (complex
    block-tridiagonal LU over the grid slabs): data of both kinds and the
    joint misfit gradient."""
    mesh, survey, m = syn.dc2d_large(seed=0)
    eng = TorchCR2D(mesh, survey, nky=12, device=cuda, ip_scale=1000.0)
    dc = eng.dc
    ops = dc._ops
    op = dict(Lstack=dc._L, crow=ops.crow, col=ops.col, nN=ops.nN, Q=ops.q.toarray(),
              Pd=ops.Pd, sidx=ops.sidx, wq=dc.wq_np,
              slab=O.grid_slabs(mesh.node_grid_index()))
    chg = np.random.default_rng(3).uniform(0.01, 0.2, ops.nC)
    mm = np.concatenate([m, chg])
    dr, di = O.cr_dpred_2d(op, m, chg, 1000.0, "magnitude")
    dobs_r = dr * (1.0 + 0.03 * np.random.default_rng(4).standard_normal(dr.size))
    w_r = 1.0 / np.abs(dobs_r)
    dobs_i = di + 2.0
    w_i = np.full(di.size, 0.5)
    phi_o, g_o = O.cr_misfit_grad_2d(op, mm, 1000.0, "magnitude", dobs_r, w_r, dobs_i,
                                     w_i, 0.7)
    x = torch.tensor(mm, device=cuda, requires_grad=True)
    phi = eng.misfit(x, *(torch.tensor(a, device=cuda) for a in (dobs_r, w_r, dobs_i, w_i)),
                     lam=0.7)
    phi.backward()
    with torch.no_grad():
        d_rho, d_ip = eng.dpred(x)
    eng.check()
    assert rel(d_rho, dr) < 1e-10 and rel(d_ip, di) < 1e-10
    assert abs(float(phi.detach()) - phi_o) <= 1e-9 * phi_o
    assert rel(x.grad, g_o) < 1e-9
