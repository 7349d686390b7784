"""Solver-level parity on the GPU, through the C ABI (dct_factorize/dct_solve
and the gather-contract kernel), against the reference's own outputs
(dctorch/tests/test_solver.py specs: solve < 1e-11, FD gradients < 1e-5,
narrow right-hand sides < 1e-13)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

from conftest import golden
from simpeg_dc_torch_b200 import (DCTBatchSolver, DCTSolver, make_batch_solver,
                                  make_solver, sparse_solve, sparse_solve_batch,
                                  sparse_solve_batch_prefactored)

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


def laplacian(nx):
    T = sp.diags([-1.0, 2.0, -1.0], [-1, 0, 1], shape=(nx, nx))
    I = sp.eye(nx)
    A = (sp.kron(I, T) + sp.kron(T, I) + 0.1 * sp.eye(nx * nx)).tocsr()
    A.sort_indices()
    return A


def test_solve_matches_reference(cuda):
    g = golden("solver_nx40")
    n = g["crow"].size - 1
    slv = make_solver(torch.tensor(g["crow"]), torch.tensor(g["col"]), n,
                      g["b"].shape[1], device=cuda)
    assert isinstance(slv, DCTSolver)
    x = sparse_solve(torch.tensor(g["vals"], device=cuda),
                     torch.tensor(g["b"], device=cuda), slv)
    assert rel(x.cpu(), torch.tensor(g["x"])) < 1e-11
    assert slv.check() == 0.0


def test_gradients_match_reference(cuda):
    g = golden("solver_nx12")
    n = g["crow"].size - 1
    slv = DCTSolver(torch.tensor(g["crow"]), torch.tensor(g["col"]), n,
                    g["b"].shape[1], device=cuda)
    vals = torch.tensor(g["vals"], device=cuda, requires_grad=True)
    b = torch.tensor(g["b"], device=cuda, requires_grad=True)
    (torch.tensor(g["w"], device=cuda) * sparse_solve(vals, b, slv)).sum().backward()
    assert rel(vals.grad.cpu(), torch.tensor(g["grad_vals"])) < 1e-11
    assert rel(b.grad.cpu(), torch.tensor(g["grad_b"])) < 1e-11
    # finite differences as in the reference test (eps 1e-6, rel < 1e-5)
    A = sp.csr_matrix((g["vals"], g["col"], g["crow"]), shape=(n, n))

    def loss(data):
        Am = sp.csr_matrix((data, g["col"], g["crow"]), shape=(n, n))
        return float((g["w"] * spla.spsolve(Am.tocsc(), g["b"])).sum())

    rng = np.random.default_rng(1)
    for p in rng.choice(A.nnz, 6, replace=False):
        d = g["vals"].copy()
        d[p] += 1e-6
        fd = (loss(d) - loss(g["vals"])) / 1e-6
        assert abs(fd - float(vals.grad[p])) <= 1e-5 * (abs(fd) + 1e-12)


def test_narrow_rhs_reuses_the_plan(cuda):
    A = laplacian(95)
    n = A.shape[0]
    rng = np.random.default_rng(0)
    b = torch.tensor(rng.standard_normal((n, 140)), device=cuda)
    slv = DCTSolver(torch.tensor(A.indptr), torch.tensor(A.indices), n, 140,
                    device=cuda)
    vals = torch.tensor(A.data, device=cuda)
    x = sparse_solve(vals, b, slv)
    xn = sparse_solve(vals, b[:, :7], slv)
    assert rel(xn, x[:, :7]) < 1e-13
    xr = spla.spsolve(A.tocsc(), b[:, :3].cpu().numpy())
    assert rel(x[:, :3].cpu(), torch.tensor(xr)) < 1e-11


@pytest.mark.parametrize("shared", [True, False])
def test_batch_solver_shared_and_batched_rhs(cuda, shared):
    A = laplacian(30)
    n = A.shape[0]
    nb = 5
    rng = np.random.default_rng(2)
    scale = 1.0 + rng.random(nb)
    vals = torch.tensor(np.stack([A.data * s + 0.05 * s for s in scale]),
                        device=cuda)
    # diagonal shift keeps every system SPD on the same pattern
    diag = torch.tensor((A.indices == np.repeat(np.arange(n), np.diff(A.indptr)))
                        .astype(float), device=cuda)
    vals = vals + 0.3 * diag
    slv = make_batch_solver(torch.tensor(A.indptr), torch.tensor(A.indices), n,
                            4, nb, device=cuda)
    assert isinstance(slv, DCTBatchSolver)
    b = torch.tensor(rng.standard_normal((n, 4) if shared else (nb, n, 4)),
                     device=cuda)
    vr = vals.clone().requires_grad_(True)
    br = b.clone().requires_grad_(True)
    x = sparse_solve_batch(vr, br, slv)
    wgt = torch.tensor(rng.standard_normal(x.shape), device=cuda)
    (wgt * x).sum().backward()
    for k in range(nb):
        Ak = sp.csr_matrix((vals[k].cpu().numpy(), A.indices, A.indptr), shape=(n, n))
        bk = b.cpu().numpy() if shared else b[k].cpu().numpy()
        xk = spla.spsolve(Ak.tocsc(), bk)
        assert rel(x[k].detach().cpu(), torch.tensor(xk)) < 1e-11
        adj = spla.spsolve(Ak.tocsc(), wgt[k].cpu().numpy())
        row = np.repeat(np.arange(n), np.diff(A.indptr))
        gv = -(adj[row] * xk[A.indices]).sum(1)
        assert rel(vr.grad[k].cpu(), torch.tensor(gv)) < 1e-10
    assert br.grad.shape == b.shape
    # prefactored: same values, same gradients
    slv.factorize(vals)
    vp = vals.clone().requires_grad_(True)
    xp = sparse_solve_batch_prefactored(vp, b, slv)
    (wgt * xp).sum().backward()
    assert rel(xp.detach(), x.detach()) < 1e-13
    assert rel(vp.grad, vr.grad) < 1e-12
    assert slv.stamp >= 2


def test_float32_solver_with_refinement(cuda):
    g = golden("solver_nx40")
    n = g["crow"].size - 1
    crow, col = torch.tensor(g["crow"]), torch.tensor(g["col"])
    plain = DCTSolver(crow, col, n, 5, device=cuda, dtype=torch.float32, refine=0)
    refined = DCTSolver(crow, col, n, 5, device=cuda, dtype=torch.float32, refine=2)
    vals = torch.tensor(g["vals"], device=cuda)
    b = torch.tensor(g["b"], device=cuda, dtype=torch.float32)
    x0 = sparse_solve(vals, b, plain).double().cpu()
    x2 = sparse_solve(vals, b, refined).double().cpu()
    xr = torch.tensor(g["x"])
    e0, e2 = rel(x0, xr), rel(x2, xr)
    assert e0 < 1e-4
    assert e2 < 1e-6 and e2 <= e0
    res = refined.check()
    assert res < 1e-7


@pytest.mark.parametrize("k", [4, 3])
def test_wide_supernode_blocked_update(cuda, k):
    """A dense 330 x 330 block coupled to a 2-D grid: a supernode of six
    64-column panels, so the float32 factorization runs its narrow updates
    inside a block of four panels and the deferred K = 256 update beyond it
    (one TMEM accumulator per panel), then a partial second block; k = 4
    takes the bulk-reduction epilogue of the substitution, k = 3 the
    atomics.  Float64 and float32 + refinement against scipy."""
    rng = np.random.default_rng(3)
    G = rng.standard_normal((330, 330))
    D = sp.csr_matrix(G @ G.T / 330 + 4 * np.eye(330))
    L = laplacian(12)
    C = sp.random(L.shape[0], 330, density=0.02, random_state=4) * 0.05
    A = sp.bmat([[L + 2 * sp.eye(L.shape[0]), C], [C.T, D]]).tocsr()
    A = ((A + A.T) * 0.5).tocsr()
    A.sort_indices()
    n = A.shape[0]
    b = rng.standard_normal((n, k))
    xr = torch.tensor(spla.spsolve(A.tocsc(), b))
    crow, col = torch.tensor(A.indptr), torch.tensor(A.indices)
    vals = torch.tensor(A.data, device=cuda)
    for dtype, refine, tol in ((torch.float64, None, 1e-11), (torch.float32, 2, 1e-7)):
        slv = DCTSolver(crow, col, n, k, device=cuda, dtype=dtype,
                        **({} if refine is None else {"refine": refine}))
        bt = torch.tensor(b, device=cuda, dtype=dtype)
        x = sparse_solve(vals, bt, slv).double().cpu()
        assert rel(x, xr) < tol, (dtype, rel(x, xr))
        slv.check()


def test_zero_pivot_is_reported_not_trapped(cuda):
    A = laplacian(8)
    n = A.shape[0]
    vals = torch.tensor(-A.data, device=cuda)      # negative definite
    slv = DCTSolver(torch.tensor(A.indptr), torch.tensor(A.indices), n, 1,
                    device=cuda)
    slv.factorize(vals)
    with pytest.raises(RuntimeError):
        slv.check()
    # the context is still usable afterwards
    slv.factorize(torch.tensor(A.data, device=cuda))
    assert slv.check() == 0.0


def test_cpu_device_is_refused():
    with pytest.raises(NotImplementedError):
        make_solver(torch.tensor([0, 1]), torch.tensor([0]), 1, 1, device="cpu")


def _regularisation_hm(nx, ny, alpha_s, alpha_x, alpha_y, rng):
    """H_m = alpha_s W_s + alpha_x Dx^T Wx Dx + alpha_y Dy^T Wy Dy on an
    nx x ny cell grid (positive weights): SPD for alpha_s > 0, the shape of
    the Gauss-Newton model Hessian the reference solves on the GPU."""
    def diff(n):
        return sp.diags([-np.ones(n - 1), np.ones(n - 1)], [0, 1], shape=(n - 1, n))
    Dx = sp.kron(sp.eye(ny), diff(nx))
    Dy = sp.kron(diff(ny), sp.eye(nx))
    ws = sp.diags(rng.uniform(0.5, 2.0, nx * ny))
    wx = sp.diags(rng.uniform(0.5, 2.0, Dx.shape[0]))
    wy = sp.diags(rng.uniform(0.5, 2.0, Dy.shape[0]))
    H = (alpha_s * ws + alpha_x * Dx.T @ wx @ Dx + alpha_y * Dy.T @ wy @ Dy).tocsr()
    H.sort_indices()
    return H


@pytest.mark.parametrize("k", [1, 3])
def test_gauss_newton_hm_solve_call_site(cuda, k):
    """The reference's TorchGaussNewton._hm_solve_gpu (dctorch/optimization.py:
    727-761) plans once per pattern with make_solver(..., matrix_type='spd'),
    refactorizes per step and accepts the solve when ||H X - rhs|| / ||rhs||
    <= 1e-8.  The same sequence on this package's solver, two steps with
    different values on one plan."""
    rng = np.random.default_rng(11)
    H = _regularisation_hm(90, 40, 1e-3, 1.0, 0.5, rng)
    n = H.shape[0]
    crow = torch.as_tensor(H.indptr, dtype=torch.int32, device=cuda)
    col = torch.as_tensor(H.indices, dtype=torch.int32, device=cuda)
    slv = make_solver(crow, col, n, k, device=cuda, dtype=torch.float64,
                      matrix_type="spd")
    for step in range(2):
        Hs = H.copy()
        Hs.data = Hs.data * (1.0 + 0.5 * step)
        rhs = torch.as_tensor(rng.standard_normal((n, k)), device=cuda)
        vals = torch.as_tensor(Hs.data, dtype=torch.float64, device=cuda)
        slv.factorize(vals)
        X = slv.solve(rhs.contiguous())
        Ht = torch.sparse_csr_tensor(crow.long(), col.long(), vals, (n, n))
        res = torch.linalg.norm(Ht @ X - rhs) / torch.linalg.norm(rhs)
        assert float(res) <= 1e-8
        ref = spla.spsolve(Hs.tocsc(), rhs.cpu().numpy())
        assert rel(X.cpu(), torch.as_tensor(ref.reshape(n, k))) < 1e-10
    assert slv.check() == 0.0
