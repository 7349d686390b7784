"""General (unsymmetric-valued) systems on the GPU: float64 plans of
matrix_type "general" (cuDSS's GENERAL, dctorch/solver.py:44-47) factor
P A P^T = L U with static pivoting on the symmetric plans' analysis and
schedules.  Checked against SuperLU on 2.5-D and 3-D nodal patterns (the
3-D one has fronts beyond one CTA's shared memory, so the blocked panel LU,
both panel TRSMs and the two-buffer trailing update run): A x = b and
A^T x = b, shared and per-system right-hand sides, and the autograd
gradients of a batched solve, whose adjoint is the transposed solve."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

from simpeg_dc_torch_b200 import _native as nat
from simpeg_dc_torch_b200 import make_batch_solver, make_solver, sparse_solve_batch
from simpeg_dc_torch_b200 import synthetic as syn
from simpeg_dc_torch_b200.operators import nodal_operators

import oracle.dc_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a.detach().cpu() if torch.is_tensor(a) else a)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _general_systems(kind, nbatch, seed):
    """nbatch unsymmetric systems on a nodal pattern: the SPD operator at a
    random conductivity plus an antisymmetric coupling of a quarter of each
    off-diagonal entry (a convection-like term)."""
    if kind == "2d":
        mesh, survey, _ = syn.suite_case("2d-tensor")
        ops = nodal_operators(mesh, survey)
        L = ops.L_ky(0.1)
    else:
        mesh, survey, _ = syn.suite_case("3d-tensor")
        ops = nodal_operators(mesh, survey)
        L = ops.L3()
    rng = np.random.default_rng(seed)
    crow, col, n = ops.crow, ops.col, ops.nN
    r = O.row_of(crow)
    vals = []
    for _ in range(nbatch):
        v = L @ np.exp(rng.uniform(-2, 1, ops.nC))
        A = sp.csr_matrix((v, col, crow), shape=(n, n))
        K = sp.triu(A, 1) * rng.uniform(0.1, 0.25)
        K = K - K.T                        # antisymmetric, same pattern
        B = (A + K).tocsr()
        B.sort_indices()
        vals.append(np.asarray(B[r, col]).ravel())
    return crow, col, n, np.stack(vals)


@pytest.mark.parametrize("kind", ["2d", "3d"])
def test_general_solve_and_transposed_solve(cuda, kind):
    crow, col, n, vals = _general_systems(kind, 2, 1)
    rng = np.random.default_rng(2)
    k = 4
    B = rng.standard_normal((n, k))
    Bb = rng.standard_normal((2, n, k))
    s = make_batch_solver(torch.tensor(crow), torch.tensor(col), n, k, 2, device=cuda,
                          matrix_type="general")
    s.factorize(torch.tensor(vals, device=cuda))
    X = s.solve(torch.tensor(B, device=cuda)).cpu().numpy()
    Xb = s.solve(torch.tensor(Bb, device=cuda)).cpu().numpy()
    Xt = s.solve(torch.tensor(B, device=cuda), transposed=True).cpu().numpy()
    s.check()
    assert s.static_pivots() == 0
    for i in range(2):
        A = sp.csr_matrix((vals[i], col, crow), shape=(n, n))
        assert abs(A - A.T).max() > 1e-3 * abs(A).max()      # really unsymmetric
        lu = spla.splu(A.tocsc())
        assert rel(X[i], lu.solve(B)) < 1e-11
        assert rel(Xb[i], lu.solve(Bb[i])) < 1e-11
        assert rel(Xt[i], lu.solve(B, trans="T")) < 1e-11
    s.free()


def test_general_single_solver(cuda):
    crow, col, n, vals = _general_systems("2d", 1, 3)
    s = make_solver(torch.tensor(crow), torch.tensor(col), n, 2, device=cuda,
                    matrix_type="general")
    s.factorize(torch.tensor(vals[0], device=cuda))
    b = np.random.default_rng(4).standard_normal(n)
    x = s.solve(torch.tensor(b, device=cuda)).cpu().numpy()
    A = sp.csr_matrix((vals[0], col, crow), shape=(n, n))
    assert np.linalg.norm(A @ x - b) / np.linalg.norm(b) < 1e-12
    s.free()


def test_general_autograd_uses_the_transposed_solve(cuda):
    """For the loss sum (x - t)^2 of x = A^{-1} b: grad_vals = -adj_row x_col
    and grad_b = sum_systems adj, with adj = A^{-T} 2 (x - t)."""
    crow, col, n, vals = _general_systems("2d", 2, 5)
    rng = np.random.default_rng(6)
    k = 3
    B = rng.standard_normal((n, k))
    T = rng.standard_normal((2, n, k))
    s = make_batch_solver(torch.tensor(crow), torch.tensor(col), n, k, 2, device=cuda,
                          matrix_type="general")
    v = torch.tensor(vals, device=cuda, requires_grad=True)
    b = torch.tensor(B, device=cuda, requires_grad=True)
    x = sparse_solve_batch(v, b, s)
    ((x - torch.tensor(T, device=cuda)) ** 2).sum().backward()
    s.check()
    r = O.row_of(crow)
    X, ADJ = [], []
    for i in range(2):
        A = sp.csr_matrix((vals[i], col, crow), shape=(n, n)).tocsc()
        lu = spla.splu(A)
        xi = lu.solve(B)
        X.append(xi)
        ADJ.append(lu.solve(2.0 * (xi - T[i]), trans="T"))
    X, ADJ = np.stack(X), np.stack(ADJ)
    gv = -np.einsum("bes,bes->be", ADJ[:, r], X[:, col])
    assert rel(x, X) < 1e-11
    assert rel(v.grad, gv) < 1e-10
    assert rel(b.grad, ADJ.sum(0)) < 1e-10
    s.free()


def test_general_rejects_unsymmetric_patterns_and_other_dtypes(cuda):
    crow = np.array([0, 2, 3, 4], np.int32)          # (0,1) without (1,0)
    col = np.array([0, 1, 1, 2], np.int32)
    with pytest.raises(nat.DCTError):
        make_solver(torch.tensor(crow), torch.tensor(col), 3, 1, device=cuda,
                    matrix_type="general")
    c2, k2, n2, _ = _general_systems("2d", 1, 7)
    with pytest.raises(NotImplementedError):
        make_solver(torch.tensor(c2), torch.tensor(k2), n2, 1, device=cuda,
                    dtype=torch.float32, matrix_type="general")


def test_general_static_pivoting_and_nonfinite_pivots(cuda):
    """A zero diagonal (every pivot of the first elimination step zero) is
    replaced by the static bound and counted, with finite results; a NaN
    value records a zero-pivot error that check() raises."""
    crow, col, n, vals = _general_systems("2d", 1, 8)
    r = O.row_of(crow)
    v = vals[0].copy()
    v[r == col] = 0.0
    s = make_solver(torch.tensor(crow), torch.tensor(col), n, 1, device=cuda,
                    matrix_type="general")
    s.factorize(torch.tensor(v, device=cuda))
    x = s.solve(torch.tensor(np.ones(n), device=cuda))
    s.check()
    assert s.static_pivots() > 0
    assert torch.isfinite(x).all()
    v2 = vals[0].copy()
    v2[0] = np.nan
    s.factorize(torch.tensor(v2, device=cuda))
    s.solve(torch.tensor(np.ones(n), device=cuda))
    with pytest.raises(nat.DCTError):
        s.check()
    s.free()
