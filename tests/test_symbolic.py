"""libdct without a GPU: exported symbols, the nested-dissection analysis and
a task-by-task CPU replay of the factor/solve launch schedules."""
import re
import os

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import pytest

from conftest import ROOT
from schedule_replay import Struct, replay_factor, replay_solve
from simpeg_dc_torch_b200 import _native as nat
from simpeg_dc_torch_b200 import synthetic as syn
from simpeg_dc_torch_b200.operators import nodal_operators


def test_library_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "dct.h")).read()
    declared = set(re.findall(r"^\s*(?:int|void|int64_t|const char\*)\s+(dct_\w+)\s*\(",
                              hdr, re.M))
    assert declared
    L = nat.lib()
    for name in declared:
        assert hasattr(L, name), name
    assert declared <= set(nat.exported_symbols())
    assert L.dct_version() >= 10000


def laplacian(nx):
    T = sp.diags([-1.0, 2.0, -1.0], [-1, 0, 1], shape=(nx, nx))
    I = sp.eye(nx)
    A = (sp.kron(I, T) + sp.kron(T, I) + 0.1 * sp.eye(nx * nx)).tocsr()
    A.sort_indices()
    return A


def _check(A, coords, leaf, rhs, dtype=0):
    sym = nat.Symbolic(A.indptr, A.indices, coords, leaf)
    S = Struct(sym)
    n = A.shape[0]
    assert np.array_equal(np.sort(S.perm), np.arange(n))
    assert np.array_equal(S.iperm[S.perm], np.arange(n))
    # supernodes tile the columns; children precede parents
    assert S.sn_first[0] == 0 and S.sn_first[-1] == n
    par = S.sn_parent
    assert np.all((par == -1) | (par > np.arange(par.size)))
    fronts, dinv = replay_factor(sym, S, A.data, dtype)
    bp = rhs[S.perm]
    xp = replay_solve(sym, S, fronts, bp, dinv, dtype)
    x = np.empty_like(xp)
    x[S.perm] = xp
    xr = spla.spsolve(A.tocsc(), rhs)
    return np.linalg.norm(x - xr) / np.linalg.norm(xr), sym.info()


@pytest.mark.parametrize("coords", [True, False])
def test_replay_2d_grid(coords):
    mesh, survey, m = syn.suite_case("2d-tensor")
    ops = nodal_operators(mesh, survey)
    A = ops.A(np.exp(-m), 0.07)
    err, info = _check(A, mesh.node_grid_index() if coords else None, 64,
                       ops.q.toarray())
    assert err < 1e-12
    assert info["nnz_L"] < 0.2 * ops.nN ** 2


@pytest.mark.parametrize("leaf,dtype", [(16, 0), (64, 0), (64, 1)])
def test_replay_3d_grid_with_large_fronts(leaf, dtype):
    """dtype 1 replays the float32 plan's schedule (128-row tensor-core tiles)."""
    mesh, survey, m = syn.suite_case("3d-tensor")
    ops = nodal_operators(mesh, survey)
    A = ops.A(np.exp(-m))
    err, info = _check(A, mesh.node_grid_index(), leaf, ops.q.toarray(), dtype)
    assert err < 1e-12
    assert info["max_front"] > 160      # the multi-CTA front path is covered


def test_replay_reference_laplacian_without_coordinates():
    A = laplacian(24)
    rhs = np.random.default_rng(0).standard_normal((A.shape[0], 5))
    err, _ = _check(A, None, 32, rhs)
    assert err < 1e-12


@pytest.mark.parametrize("dtype", [0, 1])
def test_replay_wide_supernode_blocked_update(dtype):
    """A dense 330 x 330 block coupled to a 2-D grid: one supernode of six
    panels, i.e. a full block of four panels and a partial one, so that the
    float32 schedule's deferred K = 256 updates (and the narrow updates
    inside each block) are replayed."""
    rng = np.random.default_rng(3)
    G = rng.standard_normal((330, 330))
    D = sp.csr_matrix(G @ G.T / 330 + 4 * np.eye(330))
    L = laplacian(12)
    C = sp.random(L.shape[0], 330, density=0.02, random_state=4) * 0.05
    A = sp.bmat([[L + 2 * sp.eye(L.shape[0]), C], [C.T, D]]).tocsr()
    A = ((A + A.T) * 0.5).tocsr()
    A.sort_indices()
    rhs = rng.standard_normal((A.shape[0], 3))
    err, info = _check(A, None, 32, rhs, dtype)
    assert err < 1e-11
    assert info["max_ns"] > 4 * 64


def test_disconnected_pattern():
    A = sp.block_diag([laplacian(6), laplacian(5), sp.eye(3) * 2.0]).tocsr()
    A.sort_indices()
    rhs = np.random.default_rng(1).standard_normal((A.shape[0], 2))
    err, _ = _check(A, None, 8, rhs)
    assert err < 1e-12


def test_rejects_unsymmetric_pattern():
    A = sp.csr_matrix(np.array([[2.0, 1.0, 0.0], [0.0, 2.0, 0.0],
                                [0.0, 0.0, 2.0]]))
    with pytest.raises(nat.DCTError) as ei:
        nat.Symbolic(A.indptr, A.indices)
    assert ei.value.code == 6


def test_rejects_bad_indices():
    with pytest.raises(nat.DCTError):
        nat.Symbolic(np.array([0, 1, 2]), np.array([0, 5]))


def test_schedule_counts_are_consistent():
    mesh, survey, m = syn.suite_case("3d-tensor")
    ops = nodal_operators(mesh, survey)
    sym = nat.Symbolic(ops.crow, ops.col, mesh.node_grid_index(), 64)
    for dtype in (0, 1):
        for which in (0, 1, 2, 3, 4):
            tasks, launches = sym.schedule(dtype, which)
            assert launches[:, 3].sum() == tasks.shape[0]
            assert np.all(np.diff(launches[:, 2]) >= 0)
