"""Tree meshes (octree / quadtree with hanging nodes) and their nodal
operators, on the CPU.  A tree whose leaves all share one level must give
the tensor mesh's operators exactly; a refined tree keeps the operator
symmetric, its gradient term annihilates constants, the hanging-node
interpolation reproduces linear potentials, and a pole source on a half-space
gives the analytic potential to the accuracy of the tensor discretisation."""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from simpeg_dc_torch_b200 import synthetic as syn
from simpeg_dc_torch_b200.mesh import TensorMesh
from simpeg_dc_torch_b200.operators import nodal_operators
from simpeg_dc_torch_b200.survey import (DipoleReceiver, DipoleSource, PoleReceiver,
                                         PoleSource, Survey)
from simpeg_dc_torch_b200.treemesh import TreeMesh


def _cell_perm(a, b):
    """Index into b's cells of each of a's cells (matched by centre)."""
    key = lambda c: np.round(c * 16).astype(np.int64)  # noqa: E731
    kb = {tuple(k): i for i, k in enumerate(key(b.cell_centers))}
    return np.array([kb[tuple(k)] for k in key(a.cell_centers)])


def _A(ops, L, sig):
    return sp.csr_matrix((L @ sig, ops.col, ops.crow), shape=(ops.nN, ops.nN))


def test_uniform_octree_equals_tensor_mesh():
    tm = TreeMesh([(2.0, 8)] * 3, origin=[-8, -8, -16])
    tm.refine(lambda lo, hi: np.full(lo.shape[0], 3))
    tm.finalize()
    ten = TensorMesh([[(2.0, 8)]] * 3, origin=[-8, -8, -16])
    rx = DipoleReceiver(np.array([[2.0, 0, 0], [4.0, 2, 0]]), np.array([[4.0, 0, 0], [6.0, 2, 0]]))
    sv = Survey([DipoleSource([rx], np.r_[-2.0, 0, 0], np.r_[0.0, 2, 0])])
    ot, oo = nodal_operators(tm, sv), nodal_operators(ten, sv)
    assert tm.n_hanging_nodes == 0 and ot.nN == oo.nN
    perm = _cell_perm(tm, ten)
    sig = np.exp(np.random.default_rng(0).uniform(-2, 1, ten.nC))
    At, Ao = _A(ot, ot.L3(), sig[perm]), _A(oo, oo.L3(), sig)
    assert abs(At - Ao).max() <= 1e-14 * abs(Ao).max()
    assert abs(ot.q - oo.q).max() < 1e-15 and abs(ot.Pd - oo.Pd).max() < 1e-15


def test_uniform_quadtree_equals_tensor_mesh_2p5d():
    tm = TreeMesh([(1.5, 16)] * 2, origin=[-12, -24])
    tm.refine(lambda lo, hi: np.full(lo.shape[0], 4))
    tm.finalize()
    ten = TensorMesh([[(1.5, 16)]] * 2, origin=[-12, -24])
    rx = DipoleReceiver(np.array([[3.0, 0.0]]), np.array([[4.5, 0.0]]))
    sv = Survey([PoleSource([rx], np.r_[0.0, 0.0])])
    ot, oo = nodal_operators(tm, sv), nodal_operators(ten, sv)
    perm = _cell_perm(tm, ten)
    sig = np.exp(np.random.default_rng(1).uniform(-2, 1, ten.nC))
    for ky in (0.05, 0.7):
        At, Ao = _A(ot, ot.L_ky(ky), sig[perm]), _A(oo, oo.L_ky(ky), sig)
        assert abs(At - Ao).max() <= 1e-14 * abs(Ao).max()


def _refined():
    tm = TreeMesh([(2.0, 64)] * 3, origin=[-64, -64, -128])
    tm.refine(lambda lo, hi: np.full(lo.shape[0], 2))
    tm.refine_points([[0, 0, 0]], 6, padding=10.0)
    tm.refine_points([[0, 0, 0]], 5, padding=30.0)
    tm.refine_points([[0, 0, 0]], 4, padding=60.0)
    tm.finalize()
    return tm


def test_refined_octree_operator_and_hanging_nodes():
    tm = _refined()
    assert tm.n_hanging_nodes > 0
    # 2:1 balance across faces: neighbouring leaves differ by one level at most
    lev = tm.cell_levels
    assert lev.min() >= 2 and lev.max() == 6
    # the hanging-node interpolation reproduces linear potentials
    allc = tm.origin + tm._all_nodes_f * tm.h0
    u = allc @ np.array([0.3, -1.1, 0.7]) + 2.0
    assert np.abs(tm.P @ u[tm._free] - u).max() < 1e-12
    sv = Survey([PoleSource([PoleReceiver(np.array([[6.0, 0, 0]]))], np.r_[0.0, 0, 0])])
    o = nodal_operators(tm, sv)
    sig = np.exp(np.random.default_rng(2).uniform(-2, 1, tm.nC))
    A = _A(o, o.L3(), sig)
    assert abs(A - A.T).max() <= 1e-14 * abs(A).max()
    Ae = _A(o, o.L_edge, sig)
    assert np.abs(Ae @ np.ones(o.nN)).max() <= 1e-12 * abs(Ae).max()


def test_refined_octree_half_space_potential():
    """Pole source on a 100 ohm-m half-space: V = rho I / (2 pi r) at
    6 - 20 m, within 5 % (no singularity removal; the tensor discretisation
    is at the same level)."""
    tm = _refined()
    pts = np.array([[x, 0.0, 0.0] for x in (6, 8, 10, 14, 20)])
    sv = Survey([PoleSource([PoleReceiver(pts)], np.r_[0.0, 0, 0])])
    o = nodal_operators(tm, sv)
    rho = 100.0
    A = _A(o, o.L3(), np.full(tm.nC, 1 / rho))
    u = spla.spsolve(A.tocsc(), o.q.toarray()[:, 0])
    v = o.Pd @ u
    ana = rho / (2 * np.pi * pts[:, 0])
    assert np.abs(v / ana - 1).max() < 0.05, v / ana


def test_refined_3d_workload_builder_shapes():
    tm, sv, m = syn.dc3d_tree(seed=0, max_level=6, n_el=7, n_sources=12, n_rx=5,
                              refine=((6, 10.0), (5, 30.0), (4, 60.0)))
    assert m.size == tm.nC and np.all(np.isfinite(m))
    assert len(sv.source_list) == 12 and sv.nD == 12 * 5
    for src in sv.source_list:
        assert np.linalg.norm(src.location_a - src.location_b) > 30.0
