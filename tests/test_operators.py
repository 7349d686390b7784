"""Build-time operators: pinned checksums, structure, and physics."""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import pytest

from conftest import golden
from simpeg_dc_torch_b200 import synthetic as syn
from simpeg_dc_torch_b200.operators import nodal_operators
from simpeg_dc_torch_b200.quadrature import (electrode_distance_range,
                                             k0_quadrature)


@pytest.mark.parametrize("name,case", [
    ("dc2d_suite", lambda: syn.suite_case("2d-tensor")),
    ("dc3d_suite", lambda: syn.suite_case("3d-tensor")),
    ("dc2d_tiny", syn.tiny_2d), ("dc3d_tiny", syn.tiny_3d)])
def test_operator_checksums_match_fixture(name, case):
    g = golden(name)
    mesh, survey, m = case()
    ops = nodal_operators(mesh, survey)
    assert ops.nnzA == g["nnzA"] and ops.nN == g["nN"] and ops.nC == g["nC"]
    for key, val in [("ck_Ledge", np.abs(ops.L_edge.data).sum()),
                     ("ck_Lnode", np.abs(ops.L_node.data).sum()),
                     ("ck_bc", np.abs(ops.L_bc(0.1).data).sum()),
                     ("ck_q", np.abs(ops.q.data).sum()),
                     ("ck_Pd", np.abs(ops.Pd.data).sum())]:
        assert abs(val - g[key]) <= 1e-12 * abs(g[key]), key
    assert np.allclose(m, g["m"])


def test_tiny_operators_equal_stored_ones():
    g = golden("dc2d_tiny")
    mesh, survey, _ = syn.tiny_2d()
    ops = nodal_operators(mesh, survey)
    L = sp.vstack([ops.L_ky(k) for k in g["kys"]]).tocsr()
    Lg = sp.csr_matrix((g["L_data"], g["L_indices"], g["L_indptr"]),
                       shape=L.shape)
    assert abs(L - Lg).max() <= 1e-14 * abs(Lg).max()
    assert np.array_equal(ops.crow, g["crow"]) and np.array_equal(ops.col, g["col"])


@pytest.mark.parametrize("case", [syn.tiny_2d, syn.tiny_3d])
def test_system_is_symmetric_positive_definite(case):
    mesh, survey, m = case()
    ops = nodal_operators(mesh, survey)
    sig = np.exp(-m)
    A = ops.A(sig, 0.05) if mesh.dim == 2 else ops.A(sig)
    assert abs(A - A.T).max() <= 1e-14 * abs(A).max()
    ev = np.linalg.eigvalsh(A.toarray())
    assert ev.min() > 0


def test_grad_term_annihilates_constants():
    mesh, survey, m = syn.tiny_3d()
    ops = nodal_operators(mesh, survey)
    A = sp.csr_matrix((ops.L_edge @ np.exp(-m), ops.col, ops.crow))
    assert np.abs(A @ np.ones(ops.nN)).max() <= 1e-12 * abs(A).max()


def test_quadrature_matches_reference_points():
    g = golden("quad")
    for i in range(4):
        lo, hi, n = g[f"args{i}"]
        p, w, info = k0_quadrature(lo, hi, int(n))
        assert np.allclose(p, g[f"pts{i}"], rtol=1e-12, atol=0)
        assert np.allclose(w, g[f"wts{i}"], rtol=1e-12, atol=0)
        assert abs(info["max_rel_err"] - g[f"err{i}"]) <= 1e-9 * g[f"err{i}"] + 1e-15


def test_half_space_2p5d_matches_analytic():
    """A homogeneous 100 ohm-m half space against rho/(2 pi) * geometric sum;
    the plain nodal method is within a few percent (no singularity removal)."""
    rho = 100.0
    mesh = syn.padded_mesh_2d(2.5, 100, 50, 15)
    xe = np.arange(21) * 5.0 - 50.0
    survey = syn.Survey(syn.dipole_dipole_2d(xe, 6))
    ops = nodal_operators(mesh, survey)
    kys, wq, _ = k0_quadrature(*electrode_distance_range(survey), 11)
    sig = np.full(ops.nC, 1 / rho)
    U = 0.0
    for k, w in zip(kys, wq):
        U = U + w * spla.spsolve(ops.A(sig, k).tocsc(), ops.q.toarray())
    d = np.asarray((ops.Pd @ U)[np.arange(ops.nD), ops.sidx]).ravel()
    truth = []
    for src in survey.source_list:
        a, b = src.location_a, src.location_b
        for rx in src.receiver_list:
            for M, N in zip(rx.locations_m, rx.locations_n):
                r = lambda p, q: np.linalg.norm(p - q)  # noqa: E731
                truth.append(rho * (1 / r(a, M) - 1 / r(b, M) - 1 / r(a, N)
                                    + 1 / r(b, N)) / (2 * np.pi))
    err = np.abs(d / np.array(truth) - 1)
    assert np.median(err) < 0.03 and err.max() < 0.1


class _DiscretizeLikeMesh:
    """Only the public attributes a discretize.TensorMesh has: h, origin, dim,
    _meshType (no private helpers of this package's TensorMesh)."""
    _meshType = "TENSOR"

    def __init__(self, h, origin):
        self.h = tuple(np.asarray(w, float) for w in h)
        self.origin = np.asarray(origin, float)
        self.dim = len(self.h)


class _SimpegLikeDipoleRx:
    def __init__(self, m, n):
        self.locations_m, self.locations_n = np.asarray(m), np.asarray(n)
        self.data_type = "volt"

    @property
    def nD(self):
        return self.locations_m.shape[0]


class _SimpegLikePoleRx:
    def __init__(self, m):
        self.locations = np.asarray(m)
        self.data_type = "volt"

    @property
    def nD(self):
        return self.locations.shape[0]


class _SimpegLikeSrc:
    def __init__(self, rxs, a, b=None, current=1.0):
        self.receiver_list = rxs
        self.location_a = np.asarray(a, float)
        # SimPEG writes a pole source's B electrode as NaN
        self.location_b = (np.full_like(self.location_a, np.nan) if b is None
                           else np.asarray(b, float))
        self.current = current


class _SimpegLikeSurvey:
    def __init__(self, srcs):
        self.source_list = srcs

    @property
    def nD(self):
        return sum(rx.nD for s in self.source_list for rx in s.receiver_list)


def _mirror(survey):
    """A SimPEG-shaped copy of one of this package's surveys."""
    out = []
    for src in survey.source_list:
        rxs = []
        for rx in src.receiver_list:
            if rx.locations_n is None:
                rxs.append(_SimpegLikePoleRx(rx.locations_m))
            else:
                rxs.append(_SimpegLikeDipoleRx(rx.locations_m, rx.locations_n))
        out.append(_SimpegLikeSrc(rxs, src.location_a, src.location_b, src.current))
    return _SimpegLikeSurvey(out)


def test_engines_accept_discretize_and_simpeg_shaped_objects():
    """The operators built from a mesh that has only discretize's public
    attributes and a survey that has only SimPEG's equal the ones built from
    this package's own classes (the reference engines take discretize /
    SimPEG objects, dctorch/simulation2d.py:37-40, simulation3d.py:47-48)."""
    from simpeg_dc_torch_b200 import synthetic as syn
    from simpeg_dc_torch_b200.mesh import as_tensor_mesh
    from simpeg_dc_torch_b200.quadrature import electrode_distance_range
    for case in (syn.tiny_2d, syn.tiny_3d):
        mesh, survey, _ = case()
        dmesh = _DiscretizeLikeMesh(mesh.h, mesh.origin)
        ssurv = _mirror(survey)
        a = nodal_operators(mesh, survey)
        b = nodal_operators(dmesh, ssurv)
        assert np.array_equal(a.crow, b.crow) and np.array_equal(a.col, b.col)
        for M, N in ((a.L_edge, b.L_edge), (a.L_node, b.L_node), (a.q, b.q),
                     (a.Pd, b.Pd)):
            assert abs(M - N).max() == 0.0
        assert np.array_equal(a.sidx, b.sidx)
        L = a.L3() if mesh.dim == 3 else a.L_ky(0.1)
        Lb = b.L3() if mesh.dim == 3 else b.L_ky(0.1)
        assert abs(L - Lb).max() == 0.0
        assert electrode_distance_range(survey) == electrode_distance_range(ssurv)
        assert np.array_equal(as_tensor_mesh(dmesh).node_grid_index(),
                              mesh.node_grid_index())

    class _Tree:
        _meshType = "TREE"
        h = ()
    with pytest.raises(NotImplementedError):
        as_tensor_mesh(_Tree())
