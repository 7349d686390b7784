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
