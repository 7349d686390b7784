"""The CPU oracle against outputs of the reference itself (golden fixtures)."""
import numpy as np
import scipy.sparse as sp

from conftest import golden
from oracle import dc_oracle as O


def _ops(g, three_d):
    n = g["crow"].size - 1
    L = sp.csr_matrix((g["L_data"], g["L_indices"], g["L_indptr"]))
    Pd = sp.csr_matrix((g["Pd_data"], g["Pd_indices"], g["Pd_indptr"]),
                       shape=(g["sidx"].size, n))
    op = dict(crow=g["crow"], col=g["col"], nN=n, Q=g["Q"], Pd=Pd,
              sidx=g["sidx"])
    if three_d:
        op["L3"] = L
    else:
        op["Lstack"] = L
        op["wq"] = g["wq"]
    return op


def test_solver_forward_and_vjp_match_reference():
    for name in ("solver_nx12", "solver_nx40"):
        g = golden(name)
        x, gv, gb = O.sparse_solve_vjp(g["crow"], g["col"], g["vals"], g["b"],
                                       g["w"])
        assert O.rel(x, g["x"]) < 1e-13
        assert O.rel(gv, g["grad_vals"]) < 1e-12
        assert O.rel(gb, g["grad_b"]) < 1e-12


def test_dc2d_tiny_matches_reference():
    g = golden("dc2d_tiny")
    op = _ops(g, False)
    m, dobs, w, v = g["m"], g["dobs"], g["w"], g["v"]
    assert O.rel(O.dpred_2d(op, m), g["dpred"]) < 1e-12
    phi, grad = O.misfit_grad_2d(op, m, dobs, w)
    assert abs(phi - g["phi"]) <= 1e-12 * abs(g["phi"])
    assert O.rel(grad, g["grad"]) < 1e-11
    assert O.rel(O.jtvec_2d(op, m, v), g["jtvec"]) < 1e-11
    # the reference's chunked products equal its whole-survey ones
    assert O.rel(g["jtvec_chunk"], g["jtvec"]) < 1e-12
    assert O.rel(g["mag_grad"], g["grad"]) < 1e-12


def test_dc3d_tiny_matches_reference():
    g = golden("dc3d_tiny")
    op = _ops(g, True)
    m, dobs, w, v = g["m"], g["dobs"], g["w"], g["v"]
    assert O.rel(O.dpred_3d(op, m), g["dpred"]) < 1e-12
    phi, grad = O.misfit_grad_3d(op, m, dobs, w)
    assert abs(phi - g["phi"]) <= 1e-12 * abs(g["phi"])
    assert O.rel(grad, g["grad"]) < 1e-11
    assert O.rel(O.jtvec_3d(op, m, v), g["jtvec"]) < 1e-11


def test_oracle_gradient_is_a_derivative():
    """Central differences of the oracle's own misfit (no reference needed)."""
    g = golden("dc2d_tiny")
    op = _ops(g, False)
    m, dobs, w = g["m"], g["dobs"], g["w"]
    _, grad = O.misfit_grad_2d(op, m, dobs, w)
    rng = np.random.default_rng(3)
    u = rng.standard_normal(m.size)
    u /= np.linalg.norm(u)
    h = 1e-5
    fd = (O.misfit_2d(op, m + h * u, dobs, w)
          - O.misfit_2d(op, m - h * u, dobs, w)) / (2 * h)
    assert abs(fd - grad @ u) <= 1e-6 * abs(fd)


def test_linearised_products_match_reference():
    """Jmatrix / Jvec / diag(J^T D J) of the oracle against the reference's
    TorchDC2D.Jmatrix, Jvec and Linearization2D (dctorch/simulation2d.py:
    439-529, 537-818), run on the dc2d_tiny problem."""
    g = golden("dc2d_tiny")
    L = golden("dc2d_lin")
    op = _ops(g, False)
    m = L["m"]
    J = O.jmatrix_2d(op, m)
    assert O.rel(J, L["jmatrix"]) < 1e-11
    assert O.rel(J, L["lin_jmatrix"]) < 1e-11
    assert O.rel(O.jvec_2d(op, m, L["u"]), L["jvec"]) < 1e-11
    assert O.rel(L["lin_jvec"], L["jvec"]) < 1e-12
    assert O.rel(O.jtvec_2d(op, m, L["v"]), L["lin_jtvec"]) < 1e-11
    assert O.rel(O.diag_jtdj_2d(op, m, L["dw"]), L["lin_diag"]) < 1e-11
    assert O.rel(O.dpred_2d(op, m), L["lin_d"]) < 1e-12
    # J is the Jacobian of dpred: its rows are the Jtvec of unit data
    u = L["u"]
    assert O.rel(J @ u, L["jvec"]) < 1e-11


def _datum_flags(survey, rx_flags):
    """Per-datum chargeability flags from per-receiver ones (survey order)."""
    out, i = [], 0
    for src in survey.source_list:
        for rx in src.receiver_list:
            out += [bool(rx_flags[i])] * rx.nD
            i += 1
    return np.array(out)


def test_ip_forward_matches_reference():
    """Linearized IP of the oracle (scale * J(m_dc) eta) against the
    reference's TorchIP2D / TorchIP3D (dctorch/ip2d.py, ip3d.py) on the tiny
    problems, every other receiver of apparent-chargeability type."""
    from simpeg_dc_torch_b200 import synthetic as syn
    ip = golden("ip_tiny")
    for tag, name, case, three_d in (("2d", "dc2d_tiny", syn.tiny_2d, False),
                                     ("3d", "dc3d_tiny", syn.tiny_3d, True)):
        op = _ops(golden(name), three_d)
        _, survey, _ = case()
        charge = _datum_flags(survey, ip[f"{tag}_flags"])
        m, eta = ip[f"{tag}_m"], ip[f"{tag}_eta"]
        v_dc = O.dpred_3d(op, m) if three_d else O.dpred_2d(op, m)
        assert O.rel(v_dc, ip[f"{tag}_vdc"]) < 1e-12
        scale = O.ip_scale(v_dc, charge)
        assert O.rel(scale, ip[f"{tag}_scale"]) < 1e-12
        assert charge.any() and (~charge).any()
        d = (O.ip_dpred_3d if three_d else O.ip_dpred_2d)(op, m, eta, charge)
        assert O.rel(d, ip[f"{tag}_d"]) < 1e-11
        w, dobs = ip[f"{tag}_w"], ip[f"{tag}_dobs"]
        g = 2.0 * w * w * (d - dobs) * scale
        grad = O.jtvec_3d(op, m, g) if three_d else O.jtvec_2d(op, m, g)
        assert O.rel(grad, ip[f"{tag}_grad"]) < 1e-10


def test_dcip_forward_matches_reference():
    """The joint non-linear DC + IP forward and misfit gradient of the oracle
    against the reference's TorchDCIP2D (dctorch/dcip2d.py) on the tiny 2-D
    problem, both DC states."""
    g = golden("dc2d_tiny")
    op = _ops(g, False)
    J = golden("dcip_tiny")
    n = J["m_rho"].size
    for state in ("total", "instantaneous"):
        mm = J[f"{state}_m"]
        eta = 0.8 / (1.0 + np.exp(-mm[n:]))
        d_dc, d_ip, _, _ = O.dcip_dpred_2d(op, mm[:n], eta, 1000.0, state)
        assert O.rel(d_dc, J[f"{state}_d_dc"]) < 1e-12
        assert O.rel(d_ip, J[f"{state}_d_ip"]) < 1e-10
        phi, grad = O.dcip_misfit_grad_2d(
            op, mm, 0.8, 1000.0, state, J[f"{state}_dobs_dc"], J[f"{state}_w_dc"],
            J[f"{state}_dobs_ip"], J[f"{state}_w_ip"], 0.7)
        assert abs(phi - J[f"{state}_phi"]) <= 1e-10 * abs(J[f"{state}_phi"])
        assert O.rel(grad, J[f"{state}_grad"]) < 1e-9


def test_cr_forward_matches_reference():
    """The complex-resistivity forward and misfit gradient of the oracle
    against the reference's TorchCR2D (dctorch/cr2d.py, complex SuperLU) on
    the tiny 2-D problem, both data conventions."""
    g = golden("dc2d_tiny")
    op = _ops(g, False)
    J = golden("cr_tiny")
    assert np.array_equal(J["wq"], g["wq"])
    n = J["m_rho"].size
    for datum in ("magnitude", "real"):
        mm = J[f"{datum}_m"]
        d_rho, d_ip = O.cr_dpred_2d(op, mm[:n], mm[n:], 1000.0, datum)
        assert O.rel(d_rho, J[f"{datum}_d_rho"]) < 1e-12
        assert O.rel(d_ip, J[f"{datum}_d_ip"]) < 1e-10
        phi, grad = O.cr_misfit_grad_2d(
            op, mm, 1000.0, datum, J[f"{datum}_dobs_rho"], J[f"{datum}_w_rho"],
            J[f"{datum}_dobs_ip"], J[f"{datum}_w_ip"], 0.7)
        assert abs(phi - J[f"{datum}_phi"]) <= 1e-10 * abs(J[f"{datum}_phi"])
        assert O.rel(grad, J[f"{datum}_grad"]) < 1e-9


def test_slab_lu_matches_superlu_real_and_complex():
    """The block-tridiagonal LU oracle solver against SuperLU on the tiny 2-D
    pattern, with complex-symmetric values (sigma (1 - i m)) and real ones,
    shared and per-system right-hand sides; and the complex-resistivity
    oracle with it equals the one on SuperLU."""
    from simpeg_dc_torch_b200 import synthetic as syn
    g = golden("dc2d_tiny")
    J = golden("cr_tiny")
    op = _ops(g, False)
    mesh, _, _ = syn.tiny_2d()
    slab = O.grid_slabs(mesh.node_grid_index())
    n = op["nN"]
    rng = np.random.default_rng(12)
    nC = op["Lstack"].shape[1]
    sig = np.exp(rng.uniform(-3, 1, nC))
    nnz = op["col"].size
    for vals in (op["Lstack"][:2 * nnz] @ sig,
                 op["Lstack"][:2 * nnz] @ sig - 1j * (op["Lstack"][:2 * nnz] @ (0.2 * sig))):
        V = vals.reshape(2, nnz)
        B = rng.standard_normal((n, 3)) + (1j * rng.standard_normal((n, 3))
                                          if np.iscomplexobj(V) else 0)
        a = O.SlabLUBatch(op["crow"], op["col"], n, slab)
        a.factorize(V)
        ref = O.SuperLUBatch(op["crow"], op["col"], n)
        ref.factorize(V)
        assert O.rel(a.solve(B), ref.solve(B)) < 1e-12
        Bb = np.stack([B, 2 * B])
        assert O.rel(a.solve(Bb), ref.solve(Bb)) < 1e-12
    n2 = J["m_rho"].size
    mm = J["magnitude_m"]
    d0 = O.cr_dpred_2d(op, mm[:n2], mm[n2:], 1000.0)
    op_s = dict(op, slab=slab)
    d1 = O.cr_dpred_2d(op_s, mm[:n2], mm[n2:], 1000.0)
    assert O.rel(d1[0], d0[0]) < 1e-12 and O.rel(d1[1], d0[1]) < 1e-11


def test_singularity_removal_matches_reference():
    """The oracle's singularity-removed 2.5-D forward and gradient against
    the reference's TorchDC2D(singularity_removal=True) (golden sr_tiny);
    the primary's background (model or fixed) cancels from the total field."""
    from simpeg_dc_torch_b200 import synthetic as syn
    g = golden("dc2d_tiny")
    S = golden("sr_tiny")
    op = _ops(g, False)
    mesh, survey, _ = syn.tiny_2d()
    widths = mesh.h_gridded
    poles, radii = [], []
    for src in survey.source_list:
        pl = [(src.location_a, 1.0)]
        if getattr(src, "location_b", None) is not None:
            pl.append((src.location_b, -1.0))
        poles.append(pl)
        radii.append([float(np.sqrt(np.prod(widths[int(mesh.point2index(
            np.asarray(loc, float)[None, :2])[0])]) / np.pi)) for loc, _ in pl])
    u1 = O.unit_primary_2d(mesh.nodes, S["kys"], poles, radii)
    m = S["m"]
    for tag in ("model", "fixed"):
        assert O.rel(O.dpred_2d_sr(op, m, u1), S[f"{tag}_dpred"]) < 1e-11
        phi, grad = O.misfit_grad_2d_sr(op, m, u1, S[f"{tag}_dobs"], S[f"{tag}_w"])
        assert abs(phi - S[f"{tag}_phi"]) <= 1e-10 * abs(S[f"{tag}_phi"])
        assert O.rel(grad, S[f"{tag}_grad"]) < 1e-9


def test_slab_solver_matches_superlu_and_reference():
    """The block-tridiagonal slab Cholesky (the oracle's solver for the large
    workloads) gives the reference's results on its golden problems and the
    SuperLU solution of a float64 system to rounding."""
    from simpeg_dc_torch_b200 import synthetic as syn
    for name, case, three_d in (("dc2d_tiny", syn.tiny_2d, False),
                                ("dc3d_tiny", syn.tiny_3d, True)):
        g = golden(name)
        mesh, _, _ = case()
        op = _ops(g, three_d)
        op["slab"] = O.grid_slabs(mesh.node_grid_index())
        assert op["slab"].size == op["nN"]
        m, dobs, w, v = g["m"], g["dobs"], g["w"], g["v"]
        dpred = O.dpred_3d if three_d else O.dpred_2d
        mgrad = O.misfit_grad_3d if three_d else O.misfit_grad_2d
        jtvec = O.jtvec_3d if three_d else O.jtvec_2d
        assert O.rel(dpred(op, m), g["dpred"]) < 1e-12
        phi, grad = mgrad(op, m, dobs, w)
        assert abs(phi - g["phi"]) <= 1e-12 * abs(g["phi"])
        assert O.rel(grad, g["grad"]) < 1e-11
        assert O.rel(jtvec(op, m, v), g["jtvec"]) < 1e-11
    # a shared right-hand side block and a batched one on one system
    mesh, survey, m = syn.tiny_3d()
    from simpeg_dc_torch_b200.operators import nodal_operators
    ops = nodal_operators(mesh, survey)
    vals = ops.L3() @ np.exp(-m)
    rng = np.random.default_rng(5)
    B = rng.standard_normal((ops.nN, 3))
    lu = O.SuperLUBatch(ops.crow, ops.col, ops.nN)
    lu.factorize(vals)
    sl = O.SlabCholeskyBatch(ops.crow, ops.col, ops.nN,
                             O.grid_slabs(mesh.node_grid_index()))
    sl.factorize(vals)
    assert O.rel(sl.solve(B), lu.solve(B)) < 1e-12
    assert O.rel(sl.solve(B[None]), lu.solve(B[None])) < 1e-12


def test_slab_solver_refuses_non_adjacent_couplings():
    crow = np.array([0, 2, 3, 5])
    col = np.array([0, 2, 1, 0, 2])
    import pytest
    with pytest.raises(ValueError):
        O.SlabCholeskyBatch(crow, col, 3, np.array([0, 1, 2]))
