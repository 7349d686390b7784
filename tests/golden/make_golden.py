"""Generate the golden fixtures from the reference implementation itself.

Run in a container that holds the reference source tree:

    python tests/golden/make_golden.py --reference /path/to/SimPEG_DC_Torch

The reference's runtime modules (dctorch/solver.py, quadrature.py,
simulation2d.py, simulation3d.py) are loaded under a stub `dctorch` package
that skips dctorch/__init__.py (which imports SimPEG, absent here).  Engines
are made with `object.__new__` and given this package's operators; every
output below is computed by the reference's own code on its CPU (SuperLU)
path in float64:

  solver_nx12.npz / solver_nx40.npz : dctorch.solver.sparse_solve on the
      5-point Laplacian + 0.1 I of dctorch/tests/test_solver.py:19-25, with
      the value/rhs gradients of loss = sum(w * x).
  quad.npz        : dctorch.quadrature.k0_quadrature points and weights.
  dc2d_tiny.npz   : a 24x12-cell 2.5-D problem, all operators stored, with
      dpred, misfit, misfit gradient, Jtvec, chunked Jtvec and
      misfit_and_grad from TorchDC2D.
  dc2d_suite.npz  : the reference suite's 2-D tensor case
      (dctorch/tests/test_suite.py:65-67), outputs + operator checksums.
  dc2d_lin.npz    : on the dc2d_tiny problem, TorchDC2D.Jmatrix and Jvec,
      and Linearization2D's d, Jvec, Jtvec, diag_JtDJ and Jmatrix.
  dc3d_tiny.npz / dc3d_suite.npz : the same for TorchDC3D.
  ip_tiny.npz     : linearized IP (dctorch/ip2d.py TorchIP2D, ip3d.py
      TorchIP3D) on the tiny 2-D and 3-D problems with every other receiver
      of data type "apparent_chargeability": V_dc, the per-datum scale, the
      IP data and the misfit gradient with respect to eta.  The IP
      constructors build their DC engine themselves (which needs SimPEG);
      here that name is pointed at the stub engines above while they run.
  sr_tiny.npz     : TorchDC2D with singularity removal
      (dctorch/simulation2d.py:306-333 with dctorch/singularity.py) on the
      tiny 2-D problem, background from the model and fixed: dpred, misfit,
      its gradient, Jtvec, chunked Jtvec and misfit_and_grad.  The primary
      is kept in host memory (no CUDA here: pin_memory is skipped).
  cr_tiny.npz     : the complex-resistivity engine (dctorch/cr2d.py
      TorchCR2D, complex-symmetric systems on SciPyBatchSolver's complex
      SuperLU) on the tiny 2-D problem for both data conventions
      ("magnitude", "real"): the (rho, ip) data of a stacked (log-rho,
      chargeability) model and the gradient of its joint misfit.
  dcip_tiny.npz   : the joint non-linear DC + IP engine (dctorch/dcip2d.py
      TorchDCIP2D) on the tiny 2-D problem for both DC states: the DC and
      IP data of a stacked (log-rho, logit-eta) model and the gradient of
      its joint misfit.
"""
from __future__ import annotations

import argparse
import os
import sys
import types

import numpy as np
import scipy.sparse as sp
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from simpeg_dc_torch_b200 import synthetic as syn  # noqa: E402
from simpeg_dc_torch_b200.operators import nodal_operators  # noqa: E402
from simpeg_dc_torch_b200.quadrature import (  # noqa: E402
    electrode_distance_range)


def load_reference(root):
    pkg = types.ModuleType("dctorch")
    pkg.__path__ = [os.path.join(root, "dctorch")]
    sys.modules["dctorch"] = pkg
    import dctorch.quadrature as Q
    import dctorch.simulation2d as S2
    import dctorch.simulation3d as S3
    import dctorch.solver as S
    return S, Q, S2, S3


def laplacian(nx):
    T = sp.diags([-1.0, 2.0, -1.0], [-1, 0, 1], shape=(nx, nx))
    I = sp.eye(nx)
    A = (sp.kron(I, T) + sp.kron(T, I) + 0.1 * sp.eye(nx * nx)).tocsr()
    A.sort_indices()
    return A


def solver_fixture(S, nx, n_rhs, seed):
    A = laplacian(nx)
    n = A.shape[0]
    rng = np.random.default_rng(seed)
    b = rng.standard_normal((n, n_rhs))
    w = rng.standard_normal((n, n_rhs))
    slv = S.SciPySolver(torch.tensor(A.indptr, dtype=torch.int32),
                        torch.tensor(A.indices, dtype=torch.int32), n, n_rhs)
    vals = torch.tensor(A.data, requires_grad=True)
    bt = torch.tensor(b, requires_grad=True)
    x = S.sparse_solve(vals, bt, slv)
    (torch.tensor(w) * x).sum().backward()
    return dict(crow=A.indptr.astype(np.int32), col=A.indices.astype(np.int32),
                vals=A.data, b=b, w=w, x=x.detach().numpy(),
                grad_vals=vals.grad.numpy(), grad_b=bt.grad.numpy())


def engine_2d(S2, ops, kys, wq, chunk=None):
    L = sp.vstack([ops.L_ky(k) for k in kys]).tocoo()
    eng = object.__new__(S2.TorchDC2D)
    dev, dt = torch.device("cpu"), torch.float64
    eng.device, eng.dtype, eng.chunk = dev, dt, chunk
    eng._sr, eng._P_inj, eng._primary = False, None, None
    eng.kys = np.asarray(kys)
    eng.nC, eng.nN, eng.nS, eng.nD = ops.nC, ops.nN, ops.nS, ops.nD
    eng.nky, eng.nnzA = len(kys), ops.nnzA
    eng.Lstack = torch.sparse_coo_tensor(
        torch.tensor(np.vstack((L.row, L.col)), dtype=torch.int64),
        torch.tensor(L.data), L.shape).coalesce()
    eng.wq = torch.tensor(np.asarray(wq))
    eng.q = torch.tensor(ops.q.toarray())
    Pd = ops.Pd.tocoo()
    eng.Pd = torch.sparse_coo_tensor(
        torch.tensor(np.vstack((Pd.row, Pd.col)), dtype=torch.int64),
        torch.tensor(Pd.data), Pd.shape).coalesce()
    eng.sidx = torch.tensor(ops.sidx)
    eng.iD = torch.arange(ops.nD)
    eng._crow = torch.tensor(ops.crow, dtype=torch.int32)
    eng._ccol = torch.tensor(ops.col, dtype=torch.int32)
    eng._solvers = {}
    eng._PdT = eng._PdTs = eng._PinjT = None
    eng.solver = eng._solver_for(ops.nS)
    return eng, sp.csr_matrix(L)


def engine_3d(S3, S, ops):
    L3 = ops.L3()
    eng = object.__new__(S3.TorchDC3D)
    eng.device, eng.dtype = torch.device("cpu"), torch.float64
    eng._P_inj = eng._P_injt = None

    def s2t(M):
        M = sp.csr_matrix(M)
        M.sort_indices()
        return torch.sparse_csr_tensor(
            torch.tensor(M.indptr, dtype=torch.int32),
            torch.tensor(M.indices, dtype=torch.int32),
            torch.tensor(M.data), size=M.shape)
    eng.nC, eng.nN, eng.nS, eng.nD = ops.nC, ops.nN, ops.nS, ops.nD
    eng.nnzA = ops.nnzA
    eng.L3 = s2t(L3)
    eng.L3t = s2t(L3.T)
    eng.q = torch.tensor(ops.q.toarray())
    eng.Pd = s2t(ops.Pd)
    eng.sidx = torch.tensor(ops.sidx)
    eng.iD = torch.arange(ops.nD)
    eng.solver = S.make_solver(torch.tensor(ops.crow, dtype=torch.int32),
                               torch.tensor(ops.col, dtype=torch.int32),
                               ops.nN, ops.nS, device="cpu")
    return eng, L3


def run_engine(eng, m, dobs, w, v, two_d):
    mt = torch.tensor(m, requires_grad=True)
    phi = eng.misfit(mt, torch.tensor(dobs), torch.tensor(w))
    phi.backward()
    out = dict(phi=float(phi), grad=mt.grad.numpy().copy())
    with torch.no_grad():
        out["dpred"] = eng.dpred(torch.tensor(m)).numpy()
    out["jtvec"] = eng.Jtvec(torch.tensor(m), torch.tensor(v)).numpy()
    if two_d:
        ch = max(1, eng.nS // 3)
        out["jtvec_chunk"] = eng.Jtvec(torch.tensor(m), torch.tensor(v),
                                       chunk=ch).numpy()
        f, g = eng.misfit_and_grad(torch.tensor(m), torch.tensor(dobs),
                                   torch.tensor(w), chunk=ch)
        out["mag_phi"] = float(f)
        out["mag_grad"] = g.numpy()
        out["chunk"] = ch
    return out


def data_vectors(eng, m, seed):
    rng = np.random.default_rng(seed)
    with torch.no_grad():
        d = eng.dpred(torch.tensor(m)).numpy()
    dobs, w = syn.observed(d, rng, 0.05)
    v = rng.standard_normal(d.size)
    return dobs, w, v


def checksums(ops):
    return dict(ck_Ledge=float(np.abs(ops.L_edge.data).sum()),
                ck_Lnode=float(np.abs(ops.L_node.data).sum()),
                ck_bc=float(np.abs(ops.L_bc(0.1).data).sum()),
                ck_q=float(np.abs(ops.q.data).sum()),
                ck_Pd=float(np.abs(ops.Pd.data).sum()),
                nnzA=ops.nnzA, nN=ops.nN, nC=ops.nC)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True)
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    S, Q, S2, S3 = load_reference(a.reference)
    out = a.out

    np.savez_compressed(os.path.join(out, "solver_nx12.npz"),
                        **solver_fixture(S, 12, 3, 1))
    np.savez_compressed(os.path.join(out, "solver_nx40.npz"),
                        **solver_fixture(S, 40, 5, 0))

    qd = {}
    for i, (lo, hi, n) in enumerate([(5.0, 120.0, 11), (5.0, 120.0, 7),
                                     (2.0, 90.0, 12), (1.0, 60.0, 5)]):
        p, w, info = Q.k0_quadrature(lo, hi, n)
        qd[f"args{i}"] = np.array([lo, hi, n])
        qd[f"pts{i}"] = p
        qd[f"wts{i}"] = w
        qd[f"err{i}"] = info["max_rel_err"]
    np.savez_compressed(os.path.join(out, "quad.npz"), **qd)

    for name, (mesh, survey, m), nky, store_ops in [
            ("dc2d_tiny", syn.tiny_2d(), 7, True),
            ("dc2d_suite", syn.suite_case("2d-tensor"), 11, False)]:
        ops = nodal_operators(mesh, survey)
        rmin, rmax = electrode_distance_range(survey)
        kys, wq, _ = Q.k0_quadrature(rmin, rmax, nky)
        eng, L = engine_2d(S2, ops, kys, wq)
        dobs, w, v = data_vectors(eng, m, 21)
        res = run_engine(eng, m, dobs, w, v, True)
        rec = dict(m=m, dobs=dobs, w=w, v=v, kys=kys, wq=wq, **res,
                   **checksums(ops))
        if store_ops:
            rec.update(L_indptr=L.indptr, L_indices=L.indices, L_data=L.data,
                       crow=ops.crow, col=ops.col, Q=ops.q.toarray(),
                       Pd_indptr=ops.Pd.indptr, Pd_indices=ops.Pd.indices,
                       Pd_data=ops.Pd.data, sidx=ops.sidx)
        np.savez_compressed(os.path.join(out, name + ".npz"), **rec)
        print(name, "nN", ops.nN, "nD", ops.nD, "nky", len(kys))

    # linearised products of the 2.5-D engine on the tiny problem (its
    # operators are stored in dc2d_tiny.npz): TorchDC2D.Jmatrix / Jvec and
    # Linearization2D.Jvec / Jtvec / diag_JtDJ / Jmatrix
    mesh, survey, m = syn.tiny_2d()
    ops = nodal_operators(mesh, survey)
    rmin, rmax = electrode_distance_range(survey)
    kys, wq, _ = Q.k0_quadrature(rmin, rmax, 7)
    eng, _ = engine_2d(S2, ops, kys, wq)
    rng = np.random.default_rng(23)
    u = rng.standard_normal(ops.nC)
    v = rng.standard_normal(ops.nD)
    dw = rng.uniform(0.5, 2.0, ops.nD)
    mt = torch.tensor(m)
    rec = dict(m=m, u=u, v=v, dw=dw)
    rec["jmatrix"] = eng.Jmatrix(mt, block=5).numpy()
    rec["jvec"] = eng.Jvec(mt, torch.tensor(u)).numpy()
    lin = eng.linearize(mt)
    rec["lin_d"] = lin.d.numpy()
    rec["lin_jvec"] = lin.Jvec(torch.tensor(u)).numpy()
    rec["lin_jtvec"] = lin.Jtvec(torch.tensor(v)).numpy()
    rec["lin_diag"] = lin.diag_JtDJ(torch.tensor(dw), sub=3).numpy()
    rec["lin_jmatrix"] = lin.Jmatrix(sub=4).numpy()
    np.savez_compressed(os.path.join(out, "dc2d_lin.npz"), **rec)
    print("dc2d_lin", rec["jmatrix"].shape)

    for name, (mesh, survey, m), store_ops in [
            ("dc3d_tiny", syn.tiny_3d(), True),
            ("dc3d_suite", syn.suite_case("3d-tensor"), False)]:
        ops = nodal_operators(mesh, survey)
        eng, L3 = engine_3d(S3, S, ops)
        dobs, w, v = data_vectors(eng, m, 22)
        res = run_engine(eng, m, dobs, w, v, False)
        rec = dict(m=m, dobs=dobs, w=w, v=v, **res, **checksums(ops))
        if store_ops:
            rec.update(L_indptr=L3.indptr, L_indices=L3.indices,
                       L_data=L3.data, crow=ops.crow, col=ops.col,
                       Q=ops.q.toarray(), Pd_indptr=ops.Pd.indptr,
                       Pd_indices=ops.Pd.indices, Pd_data=ops.Pd.data,
                       sidx=ops.sidx)
        np.savez_compressed(os.path.join(out, name + ".npz"), **rec)
        print(name, "nN", ops.nN, "nD", ops.nD)

    np.savez_compressed(os.path.join(out, "ip_tiny.npz"),
                        **ip_fixture(a.reference, S, Q, S2, S3))
    np.savez_compressed(os.path.join(out, "dcip_tiny.npz"), **dcip_fixture(S, Q, S2))
    np.savez_compressed(os.path.join(out, "cr_tiny.npz"), **cr_fixture(S, Q, S2))
    np.savez_compressed(os.path.join(out, "sr_tiny.npz"), **sr_fixture(Q, S2))


def mark_chargeability(survey):
    """Every other receiver (in survey order) becomes an apparent-
    chargeability receiver; returns the per-receiver flags."""
    flags = []
    for src in survey.source_list:
        for rx in src.receiver_list:
            if len(flags) % 2 == 1:
                rx.data_type = "apparent_chargeability"
            flags.append(rx.data_type == "apparent_chargeability")
    return np.array(flags)


def ip_fixture(root, S, Q, S2, S3):
    import dctorch.ip2d as I2
    import dctorch.ip3d as I3
    rec = {}
    for tag, (mesh, survey, m) in (("2d", syn.tiny_2d()), ("3d", syn.tiny_3d())):
        flags = mark_chargeability(survey)
        ops = nodal_operators(mesh, survey)
        if tag == "2d":
            rmin, rmax = electrode_distance_range(survey)
            kys, wq, _ = Q.k0_quadrature(rmin, rmax, 7)
            eng, _ = engine_2d(S2, ops, kys, wq)
            saved, S2.TorchDC2D = S2.TorchDC2D, (lambda *a, **k: eng)
            try:
                ip = I2.TorchIP2D(mesh, survey, m, nky=7, device="cpu",
                                  dtype=torch.float64, quadrature=(kys, wq))
            finally:
                S2.TorchDC2D = saved
            rec.update(kys=kys, wq=wq)
        else:
            eng, _ = engine_3d(S3, S, ops)
            saved, S3.TorchDC3D = S3.TorchDC3D, (lambda *a, **k: eng)
            try:
                ip = I3.TorchIP3D(mesh, survey, m, device="cpu", dtype=torch.float64)
            finally:
                S3.TorchDC3D = saved
        rng = np.random.default_rng(31)
        eta = rng.uniform(0.0, 0.1, ops.nC)
        with torch.no_grad():
            d = ip.dpred(torch.tensor(eta)).numpy()
        dobs = d * (1.0 + 0.05 * rng.standard_normal(d.size))
        w = 1.0 / (0.05 * np.abs(dobs) + 1e-3 * np.abs(dobs).max())
        et = torch.tensor(eta, requires_grad=True)
        phi = ip.misfit(et, torch.tensor(dobs), torch.tensor(w))
        phi.backward()
        rec.update({f"{tag}_m": m, f"{tag}_flags": flags, f"{tag}_eta": eta,
                    f"{tag}_dobs": dobs, f"{tag}_w": w,
                    f"{tag}_vdc": ip.v_dc.numpy(), f"{tag}_scale": ip._scale.numpy(),
                    f"{tag}_d": d, f"{tag}_phi": float(phi),
                    f"{tag}_grad": et.grad.numpy()})
        print("ip", tag, "nD", d.size, "chargeability data",
              int((ip._scale.numpy() != 1.0).sum()))
    return rec


def sr_fixture(Q, S2):
    mesh, survey, m = syn.tiny_2d()
    ops = nodal_operators(mesh, survey)
    rmin, rmax = electrode_distance_range(survey)
    kys, wq, _ = Q.k0_quadrature(rmin, rmax, 7)
    rec = dict(kys=kys, wq=wq, m=m)
    pin = torch.Tensor.pin_memory
    torch.Tensor.pin_memory = lambda self, *a, **k: self
    try:
        for tag, rho_p in (("model", None), ("fixed", 50.0)):
            eng, _ = engine_2d(S2, ops, kys, wq)
            eng._sr, eng._rho_p, eng._mesh, eng._survey = True, rho_p, mesh, survey
            dobs, w, v = data_vectors(eng, m, 51)
            res = run_engine(eng, m, dobs, w, v, True)
            rec.update({f"{tag}_{k}": x for k, x in
                        dict(dobs=dobs, w=w, v=v, **res).items()})
            print("sr", tag, "nD", dobs.size)
    finally:
        torch.Tensor.pin_memory = pin
    return rec


def dcip_fixture(S, Q, S2):
    import dctorch.dcip2d as D2
    mesh, survey, m = syn.tiny_2d()
    ops = nodal_operators(mesh, survey)
    rmin, rmax = electrode_distance_range(survey)
    kys, wq, _ = Q.k0_quadrature(rmin, rmax, 7)
    rec = dict(kys=kys, wq=wq, m_rho=m)
    for state in ("total", "instantaneous"):
        eng, _ = engine_2d(S2, ops, kys, wq)
        saved, S2.TorchDC2D = S2.TorchDC2D, (lambda *a, **k: eng)
        try:
            dcip = D2.TorchDCIP2D(mesh, survey, nky=7, device="cpu",
                                  dtype=torch.float64, eta_max=0.8,
                                  ip_scale=1000.0, dc_state=state,
                                  quadrature=(kys, wq))
        finally:
            S2.TorchDC2D = saved
        rng = np.random.default_rng(41)
        eta = rng.uniform(0.02, 0.3, ops.nC)
        mm = np.concatenate([m, dcip.m_eta_of(eta)])
        with torch.no_grad():
            d_dc, d_ip = (x.numpy() for x in dcip.dpred(torch.tensor(mm)))
        dobs_dc = d_dc * (1.0 + 0.03 * rng.standard_normal(d_dc.size))
        w_dc = 1.0 / (0.03 * np.abs(dobs_dc) + 1e-3 * np.abs(dobs_dc).max())
        dobs_ip = d_ip + 2.0 * rng.standard_normal(d_ip.size)
        w_ip = np.full(d_ip.size, 0.5)
        mt = torch.tensor(mm, requires_grad=True)
        phi = dcip.misfit(mt, torch.tensor(dobs_dc), torch.tensor(w_dc),
                          torch.tensor(dobs_ip), torch.tensor(w_ip), lam=0.7)
        phi.backward()
        rec.update({f"{state}_m": mm, f"{state}_d_dc": d_dc, f"{state}_d_ip": d_ip,
                    f"{state}_dobs_dc": dobs_dc, f"{state}_w_dc": w_dc,
                    f"{state}_dobs_ip": dobs_ip, f"{state}_w_ip": w_ip,
                    f"{state}_phi": float(phi), f"{state}_grad": mt.grad.numpy()})
        print("dcip", state, "nD", d_dc.size, "max d_ip", float(np.abs(d_ip).max()))
    return rec


def cr_fixture(S, Q, S2):
    import dctorch.cr2d as C2
    mesh, survey, m = syn.tiny_2d()
    ops = nodal_operators(mesh, survey)
    rmin, rmax = electrode_distance_range(survey)
    kys, wq, _ = Q.k0_quadrature(rmin, rmax, 7)
    rec = dict(kys=kys, wq=wq, m_rho=m)
    rng = np.random.default_rng(43)
    chg = rng.uniform(0.01, 0.2, ops.nC)
    for datum in ("magnitude", "real"):
        eng, _ = engine_2d(S2, ops, kys, wq)
        saved, S2.TorchDC2D = S2.TorchDC2D, (lambda *a, **k: eng)
        try:
            cr = C2.TorchCR2D(mesh, survey, nky=7, device="cpu",
                              dtype=torch.complex128, ip_scale=1000.0,
                              dc_datum=datum, quadrature=(kys, wq))
        finally:
            S2.TorchDC2D = saved
        mm = np.concatenate([m, chg])
        with torch.no_grad():
            d_r, d_i = (x.numpy() for x in cr.dpred(torch.tensor(mm)))
        dobs_r = d_r * (1.0 + 0.03 * rng.standard_normal(d_r.size))
        w_r = 1.0 / (0.03 * np.abs(dobs_r) + 1e-3 * np.abs(dobs_r).max())
        dobs_i = d_i + 2.0 * rng.standard_normal(d_i.size)
        w_i = np.full(d_i.size, 0.5)
        mt = torch.tensor(mm, requires_grad=True)
        phi = cr.misfit(mt, torch.tensor(dobs_r), torch.tensor(w_r),
                        torch.tensor(dobs_i), torch.tensor(w_i), lam=0.7)
        phi.backward()
        rec.update({f"{datum}_m": mm, f"{datum}_d_rho": d_r, f"{datum}_d_ip": d_i,
                    f"{datum}_dobs_rho": dobs_r, f"{datum}_w_rho": w_r,
                    f"{datum}_dobs_ip": dobs_i, f"{datum}_w_ip": w_i,
                    f"{datum}_phi": float(phi), f"{datum}_grad": mt.grad.numpy()})
        print("cr", datum, "nD", d_r.size, "max |d_ip|", float(np.abs(d_i).max()))
    return rec


if __name__ == "__main__":
    main()
