"""Differentiable 2.5-D DC resistivity on a B200 (drop-in for dctorch's
`TorchDC2D`, dctorch/simulation2d.py:34-534).

The constructor, `dpred`, `misfit`, `misfit_and_grad` and `Jtvec` keep the
reference's signatures and results.  At build time the sigma-linear maps
L_ky, the sources q, the receiver projection Pd and the wavenumber quadrature
are assembled from the mesh (see `operators.py` and `quadrature.py`); at run
time the whole forward + adjoint chain runs in the hand-written CUDA kernels
of libdct (see `_fused.py`): all nky wavenumbers and all sources are factored
and solved in the same launches.

Precision: `dtype=torch.float64` (default) factors and solves in float64;
`dtype=torch.float32` factors and solves in float32 with float64 iterative
refinement (at most `refine` corrections, default 2, ending once the
estimated error of the fields is below `refine_tol`, default 1e-9: measured
on the 56,525-node workload, one correction leaves the gradient within
5e-8 of float64).  The quadrature sum, the data and the misfit are float64 in both.
Data come back in the model's dtype.

Singularity removal (`singularity_removal=True`, `rho_primary`) solves for
the field as the analytic half-space primary plus a smooth remainder (see
`primary.py`).  Not provided: SimPEG's own wavenumber fit
(`quadrature="simpeg"`), which needs SimPEG's optimizer run.
"""
from __future__ import annotations

import os

import numpy as np
import scipy.sparse as sp
import torch

from .primary import source_cells, unit_primary
from ._fused import FusedDpred, FusedPath
from .mesh import as_tensor_mesh
from .operators import nodal_operators
from .quadrature import (amplification, electrode_distance_range,
                         k0_quadrature, transform_error)


def _to_coo_tensor(M, device, dtype):
    M = sp.coo_matrix(M)
    return torch.sparse_coo_tensor(
        torch.as_tensor(np.vstack((M.row, M.col)), dtype=torch.int64,
                        device=device),
        torch.as_tensor(M.data, dtype=dtype, device=device),
        M.shape).coalesce()


class _ActiveCells:
    """m_full = P m + v_inactive (dctorch/simulation2d.py:122-134, 299-304)."""

    def __init__(self, active_cells, val_inactive, nC, device):
        act = np.asarray(active_cells, dtype=bool)
        if act.size != nC:
            raise ValueError("active_cells must have one entry per cell")
        self.idx = torch.as_tensor(np.where(act)[0], device=device)
        v = np.full(nC, float(val_inactive))
        v[act] = 0.0
        self.v = torch.as_tensor(v, dtype=torch.float64, device=device)
        self.nA = int(act.sum())

    def full(self, m):
        return self.v.to(m.dtype).index_add(0, self.idx, m)

    def inject(self, v):
        """P v: a perturbation of the active cells on the full mesh."""
        out = torch.zeros(self.v.numel(), dtype=v.dtype, device=v.device)
        return out.index_add(0, self.idx, v)

    def restrict(self, g_full):
        return g_full[self.idx]


class TorchDC2D:
    """Differentiable dpred/misfit for 2.5-D nodal DC on a fixed mesh+survey."""

    def __init__(self, mesh, survey, nky=12, device="cuda",
                 dtype=torch.float64, active_cells=None, val_inactive=None,
                 chunk=None, singularity_removal=False, rho_primary=None,
                 quadrature=None, refine=None, refine_fields=None,
                 refine_tol=None, leaf_size=64):
        if quadrature is None:
            quadrature = os.environ.get("DCTORCH_QUADRATURE", "electrodes")
        if isinstance(quadrature, str) and quadrature != "electrodes":
            raise NotImplementedError(
                f"quadrature={quadrature!r} needs SimPEG's own wavenumber fit; "
                "use 'electrodes' or pass (points, weights)")
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise NotImplementedError("TorchDC2D here runs on CUDA devices only")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.dtype = dtype
        self.chunk = None if chunk is None else int(chunk)
        self._sr = bool(singularity_removal)
        self._rho_p = None if rho_primary is None else float(rho_primary)

        rmin, rmax = electrode_distance_range(survey)
        if isinstance(quadrature, str):
            kys, wq, info = k0_quadrature(rmin, rmax, nky)
            self.quadrature_info = {
                "source": "electrodes", "r_range": (rmin, rmax),
                "max_rel_err": info["max_rel_err"],
                "amplification": info["amplification"],
                "n_used": info["n_used"]}
        else:
            kys, wq = (np.asarray(a, float) for a in quadrature)
            self.quadrature_info = {
                "source": "given", "r_range": (rmin, rmax),
                "max_rel_err": transform_error(kys, wq, rmin, rmax),
                "amplification": amplification(wq), "n_used": int(kys.size)}

        mesh = as_tensor_mesh(mesh)
        ops = nodal_operators(mesh, survey)
        self._ops = ops
        self.kys = np.asarray(kys, float)
        self.wq_np = np.asarray(wq, float)
        self.nC, self.nN, self.nS, self.nD = ops.nC, ops.nN, ops.nS, ops.nD
        self.nky = int(self.kys.size)
        self.nnzA = ops.nnzA
        L = sp.vstack([ops.L_ky(k) for k in self.kys]).tocsr()
        self._L = L
        self._check_symmetric(L)
        precision = "fp64" if dtype == torch.float64 else "fp32_ir"
        self.precision = precision
        self._path = FusedPath(ops.crow, ops.col, L, self.wq_np, ops.q, ops.Pd,
                               ops.sidx, self.device, precision,
                               coords=mesh.node_grid_index()
                               if hasattr(mesh, "node_grid_index") else None,
                               refine=refine, refine_fields=refine_fields,
                               leaf_size=leaf_size,
                               refine_tol=(1e-9 if refine_tol is None
                                           else refine_tol))
        self.solver = self._path.solver
        if self._sr:
            # fields by the split u = rho_s u_1 + u_s (primary.py); the
            # geometric primary and A(1) u_1 are formed once here
            self._path.set_primary(
                unit_primary(mesh, survey, self.kys),
                (L @ np.ones(self.nC)).reshape(self.nky, self.nnzA),
                source_cells(mesh, survey), self._rho_p)
        self.sidx = torch.as_tensor(ops.sidx, device=self.device)
        self.iD = torch.arange(self.nD, device=self.device)
        self.wq = torch.as_tensor(self.wq_np, dtype=torch.float64,
                                  device=self.device)
        self._inj = None
        if active_cells is not None:
            self._inj = _ActiveCells(active_cells, val_inactive, self.nC,
                                     self.device)
        self._mesh, self._survey = mesh, survey
        self._lstack = None

    # ------------------------------------------------------------ helpers
    def _check_symmetric(self, L):
        """The factorization is Cholesky: A must be symmetric for every ky
        (checked once at build time at a reference model)."""
        sig = np.full(self.nC, 0.01)
        v = L[:self.nnzA] @ sig
        A = sp.csr_matrix((v, self._ops.col, self._ops.crow),
                          shape=(self.nN, self.nN))
        if abs(A - A.T).max() > 1e-12 * abs(A).max():
            raise ValueError("assembled operator is not symmetric")

    @property
    def Lstack(self):
        """The stacked assembly map (nky*nnzA, nC) as a torch sparse tensor
        (the reference engine's attribute)."""
        if self._lstack is None:
            self._lstack = _to_coo_tensor(self._L, self.device, torch.float64)
        return self._lstack

    @property
    def q(self):
        return torch.as_tensor(self._ops.q.toarray(), dtype=torch.float64,
                               device=self.device)

    @property
    def Pd(self):
        return _to_coo_tensor(self._ops.Pd, self.device, torch.float64)

    def _model_to_full(self, m):
        m_loc = m.to(device=self.device, dtype=torch.float64).reshape(-1)
        if self._inj is not None:
            m_loc = self._inj.full(m_loc)
        return m_loc

    def _grad_to_model(self, g_full, m):
        g = g_full if self._inj is None else self._inj.restrict(g_full)
        return g.to(device=m.device, dtype=m.dtype)

    # ------------------------------------------------------------ runtime
    def dpred(self, m):
        """Predicted data (nD,) for m = log(rho). Autograd-traceable."""
        dev0, dt0 = m.device, m.dtype
        m_full = self._model_to_full(m)
        d = FusedDpred.apply(m_full, self._path)
        return d.to(device=dev0, dtype=dt0)

    def misfit(self, m, dobs, w):
        """phi_d = ||w*(dpred-dobs)||^2 (no 1/2 factor)."""
        r = w * (self.dpred(m) - dobs)
        return (r ** 2).sum()

    def misfit_and_grad(self, m, dobs, w, chunk=None):
        """(phi_d, dphi_d/dm) outside the autograd graph
        (dctorch/simulation2d.py:345-375).  All sources are solved against one
        factorization; `chunk` is accepted for compatibility."""
        with torch.no_grad():
            m_full = self._model_to_full(m)
            d, sigma, U, _ = self._path.forward(m_full)
            wd = w.to(self.device, torch.float64)
            r = wd * (d - dobs.to(self.device, torch.float64))
            phi = (r ** 2).sum()
            g = self._path.adjoint(2.0 * wd * r, U, sigma)
        return float(phi), self._grad_to_model(g, m)

    def Jtvec(self, m, v, chunk=None):
        """J^T v without forming J (dctorch/simulation2d.py:398-437)."""
        with torch.no_grad():
            m_full = self._model_to_full(m)
            _, sigma, U, _ = self._path.forward(m_full)
            g = self._path.adjoint(v.reshape(-1), U, sigma)
        return self._grad_to_model(g, m)

    # ------------------------------------------------ linearised products
    def _jac_rows(self, sigma, U, a, b):
        """Rows a..b of J as an (nM, b - a) block (active cells only)."""
        Jb = self._path.jac_block(a, b, sigma, U)
        return Jb if self._inj is None else Jb[self._inj.idx]

    def Jmatrix(self, m, block=32):
        """The explicit (nD, nM) Jacobian from one factorization
        (dctorch/simulation2d.py:439-518): the adjoint right-hand sides are the
        columns of Pd^T, solved `block` data at a time on the same factors.
        Returned outside the autograd graph on m's device and dtype."""
        self._plain_only("Jmatrix")
        block = max(1, min(int(block), self.nD, self._path.width))
        with torch.no_grad():
            m_full = self._model_to_full(m)
            _, sigma, U, _ = self._path.forward(m_full)
            J = torch.empty((self.nD, self._nM()), dtype=torch.float64,
                            device=self.device)
            for a in range(0, self.nD, block):
                b = min(a + block, self.nD)
                J[a:b] = self._jac_rows(sigma, U, a, b).T
        return J.to(device=m.device, dtype=m.dtype)

    def linearize(self, m, store_fields=None, fields_max_gib=2.0):
        """The forward frozen at m: one factorization, the fields kept, and
        J v / J^T v as one batched solve each (see `Linearization2D`)."""
        self._plain_only("linearize")
        return Linearization2D(self, m, store_fields=store_fields,
                               fields_max_gib=fields_max_gib)

    def _plain_only(self, what):
        if self._sr:
            raise NotImplementedError(
                f"{what} is built for the plain formulation only (as in "
                "dctorch/simulation2d.py:471-476, 572-577); with singularity "
                "removal use dpred, misfit, misfit_and_grad or Jtvec")

    def Jvec(self, m, v):
        """J v without forming J (dctorch/simulation2d.py:526-529)."""
        return self.linearize(m).Jvec(v)

    def _nM(self):
        return self.nC if self._inj is None else self._inj.nA

    def check(self):
        """Synchronise and raise if a kernel reported an error."""
        return self.solver.check()


class Linearization2D:
    """The 2.5-D forward frozen at one model, for Gauss-Newton
    (dctorch/simulation2d.py:537-818).

    The systems are factorized once and the fields U_k = A_k^{-1} q are kept
    on the device (when they fit `fields_max_gib`, otherwise re-solved from
    the stored factors for each product).  Then

        J v   :  A_k dU_k = -A_k(dsigma) U_k, dsigma = -sigma v;  J v = Pd sum_k w_k dU_k
        J^T v :  A_k Y_k = Pd^T v on the same factors; contraction with U_k, L^T, -sigma

    each one batched solve over all wavenumbers and sources.  `diag_JtDJ` and
    `Jmatrix` form rows of J `sub` data at a time (one adjoint solve per
    block) and never hold more than one block.  The solver is shared with the
    engine: if anything else refactorizes it (a line-search `dpred`), its
    stamp changes and this factorization is restored before the next product.
    """

    def __init__(self, eng, m, store_fields=None, fields_max_gib=2.0):
        self.eng = eng
        self.m_dtype, self.m_device = m.dtype, m.device
        path = eng._path
        with torch.no_grad():
            self.m_full = eng._model_to_full(m)
            self.sigma, self.vals = path.values(self.m_full)
            path.factorize(self.vals)
            self._stamp = path.solver.stamp
            U = path.fields()
            self.d = path.project(U).to(self.m_device, self.m_dtype)
        nbytes = U.numel() * U.element_size()
        if store_fields is None:
            store_fields = nbytes <= fields_max_gib * 2 ** 30
        self._U = U if store_fields else None
        self.width = path.width

    def _ensure(self):
        path = self.eng._path
        if path.solver.stamp != self._stamp:
            path.factorize(self.vals)
            self._stamp = path.solver.stamp

    def _fields(self):
        self._ensure()
        return self._U if self._U is not None else self.eng._path.fields()

    def _v_full(self, v):
        v = v.to(self.eng.device, torch.float64).reshape(-1)
        return v if self.eng._inj is None else self.eng._inj.inject(v)

    def _out(self, x):
        return x.to(self.m_device, self.m_dtype)

    @torch.no_grad()
    def Jvec(self, v):
        """J v, (nD,)."""
        U = self._fields()
        return self._out(self.eng._path.jvec(self._v_full(v), self.sigma, U))

    @torch.no_grad()
    def Jtvec(self, v):
        """J^T v, (nM,)."""
        U = self._fields()
        g = self.eng._path.adjoint(v.reshape(-1), U, self.sigma)
        return self._out(g if self.eng._inj is None else self.eng._inj.restrict(g))

    def _blocks(self, sub):
        nb = self.width if not sub else max(1, min(int(sub), self.width))
        U = self._fields()
        for a in range(0, self.eng.nD, nb):
            b = min(a + nb, self.eng.nD)
            yield a, b, self.eng._jac_rows(self.sigma, U, a, b)

    @torch.no_grad()
    def diag_JtDJ(self, dw, sub=None):
        """diag(J^T diag(dw) J), (nM,), exact, without storing J."""
        dw = dw.to(self.eng.device, torch.float64).reshape(-1)
        out = torch.zeros(self.eng._nM(), dtype=torch.float64, device=self.eng.device)
        for a, b, Jb in self._blocks(sub):
            out += (Jb ** 2) @ dw[a:b]
        return self._out(out)

    @torch.no_grad()
    def Jmatrix(self, sub=None):
        """The explicit J (nD, nM) from this linearization's factors and fields."""
        J = torch.empty((self.eng.nD, self.eng._nM()), dtype=torch.float64,
                        device=self.eng.device)
        for a, b, Jb in self._blocks(sub):
            J[a:b] = Jb.T
        return self._out(J)
