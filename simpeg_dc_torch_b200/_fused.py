"""The fused forward + adjoint path shared by the 2.5-D and 3-D engines.

One call of `forward` runs, on the engine's CUDA stream,

    sigma = exp(-m);  VALS = L sigma                  (dct_sigma_values)
    factor every system                               (dct_factorize)
    U = A^{-1} Q for all sources, all systems         (dct_scatter_rhs + dct_solve_permuted)
    d_i = sum_k w_k (Pd U_k)[i, sidx_i]               (dct_project_data)

and `adjoint(gd)` the reverse pass for dL/dd = gd on the same factors,

    R = Pd^T G (scattered into source columns)        (dct_scatter_rhs)
    Y = A^{-1} R                                      (dct_solve_permuted)
    gv[k, e] = -w_k sum_s Y_k[row_e, s] U_k[col_e, s] (dct_gather_contract)
    dL/dm = -sigma * (L^T gv)                         (dct_values_vjp)

which is the chain the reference builds from torch ops and cuDSS calls
(dctorch/simulation2d.py:378-396 with solver.py:236-281; simulation3d.py:
197-207).  Fields stay in the solver's permuted row order on the device.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import torch

from . import _native as nat
from .solver import DCTBatchSolver, _stream_ptr


def _csr64(M: sp.csr_matrix, device):
    M = sp.csr_matrix(M)
    M.sum_duplicates()
    M.sort_indices()
    return (torch.as_tensor(M.indptr.astype(np.int64), device=device),
            torch.as_tensor(M.indices.astype(np.int32), device=device),
            torch.as_tensor(M.data.astype(np.float64), device=device))


class FusedPath:
    """Device operators + solver for one mesh/survey.

    L      : (nbatch*nnzA, nC) assembly map (scipy CSR), system k in rows
             k*nnzA .. (k+1)*nnzA
    w      : per-system weights of the data sum (None: all ones)
    Q      : (nN, nS) scipy sparse sources;  Pd (nD, nN) CSR; sidx (nD,)
    """

    def __init__(self, crow, col, L, w, Q, Pd, sidx, device, precision,
                 coords=None, refine=None, n_rhs=None, refine_fields=None,
                 refine_tol=None, tuning=None, leaf_size=64, refine_tol_fields=None):
        self.device = device
        nN = crow.size - 1
        self.nN, self.nnzA = nN, col.size
        self.nbatch = L.shape[0] // self.nnzA
        self.nC = L.shape[1]
        self.nS = Q.shape[1]
        self.nD = Pd.shape[0]
        dt = torch.float64 if precision == "fp64" else torch.float32
        self.width = int(n_rhs or self.nS)
        self._pri = None      # singularity-removal split (set_primary)
        self.solver = DCTBatchSolver(crow, col, nN, self.width, self.nbatch,
                                     device=device, dtype=dt, coords=coords,
                                     refine=refine, refine_tol=refine_tol,
                                     tuning=tuning, leaf_size=leaf_size)
        plan = self.solver.plan
        self._plan = plan
        # float32 plans: most refinement corrections of the forward and of
        # the adjoint fields (each stops early at the plan's tolerance).  The
        # gradient contracts both fields at every node, so their errors
        # reach it amplified (measured on the 3-D benchmark: fields at
        # 1e-10 give a gradient within 3e-6 of float64, at 5e-12 within 3e-9).
        self.refine_adj = self.solver.refine
        # with record_refinement set, every solve of the path synchronises
        # and keeps its refinement record in last_refinement (diagnostics)
        self.record_refinement = False
        self.last_refinement = {}
        self.refine_fields = (self.refine_adj if refine_fields is None
                              else int(refine_fields))
        # stopping tolerances of the forward-field and of the adjoint
        # solves (0: a fixed number of corrections)
        self.tol_adj = self.solver.refine_tol
        self.tol_fields = self.tol_adj if refine_tol_fields is None else float(refine_tol_fields)
        self._iperm_ptr = plan.d_iperm
        perm = self.solver._sym.array("perm")
        iperm = np.empty_like(perm)
        iperm[perm] = np.arange(perm.size, dtype=perm.dtype)
        self.iperm_host = iperm
        self.iperm_d = torch.as_tensor(iperm.astype(np.int64), device=device)
        self.L_ptr, self.L_col, self.L_val = _csr64(L, device)
        self.Lt_ptr, self.Lt_col, self.Lt_val = _csr64(sp.csr_matrix(L.T), device)
        self.w = None if w is None else torch.as_tensor(
            np.asarray(w, float), device=device)
        self.row_e = self.solver.row
        self.col_e = self.solver.col
        # sources: one pair per nonzero (node, source)
        Qc = sp.coo_matrix(Q)
        self._q = self._pairs(iperm[Qc.row], Qc.col,
                              [[(0, v)] for v in Qc.data])
        # receivers: CSR of Pd and the adjoint pairs (node, source) <- data
        Pd = sp.csr_matrix(Pd)
        Pd.sort_indices()
        self.Pd_ptr = torch.as_tensor(Pd.indptr.astype(np.int32), device=device)
        self.Pd_col = torch.as_tensor(Pd.indices.astype(np.int32), device=device)
        self.Pd_val = torch.as_tensor(Pd.data.astype(np.float64), device=device)
        self.Pd_indptr = Pd.indptr.astype(np.int64)
        self.Pd_row = torch.as_tensor(
            np.repeat(np.arange(Pd.shape[0]), np.diff(Pd.indptr)).astype(np.int64),
            device=device)
        self.sidx = np.asarray(sidx, dtype=np.int64)
        self.sidx_d = torch.as_tensor(self.sidx.astype(np.int32), device=device)
        groups = {}
        Pc = Pd.tocoo()
        for i, j, v in zip(Pc.row, Pc.col, Pc.data):
            key = (int(iperm[j]), int(self.sidx[i]))
            groups.setdefault(key, []).append((int(i), float(v)))
        keys = sorted(groups)
        self._adj = self._pairs(np.array([k[0] for k in keys], dtype=np.int64),
                                np.array([k[1] for k in keys], dtype=np.int64),
                                [groups[k] for k in keys])

    def _pairs(self, rows, srcs, lists):
        ptr = np.zeros(len(lists) + 1, dtype=np.int64)
        ptr[1:] = np.cumsum([len(x) for x in lists])
        datum = np.array([d for x in lists for d, _ in x], dtype=np.int32)
        coef = np.array([c for x in lists for _, c in x], dtype=np.float64)
        dev = self.device
        return dict(n=len(lists),
                    ptr=torch.as_tensor(ptr, device=dev),
                    row=torch.as_tensor(np.asarray(rows, np.int32), device=dev),
                    src=torch.as_tensor(np.asarray(srcs, np.int32), device=dev),
                    datum=torch.as_tensor(datum, device=dev),
                    coef=torch.as_tensor(coef, device=dev))

    # ------------------------------------------------------------ kernels
    def _st(self):
        return _stream_ptr(self.device)

    def values(self, m_full):
        """sigma, VALS (nbatch, nnzA) for the full-mesh log-resistivity."""
        m = m_full.detach().to(self.device, torch.float64).contiguous()
        sigma = torch.empty(self.nC, dtype=torch.float64, device=self.device)
        vals = torch.empty(self.nbatch * self.nnzA, dtype=torch.float64,
                           device=self.device)
        nat.check(nat.lib().dct_sigma_values(
            vals.numel(), self.L_ptr.data_ptr(), self.L_col.data_ptr(),
            self.L_val.data_ptr(), self.nC, m.data_ptr(), sigma.data_ptr(),
            vals.data_ptr(), self._st()), "dct_sigma_values")
        return sigma, vals.view(self.nbatch, self.nnzA)

    def factorize(self, vals):
        self.solver.factorize(vals)

    def _scatter(self, pairs, g, k):
        dst = torch.empty((self.nN, k), dtype=torch.float64, device=self.device)
        nat.check(nat.lib().dct_scatter_rhs(
            self.nN, k, pairs["n"], pairs["ptr"].data_ptr(),
            pairs["row"].data_ptr(), pairs["src"].data_ptr(),
            pairs["datum"].data_ptr(), pairs["coef"].data_ptr(),
            None if g is None else g.data_ptr(), dst.data_ptr(), self._st()),
            "dct_scatter_rhs")
        return dst

    def _solve_perm(self, rhs_shared, k):
        x = torch.empty((self.nbatch, self.nN, k), dtype=torch.float64,
                        device=self.device)
        self._plan.solve_permuted(rhs_shared.data_ptr(), 0, k, x.data_ptr(),
                                  self._st())
        return x

    def _set_refinement(self, iters, tol):
        self._plan.set_refinement(iters)
        self._plan.set_refinement_tolerance(tol)

    def _record(self, what):
        if self.record_refinement and self.solver.dtype == torch.float32:
            self.last_refinement[what] = self.solver.refinement_info()

    def fields(self):
        """U = A^{-1} Q, permuted (nbatch, nN, nS)."""
        self._set_refinement(self.refine_fields, self.tol_fields)
        U = self._solve_perm(self._scatter(self._q, None, self.nS), self.nS)
        self._record("fields")
        return U

    # ------------------------------------------------ singularity removal
    def set_primary(self, u1, vals_one, src_cell, rho_fixed=None):
        """Use the split u = rho_s u_1 + u_s (see primary.py) for the fields
        of `forward`: u1 (nbatch, nN, nS) unit primary in node order,
        vals_one (nbatch, nnzA) the system values at unit conductivity,
        src_cell (nS,) the cell of each source's A electrode, rho_fixed an
        optional fixed background."""
        X = torch.empty((self.nbatch, self.nN, self.nS), dtype=torch.float64,
                        device=self.device)
        X[:, self.iperm_d, :] = torch.as_tensor(np.asarray(u1, float), device=self.device)
        X = X.contiguous()
        v1 = torch.as_tensor(np.asarray(vals_one, float).reshape(-1),
                             device=self.device).contiguous()
        # A(1) u_1 depends on nothing but the geometry: formed once
        R1 = self._pattern_product(v1, X, 1.0)
        self._pri = dict(X=X, R1=R1,
                         cell=torch.as_tensor(np.asarray(src_cell, np.int64),
                                              device=self.device),
                         fixed=None if rho_fixed is None else float(rho_fixed))

    def _pattern_product(self, vals, X, alpha):
        """alpha A(vals) X for every system, X and the result permuted."""
        Y = torch.empty_like(X)
        nat.check(nat.lib().dct_pattern_spmm(
            self.nbatch, self.nN, X.shape[-1], self.solver.crow.data_ptr(),
            self.col_e.data_ptr(), self._iperm_ptr, vals.data_ptr(), self.nnzA,
            float(alpha), X.data_ptr(), Y.data_ptr(), self._st()), "dct_pattern_spmm")
        return Y

    def _fields_split(self, m_full, vals):
        """U = rho_s u_1 + A^{-1} (A(1) u_1 - A(sigma) rho_s u_1), permuted."""
        p = self._pri
        if p["fixed"] is not None:
            rho = torch.full((self.nS,), p["fixed"], dtype=torch.float64, device=self.device)
        else:
            rho = torch.exp(m_full.detach().to(self.device, torch.float64)[p["cell"]])
        Xs = (p["X"] * rho.view(1, 1, -1)).contiguous()
        rhs = p["R1"] + self._pattern_product(vals.reshape(-1).contiguous(), Xs, -1.0)
        self._set_refinement(self.refine_fields, self.tol_fields)
        Us = torch.empty_like(rhs)
        self._plan.solve_permuted(rhs.data_ptr(), 1, self.nS, Us.data_ptr(), self._st())
        self._record("fields")
        return Xs + Us

    def project(self, U):
        d = torch.empty(self.nD, dtype=torch.float64, device=self.device)
        nat.check(nat.lib().dct_project_data(
            self.nbatch, self.nN, U.shape[-1], self.nD, self.Pd_ptr.data_ptr(),
            self.Pd_col.data_ptr(), self.Pd_val.data_ptr(),
            self.sidx_d.data_ptr(), self._iperm_ptr,
            None if self.w is None else self.w.data_ptr(), U.data_ptr(),
            d.data_ptr(), self._st()), "dct_project_data")
        return d

    def forward(self, m_full):
        """(d, sigma, U, stamp): data, conductivity, permuted fields and the
        solver stamp of the factorization they were computed with."""
        sigma, vals = self.values(m_full)
        self.factorize(vals)
        U = self.fields() if self._pri is None else self._fields_split(m_full, vals)
        d = self.project(U)
        return d, sigma, U, self.solver.stamp

    def ensure_factors(self, m_full, stamp):
        """Refactorize at m_full if another call replaced the factors."""
        if self.solver.stamp != stamp:
            self.factorize(self.values(m_full)[1])
        return self.solver.stamp

    def adjoint(self, gd, U, sigma):
        """dL/dm_full for dL/dd = gd on the current factorization."""
        g = gd.detach().to(self.device, torch.float64).contiguous()
        R = self._scatter(self._adj, g, self.nS)
        self._set_refinement(self.refine_adj, self.tol_adj)
        Y = self._solve_perm(R, self.nS)
        self._record("adjoint")
        gv = torch.empty(self.nbatch * self.nnzA, dtype=torch.float64,
                         device=self.device)
        nat.check(nat.lib().dct_gather_contract(
            self.nbatch, self.nN, self.nnzA, self.nS, self.row_e.data_ptr(),
            self.col_e.data_ptr(), self._iperm_ptr,
            None if self.w is None else self.w.data_ptr(), Y.data_ptr(),
            U.data_ptr(), gv.data_ptr(), self._st()), "dct_gather_contract")
        gm = torch.empty(self.nC, dtype=torch.float64, device=self.device)
        nat.check(nat.lib().dct_values_vjp(
            self.nC, self.Lt_ptr.data_ptr(), self.Lt_col.data_ptr(),
            self.Lt_val.data_ptr(), sigma.data_ptr(), gv.data_ptr(),
            gm.data_ptr(), self._st()), "dct_values_vjp")
        return gm


    # ------------------------------------------------ linearised products
    def jvec(self, v_full, sigma, U):
        """J v (nD,) on the current factorization and fields U:
        A_k dU_k = -A_k(dvals) U_k with dvals = L (-sigma v), then the
        weighted projection of dU (dctorch/simulation2d.py:689-710)."""
        x = (-sigma * v_full.to(self.device, torch.float64)).contiguous()
        dvals = torch.empty(self.nbatch * self.nnzA, dtype=torch.float64,
                            device=self.device)
        nat.check(nat.lib().dct_csr_spmv(
            dvals.numel(), self.L_ptr.data_ptr(), self.L_col.data_ptr(),
            self.L_val.data_ptr(), x.data_ptr(), dvals.data_ptr(), self._st()),
            "dct_csr_spmv")
        k = U.shape[-1]
        rhs = torch.empty_like(U)
        nat.check(nat.lib().dct_pattern_spmm(
            self.nbatch, self.nN, k, self.solver.crow.data_ptr(),
            self.col_e.data_ptr(), self._iperm_ptr, dvals.data_ptr(),
            self.nnzA, -1.0, U.data_ptr(), rhs.data_ptr(), self._st()),
            "dct_pattern_spmm")
        self._set_refinement(self.refine_fields, self.tol_fields)
        dU = torch.empty_like(rhs)
        self._plan.solve_permuted(rhs.data_ptr(), 1, k, dU.data_ptr(), self._st())
        return self.project(dU)

    def jac_block(self, a, b, sigma, U):
        """Rows a..b of the Jacobian w.r.t. m_full as an (nC, b - a) block:
        one adjoint solve with the columns a..b of Pd^T and the pairwise
        contraction with each datum's own source field
        (dctorch/simulation2d.py:439-518, 727-776)."""
        nb = b - a
        p0, p1 = int(self.Pd_indptr[a]), int(self.Pd_indptr[b])
        rhs = torch.zeros((self.nN, nb), dtype=torch.float64, device=self.device)
        rhs.index_put_((self.iperm_d[self.Pd_col[p0:p1].long()],
                        self.Pd_row[p0:p1] - a), self.Pd_val[p0:p1],
                       accumulate=True)
        self._set_refinement(self.refine_adj, self.tol_adj)
        Y = self._solve_perm(rhs, nb)
        gv = torch.empty((self.nbatch * self.nnzA, nb), dtype=torch.float64,
                         device=self.device)
        nat.check(nat.lib().dct_gather_pairwise(
            self.nbatch, self.nN, self.nnzA, nb, U.shape[-1],
            self.row_e.data_ptr(), self.col_e.data_ptr(), self._iperm_ptr,
            None if self.w is None else self.w.data_ptr(),
            self.sidx_d[a:b].contiguous().data_ptr(), Y.data_ptr(), U.data_ptr(),
            gv.data_ptr(), self._st()), "dct_gather_pairwise")
        Jb = torch.empty((self.nC, nb), dtype=torch.float64, device=self.device)
        nat.check(nat.lib().dct_values_vjp_multi(
            self.nC, nb, self.Lt_ptr.data_ptr(), self.Lt_col.data_ptr(),
            self.Lt_val.data_ptr(), sigma.data_ptr(), gv.data_ptr(),
            Jb.data_ptr(), self._st()), "dct_values_vjp_multi")
        return Jb


class FusedDpred(torch.autograd.Function):
    """d = dpred(m_full) with the hand-written adjoint as its backward."""

    @staticmethod
    def forward(ctx, m_full, path):
        d, sigma, U, stamp = path.forward(m_full)
        ctx.path, ctx.stamp = path, stamp
        ctx.save_for_backward(m_full.detach(), sigma, U)
        return d

    @staticmethod
    def backward(ctx, gd):
        m_full, sigma, U = ctx.saved_tensors
        path = ctx.path
        path.ensure_factors(m_full, ctx.stamp)
        return path.adjoint(gd, U, sigma).to(m_full.dtype), None
