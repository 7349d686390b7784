"""CPU oracle (TEST INFRASTRUCTURE ONLY) for dctorch's forward + adjoint path.

A float64 numpy/scipy restatement of what the reference computes at run
time, given the build-time operators.  It is used by the tests as the checker
and by bench.py as the timed CPU baseline; the product never calls it.

Pinned: `tests/golden/*.npz` hold outputs of the reference itself (its
`SciPySolver`/`SciPyBatchSolver` SuperLU path and its `TorchDC2D`/`TorchDC3D`
runtime, driven with the same operators); `tests/test_oracle.py` checks this
module against them.

Three exact solvers stand behind it: `SuperLUBatch` (the reference's own
CPU solver, scipy SuperLU, real or complex), `SlabCholeskyBatch`, a
block-tridiagonal dense Cholesky over the grid slabs for the float64
workloads at which SuperLU takes minutes per factorization (selected by an
operator set's "slab" entry), and `SlabLUBatch`, the same slabs factored by
block LU for complex-symmetric (complex resistivity) and general systems.

Operators (names as in the reference engines):
  Lstack  : CSR (nky*nnzA, nC), values of A_k = rows k*nnzA .. (k+1)*nnzA
  crow,col: CSR pattern of A (nN+1,), (nnzA,)
  wq      : (nky,) quadrature weights            (2.5-D only)
  Q       : (nN, nS) dense sources
  Pd      : CSR (nD, nN) receiver projection;  sidx (nD,) source of datum
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


# ------------------------------------------------------------- solver level
class SuperLUBatch:
    """SuperLU factorizations of nbatch systems on one pattern
    (dctorch/solver.py:314-374, SciPySolver / SciPyBatchSolver)."""

    def __init__(self, crow, col, n):
        self.crow = np.asarray(crow)
        self.col = np.asarray(col)
        self.n = int(n)
        self.lu = []

    def factorize(self, vals):
        vals = np.atleast_2d(np.asarray(vals))
        if not np.iscomplexobj(vals):
            vals = vals.astype(float)
        self.dtype = vals.dtype
        self.lu = [spla.splu(sp.csr_matrix((v, self.col, self.crow),
                                           shape=(self.n, self.n)).tocsc())
                   for v in vals]

    def solve(self, B):
        """B: (n, k) shared, or (nbatch, n, k); returns (nbatch, n, k)."""
        B = np.asarray(B, np.result_type(self.dtype, np.asarray(B).dtype, float))
        if B.ndim == 2:
            return np.stack([lu.solve(B) for lu in self.lu])
        return np.stack([lu.solve(B[i]) for i, lu in enumerate(self.lu)])


def row_of(crow):
    return np.repeat(np.arange(len(crow) - 1), np.diff(crow))


class SlabCholeskyBatch:
    """Exact float64 solves of nbatch SPD systems on one grid pattern by a
    block-tridiagonal dense Cholesky, for problems too large for SuperLU's
    single-threaded factorization and column-by-column solves.  It computes
    the same x = A^{-1} b as `SuperLUBatch` (dctorch/solver.py:314-374) to
    rounding, by another direct method, which `tests/test_oracle.py` checks.

    `slab[i]` is the grid slab of node i (its index along one mesh axis); the
    nodal stencil couples only nodes of the same or adjacent slabs, so with
    the nodes grouped slab by slab A is block tridiagonal:
        L_ii L_ii^T = A_ii - L_i,i-1 L_i,i-1^T,
        L_i+1,i     = A_i+1,i L_ii^{-T},
    and the solves are blocked forward / backward substitutions over the
    slabs (LAPACK potrf / trsm / gemm on dense blocks)."""

    def __init__(self, crow, col, n, slab):
        self.crow = np.asarray(crow)
        self.col = np.asarray(col)
        self.n = int(n)
        slab = np.asarray(slab, dtype=np.int64)
        if slab.shape != (self.n,):
            raise ValueError("one slab index per node")
        r = row_of(self.crow)
        if np.abs(slab[r] - slab[self.col]).max(initial=0) > 1:
            raise ValueError("the pattern couples nodes of non-adjacent slabs")
        self.order = np.argsort(slab, kind="stable")
        self.starts = np.searchsorted(slab[self.order],
                                      np.arange(int(slab.max()) + 2))
        self.fac = []

    # BLAS threads of the dense block kernels: the blocks are small (one
    # grid slab), and more threads than this only add synchronisation
    BLAS_THREADS = 4

    def _threads(self):
        import os
        from threadpoolctl import threadpool_limits
        return threadpool_limits(limits=max(1, min(self.BLAS_THREADS,
                                                   os.cpu_count() or 1)),
                                 user_api="blas")

    def factorize(self, vals):
        with self._threads():
            self._factorize(vals)

    def _factorize(self, vals):
        import scipy.linalg as sla
        vals = np.atleast_2d(np.asarray(vals, float))
        o, st = self.order, self.starts
        self.fac = []
        for v in vals:
            A = sp.csr_matrix((v, self.col, self.crow), shape=(self.n, self.n))
            A = A[o][:, o].tocsr()
            diag, sub = [], []
            prev = None
            for i in range(len(st) - 1):
                a, b = st[i], st[i + 1]
                D = A[a:b, a:b].toarray()
                if prev is not None:
                    D -= prev @ prev.T
                Lii = sla.cholesky(D, lower=True, check_finite=False)
                diag.append(Lii)
                if i + 2 < len(st):
                    B = A[b:st[i + 2], a:b].toarray()
                    prev = _flush_tiny(sla.solve_triangular(
                        Lii, B.T, lower=True, check_finite=False).T)
                    sub.append(prev)
            self.fac.append((diag, sub))

    def _solve_one(self, f, B):
        import scipy.linalg as sla
        diag, sub = f
        st = self.starts
        X = np.array(B[self.order], dtype=float)
        ns = len(st) - 1
        for i in range(ns):
            a, b = st[i], st[i + 1]
            rhs = X[a:b]
            if i > 0:
                rhs = rhs - sub[i - 1] @ X[st[i - 1]:a]
            X[a:b] = _flush_tiny(sla.solve_triangular(diag[i], rhs, lower=True,
                                                      check_finite=False))
        for i in range(ns - 1, -1, -1):
            a, b = st[i], st[i + 1]
            rhs = X[a:b]
            if i + 1 < ns:
                rhs = rhs - sub[i].T @ X[b:st[i + 2]]
            X[a:b] = _flush_tiny(sla.solve_triangular(diag[i], rhs, lower=True,
                                                      trans="T", check_finite=False))
        out = np.empty_like(X)
        out[self.order] = X
        return out

    def solve(self, B):
        """B: (n, k) shared, or (nbatch, n, k); returns (nbatch, n, k)."""
        B = np.asarray(B, float)
        with self._threads():
            if B.ndim == 2:
                return np.stack([self._solve_one(f, B) for f in self.fac])
            return np.stack([self._solve_one(f, B[i]) for i, f in enumerate(self.fac)])


class SlabLUBatch:
    """Exact solves of nbatch systems on one grid pattern, real or complex
    (complex-symmetric A of the complex-resistivity engine), by block
    tridiagonal LU over the grid slabs (as `SlabCholeskyBatch`, without
    symmetry): U_1 = A_11, L_i+1,i = A_i+1,i U_i^{-1},
    U_i+1 = A_i+1,i+1 - L_i+1,i A_i,i+1, each U_i factored by dense LU with
    partial pivoting inside the block (LAPACK getrf).  It computes the same
    x = A^{-1} b as `SuperLUBatch` to rounding, which `tests/test_oracle.py`
    checks."""

    def __init__(self, crow, col, n, slab):
        self._slab = SlabCholeskyBatch(crow, col, n, slab)
        self.crow, self.col, self.n = self._slab.crow, self._slab.col, self._slab.n
        self.order, self.starts = self._slab.order, self._slab.starts
        self.fac = []

    def factorize(self, vals):
        import scipy.linalg as sla
        vals = np.atleast_2d(np.asarray(vals))
        if not np.iscomplexobj(vals):
            vals = vals.astype(float)
        self.dtype = vals.dtype
        o, st = self.order, self.starts
        self.fac = []
        with self._slab._threads():
            for v in vals:
                A = sp.csr_matrix((v, self.col, self.crow), shape=(self.n, self.n))
                A = A[o][:, o].tocsr()
                lus, low, up = [], [], []
                U = A[st[0]:st[1], st[0]:st[1]].toarray()
                for i in range(len(st) - 1):
                    a, b = st[i], st[i + 1]
                    lu = sla.lu_factor(U, check_finite=False)
                    lus.append(lu)
                    if i + 2 < len(st):
                        c = st[i + 2]
                        Aup = A[a:b, b:c].toarray()
                        Alo = A[b:c, a:b].toarray()
                        # L = Alo U^{-1}:  U^T L^T = Alo^T
                        Lb = _flush_tiny(sla.lu_solve(lu, Alo.T, trans=1,
                                                      check_finite=False).T)
                        low.append(Lb)
                        up.append(Aup)
                        U = A[b:c, b:c].toarray() - Lb @ Aup
                self.fac.append((lus, low, up))

    def _solve_one(self, f, B):
        import scipy.linalg as sla
        lus, low, up = f
        st = self.starts
        X = np.array(B[self.order], dtype=np.result_type(self.dtype, B.dtype))
        ns = len(st) - 1
        for i in range(1, ns):
            a, b = st[i], st[i + 1]
            X[a:b] -= low[i - 1] @ X[st[i - 1]:a]
        for i in range(ns - 1, -1, -1):
            a, b = st[i], st[i + 1]
            rhs = X[a:b]
            if i + 1 < ns:
                rhs = rhs - up[i] @ X[b:st[i + 2]]
            X[a:b] = _flush_tiny(sla.lu_solve(lus[i], rhs, check_finite=False))
        out = np.empty_like(X)
        out[self.order] = X
        return out

    def solve(self, B):
        """B: (n, k) shared, or (nbatch, n, k); returns (nbatch, n, k)."""
        B = np.asarray(B)
        with self._slab._threads():
            if B.ndim == 2:
                return np.stack([self._solve_one(f, B) for f in self.fac])
            return np.stack([self._solve_one(f, B[i]) for i, f in enumerate(self.fac)])


def _flush_tiny(X):
    """Entries below 1e-100 of the block's largest set to zero: the coupling
    blocks decay geometrically away from the slab interface, and products
    of such entries would otherwise fall into subnormal floating point,
    which slows the dense kernels by orders of magnitude.  The perturbation
    is 1e-100 relative, far below float64 rounding."""
    big = np.abs(X).max(initial=0.0)
    if big > 0.0:
        X[np.abs(X) < 1e-100 * big] = 0.0
    return X


def grid_slabs(node_grid):
    """Slab index of every node for `SlabCholeskyBatch`: its grid index along
    the axis with the most nodes (the smallest dense blocks)."""
    g = np.asarray(node_grid)
    ax = int(np.argmax(g.max(axis=0)))
    return g[:, ax]


def _batch_solver(op):
    """The exact solver of the operator set: SuperLU (the reference's CPU
    solver) unless op carries grid slabs for the block solver."""
    if op.get("slab") is not None:
        return SlabCholeskyBatch(op["crow"], op["col"], op["nN"], op["slab"])
    return SuperLUBatch(op["crow"], op["col"], op["nN"])


def sparse_solve_vjp(crow, col, vals, b, gx):
    """x = A^{-1} b and the vector-Jacobian products of a loss with dL/dx = gx
    (dctorch/solver.py:141-173 and 261-281):
        adj = A^{-1} gx;  dL/dvals[e] = -sum_s adj[row_e, s] x[col_e, s];
        dL/db = adj  (summed over the batch when b is shared).
    vals: (nnz,) or (nb, nnz); b: (n,k) or (nb,n,k); gx like x.
    """
    vals = np.asarray(vals, float)
    single = vals.ndim == 1
    V = vals[None] if single else vals
    n = len(crow) - 1
    slv = SuperLUBatch(crow, col, n)
    slv.factorize(V)
    b = np.asarray(b, float)
    b2 = b.reshape(n, -1) if (single and b.ndim <= 2) else b
    x = slv.solve(b2 if b2.ndim == 2 else b2)
    gx = np.asarray(gx, float)
    G = gx.reshape(x.shape)
    adj = slv.solve(G) if G.ndim == 3 else slv.solve(G)
    r = row_of(crow)
    gvals = -np.einsum("bes,bes->be", adj[:, r, :], x[:, col, :])
    shared = b.ndim == 2 or single
    gb = adj.sum(0) if (shared and not single) else adj
    if single:
        return x[0].reshape(b.shape), gvals[0], adj[0].reshape(b.shape)
    return x, gvals, gb


# ---------------------------------------------------------- engine level
def sigma_of(m):
    return np.exp(-np.asarray(m, float))


def vals_2d(Lstack, m, nky):
    """VALS = (Lstack @ exp(-m)).view(nky, nnzA)  (simulation2d.py:391-392)."""
    v = Lstack @ sigma_of(m)
    return v.reshape(nky, -1)


def dpred_2d(op, m, return_fields=False):
    """Predicted data (simulation2d.py:378-396): Ubar = sum_k wq_k U_k,
    d = (Pd Ubar)[i, sidx[i]]."""
    nky = len(op["wq"])
    VALS = vals_2d(op["Lstack"], m, nky)
    slv = _batch_solver(op)
    slv.factorize(VALS)
    U = slv.solve(op["Q"])
    Ubar = np.tensordot(op["wq"], U, axes=(0, 0))
    PU = op["Pd"] @ Ubar
    d = PU[np.arange(PU.shape[0]), op["sidx"]]
    if return_fields:
        return d, VALS, slv, U
    return d


def _adjoint_2d(op, m, g_data, fields=None):
    """dL/dm for dL/dd = g_data through the 2.5-D chain (the autograd path of
    simulation2d.py:378-396 with solver.py:261-281 and the Lstack vjp).
    `fields` = dpred_2d(..., return_fields=True) reuses that factorization."""
    nky = len(op["wq"])
    d, VALS, slv, U = fields or dpred_2d(op, m, return_fields=True)
    nS = op["Q"].shape[1]
    nN = op["nN"]
    # dL/dUbar[:, s] = Pd^T (g restricted to source s)
    G = np.zeros((op["Pd"].shape[0], nS))
    G[np.arange(G.shape[0]), op["sidx"]] = g_data
    GU = op["Pd"].T @ G                         # (nN, nS)
    Y = slv.solve(GU)                           # A_k^{-1} Pd^T G (unweighted)
    r = row_of(op["crow"])
    gv = np.empty((nky, len(op["col"])))
    for k in range(nky):
        gv[k] = -op["wq"][k] * np.einsum("es,es->e", Y[k][r], U[k][op["col"]])
    gsig = op["Lstack"].T @ gv.reshape(-1)
    return d, -sigma_of(m) * gsig


def misfit_2d(op, m, dobs, w):
    """phi = sum (w (d - dobs))^2 (simulation2d.py:531-534)."""
    d = dpred_2d(op, m)
    r = w * (d - dobs)
    return float((r ** 2).sum())


def misfit_grad_2d(op, m, dobs, w):
    """(phi, dphi/dm) with one factorization, as misfit().backward() does."""
    fields = dpred_2d(op, m, return_fields=True)
    r = w * (fields[0] - dobs)
    _, g = _adjoint_2d(op, m, 2.0 * w * r, fields)
    return float((r ** 2).sum()), g


def jtvec_2d(op, m, v):
    """J^T v (simulation2d.py:398-437)."""
    return _adjoint_2d(op, m, np.asarray(v, float))[1]


def jvec_2d(op, m, u, fields=None):
    """J u for J = d(dpred)/dm (simulation2d.py:526-529 through
    Linearization2D.Jvec, 689-710): A_k dU_k = -A_k(dsigma) U_k with
    dsigma = -sigma u, then J u = (Pd sum_k wq_k dU_k)[i, sidx_i].
    `fields` = dpred_2d(..., return_fields=True) reuses that factorization."""
    nky = len(op["wq"])
    d, VALS, slv, U = fields or dpred_2d(op, m, return_fields=True)
    dvals = (op["Lstack"] @ (-sigma_of(m) * np.asarray(u, float))).reshape(nky, -1)
    n = op["nN"]
    rhs = np.stack([-(sp.csr_matrix((dvals[k], op["col"], op["crow"]),
                                    shape=(n, n)) @ U[k]) for k in range(nky)])
    dU = slv.solve(rhs)
    dbar = np.tensordot(op["wq"], dU, axes=(0, 0))
    PU = op["Pd"] @ dbar
    return PU[np.arange(PU.shape[0]), op["sidx"]]


def jmatrix_2d(op, m):
    """The explicit (nD, nC) sensitivity matrix (simulation2d.py:439-518):
    Y_k = A_k^{-1} Pd^T (one column per datum r);
    J[r] = -sigma * L^T (-wq_k Y_k[row_e, r] U_k[col_e, sidx_r])."""
    nky = len(op["wq"])
    d, VALS, slv, U = dpred_2d(op, m, return_fields=True)
    Y = slv.solve(op["Pd"].T.toarray())            # (nky, nN, nD)
    r = row_of(op["crow"])
    c = op["col"]
    sidx = op["sidx"]
    nD = op["Pd"].shape[0]
    gv = np.empty((nky, len(c), nD))
    for k in range(nky):
        gv[k] = -op["wq"][k] * Y[k][r] * U[k][c][:, sidx]
    J = op["Lstack"].T @ gv.reshape(nky * len(c), nD)  # (nC, nD)
    return (-sigma_of(m)[:, None] * J).T


def diag_jtdj_2d(op, m, dw):
    """diag(J^T diag(dw) J) (simulation2d.py:778-793)."""
    J = jmatrix_2d(op, m)
    return (J ** 2).T @ np.asarray(dw, float)


# ------------------------------------------------------------------- 3-D
def dpred_3d(op, m, return_fields=False):
    """simulation3d.py:197-207: VALS = L3 exp(-m); U = A^{-1} q; d = (Pd U)[i, sidx]."""
    vals = op["L3"] @ sigma_of(m)
    slv = _batch_solver(op)
    slv.factorize(vals[None])
    U = slv.solve(op["Q"])[0]
    PU = op["Pd"] @ U
    d = PU[np.arange(PU.shape[0]), op["sidx"]]
    if return_fields:
        return d, slv, U
    return d


def _adjoint_3d(op, m, g_data, fields=None):
    d, slv, U = fields or dpred_3d(op, m, return_fields=True)
    G = np.zeros((op["Pd"].shape[0], op["Q"].shape[1]))
    G[np.arange(G.shape[0]), op["sidx"]] = g_data
    Y = slv.solve(op["Pd"].T @ G)[0]
    r = row_of(op["crow"])
    gv = -np.einsum("es,es->e", Y[r], U[op["col"]])
    return d, -sigma_of(m) * (op["L3"].T @ gv)


def misfit_grad_3d(op, m, dobs, w):
    """(phi, dphi/dm) with one factorization (simulation3d.py:224-227 + backward)."""
    fields = dpred_3d(op, m, return_fields=True)
    r = w * (fields[0] - dobs)
    _, g = _adjoint_3d(op, m, 2.0 * w * r, fields)
    return float((r ** 2).sum()), g


def jtvec_3d(op, m, v):
    """simulation3d.py:209-222."""
    return _adjoint_3d(op, m, np.asarray(v, float))[1]


def rel(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def jvec_3d(op, m, u):
    """J u for the 3-D engine: A dU = -A(dvals) U with dvals = L3 (-sigma u),
    J u = (Pd dU)[i, sidx_i] (the product of dctorch/ip3d.py:150-163 before
    its scale)."""
    d, slv, U = dpred_3d(op, m, return_fields=True)
    n = op["nN"]
    dvals = op["L3"] @ (-sigma_of(m) * np.asarray(u, float))
    rhs = -(sp.csr_matrix((dvals, op["col"], op["crow"]), shape=(n, n)) @ U)
    dU = slv.solve(rhs[None])[0]
    PU = op["Pd"] @ dU
    return PU[np.arange(PU.shape[0]), op["sidx"]]


def ip_scale(v_dc, chargeability):
    """Per-datum IP scale: 1 / V_dc where the receiver's data type is
    apparent chargeability, else 1 (dctorch/ip2d.py:96-106, ip3d.py:125-135)."""
    s = np.ones_like(np.asarray(v_dc, float))
    c = np.asarray(chargeability, bool)
    s[c] = 1.0 / np.asarray(v_dc, float)[c]
    return s


def ip_dpred_2d(op, m_dc, eta, chargeability):
    """Linearized 2.5-D IP data scale * J(m_dc) eta (dctorch/ip2d.py:112-133)."""
    return ip_scale(dpred_2d(op, m_dc), chargeability) * jvec_2d(op, m_dc, eta)


def ip_dpred_3d(op, m_dc, eta, chargeability):
    """Linearized 3-D IP data scale * J(m_dc) eta (dctorch/ip3d.py:150-163)."""
    return ip_scale(dpred_3d(op, m_dc), chargeability) * jvec_3d(op, m_dc, eta)



def dcip_dpred_2d(op, m_rho, eta, ip_scale=1.0, dc_state="total"):
    """Joint non-linear DC + IP data (dctorch/dcip2d.py:152-180): V0 at
    sigma = exp(-m_rho), V1 at sigma (1 - eta); d_IP = ip_scale (V1 - V0) / V1,
    d_DC = V1 ("total") or V0 ("instantaneous").  Returns (d_DC, d_IP, V0, V1)."""
    eta = np.asarray(eta, float)
    v0 = dpred_2d(op, m_rho)
    v1 = dpred_2d(op, np.asarray(m_rho, float) - np.log1p(-eta))
    d_dc = v1 if dc_state == "total" else v0
    return d_dc, ip_scale * (v1 - v0) / v1, v0, v1


def dcip_misfit_grad_2d(op, m, eta_max, ip_scale, dc_state, dobs_dc, w_dc,
                        dobs_ip, w_ip, lam):
    """(phi, dphi/dm) of the joint misfit for the stacked model
    m = cat(log-rho, logit(eta / eta_max)) (dctorch/dcip2d.py:182-193), by
    the chain rule through both states' adjoints."""
    m = np.asarray(m, float)
    n = m.size // 2
    m_rho, m_eta = m[:n], m[n:]
    s = 1.0 / (1.0 + np.exp(-m_eta))
    eta = eta_max * s
    d_dc, d_ip, v0, v1 = dcip_dpred_2d(op, m_rho, eta, ip_scale, dc_state)
    r_dc = w_dc * (d_dc - dobs_dc)
    r_ip = w_ip * (d_ip - dobs_ip)
    phi = float((r_dc ** 2).sum() + lam * (r_ip ** 2).sum())
    g_dc = 2.0 * w_dc * r_dc
    g_ip = 2.0 * lam * w_ip * r_ip
    g0 = -g_ip * ip_scale / v1
    g1 = g_ip * ip_scale * v0 / v1 ** 2
    if dc_state == "total":
        g1 = g1 + g_dc
    else:
        g0 = g0 + g_dc
    m_eff = m_rho - np.log1p(-eta)
    j1 = jtvec_2d(op, m_eff, g1)
    grad_rho = jtvec_2d(op, m_rho, g0) + j1
    grad_eta = j1 / (1.0 - eta) * eta_max * s * (1.0 - s)
    return phi, np.concatenate([grad_rho, grad_eta])


def cr_dpred_2d(op, m_rho, chg, ip_scale=1.0, dc_datum="magnitude",
                return_fields=False):
    """Complex-resistivity 2.5-D data (dctorch/cr2d.py:74-97): the complex
    conductivity sigma* = sigma (1 - i m) with sigma = exp(-m_rho), complex
    values VALS = Lstack sigma*, U_k = A_k^{-1} q on complex SuperLU
    (complex-symmetric A_k; the block LU `SlabLUBatch` when op carries grid
    slabs), Ubar = sum_k wq_k U_k, V = (Pd Ubar)[i, sidx_i];
    d_rho = |V| ("magnitude") or Re V ("real"), d_ip = ip_scale Im V / Re V.
    Returns (d_rho, d_ip) or, with return_fields, also (V, sigma*, lu, U)."""
    nky = len(op["wq"])
    sig = sigma_of(m_rho)
    sstar = sig * (1.0 - 1j * np.asarray(chg, float))
    L = op["Lstack"]
    VALS = (L @ sstar.real + 1j * (L @ sstar.imag)).reshape(nky, -1)
    n = op["nN"]
    lu = (SlabLUBatch(op["crow"], op["col"], n, op["slab"]) if op.get("slab") is not None
          else SuperLUBatch(op["crow"], op["col"], n))
    lu.factorize(VALS)
    U = lu.solve(np.asarray(op["Q"], complex))
    Ubar = np.tensordot(op["wq"], U, axes=(0, 0))
    PU = op["Pd"] @ Ubar
    V = PU[np.arange(PU.shape[0]), op["sidx"]]
    d_rho = np.abs(V) if dc_datum == "magnitude" else V.real.copy()
    d_ip = ip_scale * V.imag / V.real
    if return_fields:
        return d_rho, d_ip, (V, sstar, lu, U)
    return d_rho, d_ip


def cr_misfit_grad_2d(op, m, ip_scale, dc_datum, dobs_rho, w_rho, dobs_ip, w_ip,
                      lam):
    """(phi, dphi/dm) of the complex-resistivity misfit (dctorch/cr2d.py:
    104-108) for the stacked model m = cat(log-rho, chargeability).

    V is holomorphic in sigma*, so for the real loss dphi = Re(G dV) with
    G = dphi/dRe V - i dphi/dIm V.  The adjoint fields Y_k = A_k^{-1} Pd^T G
    (complex, A_k^T = A_k) give h = Lstack^T gv, gv_k[e] = -wq_k sum_s
    Y_k[row_e, s] U_k[col_e, s]; with dsigma* = -sigma* dm_rho - i sigma dm,
    dphi/dm_rho = Re(-sigma* h) and dphi/dm = sigma Im(h)."""
    m = np.asarray(m, float)
    n = m.size // 2
    m_rho, chg = m[:n], m[n:]
    d_rho, d_ip, (V, sstar, lu, U) = cr_dpred_2d(op, m_rho, chg, ip_scale,
                                                 dc_datum, return_fields=True)
    r_rho = w_rho * (d_rho - dobs_rho)
    r_ip = w_ip * (d_ip - dobs_ip)
    phi = float((r_rho ** 2).sum() + lam * (r_ip ** 2).sum())
    g_rho = 2.0 * w_rho * r_rho
    g_ip = 2.0 * lam * w_ip * r_ip
    Vr, Vi = V.real, V.imag
    if dc_datum == "magnitude":
        a = np.abs(V)
        gr, gi = g_rho * Vr / a, g_rho * Vi / a
    else:
        gr, gi = g_rho.copy(), np.zeros_like(g_rho)
    gr = gr - g_ip * ip_scale * Vi / Vr ** 2
    gi = gi + g_ip * ip_scale / Vr
    G = np.zeros((op["Pd"].shape[0], op["Q"].shape[1]), complex)
    G[np.arange(G.shape[0]), op["sidx"]] = gr - 1j * gi
    R = op["Pd"].T @ G
    r = row_of(op["crow"])
    nky = len(op["wq"])
    gv = np.empty((nky, len(op["col"])), complex)
    Y = lu.solve(R)
    for k in range(nky):
        gv[k] = -op["wq"][k] * np.einsum("es,es->e", Y[k][r], U[k][op["col"]])
    L = op["Lstack"]
    gvf = gv.reshape(-1)
    h = L.T @ gvf.real + 1j * (L.T @ gvf.imag)
    sig = sstar.real
    return phi, np.concatenate([np.real(-sstar * h), sig * h.imag])


def unit_primary_2d(nodes, kys, poles, radii):
    """Unit-resistivity half-space primary (dctorch/singularity.py:47-82):
    K_0(ky r) / pi summed over each source's poles (location, sign), and at
    a pole's own node the mean of K_0 over a disc of radius R,
    2 (1 - a K_1(a)) / a^2 / pi with a = ky R.  poles[j] lists the poles of
    source j, radii[j] the disc radius of each.  Returns (nky, nN, nS)."""
    from scipy.special import k0, k1
    nodes = np.asarray(nodes, float)
    tol = 1e-9 * max(1.0, float(np.abs(nodes).max()))
    out = np.zeros((len(kys), nodes.shape[0], len(poles)))
    for j, plist in enumerate(poles):
        for (loc, sign), R in zip(plist, radii[j]):
            r = np.sqrt(((nodes - np.asarray(loc, float)[None, :2]) ** 2).sum(1))
            for ik, ky in enumerate(kys):
                v = k0(np.maximum(ky * r, 1e-300)) / np.pi
                at = r < tol
                if at.any():
                    a = ky * R
                    v[at] = 2.0 * (1.0 - a * k1(a)) / a ** 2 / np.pi
                out[ik, :, j] += sign * v
    return out


def dpred_2d_sr(op, m, u1, return_fields=False):
    """Singularity-removed data (dctorch/simulation2d.py:316-333): the total
    field rho_s u_1 + A^{-1}(A(1) u_1 - A(sigma) rho_s u_1), which equals
    A(sigma)^{-1} A(1) u_1 for any background rho_s."""
    nky = len(op["wq"])
    VALS = vals_2d(op["Lstack"], m, nky)
    ONES = (op["Lstack"] @ np.ones(op["Lstack"].shape[1])).reshape(nky, -1)
    n = op["nN"]
    slv = _batch_solver(op)
    slv.factorize(VALS)
    B = np.stack([sp.csr_matrix((ONES[k], op["col"], op["crow"]), shape=(n, n)) @ u1[k]
                  for k in range(nky)])
    U = slv.solve(B)
    Ubar = np.tensordot(op["wq"], U, axes=(0, 0))
    PU = op["Pd"] @ Ubar
    d = PU[np.arange(PU.shape[0]), op["sidx"]]
    if return_fields:
        return d, VALS, slv, U
    return d


def misfit_grad_2d_sr(op, m, u1, dobs, w):
    """(phi, dphi/dm) under singularity removal: the right-hand side A(1) u_1
    does not depend on the model, so the plain adjoint with the total field."""
    fields = dpred_2d_sr(op, m, u1, return_fields=True)
    r = w * (fields[0] - dobs)
    _, g = _adjoint_2d(op, m, 2.0 * w * r, fields)
    return float((r ** 2).sum()), g
