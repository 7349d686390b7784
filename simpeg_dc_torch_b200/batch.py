"""Many independent 2.5-D DC surveys of uneven size, factored and solved in
the same launches.

The reference batches the nky wavenumber systems of one survey on one
pattern (`CuDSSBatchSolver`, dctorch/solver.py:181-233) and runs surveys one
after another.  Here every survey's wavenumber systems are assembled side by
side into one block-diagonal pattern: system k of the batch holds survey
b's k-th wavenumber system in the rows of survey b, for every b at once.
The nested dissection splits the disconnected blocks first (empty
separators), so the assembly forest has one tree per survey and every
level-synchronous factor or substitution launch covers the fronts of all
surveys at that level.

Each survey keeps its own wavenumbers and weights (the reference's default
"electrodes" fit over its own electrode distances, dctorch/quadrature.py).
The weight w_bk of survey b's k-th wavenumber is folded into that block of
the system, A'_bk = A_bk / w_bk (rows of its assembly map scaled by 1/w_bk),
so that A'_bk^{-1} q = w_bk A_bk^{-1} q and the batch's data are a plain sum
over the systems; the adjoint through the scaled map is then the exact
gradient of the same data.  A survey whose fit kept fewer points than
another's has its heaviest point split into equal halves (two systems of
weight w/2, the same sum) until the counts agree.

Sources of all surveys share the right-hand-side columns (survey b's source
s is column s in b's rows); data, models and gradients are the surveys'
concatenated in order (`split_model`, `split_data`, `join`).  With
`tune=True` the solver's schedule shapes come from the autotuner
(`tuning.py`) timed on this batch's own pattern.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp
import torch

from ._fused import FusedDpred, FusedPath
from .mesh import as_tensor_mesh
from .operators import nodal_operators
from .quadrature import electrode_distance_range, k0_quadrature


def _equalise(kys, wq, n):
    """Split the heaviest point in halves until there are n points."""
    kys, wq = list(kys), list(wq)
    while len(kys) < n:
        i = int(np.argmax(wq))
        kys.insert(i + 1, kys[i])
        wq[i] *= 0.5
        wq.insert(i + 1, wq[i])
    return np.asarray(kys, float), np.asarray(wq, float)


@dataclass
class BatchOperators:
    """Block-diagonal operators of a batch of 2.5-D surveys."""
    crow: np.ndarray           # (N+1,) int32 block-diagonal pattern
    col: np.ndarray            # (nnz,) int32
    L: sp.csr_matrix           # (nky*nnz, nC): system k in rows k*nnz.., scaled by 1/w
    Q: sp.csc_matrix           # (N, max nS)
    Pd: sp.csr_matrix          # (nD, N)
    sidx: np.ndarray           # (nD,) source column of each datum
    coords: np.ndarray         # (N, 2) grid coordinates, surveys side by side
    nky: int
    kys: list                  # per survey (nky,) wavenumbers (after splitting)
    wq: list                   # per survey (nky,) weights (after splitting)
    node_off: np.ndarray       # (B+1,) node offsets
    cell_off: np.ndarray       # (B+1,) cell offsets
    data_off: np.ndarray       # (B+1,) data offsets
    nS: np.ndarray             # (B,) sources per survey
    ops: list                  # per survey NodalOperators


def batch_operators(problems, nky=12):
    """Block-diagonal operators of [(mesh, survey), ...] (host, float64)."""
    ops, kys, wqs, meshes = [], [], [], []
    for mesh, survey in problems:
        mesh = as_tensor_mesh(mesh)
        meshes.append(mesh)
        o = nodal_operators(mesh, survey)
        k, w, _ = k0_quadrature(*electrode_distance_range(survey), nky)
        ops.append(o)
        kys.append(np.asarray(k, float))
        wqs.append(np.asarray(w, float))
    n_used = max(k.size for k in kys)
    for b in range(len(ops)):
        kys[b], wqs[b] = _equalise(kys[b], wqs[b], n_used)
    B = len(ops)
    node_off = np.zeros(B + 1, np.int64)
    cell_off = np.zeros(B + 1, np.int64)
    data_off = np.zeros(B + 1, np.int64)
    nnz_off = np.zeros(B + 1, np.int64)
    for b, o in enumerate(ops):
        node_off[b + 1] = node_off[b] + o.nN
        cell_off[b + 1] = cell_off[b] + o.nC
        data_off[b + 1] = data_off[b] + o.nD
        nnz_off[b + 1] = nnz_off[b] + o.nnzA
    N, nnz = int(node_off[-1]), int(nnz_off[-1])
    crow = np.zeros(N + 1, np.int64)
    col = np.zeros(nnz, np.int64)
    for b, o in enumerate(ops):
        crow[node_off[b] + 1:node_off[b + 1] + 1] = nnz_off[b] + o.crow[1:]
        col[nnz_off[b]:nnz_off[b + 1]] = node_off[b] + o.col
    blocks = []
    for k in range(n_used):
        blocks.append(sp.block_diag([o.L_ky(kys[b][k]) / wqs[b][k]
                                     for b, o in enumerate(ops)], format="csr"))
    L = sp.vstack(blocks).tocsr()
    nS = np.array([o.nS for o in ops])
    Q = sp.lil_matrix((N, int(nS.max())))
    for b, o in enumerate(ops):
        Q[node_off[b]:node_off[b + 1], :o.nS] = o.q
    Pd = sp.block_diag([o.Pd for o in ops], format="csr")
    sidx = np.concatenate([o.sidx for o in ops])
    coords, x0 = [], 0
    for mesh in meshes:
        g = mesh.node_grid_index().astype(np.int64)
        g[:, 0] += x0
        x0 = int(g[:, 0].max()) + 2
        coords.append(g)
    coords = np.vstack(coords)
    if coords.max() >= 2 ** 31:
        raise ValueError("batch too large for int32 grid coordinates")
    return BatchOperators(crow=crow.astype(np.int32), col=col.astype(np.int32),
                          L=L, Q=sp.csc_matrix(Q), Pd=Pd, sidx=sidx,
                          coords=coords.astype(np.int32), nky=n_used, kys=kys,
                          wq=wqs, node_off=node_off, cell_off=cell_off,
                          data_off=data_off, nS=nS, ops=ops)


class TorchDC2DBatch:
    """dpred / misfit / gradient of many independent 2.5-D surveys at once.

    problems : [(mesh, survey), ...] -- tensor meshes (this package's or
    discretize's) and DC surveys, of any sizes.  Models, data and gradients
    are the surveys' concatenated (see split_model / split_data / join)."""

    def __init__(self, problems, nky=12, device="cuda", dtype=torch.float64,
                 refine=None, refine_tol=None, tune=False):
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise NotImplementedError("TorchDC2DBatch runs on CUDA devices only")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.dtype = dtype
        bo = batch_operators(problems, nky)
        self._bo = bo
        self.nsurveys = len(bo.ops)
        self.nky = bo.nky
        self.nC = int(bo.cell_off[-1])
        self.nN = int(bo.node_off[-1])
        self.nD = int(bo.data_off[-1])
        self.nS = int(bo.nS.max())
        precision = "fp64" if dtype == torch.float64 else "fp32_ir"
        refine_tol = 1e-9 if refine_tol is None else refine_tol
        self.tuning, self.tuning_table = None, None
        if tune:
            from .tuning import tune_schedule
            vals = bo.L @ np.full(self.nC, 0.01)
            self.tuning, self.tuning_table = tune_schedule(
                bo.crow, bo.col, self.nN, self.nS, self.nky, self.device, dtype,
                vals.reshape(self.nky, -1), bo.coords,
                refine=2 if refine is None else int(refine))
        self._path = FusedPath(bo.crow, bo.col, bo.L, None, bo.Q, bo.Pd, bo.sidx,
                               self.device, precision, coords=bo.coords,
                               refine=refine, refine_tol=refine_tol,
                               tuning=self.tuning)
        self.solver = self._path.solver

    # ---------------------------------------------------------- layout
    def split_model(self, m):
        o = self._bo.cell_off
        return [m[o[b]:o[b + 1]] for b in range(self.nsurveys)]

    def split_data(self, d):
        o = self._bo.data_off
        return [d[o[b]:o[b + 1]] for b in range(self.nsurveys)]

    @staticmethod
    def join(parts):
        if isinstance(parts[0], torch.Tensor):
            return torch.cat([p.reshape(-1) for p in parts])
        return np.concatenate([np.asarray(p, float).reshape(-1) for p in parts])

    # ---------------------------------------------------------- runtime
    def dpred(self, m):
        """Data of every survey (nD,) for the concatenated log-resistivities
        m (nC,).  Autograd-traceable."""
        dev0, dt0 = m.device, m.dtype
        m_full = m.to(device=self.device, dtype=torch.float64).reshape(-1)
        d = FusedDpred.apply(m_full, self._path)
        return d.to(device=dev0, dtype=dt0)

    def misfit(self, m, dobs, w):
        """sum over surveys of ||w (dpred - dobs)||^2; its gradient holds
        each survey's own misfit gradient in that survey's cells."""
        d = self.dpred(m)
        r = w.to(d.dtype) * (d - dobs.to(d.dtype))
        return (r * r).sum()

    def check(self):
        return self.solver.check()
