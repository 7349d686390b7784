"""Sparse SPD direct solve on a B200 as torch autograd ops (drop-in for
dctorch/solver.py on CUDA devices).

The classes mirror the reference's solver surface: `DCTSolver` replaces
`CuDSSSolver` (dctorch/solver.py:76-138), `DCTBatchSolver` replaces
`CuDSSBatchSolver` (dctorch/solver.py:181-233); `make_solver` and
`make_batch_solver` (dctorch/solver.py:383-399) return them for CUDA devices.
Attributes `n, n_rhs, nbatch, device, dtype, crow, col, row, stamp` and methods
`factorize(values)`, `solve(b)`, `free()` keep the reference's meaning and
shapes.  The symbolic analysis (nested dissection + assembly tree) runs once
per instance; `factorize` is a numeric refactorization of new values on the
same pattern.

Precision: a float64 solver factors and solves in float64.  A float32 solver
factors and solves in float32 and refines every solution with residuals
b - A x formed in float64: at most `refine` corrections (default 2; 0 gives
the plain float32 solve of the reference).  With `refine_tol` > 0 the
refinement stops once the estimated relative error of the solution is below
it, and when the corrections stagnate or run out above it `check()` raises
(status "iterative refinement did not converge"); `refine_tol` = 0 (the
default) runs the fixed number of corrections.

The differentiable ops `sparse_solve`, `sparse_solve_batch` and
`sparse_solve_batch_prefactored` have the reference's contract
(dctorch/solver.py:141-178, 236-311): the backward solves the adjoint on the
same factors (A symmetric) and contracts it with the solution on the pattern,
grad_vals[e] = -sum_s adj[row_e, s] x[col_e, s], here in one CUDA kernel.

Only CUDA devices are served; there is no CPU path in this package.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _native as nat

# real SPD systems, complex-symmetric ones (A^T = A, not Hermitian;
# factored A = L L^T without conjugation) and general real ones (float64
# P A P^T = L U with static pivoting, structurally symmetric patterns)
_MATRIX_TYPES = ("spd", "symmetric", "general")


def _require_cuda(device):
    device = torch.device(device)
    if device.type != "cuda":
        raise NotImplementedError(
            "simpeg_dc_torch_b200 implements the CUDA solver path only; "
            f"got device {device}")
    if not torch.cuda.is_available():
        raise RuntimeError("a CUDA device was requested but none is available")
    if device.index is None:
        device = torch.device("cuda", torch.cuda.current_device())
    return device


def _stream_ptr(device):
    return torch.cuda.current_stream(device).cuda_stream


def _dtype_code(dt):
    if dt == torch.float64:
        return nat.F64
    if dt == torch.float32:
        return nat.F32
    if dt in (torch.complex128, torch.complex64):
        return nat.C128
    raise TypeError(f"unsupported dtype {dt}; float64, float32 or complex expected")


def _work_dtype(dt):
    """The dtype of the buffers the library reads and writes: complex64
    systems are factored and solved in complex128."""
    return torch.complex128 if dt.is_complex else dt


class _PlanSolver:
    """Shared machinery of the single and batched solvers."""

    def __init__(self, crow, col, n, n_rhs, nbatch, device, dtype,
                 matrix_type, coords, refine, leaf_size, refine_tol=None,
                 tuning=None):
        if matrix_type not in _MATRIX_TYPES or (
                (matrix_type == "symmetric") != bool(dtype.is_complex)) or (
                matrix_type == "general" and dtype != torch.float64):
            raise NotImplementedError(
                f"matrix_type {matrix_type!r} with dtype {dtype}: real SPD "
                "systems ('spd', Cholesky), complex-symmetric ones "
                "('symmetric', L L^T) and float64 general ones ('general', "
                "L U with static pivoting) are factored here")
        self.matrix_type = matrix_type
        self.general = matrix_type == "general"
        self.device = _require_cuda(device)
        self.dtype = dtype
        self._code = _dtype_code(dtype)
        self.n, self.n_rhs, self.nbatch = int(n), int(n_rhs), int(nbatch)
        crow_np = np.asarray(torch.as_tensor(crow).cpu().numpy(), dtype=np.int32)
        col_np = np.asarray(torch.as_tensor(col).cpu().numpy(), dtype=np.int32)
        if crow_np.size != self.n + 1:
            raise ValueError("crow must have n+1 entries")
        self.crow = torch.as_tensor(crow_np).to(self.device)
        self.col = torch.as_tensor(col_np).to(self.device)
        counts = self.crow[1:] - self.crow[:-1]
        self.row = torch.repeat_interleave(
            torch.arange(self.n, device=self.device, dtype=torch.int32),
            counts)
        self.nnz = int(col_np.size)
        self._sym = nat.Symbolic(crow_np, col_np, coords, leaf_size)
        with torch.cuda.device(self.device):
            self._plan = nat.Plan(self._sym, self.nbatch, self.n_rhs,
                                  self._code, self.device.index, tuning,
                                  general=self.general)
        # refinement of float32 plans: at most `refine` corrections (the
        # library default is 2), fewer once the estimated error is below
        # `refine_tol` (0, the library default: a fixed count)
        self.refine = 2 if refine is None else int(refine)
        self._plan.set_refinement(self.refine)
        self.refine_tol = 0.0 if refine_tol is None else float(refine_tol)
        self._plan.set_refinement_tolerance(self.refine_tol)
        self.stamp = 0

    # ---- introspection
    @property
    def plan(self):
        return self._plan

    def analysis(self):
        """Statistics of the symbolic analysis (fronts, nnz(L), flops)."""
        return self._sym.info()

    def check(self):
        """Synchronise and raise if a kernel reported an error since the last
        check (a non-positive pivot, a refinement that did not converge, a
        timed-out device wait).  Returns the last refinement residual ratio
        max|b - A x| / max|b|."""
        code, where, res = self._plan.status(_stream_ptr(self.device))
        if code == 5:
            it, _, est, _ = self._plan.refinement_info(_stream_ptr(self.device))
            raise nat.DCTError(code, "solve",
                               f"estimated error {est:.3g} after {it} corrections "
                               f"(tolerance {self.refine_tol:.3g}, residual "
                               f"ratio {res:.3g})")
        if code != 0:
            raise nat.DCTError(code, "factorization", f"at supernode {where}")
        return res

    def refinement_info(self):
        """Refinement record of the last float32 solve: {"iters",
        "converged", "est_error", "rho"} (synchronises the stream)."""
        it, conv, est, rho = self._plan.refinement_info(_stream_ptr(self.device))
        return {"iters": it, "converged": conv, "est_error": est, "rho": rho}

    # ---- numeric phases
    def _factorize(self, values):
        v = values.detach()
        if self._code == nat.C128:
            v = v.to(torch.complex128)
        elif v.dtype not in (torch.float64, torch.float32):
            v = v.to(torch.float64)
        v = v.to(self.device).contiguous()
        if v.dim() == 1:
            v = v.unsqueeze(0)
        if v.shape != (self.nbatch, self.nnz):
            raise ValueError(f"values must be ({self.nbatch}, {self.nnz}), "
                             f"got {tuple(v.shape)}")
        self._plan.factorize(v.data_ptr(), _dtype_code(v.dtype), self.nnz,
                             _stream_ptr(self.device))
        self._vals_keepalive = v
        self.stamp += 1

    def _solve(self, b2, batched, transposed=False):
        """b2: (n, k) or (nbatch, n, k) in self.dtype; returns (nbatch, n, k).
        transposed: solve A^T x = b (differs from A x = b for general plans)."""
        k = b2.shape[-1]
        if k > self.n_rhs:
            raise ValueError(f"{k} right-hand sides exceed n_rhs={self.n_rhs}")
        wdt = _work_dtype(self.dtype)
        b2 = b2.to(wdt).contiguous()
        x = torch.empty((self.nbatch, self.n, k), dtype=wdt, device=self.device)
        fn = self._plan.solve_transposed if transposed else self._plan.solve
        fn(b2.data_ptr(), _dtype_code(wdt), 1 if batched else 0, k,
           x.data_ptr(), _stream_ptr(self.device))
        return x.to(self.dtype)

    def static_pivots(self):
        """Pivots replaced by static pivoting in the last factorization of a
        general plan (synchronises the stream); 0 for the other types."""
        return self._plan.static_pivots(_stream_ptr(self.device)) if self.general else 0

    def free(self):
        if getattr(self, "_plan", None) is not None:
            self._plan.free()
            self._plan = None


class DCTSolver(_PlanSolver):
    """Stateful SPD solver bound to one pattern and RHS width
    (the interface of dctorch's CuDSSSolver)."""

    def __init__(self, crow, col, n, n_rhs, device="cuda",
                 dtype=torch.float64, matrix_type="spd", coords=None,
                 refine=None, leaf_size=64, refine_tol=None, tuning=None):
        super().__init__(crow, col, n, n_rhs, 1, device, dtype, matrix_type,
                         coords, refine, leaf_size, refine_tol, tuning)

    def factorize(self, values):
        """Numeric refactorization with new values (nnz,), same pattern."""
        self._factorize(values.reshape(1, -1))

    def solve(self, b, transposed=False):
        """Solve A x = b (A^T x = b with transposed) for the current
        factorization; b (n,) or (n, k)."""
        b2 = b.detach().to(device=self.device, dtype=self.dtype)
        b2 = b2.reshape(self.n, -1).contiguous()
        x = self._solve(b2, False, transposed)
        return x[0].reshape(b.shape)


class DCTBatchSolver(_PlanSolver):
    """`nbatch` SPD systems on one shared pattern (the interface of dctorch's
    CuDSSBatchSolver): one analysis, every system factored and solved in the
    same launches."""

    def __init__(self, crow, col, n, n_rhs, nbatch, device="cuda",
                 dtype=torch.float64, matrix_type="spd", coords=None,
                 refine=None, leaf_size=64, refine_tol=None, tuning=None):
        super().__init__(crow, col, n, n_rhs, nbatch, device, dtype,
                         matrix_type, coords, refine, leaf_size, refine_tol, tuning)

    def factorize(self, values):
        """values: (nbatch, nnz) -- refactorize every system."""
        self._factorize(values)

    def solve(self, b, transposed=False):
        """b: (nbatch, n, k) or shared (n, k); returns (nbatch, n, k)
        (A^T x = b with transposed)."""
        shared = b.dim() == 2
        b2 = b.detach().to(device=self.device, dtype=self.dtype).contiguous()
        return self._solve(b2, not shared, transposed)


# --------------------------------------------------------------- autograd
def _grad_vals(solver, adj, x):
    """-sum_s adj[b, row_e, s] x[b, col_e, s] for every pattern entry."""
    nb = adj.shape[0]
    k = adj.shape[-1]
    wdt = _work_dtype(adj.dtype)
    adj, x = adj.to(wdt).contiguous(), x.to(wdt).contiguous()
    out = torch.empty((nb, solver.nnz), dtype=wdt, device=adj.device)
    nat.check(nat.lib().dct_gather_contract_plain(
        nb, solver.n, solver.nnz, k, solver.row.data_ptr(),
        solver.col.data_ptr(), _dtype_code(wdt),
        adj.data_ptr(), x.data_ptr(),
        out.data_ptr(), _stream_ptr(solver.device)), "gather_contract")
    return out


class _SparseSolveFn(torch.autograd.Function):
    """x = A(values)^{-1} b, differentiable in values and b (A SPD)."""

    @staticmethod
    def forward(ctx, values, b, solver):
        solver.factorize(values.detach())
        x = solver.solve(b.detach())
        ctx.solver = solver
        ctx.dt_vals, ctx.dt_b = values.dtype, b.dtype
        ctx.save_for_backward(x)
        return x

    @staticmethod
    def backward(ctx, grad_x):
        (x,) = ctx.saved_tensors
        solver = ctx.solver
        # complex-safe (a no-op on real tensors): torch hands backward the
        # conjugate Wirtinger derivative G = dL/dx*; with x holomorphic in A,
        # dL/dA*_ij = -conj(adj_i x_j), dL/db* = conj(adj) for
        # adj = A^{-T} conj(G) (dctorch/solver.py:236-281, where A^T = A); a
        # general plan solves with A^T on the same factors
        adj = solver.solve(grad_x.conj().resolve_conj().contiguous(),
                           transposed=getattr(solver, "general", False))
        grad_vals = grad_b = None
        if ctx.needs_input_grad[0]:
            gv = _grad_vals(solver, adj.reshape(1, solver.n, -1),
                            x.reshape(1, solver.n, -1))
            grad_vals = gv[0].conj().resolve_conj().to(ctx.dt_vals)
        if ctx.needs_input_grad[1]:
            grad_b = adj.conj().resolve_conj().to(ctx.dt_b)
        return grad_vals, grad_b, None


def sparse_solve(values, b, solver):
    """Differentiable sparse SPD solve (dctorch/solver.py:176-178)."""
    return _SparseSolveFn.apply(values, b, solver)


class _SparseSolveBatchFn(torch.autograd.Function):
    """x_i = A_i(values_i)^{-1} b on one shared pattern (real SPD)."""

    @staticmethod
    def forward(ctx, values, b, solver):
        solver.factorize(values.detach())
        x = solver.solve(b.detach())
        ctx.solver = solver
        ctx.b_shared = b.dim() == 2
        ctx.dt_vals, ctx.dt_b = values.dtype, b.dtype
        ctx.save_for_backward(x)
        return x

    @staticmethod
    def backward(ctx, grad_x):
        (x,) = ctx.saved_tensors
        solver = ctx.solver
        # complex-safe, as _SparseSolveFn.backward (A^T for general plans)
        adj = solver.solve(grad_x.conj().resolve_conj().contiguous(),
                           transposed=getattr(solver, "general", False))
        grad_vals = grad_b = None
        if ctx.needs_input_grad[0]:
            grad_vals = _grad_vals(solver, adj, x).conj().resolve_conj().to(ctx.dt_vals)
        if ctx.needs_input_grad[1]:
            gb = adj.sum(0) if ctx.b_shared else adj
            grad_b = gb.conj().resolve_conj().to(ctx.dt_b)
        return grad_vals, grad_b, None


class _SparseSolveBatchPreFn(torch.autograd.Function):
    """As _SparseSolveBatchFn for an A the caller already factorized."""

    @staticmethod
    def forward(ctx, values, b, solver):
        x = solver.solve(b.detach())
        ctx.solver = solver
        ctx.b_shared = b.dim() == 2
        ctx.dt_vals, ctx.dt_b = values.dtype, b.dtype
        ctx.save_for_backward(x)
        return x

    backward = _SparseSolveBatchFn.backward


def sparse_solve_batch(values, b, solver):
    """values: (nbatch, nnz) | b: (nbatch, n, k) or shared (n, k)."""
    return _SparseSolveBatchFn.apply(values, b, solver)


def sparse_solve_batch_prefactored(values, b, solver):
    """Differentiable solve on an already-factorized A."""
    return _SparseSolveBatchPreFn.apply(values, b, solver)


def _default_mtype(dtype, matrix_type):
    if matrix_type is not None:
        return matrix_type
    return "symmetric" if dtype.is_complex else "spd"


def make_solver(crow, col, n, n_rhs, device="cuda", dtype=torch.float64,
                matrix_type=None, **kw):
    """Factory (dctorch/solver.py:383-390): the B200 solver for CUDA devices."""
    mt = _default_mtype(dtype, matrix_type)
    return DCTSolver(crow, col, n, n_rhs, device=device, dtype=dtype,
                     matrix_type=mt, **kw)


def make_batch_solver(crow, col, n, n_rhs, nbatch, device="cuda",
                      dtype=torch.float64, matrix_type=None, **kw):
    """Factory (dctorch/solver.py:393-399)."""
    mt = _default_mtype(dtype, matrix_type)
    return DCTBatchSolver(crow, col, n, n_rhs, nbatch, device=device,
                          dtype=dtype, matrix_type=mt, **kw)


# the reference's class names, for `from ... import CuDSSSolver` call sites
CuDSSSolver = DCTSolver
CuDSSBatchSolver = DCTBatchSolver
