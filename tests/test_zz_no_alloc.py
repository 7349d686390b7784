"""The allocation-free small solve (dct_solve_small_noalloc).

It exists for callers that cannot allocate device memory -- hosts whose
framework owns the device memory through its own pool, loops that cannot
take cudaMalloc's device synchronisation -- and keeps its only scratch in a
fixed array inside the library.  These tests call it through the C ABI three
times in a row (the scratch keeps the previous call's contents, which must
not leak into the next result) and compare each result with the regular
allocating entry point (dct_solve via DCTSolver) and with scipy's float64
sparse solve, within 1e-10 relative; they check that the calls change
neither torch's allocation count nor the device's free memory (after the
first call, which sets the entry point up on the device), that a matrix
that is not positive definite comes back as NaN, and that sizes beyond the
limit are refused."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

from simpeg_dc_torch_b200 import DCTSolver, sparse_solve
from simpeg_dc_torch_b200 import _native as nat
from simpeg_dc_torch_b200 import synthetic as syn
from simpeg_dc_torch_b200.operators import nodal_operators

pytestmark = pytest.mark.gpu


def _noalloc(crow, col, vals, b, x, dev):
    n, k = b.shape
    rc = nat.lib().dct_solve_small_noalloc(
        n, C.c_void_p(crow.data_ptr()), C.c_void_p(col.data_ptr()),
        C.c_void_p(vals.data_ptr()), C.c_void_p(b.data_ptr()), k,
        C.c_void_p(x.data_ptr()),
        C.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    nat.check(rc, "dct_solve_small_noalloc")


def _free_bytes(dev):
    free, _ = torch.cuda.mem_get_info(dev)
    return free


def test_noalloc_solve_matches_allocating_solve(cuda):
    mesh, survey, m = syn.tiny_2d()                 # 325 nodes
    ops = nodal_operators(mesh, survey)
    n = ops.nN
    crow = torch.tensor(ops.crow, device=cuda)
    col = torch.tensor(ops.col, device=cuda)
    rng = np.random.default_rng(7)
    cases = []
    for call, ky in enumerate((0.05, 0.4, 1.5)):    # three calls in a row
        A = ops.A(np.exp(-(m + 0.2 * call)), ky)
        vals = torch.tensor(A.data, device=cuda)
        b_np = rng.standard_normal((n, 6))
        b = torch.tensor(b_np, device=cuda)
        x = torch.full_like(b, np.nan)
        cases.append((A, vals, b_np, b, x))
    # the allocating reference solutions first, so that the no-alloc calls
    # below run back to back with every buffer already in place
    refs = [sparse_solve(vals, b, DCTSolver(crow, col, n, 6, device=cuda))
            for _, vals, _, b, _ in cases]
    # the first call on the device looks up the scratch address and loads
    # the kernels (lazy module loading may take device memory for code);
    # the two calls after it must change neither count
    _noalloc(crow, col, cases[0][1], cases[0][3], cases[0][4], cuda)
    torch.cuda.synchronize()
    alloc0, free0 = torch.cuda.memory_allocated(cuda), _free_bytes(cuda)
    for _, vals, _, b, x in cases[1:]:
        _noalloc(crow, col, vals, b, x, cuda)
    torch.cuda.synchronize()
    assert torch.cuda.memory_allocated(cuda) == alloc0
    assert _free_bytes(cuda) == free0
    for (A, _, b_np, _, x), ref in zip(cases, refs):
        xs = spla.spsolve(sp.csc_matrix(A), b_np)
        xh = x.cpu().numpy()
        assert np.linalg.norm(xh - xs) <= 1e-10 * np.linalg.norm(xs)
        err = float(torch.linalg.norm(x - ref) / torch.linalg.norm(ref))
        assert err < 1e-10, err


def test_noalloc_marks_an_indefinite_matrix_with_nan(cuda):
    n = 40
    A = sp.diags([-np.ones(n - 1), 2.0 * np.ones(n), -np.ones(n - 1)],
                 [-1, 0, 1]).tocsr()
    A[7, 7] = -3.0                                   # not positive definite
    A = sp.csr_matrix(A)
    A.sort_indices()
    crow = torch.tensor(A.indptr.astype(np.int32), device=cuda)
    col = torch.tensor(A.indices.astype(np.int32), device=cuda)
    vals = torch.tensor(A.data, device=cuda)
    b = torch.ones((n, 2), dtype=torch.float64, device=cuda)
    x = torch.zeros_like(b)
    _noalloc(crow, col, vals, b, x, cuda)
    torch.cuda.synchronize()
    assert bool(torch.isnan(x).all())


def test_noalloc_rejects_sizes_beyond_its_limit(cuda):
    n = 513
    crow = torch.zeros(n + 1, dtype=torch.int32, device=cuda)
    col = torch.zeros(1, dtype=torch.int32, device=cuda)
    vals = torch.ones(1, dtype=torch.float64, device=cuda)
    b = torch.zeros((n, 1), dtype=torch.float64, device=cuda)
    with pytest.raises(nat.DCTError) as ei:
        _noalloc(crow, col, vals, b, b.clone(), cuda)
    assert ei.value.code == 1
