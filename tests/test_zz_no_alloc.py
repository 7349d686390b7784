"""The allocation-free small solve (dct_solve_small_noalloc).

It exists for callers that cannot allocate device memory -- code running
while a stream is captured into a CUDA graph, hosts whose framework owns the
device memory, loops that cannot take cudaMalloc's device synchronisation --
and keeps its only scratch in a fixed array inside the library.  This test
calls it through the C ABI twice in a row (the scratch keeps the previous
call's contents, which must not leak into the next result) and compares each
result with the regular allocating entry point (dct_solve via DCTSolver)."""
import ctypes as C

import numpy as np
import pytest
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


def test_noalloc_solve_matches_allocating_solve(cuda):
    mesh, survey, m = syn.tiny_2d()                 # 325 nodes
    ops = nodal_operators(mesh, survey)
    n = ops.nN
    crow = torch.tensor(ops.crow, device=cuda)
    col = torch.tensor(ops.col, device=cuda)
    rng = np.random.default_rng(7)
    results = []
    for call, ky in enumerate((0.05, 0.4)):         # two calls in a row
        A = ops.A(np.exp(-(m + 0.2 * call)), ky)
        vals = torch.tensor(A.data, device=cuda)
        b = torch.tensor(rng.standard_normal((n, 6)), device=cuda)
        x = torch.full_like(b, np.nan)
        _noalloc(crow, col, vals, b, x, cuda)
        ref = sparse_solve(vals, b, DCTSolver(crow, col, n, 6, device=cuda))
        torch.cuda.synchronize()
        err = float(torch.linalg.norm(x - ref) / torch.linalg.norm(ref))
        results.append(err)
        assert err < 1e-10, (call, err)
    assert len(results) == 2


def test_noalloc_rejects_sizes_beyond_its_limit(cuda):
    n = 513
    crow = torch.zeros(n + 1, dtype=torch.int32, device=cuda)
    col = torch.zeros(1, dtype=torch.int32, device=cuda)
    vals = torch.ones(1, dtype=torch.float64, device=cuda)
    b = torch.zeros((n, 1), dtype=torch.float64, device=cuda)
    with pytest.raises(nat.DCTError) as ei:
        _noalloc(crow, col, vals, b, b.clone(), cuda)
    assert ei.value.code == 1
