"""Failure detection on the GPU without a fault: the bounded mbarrier wait of
the tensor-core kernels, made to run out on a barrier that nothing arrives
on, records DCT_ERR_DEVICE_TIMEOUT and returns; the context stays usable (a
solve right after it is exact)."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from simpeg_dc_torch_b200 import _native as nat
from simpeg_dc_torch_b200 import make_solver

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_context_survives(cuda):
    code, done = C.c_int32(0), C.c_int32(-1)
    st = torch.cuda.current_stream(cuda).cuda_stream
    rc = nat.lib().dct_selftest_wait_timeout(64, C.byref(code), C.byref(done), st)
    assert rc == 0
    assert code.value == 9          # DCT_ERR_DEVICE_TIMEOUT
    assert done.value == 0
    # the context still runs kernels correctly
    n = 50
    A = sp.diags([-np.ones(n - 1), 2.5 * np.ones(n), -np.ones(n - 1)], [-1, 0, 1]).tocsr()
    A.sort_indices()
    s = make_solver(torch.tensor(A.indptr, dtype=torch.int32),
                    torch.tensor(A.indices, dtype=torch.int32), n, 1, device=cuda)
    s.factorize(torch.tensor(A.data, device=cuda))
    b = np.arange(n, dtype=float)
    x = s.solve(torch.tensor(b, device=cuda)).cpu().numpy()
    s.check()
    assert np.linalg.norm(A @ x - b) / np.linalg.norm(b) < 1e-13


def test_selftest_rejects_bad_arguments(cuda):
    code = C.c_int32(0)
    st = torch.cuda.current_stream(cuda).cuda_stream
    assert nat.lib().dct_selftest_wait_timeout(0, C.byref(code), None, st) == 1
    assert nat.lib().dct_selftest_wait_timeout(1 << 20, C.byref(code), None, st) == 1
