"""The value-gradient contraction of the fused adjoint (dct_gather_contract):
gv[b, e] = -scale[b] sum_r Y[b, iperm[row_e], r] X[b, iperm[col_e], r] against
a float64 torch evaluation, for right-hand-side counts on every kernel path
(one warp per run of entries with the row of Y in registers for k <= 64, 128,
256; one warp per entry above), entries in CSR order and shuffled, and a
batch with per-system scales (the 2.5-D quadrature weights)."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

from simpeg_dc_torch_b200 import _native as nat

pytestmark = pytest.mark.gpu


def _case(rng, n, k, nbatch, shuffle):
    A = sp.random(n, n, density=8.0 / n, random_state=rng, format="csr")
    A = (A + A.T + sp.eye(n)).tocsr()
    A.sort_indices()
    coo = A.tocoo()
    row, col = coo.row.astype(np.int32), coo.col.astype(np.int32)
    if shuffle:
        p = rng.permutation(row.size)
        row, col = row[p], col[p]
    iperm = rng.permutation(n).astype(np.int32)
    Y = rng.standard_normal((nbatch, n, k))
    X = rng.standard_normal((nbatch, n, k))
    scale = rng.uniform(0.5, 2.0, nbatch)
    return row, col, iperm, Y, X, scale


@pytest.mark.parametrize("k", [40, 100, 200, 300])
@pytest.mark.parametrize("shuffle", [False, True])
def test_gather_contract_against_torch(cuda, k, shuffle):
    rng = np.random.default_rng(k + int(shuffle))
    n, nbatch = 3000, 3
    row, col, iperm, Y, X, scale = _case(rng, n, k, nbatch, shuffle)
    t = lambda a: torch.as_tensor(a, device=cuda).contiguous()  # noqa: E731
    d_row, d_col, d_iperm = t(row), t(col), t(iperm)
    dY, dX, dscale = t(Y), t(X), t(scale)
    nnz = row.size
    gv = torch.empty(nbatch * nnz, dtype=torch.float64, device=cuda)
    nat.check(nat.lib().dct_gather_contract(
        nbatch, n, nnz, k, d_row.data_ptr(), d_col.data_ptr(), d_iperm.data_ptr(),
        dscale.data_ptr(), dY.data_ptr(), dX.data_ptr(), gv.data_ptr(),
        torch.cuda.current_stream(cuda).cuda_stream), "dct_gather_contract")
    r = d_iperm[d_row.long()].long()
    c = d_iperm[d_col.long()].long()
    ref = -(dscale.view(-1, 1) * (dY[:, r, :] * dX[:, c, :]).sum(-1)).reshape(-1)
    err = (gv - ref).abs().max() / ref.abs().max()
    assert float(err) < 1e-13
