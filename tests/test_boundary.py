"""The drop-in boundary on a machine without a GPU: the solver factories and
the engines have no CPU path and say so (no silent fallback), and matrix
types the library does not factor are refused before any device work
(dctorch/solver.py:383-399 for the factories' signatures)."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

from simpeg_dc_torch_b200 import TorchDC2D, TorchDC3D, make_batch_solver, make_solver
from simpeg_dc_torch_b200 import synthetic as syn


def _pattern(n=50):
    A = sp.diags([np.full(n - 1, -1.0), np.full(n, 4.0), np.full(n - 1, -1.0)],
                 [-1, 0, 1], format="csr")
    return torch.as_tensor(A.indptr), torch.as_tensor(A.indices), n


@pytest.mark.parametrize("factory", ["single", "batch"])
def test_no_cpu_path(factory):
    crow, col, n = _pattern()
    with pytest.raises(NotImplementedError, match="CUDA solver path only"):
        if factory == "single":
            make_solver(crow, col, n, 2, device="cpu")
        else:
            make_batch_solver(crow, col, n, 2, 3, device="cpu")


@pytest.mark.parametrize("mt,dt", [("general", torch.float32), ("symmetric", torch.float64),
                                   ("spd", torch.complex128), ("hermitian", torch.float64)])
def test_unsupported_matrix_types_refused(mt, dt):
    crow, col, n = _pattern()
    with pytest.raises(NotImplementedError, match="matrix_type"):
        make_solver(crow, col, n, 2, device="cuda", dtype=dt, matrix_type=mt)


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU message")
def test_cuda_requested_without_a_gpu():
    crow, col, n = _pattern()
    with pytest.raises(RuntimeError, match="none is available"):
        make_solver(crow, col, n, 2, device="cuda")


def test_engines_refuse_cpu():
    mesh, survey, _ = syn.tiny_2d()
    with pytest.raises(NotImplementedError):
        TorchDC2D(mesh, survey, nky=3, device="cpu")
    mesh3, survey3, _ = syn.tiny_3d()[:3]
    with pytest.raises(NotImplementedError):
        TorchDC3D(mesh3, survey3, device="cpu")
