"""simpeg_dc_torch_b200 -- the dctorch DC forward + adjoint hot path on B200.

A from-scratch sm_100a implementation (sparse supernodal Cholesky, multi-RHS
substitution, fused assembly / projection / adjoint kernels) behind the
reference's solver and engine interfaces:

    make_solver, make_batch_solver, DCTSolver, DCTBatchSolver,
    sparse_solve, sparse_solve_batch, sparse_solve_batch_prefactored,
    TorchDC2D, TorchDC3D, Linearization2D,
    TorchIP2D, TorchIP3D (linearized IP), TorchDCIP2D (joint DC + IP),
    TorchCR2D (complex resistivity, complex-symmetric systems),
    TorchDC2DBatch (many uneven 2.5-D surveys in the same launches),
    GraphedMisfitGrad (an engine's eval + gradient replayed from a CUDA graph)

Mesh/survey helpers (`TensorMesh`, `TreeMesh` -- octree / quadtree with
hanging nodes --, `Survey`, sources, receivers) stand in for discretize /
SimPEG objects.  The engines also take a discretize
`TensorMesh` (or any tensor mesh with its public `h` and `origin`) and
SimPEG-shaped DC surveys (`source_list`, `location_a/b`, `locations_m/n`,
`current`), reading only those public attributes.
"""
__version__ = "0.1.0"

from .mesh import TensorMesh  # noqa: F401
from .treemesh import TreeMesh  # noqa: F401
from .survey import (DipoleReceiver, DipoleSource, PoleReceiver,  # noqa: F401
                     PoleSource, Survey)
from .solver import (CuDSSBatchSolver, CuDSSSolver, DCTBatchSolver,  # noqa: F401
                     DCTSolver, make_batch_solver, make_solver, sparse_solve,
                     sparse_solve_batch, sparse_solve_batch_prefactored)
from .simulation2d import Linearization2D, TorchDC2D  # noqa: F401
from .simulation3d import TorchDC3D  # noqa: F401
from .ip import TorchIP2D, TorchIP3D  # noqa: F401
from .dcip import TorchDCIP2D  # noqa: F401
from .cr2d import TorchCR2D  # noqa: F401
from .batch import TorchDC2DBatch  # noqa: F401
from .graphs import GraphedMisfitGrad  # noqa: F401
