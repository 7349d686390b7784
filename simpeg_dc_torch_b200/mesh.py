"""Rectilinear (tensor) meshes for the nodal DC discretisation.

`TensorMesh` carries the subset of `discretize.TensorMesh` that the engines
read: cell widths `h`, `origin`, the node/cell counts and coordinates, cell
volumes, and node interpolation.  The engines accept any tensor mesh that
exposes discretize's public `h` (per-axis cell widths) and `origin` (or the
older `x0`): `as_tensor_mesh` rebuilds it as this class, so a
`discretize.TensorMesh` can be handed to them directly.

Ordering conventions are discretize's: nodes and cells are numbered with x
fastest, then y, then z (Fortran order).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def _expand_widths(spec) -> np.ndarray:
    """Cell widths of one axis from a discretize-style spec.

    Accepts an array of widths, or a list of tuples `(dx, n)` (n cells of
    width dx) and `(dx, n, r)` (n cells growing geometrically by |r| from dx;
    r < 0 lists them in decreasing order, which is how left/bottom padding
    is written).
    """
    if isinstance(spec, np.ndarray) or (
            isinstance(spec, (list, tuple)) and len(spec) > 0
            and np.isscalar(spec[0])):
        return np.asarray(spec, dtype=float)
    out = []
    for item in spec:
        if np.isscalar(item):
            out.append(np.array([float(item)]))
            continue
        dx, n = float(item[0]), int(item[1])
        if len(item) == 2:
            out.append(np.full(n, dx))
        else:
            r = float(item[2])
            w = dx * abs(r) ** np.arange(1, n + 1)
            out.append(w[::-1] if r < 0 else w)
    return np.concatenate(out) if out else np.zeros(0)


class TensorMesh:
    """A 2-D or 3-D tensor mesh.

    Parameters
    ----------
    h : list of per-axis width specs (see `_expand_widths`).
    origin : per-axis origin; a number, or "0" (start at 0), "C" (centred on
        0), "N" (ending at 0).  A string such as "CN" gives one letter per axis.
    """

    _meshType = "TENSOR"

    def __init__(self, h, origin=None):
        self.h = [_expand_widths(s) for s in h]
        self.dim = len(self.h)
        if self.dim not in (2, 3):
            raise ValueError("TensorMesh supports 2 or 3 dimensions")
        if origin is None:
            origin = [0.0] * self.dim
        if isinstance(origin, str):
            origin = list(origin)
        o = []
        for ax, val in enumerate(origin):
            ext = float(self.h[ax].sum())
            if isinstance(val, str):
                o.append({"0": 0.0, "C": -0.5 * ext, "N": -ext}[val.upper()])
            else:
                o.append(float(val))
        self.origin = np.asarray(o, dtype=float)

    # ------------------------------------------------------------ counts
    @property
    def shape_cells(self):
        return tuple(len(w) for w in self.h)

    @property
    def shape_nodes(self):
        return tuple(len(w) + 1 for w in self.h)

    @property
    def nC(self):
        return int(np.prod(self.shape_cells))

    n_cells = nC

    @property
    def n_nodes(self):
        return int(np.prod(self.shape_nodes))

    # ------------------------------------------------------- coordinates
    def _axis_nodes(self, ax):
        return self.origin[ax] + np.r_[0.0, np.cumsum(self.h[ax])]

    def _axis_centers(self, ax):
        n = self._axis_nodes(ax)
        return 0.5 * (n[1:] + n[:-1])

    @property
    def nodes_x(self):
        return self._axis_nodes(0)

    @property
    def nodes_y(self):
        return self._axis_nodes(1)

    @property
    def nodes_z(self):
        return self._axis_nodes(2)

    @property
    def nodes(self):
        g = np.meshgrid(*[self._axis_nodes(a) for a in range(self.dim)],
                        indexing="ij")
        return np.column_stack([x.reshape(-1, order="F") for x in g])

    @property
    def cell_centers(self):
        g = np.meshgrid(*[self._axis_centers(a) for a in range(self.dim)],
                        indexing="ij")
        return np.column_stack([x.reshape(-1, order="F") for x in g])

    @property
    def cell_volumes(self):
        v = self.h[0]
        for ax in range(1, self.dim):
            v = np.multiply.outer(v, self.h[ax])
        return v.reshape(-1, order="F")

    @property
    def h_gridded(self):
        """Cell widths (nC, dim), cell order (first axis fastest)."""
        g = np.meshgrid(*self.h, indexing="ij")
        return np.column_stack([x.reshape(-1, order="F") for x in g])

    def point2index(self, locs):
        """Index of the cell holding each point (nP, dim): along each axis the
        cell [x_i, x_{i+1}) that contains the coordinate, the last cell for
        the far boundary."""
        locs = np.atleast_2d(np.asarray(locs, float))
        idx = np.zeros(locs.shape[0], dtype=np.int64)
        stride = 1
        for ax in range(self.dim):
            nodes = self._axis_nodes(ax)
            i = np.searchsorted(nodes, locs[:, ax], side="right") - 1
            i = np.clip(i, 0, len(self.h[ax]) - 1)
            idx += i * stride
            stride *= len(self.h[ax])
        return idx

    def node_grid_index(self):
        """Integer (i, j[, k]) grid coordinates of every node, node order."""
        g = np.meshgrid(*[np.arange(n) for n in self.shape_nodes],
                        indexing="ij")
        return np.column_stack([x.reshape(-1, order="F") for x in g]).astype(
            np.int32)

    # ------------------------------------------------------ interpolation
    def get_interpolation_matrix(self, locs, location_type="N"):
        """Multilinear interpolation from nodes to `locs` (npts, dim), CSR.

        Points outside the mesh raise ValueError.  Only nodal interpolation is
        needed by the DC engines.
        """
        if location_type not in ("N", "nodes"):
            raise NotImplementedError("only nodal interpolation is provided")
        locs = np.atleast_2d(np.asarray(locs, dtype=float))[:, :self.dim]
        npts = locs.shape[0]
        shape = self.shape_nodes
        idx_lists, w_lists = [], []
        for ax in range(self.dim):
            xn = self._axis_nodes(ax)
            x = locs[:, ax]
            tol = 1e-9 * max(1.0, float(np.abs(xn).max()))
            if np.any(x < xn[0] - tol) or np.any(x > xn[-1] + tol):
                raise ValueError("interpolation point outside the mesh")
            i = np.clip(np.searchsorted(xn, x, side="right") - 1, 0,
                        len(xn) - 2)
            t = np.clip((x - xn[i]) / (xn[i + 1] - xn[i]), 0.0, 1.0)
            idx_lists.append((i, i + 1))
            w_lists.append((1.0 - t, t))
        rows, cols, vals = [], [], []
        for corner in range(2 ** self.dim):
            flat = np.zeros(npts, dtype=np.int64)
            w = np.ones(npts)
            stride = 1
            for ax in range(self.dim):
                bit = (corner >> ax) & 1
                flat += idx_lists[ax][bit] * stride
                w = w * w_lists[ax][bit]
                stride *= shape[ax]
            rows.append(np.arange(npts))
            cols.append(flat)
            vals.append(w)
        P = sp.csr_matrix((np.concatenate(vals),
                           (np.concatenate(rows), np.concatenate(cols))),
                          shape=(npts, self.n_nodes))
        P.eliminate_zeros()
        P.sum_duplicates()
        return P


def as_tensor_mesh(mesh):
    """This package's TensorMesh for `mesh`: the mesh itself, or a rebuild of
    any tensor mesh that exposes discretize's public `h` (per-axis widths)
    and `origin` (or `x0`), such as `discretize.TensorMesh`
    (dctorch/simulation2d.py:37-40 and simulation3d.py:47-48 take those).
    This package's `TreeMesh` passes through; other mesh types (a discretize
    `TreeMesh`, ...) raise NotImplementedError."""
    if isinstance(mesh, TensorMesh):
        return mesh
    from .treemesh import TreeMesh
    if isinstance(mesh, TreeMesh):
        return mesh          # this package's tree meshes pass through
    kind = str(getattr(mesh, "_meshType", "TENSOR")).upper()
    if kind != "TENSOR" or not hasattr(mesh, "h"):
        raise NotImplementedError(
            f"only tensor meshes are supported (got {type(mesh).__name__})")
    origin = getattr(mesh, "origin", None)
    if origin is None:
        origin = getattr(mesh, "x0", None)
    h = [np.asarray(w, dtype=float).reshape(-1) for w in mesh.h]
    return TensorMesh(h, origin=None if origin is None
                      else [float(v) for v in np.asarray(origin, float)])
