"""Octree (3-D) and quadtree (2-D) meshes with hanging nodes, for the nodal
DC operators on refined meshes (the reference extracts them from SimPEG on a
discretize TreeMesh, dctorch/simulation2d.py:173-195, simulation3d.py:
103-121; neither package is available here, so the mesh and its operators
are built directly).

A `TreeMesh` covers a box of 2**max_level finest cells per axis (finest
widths h0 per axis).  Leaves are cells (level l, index i per axis) covering
finest indices [i 2**(max_level-l), (i+1) 2**(max_level-l)); level 0 is the
whole box.  `refine(fn)` splits leaves until each reaches the level fn gives
for it; `finalize()` enforces the 2:1 balance across faces, edges and
corners and numbers cells and nodes.

Nodes are the corners of the leaves.  A corner that lies inside an edge or a
face of a coarser leaf is hanging: its value is the linear interpolation of
that edge's two end nodes or that face's four corners (applied recursively
when those are hanging in turn), so the potential stays continuous.  The free
(non-hanging) nodes are the unknowns; `P` (all nodes x free nodes) is the
interpolation.  The nodal operators follow the tensor-mesh ones cell by cell
(every leaf gives each of its edges vol sigma / 2**(dim-1) / len**2 of
Grad^T Me Grad, each of its corners vol / 2**dim of the nodal mass, each of
its boundary faces the Robin term), assembled on all nodes and mapped to the
free ones by P^T (.) P.  On a tree whose leaves all share one level they are
the tensor mesh's own.
"""
from __future__ import annotations

import itertools

import numpy as np
import scipy.sparse as sp


class TreeMesh:
    """2:1 balanced tree mesh.

    h       : per axis, the finest cell width (a number) and, optionally, the
              number of finest cells (a power of two, equal on all axes);
              given as [(h0, n)] per axis, or h0 values with max_level.
    origin  : the box's lowest corner.
    """

    def __init__(self, h, origin=None, max_level=None):
        h0, ns = [], []
        for a in h:
            if np.ndim(a) == 0:
                h0.append(float(a))
                ns.append(None)
            else:
                w, n = a
                h0.append(float(w))
                ns.append(int(n))
        self.dim = len(h0)
        if max_level is None:
            n = ns[0]
            if n is None or any(x != n for x in ns):
                raise ValueError("give max_level or the same power-of-two count on every axis")
            max_level = int(round(np.log2(n)))
            if 2 ** max_level != n:
                raise ValueError("the number of finest cells must be a power of two")
        self.max_level = int(max_level)
        self.h0 = np.asarray(h0, float)
        self.n_finest = 2 ** self.max_level
        self.origin = np.zeros(self.dim) if origin is None else np.asarray(origin, float)
        self._leaves = {(0,) + (0,) * self.dim}
        self._final = False

    # ------------------------------------------------------------ building
    def _extent(self, leaf):
        l, idx = leaf[0], np.asarray(leaf[1:])
        s = 2 ** (self.max_level - l)
        lo = self.origin + idx * s * self.h0
        return lo, lo + s * self.h0

    def refine(self, level_fn):
        """Split leaves until every leaf's level is at least level_fn(lo, hi)
        (arrays of its lowest and highest corner, (k, dim) batches)."""
        self._final = False
        changed = True
        while changed:
            changed = False
            leaves = np.array(sorted(self._leaves), dtype=np.int64)
            if leaves.size == 0:
                break
            s = 2 ** (self.max_level - leaves[:, 0])
            lo = self.origin + leaves[:, 1:] * (s[:, None] * self.h0)
            hi = lo + s[:, None] * self.h0
            want = np.asarray(level_fn(lo, hi), dtype=np.int64)
            split = (leaves[:, 0] < np.minimum(want, self.max_level))
            for leaf in map(tuple, leaves[split]):
                self._split(leaf)
                changed = True

    def refine_points(self, points, level, padding=0.0):
        """Leaves that come within `padding` of any of the points reach
        `level` (the test uses the leaf's bounding sphere: a leaf whose
        centre is within padding + half its diagonal of a point)."""
        from scipy.spatial import cKDTree
        pts = np.atleast_2d(np.asarray(points, float))
        kd = cKDTree(pts)

        def fn(lo, hi):
            ctr = 0.5 * (lo + hi)
            rad = 0.5 * np.linalg.norm(hi - lo, axis=1)
            d, _ = kd.query(ctr)
            return np.where(d - rad <= padding, level, 0)
        self.refine(fn)

    def _split(self, leaf):
        self._leaves.discard(leaf)
        l, idx = leaf[0], leaf[1:]
        for off in itertools.product((0, 1), repeat=self.dim):
            self._leaves.add((l + 1,) + tuple(2 * i + o for i, o in zip(idx, off)))

    def _level_map(self):
        """Level of the leaf covering every finest cell, an int8 array
        indexed [x, y(, z)] by finest-grid cell index."""
        L, dim = self.max_level, self.dim
        V = np.full((self.n_finest,) * dim, -1, dtype=np.int8)
        leaves = np.array(sorted(self._leaves), dtype=np.int64)
        for l in np.unique(leaves[:, 0]):
            sel = leaves[leaves[:, 0] == l, 1:]
            M = np.zeros((2 ** int(l),) * dim, dtype=bool)
            M[tuple(sel.T)] = True
            s = 2 ** (L - int(l))
            for a in range(dim):
                M = np.repeat(M, s, axis=a)
            V[M] = l
        return V

    def _balance(self):
        """2:1 balance: no leaf touches (face, edge or corner) a leaf more
        than one level coarser."""
        L, dim, nf = self.max_level, self.dim, self.n_finest
        offs = np.array([o for o in itertools.product((-1, 0, 1), repeat=dim) if any(o)])
        while True:
            V = self._level_map()
            leaves = np.array(sorted(self._leaves), dtype=np.int64)
            lev = leaves[:, 0]
            s = 2 ** (L - lev)
            base = leaves[:, 1:] * s[:, None]
            split = set()
            for o in offs:
                probe = np.where(o < 0, base - 1, np.where(o > 0, base + s[:, None], base))
                ok = np.all((probe >= 0) & (probe < nf), axis=1)
                pr = probe[ok]
                nl = V[tuple(pr.T)].astype(np.int64)
                bad = nl < lev[ok] - 1
                if not bad.any():
                    continue
                pb, lb = pr[bad], nl[bad]
                keys = np.column_stack([lb, pb >> (L - lb)[:, None]])
                split.update(map(tuple, np.unique(keys, axis=0)))
            if not split:
                return
            for leaf in split:
                if leaf in self._leaves:
                    self._split(leaf)

    def finalize(self):
        """Balance the tree and number its cells and nodes."""
        self._balance()
        L = self.max_level
        leaves = np.array(sorted(self._leaves), dtype=np.int64)
        s = 2 ** (L - leaves[:, 0])
        lo_f = leaves[:, 1:] * s[:, None]            # finest-grid lowest corner
        # cells in Morton order of their lowest corner (neighbours close)
        order = np.argsort(_morton(lo_f, L), kind="stable")
        self._cell_level = leaves[order, 0]
        self._cell_lo = lo_f[order]
        self._cell_size = s[order]
        code = _morton(self._cell_lo, L) * (L + 1) + self._cell_level
        self._cell_code_order = np.argsort(code, kind="stable")
        self._cell_code_sorted = code[self._cell_code_order]
        self._vmap = None
        self._final = True
        self._build_nodes()

    # ------------------------------------------------------------ geometry
    @property
    def nC(self):
        return int(self._cell_level.size)

    n_cells = nC

    @property
    def cell_centers(self):
        return self.origin + (self._cell_lo + 0.5 * self._cell_size[:, None]) * self.h0

    @property
    def cell_volumes(self):
        return np.prod(self._cell_size[:, None] * self.h0, axis=1)

    @property
    def h_gridded(self):
        return self._cell_size[:, None] * self.h0

    @property
    def cell_levels(self):
        return self._cell_level.copy()

    def _build_nodes(self):
        dim, L = self.dim, self.max_level
        corners = np.array(list(itertools.product((0, 1), repeat=dim)))[:, ::-1]  # x fastest
        all_pts = (self._cell_lo[:, None, :] + corners[None] * self._cell_size[:, None, None])
        flat = all_pts.reshape(-1, dim)
        keys = _key(flat, L)
        uniq, inv = np.unique(keys, return_inverse=True)
        self._all_nodes_f = _unkey(uniq, L, dim)        # finest-grid coords
        self._cell_nodes = inv.reshape(self.nC, 2 ** dim)
        n_all = uniq.size
        # hanging nodes: midpoints of leaf edges and centres of leaf faces
        # that are nodes of the mesh, constrained to the edge's end nodes or
        # the face's corners
        big = self._cell_size >= 2
        lo = self._cell_lo[big]
        sz = self._cell_size[big][:, None]
        half = sz // 2

        def node_of(pts):
            k = _key(pts, L)
            p = np.searchsorted(uniq, k)
            p = np.minimum(p, n_all - 1)
            return p, uniq[p] == k

        H, Cn, W = [], [], []
        for a in range(dim):
            others = [o for o in range(dim) if o != a]
            ea = np.zeros(dim, np.int64)
            ea[a] = 1
            for bits in itertools.product((0, 1), repeat=dim - 1):
                off = np.zeros(dim, np.int64)
                for o, bv in zip(others, bits):
                    off[o] = bv
                p = lo + off * sz
                m, hit = node_of(p + ea * half)
                if not hit.any():
                    continue
                e0, _ = node_of(p[hit])
                e1, _ = node_of(p[hit] + ea * sz[hit])
                for q in (e0, e1):
                    H.append(m[hit])
                    Cn.append(q)
                    W.append(np.full(q.size, 0.5))
        if dim == 3:
            for a in range(dim):
                others = [o for o in range(dim) if o != a]
                for side in (0, 1):
                    base = lo.copy()
                    base[:, a] += side * sz[:, 0]
                    ctr = base.copy()
                    for o in others:
                        ctr[:, o] += half[:, 0]
                    m, hit = node_of(ctr)
                    if not hit.any():
                        continue
                    for bits in itertools.product((0, 1), repeat=2):
                        q = base[hit].copy()
                        for o, bv in zip(others, bits):
                            q[:, o] += bv * sz[hit, 0]
                        qi, _ = node_of(q)
                        H.append(m[hit])
                        Cn.append(qi)
                        W.append(np.full(qi.size, 0.25))
        hanging = np.zeros(n_all, bool)
        if H:
            H, Cn, W = np.concatenate(H), np.concatenate(Cn), np.concatenate(W)
            # a node found hanging from several coarse cells: one constraint
            # (the same one) kept
            hanging[H] = True
            rows, first = np.unique(np.column_stack([H, Cn]), axis=0, return_index=True)
            H, Cn, W = H[first], Cn[first], W[first]
        # C: all nodes -> all nodes, identity on free nodes, the constraint
        # on hanging ones; applied until no hanging node remains on the right
        free = np.flatnonzero(~hanging)
        Cr = np.concatenate([free, H]) if len(H) else free
        Cc = np.concatenate([free, Cn]) if len(H) else free
        Cv = np.concatenate([np.ones(free.size), W]) if len(H) else np.ones(free.size)
        C = sp.csr_matrix((Cv, (Cr, Cc)), shape=(n_all, n_all))
        Pm = C.copy()
        for _ in range(64):
            if not hanging[Pm.indices].any():
                break
            Pm = (Pm @ C).tocsr()
        else:
            raise AssertionError("hanging-node constraints do not resolve")
        free_id = -np.ones(n_all, np.int64)
        free_id[free] = np.arange(free.size)
        Pm = Pm.tocoo()
        self.P = sp.csr_matrix((Pm.data, (Pm.row, free_id[Pm.col])), shape=(n_all, free.size))
        self.P.sum_duplicates()
        self._free = free
        self._hanging = hanging

    @property
    def n_nodes(self):
        return int(self._free.size)

    @property
    def nodes(self):
        """Coordinates of the free nodes (the unknowns)."""
        return self.origin + self._all_nodes_f[self._free] * self.h0

    @property
    def n_hanging_nodes(self):
        return int(self._hanging.sum())

    def node_grid_index(self):
        """Finest-grid integer coordinates of the free nodes (for the
        geometric nested dissection)."""
        return self._all_nodes_f[self._free].astype(np.int32)

    # ------------------------------------------------------------ lookup
    def cells_of_points(self, points):
        """Index of the leaf containing each point (on a shared boundary, the
        leaf on the high side)."""
        pts = np.atleast_2d(np.asarray(points, float))
        L = self.max_level
        f = np.floor((pts - self.origin) / self.h0).astype(np.int64)
        f = np.clip(f, 0, self.n_finest - 1)
        if self._vmap is None:
            self._vmap = self._level_map()
        lev = self._vmap[tuple(f.T)].astype(np.int64)
        lo = (f >> (L - lev)[:, None]) << (L - lev)[:, None]
        code = _morton(lo, L) * (L + 1) + lev
        pos = np.searchsorted(self._cell_code_sorted, code)
        if not np.all(self._cell_code_sorted[np.minimum(pos, self.nC - 1)] == code):
            raise AssertionError("point outside every leaf")
        return self._cell_code_order[pos]

    def point2index(self, locs):
        """discretize's name: the cell containing each point."""
        return self.cells_of_points(locs)

    def get_interpolation_matrix(self, locs, location_type="N"):
        """discretize's name: nodal ("N") interpolation onto the free nodes."""
        if location_type not in ("N", "nodes"):
            raise NotImplementedError("tree meshes interpolate nodal values only")
        return self.interpolation_matrix(locs)

    def interpolation_matrix(self, points):
        """(npoints, n_nodes) multilinear interpolation of the free nodal
        values at the points (through the leaf that contains each point)."""
        pts = np.atleast_2d(np.asarray(points, float))
        cells = self.cells_of_points(pts)
        dim = self.dim
        corners = np.array(list(itertools.product((0, 1), repeat=dim)))[:, ::-1]
        lo = self.origin + self._cell_lo[cells] * self.h0
        wdt = self._cell_size[cells][:, None] * self.h0
        t = np.clip((pts - lo) / wdt, 0.0, 1.0)
        R, C, V = [], [], []
        for k, cb in enumerate(corners):
            w = np.prod(np.where(cb[None] == 1, t, 1.0 - t), axis=1)
            R.append(np.arange(len(pts)))
            C.append(self._cell_nodes[cells, k])
            V.append(w)
        W = sp.csr_matrix((np.concatenate(V), (np.concatenate(R), np.concatenate(C))),
                          shape=(len(pts), self.P.shape[0]))
        return (W @ self.P).tocsr()


def _morton(f, L):
    f = np.asarray(f, np.int64)
    code = np.zeros(f.shape[0], np.int64)
    dim = f.shape[1]
    for bit in range(L + 1):
        for a in range(dim):
            code |= ((f[:, a] >> bit) & 1) << (bit * dim + a)
    return code


def _key(f, L):
    f = np.asarray(f, np.int64)
    n = (1 << L) + 1
    k = np.zeros(f.shape[0], np.int64)
    for a in range(f.shape[1] - 1, -1, -1):
        k = k * n + f[:, a]
    return k


def _unkey(k, L, dim):
    n = (1 << L) + 1
    k = np.asarray(k, np.int64).copy()
    out = np.empty((k.size, dim), np.int64)
    for a in range(dim):
        out[:, a] = k % n
        k //= n
    return out
