"""Build-time operators of the nodal DC discretisation on a tensor mesh.

The reference obtains these by running stock SimPEG once and reading its
matrices back (dctorch/simulation2d.py:141-270, dctorch/simulation3d.py:84-195).
SimPEG is not a dependency here, so the same matrices are assembled directly
from the mesh.  Every system-matrix value is linear in the cell conductivity
sigma, and the decomposition is the reference's own
(dctorch/simulation2d.py:217-219):

    A(ky).data = L_ky @ sigma,   L_ky = L_edge + ky^2 L_node + L_bc(ky)
    A.data     = L3 @ sigma,     L3   = L_edge + L_bc              (3-D)

with
  * L_edge : Grad^T diag(Me(sigma)) Grad scattered onto A's CSR entries.
    Me is the diagonal edge inner product of a tensor mesh with isotropic
    sigma, Me_e = sum over the cells touching edge e of vol_c sigma_c /
    2^(dim-1), and Grad the nodal gradient (difference / edge length).
  * L_node : the nodal mass aveN2CC^T diag(vol) on the diagonal (each cell
    gives vol_c / 2^dim to each of its corner nodes).
  * L_bc   : the mixed (Robin) boundary term diag(AvgBC @ sigma) on the
    diagonal.  On every boundary face but the top one, alpha_f =
    ky K1(ky r)/K0(ky r) (r_hat . n) in 2.5-D and (r_hat . n) / r in 3-D,
    r measured from the top-centre of the mesh; the face contributes
    alpha_f area_f sigma_(adjacent cell) / (nodes per face) to each of its
    nodes.
  * q      : one column per source, I (P_A - P_B) through nodal
    interpolation;  Pd : the stacked receiver projections P_M - P_N with
    `sidx` giving the source of each datum, in survey order.

Node, cell and CSR orderings follow discretize (x fastest).  The CSR pattern
is the nodal 5-point (2-D) / 7-point (3-D) stencil with sorted columns.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp
from scipy.special import k0e, k1e

from .mesh import as_tensor_mesh
from .survey import receiver_projection, source_term


@dataclass
class NodalOperators:
    dim: int
    nC: int
    nN: int
    nnzA: int
    crow: np.ndarray            # (nN+1,) int32, CSR of A
    col: np.ndarray             # (nnzA,) int32
    L_edge: sp.csr_matrix       # (nnzA, nC)
    L_node: sp.csr_matrix       # (nnzA, nC)   (2.5-D only term; zero use in 3-D)
    bc_faces: dict              # geometry of the Robin term (see _boundary_faces)
    q: sp.csc_matrix            # (nN, nS)
    Pd: sp.csr_matrix           # (nD, nN)
    sidx: np.ndarray            # (nD,) int64
    extra: dict = field(default_factory=dict)

    @property
    def nS(self):
        return self.q.shape[1]

    @property
    def nD(self):
        return self.Pd.shape[0]

    # ------------------------------------------------------------ per-ky maps
    def L_bc(self, ky=None) -> sp.csr_matrix:
        """Robin term: (nnzA, nC).  `ky=None` gives the 3-D coefficient."""
        f = self.bc_faces
        r, rdn = f["r"], f["r_dot_n"]
        alpha = np.zeros_like(r)
        nt = f["not_top"]
        if ky is None:
            alpha[nt] = (rdn / r)[nt]
        else:
            kr = ky * r
            alpha[nt] = (ky * k1e(kr) / k0e(kr) * rdn)[nt]
        coef = alpha * f["area"] / f["nodes"].shape[1]
        npf = f["nodes"].shape[1]
        if "exp_pos" in f:
            # tree meshes: each face's corner terms through the hanging-node
            # interpolation (entries off the diagonal included)
            fc = f["exp_face"]
            return sp.csr_matrix((coef[fc] * f["exp_w"], (f["exp_pos"], f["cell"][fc])),
                                 shape=(self.nnzA, self.nC))
        rows = np.repeat(f["diag_pos"], 1).reshape(-1)
        vals = np.repeat(coef, npf)
        cells = np.repeat(f["cell"], npf)
        return sp.csr_matrix((vals, (rows, cells)), shape=(self.nnzA, self.nC))

    def L_ky(self, ky) -> sp.csr_matrix:
        return (self.L_edge + (ky ** 2) * self.L_node + self.L_bc(ky)).tocsr()

    def L3(self) -> sp.csr_matrix:
        return (self.L_edge + self.L_bc(None)).tocsr()

    def A(self, sigma, ky=None):
        """The assembled system matrix (scipy CSR) at conductivity sigma."""
        L = self.L3() if ky is None else self.L_ky(ky)
        return sp.csr_matrix((L @ sigma, self.col, self.crow),
                             shape=(self.nN, self.nN))


def _node_index(shape_nodes, idx):
    """Flat node id from per-axis integer index arrays (x fastest)."""
    flat = np.zeros_like(idx[0], dtype=np.int64)
    stride = 1
    for ax, n in enumerate(shape_nodes):
        flat = flat + idx[ax].astype(np.int64) * stride
        stride *= n
    return flat


def _cell_index(shape_cells, idx):
    flat = np.zeros_like(idx[0], dtype=np.int64)
    stride = 1
    for ax, n in enumerate(shape_cells):
        flat = flat + idx[ax].astype(np.int64) * stride
        stride *= n
    return flat


def _edges(mesh):
    """All edges as (node_a, node_b, axis, length, per-axis node index)."""
    sn = mesh.shape_nodes
    out = []
    for ax in range(mesh.dim):
        rng = [np.arange(n - 1 if a == ax else n) for a, n in enumerate(sn)]
        g = np.meshgrid(*rng, indexing="ij")
        g = [x.reshape(-1, order="F") for x in g]
        a = _node_index(sn, g)
        gb = list(g)
        gb[ax] = gb[ax] + 1
        b = _node_index(sn, gb)
        out.append((a, b, ax, mesh.h[ax][g[ax]], g))
    return out


def _pattern(mesh, edges):
    nN = mesh.n_nodes
    r = [np.arange(nN)]
    c = [np.arange(nN)]
    for a, b, *_ in edges:
        r += [a, b]
        c += [b, a]
    r = np.concatenate(r)
    c = np.concatenate(c)
    P = sp.csr_matrix((np.ones(r.size), (r, c)), shape=(nN, nN))
    P.sort_indices()
    return P.indptr.astype(np.int64), P.indices.astype(np.int64)


def _boundary_faces(mesh, pos_of):
    """Boundary faces: centre, outward normal, area, adjacent cell, nodes."""
    dim = mesh.dim
    sn, sc = mesh.shape_nodes, mesh.shape_cells
    cen, nrm, area, cell, nodes, top = [], [], [], [], [], []
    centers = [mesh._axis_centers(a) for a in range(dim)]
    coords = [mesh._axis_nodes(a) for a in range(dim)]
    for ax in range(dim):
        others = [a for a in range(dim) if a != ax]
        for side in (0, 1):
            ia = 0 if side == 0 else sn[ax] - 1
            ca = 0 if side == 0 else sc[ax] - 1
            g = np.meshgrid(*[np.arange(sc[a]) for a in others], indexing="ij")
            g = [x.reshape(-1, order="F") for x in g]
            nf = g[0].size
            cidx = [None] * dim
            cidx[ax] = np.full(nf, ca)
            ctr = np.zeros((nf, dim))
            ctr[:, ax] = coords[ax][ia]
            ar = np.ones(nf)
            for k, a in enumerate(others):
                cidx[a] = g[k]
                ctr[:, a] = centers[a][g[k]]
                ar = ar * mesh.h[a][g[k]]
            nv = np.zeros((nf, dim))
            nv[:, ax] = -1.0 if side == 0 else 1.0
            corner_nodes = []
            for corner in range(2 ** (dim - 1)):
                nidx = [None] * dim
                nidx[ax] = np.full(nf, ia)
                for k, a in enumerate(others):
                    nidx[a] = g[k] + ((corner >> k) & 1)
                corner_nodes.append(_node_index(sn, nidx))
            cen.append(ctr)
            nrm.append(nv)
            area.append(ar)
            cell.append(_cell_index(sc, cidx))
            nodes.append(np.column_stack(corner_nodes))
            top.append(np.full(nf, ax == dim - 1 and side == 1))
    cen = np.vstack(cen)
    nrm = np.vstack(nrm)
    nodes = np.vstack(nodes)
    nodes_all = mesh.nodes
    middle = np.median(nodes_all, axis=0)
    top_v = np.max(nodes_all[:, -1])
    src_pt = np.r_[middle[:-1], top_v]
    rv = cen - src_pt
    r = np.linalg.norm(rv, axis=-1)
    rdn = np.einsum("ij,ij->i", rv / r[:, None], nrm)
    return {
        "r": r, "r_dot_n": rdn, "area": np.concatenate(area),
        "cell": np.concatenate(cell), "nodes": nodes,
        "not_top": ~np.concatenate(top),
        "diag_pos": pos_of(nodes.reshape(-1), nodes.reshape(-1)),
    }


def nodal_operators(mesh, survey) -> NodalOperators:
    """Assemble the sigma-linear maps, sources and receivers for a tensor mesh
    (this package's, or any with discretize's public `h` and `origin`) or a
    `TreeMesh` of this package."""
    from .treemesh import TreeMesh
    if isinstance(mesh, TreeMesh):
        return tree_nodal_operators(mesh, survey)
    mesh = as_tensor_mesh(mesh)
    dim = mesh.dim
    nC, nN = mesh.nC, mesh.n_nodes
    edges = _edges(mesh)
    indptr, indices = _pattern(mesh, edges)
    nnzA = indices.size
    rows_of = np.repeat(np.arange(nN, dtype=np.int64), np.diff(indptr))
    keys = rows_of * nN + indices

    def pos_of(r, c):
        k = np.asarray(r, np.int64) * nN + np.asarray(c, np.int64)
        p = np.searchsorted(keys, k)
        if not np.all(keys[p] == k):
            raise AssertionError("entry missing from the A pattern")
        return p

    # ---- Grad^T diag(Me) Grad : per edge, per adjacent cell
    sc = mesh.shape_cells
    vol = mesh.cell_volumes
    share = 1.0 / 2 ** (dim - 1)
    R, Cc, V = [], [], []
    for a, b, ax, length, g in edges:
        others = [o for o in range(dim) if o != ax]
        p_ab, p_ba = pos_of(a, b), pos_of(b, a)
        p_aa, p_bb = pos_of(a, a), pos_of(b, b)
        for corner in range(2 ** (dim - 1)):
            cidx = [None] * dim
            cidx[ax] = g[ax]
            ok = np.ones(a.size, dtype=bool)
            for k, o in enumerate(others):
                ci = g[o] - 1 + ((corner >> k) & 1)
                ok &= (ci >= 0) & (ci < sc[o])
                cidx[o] = np.clip(ci, 0, sc[o] - 1)
            cell = _cell_index(sc, cidx)[ok]
            w = (share * vol[cell]) / length[ok] ** 2
            for p, s in ((p_ab, -1.0), (p_ba, -1.0), (p_aa, 1.0), (p_bb, 1.0)):
                R.append(p[ok])
                Cc.append(cell)
                V.append(s * w)
    L_edge = sp.csr_matrix((np.concatenate(V), (np.concatenate(R),
                                                 np.concatenate(Cc))),
                           shape=(nnzA, nC))
    L_edge.sum_duplicates()
    L_edge.sort_indices()

    # ---- nodal mass aveN2CC^T diag(vol): each cell -> its 2^dim corners
    cg = np.meshgrid(*[np.arange(n) for n in sc], indexing="ij")
    cg = [x.reshape(-1, order="F") for x in cg]
    cells = _cell_index(sc, cg)
    R, Cc, V = [], [], []
    for corner in range(2 ** dim):
        nidx = [cg[ax] + ((corner >> ax) & 1) for ax in range(dim)]
        nd = _node_index(mesh.shape_nodes, nidx)
        R.append(pos_of(nd, nd))
        Cc.append(cells)
        V.append(vol[cells] / 2 ** dim)
    L_node = sp.csr_matrix((np.concatenate(V), (np.concatenate(R),
                                                 np.concatenate(Cc))),
                           shape=(nnzA, nC))
    L_node.sum_duplicates()
    L_node.sort_indices()

    bcf = _boundary_faces(mesh, pos_of)

    # ---- sources (dense columns are tiny: a few nodes each) and receivers
    qcols = [sp.csc_matrix(source_term(src, mesh).reshape(-1, 1))
             for src in survey.source_list]
    q = sp.hstack(qcols).tocsc() if qcols else sp.csc_matrix((nN, 0))
    Pb, sidx = [], []
    for isrc, src in enumerate(survey.source_list):
        for rx in src.receiver_list:
            P = receiver_projection(rx, mesh)
            Pb.append(P)
            sidx += [isrc] * P.shape[0]
    Pd = sp.vstack(Pb).tocsr() if Pb else sp.csr_matrix((0, nN))
    Pd.sort_indices()
    return NodalOperators(
        dim=dim, nC=nC, nN=nN, nnzA=nnzA,
        crow=indptr.astype(np.int32), col=indices.astype(np.int32),
        L_edge=L_edge, L_node=L_node, bc_faces=bcf, q=q, Pd=Pd,
        sidx=np.asarray(sidx, dtype=np.int64))


# ------------------------------------------------------------------ trees
def _outer_entries(G, weights):
    """For every row r of the sparse G (rows x n): the entries
    weights[r] * G[r, i] * G[r, j] of the rank-one term G[r]^T G[r], as
    (i, j, value, r) arrays."""
    G = sp.csr_matrix(G)
    G.sum_duplicates()
    nnz_row = np.diff(G.indptr)
    I, J, V, R = [], [], [], []
    for k in np.unique(nnz_row):
        if k == 0:
            continue
        rows = np.flatnonzero(nnz_row == k)
        starts = G.indptr[rows]
        idx = starts[:, None] + np.arange(k)[None, :]
        cols = G.indices[idx]
        vals = G.data[idx]
        cols = cols.astype(np.int64)          # i n + j keys exceed 32 bits
        I.append(np.repeat(cols, k, axis=1).reshape(-1))
        J.append(np.tile(cols, (1, k)).reshape(-1))
        V.append((vals[:, :, None] * vals[:, None, :] * weights[rows][:, None, None]).reshape(-1))
        R.append(np.repeat(rows, k * k))
    if not I:
        e = np.zeros(0, np.int64)
        return e, e, np.zeros(0), e
    return np.concatenate(I), np.concatenate(J), np.concatenate(V), np.concatenate(R)


def tree_nodal_operators(mesh, survey) -> NodalOperators:
    """The sigma-linear maps, sources and receivers on a `TreeMesh`: the
    tensor-mesh operators cell by cell on all leaf corners, mapped to the
    free nodes through the hanging-node interpolation P (see treemesh.py)."""
    from .treemesh import TreeMesh
    if not isinstance(mesh, TreeMesh) or not mesh._final:
        raise ValueError("a finalized TreeMesh is expected")
    dim = mesh.dim
    nC, nN = mesh.nC, mesh.n_nodes
    Pm = mesh.P.tocsr()
    n_all = Pm.shape[0]
    cn = mesh._cell_nodes                     # (nC, 2^dim) all-node ids, x fastest
    size = mesh._cell_size
    vol = mesh.cell_volumes
    # ---- element edges: rows (cell, edge), G = (E1 - E0) P
    e0, e1, wts, cells = [], [], [], []
    for ax in range(dim):
        ln = size * mesh.h0[ax]
        for k in range(2 ** dim):
            if (k >> ax) & 1:
                continue
            e0.append(cn[:, k])
            e1.append(cn[:, k | (1 << ax)])
            wts.append(vol / 2 ** (dim - 1) / ln ** 2)
            cells.append(np.arange(nC))
    e0, e1 = np.concatenate(e0), np.concatenate(e1)
    wts, cells = np.concatenate(wts), np.concatenate(cells)
    nr = e0.size
    E = sp.csr_matrix((np.r_[np.ones(nr), -np.ones(nr)],
                       (np.r_[np.arange(nr), np.arange(nr)], np.r_[e1, e0])),
                      shape=(nr, n_all))
    G = (E @ Pm).tocsr()
    gi, gj, gv, gr = _outer_entries(G, wts)
    # ---- nodal mass: rows (cell, corner), vector P[corner]
    Mr = sp.csr_matrix((np.ones(nC * 2 ** dim), (np.arange(nC * 2 ** dim), cn.reshape(-1))),
                       shape=(nC * 2 ** dim, n_all))
    Nm = (Mr @ Pm).tocsr()
    mw = np.repeat(vol / 2 ** dim, 2 ** dim)
    mi, mj, mv, mr = _outer_entries(Nm, mw)
    mcell = mr // (2 ** dim)
    # ---- boundary faces (all but the top): geometry and corner vectors
    nf = mesh.n_finest
    lo = mesh._cell_lo
    fcell, fctr, fnrm, farea, fnodes, ftop = [], [], [], [], [], []
    for ax in range(dim):
        others = [o for o in range(dim) if o != ax]
        for side in (0, 1):
            on = (lo[:, ax] == 0) if side == 0 else (lo[:, ax] + size == nf)
            c = np.flatnonzero(on)
            if c.size == 0:
                continue
            ctr = mesh.origin + (lo[c] + 0.5 * size[c, None]) * mesh.h0
            ctr[:, ax] = mesh.origin[ax] + (0 if side == 0 else nf) * mesh.h0[ax]
            nv = np.zeros((c.size, dim))
            nv[:, ax] = -1.0 if side == 0 else 1.0
            ar = np.ones(c.size)
            for o in others:
                ar = ar * size[c] * mesh.h0[o]
            ks = [k for k in range(2 ** dim) if ((k >> ax) & 1) == side]
            fcell.append(c)
            fctr.append(ctr)
            fnrm.append(nv)
            farea.append(ar)
            fnodes.append(cn[c][:, ks])
            ftop.append(np.full(c.size, ax == dim - 1 and side == 1))
    fcell = np.concatenate(fcell)
    fctr, fnrm = np.vstack(fctr), np.vstack(fnrm)
    farea, fnodes = np.concatenate(farea), np.vstack(fnodes)
    ftop = np.concatenate(ftop)
    npf = fnodes.shape[1]
    Fr = sp.csr_matrix((np.ones(fnodes.size), (np.arange(fnodes.size), fnodes.reshape(-1))),
                       shape=(fnodes.size, n_all))
    Fm = (Fr @ Pm).tocsr()
    bi, bj, bv, br = _outer_entries(Fm, np.ones(fnodes.size))
    bface = br // npf
    # ---- the A pattern: every entry any term touches, plus the diagonal
    keys = np.unique(np.concatenate([gi * nN + gj, mi * nN + mj, bi * nN + bj,
                                     np.arange(nN, dtype=np.int64) * (nN + 1)]))
    rows_k, cols_k = keys // nN, keys % nN
    indptr = np.zeros(nN + 1, np.int64)
    np.add.at(indptr, rows_k + 1, 1)
    indptr = np.cumsum(indptr)
    nnzA = keys.size

    def pos(i, j):
        return np.searchsorted(keys, np.asarray(i, np.int64) * nN + np.asarray(j, np.int64))

    L_edge = sp.csr_matrix((gv, (pos(gi, gj), cells[gr])), shape=(nnzA, nC))
    L_edge.sum_duplicates()
    L_edge.sort_indices()
    L_node = sp.csr_matrix((mv, (pos(mi, mj), mcell)), shape=(nnzA, nC))
    L_node.sum_duplicates()
    L_node.sort_indices()
    nodes_all = mesh.nodes
    middle = np.median(nodes_all, axis=0)
    src_pt = np.r_[middle[:-1], np.max(nodes_all[:, -1])]
    rv = fctr - src_pt
    r = np.linalg.norm(rv, axis=-1)
    rdn = np.einsum("ij,ij->i", rv / r[:, None], fnrm)
    bcf = {"r": r, "r_dot_n": rdn, "area": farea, "cell": fcell,
           "nodes": fnodes, "not_top": ~ftop,
           # the P-mapped corner terms: entry, face, weight
           "exp_pos": pos(bi, bj), "exp_face": bface, "exp_w": bv}
    qcols = [sp.csc_matrix(source_term(src, mesh).reshape(-1, 1))
             for src in survey.source_list]
    q = sp.hstack(qcols).tocsc() if qcols else sp.csc_matrix((nN, 0))
    Pb, sidx = [], []
    for isrc, src in enumerate(survey.source_list):
        for rx in src.receiver_list:
            P = receiver_projection(rx, mesh)
            Pb.append(P)
            sidx += [isrc] * P.shape[0]
    Pd = sp.vstack(Pb).tocsr() if Pb else sp.csr_matrix((0, nN))
    Pd.sort_indices()
    return NodalOperators(
        dim=dim, nC=nC, nN=nN, nnzA=nnzA,
        crow=indptr.astype(np.int32), col=cols_k.astype(np.int32),
        L_edge=L_edge, L_node=L_node, bc_faces=bcf, q=q, Pd=Pd,
        sidx=np.asarray(sidx, dtype=np.int64))
