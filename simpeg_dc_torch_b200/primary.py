"""Analytic primary potential for singularity removal in the 2.5-D engine.

A point current I on the surface of a homogeneous half space of resistivity
rho has, in the wavenumber domain, the potential rho I / pi * K_0(ky r)
(the whole-space 1/(2 pi) doubled by the image in the free surface).  The
singularity-removed formulation (dctorch/singularity.py:1-44) writes the
field as u = u_p + u_s with u_p that potential and solves

    A(sigma) u_s = A(1) u_1 - A(sigma) (rho_s u_1),    u = rho_s u_1 + u_s,

u_1 the unit-resistivity primary and rho_s the background of source s (the
model's resistivity in the cell holding its A electrode, or a fixed value).
At the source node itself, where K_0 diverges, the value is the mean of K_0
over a disc of the cell's area, 2 (1 - a K_1(a)) / a^2 with a = ky R and
R = sqrt(area / pi) (an exact integral: d/da [-a K_1(a)] = a K_0(a)).

The total field equals A(sigma)^{-1} A(1) u_1 whatever rho_s is, and A(1)
u_1 does not depend on the model, so the adjoint of the plain formulation,
contracted with the total field, is also the adjoint of this one.
"""
from __future__ import annotations

import numpy as np

from .survey import source_electrodes


def unit_primary(mesh, survey, kys):
    """u_1: the unit-resistivity primary at every node, (nky, nN, nS)."""
    from scipy.special import k0, k1

    nodes = np.asarray(mesh.nodes, float)
    kys = np.asarray(kys, float)
    widths = np.asarray(mesh.h_gridded, float)
    tol = 1e-9 * max(1.0, float(np.abs(nodes).max()))
    srcs = survey.source_list
    out = np.zeros((kys.size, nodes.shape[0], len(srcs)))
    for j, src in enumerate(srcs):
        a, b = source_electrodes(src)
        poles = [(a, 1.0)] + ([] if b is None else [(b, -1.0)])
        for loc, sign in poles:
            r = np.hypot(nodes[:, 0] - loc[0], nodes[:, 1] - loc[1])
            on_node = r < tol
            cell = int(np.atleast_1d(mesh.point2index(loc[None, :2]))[0])
            radius = float(np.sqrt(np.prod(widths[cell]) / np.pi))
            for ik, ky in enumerate(kys):
                col = k0(np.maximum(ky * r, 1e-300)) / np.pi
                if on_node.any():
                    a = ky * radius
                    col[on_node] = 2.0 * (1.0 - a * k1(a)) / (a * a) / np.pi
                out[ik, :, j] += sign * col
    return out


def source_cells(mesh, survey):
    """Cell holding each source's A electrode, (nS,)."""
    return np.array([int(np.atleast_1d(mesh.point2index(
        source_electrodes(s)[0][None, :2]))[0]) for s in survey.source_list],
        dtype=np.int64)
