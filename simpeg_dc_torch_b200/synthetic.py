"""Seeded synthetic DC problems (meshes, surveys, log-resistivity models).

The workloads used by the tests and the benchmark:

  * `regression_2d`     : TensorMesh 100x50 @ 1 m, 21 electrodes on -30..30 m,
                          dipole-dipole n = 1..6, a 10 ohm-m block in 100 ohm-m
                          (the reference's own regression case,
                          dctorch/tests/test_simulation2d.py:24-56).
  * `suite_case`        : the reference coverage-suite tensor cases
                          (dctorch/tests/test_suite.py:62-87): 2-D 64x32 @ 1 m
                          and 3-D 20x20x10 @ 2 m, m = log 100 + 0.3 N(0,1).
  * `dc2d_small`        : 100x50 core cells of 2.5 m + 10 padding cells (x1.3)
                          left, right and below; 21 electrodes @ 5 m;
                          dipole-dipole n = 1..6; nky = 11.
  * `dc2d_large`        : 400x120 core @ 1 m + padding (x1.3); 96 electrodes
                          @ 4 m; dipole-dipole (a = 1, n = 1..20) + Wenner
                          (a = 1); nky = 12.
  * `dc2d_batch`        : 64 independent 2.5-D problems, 5k-40k cells,
                          24-64 electrodes, dipole-dipole, nky = 12.
  * `dc3d`              : 64x64x32 core @ 5 m + 8 padding cells per face
                          (x1.3, none above); 10x10 surface grid; 200
                          pole-dipole sources with ~30 receivers each.

Models are m = log(rho): a background with seeded blocks/ellipsoids plus
N(0, 0.1^2) cell noise, as the workload definitions ask.
"""
from __future__ import annotations

import numpy as np

from .mesh import TensorMesh
from .survey import (DipoleReceiver, DipoleSource, PoleSource, Survey)


# ----------------------------------------------------------------- surveys
def dipole_dipole_2d(xe, nmax, a=1, z=0.0):
    """Dipole-dipole on electrodes xe: AB = (i, i+a), MN = (B + n a, B + (n+1) a)."""
    xe = np.asarray(xe, float)
    srcs = []
    for i in range(len(xe) - a):
        lm, ln = [], []
        for n in range(1, nmax + 1):
            jm, jn = i + a + n * a, i + a + (n + 1) * a
            if jn >= len(xe):
                break
            lm.append([xe[jm], z])
            ln.append([xe[jn], z])
        if lm:
            rx = DipoleReceiver(np.array(lm), np.array(ln))
            srcs.append(DipoleSource([rx], np.r_[xe[i], z], np.r_[xe[i + a], z]))
    return srcs


def reference_dd_survey(xe, nmax):
    """The reference tests' dipole-dipole (dctorch/tests/test_simulation2d.py:
    147-161): AB = (i, i+1), MN = (i+1+n, i+2+n), n = 1..nmax."""
    return Survey(dipole_dipole_2d(xe, nmax, a=1))


def wenner_2d(xe, a=1, z=0.0):
    xe = np.asarray(xe, float)
    srcs = []
    for i in range(len(xe) - 3 * a):
        rx = DipoleReceiver(np.array([[xe[i + a], z]]),
                            np.array([[xe[i + 2 * a], z]]))
        srcs.append(DipoleSource([rx], np.r_[xe[i], z], np.r_[xe[i + 3 * a], z]))
    return srcs


# ------------------------------------------------------------------ meshes
def padded_mesh_2d(dx, ncx, ncy, npad, growth=1.3):
    hx = [(dx, npad, -growth), (dx, ncx), (dx, npad, growth)]
    hy = [(dx, npad, -growth), (dx, ncy)]
    return TensorMesh([hx, hy], origin="CN")


def padded_mesh_3d(dx, ncx, ncy, ncz, npad, growth=1.3):
    hx = [(dx, npad, -growth), (dx, ncx), (dx, npad, growth)]
    hy = [(dx, npad, -growth), (dx, ncy), (dx, npad, growth)]
    hz = [(dx, npad, -growth), (dx, ncz)]
    return TensorMesh([hx, hy, hz], origin="CCN")


# ------------------------------------------------------------------ models
def block_model_2d(mesh, rng, core_x, core_depth, rho_bg=100.0,
                   rhos=(10.0, 1000.0), noise=0.1):
    cc = mesh.cell_centers
    m = np.full(mesh.nC, np.log(rho_bg))
    for rho in rhos:
        w = rng.uniform(0.1, 0.25) * (core_x[1] - core_x[0])
        h = rng.uniform(0.1, 0.3) * core_depth
        x0 = rng.uniform(core_x[0] + 0.1 * (core_x[1] - core_x[0]),
                         core_x[1] - 0.1 * (core_x[1] - core_x[0]) - w)
        z0 = -rng.uniform(0.05, 0.5) * core_depth
        blk = ((cc[:, 0] > x0) & (cc[:, 0] < x0 + w)
               & (cc[:, 1] < z0) & (cc[:, 1] > z0 - h))
        m[blk] = np.log(rho)
    return m + noise * rng.standard_normal(mesh.nC)


# ------------------------------------------------------------------ cases
def regression_2d():
    mesh = TensorMesh([[(1.0, 100)], [(1.0, 50)]], origin="CN")
    survey = reference_dd_survey(np.linspace(-30, 30, 21), 6)
    m = np.log(100.0) * np.ones(mesh.nC)
    cc = mesh.cell_centers
    blk = (np.abs(cc[:, 0] - 5) < 8) & (cc[:, 1] < -3) & (cc[:, 1] > -10)
    m[blk] = np.log(10.0)
    return mesh, survey, m


def suite_case(kind):
    rng = np.random.default_rng(11)
    if kind == "2d-tensor":
        mesh = TensorMesh([[(1.0, 64)], [(1.0, 32)]], origin="CN")
        xe = np.linspace(-20, 20, 15)
        survey = Survey(dipole_dipole_2d(xe, 4, a=1))
    elif kind == "3d-tensor":
        mesh = TensorMesh([[(2.0, 20)], [(2.0, 20)], [(2.0, 10)]],
                          origin="CCN")
        xe = np.linspace(-14, 14, 9)
        srcs = []
        for i in range(len(xe) - 1):
            lm, ln = [], []
            for n in range(1, 4):
                jm, jn = i + 1 + n, i + 2 + n
                if jn >= len(xe):
                    break
                lm.append([xe[jm], 0.0, 0.0])
                ln.append([xe[jn], 0.0, 0.0])
            if lm:
                rx = DipoleReceiver(np.array(lm), np.array(ln))
                srcs.append(DipoleSource([rx], np.r_[xe[i], 0.0, 0.0],
                                         np.r_[xe[i + 1], 0.0, 0.0]))
        survey = Survey(srcs)
    else:
        raise ValueError(kind)
    m = np.log(100.0) * np.ones(mesh.nC) + 0.3 * rng.standard_normal(mesh.nC)
    return mesh, survey, m


def tiny_2d():
    """A 24x12-cell padded 2.5-D case (golden fixtures hold its operators)."""
    mesh = TensorMesh([[(2.0, 4, -1.3), (1.0, 16), (2.0, 4, 1.3)],
                       [(2.0, 4, -1.3), (1.0, 8)]], origin="CN")
    xe = np.linspace(-6, 6, 7)
    survey = Survey(dipole_dipole_2d(xe, 3))
    rng = np.random.default_rng(5)
    m = np.log(100.0) + 0.3 * rng.standard_normal(mesh.nC)
    return mesh, survey, m


def tiny_3d():
    """A 10x10x6-cell padded 3-D case with a pole source (golden fixtures)."""
    mesh = TensorMesh([[(2.0, 2, -1.3), (1.0, 6), (2.0, 2, 1.3)],
                       [(2.0, 2, -1.3), (1.0, 6), (2.0, 2, 1.3)],
                       [(2.0, 2, -1.3), (1.0, 4)]], origin="CCN")
    xe = np.linspace(-2, 2, 5)
    srcs = []
    for i in range(len(xe) - 3):
        rx = DipoleReceiver(np.array([[xe[i + 2], 0, 0]]),
                                np.array([[xe[i + 3], 0, 0]]))
        srcs.append(DipoleSource([rx], np.r_[xe[i], 0, 0],
                                     np.r_[xe[i + 1], 0, 0]))
    srcs.append(PoleSource([DipoleReceiver(
        np.array([[1.0, 1.0, 0.0], [2.0, 1.0, 0.0]]),
        np.array([[2.0, 1.0, 0.0], [2.0, 2.0, 0.0]]))], np.r_[-1.0, -1.0, 0.0]))
    survey = Survey(srcs)
    rng = np.random.default_rng(6)
    m = np.log(100.0) + 0.3 * rng.standard_normal(mesh.nC)
    return mesh, survey, m


def dc2d_small(seed=0):
    mesh = padded_mesh_2d(2.5, 100, 50, 10)
    xe = np.arange(21) * 5.0 - 50.0
    survey = Survey(dipole_dipole_2d(xe, 6, a=1))
    rng = np.random.default_rng(seed)
    m = block_model_2d(mesh, rng, (-125.0, 125.0), 125.0)
    return mesh, survey, m


def dc2d_large(seed=0):
    mesh = padded_mesh_2d(1.0, 400, 120, 12)
    xe = np.arange(96) * 4.0 - 190.0
    srcs = dipole_dipole_2d(xe, 20, a=1) + wenner_2d(xe, a=1)
    survey = Survey(srcs)
    rng = np.random.default_rng(seed)
    m = block_model_2d(mesh, rng, (-200.0, 200.0), 120.0)
    return mesh, survey, m


def dc2d_batch(n_problems=64, seed=0, scale=1.0):
    """List of (mesh, survey, m) of uneven size (5k-40k cells; `scale`
    multiplies the cell counts, for small test batches)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_problems):
        target = rng.uniform(5e3, 4e4) * scale
        npad = 8
        ncy = int(np.sqrt(target / 3.0))
        ncx = max(int(target / (ncy + npad)) - 2 * npad, 40)
        dx = 1.0
        mesh = padded_mesh_2d(dx, ncx, ncy, npad)
        ne = int(rng.integers(24, 65))
        span = 0.8 * ncx * dx
        xe = np.linspace(-span / 2, span / 2, ne)
        xe = np.round(xe / dx) * dx
        xe = np.unique(xe)
        survey = Survey(dipole_dipole_2d(xe, 6, a=1))
        cc = mesh.cell_centers
        m = np.full(mesh.nC, np.log(10.0) * rng.uniform(1.0, 3.5) / np.log(10.0))
        for _b in range(3):
            x0 = rng.uniform(-span / 2, span / 2)
            z0 = -rng.uniform(0.05, 0.6) * ncy * dx
            w, h = rng.uniform(0.05, 0.2) * span, rng.uniform(0.05, 0.3) * ncy
            blk = (np.abs(cc[:, 0] - x0) < w / 2) & (np.abs(cc[:, 1] - z0) < h / 2)
            m[blk] = np.log(10.0) * rng.uniform(1.0, 3.5)
        out.append((mesh, survey, m))
    return out


def dc3d(seed=0, ncore=(64, 64, 32), dx=5.0, npad=8, n_grid=10,
         n_sources=200, n_rx=30):
    mesh = padded_mesh_3d(dx, ncore[0], ncore[1], ncore[2], npad)
    span = (ncore[0] - 10) * dx
    g = np.linspace(-span / 2, span / 2, n_grid)
    g = np.round(g / dx) * dx
    ex, ey = np.meshgrid(g, g, indexing="ij")
    elec = np.c_[ex.ravel(), ey.ravel(), np.zeros(ex.size)]
    # the second half of the sources sits on the half-spacing offset grid
    step = g[1] - g[0]
    go = np.round((g[:-1] + step / 2) / dx) * dx
    ox, oy = np.meshgrid(go, go, indexing="ij")
    elec2 = np.c_[ox.ravel(), oy.ravel(), np.zeros(ox.size)]
    cand = np.vstack([elec, elec2])
    rng = np.random.default_rng(seed)
    pick = rng.choice(cand.shape[0], size=min(n_sources, cand.shape[0]),
                      replace=False)
    src_locs = cand[np.sort(pick)]
    if src_locs.shape[0] < n_sources:
        extra = cand[rng.choice(cand.shape[0], n_sources - src_locs.shape[0])]
        src_locs = np.vstack([src_locs, extra + np.r_[dx, 0, 0]])
    # receiver dipoles: adjacent-electrode pairs along x and y
    pairs = []
    for i in range(n_grid):
        for j in range(n_grid):
            a = i * n_grid + j
            if i + 1 < n_grid:
                pairs.append((a, (i + 1) * n_grid + j))
            if j + 1 < n_grid:
                pairs.append((a, i * n_grid + j + 1))
    pairs = np.array(pairs)
    mid = 0.5 * (elec[pairs[:, 0]] + elec[pairs[:, 1]])
    srcs = []
    for s in src_locs:
        d = np.linalg.norm(mid - s, axis=1)
        ok = (np.linalg.norm(elec[pairs[:, 0]] - s, axis=1) > 1e-6) & \
             (np.linalg.norm(elec[pairs[:, 1]] - s, axis=1) > 1e-6)
        order = np.argsort(np.where(ok, d, np.inf))[:n_rx]
        rx = DipoleReceiver(elec[pairs[order, 0]], elec[pairs[order, 1]])
        srcs.append(PoleSource([rx], s))
    survey = Survey(srcs)
    cc = mesh.cell_centers
    z = cc[:, 2]
    m = np.where(z > -20.0, np.log(200.0),
                 np.where(z > -80.0, np.log(50.0), np.log(500.0)))
    for rho in (5.0, 2000.0):
        c = np.r_[rng.uniform(-0.3, 0.3, 2) * span, -rng.uniform(30.0, 90.0)]
        ax = np.r_[rng.uniform(20.0, 60.0, 2), rng.uniform(15.0, 30.0)]
        inside = (((cc - c) / ax) ** 2).sum(1) < 1.0
        m[inside] = np.log(rho)
    m = m + 0.1 * rng.standard_normal(mesh.nC)
    return mesh, survey, m


def gaussian_random_field(points, rng, corr=50.0, sigma=0.5, spacing=None, extent=None):
    """A seeded smooth random field at `points` (n, dim): white noise on a
    regular grid filtered by a Gaussian kernel of correlation length `corr`
    (FFT), scaled to standard deviation `sigma`, interpolated linearly."""
    from scipy.interpolate import RegularGridInterpolator
    pts = np.atleast_2d(np.asarray(points, float))
    lo = pts.min(0) if extent is None else np.asarray(extent[0], float)
    hi = pts.max(0) if extent is None else np.asarray(extent[1], float)
    d = corr / 4.0 if spacing is None else float(spacing)
    n = [int(np.ceil((h - l) / d)) + 1 for l, h in zip(lo, hi)]
    noise = rng.standard_normal(n)
    k = np.meshgrid(*[np.fft.fftfreq(m, d=d) for m in n], indexing="ij")
    k2 = sum(ki ** 2 for ki in k)
    field = np.real(np.fft.ifftn(np.fft.fftn(noise) * np.exp(-0.5 * (2 * np.pi) ** 2 * k2 *
                                                              (corr / 2.0) ** 2)))
    field = (field - field.mean()) / (field.std() + 1e-30) * sigma
    axes = [l + d * np.arange(m) for l, m in zip(lo, n)]
    f = RegularGridInterpolator(axes, field, bounds_error=False, fill_value=None)
    return f(np.clip(pts, lo, hi))


def dc3d_tree(seed=0, max_level=8, h0=5.0, n_el=21, spacing=10.0, n_sources=400, n_rx=40,
              refine=((8, 130.0), (7, 250.0), (6, 400.0), (5, 600.0))):
    """The refined 3-D workload: an octree refined around a surface electrode grid
    (n_el x n_el at `spacing`), gradient-array sources (far-apart A, B pairs,
    each with n_rx adjacent-electrode potential dipoles between them) and a
    Gaussian random field log-rho (50 m correlation, sigma 0.5 around
    log 100).  Returns (mesh, survey, m)."""
    from .treemesh import TreeMesh
    rng = np.random.default_rng(seed)
    nf = 2 ** max_level
    width = nf * h0
    tm = TreeMesh([(h0, nf)] * 3, origin=[-width / 2, -width / 2, -width])
    half = (n_el - 1) * spacing / 2
    g = np.linspace(-half, half, n_el)
    ex, ey = np.meshgrid(g, g, indexing="ij")
    elec = np.c_[ex.ravel(), ey.ravel(), np.zeros(ex.size)]
    tm.refine(lambda lo, hi: np.full(lo.shape[0], 3))
    for level, pad in refine:
        tm.refine_points(elec, level, padding=pad)
    tm.finalize()
    idx = np.arange(elec.shape[0]).reshape(n_el, n_el)
    pairs = np.r_[np.c_[idx[:-1, :].ravel(), idx[1:, :].ravel()],
                  np.c_[idx[:, :-1].ravel(), idx[:, 1:].ravel()]]
    mid = 0.5 * (elec[pairs[:, 0]] + elec[pairs[:, 1]])
    srcs = []
    while len(srcs) < n_sources:
        a, b = rng.choice(elec.shape[0], 2, replace=False)
        A, B = elec[a], elec[b]
        if np.linalg.norm(A - B) < 0.6 * (2 * half):
            continue
        # dipoles in the middle third between A and B (the gradient array's
        # potential electrodes), nearest to the segment first
        t = np.clip(((mid - A) @ (B - A)) / ((B - A) @ (B - A)), 0.0, 1.0)
        dseg = np.linalg.norm(mid - (A + t[:, None] * (B - A)), axis=1)
        ok = (t > 1 / 3) & (t < 2 / 3)
        ok &= np.all(pairs != a, axis=1) & np.all(pairs != b, axis=1)
        order = np.argsort(np.where(ok, dseg, np.inf))[:n_rx]
        rx = DipoleReceiver(elec[pairs[order, 0]], elec[pairs[order, 1]])
        srcs.append(DipoleSource([rx], A, B))
    survey = Survey(srcs)
    m = np.log(100.0) + gaussian_random_field(tm.cell_centers, rng, corr=50.0, sigma=0.5,
                                              spacing=10.0,
                                              extent=(tm.origin, tm.origin + width))
    return tm, survey, m


def tree_small(seed=0):
    """A small 3-D octree case (a few thousand nodes) for parity tests."""
    return dc3d_tree(seed=seed, max_level=6, h0=5.0, n_el=5, spacing=10.0, n_sources=6,
                     n_rx=4, refine=((6, 8.0), (5, 20.0), (4, 45.0)))


def observed(d_true, rng, rel_noise=0.05):
    """dobs = d (1 + rel N(0,1)), w = 1 / (rel |dobs|) (the workloads' noise)."""
    dobs = d_true * (1.0 + rel_noise * rng.standard_normal(d_true.shape))
    w = 1.0 / (rel_noise * np.abs(dobs) + 1e-30)
    return dobs, w
