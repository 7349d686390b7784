"""Wavenumber quadrature of the 2.5-D transform, fitted on electrode distances.

The 2.5-D potential is a weighted sum of 2-D solves, u = sum_k w_k u_k.  The
points k and weights w are chosen so that sum_k 2 w_k K0(k r) reproduces 1/r
over the distances the survey's electrode pairs span (w = g/2, SimPEG's
convention).  This restates the reference's algorithm
(dctorch/quadrature.py:100-154):

  1. sample r log-uniformly on [r_min/margin, r_max*margin];
  2. for a set of log10-wavenumbers, the weights are the non-negative
     least-squares fit of r K0(k r) g = 1 with column normalisation
     (quadrature.py:73-86), falling back to bounded least squares;
  3. the log-wavenumbers are optimised by `least_squares` (TRF) on that
     residual (quadrature.py:128-133);
  4. continuation: start from `n_start` points spread over [-log r_max,
     -log r_min]; add one point at a time in the widest gap (the two ends
     count as gaps of half a decade) and refit (quadrature.py:135-145);
  5. points with zero weight are dropped (quadrature.py:147-149).

The same scipy routines and tolerances are used, so the points and weights
agree with the reference's to round-off; a committed fixture pins that.
"""
from __future__ import annotations

import warnings

import numpy as np

from .survey import source_electrodes


def electrode_distance_range(survey):
    """(r_min, r_max) over current/potential electrode pairs (horizontal and
    vertical coordinates only), as in dctorch/quadrature.py:38-61."""
    lo, hi = np.inf, 0.0
    for src in survey.source_list:
        a, b = source_electrodes(src)
        cur = [np.atleast_2d(a)] + ([] if b is None else [np.atleast_2d(b)])
        cur = np.vstack(cur)[:, :2]
        cur = cur[np.isfinite(cur).all(axis=1)]
        for rx in src.receiver_list:
            pm = getattr(rx, "locations_m", None)
            if pm is None:
                pm = rx.locations
            pts = [np.atleast_2d(np.asarray(pm, float))]
            pn = getattr(rx, "locations_n", None)
            if pn is not None:
                pts.append(np.atleast_2d(np.asarray(pn, float)))
            pts = np.vstack(pts)[:, :2]
            pts = pts[np.isfinite(pts).all(axis=1)]
            d = np.sqrt(((cur[:, None, :] - pts[None, :, :]) ** 2).sum(-1))
            d = d.reshape(-1)
            d = d[d > 1e-9]
            if d.size:
                lo = min(lo, float(d.min()))
                hi = max(hi, float(d.max()))
    if not np.isfinite(lo):
        raise ValueError("no separated current/potential electrode pair")
    return lo, hi


def amplification(weights):
    """sum|w| / |sum w| (1 for non-negative weights)."""
    w = np.asarray(weights, float)
    return float(np.abs(w).sum() / abs(w.sum()))


def _k0_columns(r, k):
    from scipy.special import k0
    return r[:, None] * k0(np.outer(r, k))


def _nonneg_fit(A, rhs):
    from scipy.optimize import lsq_linear, nnls
    norms = np.linalg.norm(A, axis=0)
    norms[norms == 0.0] = 1.0
    An = A / norms
    try:
        g = nnls(An, rhs, maxiter=50 * A.shape[1])[0]
    except RuntimeError:
        g = lsq_linear(An, rhs, bounds=(0.0, np.inf), method="bvls").x
    return g / norms


def transform_error(points, weights, r_min, r_max, n=400):
    """max |sum_k 2 w_k r K0(k r) - 1| on a log grid over [r_min, r_max]."""
    r = np.logspace(np.log10(r_min), np.log10(r_max), n)
    approx = _k0_columns(r, np.asarray(points)) @ (2.0 * np.asarray(weights))
    return float(np.abs(approx - 1.0).max())


def k0_quadrature(r_min, r_max, nky, margin=2.0, n_samples=200, n_start=4):
    """(points, weights, info) for the 2.5-D transform; see module docstring."""
    from scipy.optimize import least_squares

    r = np.logspace(np.log10(r_min / margin), np.log10(r_max * margin),
                    n_samples)
    ones = np.ones_like(r)

    def weights_of(logk):
        return _nonneg_fit(_k0_columns(r, 10.0 ** logk), ones)

    def residual(logk):
        A = _k0_columns(r, 10.0 ** logk)
        return A @ _nonneg_fit(A, ones) - ones

    def refit(logk0):
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)
            res = least_squares(residual, logk0, method="trf", xtol=1e-12,
                                ftol=1e-12, max_nfev=200 * logk0.size)
        return np.sort(res.x), bool(res.success)

    left, right = -np.log10(r.max()), -np.log10(r.min())
    n_first = min(n_start, nky)
    logk, ok = refit(np.linspace(left, right, n_first))
    errs = {n_first: transform_error(10.0 ** logk, weights_of(logk) / 2.0,
                                     r_min, r_max)}
    for n in range(n_first + 1, nky + 1):
        bounds = np.concatenate(([left - 0.5], logk, [right + 0.5]))
        gap = int(np.argmax(np.diff(bounds)))
        new = 0.5 * (bounds[gap] + bounds[gap + 1])
        logk, ok = refit(np.sort(np.concatenate((logk, [new]))))
        errs[n] = transform_error(10.0 ** logk, weights_of(logk) / 2.0,
                                  r_min, r_max)
    pts = 10.0 ** logk
    wts = weights_of(logk) / 2.0
    pos = wts > 0
    if not pos.all():
        pts, wts = pts[pos], wts[pos]
    info = {"success": ok and bool(np.isfinite(wts).all()),
            "max_rel_err": errs[nky], "r_range": (float(r_min), float(r_max)),
            "err_by_n": errs, "n_used": int(pts.size),
            "amplification": amplification(wts)}
    return pts, wts, info
