"""Linearized induced-polarization (Seigel) forward on the DC engines.

The IP data of a chargeability model eta are the DC sensitivity applied to
the conductivity change -sigma_bg eta, scaled per datum
(dctorch/ip2d.py:1-26, ip3d.py:1-23):

    d_IP = scale * J_m(m_dc) eta,   J_m = dd/dm at the background m = log(rho),
    scale = 1 / V_dc on receivers of data type "apparent_chargeability", else 1.

Here that is one fixed factorization of the background (and its fields)
kept by the DC engine's fused path, and per evaluation one batched solve of
-A_k(dvals) U_k on those factors (the same product as the engines' J v);
the gradient with respect to eta is the adjoint product J_m^T (scale * g).
`dpred` is differentiable in eta only; the background never changes.  If
something else refactorizes the wrapped engine, the background factors are
restored before the next product.
"""
from __future__ import annotations

import numpy as np
import torch

from .simulation2d import TorchDC2D, _ActiveCells
from .simulation3d import TorchDC3D


class _LinearIPFn(torch.autograd.Function):
    """d = scale * J e (e on the full mesh, float64); backward J^T (scale g)."""

    @staticmethod
    def forward(ctx, e_full, ip):
        ctx.ip = ip
        with torch.no_grad():
            return ip._scale * ip._jvec(e_full)

    @staticmethod
    def backward(ctx, g):
        ip = ctx.ip
        with torch.no_grad():
            return ip._jtvec(ip._scale * g.to(torch.float64)), None


class _LinearIP:
    """Shared runtime of TorchIP2D / TorchIP3D."""

    def _setup(self, dc, m_full, survey, eta_cells):
        self.dc = dc
        self.device, self.dtype = dc.device, dc.dtype
        self._eta = eta_cells      # active-cell map of eta, or None
        path = dc._path
        with torch.no_grad():
            self._sigma, self._vals = path.values(m_full)
            path.factorize(self._vals)
            self._stamp = path.solver.stamp
            self._U = path.fields()
            v_dc = path.project(self._U)
        self.v_dc = v_dc.to(self.dtype)
        # per-datum scale in survey order (the order of the engine's data)
        scale = torch.ones(dc.nD, dtype=torch.float64, device=self.device)
        i0 = 0
        for src in survey.source_list:
            for rx in src.receiver_list:
                i1 = i0 + rx.nD
                if getattr(rx, "data_type", "volt") == "apparent_chargeability":
                    scale[i0:i1] = 1.0 / v_dc[i0:i1]
                i0 = i1
        if i0 != dc.nD:
            raise ValueError("survey data count does not match the engine's")
        self._scale = scale

    def _ensure(self):
        path = self.dc._path
        if path.solver.stamp != self._stamp:
            path.factorize(self._vals)
            self._stamp = path.solver.stamp

    def _jvec(self, e_full):
        self._ensure()
        return self.dc._path.jvec(e_full, self._sigma, self._U)

    def _jtvec(self, g):
        """J^T g on the full mesh (the active-cell injection of eta is a
        torch op, whose backward restricts it)."""
        self._ensure()
        return self.dc._path.adjoint(g.reshape(-1).contiguous(), self._U, self._sigma)

    def dpred(self, eta):
        """Predicted IP data (nD,) for eta (on the active cells when built
        with active_cells, else on the full mesh); linear and differentiable."""
        dev0, dt0 = eta.device, eta.dtype
        e = eta.to(device=self.device, dtype=torch.float64).reshape(-1)
        if self._eta is not None:
            e = self._eta.inject(e)
        d = _LinearIPFn.apply(e, self)
        return d.to(device=dev0, dtype=dt0)

    def misfit(self, eta, dobs, w):
        """phi_d = ||w*(dpred-dobs)||^2 (no 1/2 factor)."""
        r = w * (self.dpred(eta) - dobs)
        return (r ** 2).sum()

    def check(self):
        return self.dc.check()


class TorchIP2D(_LinearIP):
    """Linearized 2.5-D IP on a fixed mesh, survey and background
    (dctorch/ip2d.py:51-158).  m_dc: (nC,) log-rho background on the full
    mesh; active_cells: optional mask for eta (inactive eta = 0)."""

    def __init__(self, mesh, survey, m_dc, nky=12, device="cuda",
                 dtype=torch.float64, active_cells=None, quadrature=None):
        dc = TorchDC2D(mesh, survey, nky=nky, device=device, dtype=dtype,
                       quadrature=quadrature)
        m_bg = np.asarray(m_dc, dtype=float).reshape(-1)
        if m_bg.size != dc.nC:
            raise ValueError("m_dc must live on the full mesh")
        eta = None
        if active_cells is not None:
            eta = _ActiveCells(active_cells, 0.0, dc.nC, dc.device)
        m_full = torch.as_tensor(m_bg, dtype=torch.float64, device=dc.device)
        self._setup(dc, m_full, survey, eta)


class TorchIP3D(_LinearIP):
    """Linearized 3-D IP on a fixed mesh, survey and background
    (dctorch/ip3d.py:75-175).  m_dc: log-rho background on the active cells
    when active_cells is given (inactive cells take val_inactive), else on
    the full mesh; eta lives on the same cells."""

    def __init__(self, mesh, survey, m_dc, device="cuda", dtype=torch.float64,
                 active_cells=None, val_inactive=None, bc_type="Robin"):
        dc = TorchDC3D(mesh, survey, device=device, dtype=dtype,
                       active_cells=active_cells, val_inactive=val_inactive,
                       bc_type=bc_type)
        m_bg = torch.as_tensor(np.asarray(m_dc, dtype=float).reshape(-1),
                               dtype=torch.float64, device=dc.device)
        if dc._inj is not None:
            if m_bg.numel() != dc._inj.nA:
                raise ValueError("m_dc must live on the active cells")
        elif m_bg.numel() != dc.nC:
            raise ValueError("m_dc must live on the full mesh")
        self._setup(dc, dc._model_to_full(m_bg), survey, dc._inj)
