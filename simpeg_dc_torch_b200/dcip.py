"""Joint non-linear DC + IP 2.5-D forward (Seigel, not linearized).

The two states of a chargeable medium (dctorch/dcip2d.py:1-54):

    sigma     = exp(-m_rho)                  instantaneous (un-polarized)
    eta       = eta_max * sigmoid(m_eta)     chargeability in (0, eta_max)
    sigma_eff = sigma * (1 - eta)            fully polarized steady state

    V0 = F(sigma),  V1 = F(sigma_eff)
    d_IP = ip_scale * (V1 - V0) / V1
    d_DC = V1 (dc_state "total") or V0 ("instantaneous")

Both voltages come from the fused 2.5-D evaluation of this package (values,
factorization, all sources in one batched solve, projection), once with the
log-resistivity m_rho and once with m_rho - log(1 - eta), on two engines
that share the mesh and survey, so each state keeps its own factors for the
adjoint.  The gradient with respect to both model blocks is the adjoint of
the two evaluations, through autograd.
"""
from __future__ import annotations

import numpy as np
import torch

from .simulation2d import TorchDC2D, _ActiveCells


class TorchDCIP2D:
    """Differentiable joint (rho, eta) 2.5-D nodal DC-IP forward with the
    constructor and methods of dctorch.dcip2d.TorchDCIP2D (dcip2d.py:62-193).

    The model is m = cat(m_rho, m_eta), each on the active cells (or the
    full mesh): m_rho = log(rho), m_eta = logit(eta / eta_max); inactive
    cells take val_inactive (log-rho) and eta = 0.  idx_dc / idx_ip select
    the DC and IP data from the survey's data ordering (default: all).
    """

    def __init__(self, mesh, survey, nky=12, device="cuda",
                 dtype=torch.float64, active_cells=None, val_inactive=None,
                 idx_dc=None, idx_ip=None, eta_max=1.0, ip_scale=1.0,
                 dc_state="total", quadrature=None):
        if dc_state not in ("total", "instantaneous"):
            raise ValueError(f"dc_state must be 'total' or 'instantaneous', not {dc_state!r}")
        # one engine per state: each keeps its own factorization
        self.dc = TorchDC2D(mesh, survey, nky=nky, device=device, dtype=dtype,
                            quadrature=quadrature)
        self._dc_eff = TorchDC2D(mesh, survey, nky=nky, device=device, dtype=dtype,
                                 quadrature=(self.dc.kys, self.dc.wq_np))
        dc = self.dc
        self.device, self.dtype = dc.device, dc.dtype
        self.nky, self.nD = dc.nky, dc.nD
        self._act = None
        if active_cells is not None:
            if val_inactive is None:
                raise ValueError("val_inactive is required with active_cells")
            self._act = _ActiveCells(active_cells, val_inactive, dc.nC, dc.device)
        self.nP = dc.nC if self._act is None else self._act.nA
        self.eta_max = float(eta_max)
        self.ip_scale = float(ip_scale)
        self.dc_state = dc_state

        def _idx(a):
            if a is None:
                return torch.arange(dc.nD, dtype=torch.int64, device=self.device)
            return torch.as_tensor(np.asarray(a, dtype=np.int64), device=self.device)

        self.idx_dc, self.idx_ip = _idx(idx_dc), _idx(idx_ip)
        self.nD_dc = int(self.idx_dc.numel())
        self.nD_ip = int(self.idx_ip.numel())

    # ------------------------------------------------ model <-> fields
    def _inject_rho(self, m_rho):
        return m_rho if self._act is None else self._act.full(m_rho)

    def _inject_eta(self, eta):
        return eta if self._act is None else self._act.inject(eta)

    def split(self, m):
        """(m_rho, m_eta) blocks of the stacked model."""
        m = m.reshape(-1)
        if m.numel() != 2 * self.nP:
            raise ValueError(f"model must be 2*{self.nP} long, got {m.numel()}")
        return m[:self.nP], m[self.nP:]

    def eta_of(self, m_eta):
        """Physical eta (on the model's cells) from the logit block."""
        return self.eta_max * torch.sigmoid(m_eta)

    def m_eta_of(self, eta):
        """The logit block of a physical eta (numpy or tensor)."""
        if not torch.is_tensor(eta):
            e = np.clip(np.asarray(eta, dtype=float) / self.eta_max, 1e-12, 1 - 1e-12)
            return np.log(e / (1 - e))
        e = (eta / self.eta_max).clamp(1e-12, 1 - 1e-12)
        return torch.log(e / (1 - e))

    # ------------------------------------------------ runtime
    def _voltages(self, m_rho_full, eta_full):
        """(V0, V1): the un-polarized and the fully polarized data."""
        v0 = self.dc.dpred(m_rho_full)
        v1 = self._dc_eff.dpred(m_rho_full - torch.log1p(-eta_full))
        return v0, v1

    def dpred_from_fields(self, m_rho, eta):
        """(d_DC, d_IP) from log-rho and physical eta (both on the model's
        cells), bypassing the sigmoid."""
        dev0, dt0 = m_rho.device, m_rho.dtype
        mr = m_rho.to(device=self.device, dtype=torch.float64).reshape(-1)
        e = eta.to(device=self.device, dtype=torch.float64).reshape(-1)
        v0, v1 = self._voltages(self._inject_rho(mr), self._inject_eta(e))
        d_dc = (v1 if self.dc_state == "total" else v0)[self.idx_dc]
        d_ip = self.ip_scale * (v1[self.idx_ip] - v0[self.idx_ip]) / v1[self.idx_ip]
        return d_dc.to(device=dev0, dtype=dt0), d_ip.to(device=dev0, dtype=dt0)

    def dpred(self, m):
        """(d_DC, d_IP) for the stacked model m = cat(log-rho, logit-eta)."""
        m_rho, m_eta = self.split(m)
        return self.dpred_from_fields(m_rho, self.eta_of(m_eta))

    def misfit(self, m, dobs_dc, w_dc, dobs_ip, w_ip, lam=1.0):
        """phi_DC + lam * phi_IP, each ||w*(dpred-dobs)||^2 (no 1/2)."""
        d_dc, d_ip = self.dpred(m)
        r0 = w_dc * (d_dc - dobs_dc)
        r1 = w_ip * (d_ip - dobs_ip)
        return (r0 ** 2).sum() + lam * (r1 ** 2).sum()

    def check(self):
        self.dc.check()
        return self._dc_eff.check()
