"""Complex-resistivity 2.5-D forward (drop-in for dctorch's `TorchCR2D`,
dctorch/cr2d.py:13-108).

The medium has the complex conductivity

    sigma* = sigma (1 - i m),   sigma = exp(-m_rho),   m the chargeability

so every wavenumber system A_k(sigma*) is complex symmetric (A^T = A, not
Hermitian).  The systems are factored A = L L^T without conjugation by the
same multifrontal kernels as the real path, instantiated in complex128 (a
`DCT_C128` plan), and all wavenumbers and sources are solved in the same
launches.  The data are

    V = (Pd sum_k w_k U_k)[i, sidx_i],  U_k = A_k^{-1} q
    d_rho = |V| ("magnitude") or Re V ("real"),  d_ip = ip_scale Im V / Re V

and the gradient of a real loss runs through the complex-safe adjoint of the
batched solve (the conjugate Wirtinger derivative, one adjoint solve on the
same factors, the pattern contraction in one kernel).  Values and the
receiver projection are formed with torch sparse products, as the reference
does.
"""
from __future__ import annotations

import torch

from .simulation2d import TorchDC2D, _to_coo_tensor
from .solver import make_batch_solver, sparse_solve_batch


class TorchCR2D:
    """Differentiable complex-resistivity 2.5-D nodal forward.

    mesh, survey : receivers of plain voltage (the ratio is formed here).
    ip_scale     : multiplies d_ip (1000 for chargeability in mV/V, also
                   ~mrad of phase).
    dc_datum     : "magnitude" (|V|, the magnitude/phase pair) or "real" (Re V).
    dtype        : complex128, or complex64 (factored and solved in
                   complex128; data come back in the model's dtype).
    """

    def __init__(self, mesh, survey, nky=12, device="cuda",
                 dtype=torch.complex128, active_cells=None, val_inactive=None,
                 ip_scale=1.0, dc_datum="magnitude", quadrature=None,
                 leaf_size=64):
        if not dtype.is_complex:
            raise TypeError(f"TorchCR2D needs a complex dtype, got {dtype}")
        if dc_datum not in ("magnitude", "real"):
            raise ValueError(f"dc_datum must be 'magnitude' or 'real', not {dc_datum!r}")
        dc = TorchDC2D(mesh, survey, nky=nky, device=device, dtype=torch.float64,
                       active_cells=active_cells, val_inactive=val_inactive,
                       quadrature=quadrature, leaf_size=leaf_size)
        self.dc = dc
        self.device, self.dtype = dc.device, dtype
        self.rdtype = torch.float64 if dtype == torch.complex128 else torch.float32
        self.nky, self.nD = dc.nky, dc.nD
        self.nP = dc.nC if dc._inj is None else dc._inj.nA
        self.ip_scale = float(ip_scale)
        self.dc_datum = dc_datum
        # the real SPD plan is replaced by a complex-symmetric one on the
        # same pattern and dissection coordinates
        crow, col = dc.solver.crow, dc.solver.col
        dc.solver.free()
        dc.solver = None
        mesh_t = dc._mesh
        coords = mesh_t.node_grid_index() if hasattr(mesh_t, "node_grid_index") else None
        self.solver = make_batch_solver(crow, col, dc.nN, dc.nS, dc.nky,
                                        device=self.device, dtype=torch.complex128,
                                        matrix_type="symmetric", coords=coords,
                                        leaf_size=leaf_size)
        self.q = dc.q.to(torch.complex128)
        self._L = dc.Lstack
        self._Pd = _to_coo_tensor(dc._ops.Pd, self.device, torch.float64)
        self._wq = dc.wq.to(torch.complex128).view(-1, 1, 1)

    # ------------------------------------------------ model <-> fields
    def _inject_rho(self, m_rho):
        return m_rho if self.dc._inj is None else self.dc._inj.full(m_rho)

    def _inject_ip(self, m_ip):
        return m_ip if self.dc._inj is None else self.dc._inj.inject(m_ip)

    def split(self, m):
        """(log-rho, chargeability) blocks of the stacked model."""
        m = m.reshape(-1)
        if m.numel() != 2 * self.nP:
            raise ValueError(f"model must be 2*{self.nP} long, got {m.numel()}")
        return m[:self.nP], m[self.nP:]

    # ------------------------------------------------ runtime
    def _spmm(self, M, v):
        return torch.sparse.mm(M, v.unsqueeze(1)).squeeze(1)

    def voltages(self, m_rho, m_ip):
        """The complex data V (nD,) for log-rho and chargeability on the
        model's cells (complex128 on the engine's device)."""
        dc = self.dc
        mr = m_rho.to(device=self.device, dtype=torch.float64).reshape(-1)
        mi = m_ip.to(device=self.device, dtype=torch.float64).reshape(-1)
        sig = torch.exp(-self._inject_rho(mr))
        chg = self._inject_ip(mi)
        # sigma* = sigma (1 - i m): two real products, then recombined
        vre = self._spmm(self._L, sig).view(dc.nky, dc.nnzA)
        vim = self._spmm(self._L, -sig * chg).view(dc.nky, dc.nnzA)
        U = sparse_solve_batch(torch.complex(vre, vim), self.q, self.solver)
        Ubar = (self._wq * U).sum(0)
        Vr = torch.sparse.mm(self._Pd, Ubar.real)[dc.iD, dc.sidx]
        Vi = torch.sparse.mm(self._Pd, Ubar.imag)[dc.iD, dc.sidx]
        return torch.complex(Vr, Vi)

    def dpred_from_fields(self, m_rho, m_ip):
        """(d_rho, d_ip) from log-rho and chargeability (model cells)."""
        dev0, dt0 = m_rho.device, m_rho.dtype
        V = self.voltages(m_rho, m_ip)
        Vr, Vi = V.real, V.imag
        d_rho = torch.sqrt(Vr ** 2 + Vi ** 2) if self.dc_datum == "magnitude" else Vr
        d_ip = self.ip_scale * Vi / Vr
        return d_rho.to(device=dev0, dtype=dt0), d_ip.to(device=dev0, dtype=dt0)

    def dpred(self, m):
        """(d_rho, d_ip) for the stacked model m = cat(log-rho, chargeability)."""
        m_rho, m_ip = self.split(m)
        return self.dpred_from_fields(m_rho, m_ip)

    def misfit(self, m, dobs_rho, w_rho, dobs_ip, w_ip, lam=1.0):
        """phi_rho + lam * phi_ip, each ||w (dpred - dobs)||^2 (no 1/2)."""
        d_r, d_i = self.dpred(m)
        return ((w_rho * (d_r - dobs_rho)) ** 2).sum() \
            + lam * ((w_ip * (d_i - dobs_ip)) ** 2).sum()

    def check(self):
        """Synchronise and raise if a kernel reported an error."""
        return self.solver.check()
