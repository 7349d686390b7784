"""Eval + gradient of an engine replayed from one CUDA graph.

One misfit-and-gradient evaluation of the fused path is a fixed sequence of
launches for a given mesh, survey and plan: assembly of the values,
factorization, source scatter, refined solve, projection, misfit, adjoint
scatter, refined adjoint solve, gather-contract and L^T product.  The
refinement decides on the device when to stop (later correction launches see
a flag and return), so nothing in the sequence waits for the host.
`GraphedMisfitGrad` captures that sequence once on a side stream and replays
it for every new model: one graph launch per evaluation instead of several
hundred kernel launches from the host.

The graph reads the model, observed data and weights from its own input
buffers and writes phi and the gradient into its own output buffers (the
call copies them in and returns copies).  Replays overwrite the solver's
factors, so the solver's stamp is advanced on every call: an autograd
backward of an earlier eager `dpred` then refactorizes before it runs.
"""
from __future__ import annotations

import torch


class GraphedMisfitGrad:
    """(phi, dphi/dm) of `eng.misfit_and_grad` from one captured CUDA graph.

    eng   : a TorchDC2D, TorchDC3D or TorchDC2DBatch engine (its fused path
            `_path`, and `_model_to_full` / `_inj` where it has active cells)
    m, dobs, w : example inputs; their shapes and the engine fix the graph
    warmup: eager evaluations on the capture stream before the capture (the
            plan's lazily made buffers exist before capturing)
    """

    def __init__(self, eng, m, dobs, w, warmup=2):
        path = getattr(eng, "_path", None)
        if path is None or getattr(path, "_pri", None) is not None:
            raise NotImplementedError(
                "graph capture needs the plain fused path (no singularity removal)")
        self.eng, self.path = eng, path
        dev = eng.device
        self.m_dtype, self.m_device = m.dtype, m.device
        self._m = m.detach().to(dev, torch.float64).reshape(-1).clone()
        self._dobs = dobs.detach().to(dev, torch.float64).reshape(-1).clone()
        self._w = w.detach().to(dev, torch.float64).reshape(-1).clone()
        if path.record_refinement:
            raise ValueError("record_refinement synchronises; switch it off first")
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            for _ in range(max(1, int(warmup))):
                self._body()
        torch.cuda.current_stream(dev).wait_stream(side)
        torch.cuda.synchronize(dev)
        self.graph = torch.cuda.CUDAGraph()
        # thread-local capture: other threads' CUDA calls are not captured
        with torch.cuda.graph(self.graph, stream=side, capture_error_mode="thread_local"):
            self._phi, self._grad = self._body()
        torch.cuda.synchronize(dev)
        self.path.solver.stamp += 1

    def _body(self):
        eng, path = self.eng, self.path
        to_full = getattr(eng, "_model_to_full", None)
        inj = getattr(eng, "_inj", None)
        with torch.no_grad():
            m_full = self._m if to_full is None else to_full(self._m)
            d, sigma, U, _ = path.forward(m_full)
            r = self._w * (d - self._dobs)
            phi = (r * r).sum()
            g = path.adjoint(2.0 * self._w * r, U, sigma)
            g = g if inj is None else inj.restrict(g)
        return phi, g

    def replay(self, m, dobs=None, w=None):
        """Replay on the current stream without copying the outputs out:
        returns the graph's own (phi, grad) tensors (overwritten by the next
        replay)."""
        self._m.copy_(m.detach().reshape(-1))
        if dobs is not None:
            self._dobs.copy_(dobs.detach().reshape(-1))
        if w is not None:
            self._w.copy_(w.detach().reshape(-1))
        self.graph.replay()
        self.path.solver.stamp += 1
        return self._phi, self._grad

    def __call__(self, m, dobs=None, w=None):
        """(phi as float, gradient in m's dtype and device)."""
        phi, g = self.replay(m, dobs, w)
        return float(phi), g.to(device=self.m_device, dtype=self.m_dtype, copy=True)
