"""The optimizer contracts of the reference on this package's engines:
one torch.optim.LBFGS step with TorchLBFGS's closure over the 3-D
benchmark's engine (dctorch/optimization.py:330-402, the closure at
372-381), and one Gauss-Newton step on the full 2.5-D large workload with
TorchGaussNewton's call sequence (dctorch/optimization.py:586-618, 858-979:
the gradient through the linearization, a Jacobi-preconditioned truncated CG
on J^T D J + beta H_m, an Armijo line search).  TorchGaussNewton itself
cannot be imported without SimPEG, so its sequence is restated here.  Each
step must decrease the objective; the gradient of the float32 closure must
match float64 within 1e-5, and the linearization's J v and J^T v the oracle
within 1e-9 (float64)."""
import numpy as np
import pytest
import torch

from oracle import dc_oracle as O
from simpeg_dc_torch_b200 import TorchDC2D, TorchDC3D
from simpeg_dc_torch_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = torch.as_tensor(a, dtype=torch.float64).cpu()
    b = torch.as_tensor(b, dtype=torch.float64).cpu()
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


def pcg(apply_H, b, Minv, maxiter, rtol):
    """Preconditioned conjugate gradients on H x = b from x = 0, stopped at
    ||r|| <= rtol ||b|| (the truncated inner solve of a Gauss-Newton step)."""
    x = torch.zeros_like(b)
    r = b.clone()
    z = Minv * r
    p = z.clone()
    rz = float(r @ z)
    nb = float(torch.linalg.norm(b))
    it = 0
    for it in range(1, maxiter + 1):
        Hp = apply_H(p)
        alpha = rz / float(p @ Hp)
        x += alpha * p
        r -= alpha * Hp
        if float(torch.linalg.norm(r)) <= rtol * nb:
            break
        z = Minv * r
        rz_new = float(r @ z)
        p = z + (rz_new / rz) * p
        rz = rz_new
    return x, it


def test_lbfgs_iteration_on_the_3d_benchmark(cuda):
    """The 3-D benchmark (269,001 nodes, 200 sources), float32 + refinement engine."""
    mesh, survey, m_true = syn.dc3d(seed=0)
    e32 = TorchDC3D(mesh, survey, device=cuda, dtype=torch.float32)
    with torch.no_grad():
        d_true = e32.dpred(torch.tensor(m_true, device=cuda)).cpu().numpy()
    dobs_np, w_np = syn.observed(d_true, np.random.default_rng(11))
    dobs = torch.tensor(dobs_np, device=cuda)
    w = torch.tensor(w_np, device=cuda)
    m0 = np.full_like(m_true, float(np.median(m_true)))
    m_ref = torch.tensor(m0, device=cuda)
    beta = 1e-2

    def objective(mc):
        return e32.misfit(mc, dobs, w) + beta * ((mc - m_ref) ** 2).sum()

    m = torch.tensor(m0, device=cuda, requires_grad=True)
    opt = torch.optim.LBFGS([m], lr=1.0, max_iter=4, history_size=10,
                            line_search_fn="strong_wolfe")
    grads = []

    def closure():                        # dctorch/optimization.py:372-381
        opt.zero_grad()
        loss = objective(m)
        loss.backward()
        grads.append(m.grad.detach().clone())
        return loss

    with torch.no_grad():
        f0 = float(objective(m))
    opt.step(closure)
    with torch.no_grad():
        f1 = float(objective(m))
    e32.check()
    assert f1 < f0, (f0, f1)
    # the first closure's gradient is the float64 engine's within 1e-5
    del opt, e32
    torch.cuda.empty_cache()
    e64 = TorchDC3D(mesh, survey, device=cuda, dtype=torch.float64)
    x = torch.tensor(m0, device=cuda, requires_grad=True)
    (e64.misfit(x, dobs, w) + beta * ((x - m_ref) ** 2).sum()).backward()
    assert rel(grads[0], x.grad) < 1e-5


def test_gauss_newton_step_on_the_2d_large_workload(cuda):
    """The large 2.5-D workload (56,525 nodes, 12 wavenumbers, 186 sources), float64."""
    mesh, survey, m_true = syn.dc2d_large(seed=0)
    eng = TorchDC2D(mesh, survey, nky=12, device=cuda)
    with torch.no_grad():
        d_true = eng.dpred(torch.tensor(m_true, device=cuda)).cpu().numpy()
    dobs_np, w_np = syn.observed(d_true, np.random.default_rng(12))
    dobs = torch.tensor(dobs_np, device=cuda)
    w = torch.tensor(w_np, device=cuda)
    m0_np = np.full_like(m_true, float(np.median(m_true)))
    m0 = torch.tensor(m0_np, device=cuda)
    # the point: data, gradient and the linearization (optimization.py:586-618)
    lin = eng.linearize(m0)
    d0 = lin.d
    r = w * (d0 - dobs)
    D = 2.0 * w ** 2
    g = lin.Jtvec(w * 2.0 * r)          # the smallness term's gradient is 0 at m0
    diag = lin.diag_JtDJ(D)
    beta = 1e-3 * float(diag.mean())

    def f(mc, d=None):                  # phi_d + beta ||m - m0||^2
        with torch.no_grad():
            d = eng.dpred(mc) if d is None else d
            return float(((w * (d - dobs)) ** 2).sum()
                         + beta * ((mc - m0) ** 2).sum())

    f0 = f(m0, d0)

    def H(v):
        return lin.Jtvec(D * lin.Jvec(v)) + beta * 2.0 * v

    Minv = 1.0 / torch.clamp(diag + 2.0 * beta, min=1e-12 * float(diag.max()))
    p, it = pcg(H, -g, Minv, maxiter=20, rtol=1e-2)
    slope = float(g @ p)
    assert slope < 0.0
    # Armijo line search along p (optimization.py:947-975)
    a, accepted, f1 = 1.0, False, f0
    for _ in range(8):
        ft = f(m0 + a * p)
        if ft <= f0 + 1e-4 * a * slope:
            accepted, f1 = True, ft
            break
        a *= 0.5
    eng.check()
    assert accepted and f1 < f0, (f0, f1, a, it)
    # the linearization's products against the oracle at m0
    ops = eng._ops
    op = dict(Lstack=eng._L, crow=ops.crow, col=ops.col, nN=ops.nN,
              Q=ops.q.toarray(), Pd=ops.Pd, sidx=ops.sidx, wq=eng.wq_np,
              slab=O.grid_slabs(mesh.node_grid_index()))
    fields = O.dpred_2d(op, m0_np, return_fields=True)
    rng = np.random.default_rng(13)
    u = rng.standard_normal(m0_np.size)
    v = rng.standard_normal(d0.numel())
    jv = lin.Jvec(torch.tensor(u, device=cuda)).cpu().numpy()
    jt = lin.Jtvec(torch.tensor(v, device=cuda)).cpu().numpy()
    assert rel(jv, O.jvec_2d(op, m0_np, u, fields)) < 1e-9
    assert rel(jt, O._adjoint_2d(op, m0_np, v, fields)[1]) < 1e-9
