"""Adjoint substep (PIC, labels fixed per substep) against central finite
differences of an FP64 CPU forward (oracle/pic64.py) run on the same per-
substep labels.  The directional derivative <grad, d> of the GPU adjoint must
match (L(c + eps d) - L(c - eps d)) / (2 eps) within 1e-3 relative, and the
whole gradient must match the FP64 reverse-mode gradient of the same forward
(itself checked against finite differences on the CPU) within 1e-4 relative
L2."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _check(problem, control, n_dirs, eps, tol, seed, tol_l2=1e-4):
    import torch
    from oracle.pic64 import PicFP64
    c_t = torch.from_numpy(control).cuda()
    loss_gpu, ckpts = problem.forward(c_t, keep_labels=True)
    grad = problem.backward(c_t, ckpts).cpu().numpy().astype(np.float64)
    labels = [l.cpu().numpy() for l in problem.labels_log]
    x0 = problem.x0.cpu().numpy()
    target = problem.target.cpu().numpy().astype(np.float64)
    ref = PicFP64(problem.n)
    apic = problem.transfer == "apic"
    loss_fn = ref.loss_apic if apic else ref.loss
    grad_fn = ref.grad_apic if apic else ref.grad
    L0 = loss_fn(control, x0, labels, problem.dt, target)
    assert abs(L0 - loss_gpu) <= 1e-6 * abs(L0), (L0, loss_gpu)
    g64 = grad_fn(control, x0, labels, problem.dt, target)
    rel = np.linalg.norm(grad - g64) / np.linalg.norm(g64)
    assert rel < tol_l2, rel
    rng = np.random.default_rng(seed)
    ad, fd = [], []
    for _ in range(n_dirs):
        d = rng.normal(size=control.shape)
        d /= np.linalg.norm(d)
        lp = loss_fn(control + eps * d, x0, labels, problem.dt, target)
        lm = loss_fn(control - eps * d, x0, labels, problem.dt, target)
        fd.append((lp - lm) / (2 * eps))
        ad.append(float((grad * d).sum()))
    ad, fd = np.array(ad), np.array(fd)
    scale = np.maximum(np.abs(fd), 0.05 * np.abs(fd).max())
    err = np.abs(ad - fd) / scale
    assert err.max() < tol, list(zip(ad, fd, err))
    return err


def test_adjoint_small_uneven_segments(gf):
    """32^3, 7 substeps with checkpoints every 3 (a short last segment)."""
    from gpufluid_b200.adjoint import DropShaping
    prob = DropShaping(n=32, T=7, k=3)
    control = np.random.default_rng(1).normal(0, 0.1, (3, 32, 32, 32)).astype(np.float32)
    _check(prob, control, n_dirs=6, eps=1e-3, tol=1e-3, seed=11)


def test_adjoint_drop_shaping_64(gf):
    """The 64^3 drop-shaping problem: 40 substeps at dt 1/240, checkpoints
    every 10, 16 seeded directions, eps 1e-3."""
    from gpufluid_b200.adjoint import DropShaping
    prob = DropShaping(n=64, T=40, k=10)
    control = np.random.default_rng(4).normal(0, 0.1, (3, 64, 64, 64)).astype(np.float32)
    _check(prob, control, n_dirs=16, eps=1e-3, tol=1e-3, seed=7)


def test_rollout_loss_autograd(gf):
    import torch
    from gpufluid_b200.adjoint import DropShaping, RolloutLoss
    prob = DropShaping(n=32, T=4, k=2)
    control = torch.from_numpy(
        np.random.default_rng(2).normal(0, 0.1, (3, 32, 32, 32)).astype(np.float32)).cuda()
    control.requires_grad_(True)
    loss = RolloutLoss.apply(control, prob)
    loss.backward()
    _, ck = prob.forward(control.detach())
    g2 = prob.backward(control.detach(), ck)
    assert control.grad is not None and control.grad.shape == control.shape
    assert torch.allclose(control.grad, g2, rtol=1e-4, atol=1e-7 * float(g2.abs().max()))


def test_adjoint_apic_small_uneven_segments(gf):
    """APIC transfer: 32^3, 7 substeps with checkpoints every 3; the affine
    matrices' adjoint is carried through the substeps."""
    from gpufluid_b200.adjoint import DropShaping
    prob = DropShaping(n=32, T=7, k=3, transfer="apic")
    control = np.random.default_rng(1).normal(0, 0.1, (3, 32, 32, 32)).astype(np.float32)
    _check(prob, control, n_dirs=6, eps=1e-3, tol=1e-3, seed=11)


def test_adjoint_apic_drop_shaping_64(gf):
    """The 64^3 drop-shaping problem with APIC transfer: 40 substeps at dt
    1/240, checkpoints every 10, 16 seeded directions, eps 1e-3."""
    from gpufluid_b200.adjoint import DropShaping
    prob = DropShaping(n=64, T=40, k=10, transfer="apic")
    control = np.random.default_rng(4).normal(0, 0.1, (3, 64, 64, 64)).astype(np.float32)
    _check(prob, control, n_dirs=16, eps=1e-3, tol=1e-3, seed=7)
