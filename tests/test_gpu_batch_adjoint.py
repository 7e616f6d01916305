"""Batched forward+adjoint of the drop-shaping loss over scenes of uneven
sizes (one batch context, one launch per kernel for all scenes).  Each
scene's block of the batched gradient is checked against the FP64 reverse-
mode gradient of that scene alone (oracle/pic64.py, on the scene's own
per-substep labels from the batched run) and against the single-scene GPU
adjoint; each scene's loss against the FP64 loss."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _controls(sides, seed):
    rng = np.random.default_rng(seed)
    return [rng.normal(0, 0.1, (3, n, n, n)).astype(np.float32) for n in sides]


def _check_batch(sides, T, k, transfer, seed):
    import torch
    from gpufluid_b200.adjoint import BatchedDropShaping, DropShaping
    from oracle.pic64 import PicFP64
    prob = BatchedDropShaping(sides, T=T, k=k, transfer=transfer)
    ctrl = _controls(sides, seed)
    c_t = torch.zeros(prob.control_shape, dtype=torch.float32, device="cuda")
    for s, c in enumerate(ctrl):
        prob.scene_control(c_t, s).copy_(torch.from_numpy(c))
    loss, ckpts = prob.forward(c_t, keep_labels=True)
    losses = prob.scene_losses()
    # a second splat (float atomics in another order) differs in the last bits
    assert abs(losses.sum() - loss) <= 1e-6 * abs(loss)
    grad = prob.backward(c_t, ckpts)
    x0 = prob.x0.cpu().numpy()
    part0 = prob.solver.part0
    target = prob.target.cpu().numpy().astype(np.float64)
    apic = transfer == "apic"
    for s, n in enumerate(sides):
        c0 = prob.cell0[s]
        labels = [l[c0:c0 + n ** 3].cpu().numpy().reshape(n, n, n) for l in prob.labels_log]
        xs = x0[part0[s]:part0[s + 1]]
        ts = target[c0:c0 + n ** 3].reshape(n, n, n)
        ref = PicFP64(n)
        loss_fn = ref.loss_apic if apic else ref.loss
        grad_fn = ref.grad_apic if apic else ref.grad
        L64 = loss_fn(ctrl[s], xs, labels, prob.dt, ts)
        assert abs(L64 - losses[s]) <= 1e-6 * abs(L64), (s, L64, losses[s])
        g = prob.scene_control(grad, s).cpu().numpy().astype(np.float64)
        g64 = grad_fn(ctrl[s], xs, labels, prob.dt, ts)
        rel = np.linalg.norm(g - g64) / np.linalg.norm(g64)
        assert rel < 1e-4, (s, rel)
        # the scene run alone on a single-grid context
        one = DropShaping(n=n, T=T, k=k, transfer=transfer)
        cs = torch.from_numpy(ctrl[s]).cuda()
        l1, ck1 = one.forward(cs)
        g1 = one.backward(cs, ck1).cpu().numpy().astype(np.float64)
        assert abs(l1 - losses[s]) <= 1e-5 * abs(l1), (s, l1, losses[s])
        rel1 = np.linalg.norm(g - g1) / np.linalg.norm(g1)
        assert rel1 < 1e-4, (s, rel1)


def test_batched_adjoint_pic_uneven(gf):
    """Three scenes (24^3, 16^3, 32^3): 5 substeps, checkpoints every 2."""
    _check_batch((24, 16, 32), T=5, k=2, transfer="pic", seed=3)


def test_batched_adjoint_apic_uneven(gf):
    """The same scenes with APIC transfer (affine-matrix adjoint carried)."""
    _check_batch((24, 16, 32), T=5, k=2, transfer="apic", seed=5)


def test_batched_rollout_autograd(gf):
    import torch
    from gpufluid_b200.adjoint import BatchedDropShaping, RolloutLoss
    prob = BatchedDropShaping((16, 24), T=3, k=2)
    control = torch.zeros(prob.control_shape, dtype=torch.float32, device="cuda")
    for s, c in enumerate(_controls((16, 24), 9)):
        prob.scene_control(control, s).copy_(torch.from_numpy(c))
    control.requires_grad_(True)
    loss = RolloutLoss.apply(control, prob)
    loss.backward()
    assert control.grad is not None and control.grad.shape == control.shape
    assert float(control.grad.abs().sum()) > 0
