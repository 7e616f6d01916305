"""The FP64 finite-difference reference (oracle/pic64.py) against the
golden-pinned float32 oracle: one PIC substep, same labels, agreement to
float32 rounding."""
import numpy as np

from helpers import rel_l2


def test_pic64_substep_matches_fp32_oracle(oracle):
    from oracle.pic64 import PicFP64
    n = 24
    o = oracle.OracleFlip(n, n, n, transfer_mode="pic", flip_blend=0.0)
    pos = oracle.seed_box(o.dx, (0.2, 0.1, 0.25), (0.6, 0.55, 0.7))
    rng = np.random.default_rng(3)
    vel = rng.normal(0, 0.3, pos.shape).astype(np.float32)
    o.set_particles(pos, vel)
    dt = 1.0 / 240.0
    o.step(dt, pressure_iters=2000, pressure_solver="pcg64", tol=1e-13)
    ref = PicFP64(n)
    lab = oracle.wall_marker(n, n, n)
    o2 = oracle.OracleFlip(n, n, n, transfer_mode="pic", flip_blend=0.0)
    o2.set_particles(pos, vel)
    o2.clear(); o2.p2g()
    lab = o2.marker.copy()
    x, v = ref.substep(pos.astype(np.float64), vel.astype(np.float64), lab, dt, key=0)
    assert rel_l2(v, o.vel) < 1e-5, rel_l2(v, o.vel)
    assert rel_l2(x, o.pos) < 1e-6


def test_pic64_splat_matches_fp32_oracle(oracle):
    from oracle.pic64 import PicFP64
    n = 20
    rng = np.random.default_rng(0)
    pos = (rng.random((5000, 3)) * 0.9 + 0.05).astype(np.float32)
    a = PicFP64(n).splat(pos.astype(np.float64))
    b = oracle.density_splat(n, n, n, 1.0 / n, pos)
    assert rel_l2(a, b) < 1e-6


def test_pic64_adjoint_matches_finite_differences():
    """The FP64 reverse-mode gradient of the rollout loss against central
    differences of the same FP64 forward (3 substeps, 12^3, fixed labels)."""
    from oracle.pic64 import PicFP64
    n, T, dt = 12, 3, 1.0 / 240.0
    ref = PicFP64(n)
    rng = np.random.default_rng(5)
    x0 = (rng.random((900, 3)) * 0.4 + 0.3).astype(np.float64)
    control = rng.normal(0, 0.5, (3, n, n, n))
    labels = []
    x, v = x0.copy(), ref.sample_cells(control, x0)
    for t in range(T):
        lab = np.zeros((n, n, n), np.uint8)
        lab[0] = lab[-1] = 2; lab[:, 0] = lab[:, -1] = 2; lab[:, :, 0] = lab[:, :, -1] = 2
        c = np.floor(x * n).astype(int)
        inner = lab[c[:, 0], c[:, 1], c[:, 2]] != 2
        lab[c[inner, 0], c[inner, 1], c[inner, 2]] = 1
        labels.append(lab)
        x, v = ref.substep(x, v, lab, dt, key=t)
    target = ref.splat(x0 + np.array([0.08, 0.04, 0.0]))
    g = ref.grad(control, x0, labels, dt, target)
    eps = 1e-4
    for _ in range(3):
        d = rng.normal(size=control.shape)
        d /= np.linalg.norm(d)
        fd = (ref.loss(control + eps * d, x0, labels, dt, target)
              - ref.loss(control - eps * d, x0, labels, dt, target)) / (2 * eps)
        assert abs(float((g * d).sum()) - fd) <= 1e-6 * abs(fd), (float((g * d).sum()), fd)


def test_apic64_substep_matches_fp32_oracle(oracle):
    """The FP64 APIC substep against the float32 oracle (k3_p2g_apic,
    k3_g2p_apic_advect): one substep, same labels, float32 rounding."""
    from oracle.pic64 import PicFP64
    n = 24
    pos = oracle.seed_box(1.0 / n, (0.2, 0.1, 0.25), (0.6, 0.55, 0.7))
    rng = np.random.default_rng(4)
    vel = rng.normal(0, 0.3, pos.shape).astype(np.float32)
    C = rng.normal(0, 0.5, (len(pos), 3, 3)).astype(np.float32)
    dt = 1.0 / 240.0
    o = oracle.OracleFlip(n, n, n, transfer_mode="apic")
    o.set_particles(pos, vel, C)
    o.step(dt, pressure_iters=2000, pressure_solver="pcg64", tol=1e-13)
    o2 = oracle.OracleFlip(n, n, n, transfer_mode="apic")
    o2.set_particles(pos, vel, C)
    o2.clear(); o2.p2g()
    lab = o2.marker.copy()
    x, v, Cn = PicFP64(n).substep_apic(pos.astype(np.float64), vel.astype(np.float64),
                                       C.astype(np.float64), lab, dt, key=0)
    assert rel_l2(v, o.vel) < 1e-5, rel_l2(v, o.vel)
    assert rel_l2(Cn, o.C) < 1e-4, rel_l2(Cn, o.C)
    assert rel_l2(x, o.pos) < 1e-6


def test_apic64_adjoint_matches_finite_differences():
    """The FP64 reverse-mode gradient of the APIC rollout loss against central
    differences of the same FP64 forward (3 substeps, 12^3, fixed labels)."""
    from oracle.pic64 import PicFP64
    n, T, dt = 12, 3, 1.0 / 240.0
    ref = PicFP64(n)
    rng = np.random.default_rng(5)
    x0 = rng.random((900, 3)) * 0.4 + 0.3
    control = rng.normal(0, 0.5, (3, n, n, n))
    labels = []
    x, v, C = x0.copy(), ref.sample_cells(control, x0), np.zeros((900, 3, 3))
    for t in range(T):
        lab = np.zeros((n, n, n), np.uint8)
        lab[0] = lab[-1] = 2; lab[:, 0] = lab[:, -1] = 2; lab[:, :, 0] = lab[:, :, -1] = 2
        c = np.floor(x * n).astype(int)
        inner = lab[c[:, 0], c[:, 1], c[:, 2]] != 2
        lab[c[inner, 0], c[inner, 1], c[inner, 2]] = 1
        labels.append(lab)
        x, v, C = ref.substep_apic(x, v, C, lab, dt, key=t)
    assert np.abs(C).max() > 0.1  # the affine term is exercised
    target = ref.splat(x0 + np.array([0.08, 0.04, 0.0]))
    g = ref.grad_apic(control, x0, labels, dt, target)
    eps = 1e-4
    for _ in range(3):
        d = rng.normal(size=control.shape)
        d /= np.linalg.norm(d)
        fd = (ref.loss_apic(control + eps * d, x0, labels, dt, target)
              - ref.loss_apic(control - eps * d, x0, labels, dt, target)) / (2 * eps)
        assert abs(float((g * d).sum()) - fd) <= 1e-6 * abs(fd), (float((g * d).sum()), fd)
