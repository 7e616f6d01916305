"""Parity at the benchmark workloads' sizes: the CUDA path against the CPU
oracle (the C restatement of the reference's kernels, pinned bit for bit to
src/gpufluid/solvers/solver3d.py by tests/test_oracle_golden.py) on the same
seeded inputs.

* 64^3 FLIP dam break (486,400 particles, dt = 1/240, 60 substeps):
  - Jacobi, 200 sweeps (the reference's default solver): every stage but
    P2G is bit-exact, so the two runs differ only by the float-atomic order
    of the P2G sums; labels bit-exact after substep 1, and the drift of
    particles, faces and pressure over 60 substeps is bounded below;
  - Jacobi-preconditioned PCG to 1e-5 (at most 200 iterations): the GPU's
    single-reduction CG and the oracle's reference-order CG both stop at a
    relative residual of 1e-5 but at different iterates, so the drift is the
    solver tolerance's; iteration counts agree to one check interval;
  - the reference PCG's sign (r0 = +div) for 5 substeps: same comparison.
* 128^3 APIC dam break with the sphere obstacle (3,969,024 particles,
  dt = 1/480): one substep stage by stage, from the seeded state and from
  the state after 20 substeps -- binning keys, per-cell counts, sort order and
  labels bit-exact; P2G within relative L2 2e-6 with the exact zero pattern;
  forces/BC/divergence, projection and G2P (with the C matrices) bit-exact
  given the oracle's inputs; the refined PCG (tile SGS + coarse correction)
  within 1e-6 of an FP64 solve of the oracle's system.
* 256^3 double dam break (56,088,576 particles): the first substep's
  pressure system through the global-memory PCG (the active region exceeds
  the shared-memory solver), refined to 1e-7 with the reference's Jacobi
  preconditioner and with the tile SGS one, against an FP64 CG solve of the
  same system; 20 Jacobi sweeps bit-exact against the oracle.

``GF_PARITY_OUT`` (an environment variable naming a directory) makes the
64^3 runs write their per-substep drift tables there as JSON.
"""
import ctypes
import json
import os

import numpy as np
import pytest

from helpers import assert_bitexact, rel_l2

pytestmark = pytest.mark.gpu

BOX = ((0.0, 0.0, 0.0), (0.4, 0.6, 1.0))


def _t(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _call(s, name, *args):
    from gpufluid_b200 import _lib
    s._set_stream()
    _lib.check(getattr(s._L, name)(s._ctx, *args), s._ctx, name)


def _dump(name, table):
    out = os.environ.get("GF_PARITY_OUT")
    if out:
        os.makedirs(out, exist_ok=True)
        with open(os.path.join(out, f"{name}.json"), "w") as f:
            json.dump(table, f, indent=1)


def _rollout_64(gf, oracle, solver, steps, tol=1e-5, rhs_sign=-1):
    """Step the GPU solver and the oracle side by side; per substep: label
    mismatches, relative L2 of positions, velocities, faces and pressure,
    pressure iterations of each."""
    import torch
    n, dt = 64, 1.0 / 240.0
    s = gf.FlipSolver3D(n, n, n, transfer_mode="flip", flip_blend=0.95, pressure_tol=tol,
                        pcg_rhs_sign=rhs_sign)
    s.seed_box(*BOX)
    o = oracle.OracleFlip(n, n, n, transfer_mode="flip", flip_blend=0.95, par=True)
    pos0 = oracle.seed_box(o.dx, *BOX)
    assert pos0.shape == (486400, 3)
    assert_bitexact("seeded positions", s.pos.numpy(), pos0)
    o.set_particles(pos0, np.zeros_like(pos0))
    rows = []
    for k in range(steps):
        s.step(dt, pressure_iters=200, pressure_solver=solver)
        o.step(dt, pressure_iters=200, pressure_solver=solver, tol=tol, check_every=10,
               rhs_sign=rhs_sign)
        torch.cuda.synchronize()
        pos, vel = s.get_particles()
        rows.append({
            "substep": k + 1,
            "label_mismatch": int((s.marker.numpy() != o.marker).sum()),
            "pos": rel_l2(pos, o.pos), "vel": rel_l2(vel, o.vel),
            "u": rel_l2(s.u.numpy(), o.u), "v": rel_l2(s.v.numpy(), o.v),
            "w": rel_l2(s.w.numpy(), o.w), "p": rel_l2(s.p.numpy(), o.p),
            "iters_gpu": s.last_pressure_iters, "iters_oracle": o.last_pressure_iters,
        })
    return rows


def test_cfg1_jacobi_60_substeps_track_the_oracle(gf, oracle):
    rows = _rollout_64(gf, oracle, "jacobi", 60)
    _dump("cfg1_jacobi", rows)
    first, last = rows[0], rows[-1]
    assert first["label_mismatch"] == 0
    assert first["pos"] < 1e-7 and first["vel"] < 1e-6 and first["p"] < 1e-6, first
    # drift from the float-atomic order of the P2G sums alone
    worst = {k: max(r[k] for r in rows) for k in ("pos", "vel", "u", "v", "w", "p")}
    assert worst["pos"] < 1e-5, worst
    assert worst["vel"] < 1e-3 and worst["p"] < 1e-3, worst
    assert max(r["label_mismatch"] for r in rows) <= 64, [r["label_mismatch"] for r in rows]
    assert all(r["iters_gpu"] == 200 for r in rows)
    assert np.isfinite(last["pos"])


def test_cfg1_pcg_60_substeps_track_the_oracle(gf, oracle):
    rows = _rollout_64(gf, oracle, "pcg", 60)
    _dump("cfg1_pcg", rows)
    first = rows[0]
    assert first["label_mismatch"] == 0
    assert first["pos"] < 1e-6 and first["p"] < 1e-3, first
    for r in rows:
        assert abs(r["iters_gpu"] - r["iters_oracle"]) <= 10, r
    worst = {k: max(r[k] for r in rows) for k in ("pos", "vel", "p")}
    assert worst["pos"] < 1e-4 and worst["vel"] < 2e-2 and worst["p"] < 2e-2, worst


def test_cfg1_reference_pcg_sign_tracks_the_oracle(gf, oracle):
    """The reference's PCG right-hand-side sign (it doubles the divergence
    instead of removing it): the GPU path reproduces the oracle's run."""
    rows = _rollout_64(gf, oracle, "pcg", 5, rhs_sign=+1)
    _dump("cfg1_pcg_reference_sign", rows)
    assert rows[0]["label_mismatch"] == 0
    for r in rows:
        assert abs(r["iters_gpu"] - r["iters_oracle"]) <= 10, r
        assert r["pos"] < 1e-4 and r["p"] < 1e-2, r


# ------------------------------------------------------------ 128^3 APIC
def _cfg2_solver(gf):
    from gpufluid_b200 import scene
    s = gf.FlipSolver3D(128, 128, 128, transfer_mode="apic", flip_blend=0.95, pressure_tol=1e-8,
                        pcg_preconditioner="tile_sgs", pcg_sgs_sweeps=2, pcg_coarse=True)
    s.add_solid_from_sdf(scene.sdf_sphere(s.cell_centers_np(), (0.7, 0.2, 0.5), 0.12))
    s.seed_box(*BOX)
    return s


@pytest.mark.parametrize("warm", [0, 20])
def test_cfg2_substep_stage_by_stage(gf, oracle, warm):
    import torch
    from gpufluid_b200 import _lib
    dt = 1.0 / 480.0
    s = _cfg2_solver(gf)
    assert s.n_particles == 3969024
    for _ in range(warm):
        s.step(dt, pressure_iters=4000, pressure_solver="pcg_refined")
    pos, vel = s.get_particles()
    C = s.affine_C.numpy()
    if warm:
        assert np.abs(vel).max() > 0.1 and np.abs(C).max() > 0.1
    # the oracle takes the GPU's state as its input
    o = oracle.OracleFlip(128, 128, 128, transfer_mode="apic", flip_blend=0.95, par=True)
    o.marker[...] = s._wall_marker
    o.marker[oracle.sphere_sdf(128, 128, 128, o.dx, (0.7, 0.2, 0.5), 0.12) <= 0.0] = 2
    assert_bitexact("static labels", s._marker_host, o.marker)
    o.set_particles(pos, vel, C)
    s._set_particles(pos=pos, vel=vel, C=C)  # storage order = id order
    code = _lib.GF_APIC
    # binning + labels
    _call(s, "gf_bin", code)
    torch.cuda.synchronize()
    key_o, count_o, order_o = oracle.bin_particles(128, 128, 128, s.dx, pos)
    P = pos.shape[0]
    key_g, order_g = np.empty(P, np.int32), np.empty(P, np.int32)
    count_g = np.empty(count_o.shape[0], np.int32)
    s._set_stream()
    assert s._L.gf_bin_read(s._ctx, key_g.ctypes.data, count_g.ctypes.data,
                            order_g.ctypes.data, None) == 0
    assert_bitexact("keys", key_g, key_o)
    assert_bitexact("per-cell counts", count_g, count_o)
    assert_bitexact("sort order", order_g, order_o.astype(np.int32))
    # P2G
    _call(s, "gf_p2g", code)
    torch.cuda.synchronize()
    o.clear(); o.p2g()
    assert_bitexact("labels", s.marker.numpy(), o.marker)
    for k in ("u", "v", "w"):
        g = getattr(s, "_" + k).cpu().numpy()
        assert rel_l2(g, getattr(o, k)) < 2e-6, (k, rel_l2(g, getattr(o, k)))
    for k in ("uw", "vw", "ww"):
        g = getattr(s, k).cpu().numpy()
        assert rel_l2(g, getattr(o, k)) < 2e-6, (k, rel_l2(g, getattr(o, k)))
        assert np.array_equal(g == 0, getattr(o, k) == 0), k
    # forces + BC + divergence on the oracle's P2G output
    for k in ("u", "v", "w"):
        getattr(s, "_" + k).copy_(_t(getattr(o, k)))
    for k in ("uw", "vw", "ww"):
        getattr(s, k).copy_(_t(getattr(o, k)))
    _call(s, "gf_forces_div", ctypes.c_float(s.gravity), ctypes.c_float(dt),
          ctypes.c_float(s.rho))
    torch.cuda.synchronize()
    o.normalize(); o.gravity_bc(dt); o.divergence(dt)
    for k in ("u", "v", "w", "us", "vs", "ws"):
        got = (getattr(s, "_" + k) if k in ("u", "v", "w") else getattr(s, k)).cpu().numpy()
        assert_bitexact(k, got, getattr(o, k))
    assert_bitexact("div", s.div.cpu().numpy(), o.div)
    # the headline pressure solve against FP64
    prm = s._params(dt, 4000, "pcg_refined")
    _call(s, "gf_pressure", ctypes.byref(prm), None)
    st = s.pressure_stats()
    assert st["status"] == 0 and st["kernel"] == 1 and st["coarse"] == 1, st
    assert st["relres"] <= 1e-8, st
    p64, _, rel64 = oracle.pcg64(o.marker, o.div, tol=1e-13)
    assert rel64 <= 1e-12
    err = rel_l2(s._p.cpu().numpy(), p64)
    assert err < 1e-6, err
    # projection and G2P on the same pressure (the FP64 one, rounded)
    p32 = p64.astype(np.float32)
    o.p[...] = p32
    s._p.copy_(_t(p32))
    _call(s, "gf_project", ctypes.c_float(dt), ctypes.c_float(s.rho))
    torch.cuda.synchronize()
    o.grad_bc(dt)
    for k in ("u", "v", "w"):
        assert_bitexact(k + " projected", getattr(s, "_" + k).cpu().numpy(), getattr(o, k))
    _call(s, "gf_g2p", code, ctypes.c_float(s.flip_blend), ctypes.c_float(dt))
    torch.cuda.synchronize()
    o.g2p(dt)
    assert_bitexact("pos", s.pos.numpy(), o.pos)
    assert_bitexact("vel", s.vel.numpy(), o.vel)
    assert_bitexact("C", s.affine_C.numpy(), o.C)


# ------------------------------------------------------------ 256^3
def _fp64_cg(torch, lab, b, tol=1e-13, max_iter=20000):
    """FP64 Jacobi-preconditioned CG on the device for A p = b on the fluid
    cells (A: #non-solid neighbours on the diagonal, -1 per fluid
    neighbour), built from the labels with dense tensor ops."""
    lab = lab.to(torch.int32)
    fl = lab == 1
    nx, ny, nz = lab.shape
    pad = torch.nn.functional.pad(lab, (1, 1, 1, 1, 1, 1), value=2)
    views = []
    for ax in range(3):
        for sh in (0, 2):
            sl = [slice(1, 1 + nx), slice(1, 1 + ny), slice(1, 1 + nz)]
            sl[ax] = slice(sh, sh + lab.shape[ax])
            views.append(tuple(sl))
    diag = sum((pad[v] != 2).double() for v in views)
    nbf = [(pad[v] == 1) for v in views]
    flf = fl.double()
    inv_d = torch.where(fl, 1.0 / diag.clamp(min=1.0), torch.zeros_like(diag))

    def A(x):
        xp = torch.nn.functional.pad(x, (1, 1, 1, 1, 1, 1))
        acc = sum(torch.where(m, xp[v], torch.zeros_like(x)) for m, v in zip(nbf, views))
        return (diag * x - acc) * flf

    b = torch.where(fl, b, torch.zeros_like(b))
    x = torch.zeros_like(b)
    r = b.clone()
    z = r * inv_d
    d = z.clone()
    rz = float((r * z).sum())
    bb = float(torch.linalg.vector_norm(b))
    for it in range(max_iter):
        q = A(d)
        alpha = rz / float((d * q).sum())
        x += alpha * d
        r -= alpha * q
        if it % 10 == 0 and float(torch.linalg.vector_norm(r)) < tol * bb:
            break
        z = r * inv_d
        rz_new = float((r * z).sum())
        d = z + (rz_new / rz) * d
        rz = rz_new
    return x, float(torch.linalg.vector_norm(b - A(x))) / bb


def test_cfg3_256_global_pcg_against_fp64(gf, oracle):
    import torch
    from gpufluid_b200 import _lib
    n, dt = 256, 1.0 / 960.0
    s = gf.FlipSolver3D(n, n, n, transfer_mode="flip", flip_blend=0.97, pressure_tol=1e-7)
    s.seed_box((0.0, 0.0, 0.0), (0.3, 0.7, 1.0))
    s.seed_box((0.7, 0.0, 0.0), (1.0, 0.7, 1.0), append=True)
    assert s.n_particles == 56088576
    for name, args in (("gf_bin", (0,)), ("gf_p2g", (0,)),
                       ("gf_forces_div", (ctypes.c_float(s.gravity), ctypes.c_float(dt),
                                          ctypes.c_float(s.rho)))):
        _call(s, name, *args)
    torch.cuda.synchronize()
    lab_dev, div_dev = s._label.clone(), s.div.clone()
    x64, rel = _fp64_cg(torch, lab_dev, -div_dev.double())
    assert rel < 1e-11, rel  # the reference solve: its error is far below the 1e-5 checked
    fl = lab_dev == 1
    iters = {}
    for precond in ("jacobi", "tile_sgs", "tile_sgs+coarse"):
        s.pcg_preconditioner = precond.split("+")[0]
        s.pcg_coarse = precond.endswith("coarse")
        prm = s._params(dt, 8000, "pcg_refined")
        _call(s, "gf_pressure", ctypes.byref(prm), None)
        st = s.pressure_stats()
        assert st["kernel"] == 2, st  # the global-memory solver
        assert st["coarse"] == (1 if s.pcg_coarse else 0), (precond, st)
        assert st["status"] == 0 and st["relres"] <= 1e-7, (precond, st)
        assert st["n_fluid"] > 6_000_000
        p = torch.where(fl, s._p.double(), torch.zeros_like(x64))
        err = float(torch.linalg.vector_norm(p - x64) / torch.linalg.vector_norm(x64))
        assert err < 1e-5, (precond, err)
        iters[precond] = st["iters"]
    assert iters["tile_sgs+coarse"] < iters["tile_sgs"] < iters["jacobi"], iters
    s.pcg_preconditioner = "jacobi"
    s.pcg_coarse = False
    # 20 Jacobi sweeps: bit-exact against the oracle on the same system
    prm = s._params(dt, 20, "jacobi")
    s.div.copy_(div_dev)
    s._label.copy_(lab_dev)
    _call(s, "gf_pressure", ctypes.byref(prm), None)
    torch.cuda.synchronize()
    o = oracle.OracleFlip(n, n, n, par=True)
    o.marker[...] = lab_dev.cpu().numpy().astype(np.int32)
    o.div[...] = div_dev.cpu().numpy()
    o.pressure("jacobi", 20)
    assert_bitexact("p (jacobi x20, 256^3)", s._p.cpu().numpy(), o.p)
