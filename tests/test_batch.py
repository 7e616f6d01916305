"""Batched uneven scenes: layout (CPU) and batch-vs-single parity (GPU).

A batch must step every scene exactly as a FlipSolver3D with the same grid,
particles and parameters would: labels bit-exact, grid and particle state
within the float-atomic tolerance of P2G, pressure within the solve
tolerance, with one launch per stage for the whole batch."""
import ctypes

import numpy as np
import pytest

from helpers import rel_l2

GRIDS = [(16, 16, 16), (24, 16, 20), (32, 32, 32)]
BOXES = [((0.0, 0.0, 0.0), (0.5, 0.6, 1.0)), ((0.1, 0.0, 0.2), (0.6, 0.7, 0.9)),
         ((0.0, 0.0, 0.0), (0.3, 0.5, 1.0))]


def _plan(grids):
    from gpufluid_b200 import _lib
    L = _lib.load()
    n = len(grids)
    descs = (_lib.GridDesc * n)()
    for s, (nx, ny, nz) in enumerate(grids):
        dx = 1.0 / max(nx, ny, nz)
        descs[s] = _lib.GridDesc(nx, ny, nz, dx, (ctypes.c_float * 3)(nx * dx, ny * dx, nz * dx))
    rows = (_lib.SceneLayout * n)()
    tot = _lib.BatchTotals()
    st = L.gf_batch_plan(descs, n, rows, ctypes.byref(tot))
    return st, rows, tot


def test_batch_plan_layout():
    st, rows, tot = _plan(GRIDS)
    assert st == 0
    cell = fu = fv = fw = tile = slot = 0
    for (nx, ny, nz), r in zip(GRIDS, rows):
        assert (r.cell0, r.fu0, r.fv0, r.fw0, r.tile0, r.fslot0) == (cell, fu, fv, fw, tile, slot)
        nt = -(-nx // 8) * -(-ny // 8) * -(-nz // 8)
        assert r.ntiles == nt
        cell += nx * ny * nz
        fu += (nx + 1) * ny * nz
        fv += nx * (ny + 1) * nz
        fw += nx * ny * (nz + 1)
        tile += nt
        slot += (nx + 1) * (ny + 1) * (nz + 1)
    assert (tot.ncell, tot.nu, tot.nv, tot.nw, tot.ntiles, tot.nslot) == (cell, fu, fv, fw, tile,
                                                                          slot)


def test_batch_plan_rejects_bad_scenes():
    assert _plan([(16, 0, 16)])[0] == 1
    assert _plan([])[0] == 1
    # sort keys are int32: tiles * 512 must stay below 2^31
    assert _plan([(2048, 2048, 1024)])[0] == 1


def test_cfg_uneven_scenes_is_seeded():
    from gpufluid_b200.batch import cfg_uneven_scenes
    a, b = cfg_uneven_scenes(64, seed=3), cfg_uneven_scenes(64, seed=3)
    assert a == b and len(a) == 64
    assert {s["n"] for s in a} <= {32, 48, 64, 80, 96}
    assert all(0.2 <= s["hi"][0] <= 0.5 and 0.3 <= s["hi"][1] <= 0.7 for s in a)


def _pair(transfer="flip", flip_blend=0.95, tol=1e-4, boxes=BOXES, grids=GRIDS, **kw):
    import torch
    from gpufluid_b200 import FlipSolver3D
    from gpufluid_b200.batch import BatchedFlip3D
    b = BatchedFlip3D(grids, transfer_mode=transfer, flip_blend=flip_blend, pressure_tol=tol, **kw)
    singles = []
    rng = np.random.default_rng(0)
    for s, ((nx, ny, nz), box) in enumerate(zip(grids, boxes)):
        one = FlipSolver3D(nx, ny, nz, transfer_mode=transfer, flip_blend=flip_blend,
                           pressure_tol=tol)
        if box is not None:
            b.seed_box(s, *box)
            one.seed_box(*box)
        # a solid sphere in every scene
        sdf = np.linalg.norm(one.cell_centers_np() - np.float32([0.6, 0.25, 0.5]), axis=-1) - 0.12
        one.add_solid_from_sdf(sdf)
        b.add_solid_from_sdf(s, sdf)
        singles.append(one)
    # identical random initial velocities per scene
    for s, one in enumerate(singles):
        n = one.n_particles
        v = rng.normal(0, 0.3, (n, 3)).astype(np.float32)
        one._set_particles(vel=v)
        a = int(b.part0[s])
        b._vel[a:a + n] = torch.from_numpy(v).to(b.device)
    return b, singles


def _compare(b, singles, tol_grid, tol_part, check_p=True, tol_p=None):
    for s, one in enumerate(singles):
        assert np.array_equal(b.field(s, "marker").cpu().numpy(), one._label.cpu().numpy()), s
        for name, ref in (("u", one._u), ("v", one._v), ("w", one._w)):
            assert rel_l2(b.field(s, name).cpu().numpy(), ref.cpu().numpy()) < tol_grid, (s, name)
        if check_p:
            assert rel_l2(b.field(s, "p").cpu().numpy(), one._p.cpu().numpy()) < (tol_p or tol_grid)
        if one.n_particles:
            bp, bv = b.get_particles(s)
            op, ov = one.get_particles()
            assert rel_l2(bp, op) < tol_part, s
            assert rel_l2(bv, ov) < max(tol_part, tol_grid), s


@pytest.mark.gpu
def test_batch_jacobi_matches_single_scenes(gf):
    b, singles = _pair()
    b.step(1 / 240, pressure_iters=40, pressure_solver="jacobi")
    for one in singles:
        one.step(1 / 240, pressure_iters=40, pressure_solver="jacobi")
    _compare(b, singles, 2e-5, 1e-6)


@pytest.mark.gpu
def test_batch_apic_gsrb_matches_single_scenes(gf):
    b, singles = _pair(transfer="apic")
    for _ in range(3):
        b.step(1 / 240, pressure_iters=20, pressure_solver="gsrb")
        for one in singles:
            one.step(1 / 240, pressure_iters=20, pressure_solver="gsrb")
    _compare(b, singles, 1e-4, 1e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("solver", ["pcg", "pcg_refined"])
def test_batch_pcg_per_scene_convergence(gf, solver):
    tol = 1e-5 if solver == "pcg" else 1e-8
    b, singles = _pair(tol=tol)
    b.step(1 / 240, pressure_iters=2000, pressure_solver=solver)
    for one in singles:
        one.step(1 / 240, pressure_iters=2000, pressure_solver=solver)
    stats = b.pressure_stats()
    for s, (st, one) in enumerate(zip(stats, singles)):
        assert st["status"] == 0, (s, st)
        assert 0 < st["iters"] < 2000
        if solver == "pcg_refined":
            assert st["relres"] <= tol
        # every scene stops at its own tolerance: its iteration count follows
        # its single-scene solve (the single-scene shared-memory solver is the
        # single-reduction variant, a few per cent more iterations), not the
        # slowest scene of the batch
        ref_it = one.last_pressure_iters
        assert 0.7 * ref_it - 10 <= st["iters"] <= 1.3 * ref_it + 10, (s, st, ref_it)
    assert len({st["iters"] for st in stats}) > 1
    _compare(b, singles, 1e-4, 1e-5, tol_p=1e-4 if solver == "pcg" else 1e-6)


@pytest.mark.gpu
def test_batch_pcg_tile_sgs_preconditioner(gf):
    """The segmented PCG with the tile-local SGS preconditioner: every scene
    reaches its own FP64-residual target, fewer iterations than with the
    reference's Jacobi preconditioner, the same pressures."""
    tol = 1e-8
    res = {}
    for precond in ("jacobi", "tile_sgs"):
        b, singles = _pair(tol=tol)
        b.pcg_preconditioner = precond
        b.step(1 / 240, pressure_iters=2000, pressure_solver="pcg_refined")
        for one in singles:
            one.step(1 / 240, pressure_iters=2000, pressure_solver="pcg_refined")
        stats = b.pressure_stats()
        for s, st in enumerate(stats):
            assert st["status"] == 0 and st["relres"] <= tol, (precond, s, st)
        res[precond] = [st["iters"] for st in stats]
        _compare(b, singles, 1e-4, 1e-5, tol_p=1e-6)
    assert sum(res["tile_sgs"]) < sum(res["jacobi"]), res


@pytest.mark.gpu
def test_batch_empty_scene_and_graph_replay(gf):
    import torch
    boxes = [BOXES[0], None, BOXES[2]]
    b, singles = _pair(boxes=boxes)
    b2, _ = _pair(boxes=boxes, enable_cuda_graphs=False)
    for _ in range(3):
        b.step(1 / 240, pressure_iters=500, pressure_solver="pcg_refined")
        b2.step(1 / 240, pressure_iters=500, pressure_solver="pcg_refined")
    torch.cuda.synchronize()
    st = b.pressure_stats()
    assert st[1]["status"] == 0 and st[1]["iters"] == 0
    assert float(b.field(1, "p").abs().max()) == 0.0
    for s in (0, 2):
        pa, _ = b.get_particles(s)
        pb, _ = b2.get_particles(s)
        assert rel_l2(pa, pb) < 1e-5
    assert b.launch_count() > 0


@pytest.mark.gpu
def test_batch_autotune_restores_state(gf):
    import torch
    b, _ = _pair()
    b.step(1 / 240, pressure_iters=200, pressure_solver="pcg")
    torch.cuda.synchronize()
    before = b._pos.clone(), b._vel.clone(), b._pid.clone()
    info = b.autotune(1 / 240, pressure_iters=200, pressure_solver="pcg")
    torch.cuda.synchronize()
    assert info["g2p_threads"] in (128, 256, 512)
    assert info["grid_threads"] in (128, 256, 512)
    assert info["pcg_blocks_per_sm"] in (0, 1, 2)
    assert info["step_ms_after"] > 0
    for x, y in zip(before, (b._pos, b._vel, b._pid)):
        assert torch.equal(x, y)
    b.step(1 / 240, pressure_iters=200, pressure_solver="pcg")
    assert all(s["status"] == 0 for s in b.pressure_stats())
