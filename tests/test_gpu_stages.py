"""Stage-by-stage parity of the CUDA path against the CPU oracle.

Each test loads the same inputs into the GPU solver's buffers and into the
oracle, runs ONE stage through the C ABI, and compares:

* bit-exact: cell labels, per-cell keys/counts, the (cell, particle id) sort
  order, forces+BC+divergence, Jacobi, GS-RB, projection, G2P (FLIP, PIC,
  APIC) -- deterministic stages compiled without FMA contraction;
* relative L2 <= 2e-6 (P2G face sums and weights): float atomics make the
  summation order differ from the oracle's particle order;
* PCG: the fixed-order device reductions differ from the oracle's sequential
  float32 dots, so the solution is compared within a tolerance and against
  an FP64 solve.
"""
import ctypes

import numpy as np
import pytest

from helpers import assert_bitexact, rel_l2, random_particles

pytestmark = pytest.mark.gpu

GRIDS = [(16, 12, 10), (24, 24, 24), (13, 21, 9)]


def _mk(gf, grid, transfer="flip", sphere=None):
    import torch
    nx, ny, nz = grid
    s = gf.FlipSolver3D(nx, ny, nz, transfer_mode=transfer)
    if sphere is not None:
        from gpufluid_b200 import scene
        s.add_solid_from_sdf(scene.sdf_sphere(s.cell_centers_np(), *sphere))
    return s


def _oracle(oracle, s):
    o = oracle.OracleFlip(s.nx, s.ny, s.nz, transfer_mode=s.transfer_mode,
                          flip_blend=s.flip_blend)
    o.marker[...] = s._marker_host
    return o


def _call(s, name, *args):
    from gpufluid_b200 import _lib
    s._set_stream()
    _lib.check(getattr(s._L, name)(s._ctx, *args), s._ctx, name)


def _t(a, dev="cuda"):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


@pytest.mark.parametrize("grid", GRIDS)
def test_bin_labels_keys_order_bitexact(gf, oracle, grid):
    import torch
    nx, ny, nz = grid
    s = _mk(gf, grid, sphere=((0.5 * nx / max(grid), 0.3, 0.5 * nz / max(grid)), 0.2))
    pos, vel, _ = random_particles(nx, ny, nz, s.dx, 20000, seed=nx)
    s.pos = pos
    s.vel = vel
    _call(s, "gf_bin", 0)
    torch.cuda.synchronize()
    # labels: clear + mark, as k3_clear_grid + k3_p2g
    o = _oracle(oracle, s)
    o.set_particles(pos, vel)
    o.clear(); o.p2g()
    assert_bitexact("labels", s.marker.numpy(), o.marker)
    key_o, count_o, order_o = oracle.bin_particles(nx, ny, nz, s.dx, pos)
    n = pos.shape[0]
    key_g = np.empty(n, np.int32)
    count_g = np.empty(count_o.shape[0], np.int32)
    order_g = np.empty(n, np.int32)
    nk = ctypes.c_int64()
    s._set_stream()
    assert s._L.gf_bin_read(s._ctx, key_g.ctypes.data, count_g.ctypes.data,
                            order_g.ctypes.data, ctypes.byref(nk)) == 0
    assert nk.value == count_o.shape[0]
    assert_bitexact("keys", key_g, key_o)
    assert_bitexact("per-cell counts", count_g, count_o)
    # storage order is the identity here (fresh pid = arange), so the sorted
    # order of storage slots must equal the oracle's (key, pid) order
    assert_bitexact("sort order", order_g, order_o.astype(np.int32))


@pytest.mark.parametrize("tiles_k,lanes", [(1, 0), (2, 0), (1, 1), (2, 1), (1, 2), (2, 2),
                                           (1, 3), (2, 3), (1, 4), (2, 4), (1, 5), (2, 5)])
@pytest.mark.parametrize("transfer", ["flip", "apic"])
@pytest.mark.parametrize("grid", GRIDS[:2] + [(17, 12, 40)])
def test_p2g_matches_oracle(gf, oracle, grid, transfer, tiles_k, lanes):
    """P2G with blocks of 8^3 or 8 x 8 x 16 cells per CTA and each lane
    mapping, per-cell register sums included (the autotuner's choices; 40
    cells along k give an odd tile count, so the last block holds one tile)."""
    import torch
    nx, ny, nz = grid
    s = _mk(gf, grid, transfer=transfer)
    s.set_tune(p2g_tiles_k=tiles_k, p2g_map=lanes)
    pos, vel, C = random_particles(nx, ny, nz, s.dx, 30000, seed=7)
    s._set_particles(pos=pos, vel=vel, C=C)
    _call(s, "gf_bin", 2 if transfer == "apic" else 0)
    _call(s, "gf_p2g", 2 if transfer == "apic" else 0)
    torch.cuda.synchronize()
    o = _oracle(oracle, s)
    o.set_particles(pos, vel, C)
    o.clear(); o.p2g()
    assert_bitexact("labels", s.marker.numpy(), o.marker)
    for k in ("u", "v", "w"):
        g = getattr(s, "_" + k).cpu().numpy()
        assert rel_l2(g, getattr(o, k)) < 2e-6, (k, rel_l2(g, getattr(o, k)))
    for k in ("uw", "vw", "ww"):
        g = getattr(s, k).cpu().numpy()
        assert rel_l2(g, getattr(o, k)) < 2e-6, (k, rel_l2(g, getattr(o, k)))
        # zero pattern is exact: a face has weight iff some particle reaches it
        assert np.array_equal(g == 0, getattr(o, k) == 0), k


def _load_p2g_state(s, o):
    """Copy the oracle's P2G output and labels into the solver's buffers."""
    import torch
    for k in ("u", "v", "w"):
        getattr(s, "_" + k).copy_(_t(getattr(o, k)))
    for k in ("uw", "vw", "ww"):
        getattr(s, k).copy_(_t(getattr(o, k)))
    s._label.copy_(_t(o.marker.astype(np.uint8)))


@pytest.mark.parametrize("grid", GRIDS)
def test_forces_div_bitexact(gf, oracle, grid):
    import torch
    nx, ny, nz = grid
    s = _mk(gf, grid, sphere=((0.6, 0.3, 0.4), 0.15))
    o = _oracle(oracle, s)
    pos, vel, _ = random_particles(nx, ny, nz, s.dx, 15000, seed=3)
    o.set_particles(pos, vel)
    o.clear(); o.p2g()
    _load_p2g_state(s, o)
    dt = 1.0 / 240.0
    _call(s, "gf_forces_div", ctypes.c_float(s.gravity), ctypes.c_float(dt), ctypes.c_float(s.rho))
    torch.cuda.synchronize()
    o.normalize(); o.gravity_bc(dt); o.divergence(dt)
    for k in ("u", "v", "w"):
        assert_bitexact(k, getattr(s, "_" + k).cpu().numpy(), getattr(o, k))
    for k in ("us", "vs", "ws"):
        assert_bitexact(k, getattr(s, k).cpu().numpy(), getattr(o, k))
    assert_bitexact("div", s.div.cpu().numpy(), o.div)


def _pressure_case(gf, oracle, grid, seed=5):
    nx, ny, nz = grid
    s = _mk(gf, grid, sphere=((0.55, 0.35, 0.45), 0.17))
    o = _oracle(oracle, s)
    pos, vel, _ = random_particles(nx, ny, nz, s.dx, 8 * nx * ny * nz // 3, seed=seed)
    pos[:, 1] *= 0.6  # fluid in the lower part: air cells above give a free surface
    o.set_particles(pos, vel)
    o.clear(); o.p2g(); o.normalize(); o.gravity_bc(1 / 240.0); o.divergence(1 / 240.0)
    s._label.copy_(_t(o.marker.astype(np.uint8)))
    s.div.copy_(_t(o.div))
    return s, o


def _params(gf, solver, iters, tol=1e-4, rhs_sign=-1, check_every=10, flags=0):
    from gpufluid_b200 import _lib
    return _lib.StepParams(1 / 240.0, -9.81, 1.0, 0.95, 0, _lib.SOLVER[solver], iters,
                           check_every, tol, rhs_sign, flags)


def _stats(s):
    from gpufluid_b200 import _lib
    info = _lib.PressureInfo()
    s._set_stream()
    assert s._L.gf_pressure_stats(s._ctx, ctypes.byref(info)) == 0
    return info


@pytest.mark.parametrize("solver,iters", [("jacobi", 1), ("jacobi", 37), ("gsrb", 1), ("gsrb", 25)])
@pytest.mark.parametrize("grid", GRIDS)
def test_jacobi_gsrb_bitexact(gf, oracle, grid, solver, iters):
    import torch
    s, o = _pressure_case(gf, oracle, grid)
    prm = _params(gf, solver, iters)
    it = ctypes.c_int32()
    _call(s, "gf_pressure", ctypes.byref(prm), ctypes.byref(it))
    torch.cuda.synchronize()
    o.pressure(solver, iters)
    assert it.value == iters
    assert_bitexact(f"p ({solver} x{iters})", s._p.cpu().numpy(), o.p)


@pytest.mark.parametrize("rhs_sign", [-1, +1])
@pytest.mark.parametrize("grid", [(24, 24, 24), (32, 20, 16)])
def test_pcg_matches_oracle_and_fp64(gf, oracle, grid, rhs_sign):
    import torch
    s, o = _pressure_case(gf, oracle, grid)
    tol = 1e-5
    prm = _params(gf, "pcg", 400, tol=tol, rhs_sign=rhs_sign)
    it = ctypes.c_int32()
    _call(s, "gf_pressure", ctypes.byref(prm), ctypes.byref(it))
    torch.cuda.synchronize()
    p_gpu = s._p.cpu().numpy()
    o.pressure("pcg", 400, tol=tol, rhs_sign=rhs_sign)
    # same algorithm, same stop test (every 10 iterations): counts agree to one check
    assert abs(it.value - o.last_pressure_iters) <= 10, (it.value, o.last_pressure_iters)
    p64, _, _ = oracle.pcg64(o.marker, o.div, tol=1e-13, rhs_sign=rhs_sign)
    e_gpu, e_cpu = rel_l2(p_gpu, p64), rel_l2(o.p, p64)
    assert e_gpu < 1e-3, e_gpu
    assert e_gpu < 5 * e_cpu + 1e-6, (e_gpu, e_cpu)
    assert rel_l2(p_gpu, o.p) < 1e-3


@pytest.mark.parametrize("grid", [(24, 24, 24), (40, 32, 24)])
def test_pcg_refined_reaches_fp64_accuracy(gf, oracle, grid):
    import torch
    s, o = _pressure_case(gf, oracle, grid, seed=11)
    prm = _params(gf, "pcg_refined", 2000, tol=1e-10)
    it = ctypes.c_int32()
    rel = ctypes.c_double()
    st = ctypes.c_int32()
    _call(s, "gf_pressure", ctypes.byref(prm), ctypes.byref(it))
    s._L.gf_pressure_result(s._ctx, ctypes.byref(it), ctypes.byref(rel), ctypes.byref(st))
    torch.cuda.synchronize()
    assert st.value == 0, st.value
    assert rel.value <= 1e-10, rel.value
    p64, _, _ = oracle.pcg64(o.marker, o.div, tol=1e-14)
    # the returned pressure is the FP64 iterate rounded to float32
    assert rel_l2(s._p.cpu().numpy(), p64) < 1e-6, rel_l2(s._p.cpu().numpy(), p64)


@pytest.mark.parametrize("grid", GRIDS)
def test_project_bitexact(gf, oracle, grid):
    import torch
    s, o = _pressure_case(gf, oracle, grid)
    o.pressure("jacobi", 30)
    for k in ("u", "v", "w"):
        getattr(s, "_" + k).copy_(_t(getattr(o, k)))
    s._p.copy_(_t(o.p))
    dt = 1.0 / 240.0
    _call(s, "gf_project", ctypes.c_float(dt), ctypes.c_float(s.rho))
    torch.cuda.synchronize()
    o.grad_bc(dt)
    for k in ("u", "v", "w"):
        assert_bitexact(k, getattr(s, "_" + k).cpu().numpy(), getattr(o, k))


@pytest.mark.parametrize("tiles_k", [0, 1, 2])
@pytest.mark.parametrize("transfer,blend", [("flip", 0.95), ("pic", 0.0), ("apic", 0.95)])
@pytest.mark.parametrize("grid", GRIDS + [(24, 16, 40), (32, 32, 32)])
def test_g2p_bitexact(gf, oracle, grid, transfer, blend, tiles_k):
    """G2P (the tile-staged kernel: TMA boxes where the strides allow, e.g.
    u and v at 24x16x40 and all six arrays but w, ws at 32^3, plain loads
    otherwise) with blocks of 8^3 or 8 x 8 x 16 cells, and the unstaged
    per-particle kernel (tile shape 0)."""
    import torch
    nx, ny, nz = grid
    s = _mk(gf, grid, transfer=transfer)
    s.set_tune(g2p_tiles_k=tiles_k)
    s.flip_blend = blend
    rng = np.random.default_rng(nx * 31 + ny)
    o = _oracle(oracle, s)
    for k in ("u", "v", "w", "us", "vs", "ws"):
        a = getattr(o, k)
        a[...] = rng.normal(0, 1, a.shape).astype(np.float32)
    pos, vel, C = random_particles(nx, ny, nz, s.dx, 20000, seed=nx + 1)
    s._set_particles(pos=pos, vel=vel, C=C)
    for k in ("u", "v", "w"):
        getattr(s, "_" + k).copy_(_t(getattr(o, k)))
    for k in ("us", "vs", "ws"):
        getattr(s, k).copy_(_t(getattr(o, k)))
    o.flip_blend = blend
    o.set_particles(pos, vel, C)
    code = {"flip": 0, "pic": 1, "apic": 2}[transfer]
    dt = 1.0 / 240.0
    _call(s, "gf_bin", code)
    _call(s, "gf_g2p", code, ctypes.c_float(blend), ctypes.c_float(dt))
    torch.cuda.synchronize()
    o.g2p(dt)
    assert_bitexact("pos", s.pos.numpy(), o.pos)
    assert_bitexact("vel", s.vel.numpy(), o.vel)
    if transfer == "apic":
        assert_bitexact("C", s.affine_C.numpy(), o.C)


@pytest.mark.parametrize("solver,tol", [("pcg", 1e-5), ("pcg_refined", 1e-10)])
@pytest.mark.parametrize("grid", [(24, 24, 24), (48, 40, 56)])
def test_pcg_shared_memory_matches_global_kernel(gf, oracle, grid, solver, tol):
    """The shared-memory-resident solver and the global-memory solver run the
    same recurrences; only the block partition of the dot products differs."""
    import torch
    from gpufluid_b200 import _lib
    res = {}
    for flags in (0, _lib.GF_FLAG_GLOBAL_PCG):
        s, o = _pressure_case(gf, oracle, grid, seed=21)
        prm = _params(gf, solver, 3000, tol=tol, flags=flags)
        it = ctypes.c_int32()
        _call(s, "gf_pressure", ctypes.byref(prm), ctypes.byref(it))
        torch.cuda.synchronize()
        info = _stats(s)
        assert info.kernel == (2 if flags else 1)
        assert info.status == 0
        res[flags] = (s._p.cpu().numpy(), info.iters)
    p_s, it_s = res[0]
    p_g, it_g = res[_lib.GF_FLAG_GLOBAL_PCG]
    assert abs(it_s - it_g) <= (10 if solver == "pcg" else 3), (it_s, it_g)
    assert rel_l2(p_s, p_g) < (1e-4 if solver == "pcg" else 1e-6)


def test_pcg_large_region_falls_back_to_global_kernel(gf, oracle):
    """More active tiles than the shared-memory solver holds (148 SMs x 20
    tiles): the global-memory kernel takes over and still meets the target."""
    import torch
    nx, ny, nz = 192, 64, 192
    s = gf.FlipSolver3D(nx, ny, nz)
    lab = s._marker_host.copy()
    lab[1:-1, 1:48, 1:-1] = 1  # fluid below y = 48, air above
    rng = np.random.default_rng(5)
    div = np.where(lab == 1, rng.normal(0, 1, lab.shape), 0).astype(np.float32)
    s._label.copy_(_t(lab.astype(np.uint8)))
    s.div.copy_(_t(div))
    prm = _params(gf, "pcg_refined", 4000, tol=1e-9)
    it = ctypes.c_int32()
    _call(s, "gf_pressure", ctypes.byref(prm), ctypes.byref(it))
    torch.cuda.synchronize()
    info = _stats(s)
    assert info.n_active_tiles == 24 * 6 * 24
    assert info.kernel == 2 and info.status == 0
    assert info.relres <= 1e-9


@pytest.mark.parametrize("sweeps", [1, 2, 3])
@pytest.mark.parametrize("grid", [(24, 24, 24), (48, 40, 56), (80, 80, 80)])
def test_pcg_tile_sgs_preconditioner(gf, oracle, grid, sweeps):
    """Tile-local symmetric Gauss-Seidel preconditioner (flags bits 2-3): the
    refined solve reaches the FP64 solution of the same system as the Jacobi-
    preconditioned one, in fewer iterations.  At 80^3 fluid fills y < 64 (air
    above, so the system is nonsingular): 800 tiles, several per block, so
    in-block and remote ring exchanges both run."""
    import torch
    from gpufluid_b200 import _lib
    res = {}
    for flags in (0, sweeps << _lib.GF_FLAG_SGS_SHIFT):
        s, o = _pressure_case(gf, oracle, grid, seed=23)
        if grid == (80, 80, 80):
            lab = s._marker_host.copy()
            lab[1:-1, 1:64, 1:-1] = 1
            rng = np.random.default_rng(3)
            div = np.where(lab == 1, rng.normal(0, 1, lab.shape), 0).astype(np.float32)
            s._label.copy_(_t(lab.astype(np.uint8)))
            s.div.copy_(_t(div))
            o.marker[...] = lab
            o.div[...] = div
        prm = _params(gf, "pcg_refined", 4000, tol=1e-10, flags=flags)
        it = ctypes.c_int32()
        _call(s, "gf_pressure", ctypes.byref(prm), ctypes.byref(it))
        torch.cuda.synchronize()
        info = _stats(s)
        assert info.kernel == 1 and info.status == 0, (flags, info.kernel, info.status)
        assert info.relres <= 1e-10, (flags, info.relres)
        if not res:  # the same system for both preconditioners
            p64, _, _ = oracle.pcg64(o.marker, o.div, tol=1e-14)
        assert rel_l2(s._p.cpu().numpy(), p64) < 1e-6
        res[flags] = info.iters
    assert res[sweeps << _lib.GF_FLAG_SGS_SHIFT] < res[0], res


@pytest.mark.parametrize("refined", [True, False])
@pytest.mark.parametrize("sgs", [0, 2])
@pytest.mark.parametrize("grid", [(24, 24, 24), (48, 40, 56), (80, 80, 80), (128, 128, 128)])
def test_pcg_coarse_correction(gf, oracle, grid, sgs, refined):
    """Tile coarse correction (GF_FLAG_COARSE, one region per active tile):
    the solve reaches the FP64 solution of the same system as without it, in
    fewer iterations (from 80^3; at 128^3 with the SGS preconditioner under
    0.6 of them, where an FP64 study of the bench system gives 66 against
    210).  The 128^3 dam break is the bench's system at the start."""
    import torch
    from gpufluid_b200 import _lib
    res = {}
    base = sgs << _lib.GF_FLAG_SGS_SHIFT
    for flags in (base, base | _lib.GF_FLAG_COARSE):
        s, o = _pressure_case(gf, oracle, grid, seed=29)
        if grid[0] >= 80:
            lab = s._marker_host.copy()
            n = grid[0]
            if n == 128:
                lab[1:52, 1:77, 1:-1] = 1  # dam break: x < 0.4, y < 0.6
            else:
                lab[1:-1, 1:64, 1:-1] = 1
            rng = np.random.default_rng(3)
            div = np.where(lab == 1, rng.normal(0, 1, lab.shape), 0).astype(np.float32)
            s._label.copy_(_t(lab.astype(np.uint8)))
            s.div.copy_(_t(div))
            o.marker[...] = lab
            o.div[...] = div
        prm = _params(gf, "pcg_refined" if refined else "pcg", 4000,
                      tol=1e-10 if refined else 1e-6, flags=flags)
        it = ctypes.c_int32()
        _call(s, "gf_pressure", ctypes.byref(prm), ctypes.byref(it))
        torch.cuda.synchronize()
        info = _stats(s)
        assert info.kernel == 1 and info.status == 0, (flags, info.kernel, info.status)
        assert info.coarse == (1 if flags & _lib.GF_FLAG_COARSE else 0)
        if not res:  # the same system for both
            p64, _, _ = oracle.pcg64(o.marker, o.div, tol=1e-14)
        if refined:
            assert info.relres <= 1e-10, (flags, info.relres)
            assert rel_l2(s._p.cpu().numpy(), p64) < 1e-6
        else:
            assert info.relres <= 1e-6, (flags, info.relres)
            assert rel_l2(s._p.cpu().numpy(), p64) < 1e-4
        res[flags] = info.iters
    if grid[0] >= 80:
        assert res[base | _lib.GF_FLAG_COARSE] < res[base], res
    if grid[0] == 128 and sgs:
        assert res[base | _lib.GF_FLAG_COARSE] < 0.6 * res[base], res


@pytest.mark.parametrize("refined", [True, False])
@pytest.mark.parametrize("grid", [(48, 40, 56), (80, 80, 80)])
def test_global_pcg_tile_sgs_preconditioner(gf, oracle, grid, refined):
    """The global-memory PCG (the solver for active regions beyond the
    shared-memory one) with the tile-local symmetric Gauss-Seidel
    preconditioner: same system, same FP64 answer, fewer iterations than with
    the reference's Jacobi preconditioner; 1 and 2 sweeps."""
    import torch
    from gpufluid_b200 import _lib
    res = {}
    for sweeps in (0, 1, 2):
        flags = _lib.GF_FLAG_GLOBAL_PCG | (sweeps << _lib.GF_FLAG_SGS_SHIFT)
        s, o = _pressure_case(gf, oracle, grid, seed=31)
        if grid == (80, 80, 80):
            lab = s._marker_host.copy()
            lab[1:-1, 1:64, 1:-1] = 1
            rng = np.random.default_rng(3)
            div = np.where(lab == 1, rng.normal(0, 1, lab.shape), 0).astype(np.float32)
            s._label.copy_(_t(lab.astype(np.uint8)))
            s.div.copy_(_t(div))
            o.marker[...] = lab
            o.div[...] = div
        prm = _params(gf, "pcg_refined" if refined else "pcg", 6000,
                      tol=1e-10 if refined else 1e-6, flags=flags)
        it = ctypes.c_int32()
        _call(s, "gf_pressure", ctypes.byref(prm), ctypes.byref(it))
        torch.cuda.synchronize()
        info = _stats(s)
        assert info.kernel == 2 and info.status == 0, (sweeps, info.kernel, info.status)
        if not res:
            p64, _, _ = oracle.pcg64(o.marker, o.div, tol=1e-14)
        if refined:
            assert info.relres <= 1e-10, (sweeps, info.relres)
            assert rel_l2(s._p.cpu().numpy(), p64) < 1e-6
        else:
            assert info.relres <= 1e-6, (sweeps, info.relres)
            assert rel_l2(s._p.cpu().numpy(), p64) < 1e-4
        res[sweeps] = info.iters
    assert res[2] < res[1] < res[0], res


@pytest.mark.parametrize("refined", [True, False])
@pytest.mark.parametrize("grid", [(48, 40, 56), (80, 80, 80), (128, 128, 128)])
def test_global_pcg_coarse_correction(gf, oracle, grid, refined):
    """Coarse correction of the global-memory PCG (GF_FLAG_COARSE with the
    tile SGS preconditioner; one region per cube of tiles, here one tile per
    cube): the same FP64 answer as the tile SGS alone, in fewer iterations
    from 80^3; the 128^3 system is the dam break of the shared-memory test."""
    import torch
    from gpufluid_b200 import _lib
    res = {}
    base = _lib.GF_FLAG_GLOBAL_PCG | (2 << _lib.GF_FLAG_SGS_SHIFT)
    for flags in (base, base | _lib.GF_FLAG_COARSE):
        s, o = _pressure_case(gf, oracle, grid, seed=37)
        if grid[0] >= 80:
            lab = s._marker_host.copy()
            if grid[0] == 128:
                lab[1:52, 1:77, 1:-1] = 1
            else:
                lab[1:-1, 1:64, 1:-1] = 1
            rng = np.random.default_rng(5)
            div = np.where(lab == 1, rng.normal(0, 1, lab.shape), 0).astype(np.float32)
            s._label.copy_(_t(lab.astype(np.uint8)))
            s.div.copy_(_t(div))
            o.marker[...] = lab
            o.div[...] = div
        prm = _params(gf, "pcg_refined" if refined else "pcg", 6000,
                      tol=1e-10 if refined else 1e-6, flags=flags)
        it = ctypes.c_int32()
        _call(s, "gf_pressure", ctypes.byref(prm), ctypes.byref(it))
        torch.cuda.synchronize()
        info = _stats(s)
        assert info.kernel == 2 and info.status == 0, (flags, info.kernel, info.status)
        assert info.coarse == (1 if flags & _lib.GF_FLAG_COARSE else 0), flags
        if not res:
            p64, _, _ = oracle.pcg64(o.marker, o.div, tol=1e-14)
        if refined:
            assert info.relres <= 1e-10, (flags, info.relres)
            assert rel_l2(s._p.cpu().numpy(), p64) < 1e-6
        else:
            assert info.relres <= 1e-6, (flags, info.relres)
            assert rel_l2(s._p.cpu().numpy(), p64) < 1e-4
        res[flags] = info.iters
    if grid[0] >= 80:
        assert res[base | _lib.GF_FLAG_COARSE] < res[base], res


@pytest.mark.parametrize("kernel_flags", ["global_sgs2", "global_jacobi", "smem"])
def test_refined_pcg_warm_start_both_kernels(gf, oracle, kernel_flags):
    """GF_FLAG_WARM_START on the refined PCG: after a solve, a nearby system
    (the divergence perturbed by 2%) solved from the previous pressure meets
    the same FP64 stop test relative to ||b||, gives the FP64 answer, and
    takes fewer iterations than the cold start of the same system."""
    import torch
    from gpufluid_b200 import _lib
    base = {"global_sgs2": _lib.GF_FLAG_GLOBAL_PCG | (2 << _lib.GF_FLAG_SGS_SHIFT),
            "global_jacobi": _lib.GF_FLAG_GLOBAL_PCG, "smem": 0}[kernel_flags]
    kernel = 1 if kernel_flags == "smem" else 2
    s, o = _pressure_case(gf, oracle, (48, 40, 56), seed=17)
    it = ctypes.c_int32()
    _call(s, "gf_pressure", ctypes.byref(_params(gf, "pcg_refined", 6000, tol=1e-10, flags=base)),
          ctypes.byref(it))
    rng = np.random.default_rng(4)
    div2 = np.where(o.marker == 1, o.div * (1 + 0.02 * rng.normal(0, 1, o.div.shape)), 0)
    div2 = div2.astype(np.float32)
    o.div[...] = div2
    p64, _, _ = oracle.pcg64(o.marker, o.div, tol=1e-14)
    iters = {}
    for warm in (True, False):  # the warm solve first: fields.p holds the last answer
        s.div.copy_(_t(div2))
        flags = base | (_lib.GF_FLAG_WARM_START if warm else 0)
        _call(s, "gf_pressure", ctypes.byref(_params(gf, "pcg_refined", 6000, tol=1e-10,
                                                     flags=flags)), ctypes.byref(it))
        torch.cuda.synchronize()
        info = _stats(s)
        assert info.kernel == kernel and info.status == 0, (warm, info.kernel, info.status)
        assert info.relres <= 1e-10, (warm, info.relres)
        assert rel_l2(s._p.cpu().numpy(), p64) < 1e-6
        iters[warm] = info.iters
    assert iters[True] < iters[False], iters
