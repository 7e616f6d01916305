"""Pin the CPU oracle to the reference's own outputs.

tests/golden/*.npz were produced by tests/golden/make_golden.py, which runs the
reference's FlipSolver3D source (src/gpufluid/solvers/solver3d.py) under a
sequential Warp stand-in.  Run sequentially, the oracle must reproduce every
stage of the first substep and the final state after the last one BIT FOR BIT.
"""
import glob
import os

import numpy as np
import pytest

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def _scene(path):
    d = np.load(path)
    return {k: d[k] for k in d.files}


@pytest.fixture(params=GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def golden(request):
    return _scene(request.param)


def _exact(name, got, want):
    got, want = np.asarray(got), np.asarray(want)
    assert got.shape == want.shape, (name, got.shape, want.shape)
    bad = np.flatnonzero(got.view(np.uint32 if got.dtype == np.float32 else got.dtype).ravel()
                         != want.view(np.uint32 if want.dtype == np.float32 else want.dtype).ravel())
    assert bad.size == 0, (f"{name}: {bad.size} of {got.size} differ; first at {bad[:5]}: "
                           f"got {got.ravel()[bad[:5]]} want {want.ravel()[bad[:5]]}")


def _scene_cfg(path):
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "make_golden", os.path.join(os.path.dirname(__file__), "golden", "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.SCENES[os.path.basename(path)[:-4]]


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_seed_and_walls_match_reference(oracle, path):
    """seed_box, the wall shell and the sphere SDF marking, bit for bit."""
    g, cfg = _scene(path), _scene_cfg(path)
    nx, ny, nz = cfg["grid"]
    dx = 1.0 / max(nx, ny, nz)
    pos = oracle.seed_box(dx, *cfg["box"], ppc=8)
    _exact("seed_box", pos, g["init_pos"])
    m = oracle.wall_marker(nx, ny, nz)
    if cfg["sphere"] is not None:
        m[oracle.sphere_sdf(nx, ny, nz, dx, *cfg["sphere"]) <= 0.0] = 2
    _exact("init_marker", m, g["init_marker"])


def _make(oracle, g):
    nx, ny, nz = (int(x) for x in g["grid"])
    o = oracle.OracleFlip(nx, ny, nz, flip_blend=float(g["flip_blend"]),
                          transfer_mode=str(g["transfer"]))
    assert np.float32(o.dx) == g["dx"]
    o.marker[...] = g["init_marker"]
    o.set_particles(g["init_pos"], g["init_vel"])
    return o


def test_first_substep_stages_bit_exact(oracle, golden):
    g = golden
    o = _make(oracle, g)
    dt = float(g["dt"])
    o.clear(); o.p2g()
    for k in ("u", "v", "w", "uw", "vw", "ww"):
        _exact("p2g_" + k, getattr(o, k), g["p2g_" + k])
    _exact("p2g_marker", o.marker, g["p2g_marker"])
    o.normalize()
    for k in ("u", "v", "w"):
        _exact("norm_" + k, getattr(o, k), g["norm_" + k])
    for k in ("us", "vs", "ws"):
        _exact(k, getattr(o, k), g[k])
    o.gravity_bc(dt)
    for k in ("u", "v", "w"):
        _exact("forces_" + k, getattr(o, k), g["forces_" + k])
    o.divergence(dt)
    _exact("div", o.div, g["div"])
    solver = str(g["solver"])
    # the reference's PCG starts from r = +div (rhs_sign=+1)
    o.pressure(solver, int(g["iters"]), rhs_sign=+1)
    _exact("p", o.p, g["p"])
    assert o.last_pressure_iters == int(g["pressure_iters_first"])
    o.grad_bc(dt)
    o.g2p(dt)
    _exact("g2p_pos", o.pos, g["g2p_pos"])
    _exact("g2p_vel", o.vel, g["g2p_vel"])
    if str(g["transfer"]) == "apic":
        _exact("g2p_C", o.C, g["g2p_C"])


def test_multi_substep_bit_exact(oracle, golden):
    g = golden
    o = _make(oracle, g)
    for _ in range(int(g["substeps"])):
        o.step(float(g["dt"]), pressure_iters=int(g["iters"]),
               pressure_solver=str(g["solver"]), rhs_sign=+1)
    _exact("final_pos", o.pos, g["final_pos"])
    _exact("final_vel", o.vel, g["final_vel"])
    _exact("final_marker", o.marker, g["final_marker"])
    _exact("final_p", o.p, g["final_p"])
    for k in ("u", "v", "w"):
        _exact("final_" + k, getattr(o, k), g["final_" + k])
    if str(g["transfer"]) == "apic":
        _exact("final_C", o.C, g["final_C"])
