"""CPU-only checks: the C ABI library loads and exports every declared entry
point, and the host-side scene set-up matches the reference bit for bit."""
import ctypes
import glob
import os

import numpy as np
import pytest

from helpers import assert_bitexact

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def test_library_exports_every_header_symbol(gf):
    from gpufluid_b200 import _lib
    lib = _lib.load()
    syms = _lib.header_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_struct_layouts_match_header():
    from gpufluid_b200 import _lib
    assert ctypes.sizeof(_lib.GridDesc) == 28
    assert ctypes.sizeof(_lib.Fields) == 15 * 8
    assert ctypes.sizeof(_lib.Particles) == 40
    # float dt, g, rho, blend; int transfer, solver, iters, check; double tol; int sign, reserved
    assert ctypes.sizeof(_lib.StepParams) == 48
    assert _lib.StepParams.tol.offset == 32


def test_create_rejects_bad_arguments(gf):
    from gpufluid_b200 import _lib
    L = _lib.load()
    ctx = ctypes.c_void_p()
    bad = _lib.GridDesc(0, 8, 8, 0.125, (ctypes.c_float * 3)(0, 1, 1))
    assert L.gf_create(ctypes.byref(bad), 0, ctypes.byref(ctx)) == _lib.GF_INVALID_ARG
    assert L.gf_create(None, 0, ctypes.byref(ctx)) == _lib.GF_INVALID_ARG


def test_create_without_device_reports_no_device(gf):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from gpufluid_b200 import _lib
    L = _lib.load()
    ctx = ctypes.c_void_p()
    g = _lib.GridDesc(8, 8, 8, 0.125, (ctypes.c_float * 3)(1, 1, 1))
    assert L.gf_create(ctypes.byref(g), 0, ctypes.byref(ctx)) == _lib.GF_NO_DEVICE
    assert not ctx.value


def test_solver_refuses_to_run_without_cuda(gf):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(RuntimeError, match="CUDA"):
        gf.FlipSolver3D(8, 8, 8)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_scene_setup_matches_reference(path):
    """seed_box / wall shell / sphere marking of the product's host code
    against the reference's own output stored in the golden fixtures."""
    import importlib.util
    from gpufluid_b200 import scene
    spec = importlib.util.spec_from_file_location(
        "make_golden", os.path.join(os.path.dirname(__file__), "golden", "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    cfg = mod.SCENES[os.path.basename(path)[:-4]]
    g = np.load(path)
    nx, ny, nz = cfg["grid"]
    dx = 1.0 / max(nx, ny, nz)
    assert_bitexact("seed_box", scene.seed_box_positions(dx, *cfg["box"], ppc=8), g["init_pos"])
    m = scene.wall_labels(nx, ny, nz).astype(np.int32)
    if cfg["sphere"] is not None:
        m[scene.sdf_sphere(scene.cell_centers(nx, ny, nz, dx), *cfg["sphere"]) <= 0.0] = 2
    assert_bitexact("marker", m, g["init_marker"])


def test_seed_counts_match_reference_arithmetic():
    """Particle counts of the benchmark scenes from seed_box's arithmetic."""
    from gpufluid_b200 import scene
    assert scene.seed_box_positions(1 / 64, (0, 0, 0), (0.4, 0.6, 1.0)).shape[0] == 486400
    n128 = 25 * 0 + 51 * 76 * 128 * 8
    assert n128 == 3969024


def test_cfl_host_helper():
    from gpufluid_b200 import cfl_substep_count
    v = np.array([[3.0, 4.0, 0.0], [0.0, 0.0, 1.0]], np.float32)
    assert cfl_substep_count(v, 0.1, 0.1, cfl=0.5) == 10
    assert cfl_substep_count(np.zeros((0, 3)), 0.1, 0.1) == 1
    assert cfl_substep_count(v, 0.1, 10.0, cfl=0.5, max_substeps=16) == 16
