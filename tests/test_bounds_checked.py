"""The bounds-checked build (libgfb200_checked.so, -DGF_BOUNDS_CHECK).

Every instrumented index (cell, tile key, sort slot, face, neighbour, box
position) is checked before it addresses memory; an index out of range is
skipped and counted.  The reference indexes unchecked
(src/gpufluid/solvers/solver3d.py:100-101); this build is the safety net that
needs no closed tool.  The GPU test steps the workloads' features through the
checked library in a child process (the library variant is chosen when the
package loads) and requires zero violations; it plants no bad index.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import json, numpy as np, torch
import gpufluid_b200 as gf
from gpufluid_b200 import _lib, scene
import ctypes
L = _lib.load()
out = {"lib": _lib.LIB_PATH}
# a dam break in every transfer mode, every solver, both PCG kernels, SGS,
# the coarse correction, the sphere obstacle, particles outside the grid
for transfer, solver, flags in (("flip", "jacobi", {}), ("pic", "gsrb", {}),
                                ("apic", "pcg_refined", dict(pcg_preconditioner="tile_sgs",
                                                             pcg_coarse=True)),
                                ("flip", "pcg", {})):
    s = gf.FlipSolver3D(40, 36, 44, transfer_mode=transfer, pressure_tol=1e-6, **flags)
    s.add_solid_from_sdf(scene.sdf_sphere(s.cell_centers_np(), (0.6, 0.3, 0.5), 0.12))
    s.seed_box((0.0, 0.0, 0.0), (0.45, 0.6, 0.9))
    pos = s.pos.numpy()
    pos[:50] += np.float32(0.7)  # some outside the grid: clamped cells, global paths
    s.pos = pos
    for _ in range(4):
        s.step(1 / 240, pressure_iters=300, pressure_solver=solver)
    out[f"{transfer}_{solver}_finite"] = bool(np.isfinite(s.pos.numpy()).all())
# the global-memory PCG with the tile preconditioner
s = gf.FlipSolver3D(48, 40, 56)
s.seed_box((0.0, 0.0, 0.0), (0.5, 0.6, 1.0))
s.pcg_preconditioner = "tile_sgs"
prm = s._params(1 / 240, 2000, "pcg_refined")
prm.flags |= _lib.GF_FLAG_GLOBAL_PCG
for _ in range(2):
    s._set_stream()
    _lib.check(L.gf_step(s._ctx, ctypes.byref(prm)), s._ctx, "gf_step")
out["global_pcg"] = s.pressure_stats()["kernel"]
torch.cuda.synchronize()
v, line, chk = ctypes.c_int64(), ctypes.c_int32(), ctypes.c_int32()
assert L.gf_bounds_status(0, ctypes.byref(v), ctypes.byref(line), ctypes.byref(chk)) == 0
out.update(violations=int(v.value), first_line=int(line.value), checked=int(chk.value))
print(json.dumps(out))
'''


def test_checked_library_built_and_exports():
    from gpufluid_b200 import _lib
    path = os.path.join(ROOT, "gpufluid_b200", "libgfb200_checked.so")
    assert os.path.exists(path), "build it with python -m gpufluid_b200.build --bounds-check"
    import ctypes
    lib = ctypes.CDLL(path)
    missing = [s for s in _lib.header_symbols() if not hasattr(lib, s)]
    assert not missing, missing


@pytest.mark.gpu
def test_checked_library_runs_the_workloads_without_violations():
    env = dict(os.environ, GFB200_LIB="libgfb200_checked.so", PYTHONPATH=ROOT)
    r = subprocess.run([sys.executable, "-c", CHILD], capture_output=True, text=True, env=env,
                       cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["lib"].endswith("libgfb200_checked.so")
    assert res["checked"] == 1
    assert res["global_pcg"] == 2
    assert all(v for k, v in res.items() if k.endswith("_finite")), res
    assert res["violations"] == 0, res
