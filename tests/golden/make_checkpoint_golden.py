"""Generate the cross-implementation checkpoint fixtures.

Test-fixture generator (run by hand, in a container that holds the reference
checkout; nothing at test or bench time reads the reference):

    python tests/golden/make_checkpoint_golden.py --reference <path of the GPUFLUID checkout>

It installs the sequential Warp stand-in (``warp_shim.py``) and imports the
reference's ``gpufluid.solvers.solver3d`` unmodified, then writes into
``tests/golden/checkpoint/``:

* ``reference_apic16.npz`` -- a checkpoint written by the reference's own
  ``FlipSolver3D.save_checkpoint`` (solver3d.py:4127-4157) after two APIC
  substeps of a 16^3 dam break with a sphere obstacle;
* ``reference_resume.npz`` -- the reference's state after loading that file
  into a fresh solver with its own ``load_checkpoint`` (:4159-4222) and
  stepping once more (Jacobi, 30 sweeps): the state this repo's solver must
  reach from the same file;
* ``repo_written.npz`` -- a checkpoint written by this repo's
  ``write_checkpoint`` (the writer behind ``FlipSolver3D.save_checkpoint``)
  from seeded arrays, and ``repo_loaded_by_reference.npz`` -- the arrays the
  reference's ``load_checkpoint`` read back from it (its topology and dx
  checks passed, or this script stops).
"""
from __future__ import annotations

import argparse
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "checkpoint")
ROOT = os.path.dirname(os.path.dirname(HERE))

GRID = (16, 16, 16)
DT = 1.0 / 480.0


def _reference(ref_src):
    sys.path.insert(0, HERE)
    import warp_shim  # noqa: E402
    wp = warp_shim.install()
    if "gpufluid" not in sys.modules:
        pkg = types.ModuleType("gpufluid")
        pkg.__path__ = [os.path.join(ref_src, "gpufluid")]
        sys.modules["gpufluid"] = pkg
    from gpufluid.solvers.solver3d import FlipSolver3D  # noqa: E402
    from gpufluid.primitives.sdf import sdf_sphere  # noqa: E402
    return wp, FlipSolver3D, sdf_sphere


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("GPUFLUID_REFERENCE"),
                    required="GPUFLUID_REFERENCE" not in os.environ,
                    help="GPUFLUID source checkout (or set GPUFLUID_REFERENCE)")
    a = ap.parse_args()
    wp, FlipSolver3D, sdf_sphere = _reference(os.path.join(a.reference, "src"))
    os.makedirs(OUT, exist_ok=True)

    # 1. the reference writes a checkpoint mid-simulation
    s = FlipSolver3D(*GRID, transfer_mode="apic", device="cpu")
    s.add_solid_from_sdf(sdf_sphere(s.cell_centers_np(), (0.7, 0.2, 0.5), 0.2))
    s.seed_box((0.0, 0.0, 0.0), (0.4, 0.6, 1.0), ppc=8)
    for _ in range(2):
        s.step(DT, pressure_iters=30, pressure_solver="jacobi")
    path = os.path.join(OUT, "reference_apic16.npz")
    s.save_checkpoint(path)

    # 2. the reference resumes from it and steps once more
    r = FlipSolver3D(*GRID, transfer_mode="apic", device="cpu")
    r.load_checkpoint(path)
    r.step(DT, pressure_iters=30, pressure_solver="jacobi")
    np.savez_compressed(os.path.join(OUT, "reference_resume.npz"), pos=r.pos.numpy(),
                        vel=r.vel.numpy(), affine_C=r.affine_C.numpy(), marker=r.marker.numpy(),
                        dt=np.float32(DT), iters=np.int32(30))

    # 3. this repo writes a checkpoint; the reference loads it
    sys.path.insert(0, ROOT)
    from gpufluid_b200.solver import write_checkpoint  # noqa: E402
    rng = np.random.default_rng(11)
    n = 500
    pos = (0.1 + 0.5 * rng.random((n, 3))).astype(np.float32)
    vel = rng.normal(0, 0.5, (n, 3)).astype(np.float32)
    aff = rng.normal(0, 1.0, (n, 3, 3)).astype(np.float32)
    marker = np.zeros(GRID, np.int32)
    marker[[0, -1]] = 2
    marker[:, [0, -1]] = 2
    marker[:, :, [0, -1]] = 2
    mine = os.path.join(OUT, "repo_written.npz")
    write_checkpoint(mine, pos, vel, aff, marker,
                     dict(nx=GRID[0], ny=GRID[1], nz=GRID[2], dx=1.0 / 16, gravity=-9.81,
                          flip_blend=0.95, rho=1.0, viscosity=0.0, transfer_mode="apic",
                          surface_tension=0.0))
    q = FlipSolver3D(*GRID, transfer_mode="apic", device="cpu")
    q.load_checkpoint(mine)
    got = dict(pos=q.pos.numpy(), vel=q.vel.numpy(), affine_C=q.affine_C.numpy(),
               marker=q.marker.numpy())
    for k, v in (("pos", pos), ("vel", vel), ("affine_C", aff), ("marker", marker)):
        assert np.array_equal(got[k], v), k
    np.savez_compressed(os.path.join(OUT, "repo_loaded_by_reference.npz"), **got)
    print(f"wrote {OUT}: reference checkpoint P={s.n_particles}, repo checkpoint P={n}")


if __name__ == "__main__":
    main()
