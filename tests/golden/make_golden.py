"""Generate golden vectors by running the reference's own solver source.

Test-fixture generator (run by hand, in a container that holds the reference
checkout; nothing at test or bench time reads the reference):

    python tests/golden/make_golden.py --reference <path of the GPUFLUID checkout> [--only NAME]

It installs the sequential Warp stand-in (``warp_shim.py``), imports
``gpufluid.solvers.solver3d`` from the reference checkout unmodified, builds
``FlipSolver3D`` scenes through its public API (``__init__``, ``seed_box``,
``add_solid_from_sdf``, ``step``) and records, for the first substep, the
output of every hot-path stage as the reference's ``_step_impl``
(``solver3d.py:3475-3667``) produces it, plus the state after the last substep.

Each scene is written to ``tests/golden/<name>.npz`` (float32 / int32 arrays,
C-order ``[i, j, k]`` exactly as the reference lays them out).
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# name: (grid, transfer, flip_blend, solver, iters, dt, substeps, box, sphere, init_vel_sigma)
SCENES = {
    # non-cubic grid, FLIP, Jacobi; seeded random initial velocities so the
    # FLIP blend and the advection clamp both see non-trivial values
    "flip_jacobi_16x12x10": dict(
        grid=(16, 12, 10), transfer="flip", flip_blend=0.95, solver="jacobi",
        iters=30, dt=1.0 / 240.0, substeps=3,
        box=((0.0, 0.0, 0.0), (0.4, 0.5, 0.6)), sphere=None, vel_sigma=0.5),
    # APIC + sphere obstacle + GS-RB (cfg2's features at 16^3)
    "apic_gsrb_sphere_16": dict(
        grid=(16, 16, 16), transfer="apic", flip_blend=0.95, solver="gsrb",
        iters=20, dt=1.0 / 480.0, substeps=3,
        box=((0.0, 0.0, 0.0), (0.4, 0.6, 1.0)),
        sphere=((0.7, 0.2, 0.5), 0.2), vel_sigma=0.0),
    # the reference's PCG (tol 1e-4, host-synchronised convergence checks)
    "flip_pcg_12x16x12": dict(
        grid=(12, 16, 12), transfer="flip", flip_blend=0.95, solver="pcg",
        iters=40, dt=1.0 / 240.0, substeps=2,
        box=((0.0, 0.0, 0.0), (0.5, 0.6, 0.7)), sphere=None, vel_sigma=0.3),
    # PIC (flip_blend 0) with Jacobi on a small cube
    "pic_jacobi_12": dict(
        grid=(12, 12, 12), transfer="pic", flip_blend=0.0, solver="jacobi",
        iters=20, dt=1.0 / 240.0, substeps=2,
        box=((0.1, 0.0, 0.2), (0.6, 0.5, 0.8)), sphere=((0.3, 0.7, 0.5), 0.15),
        vel_sigma=0.4),
}

# Stage snapshots taken on the first substep: kernel name -> list of
# (output key, argument index) recorded after that launch.  Argument indices
# follow each kernel's signature in solver3d.py.
_P2G = [("p2g_u", 2), ("p2g_v", 3), ("p2g_w", 4), ("p2g_uw", 5), ("p2g_vw", 6),
        ("p2g_ww", 7), ("p2g_marker", 8)]
_P2G_APIC = [("p2g_u", 3), ("p2g_v", 4), ("p2g_w", 5), ("p2g_uw", 6), ("p2g_vw", 7),
             ("p2g_ww", 8), ("p2g_marker", 9)]
_NORM = [("norm_u", 0), ("norm_v", 1), ("norm_w", 2), ("us", 6), ("vs", 7), ("ws", 8)]


def run_scene(name, cfg, ref_src):
    sys.path.insert(0, HERE)
    import warp_shim  # noqa: E402
    wp = warp_shim.install()
    # Register the package without executing its __init__ (which pulls in the
    # 2D solver, meshing and CLI modules that are not on this path).
    import types
    if "gpufluid" not in sys.modules:
        pkg = types.ModuleType("gpufluid")
        pkg.__path__ = [os.path.join(ref_src, "gpufluid")]
        sys.modules["gpufluid"] = pkg
    from gpufluid.solvers.solver3d import FlipSolver3D  # noqa: E402
    from gpufluid.primitives.sdf import sdf_sphere  # noqa: E402

    nx, ny, nz = cfg["grid"]
    s = FlipSolver3D(nx, ny, nz, flip_blend=cfg["flip_blend"],
                     transfer_mode=cfg["transfer"], device="cpu")
    if cfg["sphere"] is not None:
        c, r = cfg["sphere"]
        s.add_solid_from_sdf(sdf_sphere(s.cell_centers_np(), c, r))
    lo, hi = cfg["box"]
    s.seed_box(lo, hi, ppc=8)
    if cfg["vel_sigma"] > 0:
        rng = np.random.default_rng(1234)
        vel = rng.normal(0.0, cfg["vel_sigma"], size=(s.n_particles, 3)).astype(np.float32)
        s.vel = wp.array(vel, dtype=wp.vec3)
    out = {
        "grid": np.array([nx, ny, nz], np.int32),
        "dx": np.float32(s.dx),
        "flip_blend": np.float32(cfg["flip_blend"]),
        "transfer": np.array(cfg["transfer"]),
        "solver": np.array(cfg["solver"]),
        "iters": np.int32(cfg["iters"]),
        "dt": np.float32(cfg["dt"]),
        "substeps": np.int32(cfg["substeps"]),
        "gravity": np.float32(s.gravity),
        "rho": np.float32(s.rho),
        "init_pos": s.pos.numpy(),
        "init_vel": s.vel.numpy(),
        "init_marker": s.marker.numpy(),
    }

    state = {"n_bc": 0, "first": True}
    p2g_map = _P2G_APIC if cfg["transfer"] == "apic" else _P2G

    def hook(kname, args):
        if not state["first"]:
            return
        snap = lambda key, idx: out.__setitem__(key, np.array(args[idx]))  # noqa: E731
        if kname in ("k3_p2g", "k3_p2g_apic"):
            for key, idx in p2g_map:
                snap(key, idx)
        elif kname == "k3_normalize":
            for key, idx in _NORM:
                snap(key, idx)
        elif kname == "k3_enforce_solid_bc":
            tag = "forces" if state["n_bc"] == 0 else "final"
            state["n_bc"] += 1
            for key, idx in ((f"{tag}_u", 0), (f"{tag}_v", 1), (f"{tag}_w", 2)):
                snap(key, idx)
        elif kname == "k3_compute_divergence":
            snap("div", 3)
            snap("marker", 4)
        elif kname == "k3_subtract_pressure_grad":
            snap("p", 3)
        elif kname == "k3_g2p_and_advect":
            snap("g2p_pos", 0)
            snap("g2p_vel", 1)
        elif kname == "k3_g2p_apic_advect":
            snap("g2p_pos", 0)
            snap("g2p_vel", 1)
            snap("g2p_C", 2)

    warp_shim.LAUNCH_HOOK[0] = hook
    t0 = time.time()
    for it in range(cfg["substeps"]):
        s.step(cfg["dt"], pressure_iters=cfg["iters"], pressure_solver=cfg["solver"])
        if it == 0:
            out["pressure_iters_first"] = np.int32(s.last_pressure_iters)
        state["first"] = False
    warp_shim.LAUNCH_HOOK[0] = None
    out["final_pos"] = s.pos.numpy()
    out["final_vel"] = s.vel.numpy()
    out["final_C"] = s.affine_C.numpy()
    out["final_marker"] = s.marker.numpy()
    out["final_p"] = s.p.numpy()
    out["final_u"] = s.u.numpy()
    out["final_v"] = s.v.numpy()
    out["final_w"] = s.w.numpy()
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"{name}: P={s.n_particles} {time.time() - t0:.1f}s -> {path}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("GPUFLUID_REFERENCE"),
                    required="GPUFLUID_REFERENCE" not in os.environ,
                    help="GPUFLUID source checkout (or set GPUFLUID_REFERENCE)")
    ap.add_argument("--only", default=None)
    a = ap.parse_args()
    ref_src = os.path.join(a.reference, "src")
    for name, cfg in SCENES.items():
        if a.only and name != a.only:
            continue
        run_scene(name, cfg, ref_src)


if __name__ == "__main__":
    main()
