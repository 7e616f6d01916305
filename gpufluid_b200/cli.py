"""Command line: ``python -m gpufluid_b200 {simulate,bench,info}``.

``simulate`` follows cmd_simulate of src/gpufluid/cli/commands.py:450-901 for a
FLIP/PIC/APIC scene:
- it builds the solver from the TOML, adds the static obstacles' union SDF,
  seeds the fluid or resumes a checkpoint;
- per frame it runs round(1/(fps*dt)) substeps (or step_cfl when cfl = true),
  checks has_diverged() and the frame's pressure-solve health (a failed solve
  truncates the bake like a divergence), writes mesh/frame_NNNN.ply (binary PLY of the GPU
  iso-surface; an empty placeholder when no surface emerges) when
  [output] mesh = true, particles/frame_NNNN.npy when [output] particles =
  true, and writes checkpoints every --checkpoint-every frames;
- it writes cache.json (CacheManifest keys of src/gpufluid/io/cache.py:28-93)
  and, with --timings, timings.json;
- it returns 2 on divergence or a configuration error, else 0.

Mesh decimation (pyfqmr in the reference: third-party code) is refused with
BlockError("C7.1").
``bench`` runs the reference's fixed throughput table (commands.py:953-977)
with device-synchronised timing.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

from .config import (BlockError, FluidBoxCfg, ObstacleBoxCfg, ObstacleCylinderYCfg,
                     ObstacleMeshCfg, ObstaclePlaneCfg, ObstacleSphereCfg, load_scene)

CACHE_SCHEMA_VERSION = 1
__version__ = "0.1.0"


def build_obstacle_sdf(scene, grid_xyz):
    """Union of the static obstacles' SDFs (commands.py:42-96)."""
    from .scene import sdf_box, sdf_cylinder_y, sdf_plane, sdf_sphere
    parts = []
    for ob, motion in zip(scene.obstacle, scene.obstacle_motion or [None] * len(scene.obstacle)):
        if motion is not None:
            raise BlockError("C7.1", "animated obstacles are not part of this build")
        if isinstance(ob, ObstacleSphereCfg):
            parts.append(sdf_sphere(grid_xyz, ob.center, ob.radius))
        elif isinstance(ob, ObstacleBoxCfg):
            parts.append(sdf_box(grid_xyz, ob.center, ob.half_size))
        elif isinstance(ob, ObstacleCylinderYCfg):
            parts.append(sdf_cylinder_y(grid_xyz, ob.center, ob.radius, ob.half_height))
        elif isinstance(ob, ObstaclePlaneCfg):
            half = tuple((np.asarray(ob.bbox_hi) - np.asarray(ob.bbox_lo)) * 0.5)
            center = tuple((np.asarray(ob.bbox_hi) + np.asarray(ob.bbox_lo)) * 0.5)
            parts.append(np.maximum(sdf_plane(grid_xyz, ob.point, ob.normal),
                                    sdf_box(grid_xyz, center, half)))
        elif isinstance(ob, ObstacleMeshCfg):
            raise BlockError("C7.1", "mesh obstacles are not part of this build")
    if not parts:
        return None
    out = parts[0]
    for q in parts[1:]:
        out = np.minimum(out, q)
    return out


def check_mesh_options(out):
    """Refuse the [output] mesh options outside this build (C7.1)."""
    if not out.mesh:
        return
    if out.mesh_method not in ("trilinear", "cubic", "sdf"):
        raise BlockError("C7.1", f"output.mesh_method {out.mesh_method!r}: expected "
                                 "'trilinear', 'cubic' or 'sdf'")
    if out.mesh_smooth_passes > 0 and out.mesh_smooth_method not in ("taubin", "laplacian"):
        raise BlockError("C7.1", f"output.mesh_smooth_method {out.mesh_smooth_method!r}: "
                                 "expected 'taubin' or 'laplacian'")
    if out.decimate_ratio < 1.0:
        raise BlockError("C7.1", "output.decimate_ratio < 1 (mesh decimation) is not part of "
                                 "this build")


def make_solver(scene, args):
    from .solver import FlipSolver3D
    sim = scene.simulation
    check_mesh_options(scene.output)
    if sim.solver != "flip":
        raise BlockError("C7.1", f"solver {sim.solver!r} is not part of this build (flip only)")
    nx, ny, nz = scene.domain.resolution
    try:
        solver = FlipSolver3D(nx=nx, ny=ny, nz=nz, dx=scene.dx, gravity=sim.gravity,
                              flip_blend=sim.flip_blend, rho=sim.rho, viscosity=sim.viscosity,
                              viscosity_iters=sim.viscosity_iters,
                              surface_tension=sim.surface_tension,
                              csf_smoothing_passes=sim.csf_smoothing_passes,
                              transfer_mode=sim.transfer_mode,
                              enable_timing=bool(getattr(args, "timings", False)),
                              enable_cuda_graphs=bool(getattr(args, "enable_cuda_graphs", False)),
                              enable_sub_dense=bool(getattr(args, "enable_sub_dense", False)),
                              pressure_tol=sim.pressure_tol, pcg_rhs_sign=sim.pcg_rhs_sign,
                              pcg_check_every=sim.pcg_check_every,
                              pcg_preconditioner=sim.pcg_preconditioner,
                              pcg_sgs_sweeps=sim.pcg_sgs_sweeps, pcg_coarse=sim.pcg_coarse)
    except (NotImplementedError, ValueError) as e:
        raise BlockError("C7.1", str(e)) from None
    sdf = build_obstacle_sdf(scene, solver.cell_centers_np())
    if sdf is not None:
        solver.add_solid_from_sdf(sdf)
    # inflows / outflows (commands.py:512-530)
    from .regions import InflowBox, OutflowBox
    try:
        for inf in scene.inflow:
            solver.add_inflow(InflowBox(lo=inf.lo, hi=inf.hi, velocity=inf.velocity,
                                        rate_per_sec=inf.rate_per_sec,
                                        frame_start=inf.frame_start, frame_end=inf.frame_end,
                                        color=inf.color, temperature=inf.temperature))
        for out in scene.outflow:
            solver.add_outflow(OutflowBox(lo=out.lo, hi=out.hi, frame_start=out.frame_start,
                                          frame_end=out.frame_end))
    except ValueError as e:
        raise BlockError("C7.1", str(e)) from None
    return solver


def _seed(solver, scene):
    sources = scene.fluids if scene.fluids else [scene.fluid]
    for i, f in enumerate(sources):
        if not isinstance(f, FluidBoxCfg):
            raise BlockError("C7.1", "mesh fluid sources are not part of this build")
        if f.color is not None or f.temperature is not None:
            raise BlockError("C7.1", "colour/temperature attributes are not part of this build")
        # several [[fluids]] blocks accumulate (the reference keeps them only
        # when they carry attributes; here every block is kept)
        solver.seed_box(f.lo, f.hi, ppc=f.ppc, append=i > 0)


def cmd_simulate(args) -> int:
    scene = load_scene(args.config)
    sim = scene.simulation
    nx, ny, nz = scene.domain.resolution
    print(f"[gpufluid-b200] simulate: {args.config}")
    print(f"           resolution {nx}x{ny}x{nz}   dx={scene.dx:.5f}   domain={scene.domain_size}")
    solver = make_solver(scene, args)
    if getattr(args, "resume", None):
        try:
            solver.load_checkpoint(args.resume)
        except RuntimeError as e:
            print(f"error: resume: {e}", file=sys.stderr)
            return 2
    else:
        _seed(solver, scene)
    print(f"           particles: {solver.n_particles}")
    cache_dir = Path(scene.output.cache_dir)
    if not cache_dir.is_absolute() and scene.config_dir is not None:
        cache_dir = scene.config_dir / cache_dir
    cache_dir.mkdir(parents=True, exist_ok=True)
    mesh_dir = cache_dir / "mesh"
    mesh_dir.mkdir(exist_ok=True)
    parts_dir = cache_dir / "particles"
    if scene.output.particles:
        parts_dir.mkdir(exist_ok=True)
    extractor = None
    if scene.output.mesh:
        from .mesh import MeshExtractor, write_ply
        extractor = MeshExtractor(nx, ny, nz, scene.dx)
    t_mesh = 0.0
    verts = None
    steps_per_frame = max(1, int(round(1.0 / (sim.fps * sim.dt))))
    start_frame = int(getattr(args, "start_frame", 0))
    ckpt_every = int(getattr(args, "checkpoint_every", 0))
    t_sim = 0.0
    truncated, reason = None, None
    n_capped = 0  # pressure solves that stopped at their iteration cap
    solver.pressure_health(reset=True)
    import torch
    # reseeding every reseed_every_n_frames frames (commands.py:612-660)
    rng_reseed = np.random.default_rng(123)
    reseed_cfg = None
    if sim.reseed:
        from .reseed import ReseedConfig
        reseed_cfg = ReseedConfig(min_per_cell=sim.reseed_min_per_cell,
                                  max_per_cell=sim.reseed_max_per_cell,
                                  every_n_frames=sim.reseed_every_n_frames)
    for frame in range(start_frame, sim.frames):
        solver.prepare_frame(frame, 1.0 / sim.fps)
        if (reseed_cfg is not None and frame % reseed_cfg.every_n_frames == 0
                and solver.n_particles > 0):
            solver.reseed(reseed_cfg, rng_reseed)
        torch.cuda.synchronize()
        ts = time.time()
        if sim.cfl:
            solver.step_cfl(sim.dt * steps_per_frame, pressure_iters=sim.pressure_iters,
                            cfl=sim.cfl_factor, max_substeps=sim.cfl_max_substeps,
                            pressure_solver=sim.pressure_solver)
        else:
            for _ in range(steps_per_frame):
                solver.step(sim.dt, pressure_iters=sim.pressure_iters,
                            pressure_solver=sim.pressure_solver)
        torch.cuda.synchronize()
        t_sim += time.time() - ts
        if solver.has_diverged():
            truncated, reason = frame, "flip_divergence"
            print(f"[flip] solver diverged at frame {frame} (last dumped: {frame}/{sim.frames}).",
                  file=sys.stderr)
            break
        # the frame's pressure solves, read once: a failed solve (CG
        # breakdown, a non-finite value, a device wait that ran out) ends the
        # bake like a divergence; solves stopped at their cap are counted
        health = solver.pressure_health(reset=True)
        if health["failed"]:
            truncated, reason = frame, "pressure_solve_failed"
            print(f"[flip] pressure solve failed ({health['worst_status']}) at frame {frame} "
                  f"(last dumped: {frame}/{sim.frames}).", file=sys.stderr)
            break
        n_capped += health["not_converged"]
        if extractor is not None:
            # commands.py:721-770; the splat reads the solver's particle
            # storage directly (its order only changes float atomics' order)
            tm = time.time()
            out = scene.output
            verts, faces = extractor.extract(
                solver._pos[:solver.n_particles], iso_level=out.iso_level,
                smooth_passes=out.smooth_passes, mesh_smooth_passes=out.mesh_smooth_passes,
                mesh_smooth_method=out.mesh_smooth_method,
                wall_margin_cells=out.wall_margin_cells, decimate_ratio=out.decimate_ratio,
                mesh_method=out.mesh_method, cubic_radius_cells=out.cubic_radius_cells,
                sdf_particle_radius_cells=out.sdf_particle_radius_cells,
                sdf_search_radius_cells=out.sdf_search_radius_cells)
            t_mesh += time.time() - tm
            if verts is not None:
                write_ply(mesh_dir / f"frame_{frame:04d}.ply", verts, faces)
            else:  # an empty placeholder keeps the frame indices aligned
                write_ply(mesh_dir / f"frame_{frame:04d}.ply", np.zeros((0, 3), np.float32),
                          np.zeros((0, 3), np.int32))
        if scene.output.particles:
            pos, _ = solver.get_particles()
            np.save(parts_dir / f"frame_{frame:04d}.npy", pos.astype(np.float32))
        if frame % 10 == 0 or frame == sim.frames - 1:
            nv = len(verts) if extractor is not None and verts is not None else 0
            print(f"  frame {frame:04d}/{sim.frames} V={nv}")
        if ckpt_every > 0 and (frame + 1) % ckpt_every == 0:
            solver.save_checkpoint(cache_dir / f"checkpoint_frame_{frame:04d}.npz")
    manifest = {
        "schema_version": CACHE_SCHEMA_VERSION, "gpufluid_version": f"b200-{__version__}",
        "created_unix": time.time(), "fps": sim.fps,
        "frame_count": (truncated + 1) if truncated is not None else sim.frames,
        "mesh_pattern": "mesh/frame_{:04d}.ply",
        "particles_pattern": "particles/frame_{:04d}.npy" if scene.output.particles else None,
        "domain_size": list(scene.domain_size), "resolution": list(scene.domain.resolution),
        "dx": scene.dx,
        "notes": f"sim={t_sim:.1f}s mesh={t_mesh:.1f}s" + (
            f" pressure_at_cap={n_capped}" if n_capped else ""),
        "solver": "flip",
        "truncated_at_frame": int(truncated) if truncated is not None else None,
        "truncation_reason": reason,
    }
    (cache_dir / "cache.json").write_text(json.dumps(manifest, indent=2), encoding="utf-8")
    print(f"[gpufluid-b200] done. cache: {cache_dir}  sim total: {t_sim:.2f}s  "
          f"mesh total: {t_mesh:.2f}s")
    timings = solver._prof.summarize()
    if timings:
        (cache_dir / "timings.json").write_text(json.dumps(
            {"sections_ms": timings, "call_counts": solver._prof.call_counts,
             "sim_total_s": t_sim, "mesh_total_s": t_mesh,
             "pressure_solves_at_cap": n_capped}, indent=2, sort_keys=True))
    return 0 if truncated is None else 2


def cmd_bench(args) -> int:
    """Fixed table of commands.py:953-977, timed with device synchronisation."""
    import torch
    from .solver import FlipSolver3D
    print("[gpufluid-b200] solver throughput (3D, B200)")
    print(f"  {'resolution':>10} {'particles':>10} {'iters':>5} {'steps/s':>10} {'time/step':>10}")
    for n, ppc, iters, n_steps in [(48, 8, 50, 100), (64, 8, 50, 100), (96, 4, 40, 50)]:
        s = FlipSolver3D(nx=n, ny=n, nz=n, dx=1.0 / n)
        s.seed_box(lo=(0.05, 0.05, 0.05), hi=(0.40, 0.70, 0.40), ppc=ppc)
        for _ in range(3):
            s.step(0.005, pressure_iters=iters)
        torch.cuda.synchronize()
        t = time.time()
        for _ in range(n_steps):
            s.step(0.005, pressure_iters=iters)
        torch.cuda.synchronize()
        dt = time.time() - t
        print(f"  {n:>4}^3      {s.n_particles:>10} {iters:>5} {n_steps / dt:>10.1f} "
              f"{1000 * dt / n_steps:>9.2f}ms")
    return 0


def cmd_info(args) -> int:
    import torch
    from . import _lib
    print(f"gpufluid-b200 {__version__}")
    print(f"  library: {_lib.LIB_PATH}")
    if torch.cuda.is_available():
        p = torch.cuda.get_device_properties(0)
        print(f"  device: {p.name}, {p.multi_processor_count} SMs, "
              f"{p.total_memory / 2**30:.0f} GiB, sm_{p.major}{p.minor}")
    else:
        print("  device: none (CUDA unavailable)")
    return 0


def main(argv=None) -> int:
    p = argparse.ArgumentParser("gpufluid_b200", description="B200 FLIP fluid simulator")
    sub = p.add_subparsers(dest="cmd", required=True)
    ps = sub.add_parser("simulate", help="run a TOML scene config")
    ps.add_argument("config")
    ps.add_argument("--resume", default=None)
    ps.add_argument("--start-frame", type=int, default=0)
    ps.add_argument("--checkpoint-every", type=int, default=0)
    ps.add_argument("--timings", action="store_true")
    ps.add_argument("--enable-cuda-graphs", action="store_true")
    ps.add_argument("--enable-sub-dense", action="store_true")
    ps.add_argument("--sub-rebuild-every", type=int, default=8)
    ps.add_argument("--sub-dilation", type=int, default=4)
    ps.set_defaults(func=cmd_simulate)
    sub.add_parser("bench", help="solver throughput benchmark").set_defaults(func=cmd_bench)
    sub.add_parser("info", help="device info").set_defaults(func=cmd_info)
    args = p.parse_args(argv)
    try:
        return args.func(args)
    except BlockError as e:
        print(f"error: {e}", file=sys.stderr)
        return 2
