"""Scene TOML parsing and the simulate/info commands (tests/test_c7_cli.py of
the reference: the same minimal scene, the same C7.1 errors)."""
import json
from pathlib import Path

import numpy as np
import pytest

from gpufluid_b200 import scene as sc
from gpufluid_b200.cli import build_obstacle_sdf, main, make_solver
from gpufluid_b200.config import (BlockError, ObstacleCylinderYCfg, ObstaclePlaneCfg,
                                  ObstacleSphereCfg, SceneCfg, SimulationCfg, load_scene)


def _write_minimal(tmp_path: Path, frames: int = 2, extra_sim: str = "") -> Path:
    cfg = tmp_path / "scene.toml"
    cfg.write_text(f"""
[domain]
resolution = [16, 16, 16]

[fluid]
type = "box"
lo = [0.10, 0.30, 0.10]
hi = [0.50, 0.90, 0.50]
ppc = 8

[[obstacle]]
type = "sphere"
center = [0.5, 0.20, 0.5]
radius = 0.10

[[obstacle]]
type = "cylinder_y"
center = [0.30, 0.30, 0.30]
radius = 0.05
half_height = 0.20

[simulation]
dt = 0.005
pressure_iters = 20
frames = {frames}
fps = 24
{extra_sim}

[output]
cache_dir = "cache"
mesh = true
particles = true
iso_level = 0.5
smooth_passes = 1
""")
    return cfg


def test_parse_minimal(tmp_path):
    scene = load_scene(_write_minimal(tmp_path))
    assert isinstance(scene, SceneCfg)
    assert scene.domain.resolution == (16, 16, 16)
    assert len(scene.obstacle) == 2
    assert isinstance(scene.obstacle[0], ObstacleSphereCfg)
    assert isinstance(scene.obstacle[1], ObstacleCylinderYCfg)
    assert scene.simulation.frames == 2
    assert scene.dx == pytest.approx(1.0 / 16)
    assert scene.output.particles is True


def test_preconditioner_keys_parse(tmp_path):
    """Optional [simulation] keys of this build: the PCG preconditioner."""
    cfg = _write_minimal(tmp_path, extra_sim='pcg_preconditioner = "tile_sgs"\n'
                                             'pcg_sgs_sweeps = 3\npcg_coarse = true')
    sim = load_scene(cfg).simulation
    assert (sim.pcg_preconditioner, sim.pcg_sgs_sweeps, sim.pcg_coarse) == ("tile_sgs", 3, True)
    sim = load_scene(_write_minimal(tmp_path)).simulation
    assert (sim.pcg_preconditioner, sim.pcg_sgs_sweeps, sim.pcg_coarse) == ("jacobi", 2, False)


def test_defaults_match_reference():
    # defaults of SimulationCfg in src/gpufluid/cli/config.py
    s = SimulationCfg()
    assert (s.solver, s.dt, s.pressure_iters, s.pressure_solver) == ("flip", 0.005, 60, "jacobi")
    assert (s.cfl, s.cfl_factor, s.cfl_max_substeps) == (False, 0.5, 16)
    assert (s.flip_blend, s.gravity, s.rho, s.transfer_mode) == (0.95, -9.81, 1.0, "flip")
    assert (s.frames, s.fps) == (100, 24)


def test_unknown_obstacle_raises(tmp_path):
    cfg = tmp_path / "bad.toml"
    cfg.write_text('[[obstacle]]\ntype = "trapezohedron"\ncenter = [0,0,0]\n')
    with pytest.raises(BlockError) as ei:
        load_scene(cfg)
    assert ei.value.block_id == "C7.1"
    assert str(ei.value).startswith("[C7.1]")


def test_missing_file_raises(tmp_path):
    with pytest.raises(BlockError) as ei:
        load_scene(tmp_path / "nope.toml")
    assert ei.value.block_id == "C7.1"


def test_bad_vector_length_raises(tmp_path):
    cfg = tmp_path / "bad.toml"
    cfg.write_text('[domain]\nresolution = [16, 16]\n')
    with pytest.raises(BlockError):
        load_scene(cfg)


@pytest.mark.parametrize("extra, what", [
    ('solver = "mpm"', "flip only"),
    ("viscosity = 0.1", "viscosity"),
])
def test_out_of_scope_rejected(tmp_path, extra, what):
    scene = load_scene(_write_minimal(tmp_path, extra_sim=extra))
    with pytest.raises(BlockError) as ei:
        make_solver(scene, None)
    assert what in str(ei.value)


@pytest.mark.parametrize("key", ['mesh_method = "marching"',
                                 'mesh_smooth_method = "cotan"\nmesh_smooth_passes = 2',
                                 "decimate_ratio = 0.5"])
def test_mesh_options_outside_build_rejected(tmp_path, key):
    cfg = _write_minimal(tmp_path)
    cfg.write_text(cfg.read_text().replace("smooth_passes = 1\n", f"smooth_passes = 1\n{key}\n"))
    scene = load_scene(cfg)
    with pytest.raises(BlockError) as ei:
        make_solver(scene, None)
    assert ei.value.block_id == "C7.1" and key.split()[0] in str(ei.value)


_REGIONS = """
[[inflow]]
lo = [0.1, 0.7, 0.1]
hi = [0.3, 0.8, 0.3]
velocity = [0.0, -1.0, 0.0]
rate_per_sec = 2400.0

[[outflow]]
lo = [0.0, 0.0, 0.0]
hi = [1.0, 0.12, 1.0]
frame_start = 1
"""


def test_inflow_outflow_parse(tmp_path):
    """[[inflow]] / [[outflow]] parse with the reference's keys and defaults
    (config.py:140-166, :319-342)."""
    from gpufluid_b200.config import InflowCfg, OutflowCfg
    cfg = _write_minimal(tmp_path)
    cfg.write_text(cfg.read_text() + _REGIONS)
    scene = load_scene(cfg)
    assert scene.inflow == [InflowCfg(lo=(0.1, 0.7, 0.1), hi=(0.3, 0.8, 0.3),
                                      velocity=(0.0, -1.0, 0.0), rate_per_sec=2400.0)]
    assert scene.inflow[0].frame_end == 1_000_000 and scene.inflow[0].color is None
    assert scene.outflow == [OutflowCfg(lo=(0.0, 0.0, 0.0), hi=(1.0, 0.12, 1.0), frame_start=1)]
    (tmp_path / "b").mkdir()
    bad = _write_minimal(tmp_path / "b")
    bad.write_text(bad.read_text() + "\n[[outflow]]\nlo = [0, 0, 0]\n")
    with pytest.raises(BlockError):
        load_scene(bad)


@pytest.mark.gpu
def test_simulate_with_reseed(tmp_path):
    """reseed = true: frames 0 and 2 (every 2) reseed; the run completes and
    the particle counts stay finite."""
    cfg = _write_minimal(tmp_path, frames=3,
                         extra_sim="reseed = true\nreseed_every_n_frames = 2")
    assert main(["simulate", str(cfg)]) == 0
    last = np.load(tmp_path / "cache" / "particles" / "frame_0002.npy")
    assert len(last) > 0 and np.isfinite(last).all()


@pytest.mark.gpu
@pytest.mark.parametrize("mesh_keys", ['mesh_method = "sdf"\n',
                                       'mesh_smooth_passes = 2\nmesh_smooth_method = "laplacian"\n'])
def test_simulate_with_coarse_pcg_and_mesh_options(tmp_path, mesh_keys):
    """The preconditioner keys and the mesh options through the command line:
    refined PCG with tile SGS and the coarse correction; an sdf surface or a
    smoothed one per frame."""
    cfg = _write_minimal(tmp_path, frames=2,
                         extra_sim='pressure_solver = "pcg_refined"\n'
                                   'pcg_preconditioner = "tile_sgs"\npcg_coarse = true')
    cfg.write_text(cfg.read_text().replace("smooth_passes = 1\n", "smooth_passes = 1\n" + mesh_keys))
    assert main(["simulate", str(cfg)]) == 0
    from gpufluid_b200.mesh import read_ply
    v, t = read_ply(tmp_path / "cache" / "mesh" / "frame_0001.ply")
    assert len(v) > 0 and len(t) > 0 and np.isfinite(v).all()


@pytest.mark.gpu
def test_simulate_with_inflow_and_outflow(tmp_path):
    """The inflow adds round(2400/24) = 100 positions a frame (fewer if any
    land in a solid cell); from frame 1 the outflow slab y <= 0.12 drains."""
    cfg = _write_minimal(tmp_path, frames=3)
    cfg.write_text(cfg.read_text() + _REGIONS)
    assert main(["simulate", str(cfg)]) == 0
    counts = [len(np.load(tmp_path / "cache" / "particles" / f"frame_{f:04d}.npy"))
              for f in range(3)]
    seeded = len(sc.seed_box_positions(1.0 / 16, (0.10, 0.30, 0.10), (0.50, 0.90, 0.50), 8))
    assert counts[0] == seeded + 100
    assert counts[1] <= counts[0] + 100 and counts[2] <= counts[1] + 100
    last = np.load(tmp_path / "cache" / "particles" / "frame_0002.npy")
    assert np.isfinite(last).all()


def test_cli_error_exit_code(tmp_path, capsys):
    assert main(["simulate", str(tmp_path / "missing.toml")]) == 2
    assert "[C7.1]" in capsys.readouterr().err


def test_obstacle_sdf_union(tmp_path):
    scene = load_scene(_write_minimal(tmp_path))
    g = sc.cell_centers(16, 16, 16, 1.0 / 16)
    sdf = build_obstacle_sdf(scene, g)
    sph = np.linalg.norm(g - np.float32([0.5, 0.2, 0.5]), axis=-1) - 0.10
    assert np.allclose(np.minimum(sph, sdf), sdf)
    # sphere centre and the cylinder axis are inside; a far corner is not
    c = sc.cell_centers(16, 16, 16, 1.0 / 16)
    assert sdf[8, 3, 8] < 0           # (0.53, 0.22, 0.53)
    assert sdf[4, 4, 4] < 0           # (0.28, 0.28, 0.28), within r=0.05 of the axis
    assert sdf[15, 15, 15] > 0
    assert c.shape == (16, 16, 16, 3)


def test_sdf_cylinder_plane_values():
    pts = np.float32([[0.0, 0.0, 0.0], [0.3, 0.0, 0.0], [0.0, 0.5, 0.0], [0.3, 0.5, 0.0]])
    d = sc.sdf_cylinder_y(pts, (0, 0, 0), 0.1, 0.2)
    assert np.allclose(d, [-0.1, 0.2, 0.3, np.hypot(0.2, 0.3)], atol=1e-6)
    dp = sc.sdf_plane(np.float32([[0, 1, 0], [0, -2, 0]]), (0, 0, 0), (0, 2, 0))
    assert np.allclose(dp, [1.0, -2.0], atol=1e-6)
    ramp = SceneCfg(obstacle=[ObstaclePlaneCfg("plane", (0, 0.5, 0), (0, 1, 0), (0, 0, 0),
                                               (1, 1, 1))], obstacle_motion=[None])
    g = sc.cell_centers(8, 8, 8, 1.0 / 8)
    sdf = build_obstacle_sdf(ramp, g)
    assert (sdf[:, :4, :] < 0).all() and (sdf[:, 4:, :] > 0).all()


@pytest.mark.gpu
def test_simulate_end_to_end_creates_cache(tmp_path):
    cfg = _write_minimal(tmp_path, frames=2)
    assert main(["simulate", str(cfg), "--timings", "--checkpoint-every", "1"]) == 0
    cache = tmp_path / "cache"
    m = json.loads((cache / "cache.json").read_text())
    assert m["frame_count"] == 2 and m["fps"] == 24 and m["resolution"] == [16, 16, 16]
    assert m["schema_version"] == 1 and m["solver"] == "flip"
    assert m["particles_pattern"] == "particles/frame_{:04d}.npy"
    assert m["truncated_at_frame"] is None
    for f in range(2):
        a = np.load(cache / "particles" / f"frame_{f:04d}.npy")
        assert a.dtype == np.float32 and a.ndim == 2 and a.shape[1] == 3
        assert np.isfinite(a).all()
    # mesh/frame_NNNN.ply per frame (commands.py:721-770)
    assert m["mesh_pattern"] == "mesh/frame_{:04d}.ply"
    from gpufluid_b200.mesh import read_ply
    from oracle import mesh as om
    for f in range(2):
        v, tri = read_ply(cache / "mesh" / f"frame_{f:04d}.ply")
        assert len(v) > 0 and len(tri) > 0 and tri.max() < len(v)
        assert om.mesh_volume(v, tri) > 0
    t = json.loads((cache / "timings.json").read_text())
    assert set(t["sections_ms"]) >= {"p2g", "pressure", "g2p_advect"}
    assert t["mesh_total_s"] > 0
    ck = np.load(cache / "checkpoint_frame_0000.npz")
    assert int(ck["nx"]) == 16 and ck["pos"].shape == a.shape


@pytest.mark.gpu
def test_simulate_resume_from_checkpoint(tmp_path):
    cfg = _write_minimal(tmp_path, frames=3)
    assert main(["simulate", str(cfg), "--checkpoint-every", "2"]) == 0
    cache = tmp_path / "cache"
    ref = np.load(cache / "particles" / "frame_0002.npy")
    ck = cache / "checkpoint_frame_0001.npz"
    (cache / "particles" / "frame_0002.npy").unlink()
    assert main(["simulate", str(cfg), "--resume", str(ck), "--start-frame", "2"]) == 0
    again = np.load(cache / "particles" / "frame_0002.npy")
    assert again.shape == ref.shape
    # float-atomic P2G sums make the two runs agree to rounding only
    assert np.abs(again - ref).max() < 1e-3
