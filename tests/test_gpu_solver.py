"""End-to-end FlipSolver3D on the GPU: the reference's golden scenes and the
relational invariants the reference's own tests assert
(tests/test_f3_solver.py, test_s2_6_3_pcg.py, test_s2_6_2_gsrb.py,
test_s2_12_apic_obstacle.py, test_b5_*_graph*.py, test_f3_5_checkpoint.py,
test_s2_10_gpu_cfl.py)."""
import glob
import os

import numpy as np
import pytest

from helpers import assert_bitexact, dam_break, rel_l2

pytestmark = pytest.mark.gpu
GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_golden_scene_end_to_end(gf, path):
    """Run the reference's golden scene through the public API.  Labels after
    the first binning are exact; after several substeps the state agrees with
    the reference within the drift that float-atomic summation order causes."""
    import torch
    g = np.load(path)
    nx, ny, nz = (int(x) for x in g["grid"])
    s = gf.FlipSolver3D(nx, ny, nz, flip_blend=float(g["flip_blend"]),
                        transfer_mode=str(g["transfer"]), pcg_rhs_sign=+1)
    s._marker_host[...] = g["init_marker"]
    s._label.copy_(torch.from_numpy(g["init_marker"].astype(np.uint8)))
    s.pos = g["init_pos"]
    s.vel = g["init_vel"]
    solver, iters, dt = str(g["solver"]), int(g["iters"]), float(g["dt"])
    s.step(dt, pressure_iters=iters, pressure_solver=solver)
    torch.cuda.synchronize()
    assert_bitexact("labels after substep 1", s.marker.numpy(), g["marker"])
    assert rel_l2(s.p.numpy(), g["p"]) < 1e-4
    assert rel_l2(s.pos.numpy(), g["g2p_pos"]) < 1e-6
    assert rel_l2(s.vel.numpy(), g["g2p_vel"]) < 1e-4
    if solver == "pcg":
        assert s.last_pressure_iters == int(g["pressure_iters_first"])
    for _ in range(int(g["substeps"]) - 1):
        s.step(dt, pressure_iters=iters, pressure_solver=solver)
    torch.cuda.synchronize()
    assert rel_l2(s.pos.numpy(), g["final_pos"]) < 1e-5
    assert rel_l2(s.vel.numpy(), g["final_vel"]) < 1e-3
    assert np.mean(s.marker.numpy() != g["final_marker"]) < 2e-3


def test_shapes_and_conservation(gf):
    """test_f3_solver.py:18-39: MAC shapes, 50 steps finite, count conserved, in domain."""
    s = dam_break(gf.FlipSolver3D, (16, 16, 16), box=((0.1, 0.1, 0.1), (0.5, 0.7, 0.5)))
    assert s.u.shape == (17, 16, 16) and s.v.shape == (16, 17, 16) and s.w.shape == (16, 16, 17)
    assert s.marker.shape == (16, 16, 16)
    n0 = s.n_particles
    for _ in range(50):
        s.step(0.005, pressure_iters=40)
    pos, vel = s.get_particles()
    assert pos.shape == (n0, 3) and np.isfinite(pos).all() and np.isfinite(vel).all()
    assert (pos > 0).all() and (pos < 1).all()
    assert not s.has_diverged()


def test_centroid_falls(gf):
    """test_f3_solver.py:42-50."""
    s = dam_break(gf.FlipSolver3D, (16, 16, 16), box=((0.2, 0.4, 0.2), (0.6, 0.8, 0.6)))
    y0 = s.get_particles()[0][:, 1].mean()
    for _ in range(60):
        s.step(0.005, pressure_iters=40)
    assert y0 - s.get_particles()[0][:, 1].mean() > 0.05


@pytest.mark.parametrize("solver,iters", [("pcg", 200), ("gsrb", 100), ("pcg_refined", 400)])
def test_solvers_agree_with_jacobi(gf, solver, iters):
    """test_s2_6_3_pcg.py:23-37 / test_s2_6_2_gsrb.py:9-21: centroid within 0.05
    of a 200-iteration Jacobi run (PCG here uses the physical sign)."""
    cents = []
    for sv, it in (("jacobi", 200), (solver, iters)):
        s = dam_break(gf.FlipSolver3D, (16, 16, 16), box=((0.1, 0.1, 0.1), (0.5, 0.7, 0.5)),
                      pressure_tol=1e-5)
        for _ in range(30):
            s.step(0.005, pressure_iters=it, pressure_solver=sv)
        cents.append(s.get_particles()[0].mean(axis=0))
    assert np.linalg.norm(cents[0] - cents[1]) < 0.05


@pytest.mark.parametrize("coarse", [False, True])
def test_tile_sgs_and_coarse_agree_with_jacobi_pcg(gf, coarse):
    """The tile SGS preconditioner, with and without the coarse correction,
    changes the iteration count, not the answer: after 20 substeps of a 48^3
    dam break the particles agree with the Jacobi-preconditioned refined PCG
    (all solved to 1e-7), in fewer iterations."""
    res, its = [], []
    for pre, crs in (("jacobi", False), ("tile_sgs", coarse)):
        s = dam_break(gf.FlipSolver3D, (48, 48, 48), box=((0.0, 0.0, 0.0), (0.4, 0.6, 1.0)),
                      pressure_tol=1e-7, pcg_preconditioner=pre, pcg_coarse=crs)
        for _ in range(20):
            s.step(1 / 480, pressure_iters=2000, pressure_solver="pcg_refined")
        res.append(s.get_particles()[0])
        its.append(s.last_pressure_iters)
        if crs:
            assert s.pressure_stats()["coarse"] == 1
    err = np.linalg.norm(res[0] - res[1]) / np.linalg.norm(res[0])
    assert err < 1e-5, err
    assert its[1] < its[0], its


def test_pcg_converges_quickly(gf):
    """test_s2_6_3_pcg.py:40-47: PCG converges in < 40 iterations on 16^3."""
    s = dam_break(gf.FlipSolver3D, (16, 16, 16), box=((0.1, 0.1, 0.1), (0.5, 0.7, 0.5)))
    s.step(0.005, pressure_iters=200, pressure_solver="pcg")
    assert 0 < s.last_pressure_iters < 40


def test_apic_obstacle_energy(gf):
    """test_s2_12_apic_obstacle.py:45-67 at 32^3: APIC KE / FLIP KE < 1.2, vmax < 2x."""
    ke, vmax = {}, {}
    for mode in ("flip", "apic"):
        s = dam_break(gf.FlipSolver3D, (32, 32, 32), transfer=mode,
                      sphere=((0.7, 0.2, 0.5), 0.12))
        for _ in range(40):
            s.step(1 / 240, pressure_iters=200, pressure_solver="pcg")
        v = s.get_particles()[1]
        ke[mode] = float((v ** 2).sum())
        vmax[mode] = float(np.linalg.norm(v, axis=1).max())
    assert ke["apic"] / ke["flip"] < 1.2
    assert vmax["apic"] / vmax["flip"] < 2.0


@pytest.mark.parametrize("solver", ["jacobi", "pcg", "pcg_refined"])
def test_graph_replay_matches_direct(gf, solver):
    """test_b5_1_cuda_graph_spike.py:73-105: graph replay == direct launches.
    The scene moves (seeded random initial velocities) so every velocity
    component is well above float32 rounding noise; the comparison is over the
    whole MAC field (u, v, w together), since two direct runs already differ
    by the order of the P2G float atomics."""
    out = []
    for graphs in (False, True):
        s = dam_break(gf.FlipSolver3D, (24, 24, 24), enable_cuda_graphs=graphs,
                      box=((0.1, 0.1, 0.1), (0.5, 0.7, 0.5)))
        s.vel = np.random.default_rng(3).normal(0, 0.5, (s.n_particles, 3)).astype(np.float32)
        for _ in range(5):
            s.step(0.005, pressure_iters=60, pressure_solver=solver)
        out.append((np.concatenate([s.u.numpy().ravel(), s.v.numpy().ravel(), s.w.numpy().ravel()]),
                    s.get_particles()[0]))
        if graphs:
            assert s._cuda_graph_misses == 1 and s._cuda_graph_hits == 4
    assert rel_l2(out[1][0], out[0][0]) < 1e-4
    assert rel_l2(out[1][1], out[0][1]) < 1e-6


@pytest.mark.parametrize("solver", ["jacobi", "pcg_refined"])
def test_c_abi_graph_capture_matches_direct(gf, solver):
    """gf_graph_capture / gf_graph_replay (the reference's graph cache,
    solver3d.py:3361-3418, as C entry points): five replays give the state of
    five direct gf_step calls, and the launch count advances per replay."""
    import ctypes
    import torch
    from gpufluid_b200 import _lib
    out = []
    for use_graph in (False, True):
        s = dam_break(gf.FlipSolver3D, (24, 24, 24), box=((0.1, 0.1, 0.1), (0.5, 0.7, 0.5)))
        s.vel = np.random.default_rng(3).normal(0, 0.5, (s.n_particles, 3)).astype(np.float32)
        prm = s._params(0.005, 60, solver)
        s._set_stream()
        if use_graph:
            g = ctypes.c_void_p()
            _lib.check(s._L.gf_graph_capture(s._ctx, ctypes.byref(prm), ctypes.byref(g)),
                       s._ctx, "gf_graph_capture")
            n0 = int(s._L.gf_launch_count(s._ctx))
            for _ in range(5):
                _lib.check(s._L.gf_graph_replay(s._ctx, g), s._ctx, "gf_graph_replay")
            torch.cuda.synchronize()
            per = (int(s._L.gf_launch_count(s._ctx)) - n0) // 5
            assert per > 5
            assert s._L.gf_graph_destroy(g) == 0
        else:
            for _ in range(5):
                _lib.check(s._L.gf_step(s._ctx, ctypes.byref(prm)), s._ctx, "gf_step")
        s._pressure_stale = True
        out.append((np.concatenate([s.u.numpy().ravel(), s.v.numpy().ravel(),
                                    s.w.numpy().ravel()]), s.get_particles()[0],
                    s.pressure_health()["solves"]))
    assert rel_l2(out[1][0], out[0][0]) < 1e-4
    assert rel_l2(out[1][1], out[0][1]) < 1e-6
    assert out[0][2] == out[1][2] == 5  # the solve health is folded in on replay too


def test_checkpoint_resume_matches_continuous(gf, tmp_path):
    """test_f3_5_checkpoint.py:11-41."""
    a = dam_break(gf.FlipSolver3D, (16, 16, 16), transfer="apic")
    for _ in range(10):
        a.step(0.005, pressure_iters=40)
    a.save_checkpoint(tmp_path / "c.npz")
    b = gf.FlipSolver3D(16, 16, 16, transfer_mode="apic")
    b.load_checkpoint(tmp_path / "c.npz")
    for s in (a, b):
        for _ in range(10):
            s.step(0.005, pressure_iters=40)
    pa, pb = a.get_particles()[0], b.get_particles()[0]
    assert np.sqrt(np.mean((pa - pb) ** 2)) < 1e-3
    c = gf.FlipSolver3D(8, 8, 8)
    with pytest.raises(RuntimeError):
        c.load_checkpoint(tmp_path / "c.npz")


def test_gpu_cfl_matches_host(gf):
    """test_s2_10_gpu_cfl.py:24-39."""
    from gpufluid_b200 import cfl_substep_count, cfl_substep_count_gpu
    s = dam_break(gf.FlipSolver3D, (16, 16, 16))
    rng = np.random.default_rng(0)
    s.vel = rng.normal(0, 2.0, (s.n_particles, 3)).astype(np.float32)
    v = s.get_particles()[1]
    for t in (0.01, 0.04, 0.2):
        assert cfl_substep_count_gpu(s, s.dx, t) == cfl_substep_count(v, s.dx, t)


def test_profiler_sections(gf):
    """test_g1_9_step_profiler.py:24-56: every section fires once per step."""
    s = dam_break(gf.FlipSolver3D, (16, 16, 16), enable_timing=True)
    for _ in range(3):
        s.step(0.005, pressure_iters=20)
    counts = s._prof.call_counts
    assert set(counts) == {"clear", "p2g", "normalize", "gravity_bc", "divergence", "pressure",
                           "grad_subtract_bc", "g2p_advect", "color"}
    assert all(c == 3 for c in counts.values())
    assert s._prof.summarize()["pressure"] > 0


def test_unknown_solver_raises(gf):
    s = dam_break(gf.FlipSolver3D, (8, 8, 8))
    with pytest.raises(ValueError, match="unknown pressure_solver"):
        s.step(0.005, pressure_solver="multigrid")


def test_refined_pcg_warm_start(gf, oracle):
    """pcg_warm_start: the refined solve starts from the previous substep's
    pressure.  Same FP64-residual target (relative to ||b||), the answer
    within 1e-6 of an FP64 solve of each substep's system, fewer iterations
    than the cold start once the flow is under way."""
    from gpufluid_b200 import scene
    it = {}
    for warm in (False, True):
        s = gf.FlipSolver3D(64, 64, 64, transfer_mode="apic", pressure_tol=1e-8,
                            pcg_preconditioner="tile_sgs", pcg_coarse=True, pcg_warm_start=warm)
        s.add_solid_from_sdf(scene.sdf_sphere(s.cell_centers_np(), (0.7, 0.2, 0.5), 0.12))
        s.seed_box((0.0, 0.0, 0.0), (0.4, 0.6, 1.0))
        n = []
        for k in range(12):
            s.step(1 / 480, pressure_iters=4000, pressure_solver="pcg_refined")
            st = s.pressure_stats()
            assert st["status"] == 0 and st["kernel"] == 1 and st["relres"] <= 1e-8, (warm, st)
            n.append(st["iters"])
        p64, _, _ = oracle.pcg64(s.marker.numpy(), s.div.cpu().numpy(), tol=1e-14)
        assert rel_l2(s.p.numpy(), p64) < 1e-6
        it[warm] = n
    assert sum(it[True][4:]) < sum(it[False][4:]), it


def test_autotune_tile_shapes_and_state_restored(gf):
    """gf_autotune on a single scene: picks P2G and G2P tile shapes (8^3 or
    8 x 8 x 16 blocks), leaves the particle state where it was, and the
    tuned substep reaches the state an untuned one does."""
    out = []
    for tune in (False, True):
        s = dam_break(gf.FlipSolver3D, (48, 40, 64), transfer="apic")
        s.vel = np.random.default_rng(5).normal(0, 0.5, (s.n_particles, 3)).astype(np.float32)
        before = s.get_particles()
        if tune:
            info = s.autotune(1 / 240, 60, "jacobi")
            assert info["p2g_tiles_k"] in (1, 2) and info["g2p_tiles_k"] in (0, 1, 2), info
            assert info["p2g_map"] in (0, 1, 2, 3, 4, 5), info
            assert info["step_ms_before"] > 0 and info["step_ms_after"] > 0
            after = s.get_particles()
            assert np.array_equal(before[0], after[0]) and np.array_equal(before[1], after[1])
        for _ in range(3):
            s.step(1 / 240, pressure_iters=60, pressure_solver="jacobi")
        out.append(s.get_particles()[0])
    assert rel_l2(out[1], out[0]) < 1e-5
