"""Failure detection on the substep path, with no GPU fault.

The reference's only per-frame check is the NaN probe of has_diverged
(src/gpufluid/solvers/solver3d.py:2642-2656), after which the CLI truncates
the bake and returns 2 (src/gpufluid/cli/commands.py:712-719, :851-868).
Every failure here is made on the host or by a bounded device wait:

* NaN positions uploaded into the solver (as a --resume checkpoint): the
  substeps carry them, has_diverged() sees them, the CLI truncates, rc 2;
* a PCG capped at one iteration with tol 1e-12: NOT_CONVERGED in the
  device-side solve health, read once per frame, not an error;
* a test-only flag that makes the shared-memory PCG's first grid reduction
  wait for a count nobody publishes, with a 4096-poll limit: every block
  gives up and returns, the solve reports GF_TIMEOUT, the context keeps
  working, and the CLI truncates the bake with "pressure_solve_failed";
* truncated, damaged or inconsistent checkpoint files: RuntimeError before
  any state changes (CPU only).
"""
import ctypes
import json
from pathlib import Path

import numpy as np
import pytest

from gpufluid_b200.solver import read_checkpoint
from helpers import rel_l2


def _ckpt_arrays(n=(8, 6, 4), P=50, seed=0):
    rng = np.random.default_rng(seed)
    return dict(pos=rng.random((P, 3)).astype(np.float32) * 0.4,
                vel=rng.normal(size=(P, 3)).astype(np.float32),
                affine_C=np.zeros((P, 3, 3), np.float32),
                marker=np.zeros(n, np.int32), attr_color=np.zeros((0, 3), np.float32),
                attr_temperature=np.zeros((0,), np.float32), nx=n[0], ny=n[1], nz=n[2],
                dx=1.0 / max(n), gravity=-9.81, flip_blend=0.95, rho=1.0, viscosity=0.0,
                transfer_mode="flip", surface_tension=0.0)


def test_read_checkpoint_valid_and_rejects_bad_files(tmp_path):
    n = (8, 6, 4)
    good = tmp_path / "good.npz"
    np.savez_compressed(good, **_ckpt_arrays(n))
    d = read_checkpoint(good, n, 1.0 / 8)
    assert d["pos"].shape == (50, 3) and d["marker"].shape == n
    raw = good.read_bytes()
    cases = {
        "truncated": raw[: len(raw) // 2],
        "garbage": bytes(np.random.default_rng(1).integers(0, 256, 4096, dtype=np.uint8)),
        "empty": b"",
    }
    for name, blob in cases.items():
        p = tmp_path / f"{name}.npz"
        p.write_bytes(blob)
        with pytest.raises(RuntimeError):
            read_checkpoint(p, n, 1.0 / 8)
    # a byte flipped inside the compressed payload
    bad = bytearray(raw)
    bad[len(bad) // 3] ^= 0xFF
    (tmp_path / "flipped.npz").write_bytes(bytes(bad))
    with pytest.raises(RuntimeError):
        read_checkpoint(tmp_path / "flipped.npz", n, 1.0 / 8)
    # keys missing, wrong grid, wrong dx, inconsistent shapes
    a = _ckpt_arrays(n)
    del a["marker"]
    np.savez(tmp_path / "nokey.npz", **a)
    with pytest.raises(RuntimeError, match="keys missing"):
        read_checkpoint(tmp_path / "nokey.npz", n, 1.0 / 8)
    np.savez(tmp_path / "grid.npz", **_ckpt_arrays((8, 8, 8)))
    with pytest.raises(RuntimeError, match="grid"):
        read_checkpoint(tmp_path / "grid.npz", n, 1.0 / 8)
    a = _ckpt_arrays(n)
    a["dx"] = 0.2
    np.savez(tmp_path / "dx.npz", **a)
    with pytest.raises(RuntimeError, match="dx"):
        read_checkpoint(tmp_path / "dx.npz", n, 1.0 / 8)
    a = _ckpt_arrays(n)
    a["vel"] = a["vel"][:10]
    np.savez(tmp_path / "shape.npz", **a)
    with pytest.raises(RuntimeError, match="shapes"):
        read_checkpoint(tmp_path / "shape.npz", n, 1.0 / 8)


def _scene(tmp_path: Path, frames=2, solver="pcg", extra="") -> Path:
    cfg = tmp_path / "scene.toml"
    cfg.write_text(f"""
[domain]
resolution = [16, 16, 16]

[fluid]
type = "box"
lo = [0.10, 0.10, 0.10]
hi = [0.50, 0.60, 0.50]
ppc = 8

[simulation]
dt = 0.005
pressure_iters = 200
pressure_solver = "{solver}"
frames = {frames}
fps = 24
{extra}

[output]
cache_dir = "cache"
mesh = false
particles = true
""")
    return cfg


@pytest.mark.gpu
def test_nan_particles_are_detected(gf):
    s = gf.FlipSolver3D(16, 16, 16)
    s.seed_box((0.1, 0.1, 0.1), (0.5, 0.6, 0.5))
    assert not s.has_diverged()
    pos = s.pos.numpy()
    pos[17] = np.nan
    s.pos = pos
    assert s.has_diverged()
    s.step(0.005, pressure_iters=20)
    assert s.has_diverged()


@pytest.mark.gpu
def test_cli_truncates_bake_on_nan_resume(gf, tmp_path, capsys):
    from gpufluid_b200.cli import main
    cfg = _scene(tmp_path, frames=4)
    a = _ckpt_arrays((16, 16, 16), P=4000, seed=3)
    a["pos"] = (0.1 + 0.4 * np.random.default_rng(4).random((4000, 3))).astype(np.float32)
    a["marker"] = np.zeros((16, 16, 16), np.int32)
    a["marker"][[0, -1], :, :] = 2
    a["marker"][:, [0, -1], :] = 2
    a["marker"][:, :, [0, -1]] = 2
    a["pos"][123] = np.nan
    ck = tmp_path / "nan.npz"
    np.savez_compressed(ck, **a)
    assert main(["simulate", str(cfg), "--resume", str(ck), "--start-frame", "1"]) == 2
    m = json.loads((tmp_path / "cache" / "cache.json").read_text())
    assert m["truncated_at_frame"] == 1 and m["truncation_reason"] == "flip_divergence"
    assert m["frame_count"] == 2
    assert "diverged at frame 1" in capsys.readouterr().err


@pytest.mark.gpu
@pytest.mark.parametrize("graphs", [False, True])
def test_pcg_at_its_cap_is_reported_not_raised(gf, graphs):
    s = gf.FlipSolver3D(24, 24, 24, pressure_tol=1e-12, enable_cuda_graphs=graphs)
    s.seed_box((0.0, 0.0, 0.0), (0.4, 0.6, 1.0))
    h0 = s.pressure_health()
    assert h0["solves"] == 0 and h0["worst_status"] == "OK"
    for _ in range(3):
        s.step(1 / 240, pressure_iters=1, pressure_solver="pcg")
    h = s.check_pressure(frame=0)  # does not raise: a capped solve is not a failure
    assert h == {"worst_status": "NOT_CONVERGED", "solves": 3, "not_converged": 3,
                 "failed": 0, "last_status": "NOT_CONVERGED"}, h
    assert s.pressure_stats()["status"] == 3  # GF_NOT_CONVERGED
    assert s.pressure_health()["solves"] == 0  # reset by the read
    for _ in range(2):
        s.step(1 / 240, pressure_iters=400, pressure_solver="pcg")
    s.pressure_tol = 1e-4
    s.step(1 / 240, pressure_iters=400, pressure_solver="pcg")
    h = s.pressure_health()
    assert h["solves"] == 3 and h["failed"] == 0 and h["last_status"] == "OK", h
    # Jacobi and GS-RB run a fixed sweep count: always OK
    s.step(1 / 240, pressure_iters=10, pressure_solver="jacobi")
    assert s.pressure_health() == {"worst_status": "OK", "solves": 1, "not_converged": 0,
                                   "failed": 0, "last_status": "OK"}


def _stall_case(gf, n=32):
    import torch
    s = gf.FlipSolver3D(n, n, n)
    lab = s._marker_host.copy()
    lab[1:-1, 1:n // 2, 1:-1] = 1
    rng = np.random.default_rng(9)
    div = np.where(lab == 1, rng.normal(0, 1, lab.shape), 0).astype(np.float32)
    s._label.copy_(torch.from_numpy(lab.astype(np.uint8)).cuda())
    s.div.copy_(torch.from_numpy(div).cuda())
    return s, lab, div


@pytest.mark.gpu
def test_pcg_device_wait_runs_out_and_context_recovers(gf, oracle):
    """GF_FLAG_TEST_STALL: every block's first reduction wait runs out after
    4096 polls; the kernel returns, the status is GF_TIMEOUT, and the next
    solve on the same context succeeds."""
    import torch
    from gpufluid_b200 import _lib
    from gpufluid_b200.solver import PressureSolveError
    s, lab, div = _stall_case(gf)
    base = _lib.GF_FLAG_COARSE | (2 << _lib.GF_FLAG_SGS_SHIFT)
    for flags in (_lib.GF_FLAG_TEST_STALL, base | _lib.GF_FLAG_TEST_STALL):
        prm = _lib.StepParams(1 / 240, -9.81, 1.0, 0.95, 0, _lib.GF_PCG_REFINED, 400, 10,
                              1e-10, -1, flags)
        s._set_stream()
        assert s._L.gf_pressure(s._ctx, ctypes.byref(prm), None) == 0
        torch.cuda.synchronize()
        it, rel, st = ctypes.c_int32(), ctypes.c_double(), ctypes.c_int32()
        assert s._L.gf_pressure_result(s._ctx, ctypes.byref(it), ctypes.byref(rel),
                                       ctypes.byref(st)) == _lib.GF_TIMEOUT
        assert st.value == _lib.GF_TIMEOUT
        with pytest.raises(PressureSolveError, match="TIMEOUT"):
            s.check_pressure(frame=5)
    # the same context solves the same system afterwards
    for flags in (0, base):
        prm = _lib.StepParams(1 / 240, -9.81, 1.0, 0.95, 0, _lib.GF_PCG_REFINED, 4000, 10,
                              1e-10, -1, flags)
        s._set_stream()
        assert s._L.gf_pressure(s._ctx, ctypes.byref(prm), None) == 0
        st = s.pressure_stats()
        assert st["status"] == 0 and st["kernel"] == 1 and st["relres"] <= 1e-10, st
        p64, _, _ = oracle.pcg64(lab.astype(np.int32), div, tol=1e-14)
        assert rel_l2(s._p.cpu().numpy(), p64) < 1e-6
    h = s.pressure_health()
    assert h["failed"] == 0 and h["solves"] == 2 and h["worst_status"] == "OK", h


@pytest.mark.gpu
def test_cli_truncates_bake_on_failed_pressure_solve(gf, tmp_path, monkeypatch, capsys):
    from gpufluid_b200 import _lib
    from gpufluid_b200.cli import main
    from gpufluid_b200.solver import FlipSolver3D
    cfg = _scene(tmp_path, frames=3, solver="pcg")
    orig = FlipSolver3D._pcg_flags
    monkeypatch.setattr(FlipSolver3D, "_pcg_flags",
                        lambda self: orig(self) | _lib.GF_FLAG_TEST_STALL)
    assert main(["simulate", str(cfg)]) == 2
    m = json.loads((tmp_path / "cache" / "cache.json").read_text())
    assert m["truncated_at_frame"] == 0 and m["truncation_reason"] == "pressure_solve_failed"
    assert "pressure solve failed (TIMEOUT) at frame 0" in capsys.readouterr().err


@pytest.mark.gpu
def test_cli_rejects_damaged_resume(gf, tmp_path, capsys):
    from gpufluid_b200.cli import main
    cfg = _scene(tmp_path, frames=2)
    ck = tmp_path / "damaged.npz"
    ck.write_bytes(b"PK\x03\x04 not a checkpoint")
    assert main(["simulate", str(cfg), "--resume", str(ck)]) == 2
    assert "resume" in capsys.readouterr().err
