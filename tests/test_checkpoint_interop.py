"""Checkpoints across implementations (FlipSolver3D.save_checkpoint /
load_checkpoint, src/gpufluid/solvers/solver3d.py:4127-4222).

The fixtures in tests/golden/checkpoint/ come from the reference's own code
(tests/golden/make_checkpoint_golden.py): a checkpoint its save_checkpoint
wrote mid-simulation, its state after resuming from that file and stepping
once, and a checkpoint this repo's writer produced together with the arrays
the reference's load_checkpoint read back from it.
"""
import os

import numpy as np
import pytest

from gpufluid_b200.solver import read_checkpoint, write_checkpoint
from helpers import assert_bitexact, rel_l2

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "checkpoint")
REF = os.path.join(HERE, "reference_apic16.npz")
GRID = (16, 16, 16)


def _load(name):
    with np.load(os.path.join(HERE, name), allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def test_reference_checkpoint_reads_here():
    d = read_checkpoint(REF, GRID, 1.0 / 16, {"gravity": -9.81, "flip_blend": 0.95})
    raw = _load("reference_apic16.npz")
    for k in ("pos", "vel", "affine_C", "marker"):
        assert_bitexact(k, d[k], raw[k])
    assert raw["pos"].shape == (6912, 3) and str(raw["transfer_mode"]) == "apic"


def test_repo_writer_matches_reference_layout_and_loader(tmp_path):
    """This repo's writer gives the reference's keys and dtypes, and the file
    it wrote passed the reference loader unchanged."""
    ref, mine = _load("reference_apic16.npz"), _load("repo_written.npz")
    assert set(ref) == set(mine)
    for k in ref:
        assert ref[k].dtype == mine[k].dtype, k
    loaded = _load("repo_loaded_by_reference.npz")
    for k in ("pos", "vel", "affine_C", "marker"):
        assert_bitexact(k, loaded[k], mine[k])
    # the writer still produces that file from the same seeded arrays
    rng = np.random.default_rng(11)
    n = 500
    pos = (0.1 + 0.5 * rng.random((n, 3))).astype(np.float32)
    vel = rng.normal(0, 0.5, (n, 3)).astype(np.float32)
    aff = rng.normal(0, 1.0, (n, 3, 3)).astype(np.float32)
    p = tmp_path / "again.npz"
    write_checkpoint(p, pos, vel, aff, mine["marker"],
                     dict(nx=16, ny=16, nz=16, dx=1.0 / 16, gravity=-9.81, flip_blend=0.95,
                          rho=1.0, viscosity=0.0, transfer_mode="apic", surface_tension=0.0))
    again = dict(np.load(p, allow_pickle=False))
    assert set(again) == set(mine)
    for k in mine:
        assert np.array_equal(again[k], mine[k]), k


def test_oracle_resumes_reference_checkpoint_bit_exact(oracle):
    """The pinned oracle, resumed from the reference's checkpoint, reproduces
    the reference's next substep bit for bit (checks the fixture)."""
    d = read_checkpoint(REF, GRID, 1.0 / 16)
    want = _load("reference_resume.npz")
    o = oracle.OracleFlip(*GRID, transfer_mode="apic")
    o.marker[...] = d["marker"]
    o.set_particles(d["pos"], d["vel"], d["affine_C"])
    o.step(float(want["dt"]), pressure_iters=int(want["iters"]), pressure_solver="jacobi")
    for k, got in (("pos", o.pos), ("vel", o.vel), ("affine_C", o.C), ("marker", o.marker)):
        assert_bitexact(k, got, want[k])


@pytest.mark.gpu
def test_solver_resumes_reference_checkpoint(gf, tmp_path):
    import torch
    s = gf.FlipSolver3D(*GRID, transfer_mode="apic")
    s.load_checkpoint(REF)
    raw = _load("reference_apic16.npz")
    assert_bitexact("pos", s.pos.numpy(), raw["pos"])
    assert_bitexact("C", s.affine_C.numpy(), raw["affine_C"])
    assert_bitexact("marker", s.marker.numpy(), raw["marker"])
    want = _load("reference_resume.npz")
    s.step(float(want["dt"]), pressure_iters=int(want["iters"]), pressure_solver="jacobi")
    torch.cuda.synchronize()
    assert_bitexact("marker", s.marker.numpy(), want["marker"])
    # P2G's float atomics order the face sums differently: tolerance
    assert rel_l2(s.pos.numpy(), want["pos"]) < 1e-6
    assert rel_l2(s.vel.numpy(), want["vel"]) < 1e-5
    assert rel_l2(s.affine_C.numpy(), want["affine_C"]) < 1e-4
    # and what this solver saves has the reference's layout
    p = tmp_path / "mine.npz"
    s.save_checkpoint(p)
    mine = dict(np.load(p, allow_pickle=False))
    assert set(mine) == set(raw)
    for k in raw:
        assert mine[k].dtype == raw[k].dtype, k
