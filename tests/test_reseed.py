"""GPU particle reseeding (src/gpufluid/sim/reseed.py:275-396,
reseed_particles_gpu).

CPU: the oracle (oracle/reseed.py) against the reference function's own
output on the sequential Warp stand-in (tests/golden/reseed/reseed.npz, made
by tests/golden/make_reseed_golden.py): culling by rank in cell, solid-cell
drops, grid clamping and the jittered emission, bit for bit.  GPU:
``FlipSolver3D.reseed`` against the same vectors and against the oracle on
a dam-break state after a few substeps."""
import os

import numpy as np
import pytest

from gpufluid_b200.reseed import ReseedConfig
from oracle import reseed as orr

GOLD = os.path.join(os.path.dirname(__file__), "golden", "reseed", "reseed.npz")


def _gold():
    return dict(np.load(GOLD))


def test_oracle_matches_reference():
    g = _gold()
    p, v, ne, nc = orr.reseed(g["pos"], g["vel"], g["marker"], float(g["dx"]),
                              int(g["min_per_cell"]), int(g["max_per_cell"]),
                              float(g["jitter"]), np.random.default_rng(123))
    assert (ne, nc) == (int(g["n_emit"]), int(g["n_cull"]))
    assert np.array_equal(p, g["new_pos"]) and np.array_equal(v, g["new_vel"])


def test_config_defaults_match_reference():
    c = ReseedConfig()
    assert (c.min_per_cell, c.max_per_cell, c.jitter, c.every_n_frames) == (4, 16, 0.3, 5)


@pytest.mark.gpu
def test_reseed_matches_reference(gf):
    import torch
    g = _gold()
    nx, ny, nz = g["marker"].shape
    s = gf.FlipSolver3D(nx, ny, nz, transfer_mode="apic")
    s._set_particles(pos=g["pos"], vel=g["vel"])
    s._label.copy_(torch.from_numpy(g["marker"].astype(np.uint8)))
    ne, nc = s.reseed(ReseedConfig(), np.random.default_rng(123))
    assert (ne, nc) == (int(g["n_emit"]), int(g["n_cull"]))
    p, v = s.get_particles()
    assert np.array_equal(p, g["new_pos"]) and np.array_equal(v, g["new_vel"])
    assert np.count_nonzero(s.affine_C.numpy()) == 0
    assert np.array_equal(s.marker.numpy(), g["marker"])  # labels left as they were


@pytest.mark.gpu
def test_reseed_dam_break_matches_oracle(gf):
    """A 32^3 dam break after 6 substeps (crowded and thinned cells), with
    tighter bounds so that both culling and emission happen."""
    s = gf.FlipSolver3D(32, 32, 32)
    s.seed_box((0.0, 0.0, 0.0), (0.4, 0.6, 1.0))
    for _ in range(6):
        s.step(1.0 / 120.0, pressure_iters=40)
    pos, vel = s.get_particles()
    marker = s.marker.numpy()
    cfg = ReseedConfig(min_per_cell=6, max_per_cell=9)
    p, v, ne, nc = orr.reseed(pos, vel, marker, s.dx, cfg.min_per_cell, cfg.max_per_cell,
                              cfg.jitter, np.random.default_rng(5))
    assert ne > 0 and nc > 0
    assert s.reseed(cfg, np.random.default_rng(5)) == (ne, nc)
    gp, gv = s.get_particles()
    assert np.array_equal(gp, p) and np.array_equal(gv, v)
    s.step(1.0 / 120.0, pressure_iters=40)
    assert np.isfinite(s.pos.numpy()).all()
