"""Inflow / outflow regions (src/gpufluid/domain/regions.py, the outflow
compaction kernels solver3d.py:1945-1985 and prepare_frame :3909-4040).

CPU: the oracle (oracle/regions.py) and the package's host-side emission
against the reference module's own outputs (tests/golden/regions/regions.npz, made by
tests/golden/make_regions_golden.py), plus the reference's region tests
(tests/test_d4_7_regions.py).  GPU: ``gf_outflow_compact`` bit-exact against
the golden survivors and the oracle (order kept), edge cases, and
``FlipSolver3D.prepare_frame`` against the oracle's frame hook."""
import ctypes
import os

import numpy as np
import pytest

from gpufluid_b200.regions import InflowBox, OutflowBox, apply_inflows, outflow_box_array
from oracle import regions as orc

GOLD = os.path.join(os.path.dirname(__file__), "golden", "regions", "regions.npz")
OUT_BOXES = [((0.0, 0.0, 0.0), (0.25, 0.25, 0.25), 0, 10),
             ((0.5, 0.1, 0.6), (0.75, 0.9, 1.0), 0, 10),
             ((0.3, 0.3, 0.3), (0.6, 0.6, 0.6), 5, 10)]
IN_BOXES = [dict(lo=(0.1, 0.6, 0.1), hi=(0.3, 0.8, 0.3), velocity=(0.0, -2.0, 0.5),
                 rate_per_sec=2400.0, frame_start=0, frame_end=10),
            dict(lo=(0.55, 0.5, 0.55), hi=(0.9, 0.6, 0.9), velocity=(1.0, 0.0, 0.0),
                 rate_per_sec=1000.0, frame_start=2, frame_end=10)]


def _gold():
    return dict(np.load(GOLD))


def _active_boxes(frame):
    return [[*lo, *hi] for lo, hi, a, b in OUT_BOXES if a <= frame <= b]


# ------------------------------------------------------------------- CPU
def test_oracle_outflow_matches_reference():
    g = _gold()
    keep = orc.outflow_keep(g["out_pos"], _active_boxes(2))
    assert np.array_equal(g["out_pos"][keep], g["kept_pos"])
    assert np.array_equal(g["out_vel"][keep], g["kept_vel"])


def test_emission_matches_reference():
    """The oracle and the package's InflowBox both reproduce the reference's
    emitted positions and velocities bit for bit (same generator stream)."""
    g = _gold()
    rng_o, rng_p = np.random.default_rng(0), np.random.default_rng(0)
    boxes = [InflowBox(**b) for b in IN_BOXES]
    po, vo, pp, vp = [], [], [], []
    for f in range(4):
        a, b = orc.inflows(IN_BOXES, f, 1.0 / 24.0, rng_o)
        c, d = apply_inflows(boxes, f, 1.0 / 24.0, rng_p)
        po.append(a); vo.append(b); pp.append(c); vp.append(d)
    for got_p, got_v in ((po, vo), (pp, vp)):
        assert np.array_equal(np.concatenate(got_p), g["emit_pos"])
        assert np.array_equal(np.concatenate(got_v), g["emit_vel"])


def test_inflow_emits_within_box_and_count():
    """tests/test_d4_7_regions.py:9-18."""
    inf = InflowBox(lo=(0.0, 0.5, 0.0), hi=(0.2, 0.6, 0.2), velocity=(0, -3, 0),
                    rate_per_sec=2400)
    pos, vel = apply_inflows([inf], 5, 1.0 / 24, np.random.default_rng(1))
    assert 80 <= len(pos) <= 120 and pos.shape[1] == 3
    assert (pos >= [0.0, 0.5, 0.0]).all() and (pos <= [0.2, 0.6, 0.2]).all()
    assert np.allclose(vel, [0, -3, 0])


def test_inflow_respects_frame_range():
    """tests/test_d4_7_regions.py:21-31."""
    inf = InflowBox(lo=(0, 0, 0), hi=(1, 1, 1), rate_per_sec=1000, frame_start=10, frame_end=20)
    rng = np.random.default_rng(0)
    assert len(apply_inflows([inf], 5, 0.04, rng)[0]) == 0
    assert len(apply_inflows([inf], 15, 0.04, rng)[0]) > 0
    assert len(apply_inflows([inf], 25, 0.04, rng)[0]) == 0
    assert len(apply_inflows([], 0, 1.0 / 24, rng)[0]) == 0


def test_outflow_box_validation_and_table():
    with pytest.raises(ValueError):
        OutflowBox(lo=(0.0, 0.5, 0.0), hi=(1.0, 0.4, 1.0))
    outs = [OutflowBox(lo=lo, hi=hi, frame_start=a, frame_end=b) for lo, hi, a, b in OUT_BOXES]
    assert np.array_equal(outflow_box_array(outs, 2), np.float32(_active_boxes(2)))
    assert outflow_box_array(outs, 11).shape == (0, 6)


def test_oracle_outflow_removes_inside_only():
    """tests/test_d4_7_regions.py:34-45 (boundaries are inside)."""
    pos = np.array([[0.1, 0.1, 0.1], [0.5, 0.5, 0.5], [0.15, 0.15, 0.15], [0.2, 0.2, 0.2]],
                   np.float32)
    keep = orc.outflow_keep(pos, [[0, 0, 0, 0.2, 0.2, 0.2]])
    assert keep.tolist() == [False, True, False, False]


# ------------------------------------------------------------------- GPU
def _compact(solver, pos, vel, boxes):
    import torch
    from gpufluid_b200 import _lib
    n = len(pos)
    p = torch.from_numpy(np.ascontiguousarray(pos, np.float32)).cuda()
    v = torch.from_numpy(np.ascontiguousarray(vel, np.float32)).cuda()
    po, vo = torch.empty_like(p), torch.empty_like(v)
    b = np.ascontiguousarray(np.asarray(boxes, np.float32).reshape(-1, 6))
    nout = ctypes.c_int64(-1)
    solver._set_stream()
    st = solver._L.gf_outflow_compact(
        solver._ctx, p.data_ptr(), v.data_ptr(), n,
        b.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), len(b), po.data_ptr(), vo.data_ptr(),
        ctypes.byref(nout))
    torch.cuda.synchronize()
    m = int(nout.value)
    return st, po[:m].cpu().numpy() if m > 0 else np.zeros((0, 3), np.float32), \
        vo[:m].cpu().numpy() if m > 0 else np.zeros((0, 3), np.float32)


@pytest.mark.gpu
def test_outflow_compaction_matches_reference(gf):
    s = gf.FlipSolver3D(16, 16, 16)
    g = _gold()
    st, p, v = _compact(s, g["out_pos"], g["out_vel"], _active_boxes(2))
    assert st == 0
    assert np.array_equal(p, g["kept_pos"]) and np.array_equal(v, g["kept_vel"])


@pytest.mark.gpu
def test_outflow_compaction_large_and_edges(gf):
    """1.5 M particles (1,465 blocks: the offsets scan runs in two chunks),
    no boxes, a box holding everything, no particles, and a reversed box."""
    s = gf.FlipSolver3D(16, 16, 16)
    rng = np.random.default_rng(9)
    pos = rng.random((1_500_000, 3)).astype(np.float32)
    vel = rng.normal(size=pos.shape).astype(np.float32)
    boxes = _active_boxes(2) + [[0.9, 0.0, 0.0, 1.0, 1.0, 0.05]]
    st, p, v = _compact(s, pos, vel, boxes)
    keep = orc.outflow_keep(pos, boxes)
    assert st == 0 and np.array_equal(p, pos[keep]) and np.array_equal(v, vel[keep])
    st, p, _ = _compact(s, pos, vel, np.zeros((0, 6), np.float32))
    assert st == 0 and np.array_equal(p, pos)
    st, p, _ = _compact(s, pos, vel, [[0, 0, 0, 1, 1, 1]])
    assert st == 0 and len(p) == 0
    st, p, _ = _compact(s, pos[:0], vel[:0], boxes)
    assert st == 0 and len(p) == 0
    st, _, _ = _compact(s, pos, vel, [[0, 0.5, 0, 1, 0.4, 1]])
    assert st != 0


@pytest.mark.gpu
def test_prepare_frame_matches_oracle(gf):
    """Three frames of outflows then inflows on a 32^3 scene with a solid
    sphere under the second inflow (its emitted positions in solid cells are
    dropped); the particles after each frame hook equal the oracle's."""
    from gpufluid_b200 import scene
    s = gf.FlipSolver3D(32, 32, 32, transfer_mode="apic")
    s.add_solid_from_sdf(scene.sdf_sphere(s.cell_centers_np(), (0.7, 0.55, 0.7), 0.12))
    s.seed_box((0.0, 0.0, 0.0), (0.6, 0.5, 1.0))
    for lo, hi, a, b in OUT_BOXES:
        s.add_outflow(OutflowBox(lo=lo, hi=hi, frame_start=a, frame_end=b))
    for b in IN_BOXES:
        s.add_inflow(InflowBox(**b))
    pos, vel = s.get_particles()
    rng = np.random.default_rng(0)
    marker = s.marker.numpy()
    for f in range(3):
        s.prepare_frame(f, 1.0 / 24.0)
        pos, vel = orc.prepare_frame(pos, vel, OUT_BOXES, IN_BOXES, f, 1.0 / 24.0, rng,
                                     marker, s.dx)
        gp, gv = s.get_particles()
        assert np.array_equal(gp, pos) and np.array_equal(gv, vel), f
    # the same generator stream as the golden emission: frame 2 put some
    # positions into the sphere, so the solid filter was exercised
    g = _gold()
    assert (~orc.solid_filter(g["emit_pos"][g["emit_frame"] == 2], marker, s.dx)).any()
    assert np.count_nonzero(s.affine_C.numpy()) == 0
    s.step(1.0 / 480.0, pressure_iters=20)
    assert np.isfinite(s.pos.numpy()).all()
