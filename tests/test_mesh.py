"""Surface mesh after the substeps (src/gpufluid/meshing/surface.py:14-466,
src/gpufluid/io/ply.py).

CPU: the oracle's density field (oracle/mesh.py) against the reference
kernels' own outputs on the sequential Warp stand-in
(tests/golden/mesh/density.npz, made by tests/golden/make_mesh_golden.py),
bit for bit; the oracle's iso-surface on analytic fields (closed, consistently
oriented, enclosed volume); the PLY writer's byte layout.

GPU: ``MeshExtractor`` through ``gf_mesher_*``:
* density: within float32 atomic-order tolerance of the golden vectors, and
  bit-exact with the oracle on particles whose splat weights are dyadic (every
  order of the float adds then gives the same sum, so the blur and margin
  are checked exactly);
* iso-surface: vertices and triangles bit-exact with the oracle's on the same
  field (ragged grids, ties at the iso level, boundary-touching surfaces);
  size-independent properties at 256^3 (closed, each directed edge once,
  enclosed volume of a sphere);
* the whole extract on a solver's particles, and the CLI's mesh/ output.
"""
import os

import numpy as np
import pytest

from gpufluid_b200.config import BlockError
from gpufluid_b200.mesh import read_ply, write_ply
from oracle import mesh as om

GOLD = os.path.join(os.path.dirname(__file__), "golden", "mesh", "density.npz")
SHAPE = (16, 12, 10)


def _gold():
    return dict(np.load(GOLD))


def _cases(g):
    for c in range(5):
        cubic, passes, margin, radius = g[f"case_{c}"]
        yield (c, "cubic" if cubic else "trilinear", int(passes), int(margin), float(radius))


def _sphere(n, centre, radius, shape=None):
    shape = shape or (n, n, n)
    i, j, k = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
    r = np.sqrt((i - centre[0]) ** 2 + (j - centre[1]) ** 2 + (k - centre[2]) ** 2)
    return (radius - r).astype(np.float32)


# ------------------------------------------------------------------- CPU
def _sdf_cases(g):
    for c in range(2):
        passes, r_cells, s_cells = g[f"sdf_case_{c}"]
        yield c, int(passes), float(r_cells), float(s_cells)


def test_oracle_density_matches_reference():
    g = _gold()
    for c, method, passes, margin, radius in _cases(g):
        d = om.density_field(g["pos"], SHAPE, float(g["dx"]), passes, margin, method, radius)
        assert np.array_equal(d, g[f"density_{c}"]), (c, method)
    for c, passes, r_cells, s_cells in _sdf_cases(g):
        d = om.density_field(g["sdf_pos"], SHAPE, float(g["dx"]), passes, 0, "sdf",
                             sdf_particle_radius_cells=r_cells, sdf_search_radius_cells=s_cells)
        assert np.array_equal(d, g[f"sdf_{c}"]), c


def test_oracle_iso_surface_closed_sphere():
    n, dx = 40, 1.0 / 40
    v, t = om.iso_surface(_sphere(n, (19.3, 20.1, 18.7), 10.0), 0.0, dx)
    nb, once = om.boundary_edges(t)
    assert nb == 0 and once  # closed, each directed edge used once
    edges = np.unique(np.sort(np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]]), 1),
                      axis=0)
    assert len(v) - len(edges) + len(t) == 2  # Euler characteristic of a sphere
    vol = om.mesh_volume(v, t)
    exact = 4.0 / 3.0 * np.pi * (10 * dx) ** 3
    assert 0.98 * exact < vol < exact  # outward-facing, chordal shrink < 2 %
    # the axis-edge vertices (families 1, 2, 4) lie on the sphere
    r = np.linalg.norm(v / dx - np.float32([19.3, 20.1, 18.7]), axis=1)
    assert np.abs(r - 10.0).max() < 0.1


def test_marching_cubes_table_matches_oracle():
    """The library's generated case table (gf_marching_cubes_table, host code,
    no device) equals the oracle's per-case loop tracing; at most 5 triangles
    per case, none for the empty and the full cube, and a case and its
    complement cross the same edges."""
    import ctypes
    from gpufluid_b200 import _lib
    L = _lib.load()
    edges, ntri, tri = np.zeros(24, np.uint8), np.zeros(256, np.uint8), np.zeros(3840, np.uint8)
    assert L.gf_marching_cubes_table(edges.ctypes.data, ntri.ctypes.data, tri.ctypes.data) == 0
    assert [tuple(int(x) for x in e) for e in edges.reshape(12, 2)] == om.MC_EDGES
    tri = tri.reshape(256, 15)
    for cm in range(256):
        want = om.mc_case(cm)
        assert ntri[cm] == len(want), cm
        assert [tuple(int(x) for x in tri[cm][3 * q:3 * q + 3]) for q in range(len(want))] == want
        used = {e for t in want for e in t}
        assert used == {e for t in om.mc_case(255 - cm) for e in t}
    assert ntri.max() == 5 and ntri[0] == 0 and ntri[255] == 0
    assert L.gf_marching_cubes_table(None, ntri.ctypes.data, tri.ctypes.data) == _lib.GF_INVALID_ARG


def test_oracle_marching_cubes_closed_sphere_and_orientation():
    n, dx = 40, 1.0 / 40
    f = _sphere(n, (19.3, 20.1, 18.7), 10.0)
    v, t = om.iso_surface_mc(f, 0.0, dx)
    nb, once = om.boundary_edges(t)
    assert nb == 0 and once
    edges = np.unique(np.sort(np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]]), 1),
                      axis=0)
    assert len(v) - len(edges) + len(t) == 2
    exact = 4.0 / 3.0 * np.pi * (10 * dx) ** 3
    assert 0.98 * exact < om.mesh_volume(v, t) < exact
    r = np.linalg.norm(v / dx - np.float32([19.3, 20.1, 18.7]), axis=1)
    assert np.abs(r - 10.0).max() < 0.1
    # the tetrahedra's surface of the same field: the same axis-edge vertices
    vt, tt = om.iso_surface(f, 0.0, dx)
    assert len(vt) > len(v) and len(tt) > len(t)
    assert {tuple(x) for x in v} <= {tuple(x) for x in vt}
    # noise: every ambiguous face occurs; the surface is still closed away
    # from the grid walls and consistently oriented
    g = np.random.default_rng(3).normal(size=(20, 18, 22)).astype(np.float32)
    g[[0, -1]] = -1.0
    g[:, [0, -1]] = -1.0
    g[:, :, [0, -1]] = -1.0
    v, t = om.iso_surface_mc(g, 0.0, 1.0)
    nb, once = om.boundary_edges(t)
    assert nb == 0 and once
    assert om.mesh_volume(v, t) > 0


def test_oracle_iso_surface_open_and_inverted():
    """A slab touching the grid walls is open; the complement field gives the
    same vertices with every triangle reversed."""
    f = np.zeros((9, 7, 8), np.float32)
    f[:, :4] = 1.0
    v, t = om.iso_surface(f, 0.5, 0.1)
    nb, once = om.boundary_edges(t)
    assert nb > 0 and once
    assert np.allclose(v[:, 1], 0.35)
    v2, t2 = om.iso_surface(-f, -0.5, 0.1)
    # >= iso flips which side is inside: the crossing set is the same, but
    # the vertex sits at the same t only when no value equals the level
    assert len(v2) == len(v)
    assert om.mesh_volume(v, t) == pytest.approx(-om.mesh_volume(v2, t2))


def test_oracle_iso_surface_empty_and_degenerate():
    assert om.iso_surface(np.zeros((5, 5, 5), np.float32), 0.5, 0.1)[0].shape == (0, 3)
    assert om.iso_surface(np.ones((5, 5, 5), np.float32), 0.5, 0.1)[1].shape == (0, 3)
    assert om.iso_surface(np.eye(4, dtype=np.float32)[None, :1], 0.5, 0.1)[0].shape == (0, 3)


def test_ply_layout(tmp_path):
    """io/ply.py:10-90: ASCII header, float32 xyz, then per face uchar 3 + 3 int32."""
    v = np.float32([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1.5]])
    f = np.int32([[0, 1, 2], [0, 3, 1]])
    p = tmp_path / "m.ply"
    write_ply(p, v, f)
    raw = p.read_bytes()
    head = (b"ply\nformat binary_little_endian 1.0\nelement vertex 4\nproperty float x\n"
            b"property float y\nproperty float z\nelement face 2\n"
            b"property list uchar int vertex_indices\nend_header\n")
    assert raw.startswith(head)
    body = raw[len(head):]
    assert len(body) == 4 * 12 + 2 * 13
    assert body[:48] == v.astype("<f4").tobytes()
    assert body[48] == 3 and np.frombuffer(body[49:61], "<i4").tolist() == [0, 1, 2]
    rv, rf = read_ply(p)
    assert np.array_equal(rv, v) and np.array_equal(rf, f)
    # colours add uchar rgb after xyz; the placeholder is an empty mesh
    write_ply(p, v, f, vertex_colors=np.full((4, 3), 300))
    assert b"property uchar red\nproperty uchar green\nproperty uchar blue\n" in p.read_bytes()
    assert len(p.read_bytes().split(b"end_header\n")[1]) == 4 * 15 + 2 * 13
    write_ply(p, np.zeros((0, 3)), np.zeros((0, 3)))
    assert b"element vertex 0\n" in p.read_bytes() and b"element face 0\n" in p.read_bytes()
    with pytest.raises(BlockError):
        write_ply(p, np.zeros((3, 2)), f)
    with pytest.raises(BlockError):
        write_ply(p, v, f, vertex_colors=np.zeros((3, 3)))


def test_mesh_options_outside_build_are_refused():
    from gpufluid_b200.cli import check_mesh_options
    from gpufluid_b200.config import OutputCfg
    check_mesh_options(OutputCfg())
    check_mesh_options(OutputCfg(mesh_method="cubic"))
    check_mesh_options(OutputCfg(mesh=False, mesh_method="marching"))
    check_mesh_options(OutputCfg(mesh_smooth_passes=2))
    check_mesh_options(OutputCfg(mesh_method="sdf"))
    for kw in (dict(mesh_method="marching"),
               dict(mesh_smooth_passes=2, mesh_smooth_method="cotan"),
               dict(decimate_ratio=0.5)):
        with pytest.raises(BlockError) as e:
            check_mesh_options(OutputCfg(**kw))
        assert e.value.block_id == "C7.1"


# ------------------------------------------------------------------- GPU
def _extractor(shape, dx):
    from gpufluid_b200.mesh import MeshExtractor
    return MeshExtractor(*shape, dx)


@pytest.mark.gpu
def test_density_matches_reference(gf):
    g = _gold()
    ex = _extractor(SHAPE, float(g["dx"]))
    for c, method, passes, margin, radius in _cases(g):
        ex.density(g["pos"], passes, margin, method, radius)
        d = ex.dens.cpu().numpy()
        ref = g[f"density_{c}"]
        # float32 atomics add in arrival order: a few ulp of the largest value
        np.testing.assert_allclose(d, ref, rtol=0, atol=4e-6 * float(ref.max()), err_msg=str(c))
        assert np.array_equal(d == 0, ref == 0)


@pytest.mark.gpu
def test_sdf_density_matches_reference(gf):
    """k_sdf_field on the stand-in, bit for bit: a minimum does not depend on
    the order in which particles are met."""
    g = _gold()
    ex = _extractor(SHAPE, float(g["dx"]))
    for c, passes, r_cells, s_cells in _sdf_cases(g):
        ex.density(g["sdf_pos"], passes, 0, "sdf", sdf_particle_radius_cells=r_cells,
                   sdf_search_radius_cells=s_cells)
        assert np.array_equal(ex.dens.cpu().numpy(), g[f"sdf_{c}"]), c
    ex.density(np.zeros((0, 3), np.float32), 0, 0, "sdf")  # no particles: R - r everywhere
    d = ex.dens.cpu().numpy()
    assert np.all(d == d.flat[0]) and d.flat[0] > 0


@pytest.mark.gpu
@pytest.mark.parametrize("passes,margin", [(0, 0), (1, 0), (2, 0), (2, 3), (0, 2), (3, 1)])
def test_density_bit_exact_on_dyadic_splat(gf, passes, margin):
    """dx = 1/16 and positions on a quarter-cell lattice: every splat weight is
    a multiple of 1/64, so the atomic sums are exact in any order."""
    rng = np.random.default_rng(passes * 10 + margin)
    shape, dx = (40, 33, 29), 1.0 / 16.0
    q = rng.integers(-8, 4 * np.array(shape) + 8, size=(60000, 3))
    pos = (q.astype(np.float32) * np.float32(0.25) * np.float32(dx)).astype(np.float32)
    ex = _extractor(shape, dx)
    ex.density(pos, passes, margin)
    d = ex.dens.cpu().numpy()
    assert np.array_equal(d, om.density_field(pos, shape, dx, passes, margin))


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["marching_cubes", "marching_tetrahedra"])
@pytest.mark.parametrize("case", ["sphere", "noise", "ties", "ragged", "wall", "tiny", "flat"])
def test_iso_surface_bit_exact(gf, case, method):
    import torch
    rng = np.random.default_rng(5)
    dx, iso = 0.05, 0.0
    if case == "sphere":
        f = _sphere(48, (23.4, 22.9, 24.2), 15.3)
    elif case == "noise":
        f = rng.normal(size=(31, 27, 35)).astype(np.float32)
    elif case == "ties":  # many values exactly at the level (t = 0 vertices)
        f = rng.integers(-2, 3, size=(24, 20, 22)).astype(np.float32)
    elif case == "ragged":
        f = _sphere(0, (30.2, 6.1, 17.7), 11.6, shape=(61, 13, 37))
    elif case == "wall":  # the surface runs into the grid boundary
        f = _sphere(0, (0.0, 10.0, 10.0), 8.5, shape=(20, 20, 20))
    elif case == "tiny":
        f = np.float32([[[1, -1], [-1, 1]], [[-1, 1], [1, -1]]])
    else:  # one cell thick: no cube, no surface
        f = rng.normal(size=(1, 9, 9)).astype(np.float32)
    ex = _extractor(f.shape, dx)
    ex.surface_method = method
    v, t = ex.surface(iso, field=torch.from_numpy(f).cuda())
    ov, ot = (om.iso_surface_mc if method == "marching_cubes" else om.iso_surface)(f, iso, dx)
    if len(ot) == 0:
        assert v is None and t is None
        return
    assert np.array_equal(v, ov) and np.array_equal(t, ot)
    assert ex.n_verts == len(ov) and ex.n_tris == len(ot)
    if method == "marching_cubes":
        # the vertices are the axis-edge subset of the tetrahedra's, bit for bit
        ex.surface_method = "marching_tetrahedra"
        vt, _ = ex.surface(iso, field=torch.from_numpy(f).cuda())
        key = lambda a: a.view(np.uint32).view([("x", "u4"), ("y", "u4"), ("z", "u4")]).ravel()  # noqa: E731
        assert np.isin(key(v), key(vt)).all()
        assert len(t) <= 5 * np.prod(np.array(f.shape) - 1)


@pytest.mark.gpu
def test_iso_surface_properties_at_256(gf):
    """A 256^3 field (16.7 M nodes, 65,536 node blocks: the offsets scan runs
    in 64 chunks) holding a sphere and a wall-touching slab."""
    import torch
    n, dx = 256, 1.0 / 256
    i = torch.arange(n, device="cuda", dtype=torch.float32)
    I, J, K = torch.meshgrid(i, i, i, indexing="ij")
    sph = 60.0 - torch.sqrt((I - 127.3) ** 2 + (J - 140.6) ** 2 + (K - 120.2) ** 2)
    f = torch.maximum(sph, 20.5 - J)  # plus a floor slab y < 20.5
    ex = _extractor((n, n, n), dx)
    v, t = ex.surface(0.0, field=f.contiguous())
    assert ex.surface_method == "marching_cubes"
    assert v is not None and t.min() >= 0 and t.max() < len(v)
    nb, once = om.boundary_edges(t)
    assert once  # consistent orientation across all cubes
    # boundary edges only where the slab meets the grid walls
    e = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]])
    und, cnt = np.unique(np.sort(e, 1), axis=0, return_counts=True)
    bv = v[np.unique(und[cnt == 1])]
    on_wall = ((bv <= 1e-6) | (bv >= (n - 1) * dx - 1e-6)).any(axis=1)
    assert nb > 0 and on_wall.all()
    sel = v[:, 1] > 30 * dx  # the sphere's vertices
    r = np.linalg.norm(v[sel] / dx - np.float32([127.3, 140.6, 120.2]), axis=1)
    assert np.abs(r - 60.0).max() < 0.05
    # the sphere alone: closed, Euler characteristic 2, enclosed volume
    v, t = ex.surface(0.0, field=sph.contiguous())
    nb, once = om.boundary_edges(t)
    assert nb == 0 and once
    edges = np.unique(np.sort(np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]]), 1),
                      axis=0)
    assert len(v) - len(edges) + len(t) == 2
    exact = 4.0 / 3.0 * np.pi * (60.0 * dx) ** 3
    assert 0.995 * exact < om.mesh_volume(v, t) < exact


@pytest.mark.gpu
def test_extract_on_solver_particles(gf):
    """Dam break at 48^3 after a few substeps: the extraction's field is within
    atomic tolerance of the oracle's field; its surface is bit-exact with the
    oracle's surface of that same field; options and empty inputs."""
    import torch
    s = gf.FlipSolver3D(48, 48, 48, transfer_mode="apic")
    s.seed_box((0.05, 0.05, 0.05), (0.45, 0.6, 0.5))
    for _ in range(4):
        s.step(1.0 / 240.0, pressure_iters=80, pressure_solver="pcg")
    pos = s.pos.numpy()
    ex = _extractor((48, 48, 48), s.dx)
    v, t = ex.extract(s.pos, iso_level=0.6, smooth_passes=2, wall_margin_cells=1)
    d = ex.dens.cpu().numpy()
    ref = om.density_field(pos, (48, 48, 48), s.dx, 2, 1)
    np.testing.assert_allclose(d, ref, rtol=0, atol=4e-6 * float(ref.max()))
    ov, ot = om.iso_surface_mc(d, 0.6, s.dx)
    assert np.array_equal(v, ov) and np.array_equal(t, ot)
    assert om.boundary_edges(t)[0] == 0  # the wall margin closes the surface
    assert om.mesh_volume(v, t) > 0
    # torch tensors on the device are taken as they are
    v2, t2 = ex.extract(torch.from_numpy(pos).cuda(), iso_level=0.6, smooth_passes=2,
                        wall_margin_cells=1)
    assert len(v2) == len(v)
    assert ex.extract(np.zeros((0, 3), np.float32)) == (None, None)
    assert ex.extract(None) == (None, None)
    far = np.full((10, 3), 0.5, np.float32)  # density 10 at most: below iso 20
    assert ex.extract(far, iso_level=20.0) == (None, None)
    with pytest.raises(ValueError):
        ex.extract(pos, mesh_method="marching")
    # the "sdf" method: signed distance to the nearest particle (no atomics
    # of float sums: bit-exact), surface at its zero level, inside below it
    vd, td = ex.extract(s.pos, mesh_method="sdf", smooth_passes=1)
    dd = ex.dens.cpu().numpy()
    refd = om.density_field(pos, (48, 48, 48), s.dx, 1, 0, "sdf")
    assert np.array_equal(dd, refd)
    ov, ot = om.iso_surface_mc(dd, 0.0, s.dx, below=True)
    assert np.array_equal(vd, ov) and np.array_equal(td, ot)
    assert om.mesh_volume(vd, td) > 0  # faces outward from the fluid
    with pytest.raises(ValueError):
        ex.extract(pos, mesh_smooth_passes=1, mesh_smooth_method="cotan")
    # Taubin smoothing on the device after extraction equals the oracle's
    # smoothing of the unsmoothed surface
    vs, ts = ex.extract(s.pos, iso_level=0.6, smooth_passes=2, wall_margin_cells=1,
                        mesh_smooth_passes=2)
    d2 = ex.dens.cpu().numpy()
    ov, ot = om.iso_surface_mc(d2, 0.6, s.dx)
    assert np.array_equal(ts, ot) and np.array_equal(vs, om.smooth(ov, ot, "taubin", 2))
    with pytest.raises(ValueError):
        ex.extract(pos, decimate_ratio=0.5)
    vc, tc = ex.extract(s.pos, iso_level=3.0, mesh_method="cubic", cubic_radius_cells=2.0)
    dc = ex.dens.cpu().numpy()
    refc = om.density_field(pos, (48, 48, 48), s.dx, 2, 0, "cubic", 2.0)
    np.testing.assert_allclose(dc, refc, rtol=0, atol=4e-6 * float(refc.max()))
    ov, ot = om.iso_surface_mc(dc, 3.0, s.dx)
    assert np.array_equal(vc, ov) and np.array_equal(tc, ot)
    assert ex.launches > 0


def test_oracle_smoothing_matches_reference():
    g = dict(np.load(os.path.join(os.path.dirname(GOLD), "smoothing.npz")))
    for c in (0, 1):
        v, t = g[f"verts_{c}"], g[f"faces_{c}"]
        assert np.array_equal(om.smooth(v, t, "taubin", 2), g[f"taubin_{c}"])
        assert np.array_equal(om.smooth(v, t, "laplacian", 3, 0.4), g[f"laplacian_{c}"])


@pytest.mark.gpu
def test_smoothing_matches_reference(gf):
    """smoothing.py's functions, bit for bit: the device runs the float64
    Laplacian in the reference's order of operations."""
    from gpufluid_b200.mesh import smooth_laplacian, smooth_taubin
    g = dict(np.load(os.path.join(os.path.dirname(GOLD), "smoothing.npz")))
    for c in (0, 1):
        v, t = g[f"verts_{c}"], g[f"faces_{c}"]
        assert np.array_equal(smooth_taubin(v, t, passes=2), g[f"taubin_{c}"])
        assert np.array_equal(smooth_laplacian(v, t, passes=3, lam=0.4), g[f"laplacian_{c}"])
    # isolated vertices and a larger mesh
    v = np.concatenate([g["verts_0"], np.float32([[9.0, 9.0, 9.0]])])
    assert np.array_equal(smooth_laplacian(v, g["faces_0"], passes=2),
                          om.smooth(v, g["faces_0"], "laplacian", 2))
    f = _sphere(96, (47.3, 45.9, 48.2), 30.5)
    ov, ot = om.iso_surface(f, 0.0, 1.0 / 96)
    assert np.array_equal(smooth_taubin(ov, ot, passes=3), om.smooth(ov, ot, "taubin", 3))
    assert smooth_taubin(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.int32)).shape == (0, 3)


@pytest.mark.gpu
def test_particles_to_mesh(gf):
    from gpufluid_b200.mesh import particles_to_mesh
    rng = np.random.default_rng(2)
    pos = (np.float32([0.5, 0.5, 0.5]) + rng.normal(0, 0.06, (20000, 3))).astype(np.float32)
    v, t = particles_to_mesh(pos, 32, 32, 32, 1.0 / 32, iso_level=0.5, smooth_passes=2)
    d = om.density_field(pos, (32, 32, 32), 1.0 / 32, 2, 0)
    assert v is not None and om.mesh_volume(v, t) > 0
    # the blob's extent agrees with the oracle's field to within a cell
    ov, _ = om.iso_surface_mc(d, 0.5, 1.0 / 32)
    assert abs(len(v) - len(ov)) <= 0.01 * len(ov)
