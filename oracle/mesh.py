"""CPU oracle for the surface mesh after the substeps -- TEST INFRASTRUCTURE ONLY.

Only ``tests/`` (and the bench's CPU leg) may import this module, as the
checker; the product (``gpufluid_b200``) never does.

NumPy restatement of the reference's density field
(src/gpufluid/meshing/surface.py):

* ``splat_trilinear`` -- ``k_density_scatter`` (:14-43): f = p/dx - 0.5,
  corner weights (1-s | s) per axis, w = (wx*wy)*wz, float32 adds in thread
  (particle) order, corners (di, dj, dk) ascending;
* ``splat_cubic``     -- ``k_cubic_scatter`` (:53-84) with the host's
  radius arithmetic (:376-382);
* ``box_blur``        -- ``k_box_blur_3d`` (primitives/gridmath.py:103-121):
  float32 sum of the in-grid 3x3x3 neighbours (di, dj, dk ascending) divided
  by their count;
* ``zero_walls``      -- ``k_mc_zero_walls`` (:179-193);
* ``sdf_field``       -- ``k_sdf_field`` (:100-122) with the host radii;
* ``density_field``   -- the order of ``MeshExtractor.extract`` (:388-425);
* ``smooth``          -- ``smooth_laplacian`` / ``smooth_taubin``
  (meshing/smoothing.py:22-72).

Parity pin: ``tests/golden/mesh/density.npz`` holds the reference kernels' own
outputs run on the sequential Warp stand-in, and ``tests/golden/mesh/smoothing.npz``
the reference's smoothing functions' outputs (NumPy + SciPy, run directly)
(``tests/golden/make_mesh_golden.py``); ``tests/test_mesh.py`` checks this
restatement against them.

The iso-surface step of the reference is third-party code (scikit-image's
``marching_cubes`` below 64^3, Warp's ``MarchingCubes`` from 64^3,
surface.py:286-351); neither is installed, so that step is unpinned.  The
library's own methods are restated here independently of the CUDA code, for
bit-exact checks of the GPU extraction on the same field:

* ``iso_surface_mc`` -- marching cubes (Lorensen & Cline 1987): vertices on
  the axis edges at the linear crossing; each cube's triangles traced per
  case on the fly -- face segments (an ambiguous face cuts off its inside
  corners), loops oriented with the inside on their right as seen from outside
  the cube (decided here with floating-point midpoint geometry, where the CUDA
  table generator uses doubled integer coordinates), each loop listed from its
  lowest edge and fanned from its first vertex whose diagonals all leave the
  cube's faces;
* ``iso_surface`` -- marching tetrahedra on the Kuhn split of each cube
  (orientation from integer determinants of the tetrahedra's corners rather
  than from the permutation parity); its axis-edge vertices are the
  marching-cubes ones.
"""
from __future__ import annotations

import math

import numpy as np

F32 = np.float32


def splat_trilinear(pos, shape, dx):
    nx, ny, nz = shape
    dens = np.zeros(nx * ny * nz, F32)
    if len(pos) == 0:
        return dens.reshape(shape)
    pos = np.asarray(pos, F32)
    f = pos / F32(dx) - F32(0.5)
    i0 = np.floor(f).astype(np.int64)
    s = f - i0.astype(F32)
    idx, w = [], []
    for a in (0, 1):
        wx = (F32(1.0) - s[:, 0]) if a == 0 else s[:, 0]
        for b in (0, 1):
            wy = (F32(1.0) - s[:, 1]) if b == 0 else s[:, 1]
            for e in (0, 1):
                wz = (F32(1.0) - s[:, 2]) if e == 0 else s[:, 2]
                ii, jj, kk = i0[:, 0] + a, i0[:, 1] + b, i0[:, 2] + e
                ok = (ii >= 0) & (ii < nx) & (jj >= 0) & (jj < ny) & (kk >= 0) & (kk < nz)
                idx.append(np.where(ok, (ii * ny + jj) * nz + kk, -1))
                w.append((wx * wy) * wz)
    idx = np.stack(idx, 1).reshape(-1)  # particle-major, then corner
    w = np.stack(w, 1).reshape(-1).astype(F32)
    keep = idx >= 0
    np.add.at(dens, idx[keep], w[keep])
    return dens.reshape(shape)


def splat_cubic(pos, shape, dx, radius_cells):
    nx, ny, nz = shape
    dens = np.zeros(shape, F32)
    r_world = float(radius_cells) * float(dx)
    inv = F32(1.0 / (r_world * r_world))
    half = int(math.ceil(radius_cells)) + 1
    dx32 = F32(dx)
    for p in np.asarray(pos, F32):
        c = np.floor(p / dx32 - F32(0.5)).astype(np.int64)
        lo = np.maximum(0, c - half)
        hi = np.minimum([nx, ny, nz], c + half + 1)
        if (hi <= lo).any():
            continue
        ii = np.arange(lo[0], hi[0])
        jj = np.arange(lo[1], hi[1])
        kk = np.arange(lo[2], hi[2])
        ddx = (ii.astype(F32) + F32(0.5)) * dx32 - p[0]
        ddy = (jj.astype(F32) + F32(0.5)) * dx32 - p[1]
        ddz = (kk.astype(F32) + F32(0.5)) * dx32 - p[2]
        d_sq = (ddx[:, None, None] * ddx[:, None, None] + ddy[None, :, None] * ddy[None, :, None]
                ) + ddz[None, None, :] * ddz[None, None, :]
        r_sq = d_sq * inv
        om = F32(1.0) - r_sq
        val = (om * om) * om
        blk = dens[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]]
        blk += np.where(r_sq < F32(1.0), val, F32(0.0))
    return dens


def box_blur(src):
    src = np.asarray(src, F32)
    nx, ny, nz = src.shape
    pad = np.zeros((nx + 2, ny + 2, nz + 2), F32)
    pad[1:-1, 1:-1, 1:-1] = src
    one = np.zeros_like(pad)
    one[1:-1, 1:-1, 1:-1] = 1.0
    s = np.zeros(src.shape, F32)
    n = np.zeros(src.shape, F32)
    for di in (-1, 0, 1):
        for dj in (-1, 0, 1):
            for dk in (-1, 0, 1):
                sl = (slice(1 + di, nx + 1 + di), slice(1 + dj, ny + 1 + dj),
                      slice(1 + dk, nz + 1 + dk))
                s = s + pad[sl]  # out-of-grid neighbours add +0.0: exact
                n = n + one[sl]
    return (s / n).astype(F32)


def zero_walls(d, margin):
    d = np.array(d, F32, copy=True)
    if margin > 0:
        m = int(margin)
        d[:m], d[-m:] = 0, 0
        d[:, :m], d[:, -m:] = 0, 0
        d[:, :, :m], d[:, :, -m:] = 0, 0
    return d


def sdf_field(pos, shape, dx, particle_radius_cells=1.0, search_radius_cells=4.0):
    """``k_sdf_field`` (:100-122) with the host's radii (:405-420): phi =
    sqrt(min(R^2, d^2 to the nearest particle)) - r at the cell centres, d =
    centre - p, d^2 = (dx dx + dy dy) + dz dz in float32."""
    nx, ny, nz = shape
    R = F32(float(search_radius_cells) * float(dx))
    r = F32(float(particle_radius_cells) * float(dx))
    r2 = R * R
    best = np.full(shape, r2, F32)
    dx32 = F32(dx)
    rc = int(math.ceil(float(R) / float(dx))) + 2
    for p in np.asarray(pos, F32):
        c = np.floor(p / dx32).astype(np.int64)
        lo = np.maximum(0, c - rc)
        hi = np.minimum([nx, ny, nz], c + rc + 1)
        if (hi <= lo).any():
            continue
        ddx = (np.arange(lo[0], hi[0]).astype(F32) + F32(0.5)) * dx32 - p[0]
        ddy = (np.arange(lo[1], hi[1]).astype(F32) + F32(0.5)) * dx32 - p[1]
        ddz = (np.arange(lo[2], hi[2]).astype(F32) + F32(0.5)) * dx32 - p[2]
        d2 = (ddx[:, None, None] * ddx[:, None, None] + ddy[None, :, None] * ddy[None, :, None]
              ) + ddz[None, None, :] * ddz[None, None, :]
        blk = best[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]]
        np.minimum(blk, d2, out=blk)
    return (np.sqrt(best) - r).astype(F32)


def density_field(pos, shape, dx, smooth_passes=2, wall_margin_cells=0,
                  mesh_method="trilinear", cubic_radius_cells=2.0,
                  sdf_particle_radius_cells=1.0, sdf_search_radius_cells=4.0):
    if mesh_method == "trilinear":
        d = splat_trilinear(pos, shape, dx)
    elif mesh_method == "cubic":
        d = splat_cubic(pos, shape, dx, cubic_radius_cells)
    elif mesh_method == "sdf":
        d = sdf_field(pos, shape, dx, sdf_particle_radius_cells, sdf_search_radius_cells)
        for _ in range(smooth_passes):
            d = box_blur(d)
        return d  # no wall margin for signed distances (surface.py:422-425)
    else:
        raise ValueError(mesh_method)
    for _ in range(smooth_passes):
        d = box_blur(d)
    return zero_walls(d, wall_margin_cells)


# ---- iso-surface: marching tetrahedra on the Kuhn split ------------------
# Cube corner b = (bit0: +x, bit1: +y, bit2: +z).  The six tetrahedra share
# corners 0 and 7 and follow the axis orders of the six permutations.
_AXIS_ORDERS = [(1, 2), (1, 4), (2, 1), (2, 4), (4, 1), (4, 2)]


def _corner_xyz(b):
    return np.array([b & 1, (b >> 1) & 1, (b >> 2) & 1], np.int64)


def _det(a, b, c):
    return int(np.dot(a, np.cross(b, c)))


def iso_surface(dens, iso, dx, below=False):
    """(verts (V,3) float32, tris (T,3) int32) of {dens >= iso} ({dens <= iso}
    with ``below``); vertices ordered by (node, edge family 1..7), triangles by
    (cube, tet, triangle)."""
    d = np.asarray(dens, F32)
    nx, ny, nz = d.shape
    if nx < 2 or ny < 2 or nz < 2:  # no cube: no surface
        return np.zeros((0, 3), F32), np.zeros((0, 3), np.int32)
    iso32, dx32 = F32(iso), F32(dx)
    inside = d <= iso32 if below else d >= iso32
    cross = np.zeros((nx, ny, nz, 8), bool)
    vpos = np.zeros((nx, ny, nz, 8, 3), F32)
    gi, gj, gk = np.meshgrid(np.arange(nx, dtype=F32), np.arange(ny, dtype=F32),
                             np.arange(nz, dtype=F32), indexing="ij")
    for b in range(1, 8):
        ox, oy, oz = b & 1, (b >> 1) & 1, (b >> 2) & 1
        lo = (slice(0, nx - ox), slice(0, ny - oy), slice(0, nz - oz))
        hi = (slice(ox, nx), slice(oy, ny), slice(oz, nz))
        c = inside[lo] != inside[hi]
        cross[lo + (b,)] = c
        with np.errstate(divide="ignore", invalid="ignore"):
            t = (iso32 - d[lo]) / (d[hi] - d[lo])
        for axis, (g, o) in enumerate(((gi, ox), (gj, oy), (gk, oz))):
            base = g[lo]
            vpos[lo + (b, axis)] = ((base + t) if o else base) * dx32
    flat = cross.reshape(-1)
    verts = vpos.reshape(-1, 3)[flat]
    vid = np.full(flat.shape, -1, np.int64)
    vid[flat] = np.arange(int(flat.sum()))
    vid = vid.reshape(nx, ny, nz, 8)
    if len(verts) == 0:
        return verts.astype(F32), np.zeros((0, 3), np.int32)

    cx, cy, cz = nx - 1, ny - 1, nz - 1
    ci, cj, ck = np.meshgrid(np.arange(cx), np.arange(cy), np.arange(cz), indexing="ij")
    cube_key = (ci * ny + cj) * nz + ck   # node index of the cube's lower corner

    def corner_inside(b):
        x, y, z = _corner_xyz(b)
        return inside[x:x + cx, y:y + cy, z:z + cz]

    def edge_vid(lo_b, hi_b, sel):
        x, y, z = _corner_xyz(lo_b)
        return vid[x:x + cx, y:y + cy, z:z + cz, hi_b ^ lo_b][sel]

    keys, tris = [], []
    for t, (a, b2) in enumerate(_AXIS_ORDERS):
        cs = [0, a, a | b2, 7]
        xyz = [_corner_xyz(c) for c in cs]
        ins = [corner_inside(c) for c in cs]
        code = ins[0] * 1 + ins[1] * 2 + ins[2] * 4 + ins[3] * 8
        for m in range(1, 15):
            sel = code == m
            if not sel.any():
                continue
            members = [v for v in range(4) if (m >> v) & 1]
            if len(members) in (1, 3):
                lone_in = len(members) == 1
                l = members[0] if lone_in else [v for v in range(4) if not (m >> v) & 1][0]
                oth = [v for v in range(4) if v != l]
                e = [edge_vid(cs[min(l, o)], cs[max(l, o)], sel) for o in oth]
                det = _det(*(xyz[o] - xyz[l] for o in oth))
                away = det > 0   # triple (oth ascending) faces away from corner l
                tri = np.stack([e[0], e[1], e[2]] if away == lone_in else [e[0], e[2], e[1]], 1)
                keys.append(cube_key[sel] * 12 + t * 2)
                tris.append(tri)
            else:
                p0, p1 = members
                q0, q1 = [v for v in range(4) if not (m >> v) & 1]
                E = lambda u, x: edge_vid(cs[min(u, x)], cs[max(u, x)], sel)  # noqa: E731
                cyc = [E(p0, q0), E(p0, q1), E(p1, q1), E(p1, q0)]
                if _det(xyz[p1] - xyz[p0], xyz[q0] - xyz[p0], xyz[q1] - xyz[p0]) < 0:
                    cyc = [cyc[0], cyc[3], cyc[2], cyc[1]]
                keys.append(cube_key[sel] * 12 + t * 2)
                tris.append(np.stack([cyc[0], cyc[1], cyc[2]], 1))
                keys.append(cube_key[sel] * 12 + t * 2 + 1)
                tris.append(np.stack([cyc[0], cyc[2], cyc[3]], 1))
    if not keys:
        return verts.astype(F32), np.zeros((0, 3), np.int32)
    keys = np.concatenate(keys)
    tris = np.concatenate(tris)
    order = np.argsort(keys, kind="stable")
    return verts.astype(F32), tris[order].astype(np.int32)


# ---- marching cubes ----------------------------------------------------------
# Corner c of a cube: bit 0 +x, bit 1 +y, bit 2 +z.  Edge e: along x for
# e < 4, y for e < 8, z otherwise, from the (e % 4)-th corner (ascending)
# without that bit.
MC_EDGES = [(lo, lo | a) for a in (1, 2, 4) for lo in range(8) if not lo & a]


def _corner_pos(c):
    return np.array([c & 1, (c >> 1) & 1, (c >> 2) & 1], np.float64)


def mc_case(cm):
    """Triangles (edge-index triples) of case cm (bit c: corner c inside)."""
    inside = [(cm >> c) & 1 for c in range(8)]
    cross = [e for e, (lo, hi) in enumerate(MC_EDGES) if inside[lo] != inside[hi]]
    succ = {}
    for axis in range(3):
        a = 1 << axis
        for side in (0, a):
            on_face = [e for e in cross if (MC_EDGES[e][0] & a) == side and (MC_EDGES[e][1] & a) == side]
            if len(on_face) == 2:
                pairs = [on_face]
            elif len(on_face) == 4:  # ambiguous: each inside corner is cut off alone
                pairs = [[e for e in on_face if c in MC_EDGES[e]]
                         for c in range(8) if (c & a) == side and inside[c]]
            else:
                pairs = []
            normal = np.zeros(3)
            normal[axis] = 1.0 if side else -1.0
            for e1, e2 in pairs:
                m1 = _corner_pos(MC_EDGES[e1][0]) * 0.5 + _corner_pos(MC_EDGES[e1][1]) * 0.5
                m2 = _corner_pos(MC_EDGES[e2][0]) * 0.5 + _corner_pos(MC_EDGES[e2][1]) * 0.5
                c_in = MC_EDGES[e1][0] if inside[MC_EDGES[e1][0]] else MC_EDGES[e1][1]
                on_left = np.dot(np.cross(normal, m2 - m1), _corner_pos(c_in) - m1) > 0
                a_, b_ = (e2, e1) if on_left else (e1, e2)  # inside stays on the right
                assert a_ not in succ
                succ[a_] = b_
    assert sorted(succ) == cross
    def faces(e):  # the two cube faces holding edge e, as (axis bit, side)
        lo, hi = MC_EDGES[e]
        return {(b, lo & b) for b in (1, 2, 4) if b != hi ^ lo}

    tris, done = [], set()
    for e0 in cross:  # ascending: each loop starts at its lowest edge
        if e0 in done:
            continue
        loop, e = [], e0
        while e not in done:
            done.add(e)
            loop.append(e)
            e = succ[e]
        n = len(loop)
        # fan from the first vertex whose diagonals all leave the cube's faces
        # (a diagonal inside a face would meet the neighbouring cube's)
        s = next(k for k in range(n)
                 if all(not faces(loop[k]) & faces(loop[(k + i) % n]) for i in range(2, n - 1)))
        tris += [(loop[s], loop[(s + i) % n], loop[(s + i + 1) % n]) for i in range(1, n - 1)]
    return tris


def iso_surface_mc(dens, iso, dx, below=False):
    """Marching cubes of {dens >= iso} ({dens <= iso} with ``below``):
    (verts (V,3) float32, tris (T,3) int32); vertices ordered by (node, axis
    x y z), triangles by (cube, case triangle)."""
    d = np.asarray(dens, F32)
    nx, ny, nz = d.shape
    if nx < 2 or ny < 2 or nz < 2:
        return np.zeros((0, 3), F32), np.zeros((0, 3), np.int32)
    iso32, dx32 = F32(iso), F32(dx)
    inside = d <= iso32 if below else d >= iso32
    cross = np.zeros((nx, ny, nz, 3), bool)
    vpos = np.zeros((nx, ny, nz, 3, 3), F32)
    gi, gj, gk = np.meshgrid(np.arange(nx, dtype=F32), np.arange(ny, dtype=F32),
                             np.arange(nz, dtype=F32), indexing="ij")
    for axis in range(3):
        o = [0, 0, 0]
        o[axis] = 1
        lo = (slice(0, nx - o[0]), slice(0, ny - o[1]), slice(0, nz - o[2]))
        hi = (slice(o[0], nx), slice(o[1], ny), slice(o[2], nz))
        cross[lo + (axis,)] = inside[lo] != inside[hi]
        with np.errstate(divide="ignore", invalid="ignore"):
            t = (iso32 - d[lo]) / (d[hi] - d[lo])
        for k, g in enumerate((gi, gj, gk)):
            vpos[lo + (axis, k)] = ((g[lo] + t) if k == axis else g[lo]) * dx32
    flat = cross.reshape(-1)
    verts = vpos.reshape(-1, 3)[flat]
    vid = np.full(flat.shape, -1, np.int64)
    vid[flat] = np.arange(int(flat.sum()))
    vid = vid.reshape(nx, ny, nz, 3)
    if len(verts) == 0:
        return verts.astype(F32), np.zeros((0, 3), np.int32)
    cx, cy, cz = nx - 1, ny - 1, nz - 1
    case = np.zeros((cx, cy, cz), np.int64)
    for c in range(8):
        x, y, z = c & 1, (c >> 1) & 1, (c >> 2) & 1
        case |= inside[x:x + cx, y:y + cy, z:z + cz].astype(np.int64) << c
    ci, cj, ck = np.meshgrid(np.arange(cx), np.arange(cy), np.arange(cz), indexing="ij")
    cube_key = (ci * ny + cj) * nz + ck

    def edge_vid(e, sel):
        lo, hi = MC_EDGES[e]
        x, y, z = lo & 1, (lo >> 1) & 1, (lo >> 2) & 1
        return vid[x:x + cx, y:y + cy, z:z + cz, {1: 0, 2: 1, 4: 2}[hi ^ lo]][sel]

    keys, tris = [], []
    for cm in np.unique(case):
        sel = case == cm
        for q, (e0, e1, e2) in enumerate(mc_case(int(cm))):
            keys.append(cube_key[sel] * 8 + q)
            tris.append(np.stack([edge_vid(e0, sel), edge_vid(e1, sel), edge_vid(e2, sel)], 1))
    if not keys:
        return verts.astype(F32), np.zeros((0, 3), np.int32)
    keys = np.concatenate(keys)
    tris = np.concatenate(tris)
    order = np.argsort(keys, kind="stable")
    return verts.astype(F32), tris[order].astype(np.int32)


def smooth(verts, faces, method="taubin", passes=2, lam=0.5, mu=-0.53):
    """``smooth_laplacian`` / ``smooth_taubin`` (src/gpufluid/meshing/
    smoothing.py:22-72): L = D^-1 A - I of the distinct 1-ring neighbours
    (D = #neighbours, 1 when none; 1/D rounded to float32 as the reference's
    scipy matrices hold it), applied in float64 with each row's diagonal first
    and then its neighbours in ascending order, a multiply and an add per
    entry; v += lam L v per pass (Taubin adds v += mu L v); float32 at the end."""
    v = np.asarray(verts, np.float32).astype(np.float64)
    if len(v) == 0 or passes <= 0:
        return np.asarray(verts, np.float32)
    f = np.asarray(faces, np.int64)
    e = np.concatenate([f[:, [0, 1]], f[:, [1, 0]], f[:, [1, 2]], f[:, [2, 1]],
                        f[:, [2, 0]], f[:, [0, 2]]])
    e = np.unique(e, axis=0)  # sorted by (row, col)
    n = len(v)
    deg = np.bincount(e[:, 0], minlength=n)
    start = np.concatenate([[0], np.cumsum(deg)])
    dinv = (np.float32(1.0) / np.maximum(deg, 1).astype(np.float32)).astype(np.float64)
    maxd = int(deg.max()) if len(e) else 0
    nbr = np.zeros((n, max(maxd, 1)), np.int64)
    mask = np.zeros((n, max(maxd, 1)), bool)
    for k in range(maxd):
        has = deg > k
        nbr[has, k] = e[start[:-1][has] + k, 1]
        mask[has, k] = True
    steps = [lam] * passes if method == "laplacian" else [c for _ in range(passes) for c in (lam, mu)]
    for c in steps:
        acc = 0.0 + (-1.0 * v)
        for k in range(maxd):
            acc = np.where(mask[:, k:k + 1], acc + dinv[:, None] * v[nbr[:, k]], acc)
        v = v + c * acc
    return v.astype(np.float32)


def mesh_volume(verts, tris):
    """Signed enclosed volume (divergence theorem), float64."""
    v = np.asarray(verts, np.float64)
    a, b, c = v[tris[:, 0]], v[tris[:, 1]], v[tris[:, 2]]
    return float(np.einsum("ij,ij->i", a, np.cross(b, c)).sum() / 6.0)


def mesh_area(verts, tris):
    v = np.asarray(verts, np.float64)
    a, b, c = v[tris[:, 0]], v[tris[:, 1]], v[tris[:, 2]]
    return float(0.5 * np.linalg.norm(np.cross(b - a, c - a), axis=1).sum())


def boundary_edges(tris):
    """Number of undirected edges used by exactly one triangle (0 for a closed
    surface) and whether every interior edge appears once in each direction."""
    t = np.asarray(tris, np.int64)
    e = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]])
    und = np.sort(e, axis=1)
    _, cnt = np.unique(und, axis=0, return_counts=True)
    _, dcnt = np.unique(e, axis=0, return_counts=True)
    return int((cnt == 1).sum()), bool((dcnt == 1).all())
