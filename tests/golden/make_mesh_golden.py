"""Generate golden vectors for the mesh density field from the reference's
own kernels (src/gpufluid/meshing/surface.py:14-43 k_density_scatter, :53-84
k_cubic_scatter, :100-122 k_sdf_field, src/gpufluid/primitives/gridmath.py:
103-121 k_box_blur_3d, surface.py:179-193 k_mc_zero_walls), run in the order of
``MeshExtractor.extract`` (:353-425) for mesh_method "trilinear", "cubic" and
"sdf" (the stand-in's hash-grid query returns every point, a superset of the
points within the radius, which is all Warp's query promises).

Test-fixture generator (run by hand, in a container that holds the reference
checkout; nothing at test or bench time reads the reference):

    python tests/golden/make_mesh_golden.py --reference <path of the GPUFLUID checkout>

It installs the sequential Warp stand-in (``warp_shim.py``) and imports the
two reference modules unmodified.  The iso-surface step after them is a
third-party routine there (scikit-image's or Warp's marching cubes, neither
installed here) and is not recorded.

It also runs the reference's mesh smoothing (``meshing/smoothing.py``, NumPy +
SciPy, imported as it is) on two marching-tetrahedra surfaces.

Writes ``tests/golden/mesh/density.npz`` and ``tests/golden/mesh/smoothing.npz``.
"""
from __future__ import annotations

import argparse
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NX, NY, NZ = 16, 12, 10
DX = 1.0 / 16.0
# (mesh_method, smooth_passes, wall_margin_cells, cubic_radius_cells)
CASES = [("trilinear", 2, 0, 0.0), ("trilinear", 1, 2, 0.0), ("trilinear", 0, 0, 0.0),
         ("cubic", 1, 0, 2.0), ("cubic", 0, 1, 1.5)]
# (smooth_passes, sdf_particle_radius_cells, sdf_search_radius_cells)
SDF_CASES = [(0, 1.0, 4.0), (2, 1.5, 3.0)]


def particles():
    rng = np.random.default_rng(31)
    blob = np.float32([0.3, 0.25, 0.3]) + rng.normal(0, 0.08, (2500, 3)).astype(np.float32)
    edge = np.float32([[-0.02, 0.3, 0.3], [0.999, 0.7, 0.6], [0.5, 0.74, 0.62]])
    return np.concatenate([blob, edge]).astype(np.float32)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("GPUFLUID_REFERENCE"),
                    required="GPUFLUID_REFERENCE" not in os.environ,
                    help="GPUFLUID source checkout (or set GPUFLUID_REFERENCE)")
    args = ap.parse_args()
    sys.path.insert(0, HERE)
    import warp_shim
    wp = warp_shim.install()
    src = os.path.join(args.reference, "src", "gpufluid")
    for name, path in (("gpufluid", src), ("gpufluid.primitives", os.path.join(src, "primitives")),
                       ("gpufluid.meshing", os.path.join(src, "meshing"))):
        pkg = types.ModuleType(name)
        pkg.__path__ = [path]
        sys.modules[name] = pkg
    # surface.py imports scikit-image at module level for its CPU marching
    # cubes, which is not run here
    skimage = types.ModuleType("skimage")
    skimage.measure = types.ModuleType("skimage.measure")
    sys.modules.setdefault("skimage", skimage)
    sys.modules.setdefault("skimage.measure", skimage.measure)
    from gpufluid.primitives.gridmath import k_box_blur_3d
    from gpufluid.meshing.surface import (k_cubic_scatter, k_density_scatter, k_mc_zero_walls,
                                          k_sdf_field)

    pos = particles()
    out = {"pos": pos, "dx": DX}
    for c, (method, passes, margin, radius) in enumerate(CASES):
        dens = wp.zeros((NX, NY, NZ), dtype=float)
        tmp = wp.zeros((NX, NY, NZ), dtype=float)
        if method == "trilinear":
            wp.launch(k_density_scatter, dim=len(pos),
                      inputs=[wp.array(pos, dtype=wp.vec3), dens, DX, NX, NY, NZ])
        else:  # the host arithmetic of MeshExtractor.extract (surface.py:376-382)
            r_world = float(radius) * DX
            inv_r_world_sq = 1.0 / (r_world * r_world)
            half_cells = int(np.ceil(radius)) + 1
            wp.launch(k_cubic_scatter, dim=len(pos),
                      inputs=[wp.array(pos, dtype=wp.vec3), dens, DX, inv_r_world_sq,
                              half_cells, NX, NY, NZ])
        a, b = dens, tmp
        for _ in range(passes):
            wp.launch(k_box_blur_3d, dim=(NX, NY, NZ), inputs=[a, b])
            a, b = b, a
        if margin > 0:
            wp.launch(k_mc_zero_walls, dim=(NX, NY, NZ), inputs=[a, int(margin)])
        out[f"density_{c}"] = np.asarray(a.numpy(), np.float32)
        out[f"case_{c}"] = np.array([method == "cubic", passes, margin, radius], np.float64)
    # mesh_method "sdf" (surface.py:405-420): phi = sqrt(min(R^2, nearest d^2)) - r
    # on a subset of the particles, then the blur (no wall margin for sdf)
    sub = pos[::4]
    out["sdf_pos"] = sub
    for c, (passes, r_cells, s_cells) in enumerate(SDF_CASES):
        search_r_world = float(s_cells) * DX
        particle_r_world = float(r_cells) * DX
        phi = wp.zeros((NX, NY, NZ), dtype=float)
        tmp = wp.zeros((NX, NY, NZ), dtype=float)
        phi.fill_(search_r_world)
        grid = wp.HashGrid(64, 64, 64)
        pw = wp.array(sub, dtype=wp.vec3)
        grid.build(pw, search_r_world)
        wp.launch(k_sdf_field, dim=(NX, NY, NZ),
                  inputs=[grid.id, pw, phi, DX, NX, NY, NZ, search_r_world, particle_r_world])
        a, b = phi, tmp
        for _ in range(passes):
            wp.launch(k_box_blur_3d, dim=(NX, NY, NZ), inputs=[a, b])
            a, b = b, a
        out[f"sdf_{c}"] = np.asarray(a.numpy(), np.float32)
        out[f"sdf_case_{c}"] = np.array([passes, r_cells, s_cells], np.float64)
    d = os.path.join(HERE, "mesh")
    os.makedirs(d, exist_ok=True)
    np.savez_compressed(os.path.join(d, "density.npz"), **out)

    # mesh smoothing: the reference's functions (NumPy + SciPy) on the
    # marching-tetrahedra surfaces of two fields, one closed and one open
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle import mesh as om
    from gpufluid.meshing.smoothing import smooth_laplacian, smooth_taubin
    import scipy
    sm = {"scipy_version": np.array(scipy.__version__)}
    n = 20
    i, j, k = np.meshgrid(*[np.arange(n)] * 3, indexing="ij")
    fields = [(6.3 - np.sqrt((i - 9.4) ** 2 + (j - 10.1) ** 2 + (k - 8.7) ** 2)).astype(np.float32),
              (np.sin(i / 3.0) + np.cos(j / 4.0) - k / 10.0).astype(np.float32)]
    for c, f in enumerate(fields):
        v, t = om.iso_surface(f, 0.0, 1.0 / n)
        sm[f"verts_{c}"], sm[f"faces_{c}"] = v, t
        sm[f"taubin_{c}"] = smooth_taubin(v, t, passes=2)
        sm[f"laplacian_{c}"] = smooth_laplacian(v, t, passes=3, lam=0.4)
    np.savez_compressed(os.path.join(d, "smoothing.npz"), **sm)
    print({k: (v.shape, float(v.max())) for k, v in out.items() if k.startswith("density")})


if __name__ == "__main__":
    main()
