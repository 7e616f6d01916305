"""Generate golden vectors for GPU particle reseeding from the reference's own
``reseed_particles_gpu`` (src/gpufluid/sim/reseed.py:275-396).

Test-fixture generator (run by hand, in a container that holds the reference
checkout; nothing at test or bench time reads the reference):

    python tests/golden/make_reseed_golden.py --reference <path of the GPUFLUID checkout>

It installs the sequential Warp stand-in (``warp_shim.py``) plus a
``warp.utils.array_scan`` restated from Warp's documentation (an inclusive or
exclusive prefix sum), imports ``gpufluid.sim.reseed`` unmodified and runs
``reseed_particles_gpu`` on a 12x10x8 grid.  Sequential threads are one
valid Warp schedule: the per-cell rank of the culling kernel is then the
particles' index order.

The scene: walls, a solid block, fluid-marked cells, 1,700 particles drawn so
that some cells hold more than ``max_per_cell`` (16), some fewer than
``min_per_cell`` (4), some sit in the solid block and some lie outside the
grid (clamped to the edge cells).  ``ReseedConfig()`` defaults and the CLI's
generator ``default_rng(123)`` (commands.py:612).

Writes ``tests/golden/reseed/reseed.npz``.
"""
from __future__ import annotations

import argparse
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NX, NY, NZ = 12, 10, 8
DX = 1.0 / 12.0


def scene():
    marker = np.zeros((NX, NY, NZ), np.int32)
    marker[0], marker[-1] = 2, 2
    marker[:, 0], marker[:, -1] = 2, 2
    marker[:, :, 0], marker[:, :, -1] = 2, 2
    marker[6:9, 3:6, 2:5] = 2               # solid block
    marker[1:6, 1:5, 1:7] = 1               # cells the last step marked fluid
    rng = np.random.default_rng(77)
    dense = (np.float32([0.20, 0.20, 0.25]) +
             rng.random((900, 3)).astype(np.float32) * np.float32([0.16, 0.16, 0.16]))
    sparse = rng.random((700, 3)).astype(np.float32) * np.float32([1.0, 0.83, 0.66])
    solid = (np.float32([0.55, 0.30, 0.20]) +
             rng.random((60, 3)).astype(np.float32) * np.float32([0.2, 0.2, 0.2]))
    outside = np.float32([[-0.01, 0.5, 0.3], [1.2, 0.1, 0.1], [0.4, 0.9, 0.7],
                          [0.3, -0.2, 0.9], [0.5, 0.5, -0.05]] * 8)
    pos = np.concatenate([dense, sparse, solid, outside]).astype(np.float32)
    vel = rng.normal(size=pos.shape).astype(np.float32)
    return marker, pos, vel


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("GPUFLUID_REFERENCE"),
                    required="GPUFLUID_REFERENCE" not in os.environ,
                    help="GPUFLUID source checkout (or set GPUFLUID_REFERENCE)")
    args = ap.parse_args()
    sys.path.insert(0, HERE)
    import warp_shim
    wp = warp_shim.install()
    utils = types.ModuleType("warp.utils")

    def array_scan(src, dst, inclusive=True):
        a = np.asarray(src).view(np.ndarray).astype(np.int64)
        c = np.cumsum(a)
        if not inclusive:
            c = c - a
        dst.view(np.ndarray)[: len(c)] = c
    utils.array_scan = array_scan
    wp.utils = utils
    sys.modules["warp.utils"] = utils
    # the package's __init__ imports every solver; register bare package
    # modules so that only gpufluid.sim.reseed and its imports load
    src = os.path.join(args.reference, "src", "gpufluid")
    for name, path in (("gpufluid", src), ("gpufluid.sim", os.path.join(src, "sim")),
                       ("gpufluid.primitives", os.path.join(src, "primitives"))):
        pkg = types.ModuleType(name)
        pkg.__path__ = [path]
        sys.modules[name] = pkg
    from gpufluid.sim.reseed import ReseedConfig, reseed_particles_gpu

    marker, pos, vel = scene()
    cfg = ReseedConfig()
    rng = np.random.default_rng(123)
    new_pos, new_vel, _, _, n_emit, n_cull = reseed_particles_gpu(
        wp.array(pos, dtype=wp.vec3), wp.array(vel, dtype=wp.vec3),
        wp.array(marker, dtype=int), DX, cfg, rng, device="cpu")
    out = os.path.join(HERE, "reseed")
    os.makedirs(out, exist_ok=True)
    np.savez_compressed(os.path.join(out, "reseed.npz"), marker=marker, pos=pos, vel=vel,
                        new_pos=np.asarray(new_pos.numpy(), np.float32),
                        new_vel=np.asarray(new_vel.numpy(), np.float32),
                        n_emit=n_emit, n_cull=n_cull, dx=DX, min_per_cell=cfg.min_per_cell,
                        max_per_cell=cfg.max_per_cell, jitter=cfg.jitter)
    print("particles", len(pos), "emitted", n_emit, "culled", n_cull, "->", len(new_pos.numpy()))


if __name__ == "__main__":
    main()
