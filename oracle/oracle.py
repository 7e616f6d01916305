"""CPU oracle for the FLIP/PIC/APIC substep -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference arm may import this module, and only as the checker or the timed CPU
baseline; the product (``gpufluid_b200``) never does.

Parity pin: run sequentially (``par=False``) the C restatement in
``flip_oracle.c`` reproduces, bit for bit, the reference's own solver source
(``src/gpufluid/solvers/solver3d.py``) executed in launch order by the
sequential Warp stand-in (``tests/golden/warp_shim.py``); the committed
fixtures ``tests/golden/*.npz`` hold those reference outputs and
``tests/test_oracle_golden.py`` checks the pin.

Host-side restatements kept here (pure NumPy, float64 then float32 exactly as
the reference computes them):

* ``seed_box``      -- ``FlipSolver3D.seed_box``, solver3d.py:2826-2850
* ``wall_marker``   -- one-cell solid shell, solver3d.py:2475-2482
* ``sphere_sdf``    -- ``cell_centers`` + ``sdf_sphere``, primitives/sdf.py:31-44
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (gcc, OpenMP)."""
    if force or not os.path.exists(_LIB_PATH) or (
            os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(HERE, "flip_oracle.c"))):
        subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


def _declare(L):
    I, F, D, L64 = ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_int64
    sig = {
        "og_num_threads": ([], I),
        "og_clear_grid": ([I, I, I] + [_f32p] * 6 + [_i32p], None),
        "og_p2g_flip": ([I, I, I, F, L64, _f32p, _f32p] + [_f32p] * 6 + [_i32p, I], None),
        "og_p2g_apic": ([I, I, I, F, L64, _f32p, _f32p, _f32p] + [_f32p] * 6 + [_i32p, I], None),
        "og_normalize": ([I, I, I] + [_f32p] * 9 + [I], None),
        "og_add_gravity": ([I, I, I, _f32p, F, F, I], None),
        "og_enforce_bc": ([I, I, I, _f32p, _f32p, _f32p, _i32p, _f32p, _f32p, _f32p, I], None),
        "og_divergence": ([I, I, I, _f32p, _f32p, _f32p, _f32p, _i32p, F, F, F, I], None),
        "og_jacobi": ([I, I, I, _f32p, _f32p, _f32p, _i32p, I, I], None),
        "og_gsrb": ([I, I, I, _f32p, _f32p, _i32p, I, I], None),
        "og_pcg": ([I, I, I, _f32p, _f32p, _i32p, I, D, I, I, _f32p, I, _f32p], I),
        "og_pcg64": ([I, I, I, _f64p, _f32p, _i32p, I, D, I, _f64p, _f64p], I),
        "og_subtract_grad": ([I, I, I, _f32p, _f32p, _f32p, _f32p, _i32p, F, F, F, I], None),
        "og_g2p_flip": ([I, I, I, F, F, F, _f32p, L64, _f32p, _f32p] + [_f32p] * 6 + [I], None),
        "og_g2p_apic": ([I, I, I, F, F, _f32p, L64, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, I], None),
        "og_bin": ([I, I, I, F, L64, _f32p, _i32p, _i32p, _i32p, _i64p], None),
        "og_density_splat": ([I, I, I, F, L64, _f32p, _f32p], None),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res


def _p(a, t=_f32p):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(t)


# ------------------------------------------------------------ host set-up
def wall_marker(nx, ny, nz):
    """solver3d.py:2475-2482: marker 2 on the one-cell border, else 0."""
    m = np.zeros((nx, ny, nz), dtype=np.int32)
    m[0, :, :] = 2; m[-1, :, :] = 2
    m[:, 0, :] = 2; m[:, -1, :] = 2
    m[:, :, 0] = 2; m[:, :, -1] = 2
    return m


def sphere_sdf(nx, ny, nz, dx, center, radius):
    """cell_centers (sdf.py:31-38) + sdf_sphere (sdf.py:41-44)."""
    i = (np.arange(nx) + 0.5) * dx
    j = (np.arange(ny) + 0.5) * dx
    k = (np.arange(nz) + 0.5) * dx
    X, Y, Z = np.meshgrid(i, j, k, indexing="ij")
    g = np.stack([X, Y, Z], axis=-1).astype(np.float32)
    c = np.asarray(center, dtype=np.float32)
    return np.linalg.norm(g - c, axis=-1) - float(radius)


def seed_box(dx, lo, hi, ppc=8):
    """Vectorised restatement of seed_box, solver3d.py:2834-2850.

    One fresh ``default_rng(0)``; three draws per particle in the order
    px, py, pz; loop order i, j, k, sx, sy, sz; float64 math, float32 result.
    """
    i0, i1 = int(lo[0] / dx), int(hi[0] / dx)
    j0, j1 = int(lo[1] / dx), int(hi[1] / dx)
    k0, k1 = int(lo[2] / dx), int(hi[2] / dx)
    per_axis = int(round(ppc ** (1.0 / 3.0)))
    ni, nj, nk = max(i1 - i0, 0), max(j1 - j0, 0), max(k1 - k0, 0)
    n = ni * nj * nk * per_axis ** 3
    if n == 0:
        return np.zeros((0, 3), np.float32)
    r = np.random.default_rng(0).random(3 * n).reshape(n, 3)
    I, J, K, SX, SY, SZ = np.meshgrid(
        np.arange(i0, i1), np.arange(j0, j1), np.arange(k0, k1),
        np.arange(per_axis), np.arange(per_axis), np.arange(per_axis), indexing="ij")
    cell = np.stack([I.ravel(), J.ravel(), K.ravel()], axis=1).astype(np.float64)
    sub = np.stack([SX.ravel(), SY.ravel(), SZ.ravel()], axis=1).astype(np.float64)
    pos = (cell + (sub + 0.5 + 0.3 * (r - 0.5)) / per_axis) * dx
    return pos.astype(np.float32)


# ------------------------------------------------------------ the substep
class OracleFlip:
    """Holds one scene's state and steps it like FlipSolver3D._step_impl
    (solver3d.py:3475-3667) with the C restatement."""

    def __init__(self, nx, ny, nz, dx=None, gravity=-9.81, flip_blend=0.95, rho=1.0,
                 transfer_mode="flip", par=False):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.dx = dx if dx is not None else 1.0 / max(nx, ny, nz)
        self.dom = np.array([nx * self.dx, ny * self.dx, nz * self.dx], np.float32)
        self.gravity, self.flip_blend, self.rho = gravity, flip_blend, rho
        self.transfer_mode = transfer_mode
        self.par = int(bool(par))
        z = lambda *s: np.zeros(s, np.float32)  # noqa: E731
        self.u, self.v, self.w = z(nx + 1, ny, nz), z(nx, ny + 1, nz), z(nx, ny, nz + 1)
        self.uw, self.vw, self.ww = z(nx + 1, ny, nz), z(nx, ny + 1, nz), z(nx, ny, nz + 1)
        self.us, self.vs, self.ws = z(nx + 1, ny, nz), z(nx, ny + 1, nz), z(nx, ny, nz + 1)
        self.p, self.p_tmp, self.div = z(nx, ny, nz), z(nx, ny, nz), z(nx, ny, nz)
        self.marker = wall_marker(nx, ny, nz)
        self.pos = np.zeros((0, 3), np.float32)
        self.vel = np.zeros((0, 3), np.float32)
        self.C = np.zeros((0, 3, 3), np.float32)
        self.last_pressure_iters = 0
        self._work = None

    @property
    def n_particles(self):
        return self.pos.shape[0]

    def set_particles(self, pos, vel, C=None):
        self.pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3).copy()
        self.vel = np.ascontiguousarray(vel, np.float32).reshape(-1, 3).copy()
        self.C = (np.zeros((self.n_particles, 3, 3), np.float32) if C is None
                  else np.ascontiguousarray(C, np.float32).reshape(-1, 3, 3).copy())

    # stages ------------------------------------------------------------
    def clear(self):
        lib().og_clear_grid(self.nx, self.ny, self.nz, _p(self.u), _p(self.v), _p(self.w),
                            _p(self.uw), _p(self.vw), _p(self.ww), _p(self.marker, _i32p))

    def p2g(self):
        L, g = lib(), (self.nx, self.ny, self.nz, self.dx, self.n_particles)
        grids = (_p(self.u), _p(self.v), _p(self.w), _p(self.uw), _p(self.vw), _p(self.ww))
        if self.transfer_mode == "apic":
            L.og_p2g_apic(*g, _p(self.pos), _p(self.vel), _p(self.C), *grids,
                          _p(self.marker, _i32p), self.par)
        else:
            L.og_p2g_flip(*g, _p(self.pos), _p(self.vel), *grids, _p(self.marker, _i32p),
                          self.par)

    def normalize(self):
        lib().og_normalize(self.nx, self.ny, self.nz, _p(self.u), _p(self.v), _p(self.w),
                           _p(self.uw), _p(self.vw), _p(self.ww), _p(self.us), _p(self.vs),
                           _p(self.ws), self.par)

    def gravity_bc(self, dt):
        lib().og_add_gravity(self.nx, self.ny, self.nz, _p(self.v), self.gravity, dt, self.par)
        self.enforce_bc()

    def enforce_bc(self):
        lib().og_enforce_bc(self.nx, self.ny, self.nz, _p(self.u), _p(self.v), _p(self.w),
                            _p(self.marker, _i32p), None, None, None, self.par)

    def divergence(self, dt):
        lib().og_divergence(self.nx, self.ny, self.nz, _p(self.u), _p(self.v), _p(self.w),
                            _p(self.div), _p(self.marker, _i32p), self.dx, dt, self.rho,
                            self.par)

    def pressure(self, solver, iters, tol=1e-4, check_every=10, rhs_sign=-1):
        L, g = lib(), (self.nx, self.ny, self.nz)
        if solver == "jacobi":
            L.og_jacobi(*g, _p(self.p), _p(self.p_tmp), _p(self.div),
                        _p(self.marker, _i32p), iters, self.par)
            self.last_pressure_iters = iters
        elif solver == "gsrb":
            L.og_gsrb(*g, _p(self.p), _p(self.div), _p(self.marker, _i32p), iters, self.par)
            self.last_pressure_iters = iters
        elif solver == "pcg64":
            # FP64 Jacobi-PCG to relative residual tol (the CPU counterpart of
            # the refined solve: same residual target, FP64 throughout)
            p64, it, _ = pcg64(self.marker, self.div, tol=tol, max_iter=max(iters, 1),
                               rhs_sign=rhs_sign)
            self.p[...] = p64.astype(np.float32)
            self.last_pressure_iters = it
        elif solver == "pcg":
            if self._work is None:
                self._work = np.zeros(5 * self.nx * self.ny * self.nz, np.float32)
            self.last_pressure_iters = L.og_pcg(
                *g, _p(self.p), _p(self.div), _p(self.marker, _i32p), iters, float(tol),
                int(check_every), int(rhs_sign), _p(self._work), self.par, None)
        else:
            raise ValueError(f"unknown pressure_solver: {solver!r}")

    def grad_bc(self, dt):
        lib().og_subtract_grad(self.nx, self.ny, self.nz, _p(self.u), _p(self.v), _p(self.w),
                               _p(self.p), _p(self.marker, _i32p), self.dx, dt, self.rho,
                               self.par)
        self.enforce_bc()

    def g2p(self, dt):
        L = lib()
        if self.transfer_mode == "apic":
            L.og_g2p_apic(self.nx, self.ny, self.nz, self.dx, dt, _p(self.dom),
                          self.n_particles, _p(self.pos), _p(self.vel), _p(self.C),
                          _p(self.u), _p(self.v), _p(self.w), self.par)
        else:
            L.og_g2p_flip(self.nx, self.ny, self.nz, self.dx, dt, self.flip_blend,
                          _p(self.dom), self.n_particles, _p(self.pos), _p(self.vel),
                          _p(self.u), _p(self.v), _p(self.w), _p(self.us), _p(self.vs),
                          _p(self.ws), self.par)

    def step(self, dt, pressure_iters=80, pressure_solver="jacobi", tol=1e-4,
             check_every=10, rhs_sign=-1):
        self.clear()
        self.p2g()
        self.normalize()
        self.gravity_bc(dt)
        self.divergence(dt)
        self.pressure(pressure_solver, pressure_iters, tol, check_every, rhs_sign)
        self.grad_bc(dt)
        self.g2p(dt)


# ------------------------------------------------------------ extras
def pcg64(marker, div, tol=1e-13, max_iter=100000, rhs_sign=-1):
    """FP64 Jacobi-PCG solve of the reference's pressure operator.

    Returns (p float64 (nx,ny,nz), iterations, final relative residual)."""
    nx, ny, nz = marker.shape
    marker = np.ascontiguousarray(marker, np.int32)
    div = np.ascontiguousarray(div, np.float32)
    p = np.zeros((nx, ny, nz), np.float64)
    work = np.zeros(5 * nx * ny * nz, np.float64)
    rel = np.zeros(1, np.float64)
    it = lib().og_pcg64(nx, ny, nz, _p(p, _f64p), _p(div), _p(marker, _i32p), int(max_iter),
                        float(tol), int(rhs_sign), _p(work, _f64p), _p(rel, _f64p))
    return p, it, float(rel[0])


def bin_particles(nx, ny, nz, dx, pos, pid=None):
    """Canonical (tile-major cell key, particle id) ordering.

    Returns (key[P] int32, count[ntiles*512] int32, order[P] int64)."""
    P = pos.shape[0]
    pos = np.ascontiguousarray(pos, np.float32)
    pid = np.arange(P, dtype=np.int32) if pid is None else np.ascontiguousarray(pid, np.int32)
    nk = ((nx + 7) // 8) * ((ny + 7) // 8) * ((nz + 7) // 8) * 512
    key = np.zeros(P, np.int32)
    count = np.zeros(nk, np.int32)
    order = np.zeros(P, np.int64)
    lib().og_bin(nx, ny, nz, dx, P, _p(pos), _p(pid, _i32p), _p(key, _i32p),
                 _p(count, _i32p), _p(order, _i64p))
    return key, count, order


def density_splat(nx, ny, nz, dx, pos):
    out = np.zeros((nx, ny, nz), np.float32)
    pos = np.ascontiguousarray(pos, np.float32)
    lib().og_density_splat(nx, ny, nz, dx, pos.shape[0], _p(pos), _p(out))
    return out


def num_threads():
    return lib().og_num_threads()
