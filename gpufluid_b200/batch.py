"""Batches of independent FLIP/PIC/APIC scenes stepped together.

The reference steps one ``FlipSolver3D`` at a time; ``BatchedFlip3D`` holds
many scenes of uneven grid sizes in one library context (``gf_batch_create``)
whose arrays are the scenes' arrays concatenated in table order.  Every stage
of a substep is ONE kernel launch over all scenes (a segment table tells each
tile, face, cell or particle its scene); the pressure PCG is one persistent
kernel with per-scene scalars that stops every scene at its own tolerance; the
substep is captured in a CUDA graph and replayed; ``autotune`` picks launch
shapes by timing real substeps.  Per scene the numerics are those of a
``FlipSolver3D`` with the same grid, particles and parameters (the same
kernels on the same data; only float-atomic summation order differs).
"""
from __future__ import annotations

import ctypes
from collections import OrderedDict
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib
from . import scene as _scene


def cfg_uneven_scenes(n_scenes: int = 64, sides=(32, 48, 64, 80, 96), seed: int = 0):
    """Scene list of the batched dam-break workload: per scene a cubic grid
    side drawn uniformly from ``sides`` and a fluid block x in [0, U(0.2,0.5)],
    y in [0, U(0.3,0.7)], z in [0, 1], all draws from one seeded generator."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_scenes):
        n = int(rng.choice(np.asarray(sides)))
        hx, hy = float(rng.uniform(0.2, 0.5)), float(rng.uniform(0.3, 0.7))
        out.append({"n": n, "lo": (0.0, 0.0, 0.0), "hi": (hx, hy, 1.0)})
    return out


class BatchedFlip3D:
    """Many scenes, one context.  ``grids`` lists (nx, ny, nz) or
    (nx, ny, nz, dx) per scene (dx defaults to 1/max(n), as FlipSolver3D)."""

    _MAX_GRAPHS = 4

    def __init__(self, grids: Sequence[Sequence], gravity: float = -9.81,
                 flip_blend: float = 0.95, rho: float = 1.0, transfer_mode: str = "flip",
                 device: Optional[str] = None, pressure_tol: float = 1e-4,
                 pcg_rhs_sign: int = -1, pcg_check_every: int = 10,
                 enable_cuda_graphs: bool = True, pcg_preconditioner: str = "jacobi",
                 pcg_sgs_sweeps: int = 2):
        if transfer_mode not in _lib.TRANSFER:
            raise ValueError(f"unknown transfer_mode: {transfer_mode!r}")
        if not torch.cuda.is_available():
            raise RuntimeError("BatchedFlip3D needs a CUDA device (B200, sm_100a)")
        if len(grids) < 1:
            raise ValueError("a batch needs at least one scene")
        self.device = torch.device(device or "cuda")
        self.gravity, self.flip_blend, self.rho = gravity, flip_blend, rho
        self.transfer_mode = transfer_mode
        self.pressure_tol = float(pressure_tol)
        self.pcg_rhs_sign = -1 if pcg_rhs_sign < 0 else 1
        self.pcg_check_every = int(pcg_check_every)
        if pcg_preconditioner not in ("jacobi", "tile_sgs"):
            raise ValueError(f"unknown pcg_preconditioner: {pcg_preconditioner!r}")
        if not 1 <= int(pcg_sgs_sweeps) <= 3:
            raise ValueError("pcg_sgs_sweeps must be 1, 2 or 3")
        # "tile_sgs": tile-local symmetric Gauss-Seidel sweeps precondition
        # every scene's PCG (the reference's Jacobi by default)
        self.pcg_preconditioner = pcg_preconditioner
        self.pcg_sgs_sweeps = int(pcg_sgs_sweeps)
        self._enable_cuda_graphs = bool(enable_cuda_graphs)
        self.grids = []
        descs = (_lib.GridDesc * len(grids))()
        for s, g in enumerate(grids):
            nx, ny, nz = (int(v) for v in g[:3])
            dx = float(g[3]) if len(g) > 3 else 1.0 / max(nx, ny, nz)
            dom = np.array([nx * dx, ny * dx, nz * dx], dtype=np.float32)
            self.grids.append((nx, ny, nz, dx, dom))
            descs[s] = _lib.GridDesc(nx, ny, nz, float(np.float32(dx)),
                                     (ctypes.c_float * 3)(*(float(d) for d in dom)))
        self.n_scenes = len(grids)
        L = _lib.load()
        self._L = L
        rows = (_lib.SceneLayout * self.n_scenes)()
        tot = _lib.BatchTotals()
        _lib.check(L.gf_batch_plan(descs, self.n_scenes, rows, ctypes.byref(tot)), None,
                   "gf_batch_plan")
        self.layout = [{k: int(getattr(r, k)) for k, _ in _lib.SceneLayout._fields_} for r in rows]
        self.totals = {k: int(getattr(tot, k)) for k, _ in _lib.BatchTotals._fields_}
        dev = self.device
        z = lambda n: torch.zeros(n, dtype=torch.float32, device=dev)  # noqa: E731
        T = self.totals
        self._u, self._v, self._w = z(T["nu"]), z(T["nv"]), z(T["nw"])
        self.uw, self.vw, self.ww = z(T["nu"]), z(T["nv"]), z(T["nw"])
        self.us, self.vs, self.ws = z(T["nu"]), z(T["nv"]), z(T["nw"])
        self._p, self.div = z(T["ncell"]), z(T["ncell"])
        labels = [_scene.wall_labels(nx, ny, nz).ravel() for nx, ny, nz, _, _ in self.grids]
        self._label = torch.from_numpy(np.concatenate(labels).astype(np.uint8)).to(dev)
        self._scene_pos: list = [np.zeros((0, 3), np.float32) for _ in range(self.n_scenes)]
        self.counts = np.zeros(self.n_scenes, np.int64)
        ctx = ctypes.c_void_p()
        with torch.cuda.device(dev):
            _lib.check(L.gf_batch_create(descs, self.n_scenes, 0, ctypes.byref(ctx)), None,
                       "gf_batch_create")
        self._ctx = ctx
        self._graphs: "OrderedDict[tuple, tuple]" = OrderedDict()
        self._replayed_launches = 0
        self._commit_particles()

    def __del__(self):
        ctx = getattr(self, "_ctx", None)
        if ctx is not None and getattr(self, "_L", None) is not None:
            try:
                torch.cuda.synchronize(self.device)
            except Exception:
                pass
            self._L.gf_destroy(ctx)
            self._ctx = None

    # ------------------------------------------------------------ set-up
    def seed_box(self, scene: int, lo, hi, ppc: int = 8, append: bool = False):
        """FlipSolver3D.seed_box for one scene (solver3d.py:2826-2910)."""
        nx, ny, nz, dx, _ = self.grids[scene]
        new = _scene.seed_box_positions(dx, lo, hi, ppc)
        cur = self._scene_pos[scene]
        self._scene_pos[scene] = np.concatenate([cur, new]) if append and len(cur) else new
        self._commit_particles()

    def set_particles(self, scene: int, pos: np.ndarray):
        self._scene_pos[scene] = np.ascontiguousarray(pos, dtype=np.float32).reshape(-1, 3)
        self._commit_particles()

    def add_solid_from_sdf(self, scene: int, sdf, padding: float = 0.0):
        nx, ny, nz, _, _ = self.grids[scene]
        c0 = self.layout[scene]["cell0"]
        lab = self._label[c0:c0 + nx * ny * nz].view(nx, ny, nz)
        solid = torch.from_numpy(np.asarray(sdf) <= padding).to(self.device)
        lab[solid] = 2

    def cell_centers_np(self, scene: int):
        nx, ny, nz, dx, _ = self.grids[scene]
        return _scene.cell_centers(nx, ny, nz, dx)

    def _commit_particles(self):
        dev = self.device
        self.counts = np.array([len(p) for p in self._scene_pos], np.int64)
        n = int(self.counts.sum())
        pos = (np.concatenate(self._scene_pos) if n else np.zeros((0, 3), np.float32))
        self._pos = torch.from_numpy(np.ascontiguousarray(pos, np.float32)).to(dev)
        self._vel = torch.zeros_like(self._pos)
        self._C = torch.zeros((n, 9), dtype=torch.float32, device=dev)
        self._pid = torch.arange(n, dtype=torch.int32, device=dev)
        self.part0 = np.concatenate([[0], np.cumsum(self.counts)]).astype(np.int64)
        self._bind()

    def _bind(self):
        ptr = lambda t: t.data_ptr() if t is not None and t.numel() else None  # noqa: E731
        self._fields = _lib.Fields(
            ptr(self._u), ptr(self._v), ptr(self._w), ptr(self.uw), ptr(self.vw), ptr(self.ww),
            ptr(self.us), ptr(self.vs), ptr(self.ws), ptr(self._p), ptr(self.div),
            ptr(self._label), None, None, None)
        n = self._pos.shape[0]
        self._parts = _lib.Particles(n, ptr(self._pos), ptr(self._vel), ptr(self._C),
                                     ptr(self._pid))
        counts = (ctypes.c_int64 * self.n_scenes)(*(int(c) for c in self.counts))
        _lib.check(self._L.gf_batch_bind(self._ctx, ctypes.byref(self._fields),
                                         ctypes.byref(self._parts), counts),
                   self._ctx, "gf_batch_bind")
        self._graphs.clear()

    # --------------------------------------------------------------- step
    @property
    def n_particles(self) -> int:
        return int(self._pos.shape[0])

    def _params(self, dt, pressure_iters, pressure_solver):
        if pressure_solver not in _lib.SOLVER:
            raise ValueError(f"unknown pressure_solver: {pressure_solver!r}")
        return _lib.StepParams(float(dt), float(self.gravity), float(self.rho),
                               float(self.flip_blend), _lib.TRANSFER[self.transfer_mode],
                               _lib.SOLVER[pressure_solver], int(pressure_iters),
                               self.pcg_check_every, self.pressure_tol, self.pcg_rhs_sign,
                               (self.pcg_sgs_sweeps << _lib.GF_FLAG_SGS_SHIFT)
                               if self.pcg_preconditioner == "tile_sgs" else 0)

    def _set_stream(self):
        self._L.gf_set_stream(self._ctx, torch.cuda.current_stream(self.device).cuda_stream)

    def step(self, dt: float, pressure_iters: int = 80, pressure_solver: str = "jacobi"):
        """One substep of every scene: one launch per stage kernel for the batch."""
        prm = self._params(dt, pressure_iters, pressure_solver)
        if not self._enable_cuda_graphs:
            self._set_stream()
            _lib.check(self._L.gf_step(self._ctx, ctypes.byref(prm)), self._ctx, "gf_step")
            return
        key = (self.n_particles,) + tuple(getattr(prm, f) for f, _ in prm._fields_)
        if key in self._graphs:
            self._graphs.move_to_end(key)
        else:
            self._capture(prm, key)
        graph, launches, _ = self._graphs[key]
        graph.replay()
        self._replayed_launches += launches

    def _capture(self, prm, key):
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(self.device)
        before = int(self._L.gf_launch_count(self._ctx))
        with torch.cuda.graph(g, stream=s):
            self._L.gf_set_stream(self._ctx, s.cuda_stream)
            _lib.check(self._L.gf_step(self._ctx, ctypes.byref(prm)), self._ctx,
                       "gf_step (capture)")
        launches = int(self._L.gf_launch_count(self._ctx)) - before
        self._graphs[key] = (g, launches, s)
        while len(self._graphs) > self._MAX_GRAPHS:
            self._graphs.popitem(last=False)

    def autotune(self, dt: float, pressure_iters: int = 80,
                 pressure_solver: str = "jacobi") -> dict:
        """Pick launch shapes by timing substeps (the state is restored)."""
        prm = self._params(dt, pressure_iters, pressure_solver)
        info = _lib.TuneInfo()
        self._set_stream()
        _lib.check(self._L.gf_autotune(self._ctx, ctypes.byref(prm), ctypes.byref(info)),
                   self._ctx, "gf_autotune")
        self._graphs.clear()  # launch shapes changed
        return {k: getattr(info, k) for k, _ in _lib.TuneInfo._fields_}

    def launch_count(self) -> int:
        return int(self._L.gf_launch_count(self._ctx)) + self._replayed_launches

    # ------------------------------------------------------------ results
    def pressure_stats(self) -> list:
        n = self.n_scenes
        it = (ctypes.c_int32 * n)()
        rel = (ctypes.c_double * n)()
        st = (ctypes.c_int32 * n)()
        self._set_stream()
        _lib.check(self._L.gf_batch_pressure_stats(self._ctx, it, rel, st), self._ctx,
                   "gf_batch_pressure_stats")
        return [{"iters": it[s], "relres": rel[s], "status": st[s]} for s in range(n)]

    def get_particles(self, scene: int):
        """(pos, vel) of one scene in its original particle order."""
        a, b = int(self.part0[scene]), int(self.part0[scene + 1])
        pid = self._pid[a:b].long() - a
        pos = torch.empty_like(self._pos[a:b])
        vel = torch.empty_like(self._vel[a:b])
        pos[pid] = self._pos[a:b]
        vel[pid] = self._vel[a:b]
        return pos.cpu().numpy(), vel.cpu().numpy()

    def field(self, scene: int, name: str) -> torch.Tensor:
        """Device view of one scene's u, v, w, p, div or marker array."""
        nx, ny, nz, _, _ = self.grids[scene]
        L = self.layout[scene]
        if name in ("u", "v", "w"):
            o = L["f" + name + "0"]
            shape = {"u": (nx + 1, ny, nz), "v": (nx, ny + 1, nz), "w": (nx, ny, nz + 1)}[name]
            buf = {"u": self._u, "v": self._v, "w": self._w}[name]
        else:
            o = L["cell0"]
            shape = (nx, ny, nz)
            buf = {"p": self._p, "div": self.div, "marker": self._label}[name]
        return buf[o:o + int(np.prod(shape))].view(*shape)
