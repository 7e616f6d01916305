"""Benchmark: FLIP/APIC substeps per second at 128^3 on B200.

Workload (the 128^3 APIC dam-break configuration): 128^3 cells, dx = 1/128,
solid one-cell walls, fluid block x in [0,0.4], y in [0,0.6], z in [0,1]
seeded at 8 particles per cell (3,969,024 particles, the reference seeder's
arithmetic), a solid sphere at (0.7, 0.2, 0.5) radius 0.12, APIC transfer,
gravity -9.81, dt = 1/480.  A "step" is one full substep (binning, P2G,
forces/BC/divergence, pressure, projection, G2P + advection) of the evolving
scene.

  value   substeps/s with the pressure solved by FP32 PCG with FP64 residual
          replacement to a true relative residual of 1e-8, preconditioned by
          two sweeps of tile-local symmetric Gauss-Seidel plus a coarse
          correction over the solver blocks' regions (inputs resident in HBM;
          device time over the timed steps, max over ranks).
  refined_jacobi  the same refined solve with the reference's Jacobi
          preconditioner (the like-for-like comparison with plain).
  plain   the same substeps with plain FP32 PCG (the reference's Jacobi
          preconditioner) asked for the same 1e-8 (recursive residual), with
          the true residual it actually reached.
  e2e     the same substep through the public API with the particle state in
          pinned HOST memory: host->device copy of the full state, step,
          device->host copy of the full state, every step; HostPipeline keeps
          three independent states in flight so one state's copies overlap
          another's substep.  e2e_serial: one rollout through host buffers
          (each step's input is the previous output; no overlap possible).
  roofline  the PCG kernel: algorithmic bytes per launch / its device time,
          against the measured HBM copy bandwidth.
  cpu_baseline  the CPU oracle (a C port of the reference kernels) stepping
          one substep of the same scene on all host threads, with an FP64 CG
          pressure solve to the same 1e-8 residual.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
Multi-GPU (torchrun): independent replicas, one per rank ("replicas only":
the single-scene path does not shard); value sums the substeps of all ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import tempfile
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("FLIP substeps/s @128³ (refined vs plain FP32 PCG, same residual); fwd+adj/s")
# DRAM bytes (read + write) of one launch of the shared-memory PCG with the
# tile SGS preconditioner and the coarse correction (one region per active
# tile) on this workload, from an ncu capture: 12,928,000 read + 791,552
# written.  The solve's vectors stay in shared memory; only the input, result,
# tagged halo and coarse words, the coarse rows and the FP64 replacement steps
# touch DRAM, far below the algorithmic bytes of a streaming PCG.
PCG_DRAM_BYTES = 12928000 + 791552
GRID = 128
DT = 1.0 / 480.0
TOL = 1e-8
MAX_ITERS = 4000
SPHERE = ((0.7, 0.2, 0.5), 0.12)
BOX = ((0.0, 0.0, 0.0), (0.4, 0.6, 1.0))
SGS_SWEEPS = 2  # tile-local symmetric Gauss-Seidel sweeps of the headline solve
COARSE = True   # plus the tile coarse correction (one region per active tile)
WARM_START = True  # each refined solve starts from the previous substep's pressure
WORKLOAD = ("APIC dam break + sphere obstacle, 128^3 (dx=1/128), 8 ppc -> 3,969,024 "
            "particles, dt=1/480, pressure: FP32 PCG + FP64 residual replacement to 1e-8, "
            "tile-local symmetric Gauss-Seidel preconditioner (2 sweeps) + tile "
            "coarse correction, each solve started from the previous substep's pressure "
            "(stop test ||b - Ap|| <= 1e-8 ||b|| as from zero)")


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"gfb200_clocks_{os.getpid()}_{index}.csv")

    def start(self):
        """Start sampling and return once the first sample is written (the tool
        takes about a second to start), so the samples cover the timed region;
        samples taken before the return are not counted."""
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        self.skip = 0
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        t0 = time.time()
        while time.time() - t0 < 10.0 and self.proc.poll() is None:
            with open(self.path) as f:
                n = sum(1 for _ in f)
            if n > 0:
                self.skip = n
                return
            time.sleep(0.05)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        rows = []
        with open(self.path) as f:
            lines = f.readlines()
            lines = lines[self.skip:] or lines  # samples of the timed region
            for line in lines:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
                except ValueError:
                    continue
        if not rows:
            return None
        mx = max(r[1] for r in rows)
        load = [r for r in rows if r[0] > 0.5 * mx] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i, v in enumerate(r[2]) if v == "Active"})
        return {"sm_mhz": statistics.median(r[0] for r in load), "sm_max_mhz": mx,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------- scene
def make_solver(gf, device, graphs=True, precond="tile_sgs", coarse=COARSE, warm=WARM_START):
    from gpufluid_b200 import scene
    s = gf.FlipSolver3D(GRID, GRID, GRID, transfer_mode="apic", flip_blend=0.95,
                        device=device, pressure_tol=TOL, enable_cuda_graphs=graphs,
                        pcg_preconditioner=precond, pcg_sgs_sweeps=SGS_SWEEPS,
                        pcg_coarse=coarse, pcg_warm_start=warm)
    s.add_solid_from_sdf(scene.sdf_sphere(s.cell_centers_np(), *SPHERE))
    s.seed_box(*BOX)
    return s


def snapshot(s):
    return [t.clone() for t in (s._pos, s._vel, s._C, s._pid)]


def restore(s, snap):
    for dst, src in zip((s._pos, s._vel, s._C, s._pid), snap):
        dst.copy_(src)


def true_relres(s) -> float:
    """||b - A p|| / ||b|| in float64 for the solver's current p (host numpy,
    measurement only): A = #non-solid neighbours on the diagonal, -1 per fluid
    neighbour, fluid cells only; b = -div."""
    lab = s._label.cpu().numpy()
    p = s._p.cpu().numpy().astype(np.float64)
    b = -s.div.cpu().numpy().astype(np.float64)
    fl = lab == 1
    diag = np.zeros(lab.shape)
    acc = np.zeros(lab.shape)
    for ax in range(3):
        for sh in (-1, 1):
            nb_lab = np.full(lab.shape, 2, np.uint8)
            nb_p = np.zeros(lab.shape)
            src = [slice(None)] * 3
            dst = [slice(None)] * 3
            if sh == -1:
                dst[ax], src[ax] = slice(1, None), slice(None, -1)
            else:
                dst[ax], src[ax] = slice(None, -1), slice(1, None)
            nb_lab[tuple(dst)] = lab[tuple(src)]
            nb_p[tuple(dst)] = p[tuple(src)]
            diag += nb_lab != 2
            acc += np.where(nb_lab == 1, nb_p, 0.0)
    r = np.where(fl, b - (diag * p - acc), 0.0)
    bb = np.linalg.norm(np.where(fl, b, 0.0))
    return float(np.linalg.norm(r) / bb) if bb > 0 else 0.0


def pressure_error_fp64(torch, s, iters=6000) -> float:
    """||p - p64|| / ||p64|| for the solver's current float32 p, where p64 solves
    the same system (A p = -div on the fluid cells) in float64 by Jacobi-
    preconditioned CG on the device to a relative residual of 1e-13.
    Measurement only; the system is rebuilt from the labels with dense tensor
    ops."""
    dev = s._p.device
    lab = s._label.to(torch.int32)
    fl = lab == 1
    b = torch.where(fl, -s.div.double(), torch.zeros((), dtype=torch.float64, device=dev))
    pad_lab = torch.nn.functional.pad(lab, (1, 1, 1, 1, 1, 1), value=2)
    nx, ny, nz = lab.shape
    views = []
    for ax in range(3):
        for sh in (0, 2):
            sl = [slice(1, 1 + nx), slice(1, 1 + ny), slice(1, 1 + nz)]
            sl[ax] = slice(sh, sh + lab.shape[ax])
            views.append(tuple(sl))
    diag = sum((pad_lab[v] != 2).double() for v in views)
    nbf = [(pad_lab[v] == 1) for v in views]
    flf = fl.double()
    inv_d = torch.where(fl, 1.0 / diag.clamp(min=1.0), torch.zeros_like(diag))

    def A(x):
        xp = torch.nn.functional.pad(x, (1, 1, 1, 1, 1, 1))
        acc = sum(torch.where(m, xp[v], torch.zeros_like(x)) for m, v in zip(nbf, views))
        return (diag * x - acc) * flf

    x = torch.zeros_like(b)
    r = b.clone()
    z = r * inv_d
    pdir = z.clone()
    rz = float((r * z).sum())
    bb = float(torch.linalg.vector_norm(b))
    if bb == 0.0:
        return 0.0
    for it in range(iters):
        q = A(pdir)
        alpha = rz / float((pdir * q).sum())
        x += alpha * pdir
        r -= alpha * q
        if it % 20 == 0 and float(torch.linalg.vector_norm(r)) < 1e-13 * bb:
            break
        z = r * inv_d
        rz_new = float((r * z).sum())
        pdir = z + (rz_new / rz) * pdir
        rz = rz_new
    p32 = torch.where(fl, s._p.double(), torch.zeros_like(x))
    return float(torch.linalg.vector_norm(p32 - x) / torch.linalg.vector_norm(x))


def fp64_cpu_solve(lab, div, x0=None, tol=1e-13):
    """FP64 solve of the pressure system on the host (measurement only):
    scipy's Jacobi-preconditioned CG on the fluid cells' sparse matrix (A:
    #non-solid neighbours on the diagonal, -1 per fluid neighbour), b = -div,
    from x0 (a float32 solution: a warm start only, the answer does not
    depend on it).  Returns the dense FP64 solution and ||b - A x|| / ||b||."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    fl = lab == 1
    nf = int(fl.sum())
    idx = np.full(lab.shape, -1, np.int64)
    idx[fl] = np.arange(nf)
    diag = np.zeros(lab.shape)
    rows, cols = [], []
    for ax in range(3):
        for sh in (-1, 1):
            nb_lab = np.full(lab.shape, 2, lab.dtype)
            nb_idx = np.full(lab.shape, -1, np.int64)
            src, dst = [slice(None)] * 3, [slice(None)] * 3
            if sh == -1:
                dst[ax], src[ax] = slice(1, None), slice(None, -1)
            else:
                dst[ax], src[ax] = slice(None, -1), slice(1, None)
            nb_lab[tuple(dst)] = lab[tuple(src)]
            nb_idx[tuple(dst)] = idx[tuple(src)]
            diag += nb_lab != 2
            m = fl & (nb_lab == 1)
            rows.append(idx[m])
            cols.append(nb_idx[m])
    noff = sum(len(r) for r in rows)
    A = sp.csr_matrix((np.concatenate([-np.ones(noff), diag[fl]]),
                       (np.concatenate(rows + [np.arange(nf)]),
                        np.concatenate(cols + [np.arange(nf)]))), shape=(nf, nf))
    b = -div[fl].astype(np.float64)
    M = sp.diags(1.0 / np.maximum(diag[fl], 1.0))
    x, _ = spla.cg(A, b, x0=None if x0 is None else x0[fl].astype(np.float64), rtol=tol,
                   atol=0.0, M=M, maxiter=20000)
    out = np.zeros(lab.shape)
    out[fl] = x
    bn = float(np.linalg.norm(b))
    return out, (float(np.linalg.norm(b - A @ x)) / bn if bn > 0 else 0.0)


def fp64_error_leg(torch, s, snap0, steps=120, every=20):
    """The 128^3 workload's own protocol: 120 substeps of the refined solve
    from the seeded state; every 20 substeps the float32 pressure is compared
    with an FP64 solve of the same system on the host CPU (the solver's
    settings as timed, warm start included)."""
    restore(s, snap0)
    s._p.zero_()  # no previous pressure at the seeded state
    rows = []
    t0 = time.perf_counter()
    for k in range(1, steps + 1):
        s.step(DT, pressure_iters=MAX_ITERS, pressure_solver="pcg_refined")
        if k % every == 0:
            torch.cuda.synchronize()
            lab = s._label.cpu().numpy()
            div = s.div.cpu().numpy()
            p = s._p.cpu().numpy()
            x64, rel64 = fp64_cpu_solve(lab, div, p)
            err = float(np.linalg.norm(np.where(lab == 1, p, 0.0) - x64) / np.linalg.norm(x64))
            st = s.pressure_stats()
            rows.append({"substep": k, "rel_error_vs_fp64_cpu": err,
                         "fp64_solve_relres": rel64, "iters": st["iters"],
                         "refined_relres": st["relres"]})
    return {"protocol": f"{steps} substeps from the seeded state; every {every} substeps "
                        "||p - p64|| / ||p64||, p64 an FP64 CG solve of the same system on the "
                        "host CPU (scipy, to 1e-13)",
            "max_rel_error": max(r["rel_error_vs_fp64_cpu"] for r in rows),
            "checks": rows, "wall_s": round(time.perf_counter() - t0, 1)}


def pcg_bytes(st) -> float:
    """Algorithmic bytes of one PCG launch in the survey's accounting, over
    the cells the solver processes (N = active tiles x 512): 13 N of set-up,
    47 N per iteration (SpMV and p.Ap; x, r update and r.z; p update) and
    25 N per FP64 residual replacement.  The preconditioner's own traffic
    (tile sweeps, coarse correction) is not counted."""
    N = st["n_active_tiles"] * 512
    return float(N * (13 + 47 * st["iters"] + 25 * st["replacements"]))


def stage_bytes(P, nf, ncell_active, F):
    """Algorithmic bytes of the other APIC stages at these sizes, in the
    survey's accounting (N = cells the stage processes): sort 136P + 12N,
    P2G 60P + 4F + 2N, forces/div 8F + 5N, project 8F + 5N, G2P 72P + 4F."""
    N = ncell_active
    return {"bin_sort": 136 * P + 12 * N, "p2g": 60 * P + 4 * F + 2 * N,
            "forces_div": 8 * F + 5 * N, "project": 8 * F + 5 * N, "g2p": 72 * P + 4 * F}


# ------------------------------------------------------------- timed loops
def timed_steps(torch, s, steps, solver):
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = s.launch_count()
    e0.record(stream)
    for _ in range(steps):
        s.step(DT, pressure_iters=MAX_ITERS, pressure_solver=solver)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps, s.launch_count() - l0


def adjoint_leg(torch, device, reps=2, transfer="pic"):
    """Forward and forward+adjoint of the drop-shaping rollout (64^3 PIC sphere,
    40 substeps of 1/240 s, checkpoints every 10 substeps, refined PCG to 1e-9):
    substeps/s of each and their cost ratio, timed with device synchronisation
    around whole rollouts."""
    from gpufluid_b200.adjoint import DropShaping
    prob = DropShaping(n=64, T=40, k=10, device=device, transfer=transfer)
    g = torch.Generator(device="cpu").manual_seed(7)
    control = (0.1 * torch.randn((3, 64, 64, 64), generator=g)).to(device)
    prob.loss_and_grad(control)  # warm-up
    fwd, bwd = [], []
    for _ in range(reps):
        prob.loss_and_grad(control)
        fwd.append(prob.last_timing["forward_s"])
        bwd.append(prob.last_timing["backward_s"])
    tf, tb = float(np.median(fwd)), float(np.median(bwd))
    return {"workload": f"drop shaping 64^3 {transfer.upper()}, 40 substeps, checkpoint every 10",
            "particles": prob.P, "forward_substeps_per_s": round(prob.T / tf, 2),
            "fwd_adj_substeps_per_s": round(prob.T / (tf + tb), 2),
            "forward_ms": round(1e3 * tf, 2), "adjoint_ms": round(1e3 * tb, 2),
            "fwd_adj_over_fwd": round((tf + tb) / tf, 3)}


def batched_leg(torch, device, k_steps=10, warm=2, n_scenes=64, ranks=None):
    """64 independent dam breaks of uneven sides {32,48,64,80,96}^3 (seeded
    block extents, 8 ppc), FLIP, dt = 1/240, per-scene refined PCG to 1e-7:
    the whole batch stepped together (one launch per stage, captured graph,
    autotuned launch shapes) against the same scenes stepped one at a time
    with FlipSolver3D.  Both run `warm` untimed substeps, then `k_steps` timed
    substeps from the same state; the value is scene-substeps per second."""
    import gpufluid_b200 as gf
    from gpufluid_b200.batch import BatchedFlip3D, cfg_uneven_scenes
    from gpufluid_b200.dist import shard_scenes
    scenes = cfg_uneven_scenes(n_scenes, seed=0)
    dt, iters, tol = 1.0 / 240.0, 4000, 1e-7
    # on N GPUs each rank steps its shard of the scenes (by particle count,
    # estimated from the seeded block volumes); no exchange while stepping
    world = ranks.world if ranks else 1
    est = [int(sc["n"] ** 3 * sc["hi"][0] * sc["hi"][1] * 8) for sc in scenes]
    mine = shard_scenes(est, world)[ranks.rank if ranks else 0]
    scenes = [scenes[i] for i in mine]
    stream = torch.cuda.current_stream()

    def timed(step):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(k_steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    b = BatchedFlip3D([(sc["n"],) * 3 for sc in scenes], pressure_tol=tol, device=device,
                      pcg_preconditioner="tile_sgs", pcg_sgs_sweeps=SGS_SWEEPS)
    for i, sc in enumerate(scenes):
        b.seed_box(i, sc["lo"], sc["hi"])
    for _ in range(warm):
        b.step(dt, iters, "pcg_refined")
    tune = b.autotune(dt, iters, "pcg_refined")
    b.step(dt, iters, "pcg_refined")  # capture with the tuned shapes (untimed)
    l0 = b.launch_count()
    ms_batch = timed(lambda: b.step(dt, iters, "pcg_refined"))
    launches = (b.launch_count() - l0) // k_steps
    st = b.pressure_stats()
    n_part = b.n_particles
    del b
    ms_single = 0.0
    for sc in scenes:
        one = gf.FlipSolver3D(sc["n"], sc["n"], sc["n"], pressure_tol=tol, device=device,
                              enable_cuda_graphs=True, pcg_preconditioner="tile_sgs",
                              pcg_sgs_sweeps=SGS_SWEEPS)
        one.seed_box(sc["lo"], sc["hi"])
        for _ in range(warm + 1):
            one.step(dt, iters, "pcg_refined")
        ms_single += timed(lambda: one.step(dt, iters, "pcg_refined"))
        del one
    its = [x["iters"] for x in st]
    if ranks:  # whole-job figures: max time over ranks, totals over ranks
        ms_batch, ms_single = ranks.max(ms_batch), ranks.max(ms_single)
        n_part = int(ranks.sum(n_part))
    return {"workload": f"{n_scenes} dam breaks, sides from {{32,48,64,80,96}}^3, FLIP, 8 ppc, "
                        "dt=1/240, per-scene refined PCG to 1e-7 (tile SGS preconditioner, "
                        "batched and one at a time alike)",
            "scenes": n_scenes, "particles": n_part, "timed_substeps": k_steps,
            "sharding": f"{world} rank(s), scenes split by particle count",
            "batched_scene_substeps_per_s": round(n_scenes * k_steps * 1000.0 / ms_batch, 2),
            "one_at_a_time_scene_substeps_per_s": round(n_scenes * k_steps * 1000.0 / ms_single, 2),
            "speedup": round(ms_single / ms_batch, 3),
            "batched_ms_per_substep": round(ms_batch / k_steps, 3),
            "launches_per_batched_substep": int(launches),
            "pcg_iters_min_max": [int(min(its)), int(max(its))],
            "all_converged": bool(all(x["status"] == 0 for x in st)),
            "autotune": tune}


def batched_adjoint_leg(torch, device, n_scenes=64, reps=1, ranks=None):
    """The drop-shaping loss (sphere, PIC, 40 substeps of 1/240 s, checkpoints
    every 10, refined PCG to 1e-9) on the 64 scene sides of the batched
    workload, forward+adjoint of all scenes in one batch context against the
    same scenes' forward+adjoint one at a time (one single-grid problem per
    side, each scene with its own control).  Times are whole passes with
    device synchronisation around them; the value is scene-substeps/s."""
    from gpufluid_b200.adjoint import BatchedDropShaping, DropShaping
    from gpufluid_b200.batch import cfg_uneven_scenes
    from gpufluid_b200.dist import shard_scenes
    sides_all = [sc["n"] for sc in cfg_uneven_scenes(n_scenes, seed=0)]
    world = ranks.world if ranks else 1
    mine = shard_scenes([n ** 3 for n in sides_all], world)[ranks.rank if ranks else 0]
    sides = [sides_all[i] for i in mine]
    T = 40
    prob = BatchedDropShaping(sides, T=T, k=10, device=device)
    g = torch.Generator(device="cpu").manual_seed(7)
    control = (0.1 * torch.randn(prob.control_shape, generator=g)).to(device)
    prob.loss_and_grad(control)  # warm-up
    tb = []
    for _ in range(reps):
        prob.loss_and_grad(control)
        tb.append(prob.last_timing["forward_s"] + prob.last_timing["backward_s"])
    t_batch = float(np.median(tb))
    fwd_s = prob.last_timing["forward_s"]
    n_part = prob.P
    del prob
    singles, t_single = {}, 0.0
    for i, n in enumerate(sides):
        if n not in singles:
            singles[n] = DropShaping(n=n, T=T, k=10, device=device)
            c = (0.1 * torch.randn((3, n, n, n), generator=g)).to(device)
            singles[n].loss_and_grad(c)  # warm-up of this side
        c = (0.1 * torch.randn((3, n, n, n), generator=g)).to(device)
        singles[n].loss_and_grad(c)
        t_single += singles[n].last_timing["forward_s"] + singles[n].last_timing["backward_s"]
    del singles
    if ranks:
        t_batch, t_single = ranks.max(t_batch), ranks.max(t_single)
        n_part = int(ranks.sum(n_part))
    return {"workload": f"drop shaping on {n_scenes} scenes of sides {{32,48,64,80,96}}^3, PIC, "
                        "40 substeps, checkpoint every 10, refined PCG to 1e-9",
            "scenes": n_scenes, "particles": n_part,
            "sharding": f"{world} rank(s), scenes split by cell count",
            "batched_fwd_adj_s": round(t_batch, 3), "batched_forward_s": round(fwd_s, 3),
            "batched_fwd_adj_scene_substeps_per_s": round(n_scenes * T / t_batch, 2),
            "one_at_a_time_fwd_adj_s": round(t_single, 3),
            "one_at_a_time_fwd_adj_scene_substeps_per_s": round(n_scenes * T / t_single, 2),
            "speedup": round(t_single / t_batch, 3)}


def outflow_leg(torch, s, hbm, reps=20):
    """GPU outflow compaction (gf_outflow_compact) of the bench scene's
    particles against a slab y <= 0.05 that holds a tenth of them: device
    time per call (it synchronises for the new count) and algorithmic bytes
    (positions read twice, velocities once, survivors written: 36 B per
    particle + 24 B per survivor) against the copy peak."""
    import ctypes
    from gpufluid_b200 import _lib
    pos, vel = s._unsort(s._pos), s._unsort(s._vel)
    n = pos.shape[0]
    po, vo = torch.empty_like(pos), torch.empty_like(vel)
    box = np.ascontiguousarray(np.float32([[0.0, 0.0, 0.0, 1.0, 0.05, 1.0]]))
    bp = box.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    nout = ctypes.c_int64()
    s._set_stream()

    def call():
        _lib.check(s._L.gf_outflow_compact(s._ctx, pos.data_ptr(), vel.data_ptr(), n, bp, 1,
                                           po.data_ptr(), vo.data_ptr(), ctypes.byref(nout)),
                   s._ctx, "gf_outflow_compact")
    for _ in range(3):
        call()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        call()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    kept = int(nout.value)
    gbs = (36.0 * n + 24.0 * kept) / 1e9 / (ms / 1e3)
    return {"workload": "outflow slab y <= 0.05 over the 128^3 scene's particles",
            "particles": int(n), "kept": kept, "ms_per_call": round(ms, 4),
            "particles_per_s": round(n / (ms / 1e3), 1), "gbs": round(gbs, 1),
            "frac": round(gbs / hbm, 4)}


def reseed_leg(torch, s, snap, reps=5):
    """FlipSolver3D.reseed (device binning, rank cull and compaction; host
    emission list from the per-cell counts) on the bench scene's particle
    state with the reference's default bounds (4..16 per cell): wall time per
    call with device synchronisation, from the same state each time."""
    from gpufluid_b200.reseed import ReseedConfig
    cfg = ReseedConfig()
    restore(s, snap)
    base = [s._unsort(t).clone() for t in (s._pos, s._vel, s._C)]
    ts, res = [], None
    for r in range(reps + 1):
        s._set_particles(pos=base[0], vel=base[1], C=base[2])
        s.step(DT, pressure_iters=MAX_ITERS, pressure_solver="pcg_refined")  # labels of a substep
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = s.reseed(cfg, np.random.default_rng(123))
        torch.cuda.synchronize()
        if r:
            ts.append(time.perf_counter() - t0)
    return {"workload": "reseed of the 128^3 scene after one substep, 4..16 per cell",
            "particles_before": int(snap[0].shape[0]), "emitted": int(res[0]),
            "culled": int(res[1]), "ms_per_call": round(1e3 * float(np.median(ts)), 3)}


def e2e_pipelined(torch, gf, device, snap, steps, barrier, max_over_ranks, depth=3):
    """End to end through ``HostPipeline``: every submission copies the full
    particle state from pinned host memory, runs one refined substep and
    copies the full state back; ``depth`` solvers on their own streams keep
    that many independent states in flight.  Device time from the first
    submission to the last state's arrival in host memory, per submission."""
    from gpufluid_b200.pipeline import HostPipeline
    pipe = HostPipeline(lambda: make_solver(gf, device, graphs=True), depth=depth)
    host_in = pipe.host_buffers()
    for h, t in zip(host_in, snap):
        h.copy_(t)
    outs = [pipe.host_buffers() for _ in range(depth)]
    kw = dict(pressure_iters=MAX_ITERS, pressure_solver="pcg_refined")
    for k in range(2 * depth):  # graph captures and warm-up
        pipe.submit(host_in, outs[k % depth], DT, **kw)
    pipe.synchronize()
    torch.cuda.synchronize()
    barrier()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for st in pipe.streams:
        st.wait_stream(stream)
    for k in range(steps):
        pipe.submit(host_in, outs[k % depth], DT, **kw)
    pipe.wait_all(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / steps)
    barrier()
    del pipe
    torch.cuda.empty_cache()
    return ms, depth


def mesh_leg(torch, s, snap, hbm, reps=5):
    """MeshExtractor on the bench scene's particles with the scene TOML's
    [output] defaults (trilinear splat, 2 blur passes, iso 0.6): device time
    of the density field (zero + splat + 2 blur passes) and of the iso-surface
    (count, scan, read-back of the totals, emit), wall time of the whole
    extract including the copy of the mesh to the host, and the marching-
    tetrahedra surface of the same field for comparison.  Blur bytes: 4 B read
    + 4 B written per cell per pass (neighbour reads hit cache)."""
    from gpufluid_b200.mesh import MeshExtractor
    pos = snap[0]  # the scene's particle positions (storage order)
    ex = MeshExtractor(GRID, GRID, GRID, s.dx)
    stream = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    dens_ms, surf_ms, wall = [], [], []
    v = t = None
    for r in range(reps + 2):
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        ev[0].record(stream)
        ex.density(pos, smooth_passes=2)
        ev[1].record(stream)
        v, t = ex.surface(0.6)
        ev[2].record(stream)
        torch.cuda.synchronize()
        if r >= 2:
            wall.append(time.perf_counter() - w0)
            dens_ms.append(ev[0].elapsed_time(ev[1]))
            surf_ms.append(ev[1].elapsed_time(ev[2]))
    # the other field method and the smoothing: device time of one call each
    def dev_ms(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps
    sdf_ms = dev_ms(lambda: ex.density(pos, smooth_passes=2, mesh_method="sdf"))
    ex.density(pos, smooth_passes=2)
    smooth_ms = dev_ms(lambda: ex.surface(0.6, smooth_passes=2, smooth_method="taubin"))
    ex.surface_method = "marching_tetrahedra"
    mt_ms = dev_ms(lambda: ex.surface(0.6))
    mt_tris = ex.n_tris
    ex.surface_method = "marching_cubes"
    nc = GRID ** 3
    blur_bytes = 2 * 8 * nc
    return {"workload": f"{GRID}^3 scene particles -> trilinear density, 2 blur passes, "
                        "iso 0.6 surface (marching cubes), copied to the host",
            "particles": int(pos.shape[0]), "verts": 0 if v is None else int(len(v)),
            "tris": 0 if t is None else int(len(t)),
            "density_ms": round(float(np.median(dens_ms)), 4),
            "surface_ms": round(float(np.median(surf_ms)), 4),
            "extract_wall_ms": round(1e3 * float(np.median(wall)), 3),
            "blur_bytes": blur_bytes,
            "sdf_density_ms": round(sdf_ms, 3),
            "surface_taubin2_with_copy_ms": round(smooth_ms, 3),
            "marching_tetrahedra_surface_with_copy_ms": round(mt_ms, 3),
            "marching_tetrahedra_tris": int(mt_tris)}


def stage_bytes_flip(P, ncell_active, F):
    """Algorithmic bytes of the FLIP (non-APIC) stages in the survey's
    accounting: sort 64P + 12N, P2G 24P + 4F + 2N, forces/div 8F + 5N,
    project 8F + 5N, G2P 48P + 8F."""
    N = ncell_active
    return {"bin_sort": 64 * P + 12 * N, "p2g": 24 * P + 4 * F + 2 * N,
            "forces_div": 8 * F + 5 * N, "project": 8 * F + 5 * N, "g2p": 48 * P + 8 * F}


def extra_legs(torch, device, steps=3):
    """The other single-scene workloads, a few timed substeps each:
    64^3 FLIP dam break (box [0,.4]x[0,.6]x[0,1]), dt 1/240, Jacobi-PCG to
    1e-5 with at most 200 iterations; 256^3 double dam break (x in [0,.3] and
    [.7,1], y in [0,.7]), FLIP 0.97, dt 1/960, refined PCG to 1e-7 (the
    global-memory solver: the active region exceeds the shared-memory one)
    with the tile SGS preconditioner, then warm-started from the previous
    substep's pressure, then with the coarse correction over cubes of tiles
    (warm-started, and cold), and, from the same state, with the reference's Jacobi
    preconditioner, and 200 Jacobi sweeps as the plain comparison,
    with per-stage times and the device memory footprint."""
    import gpufluid_b200 as gf
    stream = torch.cuda.current_stream()
    out = {}

    def timed(s, dt, iters, solver, k):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(k):
            s.step(dt, pressure_iters=iters, pressure_solver=solver)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k

    s = gf.FlipSolver3D(64, 64, 64, flip_blend=0.95, pressure_tol=1e-5, device=device,
                        enable_cuda_graphs=True)
    s.seed_box((0.0, 0.0, 0.0), (0.4, 0.6, 1.0))
    for _ in range(3):
        s.step(1 / 240, pressure_iters=200, pressure_solver="pcg")
    ms = timed(s, 1 / 240, 200, "pcg", 20)
    out["dam_break_64_flip_pcg1e-5"] = {
        "particles": s.n_particles, "ms_per_substep": round(ms, 4),
        "substeps_per_s": round(1000 / ms, 2), "pcg_iters_last": s.last_pressure_iters}
    del s
    torch.cuda.empty_cache()
    free0, _ = torch.cuda.mem_get_info()
    s = gf.FlipSolver3D(256, 256, 256, flip_blend=0.97, pressure_tol=1e-7, device=device,
                        pcg_preconditioner="tile_sgs", pcg_sgs_sweeps=2)
    s.seed_box((0.0, 0.0, 0.0), (0.3, 0.7, 1.0))
    s.seed_box((0.7, 0.0, 0.0), (1.0, 0.7, 1.0), append=True)
    dt = 1 / 960
    s.step(dt, pressure_iters=4000, pressure_solver="pcg_refined")
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    snap = snapshot(s)
    ms_ref = timed(s, dt, 4000, "pcg_refined", steps)
    st_ref = s.pressure_stats()
    # the same substeps with each solve started from the previous pressure
    # (one untimed substep first, so the first timed solve starts from its
    # predecessor's answer)
    restore(s, snap)
    s.pcg_warm_start = True
    s.step(dt, pressure_iters=4000, pressure_solver="pcg_refined")
    ms_warm = timed(s, dt, 4000, "pcg_refined", steps)
    st_warm = s.pressure_stats()
    # the same substeps with the coarse correction (cubes of tiles), warm
    # started as above, then cold
    restore(s, snap)
    s.pcg_coarse = True
    s.step(dt, pressure_iters=4000, pressure_solver="pcg_refined")
    ms_cw = timed(s, dt, 4000, "pcg_refined", steps)
    st_cw = s.pressure_stats()
    restore(s, snap)
    s.pcg_warm_start = False
    ms_cc = timed(s, dt, 4000, "pcg_refined", steps)
    st_cc = s.pressure_stats()
    s.pcg_coarse = False
    # the same substeps with the reference's Jacobi preconditioner
    restore(s, snap)
    s.pcg_preconditioner = "jacobi"
    ms_ref_jac = timed(s, dt, 4000, "pcg_refined", steps)
    st_ref_jac = s.pressure_stats()
    s.pcg_preconditioner = "tile_sgs"
    restore(s, snap)
    ms_jac = timed(s, dt, 200, "jacobi", steps)
    s._prof.enabled = True
    s._L.gf_enable_timing(s._ctx, 1)
    s.step(dt, pressure_iters=4000, pressure_solver="pcg_refined")
    t = s.stage_times()
    s._L.gf_enable_timing(s._ctx, 0)
    s._prof.enabled = False
    P = s.n_particles
    F = (256 + 1) * 256 * 256 * 3
    sb = stage_bytes_flip(P, st_ref["n_active_tiles"] * 512, F)
    gbs = {k: round(sb[k] / 1e9 / (t[i] / 1e3), 1)
           for i, k in ((0, "bin_sort"), (1, "p2g"), (2, "forces_div"), (4, "project"),
                        (5, "g2p"))}
    out["double_dam_break_256"] = {
        "particles": P, "refined_pcg1e-7_ms_per_substep": round(ms_ref, 3),
        "refined_substeps_per_s": round(1000 / ms_ref, 3),
        "refined_iters_last": st_ref["iters"],
        "refined_preconditioner": "tile-local symmetric Gauss-Seidel, 2 sweeps",
        "refined_warm_start_ms_per_substep": round(ms_warm, 3),
        "refined_warm_start_substeps_per_s": round(1000 / ms_warm, 3),
        "refined_warm_start_iters_last": st_warm["iters"],
        "refined_warm_start_relres_last": st_warm["relres"],
        "refined_coarse_warm_ms_per_substep": round(ms_cw, 3),
        "refined_coarse_warm_substeps_per_s": round(1000 / ms_cw, 3),
        "refined_coarse_warm_iters_last": st_cw["iters"],
        "refined_coarse_warm_used": st_cw["coarse"],
        "refined_coarse_ms_per_substep": round(ms_cc, 3),
        "refined_coarse_iters_last": st_cc["iters"],
        "refined_coarse_used": st_cc["coarse"],
        "refined_jacobi_precond_ms_per_substep": round(ms_ref_jac, 3),
        "refined_jacobi_precond_iters_last": st_ref_jac["iters"],
        "pcg_kernel": "global-memory" if st_ref["kernel"] == 2 else "shared-memory",
        "jacobi200_ms_per_substep": round(ms_jac, 3),
        "jacobi200_substeps_per_s": round(1000 / ms_jac, 3),
        "stages_ms": {k: round(float(t[i]), 4) for i, k in enumerate(
            ("bin_sort", "p2g", "forces_div", "pressure", "project", "g2p", "total"))},
        "stages_gbs": gbs,
        "device_footprint_gb": round((free0 - free1) / 1e9, 2)}
    del s
    torch.cuda.empty_cache()
    return out


def run_ours(args):
    import torch

    import gpufluid_b200 as gf
    from gpufluid_b200.dist import Ranks

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = f"cuda:{local}"
    ranks = Ranks("nccl", device=device)
    world, rank = ranks.world, ranks.rank
    barrier = ranks.barrier
    max_over_ranks = ranks.max

    s = make_solver(gf, device, graphs=True)
    P = s.n_particles
    snap0 = snapshot(s)
    for _ in range(args.warmup):
        s.step(DT, pressure_iters=MAX_ITERS, pressure_solver="pcg_refined")
    torch.cuda.synchronize()
    snap = snapshot(s)
    p_snap = s._p.clone()  # the last solve's pressure: the warm start of the next

    # ---- plain FP32 PCG from the same state (same 1e-8 target, recursive
    # residual), with the reference's Jacobi preconditioner; every comparison
    # leg starts its solves from zero, as the reference does
    s.pcg_warm_start = False
    s.pcg_preconditioner = "jacobi"
    s.pcg_coarse = False
    s.step(DT, pressure_iters=MAX_ITERS, pressure_solver="pcg")  # capture its graph
    torch.cuda.synchronize()
    restore(s, snap)
    barrier()
    torch.cuda.synchronize()
    ms_plain, _ = timed_steps(torch, s, args.steps, "pcg")
    plain_stats = s.pressure_stats()
    check = not args.no_fp64_check
    plain_true = true_relres(s) if check else None
    plain_err = pressure_error_fp64(torch, s) if check else None
    # ---- the refined solve with the Jacobi preconditioner (like for like)
    restore(s, snap)
    s.step(DT, pressure_iters=MAX_ITERS, pressure_solver="pcg_refined")  # capture
    torch.cuda.synchronize()
    restore(s, snap)
    barrier()
    torch.cuda.synchronize()
    ms_refj, _ = timed_steps(torch, s, args.steps, "pcg_refined")
    refj_stats = s.pressure_stats()
    refj_err = pressure_error_fp64(torch, s) if check else None
    s.pcg_preconditioner = "tile_sgs"
    s.pcg_coarse = COARSE
    # ---- the headline solver with every solve started from zero
    restore(s, snap)
    s.step(DT, pressure_iters=MAX_ITERS, pressure_solver="pcg_refined")  # capture
    torch.cuda.synchronize()
    restore(s, snap)
    barrier()
    torch.cuda.synchronize()
    ms_cold, _ = timed_steps(torch, s, args.steps, "pcg_refined")
    cold_stats = s.pressure_stats()
    s.pcg_warm_start = WARM_START
    restore(s, snap)
    s._p.copy_(p_snap)
    s.step(DT, pressure_iters=MAX_ITERS, pressure_solver="pcg_refined")  # capture
    torch.cuda.synchronize()
    restore(s, snap)
    s._p.copy_(p_snap)

    # ---- refined (the value)
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    ms_ref, launches = timed_steps(torch, s, args.steps, "pcg_refined")
    clk = clocks.stop()
    barrier()
    ms_ref_max = max_over_ranks(ms_ref)
    ref_stats = s.pressure_stats()
    ref_true = true_relres(s) if check else None
    ref_err = pressure_error_fp64(torch, s) if check else None

    # ---- per-stage device times and the PCG kernel (live, same workload)
    restore(s, snap)
    s._p.copy_(p_snap)
    s._prof.enabled = True
    s._L.gf_enable_timing(s._ctx, 1)
    stage, pcg_ms, pcg_b = [], [], []
    for _ in range(max(3, min(args.steps, 10))):
        s.step(DT, pressure_iters=MAX_ITERS, pressure_solver="pcg_refined")
        t = s.stage_times()
        st = s.pressure_stats()
        stage.append(t)
        pcg_ms.append(t[7])
        pcg_b.append(pcg_bytes(st))
    s._L.gf_enable_timing(s._ctx, 0)
    s._prof.enabled = False
    stage_ms = np.mean(np.array(stage), axis=0)
    hbm, peak_kind = peaks()
    achieved = (np.sum(pcg_b) / 1e9) / (np.sum(pcg_ms) / 1e3)
    nf = st["n_fluid"]
    F = (GRID + 1) * GRID * GRID * 3
    sb = stage_bytes(P, nf, st["n_active_tiles"] * 512, F)
    stage_gbs = {k: round(sb[k] / 1e9 / (stage_ms[i] / 1e3), 1)
                 for i, k in ((0, "bin_sort"), (1, "p2g"), (2, "forces_div"), (4, "project"),
                              (5, "g2p"))}

    # ---- e2e through the public API with host buffers
    restore(s, snap)
    host = [torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for t in snap]
    for h, t in zip(host, snap):
        h.copy_(t)
    devs = (s._pos, s._vel, s._C, s._pid)
    h2d = sum(t.numel() * t.element_size() for t in host)
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        for d, h in zip(devs, host):
            d.copy_(h, non_blocking=True)
        s.step(DT, pressure_iters=MAX_ITERS, pressure_solver="pcg_refined")
        for d, h in zip(devs, host):
            h.copy_(d, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e_serial = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    barrier()
    # the same through HostPipeline: independent host-resident states, three
    # in flight, so one state's copies overlap another's substep
    ms_e2e, depth = e2e_pipelined(torch, gf, device, snap, args.steps, barrier,
                                  max_over_ranks)

    fp64_check = fp64_error_leg(torch, s, snap0) if check else None

    outflow = outflow_leg(torch, s, hbm)
    reseed = reseed_leg(torch, s, snap)
    mesh = mesh_leg(torch, s, snap, hbm)

    fwd_adj = None if args.no_adjoint else adjoint_leg(torch, device)
    fwd_adj_apic = None if args.no_adjoint else adjoint_leg(torch, device, transfer="apic")
    batched = None if args.no_batched else batched_leg(torch, device, ranks=ranks)
    batched_adj = (None if args.no_batched or args.no_adjoint
                   else batched_adjoint_leg(torch, device, ranks=ranks))
    extra = None if args.no_extra else extra_legs(torch, device)

    ms_plain_max = max_over_ranks(ms_plain)  # every rank takes part in each collective

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(steps=1)
        cpu["mesh"] = cpu_mesh_baseline(snap[0].cpu().numpy(), s.dx)

    if rank == 0:
        value = world * 1000.0 / ms_ref_max
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "substeps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_ref_max, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded seed_box lattice of the reference, sphere SDF obstacle)",
            "config": {"workload": WORKLOAD, "grid": GRID, "particles": P, "transfer": "apic",
                       "dt": DT, "pressure": "pcg_refined", "tol": TOL,
                       "preconditioner": f"tile-local symmetric Gauss-Seidel, {SGS_SWEEPS} sweeps"
                                         + (", tile coarse correction" if COARSE else ""),
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2_policy": "inputs larger than L2: particle state "
                                    f"{P * 64 / 1e6:.0f} MB + MAC grids {F * 4 * 3 / 1e6:.0f} MB "
                                    "streamed every substep"},
            "particle_updates_per_s": round(value * P, 1),
            "plain_fp32": {"substeps_per_s": round(world * 1000.0 / ms_plain_max, 3),
                           "ms_per_step": round(ms_plain, 4), "iters_last": plain_stats["iters"],
                           "recursive_relres": plain_stats["relres"],
                           "true_relres_fp64": plain_true,
                           "pressure_rel_error_vs_fp64": plain_err},
            "refined": {"ms_per_step": round(ms_ref, 4), "iters_last": ref_stats["iters"],
                        "replacements_last": ref_stats["replacements"],
                        "true_relres_fp64": ref_true,
                        "pressure_rel_error_vs_fp64": ref_err,
                        "error_vs_fp64_cpu_every_20": fp64_check,
                        "warm_start": WARM_START,
                        "time_vs_plain": round(ms_ref / ms_plain, 3)},
            "refined_cold_start": {"ms_per_step": round(ms_cold, 4),
                                   "substeps_per_s": round(1000.0 / ms_cold, 3),
                                   "iters_last": cold_stats["iters"],
                                   "note": "the headline solver with every solve started from "
                                           "zero (the reference's start)"},
            "refined_jacobi": {"ms_per_step": round(ms_refj, 4), "iters_last": refj_stats["iters"],
                               "pressure_rel_error_vs_fp64": refj_err,
                               "time_vs_plain": round(ms_refj / ms_plain, 3)},
            "e2e": {"value": round(world * 1000.0 / ms_e2e, 3), "unit": "substeps/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(h2d),
                    "mode": f"HostPipeline: {depth} independent host-resident states in flight, "
                            "each submission = H2D of the full particle state (pinned), one "
                            "substep, D2H of the full state; copies of one state overlap "
                            "another's substep",
                    "ms_per_step": round(ms_e2e, 4),
                    "serial": {"value": round(world * 1000.0 / ms_e2e_serial, 3),
                               "unit": "substeps/s", "ms_per_step": round(ms_e2e_serial, 4),
                               "mode": "one rollout: each substep's input is the previous "
                                       "substep's output, copied in and out every substep"}},
            "e2e_serial": {"value": round(world * 1000.0 / ms_e2e_serial, 3),
                           "unit": "substeps/s", "ms_per_step": round(ms_e2e_serial, 4),
                           "mode": "one rollout through host buffers: each substep's input is "
                                   "the previous substep's output, copied in and out every "
                                   "substep (no overlap possible)"},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": "k_pcg_smem<double,true,true,true> (persistent cooperative, "
                                   "shared-memory resident)",
                         "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                         "frac": round(achieved / hbm, 4), "traffic": PCG_DRAM_BYTES,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, "
                                           "one launch of this workload "
                                           "(profiles/pcg_smem_coarse_128_apic.md)",
                         "peak_source": peak_kind,
                         "bytes_per_launch": round(float(np.mean(pcg_b)), 0),
                         "ms_per_launch": round(float(np.mean(pcg_ms)), 4)},
            "stages_ms": {k: round(float(stage_ms[i]), 4) for i, k in enumerate(
                ("bin_sort", "p2g", "forces_div", "pressure", "project", "g2p", "total",
                 "pcg_kernel"))},
            "stages_gbs": stage_gbs,
            "clocks": clk,
            "cpu_baseline": cpu,
            "fwd_adj": fwd_adj,
            "fwd_adj_apic": fwd_adj_apic,
            "batched": batched,
            "batched_fwd_adj": batched_adj,
            "other_configs": extra,
            "outflow_compaction": outflow,
            "reseed": reseed,
            "mesh": mesh,
        }
        print(json.dumps(line), flush=True)
    ranks.close()


def cpu_baseline(steps=1):
    """The CPU oracle on the same scene, all host threads, FP64 CG pressure
    to the same residual; one substep from the seeded state."""
    from oracle import oracle
    oracle.build()
    o = oracle.OracleFlip(GRID, GRID, GRID, transfer_mode="apic", par=True)
    m = o.marker
    m[oracle.sphere_sdf(GRID, GRID, GRID, o.dx, *SPHERE) <= 0.0] = 2
    pos = oracle.seed_box(o.dx, *BOX)
    o.set_particles(pos, np.zeros_like(pos))
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step(DT, pressure_iters=MAX_ITERS, pressure_solver="pcg64", tol=TOL)
    dt = time.perf_counter() - t0
    return {"value": round(steps / dt, 5), "unit": "substeps/s", "cores": oracle.num_threads(),
            "kind": "port", "sample": f"{steps} substep(s) of the 128^3 APIC scene from the "
            f"seeded state ({pos.shape[0]} particles), FP64 CG pressure to {TOL}, "
            f"{dt:.1f} s wall"}


def cpu_mesh_baseline(pos, dx):
    """The oracle's density field and marching-cubes surface of the same
    particles on one host thread (the mesh leg's CPU comparison)."""
    from oracle import mesh as om
    t0 = time.perf_counter()
    d = om.density_field(pos, (GRID, GRID, GRID), dx, 2, 0)
    _, ot = om.iso_surface_mc(d, 0.6, dx)
    return {"seconds": round(time.perf_counter() - t0, 3), "cores": 1, "tris": int(len(ot)),
            "sample": f"{GRID}^3 field of {len(pos)} particles, 2 blur passes, iso 0.6"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle
    oracle.build()
    o = oracle.OracleFlip(GRID, GRID, GRID, transfer_mode="apic", par=True)
    o.marker[oracle.sphere_sdf(GRID, GRID, GRID, o.dx, *SPHERE) <= 0.0] = 2
    pos = oracle.seed_box(o.dx, *BOX)
    o.set_particles(pos, np.zeros_like(pos))
    for _ in range(args.warmup):
        o.step(DT, pressure_iters=MAX_ITERS, pressure_solver="pcg64", tol=TOL)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.step(DT, pressure_iters=MAX_ITERS, pressure_solver="pcg64", tol=TOL)
    dt = time.perf_counter() - t0
    value = args.steps / dt
    cores = oracle.num_threads()
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 5), "unit": "substeps/s",
            "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1000 * dt / args.steps, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": WORKLOAD, "grid": GRID,
                                            "particles": int(pos.shape[0])},
            "cpu_baseline": {"value": round(value, 5), "unit": "substeps/s", "cores": cores,
                             "kind": "port",
                             "sample": "the CPU oracle (C port of the reference kernels, "
                                       "OpenMP) stepping the full scene; FP64 CG pressure to "
                                       f"{TOL} (the reference's FP32 PCG cannot reach it)"},
            "e2e": {"value": round(value, 5), "unit": "substeps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the forward+adjoint rollout timing")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched uneven-scenes timing")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the 64^3 and 256^3 single-scene timings")
    ap.add_argument("--no-fp64-check", action="store_true",
                    help="skip the FP64 residual and error measurements (profiling runs)")
    ap.add_argument("--grid", type=int, default=128,
                    help="grid side (smaller sides are for profiling captures only)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    global GRID
    GRID = args.grid
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
