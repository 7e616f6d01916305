"""ctypes binding of libgfb200.so (the C ABI declared in include/gfb200.h).

The shared library is loaded from this package directory; it is built by
``python -m gpufluid_b200.build``.  There is no fallback: if the library is
missing or no sm_100 device is present, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
# GFB200_LIB=libgfb200_checked.so selects the bounds-checked build
LIB_VARIANTS = ("libgfb200.so", "libgfb200_checked.so")
_variant = os.environ.get("GFB200_LIB", LIB_VARIANTS[0])
if _variant not in LIB_VARIANTS:
    raise RuntimeError(f"GFB200_LIB={_variant!r}: expected one of {LIB_VARIANTS}")
LIB_PATH = os.path.join(HERE, _variant)
HEADER = os.path.join(os.path.dirname(HERE), "include", "gfb200.h")

GF_OK, GF_INVALID_ARG, GF_CUDA_ERROR, GF_NOT_CONVERGED = 0, 1, 2, 3
GF_NAN, GF_BREAKDOWN, GF_TIMEOUT, GF_NO_DEVICE = 4, 5, 6, 7
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "CUDA_ERROR", 3: "NOT_CONVERGED", 4: "NAN",
                5: "BREAKDOWN", 6: "TIMEOUT", 7: "NO_DEVICE"}

GF_FLIP, GF_PIC, GF_APIC = 0, 1, 2
GF_JACOBI, GF_GSRB, GF_PCG, GF_PCG_REFINED = 0, 1, 2, 3
TRANSFER = {"flip": GF_FLIP, "pic": GF_PIC, "apic": GF_APIC}
SOLVER = {"jacobi": GF_JACOBI, "gsrb": GF_GSRB, "pcg": GF_PCG, "pcg_refined": GF_PCG_REFINED}


class GfError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"gfb200 {STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_fp = ctypes.POINTER(ctypes.c_float)
_vp = ctypes.c_void_p


class GridDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
                ("dx", ctypes.c_float), ("dom", ctypes.c_float * 3)]


class Fields(ctypes.Structure):
    _fields_ = [(n, _vp) for n in ("u", "v", "w", "uw", "vw", "ww", "us", "vs", "ws", "p",
                                   "div", "label", "solid_u", "solid_v", "solid_w")]


class Particles(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("pos", _vp), ("vel", _vp), ("C", _vp), ("pid", _vp)]


class StepParams(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_float), ("gravity", ctypes.c_float), ("rho", ctypes.c_float),
                ("flip_blend", ctypes.c_float), ("transfer", ctypes.c_int32),
                ("solver", ctypes.c_int32), ("max_iters", ctypes.c_int32),
                ("check_every", ctypes.c_int32), ("tol", ctypes.c_double),
                ("rhs_sign", ctypes.c_int32), ("flags", ctypes.c_int32)]


GF_FLAG_GLOBAL_PCG = 1
GF_FLAG_TRACE = 2
GF_FLAG_SGS_SHIFT = 2  # bits 2-3: tile-local symmetric Gauss-Seidel sweeps
GF_FLAG_COARSE = 16    # tile coarse correction of the shared-memory PCG
GF_FLAG_TEST_STALL = 64  # test only: the first grid reduction of the PCG runs out its wait
GF_FLAG_WARM_START = 128  # refined PCG starts from the previous pressure
GF_NOALLOC_MAX_CELLS = 2097152


class PressureInfo(ctypes.Structure):
    _fields_ = [("iters", ctypes.c_int32), ("replacements", ctypes.c_int32),
                ("status", ctypes.c_int32), ("n_active_tiles", ctypes.c_int32),
                ("n_fluid", ctypes.c_int64), ("relres", ctypes.c_double),
                ("kernel", ctypes.c_int32), ("coarse", ctypes.c_int32)]


class Health(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in ("worst_status", "solves", "not_converged",
                                              "failed", "last_status", "wait_timeouts")]


class SceneLayout(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("cell0", "fu0", "fv0", "fw0", "tile0", "ntiles",
                                              "fslot0")]


class BatchTotals(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("ncell", "nu", "nv", "nw", "ntiles", "nslot")]


class TuneInfo(ctypes.Structure):
    _fields_ = [("g2p_threads", ctypes.c_int32), ("grid_threads", ctypes.c_int32),
                ("grid_blocks_per_sm", ctypes.c_int32), ("pcg_blocks_per_sm", ctypes.c_int32),
                ("step_ms_before", ctypes.c_float), ("step_ms_after", ctypes.c_float),
                ("p2g_tiles_k", ctypes.c_int32), ("g2p_tiles_k", ctypes.c_int32),
                ("p2g_map", ctypes.c_int32)]


GF_MESH_TRILINEAR, GF_MESH_CUBIC, GF_MESH_SDF = 0, 1, 2
MESH_METHOD = {"trilinear": GF_MESH_TRILINEAR, "cubic": GF_MESH_CUBIC, "sdf": GF_MESH_SDF}
GF_SURFACE_MARCHING_CUBES, GF_SURFACE_MARCHING_TETRAHEDRA = 0, 1
SURFACE = {"marching_cubes": GF_SURFACE_MARCHING_CUBES,
           "marching_tetrahedra": GF_SURFACE_MARCHING_TETRAHEDRA}
GF_MESH_SMOOTH_LAPLACIAN, GF_MESH_SMOOTH_TAUBIN = 0, 1
MESH_SMOOTH = {"laplacian": GF_MESH_SMOOTH_LAPLACIAN, "taubin": GF_MESH_SMOOTH_TAUBIN}


class MeshParams(ctypes.Structure):
    _fields_ = [("method", ctypes.c_int32), ("smooth_passes", ctypes.c_int32),
                ("wall_margin_cells", ctypes.c_int32), ("cubic_radius_cells", ctypes.c_float),
                ("sdf_particle_radius_cells", ctypes.c_float),
                ("sdf_search_radius_cells", ctypes.c_float)]


_SIGS = {
    "gf_create": ([ctypes.POINTER(GridDesc), ctypes.c_int64, ctypes.POINTER(_vp)], ctypes.c_int),
    "gf_destroy": ([_vp], ctypes.c_int),
    "gf_reserve_particles": ([_vp, ctypes.c_int64], ctypes.c_int),
    "gf_bind": ([_vp, ctypes.POINTER(Fields), ctypes.POINTER(Particles)], ctypes.c_int),
    "gf_set_stream": ([_vp, _vp], ctypes.c_int),
    "gf_last_error": ([_vp], ctypes.c_char_p),
    "gf_launch_count": ([_vp], ctypes.c_int64),
    "gf_bin": ([_vp, ctypes.c_int32], ctypes.c_int),
    "gf_p2g": ([_vp, ctypes.c_int32], ctypes.c_int),
    "gf_forces_div": ([_vp, ctypes.c_float, ctypes.c_float, ctypes.c_float], ctypes.c_int),
    "gf_pressure": ([_vp, ctypes.POINTER(StepParams), ctypes.POINTER(ctypes.c_int32)],
                    ctypes.c_int),
    "gf_project": ([_vp, ctypes.c_float, ctypes.c_float], ctypes.c_int),
    "gf_g2p": ([_vp, ctypes.c_int32, ctypes.c_float, ctypes.c_float], ctypes.c_int),
    "gf_step": ([_vp, ctypes.POINTER(StepParams)], ctypes.c_int),
    "gf_graph_capture": ([_vp, ctypes.POINTER(StepParams), ctypes.POINTER(_vp)], ctypes.c_int),
    "gf_graph_replay": ([_vp, _vp], ctypes.c_int),
    "gf_graph_destroy": ([_vp], ctypes.c_int),
    "gf_pressure_result": ([_vp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double),
                            ctypes.POINTER(ctypes.c_int32)], ctypes.c_int),
    "gf_bin_read": ([_vp, _vp, _vp, _vp, ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
    "gf_enable_timing": ([_vp, ctypes.c_int32], ctypes.c_int),
    "gf_stage_times": ([_vp, _fp], ctypes.c_int),
    "gf_active_tiles": ([_vp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(_vp)], ctypes.c_int),
    "gf_vmax": ([_vp, _fp], ctypes.c_int),
    "gf_outflow_compact": ([_vp, _vp, _vp, ctypes.c_int64, _fp, ctypes.c_int32, _vp, _vp,
                            ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
    "gf_compact_alive": ([_vp, _vp, _vp, ctypes.c_int64, _vp, _vp, _vp,
                          ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
    "gf_reseed_mark": ([_vp, ctypes.c_int32, _vp, _vp], ctypes.c_int),
    "gf_reseed_deficit": ([_vp, _vp, _vp, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)],
                          ctypes.c_int),
    "gf_reseed_emit": ([_vp, _vp, _vp, ctypes.c_int32, _vp, _vp], ctypes.c_int),
    "gf_pressure_stats": ([_vp, ctypes.POINTER(PressureInfo)], ctypes.c_int),
    "gf_health_read": ([_vp, ctypes.c_int32, ctypes.POINTER(Health)], ctypes.c_int),
    "gf_bounds_status": ([ctypes.c_int32, ctypes.POINTER(ctypes.c_int64),
                          ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)],
                         ctypes.c_int),
    "gf_pcg_trace": ([_vp, _vp, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)], ctypes.c_int),
    "gf_record_bytes": ([_vp, ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
    "gf_step_record": ([_vp, ctypes.POINTER(StepParams), _vp], ctypes.c_int),
    "gf_step_adjoint": ([_vp, ctypes.POINTER(StepParams), _vp, _vp, _vp, _vp, _vp], ctypes.c_int),
    "gf_step_adjoint_apic": ([_vp, ctypes.POINTER(StepParams), _vp, _vp, _vp, _vp, _vp, _vp, _vp],
                             ctypes.c_int),
    "gf_density_splat": ([_vp, _vp, ctypes.c_int64, _vp], ctypes.c_int),
    "gf_density_splat_adjoint": ([_vp, _vp, ctypes.c_int64, _vp, _vp], ctypes.c_int),
    "gf_sample_cells": ([_vp, _vp, _vp, ctypes.c_int64, _vp], ctypes.c_int),
    "gf_sample_cells_adjoint": ([_vp, _vp, ctypes.c_int64, _vp, _vp], ctypes.c_int),
    "gf_jacobi_noalloc": ([ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _vp, _vp, _vp,
                           ctypes.c_int32, _vp], ctypes.c_int),
    "gf_batch_plan": ([ctypes.POINTER(GridDesc), ctypes.c_int32, ctypes.POINTER(SceneLayout),
                       ctypes.POINTER(BatchTotals)], ctypes.c_int),
    "gf_batch_create": ([ctypes.POINTER(GridDesc), ctypes.c_int32, ctypes.c_int64,
                         ctypes.POINTER(_vp)], ctypes.c_int),
    "gf_batch_bind": ([_vp, ctypes.POINTER(Fields), ctypes.POINTER(Particles),
                       ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
    "gf_batch_pressure_stats": ([_vp, ctypes.POINTER(ctypes.c_int32),
                                 ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32)],
                                ctypes.c_int),
    "gf_autotune": ([_vp, ctypes.POINTER(StepParams), ctypes.POINTER(TuneInfo)], ctypes.c_int),
    "gf_get_tune": ([_vp, ctypes.POINTER(TuneInfo)], ctypes.c_int),
    "gf_set_tune": ([_vp, ctypes.POINTER(TuneInfo)], ctypes.c_int),
    "gf_mesher_create": ([ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_float, _vp,
                          ctypes.POINTER(_vp)], ctypes.c_int),
    "gf_mesher_destroy": ([_vp], ctypes.c_int),
    "gf_mesher_last_error": ([_vp], ctypes.c_char_p),
    "gf_mesher_set_stream": ([_vp, _vp], ctypes.c_int),
    "gf_mesher_field": ([_vp], _vp),
    "gf_mesher_launches": ([_vp], ctypes.c_int64),
    "gf_mesher_density": ([_vp, _vp, ctypes.c_int64, ctypes.POINTER(MeshParams)], ctypes.c_int),
    "gf_mesher_extract": ([_vp, _vp, ctypes.c_float, ctypes.POINTER(ctypes.c_int64),
                           ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
    "gf_mesher_copy": ([_vp, _vp, _vp], ctypes.c_int),
    "gf_mesher_copy_field": ([_vp, _vp], ctypes.c_int),
    "gf_mesher_set_inside_below": ([_vp, ctypes.c_int32], ctypes.c_int),
    "gf_mesher_set_surface": ([_vp, ctypes.c_int32], ctypes.c_int),
    "gf_marching_cubes_table": ([_vp, _vp, _vp], ctypes.c_int),
    "gf_mesher_smooth": ([_vp, _vp, ctypes.c_int64, _vp, ctypes.c_int64, ctypes.c_int32,
                          ctypes.c_int32, ctypes.c_double, ctypes.c_double], ctypes.c_int),
}

_lib = None


def header_symbols() -> list[str]:
    """Names of every function declared in include/gfb200.h."""
    with open(HEADER) as f:
        text = f.read()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|float \*|const char \*)\s*(gf_\w+)\s*\(", text,
                                 flags=re.M)))


def load():
    """Load libgfb200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with "
                               "`python -m gpufluid_b200.build` (nvcc, sm_100a)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
    return _lib


def check(status: int, ctx=None, what: str = ""):
    if status != GF_OK:
        msg = ""
        if ctx is not None:
            raw = load().gf_last_error(ctx)
            msg = raw.decode() if raw else ""
        raise GfError(status, f"{what}: {msg}" if what else msg)
