"""The allocation-free Jacobi entry point, gf_jacobi_noalloc.

It serves callers that may not allocate device memory (a host that owns all
device allocations through its own pool and forbids libraries from calling
cudaMalloc / cudaFree): its scratch is a static device array, so it must give
exactly what the regular context-based gf_pressure(GF_JACOBI) gives on the
same inputs -- also on a second call in a row, which reuses the array the
first call left behind.
This file is collected last so a failure here cannot hide any other test.
"""
import ctypes

import numpy as np
import pytest

from helpers import assert_bitexact

pytestmark = pytest.mark.gpu


def _scene(nx, ny, nz, seed):
    """Walls, a solid sphere, fluid in the lower part, seeded divergence."""
    rng = np.random.default_rng(seed)
    lab = np.zeros((nx, ny, nz), np.uint8)
    lab[0, :, :] = 2; lab[-1, :, :] = 2
    lab[:, 0, :] = 2; lab[:, -1, :] = 2
    lab[:, :, 0] = 2; lab[:, :, -1] = 2
    fluid = np.zeros_like(lab, dtype=bool)
    fluid[1:-1, 1:int(ny * 0.6), 1:-1] = True
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    sphere = (ii - nx * 0.6) ** 2 + (jj - ny * 0.3) ** 2 + (kk - nz * 0.5) ** 2 < (0.15 * nx) ** 2
    lab[fluid & (lab != 2)] = 1
    lab[sphere] = 2
    div = np.where(lab == 1, rng.normal(0.0, 1.0, lab.shape), 0.0).astype(np.float32)
    return lab, div


def _with_context(gf, lab, div, iters):
    """gf_pressure(GF_JACOBI) through a solver context (allocating path)."""
    import torch
    from gpufluid_b200 import _lib
    nx, ny, nz = lab.shape
    s = gf.FlipSolver3D(nx, ny, nz)
    s._label.copy_(torch.from_numpy(lab))
    s.div.copy_(torch.from_numpy(div))
    prm = _lib.StepParams(1 / 240.0, -9.81, 1.0, 0.95, 0, _lib.GF_JACOBI, iters, 10, 1e-4, -1, 0)
    s._set_stream()
    it = ctypes.c_int32()
    _lib.check(s._L.gf_pressure(s._ctx, ctypes.byref(prm), ctypes.byref(it)), s._ctx,
               "gf_pressure")
    return s._p.cpu().numpy()


def _noalloc(lab, div, iters):
    import torch
    from gpufluid_b200 import _lib
    L = _lib.load()
    lab_d = torch.from_numpy(lab).cuda()
    div_d = torch.from_numpy(div).cuda()
    p_d = torch.full(lab.shape, 7.0, dtype=torch.float32, device="cuda")  # garbage in
    stream = torch.cuda.current_stream().cuda_stream
    st = L.gf_jacobi_noalloc(*lab.shape, lab_d.data_ptr(), div_d.data_ptr(), p_d.data_ptr(),
                             iters, stream)
    assert st == _lib.GF_OK, st
    torch.cuda.synchronize()
    return p_d.cpu().numpy()


def test_noalloc_matches_context_entry_point_twice_in_a_row(gf):
    lab1, div1 = _scene(40, 32, 48, seed=1)
    lab2, div2 = _scene(24, 36, 20, seed=2)
    # two calls in a row: odd then even sweep counts, different grids
    for lab, div, iters in ((lab1, div1, 37), (lab2, div2, 20)):
        want = _with_context(gf, lab, div, iters)
        got = _noalloc(lab, div, iters)
        assert np.abs(want).max() > 0
        assert_bitexact(f"p ({lab.shape}, {iters} sweeps)", got, want)


def test_noalloc_rejects_grids_beyond_its_scratch(gf):
    import torch
    from gpufluid_b200 import _lib
    L = _lib.load()
    big = (130, 130, 130)
    assert big[0] * big[1] * big[2] > _lib.GF_NOALLOC_MAX_CELLS
    dummy = torch.zeros(4, device="cuda")
    st = L.gf_jacobi_noalloc(*big, dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), 5,
                             torch.cuda.current_stream().cuda_stream)
    assert st == _lib.GF_INVALID_ARG
