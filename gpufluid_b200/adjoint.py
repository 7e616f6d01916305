"""Differentiable rollouts: the adjoint substep behind ``torch.autograd``.

The reference has no differentiation (it is only planned there).  This module
chains the hand-written adjoint substep of libgfb200 (``gf_step_record`` /
``gf_step_adjoint``: PIC transfer, cell labels held fixed within a substep)
into gradients of a loss of the final particle state with respect to an
initial control, with checkpoints every ``k`` substeps and recomputation in
between.

The drop-shaping problem (``DropShaping``):

* fluid: a sphere seeded with the jittered lattice in every cell whose centre
  lies inside it (8 per cell), PIC (flip_blend 0) or APIC transfer, no
  reseeding; under APIC the affine matrices start at zero and their adjoint is
  carried through the substeps beside those of positions and velocities;
* control: a cell-centred 3-component velocity field U (3, nx, ny, nz); each
  particle starts with the trilinearly sampled velocity v_p = sum_c N_pc U_c;
* loss: L = sum_c (rho_c(x_T) - rho*_c)^2 with rho the cell-centred
  trilinear unit-mass splat (``k_density_scatter``) after T substeps, and
  rho* the splat of the same sphere translated by ``shift``, blurred by a
  Gaussian of ``sigma`` cells.

Particles are re-sorted by cell every substep, so storage order changes from
substep to substep (``pid`` records each slot's particle).  Within a
recomputed segment the records are mutually consistent; across segment
boundaries the adjoint is carried by particle id, because float-atomic P2G
sums make a recomputation differ from the first forward pass at the last bit.
"""
from __future__ import annotations

import ctypes
import time

import numpy as np
import torch

from . import _lib
from . import scene as _scene
from .solver import FlipSolver3D


def gaussian_blur(field: np.ndarray, sigma: float) -> np.ndarray:
    """Separable Gaussian blur (truncated at 4 sigma, zero outside)."""
    r = int(np.ceil(4.0 * sigma))
    x = np.arange(-r, r + 1, dtype=np.float64)
    k = np.exp(-0.5 * (x / sigma) ** 2)
    k /= k.sum()
    out = field.astype(np.float64)
    for ax in range(3):
        out = np.apply_along_axis(lambda m: np.convolve(m, k, mode="same"), ax, out)
    return out


class DropShaping:
    """Loss of the final density against a translated, blurred target."""

    def __init__(self, n=64, T=40, dt=1.0 / 240.0, k=10, center=(0.5, 0.35, 0.5), radius=0.15,
                 shift=(0.15, 0.1, 0.0), sigma=1.5, ppc=8, device="cuda",
                 pressure_solver="pcg_refined", tol=1e-9, max_iters=4000, transfer="pic"):
        if transfer not in ("pic", "apic"):
            raise ValueError("the adjoint substep supports transfer 'pic' and 'apic'")
        self.n, self.T, self.dt, self.k = n, T, dt, k
        self.transfer = transfer
        self.device = torch.device(device)
        self.solver = FlipSolver3D(n, n, n, transfer_mode=transfer, flip_blend=0.0,
                                   pressure_tol=tol, device=device)
        s = self.solver
        self.rho_shape = (n, n, n)        # splat / target buffer
        self.control_shape = (3, n, n, n)
        x0 = _scene.seed_sphere_positions(n, n, n, s.dx, center, radius, ppc)
        s._set_particles(pos=x0, vel=np.zeros_like(x0))
        self.P = x0.shape[0]
        self.x0 = s._pos.clone()
        self.pressure_solver, self.max_iters = pressure_solver, max_iters
        self.prm = s._params(dt, max_iters, pressure_solver)
        shifted = torch.from_numpy(x0 + np.asarray(shift, np.float32)).to(self.device)
        rho_t = self.splat(shifted).cpu().numpy()
        self.target = torch.from_numpy(gaussian_blur(rho_t, sigma).astype(np.float32)).to(
            self.device)
        nb = ctypes.c_int64()
        _lib.check(s._L.gf_record_bytes(s._ctx, ctypes.byref(nb)), s._ctx, "gf_record_bytes")
        self.record_bytes = nb.value
        self.records = [torch.empty(nb.value, dtype=torch.uint8, device=self.device)
                        for _ in range(k)]
        self.labels_log = None
        self.last_timing = {}

    # ---------------------------------------------------------- primitives
    def _c(self, name, *args):
        s = self.solver
        s._set_stream()
        _lib.check(getattr(s._L, name)(s._ctx, *args), s._ctx, name)

    def splat(self, pos: torch.Tensor) -> torch.Tensor:
        rho = torch.empty(self.rho_shape, dtype=torch.float32, device=self.device)
        self._c("gf_density_splat", pos.data_ptr(), pos.shape[0], rho.data_ptr())
        return rho

    def _sample(self, control: torch.Tensor, pos: torch.Tensor) -> torch.Tensor:
        vel = torch.empty_like(pos)
        self._c("gf_sample_cells", control.data_ptr(), pos.data_ptr(), pos.shape[0],
                vel.data_ptr())
        return vel

    def _load(self, pos, vel, pid, C=None):
        s = self.solver
        s._pos.copy_(pos)
        s._vel.copy_(vel)
        s._pid.copy_(pid)
        if C is None:
            s._C.zero_()
        else:
            s._C.copy_(C)

    # ------------------------------------------------------------- forward
    def forward(self, control: torch.Tensor, keep_labels: bool = False):
        """Run T substeps from the control; returns (loss, checkpoints)."""
        s = self.solver
        control = control.detach().to(self.device, torch.float32).contiguous()
        pid0 = torch.arange(self.P, dtype=torch.int32, device=self.device)
        self._load(self.x0, self._sample(control, self.x0), pid0)
        ckpts = []
        labels = [] if keep_labels else None
        for t in range(self.T):
            if t % self.k == 0:
                ckpts.append((s._pos.clone(), s._vel.clone(), s._pid.clone(), s._C.clone()))
            self._c("gf_step", ctypes.byref(self.prm))
            if keep_labels:
                labels.append(s._label.clone())
        rho = self.splat(s._pos)
        loss = float(((rho.double() - self.target.double()) ** 2).sum().item())
        self.labels_log = labels
        return loss, ckpts

    # ------------------------------------------------------------ backward
    def backward(self, control: torch.Tensor, ckpts):
        """Gradient of the loss with respect to the control (3, n, n, n)."""
        s = self.solver
        P, dev = self.P, self.device
        control = control.detach().to(dev, torch.float32).contiguous()
        apic = self.transfer == "apic"
        xbar = torch.zeros((P, 3), dtype=torch.float32, device=dev)
        vbar = torch.zeros_like(xbar)
        xin = torch.empty_like(xbar)
        vin = torch.empty_like(xbar)
        Cbar = torch.zeros((P, 9), dtype=torch.float32, device=dev)
        Cin = torch.empty_like(Cbar)
        carry_x = carry_v = carry_C = None  # adjoint by particle id across segments
        nseg = len(ckpts)
        for seg in reversed(range(nseg)):
            t0 = seg * self.k
            steps = min(self.k, self.T - t0)
            self._load(*ckpts[seg])
            for i in range(steps):
                self._c("gf_step_record", ctypes.byref(self.prm), self.records[i].data_ptr())
            if seg == nseg - 1:
                rho = self.splat(s._pos)
                rho_bar = (2.0 * (rho - self.target)).contiguous()
                self._c("gf_density_splat_adjoint", s._pos.data_ptr(), P, rho_bar.data_ptr(),
                        xbar.data_ptr())
                vbar.zero_()
                Cbar.zero_()
            else:  # bring the id-ordered adjoint into this recomputation's slot order
                idx = s._pid.long()
                xbar.copy_(carry_x[idx])
                vbar.copy_(carry_v[idx])
                Cbar.copy_(carry_C[idx])
            for i in reversed(range(steps)):
                if apic:
                    self._c("gf_step_adjoint_apic", ctypes.byref(self.prm),
                            self.records[i].data_ptr(), xbar.data_ptr(), vbar.data_ptr(),
                            Cbar.data_ptr(), xin.data_ptr(), vin.data_ptr(), Cin.data_ptr())
                    Cbar, Cin = Cin, Cbar
                else:
                    self._c("gf_step_adjoint", ctypes.byref(self.prm),
                            self.records[i].data_ptr(), xbar.data_ptr(), vbar.data_ptr(),
                            xin.data_ptr(), vin.data_ptr())
                xbar, xin = xin, xbar
                vbar, vin = vin, vbar
            # xbar, vbar (, Cbar) are now in the storage order of checkpoint seg
            idx = ckpts[seg][2].long()
            carry_x = torch.empty_like(xbar)
            carry_v = torch.empty_like(vbar)
            carry_C = torch.empty_like(Cbar)
            carry_x[idx] = xbar
            carry_v[idx] = vbar
            carry_C[idx] = Cbar
        # checkpoint 0 holds the particles in id order: carry is v(0)'s adjoint
        # (C(0) = 0 does not depend on the control)
        grad = torch.empty(self.control_shape, dtype=torch.float32, device=dev)
        self._c("gf_sample_cells_adjoint", self.x0.data_ptr(), P, carry_v.data_ptr(),
                grad.data_ptr())
        return grad

    def loss_and_grad(self, control: torch.Tensor):
        torch.cuda.synchronize(self.device)
        t0 = time.perf_counter()
        loss, ckpts = self.forward(control)
        torch.cuda.synchronize(self.device)
        t1 = time.perf_counter()
        grad = self.backward(control, ckpts)
        torch.cuda.synchronize(self.device)
        t2 = time.perf_counter()
        self.last_timing = {"forward_s": t1 - t0, "backward_s": t2 - t1}
        return loss, grad


class BatchedDropShaping(DropShaping):
    """The drop-shaping problem on many scenes of uneven sizes at once (one
    batch context: every substep, adjoint substep, splat and sampling is one
    launch per kernel for all scenes).  Scene s is the single-scene problem at
    side sides[s] (the same sphere, shift and blur in unit coordinates); the
    control is each scene's (3, n, n, n) field concatenated (flat), the loss
    the sum of the scenes' losses."""

    def __init__(self, sides, T=40, dt=1.0 / 240.0, k=10, center=(0.5, 0.35, 0.5), radius=0.15,
                 shift=(0.15, 0.1, 0.0), sigma=1.5, ppc=8, device="cuda",
                 pressure_solver="pcg_refined", tol=1e-9, max_iters=4000, transfer="pic"):
        from .batch import BatchedFlip3D
        if transfer not in ("pic", "apic"):
            raise ValueError("the adjoint substep supports transfer 'pic' and 'apic'")
        self.sides = [int(n) for n in sides]
        self.n = None
        self.T, self.dt, self.k = T, dt, k
        self.transfer = transfer
        self.device = torch.device(device)
        self.solver = BatchedFlip3D([(n, n, n) for n in self.sides], transfer_mode=transfer,
                                    flip_blend=0.0, pressure_tol=tol, device=device)
        s = self.solver
        for i, n in enumerate(self.sides):
            s.set_particles(i, _scene.seed_sphere_positions(n, n, n, 1.0 / n, center, radius, ppc))
        self.P = s.n_particles
        self.x0 = s._pos.clone()
        self.cell0 = [L["cell0"] for L in s.layout]
        ncell = s.totals["ncell"]
        self.rho_shape = (ncell,)
        self.control_shape = (3 * ncell,)
        self.pressure_solver, self.max_iters = pressure_solver, max_iters
        self.prm = s._params(dt, max_iters, pressure_solver)
        shifted = torch.from_numpy(self.x0.cpu().numpy() + np.asarray(shift, np.float32)).to(
            self.device)
        rho_t = self.splat(shifted).cpu().numpy()
        tgt = np.empty(ncell, np.float32)
        for i, n in enumerate(self.sides):
            c0 = self.cell0[i]
            tgt[c0:c0 + n ** 3] = gaussian_blur(rho_t[c0:c0 + n ** 3].reshape(n, n, n),
                                                sigma).ravel()
        self.target = torch.from_numpy(tgt).to(self.device)
        nb = ctypes.c_int64()
        _lib.check(s._L.gf_record_bytes(s._ctx, ctypes.byref(nb)), s._ctx, "gf_record_bytes")
        self.record_bytes = nb.value
        self.records = [torch.empty(nb.value, dtype=torch.uint8, device=self.device)
                        for _ in range(k)]
        self.labels_log = None
        self.last_timing = {}

    def scene_control(self, control: torch.Tensor, s: int) -> torch.Tensor:
        """View of scene s's (3, n, n, n) block of a flat control (or gradient)."""
        n = self.sides[s]
        c0 = 3 * self.cell0[s]
        return control[c0:c0 + 3 * n ** 3].view(3, n, n, n)

    def scene_losses(self) -> np.ndarray:
        """Per-scene losses at the current (final) particle state."""
        rho = self.splat(self.solver._pos)
        r = ((rho.double() - self.target.double()) ** 2).cpu().numpy()
        return np.array([r[c0:c0 + n ** 3].sum() for c0, n in zip(self.cell0, self.sides)])


class RolloutLoss(torch.autograd.Function):
    """``loss = RolloutLoss.apply(control, problem)``: the forward pass runs the
    rollout keeping only the checkpoints; backward recomputes each segment and
    runs the adjoint substeps."""

    @staticmethod
    def forward(ctx, control, problem):
        loss, ckpts = problem.forward(control)
        ctx.problem = problem
        ctx.ckpts = ckpts
        ctx.save_for_backward(control)
        return torch.tensor(loss, dtype=torch.float64, device=control.device)

    @staticmethod
    def backward(ctx, gout):
        (control,) = ctx.saved_tensors
        grad = ctx.problem.backward(control, ctx.ckpts)
        return (grad * gout.to(grad.dtype)).to(control.dtype), None
