"""FP64 CPU forward of the PIC substep with frozen labels -- TEST INFRASTRUCTURE.

Used only by tests/ as the finite-difference reference for the adjoint
(central differences of this float64 forward along seeded directions).  The
substep restates the reference kernels in float64 with vectorised NumPy:

  P2G          k3_p2g + scatter_face      solver3d.py:72-114, gridmath.py:70-95
  normalize    k3_normalize               solver3d.py:121-142
  gravity, BC  k3_add_gravity, k3_enforce_solid_bc   :149-156, :758-799
  divergence   k3_compute_divergence      :846-871
  pressure     A p = -div solved directly (the system the reference iterates)
  gradient, BC k3_subtract_pressure_grad  :1364-1407
  G2P (PIC)    k3_g2p_and_advect with flip_blend 0, sample3   :1414-1463, gridmath.py:29-63
  advect       x + v dt clamped to [1.001 dx, dom - 1.001 dx]

with the cell labels of every substep supplied by the caller (the adjoint
holds them fixed), plus the control sampling and the density-splat loss, and
the reverse-mode derivative of all of it in float64 (``substep_adjoint``,
``grad``), itself checked against central differences; and the same for the
APIC transfer (P2G with the affine term C.(x_face - x_p), k3_p2g_apic
:1475-1588; G2P gathering velocity and C, k3_g2p_apic_advect :1591-1732):
``substep_apic``, ``substep_apic_adjoint``, ``loss_apic``, ``grad_apic``.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def _corner_weights(f, dims, clamp):
    """Trilinear corners of fractional coordinates f (P,3) in a grid of dims.
    clamp=True: sample3 semantics; False: scatter_face (drop out-of-range)."""
    f = f.copy()
    dims = np.asarray(dims)
    if clamp:
        f = np.clip(f, 0.0, dims.astype(np.float64))
    i0 = np.floor(f).astype(np.int64)
    if clamp:
        i0 = np.minimum(i0, dims - 1)
        i0 = np.maximum(i0, 0)
        i1 = np.minimum(i0 + 1, dims - 1)
        s = np.clip(f - i0, 0.0, 1.0)
    else:
        i1 = i0 + 1
        s = f - i0
    out_idx, out_w = [], []
    for a in range(2):
        for b in range(2):
            for c in range(2):
                ii = np.stack([(i0, i1)[a][:, 0], (i0, i1)[b][:, 1], (i0, i1)[c][:, 2]], 1)
                w = ((1 - s[:, 0]) if a == 0 else s[:, 0]) * \
                    ((1 - s[:, 1]) if b == 0 else s[:, 1]) * \
                    ((1 - s[:, 2]) if c == 0 else s[:, 2])
                ok = np.all((ii >= 0) & (ii < dims), axis=1)
                flat = (ii[:, 0] * dims[1] + ii[:, 1]) * dims[2] + ii[:, 2]
                out_idx.append(np.where(ok, flat, 0))
                out_w.append(np.where(ok, w, 0.0))
    return np.stack(out_idx, 1), np.stack(out_w, 1)


def _corner_weights_grad(f, dims, clamp):
    """As _corner_weights, plus d(weight)/df (P,8,3) in grid units; an axis
    whose coordinate is clamped (clamp=True) has zero derivative."""
    f = f.copy()
    dims = np.asarray(dims)
    gate = np.ones_like(f)
    if clamp:
        gate = ((f >= 0.0) & (f <= dims.astype(np.float64))).astype(np.float64)
        f = np.clip(f, 0.0, dims.astype(np.float64))
    i0 = np.floor(f).astype(np.int64)
    if clamp:
        i0 = np.maximum(np.minimum(i0, dims - 1), 0)
        i1 = np.minimum(i0 + 1, dims - 1)
        raw = f - i0
        gate = gate * ((raw >= 0.0) & (raw <= 1.0))
        s = np.clip(raw, 0.0, 1.0)
    else:
        i1 = i0 + 1
        s = f - i0
    idx, w, dw = [], [], []
    for a in range(2):
        for b in range(2):
            for c in range(2):
                ii = np.stack([(i0, i1)[a][:, 0], (i0, i1)[b][:, 1], (i0, i1)[c][:, 2]], 1)
                wx = (1 - s[:, 0]) if a == 0 else s[:, 0]
                wy = (1 - s[:, 1]) if b == 0 else s[:, 1]
                wz = (1 - s[:, 2]) if c == 0 else s[:, 2]
                sg = [(-1.0, 1.0)[a], (-1.0, 1.0)[b], (-1.0, 1.0)[c]]
                ok = np.all((ii >= 0) & (ii < dims), axis=1)
                flat = (ii[:, 0] * dims[1] + ii[:, 1]) * dims[2] + ii[:, 2]
                idx.append(np.where(ok, flat, 0))
                w.append(np.where(ok, wx * wy * wz, 0.0))
                d = np.stack([sg[0] * gate[:, 0] * wy * wz, sg[1] * gate[:, 1] * wx * wz,
                              sg[2] * gate[:, 2] * wx * wy], 1)
                dw.append(np.where(ok[:, None], d, 0.0))
    return np.stack(idx, 1), np.stack(w, 1), np.stack(dw, 1)


def _corners_apic(f, dims, clamp_idx):
    """Corner flat indices, integer corner coordinates (P,8,3), weights and
    d(weight)/df (P,8,3) with unclamped weights s = f - floor(f): clamp_idx
    True clamps each corner index into the grid (apic gather, :1626-1724),
    False drops corners outside it (scatter_face with positions, :1475-1588)."""
    dims = np.asarray(dims)
    i0 = np.floor(f).astype(np.int64)
    s = f - i0
    idx, ijk, w, dw = [], [], [], []
    for a in range(2):
        for b in range(2):
            for c in range(2):
                ii = i0 + np.array([a, b, c])
                if clamp_idx:
                    ii = np.minimum(np.maximum(ii, 0), dims - 1)
                    ok = np.ones(len(f), bool)
                else:
                    ok = np.all((ii >= 0) & (ii < dims), axis=1)
                wx = (1 - s[:, 0]) if a == 0 else s[:, 0]
                wy = (1 - s[:, 1]) if b == 0 else s[:, 1]
                wz = (1 - s[:, 2]) if c == 0 else s[:, 2]
                sg = [(-1.0, 1.0)[a], (-1.0, 1.0)[b], (-1.0, 1.0)[c]]
                flat = (ii[:, 0] * dims[1] + ii[:, 1]) * dims[2] + ii[:, 2]
                idx.append(np.where(ok, flat, 0))
                ijk.append(ii)
                w.append(np.where(ok, wx * wy * wz, 0.0))
                d = np.stack([sg[0] * wy * wz, sg[1] * wx * wz, sg[2] * wx * wy], 1)
                dw.append(np.where(ok[:, None], d, 0.0))
    return np.stack(idx, 1), np.stack(ijk, 1), np.stack(w, 1), np.stack(dw, 1)


class PicFP64:
    def __init__(self, n, dx=None, gravity=-9.81, rho=1.0):
        self.n = n
        self.dx = dx if dx is not None else 1.0 / n
        self.g, self.rho = gravity, rho
        self.dims = [(n + 1, n, n), (n, n + 1, n), (n, n, n + 1)]
        self.dom = np.array([n * self.dx] * 3, np.float32).astype(np.float64)
        self._solvers = {}

    # -- pressure system on frozen labels (cached per substep key) --------
    def _system(self, key, lab):
        if key in self._solvers:
            return self._solvers[key]
        n = self.n
        fl = lab == 1
        idx = -np.ones(lab.shape, np.int64)
        idx[fl] = np.arange(int(fl.sum()))
        rows, cols, vals = [], [], []
        diag = np.zeros(lab.shape)
        for ax in range(3):
            for sh in (-1, 1):
                nb_lab = np.full(lab.shape, 2, lab.dtype)
                nb_idx = -np.ones(lab.shape, np.int64)
                src = [slice(None)] * 3
                dst = [slice(None)] * 3
                if sh == -1:
                    dst[ax], src[ax] = slice(1, None), slice(None, -1)
                else:
                    dst[ax], src[ax] = slice(None, -1), slice(1, None)
                nb_lab[tuple(dst)] = lab[tuple(src)]
                nb_idx[tuple(dst)] = idx[tuple(src)]
                diag += nb_lab != 2
                m = fl & (nb_lab == 1)
                rows.append(idx[m]); cols.append(nb_idx[m]); vals.append(-np.ones(int(m.sum())))
        rows.append(idx[fl]); cols.append(idx[fl]); vals.append(diag[fl])
        nf = int(fl.sum())
        A = sp.csc_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                          shape=(nf, nf))
        solve = spla.factorized(A) if nf else (lambda b: b)
        self._solvers[key] = (fl, idx, solve)
        return self._solvers[key]

    def _bc_masks(self, lab):
        n = self.n
        masks = []
        for c in range(3):
            d = self.dims[c]
            m = np.zeros(d, bool)
            solid = lab == 2
            if c == 0:
                left = np.zeros(d, bool); right = np.zeros(d, bool)
                left[0] = True; left[1:] = solid
                right[n] = True; right[:n] |= solid
            elif c == 1:
                left = np.zeros(d, bool); right = np.zeros(d, bool)
                left[:, 0] = True; left[:, 1:] = solid
                right[:, n] = True; right[:, :n] |= solid
            else:
                left = np.zeros(d, bool); right = np.zeros(d, bool)
                left[:, :, 0] = True; left[:, :, 1:] = solid
                right[:, :, n] = True; right[:, :, :n] |= solid
            m = left | right
            masks.append(m)
        return masks

    def substep(self, x, v, lab, dt, key):
        n, dx = self.n, self.dx
        gx = x / dx
        offs = [np.array([0.0, 0.5, 0.5]), np.array([0.5, 0.0, 0.5]), np.array([0.5, 0.5, 0.0])]
        masks = self._bc_masks(lab)
        u = []
        for c in range(3):
            idx, w = _corner_weights(gx - offs[c], self.dims[c], clamp=False)
            size = int(np.prod(self.dims[c]))
            m = np.bincount(idx.ravel(), weights=w.ravel(), minlength=size)
            q = np.bincount(idx.ravel(), weights=(w * v[:, c:c + 1]).ravel(), minlength=size)
            un = np.where(m > 1e-8, q / np.where(m > 1e-8, m, 1.0), 0.0).reshape(self.dims[c])
            if c == 1:
                un = un + self.g * dt
            un[masks[c]] = 0.0
            u.append(un)
        fl = lab == 1
        s = self.rho * dx / dt
        div = (u[0][1:] - u[0][:-1]) + (u[1][:, 1:] - u[1][:, :-1]) + (u[2][:, :, 1:] - u[2][:, :, :-1])
        div = np.where(fl, div * s, 0.0)
        fl, idx, solve = self._system(key, lab)
        p = np.zeros(lab.shape)
        if fl.any():
            p[fl] = solve(-div[fl])
        k = dt / (self.rho * dx)
        for c in range(3):
            pl = np.zeros(self.dims[c]); pr = np.zeros(self.dims[c])
            ml = np.full(self.dims[c], 2, lab.dtype); mr = np.full(self.dims[c], 2, lab.dtype)
            sl = [slice(None)] * 3; sr = [slice(None)] * 3
            sl[c] = slice(1, None); sr[c] = slice(None, -1)
            pl[tuple(sl)] = p; ml[tuple(sl)] = lab
            pr[tuple(sr)] = p; mr[tuple(sr)] = lab
            elig = ((ml == 1) | (mr == 1)) & (ml != 2) & (mr != 2)
            pl = np.where(ml == 1, pl, 0.0); pr = np.where(mr == 1, pr, 0.0)
            u[c] = np.where(elig, u[c] - k * (pr - pl), u[c])
            u[c][masks[c]] = 0.0
        vn = np.zeros_like(v)
        for c in range(3):
            idx, w = _corner_weights(gx - offs[c], self.dims[c], clamp=True)
            vn[:, c] = (w * u[c].ravel()[idx]).sum(1)
        eps = dx * 1.001
        xn = np.clip(x + vn * dt, eps, self.dom - eps)
        return xn, vn

    def substep_adjoint(self, x, v, lab, dt, key, xbar, vbar):
        """Reverse-mode derivative of substep(x, v, lab, dt, key): given the
        adjoints (xbar, vbar) of its outputs, the adjoints of its inputs."""
        n, dx = self.n, self.dx
        gx = x / dx
        offs = [np.array([0.0, 0.5, 0.5]), np.array([0.5, 0.0, 0.5]), np.array([0.5, 0.5, 0.0])]
        masks = self._bc_masks(lab)
        pw, un, ms = [], [], []
        u = []
        for c in range(3):
            idx, w, dw = _corner_weights_grad(gx - offs[c], self.dims[c], clamp=False)
            size = int(np.prod(self.dims[c]))
            m = np.bincount(idx.ravel(), weights=w.ravel(), minlength=size)
            q = np.bincount(idx.ravel(), weights=(w * v[:, c:c + 1]).ravel(), minlength=size)
            uc = np.where(m > 1e-8, q / np.where(m > 1e-8, m, 1.0), 0.0)
            pw.append((idx, w, dw)); un.append(uc); ms.append(m)
            uu = uc.reshape(self.dims[c]) + (self.g * dt if c == 1 else 0.0)
            uu[masks[c]] = 0.0
            u.append(uu)
        fl = lab == 1
        s = self.rho * dx / dt
        div = (u[0][1:] - u[0][:-1]) + (u[1][:, 1:] - u[1][:, :-1]) + (u[2][:, :, 1:] - u[2][:, :, :-1])
        div = np.where(fl, div * s, 0.0)
        fl, _, solve = self._system(key, lab)
        p = np.zeros(lab.shape)
        if fl.any():
            p[fl] = solve(-div[fl])
        k = dt / (self.rho * dx)
        u3, elig_l = [], []
        for c in range(3):
            pl = np.zeros(self.dims[c]); pr = np.zeros(self.dims[c])
            ml = np.full(self.dims[c], 2, lab.dtype); mr = np.full(self.dims[c], 2, lab.dtype)
            sl = [slice(None)] * 3; sr = [slice(None)] * 3
            sl[c] = slice(1, None); sr[c] = slice(None, -1)
            pl[tuple(sl)] = p; ml[tuple(sl)] = lab
            pr[tuple(sr)] = p; mr[tuple(sr)] = lab
            elig = ((ml == 1) | (mr == 1)) & (ml != 2) & (mr != 2) & ~masks[c]
            pl = np.where(ml == 1, pl, 0.0); pr = np.where(mr == 1, pr, 0.0)
            uc = np.where(elig, u[c] - k * (pr - pl), u[c])
            uc[masks[c]] = 0.0
            u3.append(uc); elig_l.append((elig, ml, mr))
        # G2P and advection
        g2p = [_corner_weights_grad(gx - offs[c], self.dims[c], clamp=True) for c in range(3)]
        vn = np.stack([(g2p[c][1] * u3[c].ravel()[g2p[c][0]]).sum(1) for c in range(3)], 1)
        eps = dx * 1.001
        xr = x + vn * dt
        free = (xr >= eps) & (xr <= self.dom - eps)
        xb = np.where(free, xbar, 0.0)
        vb = vbar + np.where(free, dt * xbar, 0.0)
        ub3 = []
        for c in range(3):
            idx, w, dw = g2p[c]
            size = int(np.prod(self.dims[c]))
            ub3.append(np.bincount(idx.ravel(), weights=(w * vb[:, c:c + 1]).ravel(),
                                   minlength=size).reshape(self.dims[c]))
            xb += (dw * (u3[c].ravel()[idx] * vb[:, c:c + 1])[:, :, None]).sum(1) / dx
        # projection: u3 = where(elig, u - k (pr - pl), u), masked faces 0
        pbar = np.zeros(lab.shape)
        ub = []
        for c in range(3):
            elig, ml, mr = elig_l[c]
            g = np.where(elig, ub3[c], 0.0)
            sl = [slice(None)] * 3; sr = [slice(None)] * 3
            sl[c] = slice(1, None); sr[c] = slice(None, -1)
            # face f: right cell f gets -k, left cell f-1 gets +k
            pbar += np.where(fl, -k * g[tuple(sr)] * (mr[tuple(sr)] == 1), 0.0)
            pbar += np.where(fl, k * g[tuple(sl)] * (ml[tuple(sl)] == 1), 0.0)
            ub.append(np.where(masks[c], 0.0, ub3[c]))
        lam = np.zeros(lab.shape)
        if fl.any():
            lam[fl] = solve(pbar[fl])
        divbar = np.where(fl, -lam, 0.0) * s
        for c in range(3):
            add = np.zeros(self.dims[c])
            sl = [slice(None)] * 3; sr = [slice(None)] * 3
            sl[c] = slice(1, None); sr[c] = slice(None, -1)
            add[tuple(sl)] += divbar   # the face on a cell's high side: +u
            add[tuple(sr)] -= divbar   # the face on its low side: -u
            ub[c] = np.where(masks[c], 0.0, ub[c] + add)
        vb_in = np.zeros_like(v)
        for c in range(3):
            idx, w, dw = pw[c]
            ubf = ub[c].ravel()
            m = ms[c]
            ok = m > 1e-8
            qbar = np.where(ok, ubf / np.where(ok, m, 1.0), 0.0)
            mbar = np.where(ok, -ubf * un[c] / np.where(ok, m, 1.0), 0.0)
            vb_in[:, c] = (w * qbar[idx]).sum(1)
            coef = v[:, c:c + 1] * qbar[idx] + mbar[idx]
            xb += (dw * coef[:, :, None]).sum(1) / dx
        return xb, vb_in

    def grad(self, control, x0, labels, dt, target):
        """d loss / d control by the FP64 adjoint (tape of all substeps)."""
        x = x0.astype(np.float64)
        ctl = control.astype(np.float64)
        v = self.sample_cells(ctl, x)
        tape = []
        for t, lab in enumerate(labels):
            tape.append((x, v))
            x, v = self.substep(x, v, lab, dt, key=t)
        idx, w, dw = _corner_weights_grad(x / self.dx - 0.5, (self.n,) * 3, clamp=False)
        rho = np.bincount(idx.ravel(), weights=w.ravel(), minlength=self.n ** 3)
        rbar = 2.0 * (rho - target.ravel())
        xbar = (dw * rbar[idx][:, :, None]).sum(1) / self.dx
        vbar = np.zeros_like(xbar)
        for t in reversed(range(len(labels))):
            xt, vt = tape[t]
            xbar, vbar = self.substep_adjoint(xt, vt, labels[t], dt, t, xbar, vbar)
        idx, w, _ = _corner_weights_grad(x0.astype(np.float64) / self.dx - 0.5, (self.n,) * 3,
                                         clamp=False)
        return np.stack([np.bincount(idx.ravel(), weights=(w * vbar[:, c:c + 1]).ravel(),
                                     minlength=self.n ** 3).reshape((self.n,) * 3)
                         for c in range(3)])

    # ---- APIC substep (k3_p2g_apic :1475-1588, k3_g2p_apic_advect :1591-1732)
    _OFFS = [np.array([0.0, 0.5, 0.5]), np.array([0.5, 0.0, 0.5]), np.array([0.5, 0.5, 0.0])]

    def _grid_apic(self, x, v, C, lab, dt, key):
        """P2G (APIC), forces, BC, divergence, pressure, gradient: the face
        velocities u3 plus what the adjoint needs."""
        dx = self.dx
        gx = x / dx
        masks = self._bc_masks(lab)
        pw, un, ms, u = [], [], [], []
        for c in range(3):
            idx, ijk, w, dw = _corners_apic(gx - self._OFFS[c], self.dims[c], clamp_idx=False)
            o = (ijk + self._OFFS[c]) * dx - x[:, None, :]          # x_f - x_p (P,8,3)
            val = v[:, c:c + 1] + (o * C[:, c, None, :]).sum(-1)   # (P,8)
            size = int(np.prod(self.dims[c]))
            m = np.bincount(idx.ravel(), weights=w.ravel(), minlength=size)
            q = np.bincount(idx.ravel(), weights=(w * val).ravel(), minlength=size)
            uc = np.where(m > 1e-8, q / np.where(m > 1e-8, m, 1.0), 0.0)
            pw.append((idx, w, dw, o, val)); un.append(uc); ms.append(m)
            uu = uc.reshape(self.dims[c]) + (self.g * dt if c == 1 else 0.0)
            uu[masks[c]] = 0.0
            u.append(uu)
        fl = lab == 1
        s = self.rho * dx / dt
        div = (u[0][1:] - u[0][:-1]) + (u[1][:, 1:] - u[1][:, :-1]) + (u[2][:, :, 1:] - u[2][:, :, :-1])
        div = np.where(fl, div * s, 0.0)
        fl, _, solve = self._system(key, lab)
        p = np.zeros(lab.shape)
        if fl.any():
            p[fl] = solve(-div[fl])
        k = dt / (self.rho * dx)
        u3, elig_l = [], []
        for c in range(3):
            pl = np.zeros(self.dims[c]); pr = np.zeros(self.dims[c])
            ml = np.full(self.dims[c], 2, lab.dtype); mr = np.full(self.dims[c], 2, lab.dtype)
            sl = [slice(None)] * 3; sr = [slice(None)] * 3
            sl[c] = slice(1, None); sr[c] = slice(None, -1)
            pl[tuple(sl)] = p; ml[tuple(sl)] = lab
            pr[tuple(sr)] = p; mr[tuple(sr)] = lab
            elig = ((ml == 1) | (mr == 1)) & (ml != 2) & (mr != 2) & ~masks[c]
            pl = np.where(ml == 1, pl, 0.0); pr = np.where(mr == 1, pr, 0.0)
            uc = np.where(elig, u[c] - k * (pr - pl), u[c])
            uc[masks[c]] = 0.0
            u3.append(uc); elig_l.append((elig, ml, mr))
        return dict(masks=masks, pw=pw, un=un, ms=ms, u3=u3, elig=elig_l, fl=fl, solve=solve,
                    s=s, k=k)

    def _g2p_apic(self, x, u3):
        dx = self.dx
        gx = x / dx
        inv = 3.0 / (dx * dx)
        vn = np.zeros_like(x)
        Cn = np.zeros((len(x), 3, 3))
        gath = []
        for c in range(3):
            idx, ijk, w, dw = _corners_apic(gx - self._OFFS[c], self.dims[c], clamp_idx=True)
            o = (ijk + self._OFFS[c]) * dx - x[:, None, :]
            uf = u3[c].ravel()[idx]
            vn[:, c] = (w * uf).sum(1)
            Cn[:, c, :] = ((w * uf * inv)[:, :, None] * o).sum(1)
            gath.append((idx, w, dw, o, uf))
        return vn, Cn, gath

    def substep_apic(self, x, v, C, lab, dt, key):
        g = self._grid_apic(x, v, C, lab, dt, key)
        vn, Cn, _ = self._g2p_apic(x, g["u3"])
        eps = self.dx * 1.001
        xn = np.clip(x + vn * dt, eps, self.dom - eps)
        return xn, vn, Cn

    def substep_apic_adjoint(self, x, v, C, lab, dt, key, xbar, vbar, Cbar):
        """Reverse-mode derivative of substep_apic: adjoints of (x, v, C)."""
        dx = self.dx
        inv = 3.0 / (dx * dx)
        g = self._grid_apic(x, v, C, lab, dt, key)
        vn, Cn, gath = self._g2p_apic(x, g["u3"])
        eps = dx * 1.001
        xr = x + vn * dt
        free = (xr >= eps) & (xr <= self.dom - eps)
        xb = np.where(free, xbar, 0.0)
        vb = vbar + np.where(free, dt * xbar, 0.0)
        ub3 = []
        for c in range(3):
            idx, w, dw, o, uf = gath[c]
            # g_c per corner: vb_c + inv * sum_d o_d Cbar[c][d]
            gc = vb[:, c:c + 1] + inv * (o * Cbar[:, c, None, :]).sum(-1)     # (P,8)
            size = int(np.prod(self.dims[c]))
            ub3.append(np.bincount(idx.ravel(), weights=(w * gc).ravel(),
                                   minlength=size).reshape(self.dims[c]))
            xb += (dw * (uf * gc)[:, :, None]).sum(1) / dx
            xb -= (w * uf * inv).sum(1)[:, None] * Cbar[:, c, :]
        fl, solve, s, k, masks = g["fl"], g["solve"], g["s"], g["k"], g["masks"]
        pbar = np.zeros(lab.shape)
        ub = []
        for c in range(3):
            elig, ml, mr = g["elig"][c]
            gg = np.where(elig, ub3[c], 0.0)
            sl = [slice(None)] * 3; sr = [slice(None)] * 3
            sl[c] = slice(1, None); sr[c] = slice(None, -1)
            pbar += np.where(fl, -k * gg[tuple(sr)] * (mr[tuple(sr)] == 1), 0.0)
            pbar += np.where(fl, k * gg[tuple(sl)] * (ml[tuple(sl)] == 1), 0.0)
            ub.append(np.where(masks[c], 0.0, ub3[c]))
        lam = np.zeros(lab.shape)
        if fl.any():
            lam[fl] = solve(pbar[fl])
        divbar = np.where(fl, -lam, 0.0) * s
        for c in range(3):
            add = np.zeros(self.dims[c])
            sl = [slice(None)] * 3; sr = [slice(None)] * 3
            sl[c] = slice(1, None); sr[c] = slice(None, -1)
            add[tuple(sl)] += divbar
            add[tuple(sr)] -= divbar
            ub[c] = np.where(masks[c], 0.0, ub[c] + add)
        vb_in = np.zeros_like(v)
        Cb_in = np.zeros_like(C)
        for c in range(3):
            idx, w, dw, o, val = g["pw"][c]
            ubf = ub[c].ravel()
            m = g["ms"][c]
            ok = m > 1e-8
            qbar = np.where(ok, ubf / np.where(ok, m, 1.0), 0.0)
            mbar = np.where(ok, -ubf * g["un"][c] / np.where(ok, m, 1.0), 0.0)
            wq = w * qbar[idx]
            vb_in[:, c] = wq.sum(1)
            Cb_in[:, c, :] = (wq[:, :, None] * o).sum(1)
            xb += (dw * (val * qbar[idx] + mbar[idx])[:, :, None]).sum(1) / dx
            xb -= wq.sum(1)[:, None] * C[:, c, :]
        return xb, vb_in, Cb_in

    def loss_apic(self, control, x0, labels, dt, target):
        x = x0.astype(np.float64)
        v = self.sample_cells(control.astype(np.float64), x)
        C = np.zeros((len(x), 3, 3))
        for t, lab in enumerate(labels):
            x, v, C = self.substep_apic(x, v, C, lab, dt, key=t)
        r = self.splat(x) - target
        return float((r * r).sum())

    def grad_apic(self, control, x0, labels, dt, target):
        x = x0.astype(np.float64)
        ctl = control.astype(np.float64)
        v = self.sample_cells(ctl, x)
        C = np.zeros((len(x), 3, 3))
        tape = []
        for t, lab in enumerate(labels):
            tape.append((x, v, C))
            x, v, C = self.substep_apic(x, v, C, lab, dt, key=t)
        idx, w, dw = _corner_weights_grad(x / self.dx - 0.5, (self.n,) * 3, clamp=False)
        rho = np.bincount(idx.ravel(), weights=w.ravel(), minlength=self.n ** 3)
        rbar = 2.0 * (rho - target.ravel())
        xbar = (dw * rbar[idx][:, :, None]).sum(1) / self.dx
        vbar = np.zeros_like(xbar)
        Cbar = np.zeros((len(x), 3, 3))
        for t in reversed(range(len(labels))):
            xt, vt, Ct = tape[t]
            xbar, vbar, Cbar = self.substep_apic_adjoint(xt, vt, Ct, labels[t], dt, t, xbar,
                                                         vbar, Cbar)
        idx, w, _ = _corner_weights_grad(x0.astype(np.float64) / self.dx - 0.5, (self.n,) * 3,
                                         clamp=False)
        return np.stack([np.bincount(idx.ravel(), weights=(w * vbar[:, c:c + 1]).ravel(),
                                     minlength=self.n ** 3).reshape((self.n,) * 3)
                         for c in range(3)])

    def sample_cells(self, grid3, x):
        idx, w = _corner_weights(x / self.dx - 0.5, (self.n,) * 3, clamp=False)
        return np.stack([(w * grid3[c].ravel()[idx]).sum(1) for c in range(3)], 1)

    def splat(self, x):
        idx, w = _corner_weights(x / self.dx - 0.5, (self.n,) * 3, clamp=False)
        return np.bincount(idx.ravel(), weights=w.ravel(), minlength=self.n ** 3).reshape((self.n,) * 3)

    def loss(self, control, x0, labels, dt, target):
        x = x0.astype(np.float64)
        v = self.sample_cells(control.astype(np.float64), x)
        for t, lab in enumerate(labels):
            x, v = self.substep(x, v, lab, dt, key=t)
        r = self.splat(x) - target
        return float((r * r).sum())
