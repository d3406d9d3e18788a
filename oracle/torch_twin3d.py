"""Test infrastructure, not product code: a differentiable float64 PyTorch
restatement of the 3D SSG-CPML moment-tensor step (src/Elastic3D_SSG_Tensor.py:
166-345, in the oracle's velocity3d / stress3d order) and, in TwinForce3D, of
the point-force step (src/Elastic3D_SSG_CPML.py:144-309), used as an
independent gradient oracle for the hand-written 3D adjoint kernels.  CPU, tiny grids.
Profiles, predicate bounds and coefficients come from an oracle.Oracle3D."""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F


class TwinTensor3D:
    def __init__(self, o, wavelet, rec_index):
        assert o.T == np.float64
        self.nx, self.ny, self.nz = o.shape
        self.N = o.N
        d = o.desc
        self.h = (float(d.dx), float(d.dy), float(d.dz))
        self.dt = float(d.dt)
        self.c = [float(d.c[m]) for m in range(self.N)]
        self.src = (int(d.isx), int(d.isy), int(d.isz))
        self.force = False
        self.mneg = [-float(np.float32(d.mt[q])) for q in range(6)]
        self.wav = np.asarray(wavelet, np.float32).astype(np.float64)
        self.rec = torch.as_tensor(np.asarray(rec_index, np.int64))
        self.ax = []
        for a, (arrs, (lo, hi)) in enumerate(o.axes):
            t = {k: torch.as_tensor(np.asarray(v, np.float64)) for k, v in arrs.items()}
            n = o.shape[a]
            x = (np.arange(n) - self.N) * self.h[a]
            t["in"] = torch.as_tensor((x <= lo) | (x >= hi))
            t["in_half"] = torch.as_tensor((x + self.h[a] / 2 <= lo) | (x + self.h[a] / 2 >= hi))
            self.ax.append(t)

    def _d(self, f, rng, axis, fwd):
        sl = [slice(r[0], r[1]) for r in rng]
        v = 0
        for m, c in enumerate(self.c):
            a, b = list(sl), list(sl)
            lo, hi = rng[axis]
            if fwd:
                a[axis] = slice(lo + m + 1, hi + m + 1)
                b[axis] = slice(lo - m, hi - m)
            else:
                a[axis] = slice(lo + m, hi + m)
                b[axis] = slice(lo - m - 1, hi - m - 1)
            v = v + c * (f[tuple(a)] - f[tuple(b)])
        return v / self.h[axis]

    def _prof(self, axis, name, rng):
        v = self.ax[axis][name][rng[axis][0]:rng[axis][1]]
        shape = [1, 1, 1]
        shape[axis] = -1
        return v.reshape(shape)

    def _cpml(self, d, psi, P, axis, half, rng):
        s = "_half" if half else ""
        b = self._prof(axis, "b" + s, rng)
        a = self._prof(axis, "a" + s, rng)
        k = self._prof(axis, "k" + s, rng)
        sl = tuple(slice(r[0], r[1]) for r in rng)
        reg = psi[sl]
        new = torch.where(P, b * reg + a * d, reg)
        out = torch.where(P, d / k + new, d)
        return out, psi + self._pad(new - reg, rng)

    def _pad(self, t, rng):
        (i0, i1), (j0, j1), (k0, k1) = rng
        return F.pad(t, (k0, self.nz - k1, j0, self.ny - j1, i0, self.nx - i1))

    def _pred(self, half, rng):
        p = []
        for a in range(3):
            v = self.ax[a]["in_half" if half[a] else "in"][rng[a][0]:rng[a][1]]
            shape = [1, 1, 1]
            shape[a] = -1
            p.append(v.reshape(shape))
        return p[0] | p[1] | p[2]

    def traces(self, rho, lam, mu, nt):
        nx, ny, nz, N, dt = self.nx, self.ny, self.nz, self.N, self.dt
        z = lambda: torch.zeros((nx, ny, nz), dtype=torch.float64)
        vx, vy, vz, sxx, syy, szz, sxy, sxz, syz = (z() for _ in range(9))
        m = {k: z() for k in ("xx_x", "xy_y", "xz_z", "xy_x", "yy_y", "yz_z", "xz_x", "yz_y", "zz_z",
                              "vx_x", "vy_y", "vz_z", "vy_x", "vx_y", "vz_x", "vx_z", "vz_y", "vy_z")}
        src = torch.zeros((nx, ny, nz), dtype=torch.float64)
        src[self.src] = 1.0
        out = []
        for it in range(nt):
            w = self.wav[it]
            if not self.force:
                sxx = sxx + src * (w * self.mneg[0])
                syy = syy + src * (w * self.mneg[1])
                szz = szz + src * (w * self.mneg[2])
                sxy = sxy + src * (w * self.mneg[3])
                sxz = sxz + src * (w * self.mneg[4])
                syz = syz + src * (w * self.mneg[5])
            # vx
            r = ((N, nx - N - 1), (N + 1, ny - N), (N + 1, nz - N))
            P = self._pred((True, False, False), r)
            d0, m["xx_x"] = self._cpml(self._d(sxx, r, 0, True), m["xx_x"], P, 0, True, r)
            d1, m["xy_y"] = self._cpml(self._d(sxy, r, 1, False), m["xy_y"], P, 1, False, r)
            d2, m["xz_z"] = self._cpml(self._d(sxz, r, 2, False), m["xz_z"], P, 2, False, r)
            sl = tuple(slice(a, b) for a, b in r)
            dvx = (d0 + d2 + d1) * dt / rho[sl]
            rx = r
            # vy
            r = ((N + 1, nx - N), (N, ny - N - 1), (N + 1, nz - N))
            P = self._pred((False, True, False), r)
            (i0, i1), (j0, j1), (k0, k1) = r
            rhy = 0.5 * (rho[i0:i1, j0:j1, k0:k1] + rho[i0:i1, j0 + 1:j1 + 1, k0:k1])
            d0, m["xy_x"] = self._cpml(self._d(sxy, r, 0, False), m["xy_x"], P, 0, False, r)
            d1, m["yy_y"] = self._cpml(self._d(syy, r, 1, True), m["yy_y"], P, 1, True, r)
            d2, m["yz_z"] = self._cpml(self._d(syz, r, 2, False), m["yz_z"], P, 2, False, r)
            dvy = (d0 + d1 + d2) * dt / rhy
            ry = r
            # vz
            r = ((N + 1, nx - N), (N + 1, ny - N), (N, nz - N - 1))
            P = self._pred((False, False, True), r)
            (i0, i1), (j0, j1), (k0, k1) = r
            r4 = 0.25 * (rho[i0:i1, j0:j1, k0:k1] + rho[i0:i1, j0 + 1:j1 + 1, k0:k1]
                         + rho[i0 + 1:i1 + 1, j0 + 1:j1 + 1, k0:k1] + rho[i0 + 1:i1 + 1, j0:j1, k0:k1])
            d0, m["xz_x"] = self._cpml(self._d(sxz, r, 0, False), m["xz_x"], P, 0, False, r)
            d1, m["yz_y"] = self._cpml(self._d(syz, r, 1, False), m["yz_y"], P, 1, False, r)
            d2, m["zz_z"] = self._cpml(self._d(szz, r, 2, True), m["zz_z"], P, 2, True, r)
            dvz = (d0 + d1 + d2) * dt / r4
            vx = vx + self._pad(dvx, rx)
            vy = vy + self._pad(dvy, ry)
            vz = vz + self._pad(dvz, r)
            if self.force:
                # point force after the velocity phase (Elastic3D_SSG_CPML.py:245)
                vz = vz + src * (dt * w / rho[self.src])
            # normal stresses
            r = ((N + 1, nx - N), (N + 1, ny - N), (N + 1, nz - N))
            (i0, i1), (j0, j1), (k0, k1) = r
            P = self._pred((False, False, False), r)
            lhx = 0.5 * (lam[i0:i1, j0:j1, k0:k1] + lam[i0 + 1:i1 + 1, j0:j1, k0:k1])
            mhx = 0.5 * (mu[i0:i1, j0:j1, k0:k1] + mu[i0 + 1:i1 + 1, j0:j1, k0:k1])
            lpm = lhx + 2 * mhx
            e0, m["vx_x"] = self._cpml(self._d(vx, r, 0, False), m["vx_x"], P, 0, False, r)
            e1, m["vy_y"] = self._cpml(self._d(vy, r, 1, False), m["vy_y"], P, 1, False, r)
            e2, m["vz_z"] = self._cpml(self._d(vz, r, 2, False), m["vz_z"], P, 2, False, r)
            dsxx = (lpm * e0 + lhx * (e2 + e1)) * dt
            dsyy = (lpm * e1 + lhx * (e0 + e2)) * dt
            dszz = (lpm * e2 + lhx * (e0 + e1)) * dt
            rn = r
            # sxy
            r = ((N + 1, nx - N), (N + 1, ny - N), (N, nz - N))
            (i0, i1), (j0, j1), (k0, k1) = r
            P = self._pred((True, True, False), r)
            mu0 = mu[i0:i1, j0:j1, k0:k1]
            m4 = 0.25 * (mu[i0:i1, j0 + 1:j1 + 1, k0:k1] + mu0 + mu0 + mu[i0 + 1:i1 + 1, j0:j1, k0:k1])
            f0, m["vy_x"] = self._cpml(self._d(vy, r, 0, True), m["vy_x"], P, 0, True, r)
            f1, m["vx_y"] = self._cpml(self._d(vx, r, 1, True), m["vx_y"], P, 1, True, r)
            dsxy = m4 * (f1 + f0) * dt
            rxy = r
            # sxz
            r = ((N, nx - N - 1), (N, ny - N), (N, nz - N - 1))
            (i0, i1), (j0, j1), (k0, k1) = r
            P = self._pred((True, False, True), r)
            mu0 = mu[i0:i1, j0:j1, k0:k1]
            m4 = 0.25 * (mu0 + mu[i0 + 1:i1 + 1, j0:j1, k0:k1] + mu0 + mu[i0:i1, j0 + 1:j1 + 1, k0:k1])
            g0, m["vz_x"] = self._cpml(self._d(vz, r, 0, True), m["vz_x"], P, 0, True, r)
            g1, m["vx_z"] = self._cpml(self._d(vx, r, 2, True), m["vx_z"], P, 2, True, r)
            dsxz = m4 * (g1 + g0) * dt
            rxz = r
            # syz
            r = ((N, nx - N), (N, ny - N - 1), (N, nz - N - 1))
            (i0, i1), (j0, j1), (k0, k1) = r
            P = self._pred((False, True, True), r)
            mu0 = mu[i0:i1, j0:j1, k0:k1]
            m4 = 0.25 * (mu[i0:i1, j0 + 1:j1 + 1, k0:k1] + mu0 + mu[i0:i1, j0:j1, k0 + 1:k1 + 1] + mu0)
            h0, m["vz_y"] = self._cpml(self._d(vz, r, 1, True), m["vz_y"], P, 1, True, r)
            h1, m["vy_z"] = self._cpml(self._d(vy, r, 2, True), m["vy_z"], P, 2, True, r)
            dsyz = m4 * (h0 + h1) * dt
            sxx = sxx + self._pad(dsxx, rn)
            syy = syy + self._pad(dsyy, rn)
            szz = szz + self._pad(dszz, rn)
            sxy = sxy + self._pad(dsxy, rxy)
            sxz = sxz + self._pad(dsxz, rxz)
            syz = syz + self._pad(dsyz, r)
            out.append(vx.reshape(-1)[self.rec])
        self.final = (vx, vy, vz, sxx, syy, szz, sxy, sxz, syz)
        return torch.stack(out)


class TwinForce3D(TwinTensor3D):
    """The SSG-CPML point-force step (src/Elastic3D_SSG_CPML.py:144-309): the
    same stencils, no moment tensor, vz[isx+5, isy+5, isz+5] += dt*w/rho
    after the velocity phase; receivers record vx."""

    def __init__(self, o, wavelet, rec_index):
        super().__init__(o, wavelet, rec_index)
        d = o.desc
        self.src = (int(d.isx) + 5, int(d.isy) + 5, int(d.isz) + 5)
        self.force = True
