"""Test infrastructure, not product code: a differentiable float64 PyTorch
restatement of the 2D SSG_VS step (src/Elastic2D_CPML.py:128-200) and of the
SSG_SV step (:202-275) with the moment-tensor source, used as an independent gradient oracle for the
hand-written adjoint kernels.  torch.autograd differentiates it exactly (to
float64 rounding), so its gradients with respect to rho, lambda and mu are the
discrete adjoint's reference values.  CPU only, small grids.

The CPML profiles, predicate bounds and coefficients come from an
oracle.Oracle2D instance (the oracle's own restatement of SetADEPML2D,
Elastic2D_CPML.py:392-528).
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F


def _pad(t, i0, i1, j0, j1, nx, nz):
    return F.pad(t, (j0, nz - j1, i0, nx - i1))


class TwinVS2D:
    def __init__(self, o, MT, wavelet, rec_index):
        """o: oracle.Oracle2D (float64); MT: (xx, zz, xz); wavelet: (nt,) float32
        source series; rec_index: linear receiver cells (vz)."""
        assert o.T == np.float64
        self.nx, self.nz = o.shape
        self.N = o.N
        self.dx, self.dz, self.dt = float(o.desc.dx), float(o.desc.dz), float(o.desc.dt)
        self.c = [float(o.desc.c[m]) for m in range(self.N)]
        self.isx, self.isz = int(o.desc.isx), int(o.desc.isz)
        self.mneg = [-float(np.float32(v)) for v in MT]
        self.wav = np.asarray(wavelet, np.float32).astype(np.float64)
        self.rec = torch.as_tensor(np.asarray(rec_index, np.int64))
        (ax, (xlo, xhi)), (az, (zlo, zhi)) = o.axes
        t = lambda a: torch.as_tensor(np.asarray(a, np.float64))
        self.X = {k: t(v) for k, v in ax.items()}
        self.Z = {k: t(v) for k, v in az.items()}
        N = self.N
        xi = (np.arange(self.nx) - N) * self.dx
        zj = (np.arange(self.nz) - N) * self.dz
        inx = lambda x: torch.as_tensor((x <= xlo) | (x >= xhi))
        inz = lambda z: torch.as_tensor((z <= zlo) | (z >= zhi))
        self.px, self.pxh = inx(xi), inx(xi + self.dx / 2)
        self.pz, self.pzh = inz(zj), inz(zj + self.dz / 2)

    # staggered differences over a region [i0,i1) x [j0,j1) (Differential2D.py)
    def _dx(self, f, i0, i1, j0, j1, fwd):
        v = 0
        for m, c in enumerate(self.c):
            if fwd:
                v = v + c * (f[i0 + m + 1:i1 + m + 1, j0:j1] - f[i0 - m:i1 - m, j0:j1])
            else:
                v = v + c * (f[i0 + m:i1 + m, j0:j1] - f[i0 - m - 1:i1 - m - 1, j0:j1])
        return v

    def _dz(self, f, i0, i1, j0, j1, fwd):
        v = 0
        for m, c in enumerate(self.c):
            if fwd:
                v = v + c * (f[i0:i1, j0 + m + 1:j1 + m + 1] - f[i0:i1, j0 - m:j1 - m])
            else:
                v = v + c * (f[i0:i1, j0 + m:j1 + m] - f[i0:i1, j0 - m - 1:j1 - m - 1])
        return v

    def _cpml(self, d, psi, P, b, a, k, i0, i1, j0, j1, axis):
        """CPML on one derivative over the region: returns (d', psi_new)."""
        if axis == 0:
            b, a, k = b[i0:i1, None], a[i0:i1, None], k[i0:i1, None]
        else:
            b, a, k = b[None, j0:j1], a[None, j0:j1], k[None, j0:j1]
        reg = psi[i0:i1, j0:j1]
        new = torch.where(P, b * reg + a * d, reg)
        dd = torch.where(P, d / k + new, d)
        return dd, psi + _pad(new - reg, i0, i1, j0, j1, self.nx, self.nz)

    def traces(self, rho, lam, mu, nt):
        nx, nz, N = self.nx, self.nz, self.N
        dx, dz, dt = self.dx, self.dz, self.dt
        X, Z = self.X, self.Z
        z = lambda: torch.zeros((nx, nz), dtype=torch.float64)
        vx, vz, sxx, szz, sxz = z(), z(), z(), z(), z()
        m = {k: z() for k in ("sxx_dx", "sxz_dz", "sxz_dx", "szz_dz", "dvx_dx", "dvz_dz", "dvz_dx", "dvx_dz")}
        out = []
        src = torch.zeros((nx, nz), dtype=torch.float64)
        src[self.isx, self.isz] = 1.0
        for it in range(nt):
            w = self.wav[it]
            sxx = sxx + src * (w * self.mneg[0])
            szz = szz + src * (w * self.mneg[1])
            sxz = sxz + src * (w * self.mneg[2])
            # vx :144-154
            i0, i1, j0, j1 = N + 1, nx - N, N + 1, nz - N
            P = self.px[i0:i1, None] | self.pz[None, j0:j1]
            a1 = self._dx(sxx, i0, i1, j0, j1, False) / dx
            b1 = self._dz(sxz, i0, i1, j0, j1, False) / dz
            a1, m["sxx_dx"] = self._cpml(a1, m["sxx_dx"], P, X["b"], X["a"], X["k"], i0, i1, j0, j1, 0)
            b1, m["sxz_dz"] = self._cpml(b1, m["sxz_dz"], P, Z["b"], Z["a"], Z["k"], i0, i1, j0, j1, 1)
            dvx = (a1 + b1) * dt / rho[i0:i1, j0:j1]
            # vz :156-167
            k0, k1, l0, l1 = N, nx - N - 1, N, nz - N - 1
            P = self.pxh[k0:k1, None] | self.pzh[None, l0:l1]
            r4 = 0.25 * (rho[k0:k1, l0:l1] + rho[k0:k1, l0 + 1:l1 + 1] + rho[k0 + 1:k1 + 1, l0 + 1:l1 + 1]
                         + rho[k0 + 1:k1 + 1, l0:l1])
            a2 = self._dx(sxz, k0, k1, l0, l1, True) / dx
            b2 = self._dz(szz, k0, k1, l0, l1, True) / dz
            a2, m["sxz_dx"] = self._cpml(a2, m["sxz_dx"], P, X["b_half"], X["a_half"], X["k_half"], k0, k1, l0, l1, 0)
            b2, m["szz_dz"] = self._cpml(b2, m["szz_dz"], P, Z["b_half"], Z["a_half"], Z["k_half"], k0, k1, l0, l1, 1)
            dvz = (b2 + a2) * dt / r4
            vx = vx + _pad(dvx, i0, i1, j0, j1, nx, nz)
            vz = vz + _pad(dvz, k0, k1, l0, l1, nx, nz)
            # sxx szz :172-186
            i0, i1, j0, j1 = N, nx - N - 1, N + 1, nz - N
            P = self.pxh[i0:i1, None] | self.pz[None, j0:j1]
            lhx = 0.5 * (lam[i0:i1, j0:j1] + lam[i0 + 1:i1 + 1, j0:j1])
            mhx = 0.5 * (mu[i0:i1, j0:j1] + mu[i0 + 1:i1 + 1, j0:j1])
            lpm = lhx + 2 * mhx
            p = self._dx(vx, i0, i1, j0, j1, True) / dx
            q = self._dz(vz, i0, i1, j0, j1, False) / dz
            p, m["dvx_dx"] = self._cpml(p, m["dvx_dx"], P, X["b_half"], X["a_half"], X["k_half"], i0, i1, j0, j1, 0)
            q, m["dvz_dz"] = self._cpml(q, m["dvz_dz"], P, Z["b"], Z["a"], Z["k"], i0, i1, j0, j1, 1)
            dsxx = (lpm * p + lhx * q) * dt
            dszz = (lpm * q + lhx * p) * dt
            # sxz :188-199
            k0, k1, l0, l1 = N + 1, nx - N, N, nz - N - 1
            P = self.px[k0:k1, None] | self.pzh[None, l0:l1]
            mhz = 0.5 * (mu[k0:k1, l0 + 1:l1 + 1] + mu[k0:k1, l0:l1])
            r = self._dx(vz, k0, k1, l0, l1, False) / dx
            u = self._dz(vx, k0, k1, l0, l1, True) / dz
            r, m["dvz_dx"] = self._cpml(r, m["dvz_dx"], P, X["b"], X["a"], X["k"], k0, k1, l0, l1, 0)
            u, m["dvx_dz"] = self._cpml(u, m["dvx_dz"], P, Z["b_half"], Z["a_half"], Z["k_half"], k0, k1, l0, l1, 1)
            dsxz = mhz * (u + r) * dt
            sxx = sxx + _pad(dsxx, i0, i1, j0, j1, nx, nz)
            szz = szz + _pad(dszz, i0, i1, j0, j1, nx, nz)
            sxz = sxz + _pad(dsxz, k0, k1, l0, l1, nx, nz)
            out.append(vz.reshape(-1)[self.rec])
        self.final = (vx, vz, sxx, szz, sxz)
        return torch.stack(out)


class TwinSV2D(TwinVS2D):
    """The SSG_SV step (src/Elastic2D_CPML.py:202-275) with the moment-tensor
    source injected before each velocity phase; receivers record vx."""

    def traces(self, rho, lam, mu, nt):
        nx, nz, N = self.nx, self.nz, self.N
        dx, dz, dt = self.dx, self.dz, self.dt
        X, Z = self.X, self.Z
        z = lambda: torch.zeros((nx, nz), dtype=torch.float64)
        vx, vz, sxx, szz, sxz = z(), z(), z(), z(), z()
        m = {k: z() for k in ("sxx_dx", "sxz_dz", "sxz_dx", "szz_dz", "dvx_dx", "dvz_dz", "dvz_dx", "dvx_dz")}
        out = []
        src = torch.zeros((nx, nz), dtype=torch.float64)
        src[self.isx, self.isz] = 1.0
        for it in range(nt):
            w = self.wav[it]
            sxx = sxx + src * (w * self.mneg[0])
            szz = szz + src * (w * self.mneg[1])
            sxz = sxz + src * (w * self.mneg[2])
            # vx at (i+1/2, j) :218-229
            i0, i1, j0, j1 = N, nx - N - 1, N + 1, nz - N
            P = self.pxh[i0:i1, None] | self.pz[None, j0:j1]
            r2 = (rho[i0:i1, j0:j1] + rho[i0 + 1:i1 + 1, j0:j1]) / 2
            a1 = self._dx(sxx, i0, i1, j0, j1, True) / dx
            b1 = self._dz(sxz, i0, i1, j0, j1, False) / dz
            a1, m["sxx_dx"] = self._cpml(a1, m["sxx_dx"], P, X["b_half"], X["a_half"], X["k_half"], i0, i1, j0, j1, 0)
            b1, m["sxz_dz"] = self._cpml(b1, m["sxz_dz"], P, Z["b"], Z["a"], Z["k"], i0, i1, j0, j1, 1)
            dvx = (a1 + b1) * dt / r2
            # vz at (i, j+1/2) :231-242
            k0, k1, l0, l1 = N + 1, nx - N, N, nz - N - 1
            P = self.px[k0:k1, None] | self.pzh[None, l0:l1]
            rz = 0.5 * (rho[k0:k1, l0:l1] + rho[k0:k1, l0 + 1:l1 + 1])
            a2 = self._dx(sxz, k0, k1, l0, l1, False) / dx
            b2 = self._dz(szz, k0, k1, l0, l1, True) / dz
            a2, m["sxz_dx"] = self._cpml(a2, m["sxz_dx"], P, X["b"], X["a"], X["k"], k0, k1, l0, l1, 0)
            b2, m["szz_dz"] = self._cpml(b2, m["szz_dz"], P, Z["b_half"], Z["a_half"], Z["k_half"], k0, k1, l0, l1, 1)
            dvz = (b2 + a2) * dt / rz
            vx = vx + _pad(dvx, i0, i1, j0, j1, nx, nz)
            vz = vz + _pad(dvz, k0, k1, l0, l1, nx, nz)
            # sxx szz at (i, j) :247-260
            i0, i1, j0, j1 = N + 1, nx - N, N + 1, nz - N
            P = self.px[i0:i1, None] | self.pz[None, j0:j1]
            lm = lam[i0:i1, j0:j1]
            lpm = lam[i0:i1, j0:j1] + 2 * mu[i0:i1, j0:j1]
            p = self._dx(vx, i0, i1, j0, j1, False) / dx
            q = self._dz(vz, i0, i1, j0, j1, False) / dz
            p, m["dvx_dx"] = self._cpml(p, m["dvx_dx"], P, X["b"], X["a"], X["k"], i0, i1, j0, j1, 0)
            q, m["dvz_dz"] = self._cpml(q, m["dvz_dz"], P, Z["b"], Z["a"], Z["k"], i0, i1, j0, j1, 1)
            dsxx = (lpm * p + lm * q) * dt
            dszz = (lpm * q + lm * p) * dt
            # sxz at (i+1/2, j+1/2) :262-273, same cells
            P = self.pxh[i0:i1, None] | self.pzh[None, j0:j1]
            m4 = 0.25 * (mu[i0:i1, j0 + 1:j1 + 1] + mu[i0:i1, j0:j1] + mu[i0 + 1:i1 + 1, j0 + 1:j1 + 1]
                         + mu[i0 + 1:i1 + 1, j0:j1])
            r = self._dx(vz, i0, i1, j0, j1, True) / dx
            u = self._dz(vx, i0, i1, j0, j1, True) / dz
            r, m["dvz_dx"] = self._cpml(r, m["dvz_dx"], P, X["b_half"], X["a_half"], X["k_half"], i0, i1, j0, j1, 0)
            u, m["dvx_dz"] = self._cpml(u, m["dvx_dz"], P, Z["b_half"], Z["a_half"], Z["k_half"], i0, i1, j0, j1, 1)
            dsxz = m4 * (u + r) * dt
            sxx = sxx + _pad(dsxx, i0, i1, j0, j1, nx, nz)
            szz = szz + _pad(dszz, i0, i1, j0, j1, nx, nz)
            sxz = sxz + _pad(dsxz, i0, i1, j0, j1, nx, nz)
            out.append(vx.reshape(-1)[self.rec])
        self.final = (vx, vz, sxx, szz, sxz)
        return torch.stack(out)
