"""NumPy twin of the oracle (test infrastructure only).

A second, independent transcription of six reference kernels, written
with whole-array slices instead of loops:
  * Elastic2D_CPML.update_SSG_VS        (src/Elastic2D_CPML.py:128-200)
  * Elastic2D_CPML.update_SSG_SV        (src/Elastic2D_CPML.py:203-274)
  * Elastic2D_CPML.update_RSG           (src/Elastic2D_CPML.py:277-353)
  * Elastic3D_SSG_Tensor.update_SSG      (src/Elastic3D_SSG_Tensor.py:166-345)
  * Elastic3D_SSG_CPML.update_SSG        (src/Elastic3D_SSG_CPML.py:144-309)
  * Elastic3D_SSG_SPML.update_SSG_SPML   (src/Elastic3D_SSG_SPML.py:160-393)
Every operation is an elementwise IEEE operation in the array dtype, in the
reference's order, so on the same inputs it must agree bit for bit with the
C++ oracle (sw_oracle.cpp).  Used on tiny grids only.
"""
from __future__ import annotations

import numpy as np


def _pred(vals, lo, hi):
    return (vals <= lo) | (vals >= hi)


class Twin2D:
    def __init__(self, o):
        """Build from an oracle.Oracle2D (shares its inputs, owns its state)."""
        T = o.T
        self.T = T
        self.N = o.N
        d = o.desc
        self.dx, self.dz, self.dt = T(d.dx), T(d.dz), T(d.dt)
        self.c = np.array([d.c[m] for m in range(o.N)], dtype=np.float64).astype(T)
        self.rho, self.lam, self.mu = o.rho.copy(), o.lam.copy(), o.mu.copy()
        z = lambda: np.zeros_like(o.vx)
        self.vx, self.vz, self.sxx, self.szz, self.sxz = z(), z(), z(), z(), z()
        self.mem = {k: z() for k in ("sxx_dx", "sxz_dx", "sxz_dz", "szz_dz", "dvx_dx", "dvx_dz",
                                     "dvz_dx", "dvz_dz")}
        (self.X, (self.xlo, self.xhi)), (self.Z, (self.zlo, self.zhi)) = o.axes
        self.isx, self.isz, self.rsx, self.rsz = d.isx, d.isz, d.rsx, d.rsz
        self.data = np.zeros_like(o.data)

    def _d(self, f, I, J, axis, fwd):
        T, N, c = self.T, self.N, self.c
        v = np.zeros((I.stop - I.start, J.stop - J.start), T)
        for m in range(N):
            a, b = (m + 1, -m) if fwd else (m, -m - 1)
            if axis == 0:
                hi = f[I.start + a:I.stop + a, J]
                lo = f[I.start + b:I.stop + b, J]
            else:
                hi = f[I, J.start + a:J.stop + a]
                lo = f[I, J.start + b:J.stop + b]
            v = v + c[m] * (hi - lo)
        return v

    def _mask(self, I, J, xhalf, zhalf):
        T = self.T
        i = np.arange(I.start, I.stop)
        j = np.arange(J.start, J.stop)
        x = (i - self.N).astype(T) * self.dx + (self.dx / T(2) if xhalf else T(0))
        z = (j - self.N).astype(T) * self.dz + (self.dz / T(2) if zhalf else T(0))
        return _pred(x, T(self.xlo), T(self.xhi))[:, None] | _pred(z, T(self.zlo), T(self.zhi))[None, :]

    def _pml(self, name, d, bx, ax, kx, mask, I, J, along_x):
        m = self.mem[name]
        old = m[I, J]
        if along_x:
            b, a, k = bx[I][:, None], ax[I][:, None], kx[I][:, None]
        else:
            b, a, k = bx[J][None, :], ax[J][None, :], kx[J][None, :]
        new = b * old + a * d
        m[I, J] = np.where(mask, new, old)
        return np.where(mask, d / k + new, d)

    def step(self, it, w):
        T, N, dt = self.T, self.N, self.dt
        nx, nz = self.vx.shape
        X, Z = self.X, self.Z
        # vx
        I, J = slice(N + 1, nx - N), slice(N + 1, nz - N)
        dsxxdx = self._d(self.sxx, I, J, 0, False) / self.dx
        dsxzdz = self._d(self.sxz, I, J, 1, False) / self.dz
        mk = self._mask(I, J, False, False)
        dsxxdx = self._pml("sxx_dx", dsxxdx, X["b"], X["a"], X["k"], mk, I, J, True)
        dsxzdz = self._pml("sxz_dz", dsxzdz, Z["b"], Z["a"], Z["k"], mk, I, J, False)
        self.vx[I, J] = self.vx[I, J] + (dsxxdx + dsxzdz) * dt / self.rho[I, J]
        # vz
        I, J = slice(N, nx - N - 1), slice(N, nz - N - 1)
        r = self.rho
        rh = T(0.25) * (r[I, J] + r[N:nx - N - 1, N + 1:nz - N] + r[N + 1:nx - N, N + 1:nz - N]
                        + r[N + 1:nx - N, N:nz - N - 1])
        dsxzdx = self._d(self.sxz, I, J, 0, True) / self.dx
        dszzdz = self._d(self.szz, I, J, 1, True) / self.dz
        mk = self._mask(I, J, True, True)
        dsxzdx = self._pml("sxz_dx", dsxzdx, X["b_half"], X["a_half"], X["k_half"], mk, I, J, True)
        dszzdz = self._pml("szz_dz", dszzdz, Z["b_half"], Z["a_half"], Z["k_half"], mk, I, J, False)
        self.vz[I, J] = self.vz[I, J] + (dszzdz + dsxzdx) * dt / rh
        # source
        self.vz[self.isx, self.isz] += dt * T(w) / self.rho[self.isx, self.isz]
        # sxx szz
        I, J = slice(N, nx - N - 1), slice(N + 1, nz - N)
        lhx = T(0.5) * (self.lam[I, J] + self.lam[N + 1:nx - N, J])
        mhx = T(0.5) * (self.mu[I, J] + self.mu[N + 1:nx - N, J])
        lpm = lhx + T(2) * mhx
        dvxdx = self._d(self.vx, I, J, 0, True) / self.dx
        dvzdz = self._d(self.vz, I, J, 1, False) / self.dz
        mk = self._mask(I, J, True, False)
        dvxdx = self._pml("dvx_dx", dvxdx, X["b_half"], X["a_half"], X["k_half"], mk, I, J, True)
        dvzdz = self._pml("dvz_dz", dvzdz, Z["b"], Z["a"], Z["k"], mk, I, J, False)
        self.sxx[I, J] = self.sxx[I, J] + (lpm * dvxdx + lhx * dvzdz) * dt
        self.szz[I, J] = self.szz[I, J] + (lpm * dvzdz + lhx * dvxdx) * dt
        # sxz
        I, J = slice(N + 1, nx - N), slice(N, nz - N - 1)
        mhz = T(0.5) * (self.mu[I, N + 1:nz - N] + self.mu[I, J])
        dvzdx = self._d(self.vz, I, J, 0, False) / self.dx
        dvxdz = self._d(self.vx, I, J, 1, True) / self.dz
        mk = self._mask(I, J, False, True)
        dvzdx = self._pml("dvz_dx", dvzdx, X["b"], X["a"], X["k"], mk, I, J, True)
        dvxdz = self._pml("dvx_dz", dvxdz, Z["b_half"], Z["a_half"], Z["k_half"], mk, I, J, False)
        self.sxz[I, J] = self.sxz[I, J] + mhz * (dvxdz + dvzdx) * dt
        self.data[it] = self.vz[self.rsx, self.rsz]


class Twin2DSV(Twin2D):
    """Elastic2D_CPML.update_SSG_SV (src/Elastic2D_CPML.py:203-274): vx at
    (i+1/2, j) with rho averaged over i, i+1 (as (a+b)/2); vz at (i, j+1/2)
    with 0.5*(rho[i,j] + rho[i,j+1]); the point force vx[src] += dt*w/rho[src]
    (:245); normal stresses at integer points with the cell's own lam, mu;
    sxz at (i+1/2, j+1/2) with mu averaged over the four corners; the receiver
    records vx (:274)."""

    def step(self, it, w):
        T, N, dt = self.T, self.N, self.dt
        nx, nz = self.vx.shape
        X, Z = self.X, self.Z
        r, lam, mu = self.rho, self.lam, self.mu
        # vx (:216-228)
        I, J = slice(N, nx - N - 1), slice(N + 1, nz - N)
        dsxxdx = self._d(self.sxx, I, J, 0, True) / self.dx
        dsxzdz = self._d(self.sxz, I, J, 1, False) / self.dz
        rhx = (r[I, J] + r[N + 1:nx - N, J]) / T(2)
        mk = self._mask(I, J, True, False)
        dsxxdx = self._pml("sxx_dx", dsxxdx, X["b_half"], X["a_half"], X["k_half"], mk, I, J, True)
        dsxzdz = self._pml("sxz_dz", dsxzdz, Z["b"], Z["a"], Z["k"], mk, I, J, False)
        self.vx[I, J] = self.vx[I, J] + (dsxxdx + dsxzdz) * dt / rhx
        # vz (:229-241)
        I, J = slice(N + 1, nx - N), slice(N, nz - N - 1)
        rhz = T(0.5) * (r[I, J] + r[I, N + 1:nz - N])
        dsxzdx = self._d(self.sxz, I, J, 0, False) / self.dx
        dszzdz = self._d(self.szz, I, J, 1, True) / self.dz
        mk = self._mask(I, J, False, True)
        dsxzdx = self._pml("sxz_dx", dsxzdx, X["b"], X["a"], X["k"], mk, I, J, True)
        dszzdz = self._pml("szz_dz", dszzdz, Z["b_half"], Z["a_half"], Z["k_half"], mk, I, J, False)
        self.vz[I, J] = self.vz[I, J] + (dszzdz + dsxzdx) * dt / rhz
        # point force (:245)
        self.vx[self.isx, self.isz] += dt * T(w) / r[self.isx, self.isz]
        # sxx szz (:247-259)
        I, J = slice(N + 1, nx - N), slice(N + 1, nz - N)
        lm = lam[I, J]
        l2m = lam[I, J] + T(2) * mu[I, J]
        dvxdx = self._d(self.vx, I, J, 0, False) / self.dx
        dvzdz = self._d(self.vz, I, J, 1, False) / self.dz
        mk = self._mask(I, J, False, False)
        dvxdx = self._pml("dvx_dx", dvxdx, X["b"], X["a"], X["k"], mk, I, J, True)
        dvzdz = self._pml("dvz_dz", dvzdz, Z["b"], Z["a"], Z["k"], mk, I, J, False)
        self.sxx[I, J] = self.sxx[I, J] + (l2m * dvxdx + lm * dvzdz) * dt
        self.szz[I, J] = self.szz[I, J] + (l2m * dvzdz + lm * dvxdx) * dt
        # sxz (:261-273)
        I, J = slice(N + 1, nx - N), slice(N + 1, nz - N)
        m4 = T(0.25) * (mu[I, N + 2:nz - N + 1] + mu[I, J] + mu[N + 2:nx - N + 1, N + 2:nz - N + 1]
                        + mu[N + 2:nx - N + 1, J])
        dvzdx = self._d(self.vz, I, J, 0, True) / self.dx
        dvxdz = self._d(self.vx, I, J, 1, True) / self.dz
        mk = self._mask(I, J, True, True)
        dvzdx = self._pml("dvz_dx", dvzdx, X["b_half"], X["a_half"], X["k_half"], mk, I, J, True)
        dvxdz = self._pml("dvx_dz", dvxdz, Z["b_half"], Z["a_half"], Z["k_half"], mk, I, J, False)
        self.sxz[I, J] = self.sxz[I, J] + m4 * (dvxdz + dvzdx) * dt
        self.data[it] = self.vx[self.rsx, self.rsz]


class Twin2DRSG(Twin2D):
    """Elastic2D_CPML.update_RSG (src/Elastic2D_CPML.py:277-353): rotated
    staggered grid, velocities at (i, j), stresses at (i+1/2, j+1/2);
    d/dx = (Drz - Drx)/(2 dx), d/dz = (Drz + Drx)/(2 dz) with the diagonal
    differences of src/Differential2D.py:32-56; the caller's source value is
    spread over the 2x2 block vz[isx+a, isz+b] += dt*source/(8 rho), a, b in
    {-1, 0}; no receiver."""

    # (i, j) offsets of the m-th tap's two samples, per diagonal difference
    _TAPS = {
        "rx_f": lambda m: ((m + 1, m + 1), (-m, -m)),
        "rz_f": lambda m: ((-m, m + 1), (m + 1, -m)),
        "rx_b": lambda m: ((m, m), (-m - 1, -m - 1)),
        "rz_b": lambda m: ((-m - 1, m), (m, -m - 1)),
    }

    def _dr(self, f, I, J, kind):
        T, N, c = self.T, self.N, self.c
        v = np.zeros((I.stop - I.start, J.stop - J.start), T)
        for m in range(N):
            (ai, aj), (bi, bj) = self._TAPS[kind](m)
            hi = f[I.start + ai:I.stop + ai, J.start + aj:J.stop + aj]
            lo = f[I.start + bi:I.stop + bi, J.start + bj:J.stop + bj]
            v = v + c[m] * (hi - lo)
        return v

    def step(self, it, source):
        T, N, dt = self.T, self.N, self.dt
        nx, nz = self.vx.shape
        X, Z = self.X, self.Z
        dx2, dz2 = T(2) * self.dx, T(2) * self.dz
        # velocities at integer points (:292-320)
        I, J = slice(N + 1, nx - N), slice(N + 1, nz - N)
        rx = {f: self._dr(getattr(self, f), I, J, "rx_b") for f in ("sxx", "szz", "sxz")}
        rz = {f: self._dr(getattr(self, f), I, J, "rz_b") for f in ("sxx", "szz", "sxz")}
        dsxxdx = (rz["sxx"] - rx["sxx"]) / dx2
        dszzdz = (rz["szz"] + rx["szz"]) / dz2
        dsxzdx = (rz["sxz"] - rx["sxz"]) / dx2
        dsxzdz = (rz["sxz"] + rx["sxz"]) / dz2
        mk = self._mask(I, J, False, False)
        dsxxdx = self._pml("sxx_dx", dsxxdx, X["b"], X["a"], X["k"], mk, I, J, True)
        dszzdz = self._pml("szz_dz", dszzdz, Z["b"], Z["a"], Z["k"], mk, I, J, False)
        dsxzdx = self._pml("sxz_dx", dsxzdx, X["b"], X["a"], X["k"], mk, I, J, True)
        dsxzdz = self._pml("sxz_dz", dsxzdz, Z["b"], Z["a"], Z["k"], mk, I, J, False)
        rho = self.rho[I, J]
        self.vx[I, J] = self.vx[I, J] + (dsxxdx + dsxzdz) * dt / rho
        self.vz[I, J] = self.vz[I, J] + (dszzdz + dsxzdx) * dt / rho
        # source (:322-323)
        s = T(np.float32(source))
        for a in (-1, 0):
            for b in (-1, 0):
                i, j = self.isx + a, self.isz + b
                self.vz[i, j] = self.vz[i, j] + dt * s / (T(8) * self.rho[i, j])
        # stresses at half points (:325-352), the cell's own lam and mu
        I, J = slice(N, nx - N - 1), slice(N, nz - N - 1)
        lam, mu = self.lam[I, J], self.mu[I, J]
        l2m = lam + T(2) * mu
        vxrx, vxrz = self._dr(self.vx, I, J, "rx_f"), self._dr(self.vx, I, J, "rz_f")
        vzrx, vzrz = self._dr(self.vz, I, J, "rx_f"), self._dr(self.vz, I, J, "rz_f")
        dvxdx = (vxrz - vxrx) / dx2
        dvxdz = (vxrz + vxrx) / dz2
        dvzdx = (vzrz - vzrx) / dx2
        dvzdz = (vzrz + vzrx) / dz2
        mk = self._mask(I, J, True, True)
        dvxdx = self._pml("dvx_dx", dvxdx, X["b_half"], X["a_half"], X["k_half"], mk, I, J, True)
        dvxdz = self._pml("dvx_dz", dvxdz, Z["b_half"], Z["a_half"], Z["k_half"], mk, I, J, False)
        dvzdx = self._pml("dvz_dx", dvzdx, X["b_half"], X["a_half"], X["k_half"], mk, I, J, True)
        dvzdz = self._pml("dvz_dz", dvzdz, Z["b_half"], Z["a_half"], Z["k_half"], mk, I, J, False)
        self.sxx[I, J] = self.sxx[I, J] + (l2m * dvxdx + lam * dvzdz) * dt
        self.szz[I, J] = self.szz[I, J] + (l2m * dvzdz + lam * dvxdx) * dt
        self.sxz[I, J] = self.sxz[I, J] + (mu * (dvxdz + dvzdx)) * dt


class Twin3DTensor:
    def __init__(self, o):
        """Build from an oracle.Oracle3D of scheme TENSOR."""
        T = o.T
        self.T = T
        self.N = o.N
        d = o.desc
        self.h = (T(d.dx), T(d.dy), T(d.dz))
        self.dt = T(d.dt)
        self.c = np.array([d.c[m] for m in range(o.N)], dtype=np.float64).astype(T)
        self.rho, self.lam, self.mu = o.rho.copy(), o.lam.copy(), o.mu.copy()
        z = lambda: np.zeros_like(o.vx)
        for f in ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz"):
            setattr(self, f, z())
        self.mem = {}
        self.axes = o.axes
        self.src = (d.isx, d.isy, d.isz)
        self.mt = [np.float32(d.mt[q]) for q in range(6)]
        self.rec = (o.rx, o.ry, o.rz)
        self.data = np.zeros_like(o.data)

    def _d(self, f, box, axis, fwd):
        T, N, c = self.T, self.N, self.c
        shp = tuple(s.stop - s.start for s in box)
        v = np.zeros(shp, T)
        for m in range(N):
            a, b = (m + 1, -m) if fwd else (m, -m - 1)
            hi = tuple(slice(s.start + (a if q == axis else 0), s.stop + (a if q == axis else 0))
                       for q, s in enumerate(box))
            lo = tuple(slice(s.start + (b if q == axis else 0), s.stop + (b if q == axis else 0))
                       for q, s in enumerate(box))
            v = v + c[m] * (f[hi] - f[lo])
        return v

    def _mask(self, box, half):
        T = self.T
        m = None
        for q in range(3):
            i = np.arange(box[q].start, box[q].stop)
            x = (i - self.N).astype(T) * self.h[q] + (self.h[q] / T(2) if half[q] else T(0))
            prof, (lo, hi) = self.axes[q]
            p = _pred(x, T(lo), T(hi))
            shape = [1, 1, 1]
            shape[q] = -1
            p = p.reshape(shape)
            m = p if m is None else (m | p)
        return m

    def _pml(self, name, d, q, half, mask, box):
        prof, _ = self.axes[q]
        sfx = "_half" if half else ""
        shape = [1, 1, 1]
        shape[q] = -1
        b = prof["b" + sfx][box[q]].reshape(shape)
        a = prof["a" + sfx][box[q]].reshape(shape)
        k = prof["k" + sfx][box[q]].reshape(shape)
        if name not in self.mem:
            self.mem[name] = np.zeros_like(self.vx)
        m = self.mem[name]
        old = m[box]
        new = b * old + a * d
        m[box] = np.where(mask, new, old)
        return np.where(mask, d / k + new, d)

    def step(self, it, w):
        T = self.T
        s = self.src
        src = T(np.float32(w))
        for f, q in (("sxx", 0), ("syy", 1), ("szz", 2), ("sxy", 3), ("sxz", 4), ("syz", 5)):
            getattr(self, f)[s] += src * (-T(self.mt[q]))
        self._velocity(True)
        self._stress()
        rx, ry, rz = self.rec
        self.data[it] = self.vx[rx, ry, rz].astype(np.float32)

    def _velocity(self, tensor):
        """Velocity phase; the tensor scheme sums vz's derivatives x, y, z
        (Elastic3D_SSG_Tensor.py:243), the point-force scheme z, x, y
        (Elastic3D_SSG_CPML.py:212)."""
        T, N, dt = self.T, self.N, self.dt
        nx, ny, nz = self.vx.shape
        dx, dy, dz = self.h
        S = lambda a, b: slice(a, b)
        r, lam, mu = self.rho, self.lam, self.mu
        # vx
        B = (S(N, nx - N - 1), S(N + 1, ny - N), S(N + 1, nz - N))
        d1 = self._d(self.sxx, B, 0, True) / dx
        d2 = self._d(self.sxy, B, 1, False) / dy
        d3 = self._d(self.sxz, B, 2, False) / dz
        mk = self._mask(B, (1, 0, 0))
        d1 = self._pml("sxx_dx", d1, 0, True, mk, B)
        d2 = self._pml("sxy_dy", d2, 1, False, mk, B)
        d3 = self._pml("sxz_dz", d3, 2, False, mk, B)
        self.vx[B] = self.vx[B] + (d1 + d3 + d2) * dt / r[B]
        # vy
        B = (S(N + 1, nx - N), S(N, ny - N - 1), S(N + 1, nz - N))
        Bj = (B[0], S(N + 1, ny - N), B[2])
        rhy = T(0.5) * (r[B] + r[Bj])
        d1 = self._d(self.sxy, B, 0, False) / dx
        d2 = self._d(self.syy, B, 1, True) / dy
        d3 = self._d(self.syz, B, 2, False) / dz
        mk = self._mask(B, (0, 1, 0))
        d1 = self._pml("sxy_dx", d1, 0, False, mk, B)
        d2 = self._pml("syy_dy", d2, 1, True, mk, B)
        d3 = self._pml("syz_dz", d3, 2, False, mk, B)
        self.vy[B] = self.vy[B] + (d1 + d2 + d3) * dt / rhy
        # vz
        B = (S(N + 1, nx - N), S(N + 1, ny - N), S(N, nz - N - 1))
        Bj = (B[0], S(N + 2, ny - N + 1), B[2])
        Bij = (S(N + 2, nx - N + 1), S(N + 2, ny - N + 1), B[2])
        Bi = (S(N + 2, nx - N + 1), B[1], B[2])
        r4 = T(0.25) * (r[B] + r[Bj] + r[Bij] + r[Bi])
        d1 = self._d(self.sxz, B, 0, False) / dx
        d2 = self._d(self.syz, B, 1, False) / dy
        d3 = self._d(self.szz, B, 2, True) / dz
        mk = self._mask(B, (0, 0, 1))
        d1 = self._pml("sxz_dx", d1, 0, False, mk, B)
        d2 = self._pml("syz_dy", d2, 1, False, mk, B)
        d3 = self._pml("szz_dz", d3, 2, True, mk, B)
        vz_sum = (d1 + d2 + d3) if tensor else (d3 + d1 + d2)
        self.vz[B] = self.vz[B] + vz_sum * dt / r4

    def _stress(self):
        T, N, dt = self.T, self.N, self.dt
        nx, ny, nz = self.vx.shape
        dx, dy, dz = self.h
        S = lambda a, b: slice(a, b)
        r, lam, mu = self.rho, self.lam, self.mu
        # normal stresses
        B = (S(N + 1, nx - N), S(N + 1, ny - N), S(N + 1, nz - N))
        Bi = (S(N + 2, nx - N + 1), B[1], B[2])
        lhx = T(0.5) * (lam[B] + lam[Bi])
        mhx = T(0.5) * (mu[B] + mu[Bi])
        lpm = lhx + T(2) * mhx
        e1 = self._d(self.vx, B, 0, False) / dx
        e2 = self._d(self.vy, B, 1, False) / dy
        e3 = self._d(self.vz, B, 2, False) / dz
        mk = self._mask(B, (0, 0, 0))
        e1 = self._pml("dvx_dx", e1, 0, False, mk, B)
        e2 = self._pml("dvy_dy", e2, 1, False, mk, B)
        e3 = self._pml("dvz_dz", e3, 2, False, mk, B)
        self.sxx[B] = self.sxx[B] + (lpm * e1 + lhx * (e3 + e2)) * dt
        self.syy[B] = self.syy[B] + (lpm * e2 + lhx * (e1 + e3)) * dt
        self.szz[B] = self.szz[B] + (lpm * e3 + lhx * (e1 + e2)) * dt
        # sxy
        B = (S(N + 1, nx - N), S(N + 1, ny - N), S(N, nz - N))
        Bj = (B[0], S(N + 2, ny - N + 1), B[2])
        Bi = (S(N + 2, nx - N + 1), B[1], B[2])
        m4 = T(0.25) * (mu[Bj] + mu[B] + mu[B] + mu[Bi])
        e1 = self._d(self.vy, B, 0, True) / dx
        e2 = self._d(self.vx, B, 1, True) / dy
        mk = self._mask(B, (1, 1, 0))
        e1 = self._pml("dvy_dx", e1, 0, True, mk, B)
        e2 = self._pml("dvx_dy", e2, 1, True, mk, B)
        self.sxy[B] = self.sxy[B] + m4 * (e2 + e1) * dt
        # sxz
        B = (S(N, nx - N - 1), S(N, ny - N), S(N, nz - N - 1))
        Bi = (S(N + 1, nx - N), B[1], B[2])
        Bj = (B[0], S(N + 1, ny - N + 1), B[2])
        m4 = T(0.25) * (mu[B] + mu[Bi] + mu[B] + mu[Bj])
        e1 = self._d(self.vz, B, 0, True) / dx
        e2 = self._d(self.vx, B, 2, True) / dz
        mk = self._mask(B, (1, 0, 1))
        e1 = self._pml("dvz_dx", e1, 0, True, mk, B)
        e2 = self._pml("dvx_dz", e2, 2, True, mk, B)
        self.sxz[B] = self.sxz[B] + m4 * (e2 + e1) * dt
        # syz
        B = (S(N, nx - N), S(N, ny - N - 1), S(N, nz - N - 1))
        Bj = (B[0], S(N + 1, ny - N), B[2])
        Bk = (B[0], B[1], S(N + 1, nz - N))
        m4 = T(0.25) * (mu[Bj] + mu[B] + mu[Bk] + mu[B])
        e1 = self._d(self.vz, B, 1, True) / dy
        e2 = self._d(self.vy, B, 2, True) / dz
        mk = self._mask(B, (0, 1, 1))
        e1 = self._pml("dvz_dy", e1, 1, True, mk, B)
        e2 = self._pml("dvy_dz", e2, 2, True, mk, B)
        self.syz[B] = self.syz[B] + m4 * (e1 + e2) * dt


class Twin3DCPML(Twin3DTensor):
    """Elastic3D_SSG_CPML.update_SSG (src/Elastic3D_SSG_CPML.py:144-309): the
    tensor scheme's stencils and material quirks without the moment-tensor
    injection, vz's derivatives summed z, x, y (:212), the point force
    vz[isx+5, isy+5, isz+5] += dt*w / rho there after the velocity phase
    (:245; the Dirichlet loops of :215-243 only zero cells no update touches);
    one receiver records vx (:309)."""

    def __init__(self, o):
        """Build from an oracle.Oracle3D of scheme CPML."""
        super().__init__(o)
        self.src = tuple(q + 5 for q in self.src)

    def step(self, it, w):
        T, dt = self.T, self.dt
        self._velocity(False)
        s = self.src
        self.vz[s] = self.vz[s] + (dt * T(np.float32(w))) / self.rho[s]
        self._stress()
        rx, ry, rz = self.rec
        self.data[it] = self.vx[rx[0], ry[0], rz[0]].astype(np.float32)


class Twin3DSPML(Twin3DTensor):
    """Elastic3D_SSG_SPML.update_SSG_SPML (src/Elastic3D_SSG_SPML.py:160-393):
    inside the PML predicate every component is advanced as split parts
    psi_d = ((1 - dt/2 d) psi_d + dt*term_d) / (1 + dt/2 d) (damping d only)
    and set to their sum; outside it the plain update.  Normal stresses use
    the cell's own lam, mu (:300-302); the point force is
    vz[src] += dt*w / rho[src] after the velocity phase (:294); one receiver
    records vx (:393)."""

    SPLIT = ("vx_x", "vx_y", "vx_z", "vy_x", "vy_y", "vy_z", "vz_x", "vz_y", "vz_z",
             "sxx_x", "sxx_y", "sxx_z", "syy_x", "syy_y", "syy_z",
             "sxy_x", "sxy_y", "sxz_x", "sxz_z", "syz_y", "syz_z",
             "szz_x", "szz_y", "szz_z")

    def __init__(self, o):
        """Build from an oracle.Oracle3D of scheme SPML."""
        super().__init__(o)
        self.split = {n: np.zeros_like(self.vx) for n in self.SPLIT}

    def _fac(self, q, half, box):
        """(1 - dt/2 d, 1 + dt/2 d) on axis q at the box's integer or half points."""
        T = self.T
        prof, _ = self.axes[q]
        shape = [1, 1, 1]
        shape[q] = -1
        d = prof["pml_half" if half else "pml"][box[q]].reshape(shape)
        hdt = T(0.5) * self.dt
        return T(1) - hdt * d, T(1) + hdt * d

    def _split(self, names, terms, halves, axes, mask, box):
        """Advance the split parts `names` by their terms; returns their sum."""
        total = None
        for name, term, half, q in zip(names, terms, halves, axes):
            n, d = self._fac(q, half, box)
            old = self.split[name][box]
            new = (n * old + term) / d
            self.split[name][box] = np.where(mask, new, old)
            total = new if total is None else total + new
        return total

    def step(self, it, w):
        T, N, dt = self.T, self.N, self.dt
        nx, ny, nz = self.vx.shape
        dx, dy, dz = self.h
        S = lambda a, b: slice(a, b)
        r, lam, mu = self.rho, self.lam, self.mu
        with np.errstate(all="ignore"):
            # vx :182-205
            B = (S(N, nx - N - 1), S(N + 1, ny - N), S(N + 1, nz - N))
            d1 = self._d(self.sxx, B, 0, True) / dx
            d2 = self._d(self.sxy, B, 1, False) / dy
            d3 = self._d(self.sxz, B, 2, False) / dz
            ro = T(1) / r[B]
            mk = self._mask(B, (1, 0, 0))
            sp = self._split(("vx_x", "vx_y", "vx_z"), (d1 * dt * ro, d2 * dt * ro, d3 * dt * ro),
                             (True, False, False), (0, 1, 2), mk, B)
            self.vx[B] = np.where(mk, sp, self.vx[B] + (d1 + d2 + d3) * dt * ro)
            # vy :207-233
            B = (S(N + 1, nx - N), S(N, ny - N - 1), S(N + 1, nz - N))
            Bj = (B[0], S(N + 1, ny - N), B[2])
            ro = T(1) / (T(0.5) * (r[B] + r[Bj]))
            d1 = self._d(self.sxy, B, 0, False) / dx
            d2 = self._d(self.syy, B, 1, True) / dy
            d3 = self._d(self.syz, B, 2, False) / dz
            mk = self._mask(B, (0, 1, 0))
            sp = self._split(("vy_x", "vy_y", "vy_z"), (dt * d1 * ro, dt * d2 * ro, dt * d3 * ro),
                             (False, True, False), (0, 1, 2), mk, B)
            self.vy[B] = np.where(mk, sp, self.vy[B] + (d1 + d2 + d3) * dt * ro)
            # vz :235-259
            B = (S(N + 1, nx - N), S(N + 1, ny - N), S(N, nz - N - 1))
            Bj = (B[0], S(N + 2, ny - N + 1), B[2])
            Bij = (S(N + 2, nx - N + 1), S(N + 2, ny - N + 1), B[2])
            Bi = (S(N + 2, nx - N + 1), B[1], B[2])
            ro = T(1) / (T(0.25) * (r[B] + r[Bj] + r[Bij] + r[Bi]))
            d1 = self._d(self.sxz, B, 0, False) / dx
            d2 = self._d(self.syz, B, 1, False) / dy
            d3 = self._d(self.szz, B, 2, True) / dz
            mk = self._mask(B, (0, 0, 1))
            sp = self._split(("vz_x", "vz_y", "vz_z"), (dt * d1 * ro, dt * d2 * ro, dt * d3 * ro),
                             (False, False, True), (0, 1, 2), mk, B)
            self.vz[B] = np.where(mk, sp, self.vz[B] + (d1 + d2 + d3) * dt * ro)
            # point force :294
            s = self.src
            self.vz[s] = self.vz[s] + (dt * T(np.float32(w))) / r[s]
            # normal stresses :296-333, the cell's own lam and mu
            B = (S(N + 1, nx - N), S(N + 1, ny - N), S(N + 1, nz - N))
            lm, u = lam[B], mu[B]
            l2m = lm + T(2) * u
            e1 = self._d(self.vx, B, 0, False) / dx
            e2 = self._d(self.vy, B, 1, False) / dy
            e3 = self._d(self.vz, B, 2, False) / dz
            mk = self._mask(B, (0, 0, 0))
            h3 = (False, False, False)
            xyz = (0, 1, 2)
            sxx = self._split(("sxx_x", "sxx_y", "sxx_z"), (dt * l2m * e1, dt * lm * e2, dt * lm * e3), h3, xyz,
                              mk, B)
            syy = self._split(("syy_x", "syy_y", "syy_z"), (dt * lm * e1, dt * l2m * e2, dt * lm * e3), h3, xyz,
                              mk, B)
            szz = self._split(("szz_x", "szz_y", "szz_z"), (dt * lm * e1, dt * lm * e2, dt * l2m * e3), h3, xyz,
                              mk, B)
            self.sxx[B] = np.where(mk, sxx, self.sxx[B] + (l2m * e1 + lm * (e3 + e2)) * dt)
            self.syy[B] = np.where(mk, syy, self.syy[B] + (l2m * e2 + lm * (e1 + e3)) * dt)
            self.szz[B] = np.where(mk, szz, self.szz[B] + (l2m * e3 + lm * (e1 + e2)) * dt)
            # sxy :334-350
            B = (S(N + 1, nx - N), S(N + 1, ny - N), S(N, nz - N))
            Bj = (B[0], S(N + 2, ny - N + 1), B[2])
            Bi = (S(N + 2, nx - N + 1), B[1], B[2])
            m4 = T(0.25) * (mu[Bj] + mu[B] + mu[B] + mu[Bi])
            e1 = self._d(self.vy, B, 0, True) / dx
            e2 = self._d(self.vx, B, 1, True) / dy
            mk = self._mask(B, (1, 1, 0))
            sp = self._split(("sxy_x", "sxy_y"), (dt * m4 * e1, dt * m4 * e2), (True, True), (0, 1), mk, B)
            self.sxy[B] = np.where(mk, sp, self.sxy[B] + m4 * (e2 + e1) * dt)
            # sxz :352-371
            B = (S(N, nx - N - 1), S(N, ny - N), S(N, nz - N - 1))
            Bi = (S(N + 1, nx - N), B[1], B[2])
            Bj = (B[0], S(N + 1, ny - N + 1), B[2])
            m4 = T(0.25) * (mu[B] + mu[Bi] + mu[B] + mu[Bj])
            e1 = self._d(self.vz, B, 0, True) / dx
            e3 = self._d(self.vx, B, 2, True) / dz
            mk = self._mask(B, (1, 0, 1))
            sp = self._split(("sxz_x", "sxz_z"), (dt * m4 * e1, dt * m4 * e3), (True, True), (0, 2), mk, B)
            self.sxz[B] = np.where(mk, sp, self.sxz[B] + m4 * (e3 + e1) * dt)
            # syz :373-391
            B = (S(N, nx - N), S(N, ny - N - 1), S(N, nz - N - 1))
            Bj = (B[0], S(N + 1, ny - N), B[2])
            Bk = (B[0], B[1], S(N + 1, nz - N))
            m4 = T(0.25) * (mu[Bj] + mu[B] + mu[Bk] + mu[B])
            e2 = self._d(self.vz, B, 1, True) / dy
            e3 = self._d(self.vy, B, 2, True) / dz
            mk = self._mask(B, (0, 1, 1))
            sp = self._split(("syz_y", "syz_z"), (dt * m4 * e2, dt * m4 * e3), (True, True), (1, 2), mk, B)
            self.syz[B] = np.where(mk, sp, self.syz[B] + m4 * (e3 + e2) * dt)
        rx, ry, rz = self.rec
        self.data[it] = self.vx[rx[0], ry[0], rz[0]].astype(np.float32)
