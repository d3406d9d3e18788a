// elastic2d.cu -- 2D P-SV staggered-grid kernels with ADE-CPML.
//
// Restates src/Elastic2D_CPML.py as two passes per step, one thread per cell:
//   k2_velocity<VS>  vx, vz, point source                 update_SSG_VS :144-170
//   k2_stress<VS>    sxx szz, sxz (+ receivers of v)       update_SSG_VS :172-200
//   k2_velocity<SV>  / k2_stress<SV>                       update_SSG_SV :218-274
//   k2_velocity<RSG> / k2_stress<RSG>                      update_RSG    :292-353
// Block = 32 (z, contiguous) x 8 (x).  CPML memory variables live only on their
// slabs (mem[0]: x direction (4, lo+hi, nz); mem[1]: z direction (4, nx, lo+hi)),
// components x: sxx_dx sxz_dx dvx_dx dvz_dx, z: sxz_dz szz_dz dvz_dz dvx_dz --
// the same named arrays serve all three schemes, as in the reference.
#include <algorithm>

#include "sw_device.cuh"
#include "sw_stencil2d.cuh"
#include "sw_tma.cuh"

namespace sw {

// single-shot tile: 32 (z) x 4 (x) cells, one per thread (config 1, 400^2:
// 13.3 Gcell/s against 12.8 with 32 x 8 on B200)
// Resident blocks per SM the float batched kernels are compiled for: a full
// SM (2048 threads).  Their loads of many shots' taps are latency bound, and
// full occupancy (4x32 tiles: 16 blocks, 32 registers with a few spills)
// measured 28.9 against 20.3 Gcell/s with the compiler's own register count
// (50: 9 blocks) on 64 ragged shots.  The single-shot kernels keep theirs
// (full occupancy made them slower: 12.6 against 13.3 Gcell/s at 400^2), and
// so do the double ones.
#define SW_BATCH_MINB (sizeof(T) == 4 ? 2048 / (BX * BZ) : 1)
constexpr int T2Z = 32;
constexpr int T2X = 4;

// ---------------------------------------------------------------------------
// velocity update of cell (i, j), 0 <= i < nx, 0 <= j < nz
template <typename T, int N, int SCHEME>
__device__ __forceinline__ void vel2_cell(const P2<T>& p, int i, int j, int it, T amp, int src_here) {
  const int nx = p.nx, nz = p.nz;
  const long long idx = (long long)i * nz + j;
  const T dx = p.dx, dz = p.dz, dt = p.dt;
  T c[N];
#pragma unroll
  for (int m = 0; m < N; ++m) c[m] = p.c[m];
  const T* sxx = p.f[2];
  const T* szz = p.f[3];
  const T* sxz = p.f[4];
  T* vx = p.f[0];
  T* vz = p.f[1];
  const T* rho = p.rho;
  const T* cfx = p.cf[0];
  const T* cfz = p.cf[1];
  const int xi = slab_index(i, nx, p.lo[0], p.hi[0]);
  const int zj = slab_index(j, nz, p.lo[1], p.hi[1]);
  const uint8_t fx = p.fl[0][i], fz = p.fl[1][j];
  const bool any_slab = (xi >= 0 || zj >= 0);

  if (SCHEME == SW2D_SSG_VS) {
    // vx at (i, j) :144-154; vz at (i+1/2, j+1/2) :156-167, then the source :170
    const bool ux = i >= N + 1 && i < nx - N && j >= N + 1 && j < nz - N;
    const bool uz = i >= N && i < nx - N - 1 && j >= N && j < nz - N - 1;
    const bool src = src_here && i == p.si && j == p.sk;
    // stencil sums of both components, divided by the spacings as one group
    const long long row = (long long)i * nz;
    T t0[2 * N], t1[2 * N], t2[2 * N], t3[2 * N];
    taps_x<T, N>(t0, sxx, i - N, j, nx, nz);      // Dx2bm sxx at vx
    taps_z<T, N>(t1, sxz, row, j - N, nz);        // Dz2bm sxz at vx
    taps_x<T, N>(t2, sxz, i - N + 1, j, nx, nz);  // Dx2fm sxz at vz
    taps_z<T, N>(t3, szz, row, j - N + 1, nz);    // Dz2fm szz at vz
    const long long i1 = (long long)min(i + 1, nx - 1) * nz, j1 = min(j + 1, nz - 1);
    const T r00 = ldg(rho + idx), r01 = ldg(rho + row + j1), r11 = ldg(rho + i1 + j1), r10 = ldg(rho + i1 + j);
    T sd[4] = {ux ? tapsum<T, N>(t0, c) : (T)0, ux ? tapsum<T, N>(t1, c) : (T)0,
               uz ? tapsum<T, N>(t2, c) : (T)0, uz ? tapsum<T, N>(t3, c) : (T)0};
    {
      const T hd[4] = {dx, dz, dx, dz};
      const T hr[4] = {p.rd[0], p.rd[1], p.rd[0], p.rd[1]};
      divc_group<4>(sd, hd, hr, p.fast_div & 1);
    }
    T tq[2] = {0, 0}, td[2] = {1, 1};
    if (ux) {
      T dsxxdx = sd[0], dsxzdz = sd[1];
      if (any_slab && ((fx & 1) || (fz & 1))) {
        if (xi >= 0) pml2(mx(p, 0, xi, j), cfx[CB * nx + i], cfx[CA * nx + i], cfx[CK * nx + i], dsxxdx);
        if (zj >= 0) pml2(mz(p, 0, i, zj), cfz[CB * nz + j], cfz[CA * nz + j], cfz[CK * nz + j], dsxzdz);
      }
      tq[0] = (dsxxdx + dsxzdz) * dt;
      td[0] = r00;
    }
    if (uz) {
      td[1] = (T)0.25 * (r00 + r01 + r11 + r10);
      T dsxzdx = sd[2], dszzdz = sd[3];
      if (any_slab && ((fx & 2) || (fz & 2))) {
        if (xi >= 0) pml2(mx(p, 1, xi, j), cfx[CBH * nx + i], cfx[CAH * nx + i], cfx[CKH * nx + i], dsxzdx);
        if (zj >= 0) pml2(mz(p, 1, i, zj), cfz[CBH * nz + j], cfz[CAH * nz + j], cfz[CKH * nz + j], dszzdz);
      }
      tq[1] = (dszzdz + dsxzdx) * dt;
    }
    divv_group<2>(tq, td);
    if (ux) vx[idx] = vx[idx] + tq[0];
    if (uz || src) {
      T v = vz[idx];
      if (uz) v = v + tq[1];
      if (src) {
        T t = dt * p.wav[it];
        t = div_v(t, ldg(rho + idx));
        v = v + t;
      }
      vz[idx] = v;
    }
  } else if (SCHEME == SW2D_SSG_SV) {
    // vx at (i+1/2, j) :218-229, then the source :245; vz at (i, j+1/2) :231-242
    const bool ux = i >= N && i < nx - N - 1 && j >= N + 1 && j < nz - N;
    const bool uz = i >= N + 1 && i < nx - N && j >= N && j < nz - N - 1;
    const bool src = src_here && i == p.si && j == p.sk;
    const long long row = (long long)i * nz;
    T t0[2 * N], t1[2 * N], t2[2 * N], t3[2 * N];
    taps_x<T, N>(t0, sxx, i - N + 1, j, nx, nz);  // Dx2fm sxx at vx
    taps_z<T, N>(t1, sxz, row, j - N, nz);        // Dz2bm sxz at vx
    taps_x<T, N>(t2, sxz, i - N, j, nx, nz);      // Dx2bm sxz at vz
    taps_z<T, N>(t3, szz, row, j - N + 1, nz);    // Dz2fm szz at vz
    T sd[4] = {ux ? tapsum<T, N>(t0, c) : (T)0, ux ? tapsum<T, N>(t1, c) : (T)0,
               uz ? tapsum<T, N>(t2, c) : (T)0, uz ? tapsum<T, N>(t3, c) : (T)0};
    {
      const T hd[4] = {dx, dz, dx, dz};
      const T hr[4] = {p.rd[0], p.rd[1], p.rd[0], p.rd[1]};
      divc_group<4>(sd, hd, hr, p.fast_div & 1);
    }
    T tq[2] = {0, 0}, td[2] = {1, 1};
    if (ux) {
      T dsxxdx = sd[0], dsxzdz = sd[1];
      td[0] = (ldg(rho + idx) + ldg(rho + idx + nz)) / (T)2;
      if (any_slab && ((fx & 2) || (fz & 1))) {
        if (xi >= 0) pml2(mx(p, 0, xi, j), cfx[CBH * nx + i], cfx[CAH * nx + i], cfx[CKH * nx + i], dsxxdx);
        if (zj >= 0) pml2(mz(p, 0, i, zj), cfz[CB * nz + j], cfz[CA * nz + j], cfz[CK * nz + j], dsxzdz);
      }
      tq[0] = (dsxxdx + dsxzdz) * dt;
    }
    if (uz) {
      td[1] = (T)0.5 * (ldg(rho + idx) + ldg(rho + idx + 1));
      T dsxzdx = sd[2], dszzdz = sd[3];
      if (any_slab && ((fx & 1) || (fz & 2))) {
        if (xi >= 0) pml2(mx(p, 1, xi, j), cfx[CB * nx + i], cfx[CA * nx + i], cfx[CK * nx + i], dsxzdx);
        if (zj >= 0) pml2(mz(p, 1, i, zj), cfz[CBH * nz + j], cfz[CAH * nz + j], cfz[CKH * nz + j], dszzdz);
      }
      tq[1] = (dszzdz + dsxzdx) * dt;
    }
    divv_group<2>(tq, td);
    if (ux || src) {
      T v = vx[idx];
      if (ux) v = v + tq[0];
      if (src) {
        T t = dt * p.wav[it];
        t = div_v(t, ldg(rho + idx));
        v = v + t;
      }
      vx[idx] = v;
    }
    if (uz) vz[idx] = vz[idx] + tq[1];
  } else {  // SW2D_RSG, :292-323
    const bool upd = i >= N + 1 && i < nx - N && j >= N + 1 && j < nz - N;
    const bool src = src_here && (i == p.si || i == p.si - 1) && (j == p.sk || j == p.sk - 1);
    if (upd) {
      const T dsxxrx = drx_bm<T, N>(sxx, idx, nz, c), dsxxrz = drz_bm<T, N>(sxx, idx, nz, c);
      const T dszzrx = drx_bm<T, N>(szz, idx, nz, c), dszzrz = drz_bm<T, N>(szz, idx, nz, c);
      const T dsxzrx = drx_bm<T, N>(sxz, idx, nz, c), dsxzrz = drz_bm<T, N>(sxz, idx, nz, c);
      T dsxxdx = div_c(dsxxrz - dsxxrx, (T)2 * dx, p.rd2[0], (p.fast_div >> 1) & 1);
      T dszzdz = div_c(dszzrz + dszzrx, (T)2 * dz, p.rd2[1], (p.fast_div >> 1) & 1);
      T dsxzdx = div_c(dsxzrz - dsxzrx, (T)2 * dx, p.rd2[0], (p.fast_div >> 1) & 1);
      T dsxzdz = div_c(dsxzrz + dsxzrx, (T)2 * dz, p.rd2[1], (p.fast_div >> 1) & 1);
      const T rh = ldg(rho + idx);
      if (any_slab && ((fx & 1) || (fz & 1))) {
        if (xi >= 0) {
          pml2(mx(p, 0, xi, j), cfx[CB * nx + i], cfx[CA * nx + i], cfx[CK * nx + i], dsxxdx);
          pml2(mx(p, 1, xi, j), cfx[CB * nx + i], cfx[CA * nx + i], cfx[CK * nx + i], dsxzdx);
        }
        if (zj >= 0) {
          pml2(mz(p, 1, i, zj), cfz[CB * nz + j], cfz[CA * nz + j], cfz[CK * nz + j], dszzdz);
          pml2(mz(p, 0, i, zj), cfz[CB * nz + j], cfz[CA * nz + j], cfz[CK * nz + j], dsxzdz);
        }
      }
      T t = (dsxxdx + dsxzdz) * dt;
      t = div_v(t, rh);
      vx[idx] = vx[idx] + t;
      T u = (dszzdz + dsxzdx) * dt;
      u = div_v(u, rh);
      T v = vz[idx] + u;
      if (src) {
        T s = dt * amp;
        s = div_v(s, (T)8 * rh);
        v = v + s;
      }
      vz[idx] = v;
    } else if (src) {
      T s = dt * amp;
      s = div_v(s, (T)8 * ldg(rho + idx));
      vz[idx] = vz[idx] + s;
    }
  }
}

// stress update of cell (i, j), then the next step's moment-tensor source
template <typename T, int N, int SCHEME>
// flags: bit 0 adds step it+1's moment-tensor source after the update, bit 1
// zeroes sxx on the x layer N first (the free-surface hook AEA of step it+1,
// Elastic2D_CPML.py:122-125, which precedes the source of that step)
__device__ __forceinline__ void str2_cell(const P2<T>& p, int i, int j, int it, int inject_next) {
  const int nx = p.nx, nz = p.nz;
  const long long idx = (long long)i * nz + j;
  const T dx = p.dx, dz = p.dz, dt = p.dt;
  T c[N];
#pragma unroll
  for (int m = 0; m < N; ++m) c[m] = p.c[m];
  const T* vx = p.f[0];
  const T* vz = p.f[1];
  T* sxx = p.f[2];
  T* szz = p.f[3];
  T* sxz = p.f[4];
  const T* lam = p.lam;
  const T* mu = p.mu;
  const T* cfx = p.cf[0];
  const T* cfz = p.cf[1];
  const int xi = slab_index(i, nx, p.lo[0], p.hi[0]);
  const int zj = slab_index(j, nz, p.lo[1], p.hi[1]);
  const uint8_t fx = p.fl[0][i], fz = p.fl[1][j];
  const bool any_slab = (xi >= 0 || zj >= 0);

  if (SCHEME == SW2D_SSG_VS) {
    // sxx szz at (i+1/2, j) :172-186; sxz at (i, j+1/2) :188-199
    const bool un = i >= N && i < nx - N - 1 && j >= N + 1 && j < nz - N;
    const bool us = i >= N + 1 && i < nx - N && j >= N && j < nz - N - 1;
    const long long row = (long long)i * nz;
    T t0[2 * N], t1[2 * N], t2[2 * N], t3[2 * N];
    taps_x<T, N>(t0, vx, i - N + 1, j, nx, nz);   // Dx2fm vx at sxx
    taps_z<T, N>(t1, vz, row, j - N, nz);         // Dz2bm vz at sxx
    taps_x<T, N>(t2, vz, i - N, j, nx, nz);       // Dx2bm vz at sxz
    taps_z<T, N>(t3, vx, row, j - N + 1, nz);     // Dz2fm vx at sxz
    T sd[4] = {un ? tapsum<T, N>(t0, c) : (T)0, un ? tapsum<T, N>(t1, c) : (T)0,
               us ? tapsum<T, N>(t2, c) : (T)0, us ? tapsum<T, N>(t3, c) : (T)0};
    {
      const T hd[4] = {dx, dz, dx, dz};
      const T hr[4] = {p.rd[0], p.rd[1], p.rd[0], p.rd[1]};
      divc_group<4>(sd, hd, hr, p.fast_div & 1);
    }
    if (un) {
      const T lhx = (T)0.5 * (ldg(lam + idx) + ldg(lam + idx + nz));
      const T mhx = (T)0.5 * (ldg(mu + idx) + ldg(mu + idx + nz));
      const T lpm = lhx + (T)2 * mhx;
      T dvxdx = sd[0], dvzdz = sd[1];
      if (any_slab && ((fx & 2) || (fz & 1))) {
        if (xi >= 0) pml2(mx(p, 2, xi, j), cfx[CBH * nx + i], cfx[CAH * nx + i], cfx[CKH * nx + i], dvxdx);
        if (zj >= 0) pml2(mz(p, 2, i, zj), cfz[CB * nz + j], cfz[CA * nz + j], cfz[CK * nz + j], dvzdz);
      }
      sxx[idx] = sxx[idx] + (lpm * dvxdx + lhx * dvzdz) * dt;
      szz[idx] = szz[idx] + (lpm * dvzdz + lhx * dvxdx) * dt;
    }
    if (us) {
      const T mhz = (T)0.5 * (ldg(mu + idx + 1) + ldg(mu + idx));
      T dvzdx = sd[2], dvxdz = sd[3];
      if (any_slab && ((fx & 1) || (fz & 2))) {
        if (xi >= 0) pml2(mx(p, 3, xi, j), cfx[CB * nx + i], cfx[CA * nx + i], cfx[CK * nx + i], dvzdx);
        if (zj >= 0) pml2(mz(p, 3, i, zj), cfz[CBH * nz + j], cfz[CAH * nz + j], cfz[CKH * nz + j], dvxdz);
      }
      sxz[idx] = sxz[idx] + mhz * (dvxdz + dvzdx) * dt;
    }
  } else if (SCHEME == SW2D_SSG_SV) {
    // sxx szz at (i, j) :247-260; sxz at (i+1/2, j+1/2) :262-273
    const bool un = i >= N + 1 && i < nx - N && j >= N + 1 && j < nz - N;
    const bool us = un;
    const long long row = (long long)i * nz;
    T t0[2 * N], t1[2 * N], t2[2 * N], t3[2 * N];
    taps_x<T, N>(t0, vx, i - N, j, nx, nz);       // Dx2bm vx at sxx
    taps_z<T, N>(t1, vz, row, j - N, nz);         // Dz2bm vz at sxx
    taps_x<T, N>(t2, vz, i - N + 1, j, nx, nz);   // Dx2fm vz at sxz
    taps_z<T, N>(t3, vx, row, j - N + 1, nz);     // Dz2fm vx at sxz
    T sd[4] = {un ? tapsum<T, N>(t0, c) : (T)0, un ? tapsum<T, N>(t1, c) : (T)0,
               un ? tapsum<T, N>(t2, c) : (T)0, un ? tapsum<T, N>(t3, c) : (T)0};
    {
      const T hd[4] = {dx, dz, dx, dz};
      const T hr[4] = {p.rd[0], p.rd[1], p.rd[0], p.rd[1]};
      divc_group<4>(sd, hd, hr, p.fast_div & 1);
    }
    if (un) {
      const T lm = ldg(lam + idx);
      const T lpm = ldg(lam + idx) + (T)2 * ldg(mu + idx);
      T dvxdx = sd[0], dvzdz = sd[1];
      if (any_slab && ((fx & 1) || (fz & 1))) {
        if (xi >= 0) pml2(mx(p, 2, xi, j), cfx[CB * nx + i], cfx[CA * nx + i], cfx[CK * nx + i], dvxdx);
        if (zj >= 0) pml2(mz(p, 2, i, zj), cfz[CB * nz + j], cfz[CA * nz + j], cfz[CK * nz + j], dvzdz);
      }
      sxx[idx] = sxx[idx] + (lpm * dvxdx + lm * dvzdz) * dt;
      szz[idx] = szz[idx] + (lpm * dvzdz + lm * dvxdx) * dt;
    }
    if (us) {
      const T m4 = (T)0.25 * (ldg(mu + idx + 1) + ldg(mu + idx) + ldg(mu + idx + nz + 1) + ldg(mu + idx + nz));
      T dvzdx = sd[2], dvxdz = sd[3];
      if (any_slab && ((fx & 2) || (fz & 2))) {
        if (xi >= 0) pml2(mx(p, 3, xi, j), cfx[CBH * nx + i], cfx[CAH * nx + i], cfx[CKH * nx + i], dvzdx);
        if (zj >= 0) pml2(mz(p, 3, i, zj), cfz[CBH * nz + j], cfz[CAH * nz + j], cfz[CKH * nz + j], dvxdz);
      }
      sxz[idx] = sxz[idx] + m4 * (dvxdz + dvzdx) * dt;
    }
  } else {  // RSG :326-353
    if (i >= N && i < nx - N - 1 && j >= N && j < nz - N - 1) {
      const T lm = ldg(lam + idx), u = ldg(mu + idx);
      const T lpm = lm + (T)2 * u;
      const T dvxrx = drx_fm<T, N>(vx, idx, nz, c), dvxrz = drz_fm<T, N>(vx, idx, nz, c);
      const T dvzrx = drx_fm<T, N>(vz, idx, nz, c), dvzrz = drz_fm<T, N>(vz, idx, nz, c);
      T dvxdx = div_c(dvxrz - dvxrx, (T)2 * dx, p.rd2[0], (p.fast_div >> 1) & 1);
      T dvxdz = div_c(dvxrz + dvxrx, (T)2 * dz, p.rd2[1], (p.fast_div >> 1) & 1);
      T dvzdx = div_c(dvzrz - dvzrx, (T)2 * dx, p.rd2[0], (p.fast_div >> 1) & 1);
      T dvzdz = div_c(dvzrz + dvzrx, (T)2 * dz, p.rd2[1], (p.fast_div >> 1) & 1);
      if (any_slab && ((fx & 2) || (fz & 2))) {
        if (xi >= 0) {
          pml2(mx(p, 2, xi, j), cfx[CBH * nx + i], cfx[CAH * nx + i], cfx[CKH * nx + i], dvxdx);
          pml2(mx(p, 3, xi, j), cfx[CBH * nx + i], cfx[CAH * nx + i], cfx[CKH * nx + i], dvzdx);
        }
        if (zj >= 0) {
          pml2(mz(p, 3, i, zj), cfz[CBH * nz + j], cfz[CAH * nz + j], cfz[CKH * nz + j], dvxdz);
          pml2(mz(p, 2, i, zj), cfz[CBH * nz + j], cfz[CAH * nz + j], cfz[CKH * nz + j], dvzdz);
        }
      }
      sxx[idx] = sxx[idx] + (lpm * dvxdx + lm * dvzdz) * dt;
      szz[idx] = szz[idx] + (lpm * dvzdz + lm * dvxdx) * dt;
      sxz[idx] = sxz[idx] + (u * (dvxdz + dvzdx)) * dt;
    }
  }
  // moment-tensor source of step it+1, added after this cell's own update
  // (nothing reads the stresses between here and the next velocity pass)
  if ((inject_next & 2) && i == N) sxx[idx] = (T)0;
  if ((inject_next & 1) && i == p.si && j == p.sk) {
    const T w = p.wav[it + 1];
    sxx[idx] = sxx[idx] + w * p.mneg[0];
    szz[idx] = szz[idx] + w * p.mneg[1];
    sxz[idx] = sxz[idx] + w * p.mneg[2];
  }
}

template <typename T, int N, int SCHEME>
__global__ void __launch_bounds__(T2Z * T2X)
k2_velocity(const __grid_constant__ P2<T> p, int it, T amp, int src_here) {
  const int j = blockIdx.x * T2Z + threadIdx.x;
  const int i = blockIdx.y * T2X + threadIdx.y;
  if (i >= p.nx || j >= p.nz) return;
  vel2_cell<T, N, SCHEME>(p, i, j, it, amp, src_here);
}

template <typename T, int N, int SCHEME>
__global__ void __launch_bounds__(T2Z * T2X)
k2_stress(const __grid_constant__ P2<T> p, int it, int inject_next) {
  // receivers of the velocity fields (final for this step, not written here)
  {
    const long long b = blockIdx.x + (long long)gridDim.x * blockIdx.y;
    const long long r = b * (T2Z * T2X) + threadIdx.y * T2Z + threadIdx.x;
    if (r < p.nrec) store_rec(p.rec_data, p.rec_f64, (long long)it * p.nrec + r, p.f[p.rec_field][p.rec_idx[r]]);
  }
  const int j = blockIdx.x * T2Z + threadIdx.x;
  const int i = blockIdx.y * T2X + threadIdx.y;
  if (i >= p.nx || j >= p.nz) return;
  str2_cell<T, N, SCHEME>(p, i, j, it, inject_next);
}

// moment-tensor source of step it before the velocity pass
// (2D form of Elastic3D_SSG_Tensor.py:186-193)
template <typename T>
__global__ void k2_moment_inject(const __grid_constant__ P2<T> p, int it) {
  const long long s = (long long)p.si * p.nz + p.sk;
  const T w = p.wav[it];
  p.f[2][s] = p.f[2][s] + w * p.mneg[0];
  p.f[3][s] = p.f[3][s] + w * p.mneg[1];
  p.f[4][s] = p.f[4][s] + w * p.mneg[2];
}

// free-surface hook AEA (Elastic2D_CPML.py:122-125): sxx = 0 on the x layer N
template <typename T>
__global__ void k2_aea(const __grid_constant__ P2<T> p, int n_layer) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < p.nz) p.f[2][(long long)n_layer * p.nz + j] = (T)0;
}

template <typename T>
__global__ void k2_gather(const __grid_constant__ P2<T> p, int it) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < p.nrec) store_rec(p.rec_data, p.rec_f64, (long long)it * p.nrec + r, p.f[p.rec_field][p.rec_idx[r]]);
}

// aea: bit 0 applies the free-surface hook before this step, bit 1 folds the
// next step's into this step's stress pass
template <typename T, int N, int S>
static cudaError_t launch2(const P2<T>& p, int it, T amp, bool gather_in_stress, bool pre_inject,
                           bool inject_next, int aea, cudaStream_t st) {
  dim3 block(T2Z, T2X);
  dim3 grid((p.nz + T2Z - 1) / T2Z, (p.nx + T2X - 1) / T2X);
  const bool moment = p.src_kind == SW_SRC_MOMENT;
  if (aea & 1) k2_aea<T><<<(p.nz + 255) / 256, 256, 0, st>>>(p, N);
  if (moment && pre_inject) k2_moment_inject<T><<<1, 1, 0, st>>>(p, it);
  k2_velocity<T, N, S><<<grid, block, 0, st>>>(p, it, amp, (p.src_kind != SW_SRC_NONE && !moment) ? 1 : 0);
  P2<T> q = p;
  if (!gather_in_stress) q.nrec = 0;
  k2_stress<T, N, S><<<grid, block, 0, st>>>(q, it, ((moment && inject_next) ? 1 : 0) | ((aea & 2) ? 2 : 0));
  if (!gather_in_stress && p.nrec > 0) k2_gather<T><<<(p.nrec + 255) / 256, 256, 0, st>>>(p, it);
  return cudaGetLastError();
}

template <typename T, int S>
static cudaError_t dispatch2(const P2<T>& p, int order, int it, T amp, bool g, bool pre, bool nxt, int aea,
                             cudaStream_t st) {
  switch (order) {
    case 1: return launch2<T, 1, S>(p, it, amp, g, pre, nxt, aea, st);
    case 2: return launch2<T, 2, S>(p, it, amp, g, pre, nxt, aea, st);
    case 3: return launch2<T, 3, S>(p, it, amp, g, pre, nxt, aea, st);
    case 4: return launch2<T, 4, S>(p, it, amp, g, pre, nxt, aea, st);
    case 5: return launch2<T, 5, S>(p, it, amp, g, pre, nxt, aea, st);
    case 6: return launch2<T, 6, S>(p, it, amp, g, pre, nxt, aea, st);
    case 7: return launch2<T, 7, S>(p, it, amp, g, pre, nxt, aea, st);
    case 8: return launch2<T, 8, S>(p, it, amp, g, pre, nxt, aea, st);
    default: return cudaErrorInvalidValue;
  }
}

template <typename T>
cudaError_t sw2_step(const P2<T>& p, int scheme, int order, int it, T amp, bool gather_in_stress, bool pre_inject,
                     bool inject_next, int aea, cudaStream_t st) {
  if (scheme == SW2D_SSG_VS)
    return dispatch2<T, SW2D_SSG_VS>(p, order, it, amp, gather_in_stress, pre_inject, inject_next, aea, st);
  if (scheme == SW2D_SSG_SV)
    return dispatch2<T, SW2D_SSG_SV>(p, order, it, amp, gather_in_stress, pre_inject, inject_next, aea, st);
  return dispatch2<T, SW2D_RSG>(p, order, it, amp, gather_in_stress, pre_inject, inject_next, aea, st);
}

template <typename T>
cudaError_t sw2_moment_inject(const P2<T>& p, int it, cudaStream_t st) {
  k2_moment_inject<T><<<1, 1, 0, st>>>(p, it);
  return cudaGetLastError();
}
template cudaError_t sw2_moment_inject<float>(const P2<float>&, int, cudaStream_t);
template cudaError_t sw2_moment_inject<double>(const P2<double>&, int, cudaStream_t);

// ---------------------------------------------------------------------------
// persistent path: all steps of a run in one cooperative launch
// ---------------------------------------------------------------------------
// The phases of a step (source injection when it is not folded, velocity,
// stress with the receivers, a stress-receiver gather) are separated by a
// grid barrier instead of kernel boundaries.  Block leaders count arrivals
// on one word; the last one resets it and advances the generation word, the
// others poll the generation with a bound of SW_WAIT_NS on the global timer.
// A leader that gives up sets bit 1 of the error word and its block leaves;
// every other block then leaves at its next barrier the same way, so the
// launch always ends.  The cooperative launch makes all blocks resident.
// Every cell runs the same per-cell functions in the same phase order as the
// two-launch path, so the results are identical.  Measured on B200 it is
// slower than the two launches per step replayed from a CUDA graph at every
// grid size from 96^2 to 800^2 (12.2 vs 8.9 us per step at 96^2, 17.1 vs
// 11.9 at 400^2): the two grid barriers of a step cost more than the graph's
// launch gaps, so the plan only takes this path when asked to.
struct GridBar2 {
  unsigned int* arrive;
  unsigned int* gen;
  int* err;
};

__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned int atom_add_acq_rel_gpu(unsigned int* p, unsigned int v) {
  unsigned int old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ void red_add_release_gpu(unsigned int* p, unsigned int v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// The block's writes are ordered before its leader's release-acquire
// arrival by the block barrier; the last arrival releases the new
// generation, which every other leader acquires before its block goes on.
__device__ __forceinline__ bool grid_bar(const GridBar2& b) {
  __syncthreads();
  int ok = 1;
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    const unsigned int g = ld_acquire_gpu(b.gen);
    if (atom_add_acq_rel_gpu(b.arrive, 1u) == gridDim.x - 1) {
      atomicExch(b.arrive, 0u);
      red_add_release_gpu(b.gen, 1u);
    } else {
      const uint64_t t0 = global_ns();
      while (ld_acquire_gpu(b.gen) == g) {
        if (global_ns() - t0 > SW_WAIT_NS) {
          atomicOr(b.err, 2);
          ok = 0;
          break;
        }
      }
    }
  }
  return __syncthreads_and(ok) != 0;
}

constexpr int T2PZ = 32, T2PX = 16;  // persistent block: 512 threads, 32 (z) x 16 (x) cells per tile

template <typename T, int N, int S>
__global__ void __launch_bounds__(T2PZ * T2PX)
k2p_run(const __grid_constant__ P2<T> p, int it0, int nsteps, int gather_in_stress, int fold, GridBar2 gb) {
  const int tz = (p.nz + T2PZ - 1) / T2PZ;
  const int ntile = tz * ((p.nx + T2PX - 1) / T2PX);
  const bool moment = p.src_kind == SW_SRC_MOMENT;
  const int src_here = (p.src_kind != SW_SRC_NONE && !moment) ? 1 : 0;
  const int tid = threadIdx.y * T2PZ + threadIdx.x;
  const long long nthr = (long long)gridDim.x * (T2PZ * T2PX);
  const long long gtid = (long long)blockIdx.x * (T2PZ * T2PX) + tid;
  for (int s = 0; s < nsteps; ++s) {
    const int it = it0 + s;
    // the moment-tensor source of step it: folded into the previous stress
    // phase except on the first step and when a receiver records a stress
    if (moment && (s == 0 || !fold)) {
      if (blockIdx.x == 0 && tid == 0) {
        const long long c = (long long)p.si * p.nz + p.sk;
        const T w = p.wav[it];
        p.f[2][c] = p.f[2][c] + w * p.mneg[0];
        p.f[3][c] = p.f[3][c] + w * p.mneg[1];
        p.f[4][c] = p.f[4][c] + w * p.mneg[2];
      }
      if (!grid_bar(gb)) return;
    }
    for (int t = blockIdx.x; t < ntile; t += gridDim.x) {
      const int j = (t % tz) * T2PZ + threadIdx.x, i = (t / tz) * T2PX + threadIdx.y;
      if (i < p.nx && j < p.nz) vel2_cell<T, N, S>(p, i, j, it, (T)0, src_here);
    }
    if (!grid_bar(gb)) return;
    if (gather_in_stress)
      for (long long r = gtid; r < p.nrec; r += nthr)
        store_rec(p.rec_data, p.rec_f64, (long long)it * p.nrec + r, p.f[p.rec_field][p.rec_idx[r]]);
    const int nxt = (moment && fold && s < nsteps - 1) ? 1 : 0;
    for (int t = blockIdx.x; t < ntile; t += gridDim.x) {
      const int j = (t % tz) * T2PZ + threadIdx.x, i = (t / tz) * T2PX + threadIdx.y;
      if (i < p.nx && j < p.nz) str2_cell<T, N, S>(p, i, j, it, nxt);
    }
    if (!gather_in_stress && p.nrec > 0) {
      if (!grid_bar(gb)) return;
      for (long long r = gtid; r < p.nrec; r += nthr)
        store_rec(p.rec_data, p.rec_f64, (long long)it * p.nrec + r, p.f[p.rec_field][p.rec_idx[r]]);
    }
    if (s < nsteps - 1 && !grid_bar(gb)) return;
  }
}

template <typename T, int N, int S>
static cudaError_t launch2p(const P2<T>& p, int it0, int nsteps, bool gather_in_stress, bool fold,
                            const GridBar2& gb, cudaStream_t st) {
  auto kern = k2p_run<T, N, S>;
  int dev = 0, nsm = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, T2PZ * T2PX, 0);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const long long ntile = (long long)((p.nz + T2PZ - 1) / T2PZ) * ((p.nx + T2PX - 1) / T2PX);
  const int grid = (int)std::max<long long>(1, std::min<long long>(ntile, (long long)per_sm * nsm));
  e = cudaMemsetAsync(gb.arrive, 0, sizeof(unsigned int), st);
  if (e != cudaSuccess) return e;
  int g = gather_in_stress ? 1 : 0, f = fold ? 1 : 0;
  P2<T> pp = p;
  GridBar2 b = gb;
  void* args[] = {&pp, &it0, &nsteps, &g, &f, &b};
  return cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(T2PZ, T2PX), args, 0, st);
}

template <typename T, int S>
static cudaError_t dispatch2p(const P2<T>& p, int order, int it0, int n, bool g, bool f, const GridBar2& b,
                              cudaStream_t st) {
  switch (order) {
    case 1: return launch2p<T, 1, S>(p, it0, n, g, f, b, st);
    case 2: return launch2p<T, 2, S>(p, it0, n, g, f, b, st);
    case 3: return launch2p<T, 3, S>(p, it0, n, g, f, b, st);
    case 4: return launch2p<T, 4, S>(p, it0, n, g, f, b, st);
    case 5: return launch2p<T, 5, S>(p, it0, n, g, f, b, st);
    case 6: return launch2p<T, 6, S>(p, it0, n, g, f, b, st);
    case 7: return launch2p<T, 7, S>(p, it0, n, g, f, b, st);
    case 8: return launch2p<T, 8, S>(p, it0, n, g, f, b, st);
    default: return cudaErrorInvalidValue;
  }
}

// nsteps >= 1 steps from it0 in one launch; arrive/gen/err: the plan's
// barrier words and error word
template <typename T>
cudaError_t sw2_persistent(const P2<T>& p, int scheme, int order, int it0, int nsteps, bool gather_in_stress,
                           bool fold, unsigned int* bar, int* err, cudaStream_t st) {
  const GridBar2 b{bar, bar + 1, err};
  if (scheme == SW2D_SSG_VS) return dispatch2p<T, SW2D_SSG_VS>(p, order, it0, nsteps, gather_in_stress, fold, b, st);
  if (scheme == SW2D_SSG_SV) return dispatch2p<T, SW2D_SSG_SV>(p, order, it0, nsteps, gather_in_stress, fold, b, st);
  return dispatch2p<T, SW2D_RSG>(p, order, it0, nsteps, gather_in_stress, fold, b, st);
}
template cudaError_t sw2_persistent<float>(const P2<float>&, int, int, int, int, bool, bool, unsigned int*, int*,
                                           cudaStream_t);
template cudaError_t sw2_persistent<double>(const P2<double>&, int, int, int, int, bool, bool, unsigned int*, int*,
                                            cudaStream_t);

// ---------------------------------------------------------------------------
// batched ragged shots: one launch per phase covers every tile of every shot
// ---------------------------------------------------------------------------
template <typename T, int N, int S, int BX, int BZ>
__global__ void __launch_bounds__(BX * BZ, SW_BATCH_MINB) k2b_velocity(const __grid_constant__ Batch2<T> bt, int it) {
  const int2 wk = bt.work[blockIdx.x];
  const P2<T>& p = bt.shots[wk.x - bt.first];
  const int j = (wk.y & 0xffff) * BZ + threadIdx.x, i = (wk.y >> 16) * BX + threadIdx.y;
  if (i >= p.nx || j >= p.nz) return;
  vel2_cell<T, N, S>(p, i, j, it, (T)0, p.src_kind == SW_SRC_FORCE ? 1 : 0);
}

template <typename T, int N, int S, int BX, int BZ>
__global__ void __launch_bounds__(BX * BZ, SW_BATCH_MINB) k2b_stress(const __grid_constant__ Batch2<T> bt, int it, int inject_next) {
  const int2 wk = bt.work[blockIdx.x];
  const P2<T>& p = bt.shots[wk.x - bt.first];
  const int tx = wk.y >> 16, tz = wk.y & 0xffff;
  {
    // receivers of the velocity fields: the shot's first tiles cover them
    const long long t = (long long)tx * ((p.nz + BZ - 1) / BZ) + tz;
    const long long r = t * (BX * BZ) + threadIdx.y * BZ + threadIdx.x;
    if (r < p.nrec) store_rec(p.rec_data, p.rec_f64, (long long)it * p.nrec + r, p.f[p.rec_field][p.rec_idx[r]]);
  }
  const int j = tz * BZ + threadIdx.x, i = tx * BX + threadIdx.y;
  if (i >= p.nx || j >= p.nz) return;
  str2_cell<T, N, S>(p, i, j, it, (inject_next && p.src_kind == SW_SRC_MOMENT) ? 1 : 0);
}

template <typename T>
__global__ void k2b_inject(const __grid_constant__ Batch2<T> bt, int it) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= bt.n) return;
  const P2<T>& p = bt.shots[s];
  if (p.src_kind != SW_SRC_MOMENT) return;
  const long long c = (long long)p.si * p.nz + p.sk;
  const T w = p.wav[it];
  p.f[2][c] = p.f[2][c] + w * p.mneg[0];
  p.f[3][c] = p.f[3][c] + w * p.mneg[1];
  p.f[4][c] = p.f[4][c] + w * p.mneg[2];
}

// tile shapes (x rows, z columns) the autotuner chooses from
constexpr int kBatchTiles[SW_BATCH_TILES][2] = {{8, 32}, {4, 32}, {16, 32}, {4, 64}};

template <typename T, int N, int S, int BX, int BZ>
static cudaError_t launch2b(const Batch2<T>& bt, int total, int it, bool pre, bool nxt, cudaStream_t st) {
  if (pre) k2b_inject<T><<<1, SW_BATCH_GROUP, 0, st>>>(bt, it);
  dim3 block(BZ, BX);
  k2b_velocity<T, N, S, BX, BZ><<<total, block, 0, st>>>(bt, it);
  k2b_stress<T, N, S, BX, BZ><<<total, block, 0, st>>>(bt, it, nxt ? 1 : 0);
  return cudaGetLastError();
}

template <typename T, int N, int S>
static cudaError_t tile2b(const Batch2<T>& bt, int cfg, int total, int it, bool pre, bool nxt, cudaStream_t st) {
  switch (cfg) {
    case 0: return launch2b<T, N, S, 8, 32>(bt, total, it, pre, nxt, st);
    case 1: return launch2b<T, N, S, 4, 32>(bt, total, it, pre, nxt, st);
    case 2: return launch2b<T, N, S, 16, 32>(bt, total, it, pre, nxt, st);
    case 3: return launch2b<T, N, S, 4, 64>(bt, total, it, pre, nxt, st);
    default: return cudaErrorInvalidValue;
  }
}

template <typename T, int S>
static cudaError_t order2b(const Batch2<T>& bt, int order, int cfg, int total, int it, bool pre, bool nxt,
                           cudaStream_t st) {
  switch (order) {
    case 1: return tile2b<T, 1, S>(bt, cfg, total, it, pre, nxt, st);
    case 2: return tile2b<T, 2, S>(bt, cfg, total, it, pre, nxt, st);
    case 3: return tile2b<T, 3, S>(bt, cfg, total, it, pre, nxt, st);
    case 4: return tile2b<T, 4, S>(bt, cfg, total, it, pre, nxt, st);
    case 5: return tile2b<T, 5, S>(bt, cfg, total, it, pre, nxt, st);
    case 6: return tile2b<T, 6, S>(bt, cfg, total, it, pre, nxt, st);
    case 7: return tile2b<T, 7, S>(bt, cfg, total, it, pre, nxt, st);
    case 8: return tile2b<T, 8, S>(bt, cfg, total, it, pre, nxt, st);
    default: return cudaErrorInvalidValue;
  }
}

void sw2b_tile_shape(int cfg, int* bx, int* bz) {
  *bx = kBatchTiles[cfg][0];
  *bz = kBatchTiles[cfg][1];
}

template <typename T>
cudaError_t sw2b_step(const Batch2<T>& bt, int scheme, int order, int cfg, int total, int it, bool pre, bool nxt,
                      cudaStream_t st) {
  if (scheme == SW2D_SSG_VS) return order2b<T, SW2D_SSG_VS>(bt, order, cfg, total, it, pre, nxt, st);
  return order2b<T, SW2D_SSG_SV>(bt, order, cfg, total, it, pre, nxt, st);
}
template cudaError_t sw2b_step<float>(const Batch2<float>&, int, int, int, int, int, bool, bool, cudaStream_t);
template cudaError_t sw2b_step<double>(const Batch2<double>&, int, int, int, int, int, bool, bool, cudaStream_t);

template cudaError_t sw2_step<float>(const P2<float>&, int, int, int, float, bool, bool, bool, int, cudaStream_t);
template cudaError_t sw2_step<double>(const P2<double>&, int, int, int, double, bool, bool, bool, int, cudaStream_t);

}  // namespace sw
