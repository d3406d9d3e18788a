// elastic3d_cpml.cu -- 3D staggered-grid velocity-stress kernels with ADE-CPML
// (moment-tensor and point-force variants).
//
// Restates the Taichi kernels Elastic3D_SSG_Tensor.update_SSG
// (src/Elastic3D_SSG_Tensor.py:166-345) and Elastic3D_SSG_CPML.update_SSG
// (src/Elastic3D_SSG_CPML.py:144-309) as two passes per step:
//   k3_velocity  vx, vy, vz (+ point force)          reference :194-243 / :163-245
//   k3_stress    sxx syy szz, sxy, sxz, syz (+ receivers, + next step's
//                moment-tensor injection)              reference :245-310 / :246-309
// Each CTA owns a 32 (z) x 8 (y) column tile and streams a chunk of x planes;
// the x-direction stencil taps live in per-thread register queues, the y and z
// taps are read through the read-only cache from the current plane.  CPML
// memory variables are stored only on their slabs (sw_pml_axis.lo/hi): outside
// a slab the reference's update is the identity (a = 0, kappa = 1).
#include "sw_device.cuh"

namespace sw {

constexpr int T3Z = 32;
constexpr int T3Y = 8;

template <typename T>
__device__ __forceinline__ void pml_apply(T* __restrict__ m, T b, T a, T kk, T& d) {
  T psi = b * (*m) + a * d;
  *m = psi;
  d = div_v(d, kk) + psi;
}

// ---------------------------------------------------------------------------
// velocity pass
// ---------------------------------------------------------------------------
template <typename T, int N, bool TENSOR>
__global__ void __launch_bounds__(T3Z * T3Y)
k3_velocity(const __grid_constant__ P3<T> p, int it, int force_here) {
  const int k = blockIdx.x * T3Z + threadIdx.x;
  const int j = blockIdx.y * T3Y + threadIdx.y;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  if (j < N || j >= ny - N || k < N || k >= nz - N) return;
  const int ib = max((int)blockIdx.z * p.x_chunk, N);
  const int ie = min((int)(blockIdx.z + 1) * p.x_chunk, nx - N);
  if (ib >= ie) return;

  const long long sx = (long long)ny * nz;
  const long long col = (long long)j * nz + k;
  // ranges (half-open) of Elastic3D_SSG_Tensor.py:195,211,228
  const bool vx_jk = (j >= N + 1) && (k >= N + 1);
  const bool vy_jk = (j < ny - N - 1) && (k >= N + 1);
  const bool vz_jk = (j >= N + 1) && (k < nz - N - 1);

  const int yj = slab_index(j, ny, p.lo[1], p.hi[1]);
  const int zk = slab_index(k, nz, p.lo[2], p.hi[2]);
  const uint8_t fy = p.fl[1][j], fz = p.fl[2][k];
  const T* __restrict__ cfx = p.cf[0];
  const T* __restrict__ cfy = p.cf[1];
  const T* __restrict__ cfz = p.cf[2];
  const T dx = p.dx, dy = p.dy, dz = p.dz, dt = p.dt;

  T* __restrict__ vx = p.f[0];
  T* __restrict__ vy = p.f[1];
  T* __restrict__ vz = p.f[2];
  const T* __restrict__ sxx = p.f[3];
  const T* __restrict__ syy = p.f[4];
  const T* __restrict__ szz = p.f[5];
  const T* __restrict__ sxy = p.f[6];
  const T* __restrict__ sxz = p.f[7];
  const T* __restrict__ syz = p.f[8];
  const T* __restrict__ rho = p.rho;

  T c[N];
#pragma unroll
  for (int m = 0; m < N; ++m) c[m] = p.c[m];

  // register queues along x
  //   qxx[q] = sxx[i-N+1+q]   (Dx3fm)
  //   qxy[q] = sxy[i-N+q]     (Dx3bm)
  //   qxz[q] = sxz[i-N+q]     (Dx3bm)
  T qxx[2 * N], qxy[2 * N], qxz[2 * N];
#pragma unroll
  for (int q = 0; q < 2 * N - 1; ++q) {
    qxx[q] = ldg(sxx + (long long)(ib - N + 1 + q) * sx + col);
    qxy[q] = ldg(sxy + (long long)(ib - N + q) * sx + col);
    qxz[q] = ldg(sxz + (long long)(ib - N + q) * sx + col);
  }
  T rc0 = ldg(rho + (long long)ib * sx + col);          // rho[i, j, k]
  T rn0 = ldg(rho + (long long)ib * sx + col + nz);     // rho[i, j+1, k]

  const bool src_col = force_here && (j == p.sj) && (k == p.sk);

  for (int i = ib; i < ie; ++i) {
    const long long pl = (long long)i * sx;
    qxx[2 * N - 1] = ldg(sxx + pl + (long long)N * sx + col);
    qxy[2 * N - 1] = ldg(sxy + pl + (long long)(N - 1) * sx + col);
    qxz[2 * N - 1] = ldg(sxz + pl + (long long)(N - 1) * sx + col);
    const T rc1 = ldg(rho + pl + sx + col);        // rho[i+1, j, k]
    const T rn1 = ldg(rho + pl + sx + col + nz);   // rho[i+1, j+1, k]
    const int xi = slab_index(i, nx, p.lo[0], p.hi[0]);
    const uint8_t fx = p.fl[0][i];
    const long long idx = pl + col;

    // ---- vx  (x half, y int, z int) -------------------------------------
    if (vx_jk && i < nx - N - 1) {
      T dsxxdx = 0, dsxydy = 0, dsxzdz = 0;
#pragma unroll
      for (int m = 0; m < N; ++m) dsxxdx += c[m] * (qxx[N + m] - qxx[N - 1 - m]);
#pragma unroll
      for (int m = 0; m < N; ++m) {
        const T hi = (m == 0) ? qxy[N] : ldg(sxy + idx + (long long)m * nz);
        dsxydy += c[m] * (hi - ldg(sxy + idx - (long long)(m + 1) * nz));
      }
#pragma unroll
      for (int m = 0; m < N; ++m) {
        const T hi = (m == 0) ? qxz[N] : ldg(sxz + idx + m);
        dsxzdz += c[m] * (hi - ldg(sxz + idx - (m + 1)));
      }
      dsxxdx = div_c(dsxxdx, dx, p.rd[0], p.fast_div);
      dsxydy = div_c(dsxydy, dy, p.rd[1], p.fast_div);
      dsxzdz = div_c(dsxzdz, dz, p.rd[2], p.fast_div);
      if ((xi >= 0 || yj >= 0 || zk >= 0) && ((fx & 2) || (fy & 1) || (fz & 1))) {
        if (xi >= 0)
          pml_apply(p.mem[0] + ((long long)xi * ny + j) * nz + k,
                    cfx[CBH * nx + i], cfx[CAH * nx + i], cfx[CKH * nx + i], dsxxdx);
        if (yj >= 0)
          pml_apply(p.mem[1] + ((long long)i * p.sn[1] + yj) * nz + k,
                    cfy[CB * ny + j], cfy[CA * ny + j], cfy[CK * ny + j], dsxydy);
        if (zk >= 0)
          pml_apply(p.mem[2] + ((long long)i * ny + j) * p.sn[2] + zk,
                    cfz[CB * nz + k], cfz[CA * nz + k], cfz[CK * nz + k], dsxzdz);
      }
      T t = (dsxxdx + dsxzdz + dsxydy) * dt;
      t = div_v(t, rc0);
      vx[idx] = vx[idx] + t;
    }

    // ---- vy  (x int, y half, z int) -------------------------------------
    if (vy_jk && i >= N + 1) {
      const T rhy = (T)0.5 * (rc0 + rn0);
      T dsxydx = 0, dsyydy = 0, dsyzdz = 0;
#pragma unroll
      for (int m = 0; m < N; ++m) dsxydx += c[m] * (qxy[N + m] - qxy[N - 1 - m]);
#pragma unroll
      for (int m = 0; m < N; ++m)
        dsyydy += c[m] * (ldg(syy + idx + (long long)(m + 1) * nz) - ldg(syy + idx - (long long)m * nz));
#pragma unroll
      for (int m = 0; m < N; ++m)
        dsyzdz += c[m] * (ldg(syz + idx + m) - ldg(syz + idx - (m + 1)));
      dsxydx = div_c(dsxydx, dx, p.rd[0], p.fast_div);
      dsyydy = div_c(dsyydy, dy, p.rd[1], p.fast_div);
      dsyzdz = div_c(dsyzdz, dz, p.rd[2], p.fast_div);
      if ((xi >= 0 || yj >= 0 || zk >= 0) && ((fx & 1) || (fy & 2) || (fz & 1))) {
        if (xi >= 0)
          pml_apply(p.mem[0] + p.mcomp[0] + ((long long)xi * ny + j) * nz + k,
                    cfx[CB * nx + i], cfx[CA * nx + i], cfx[CK * nx + i], dsxydx);
        if (yj >= 0)
          pml_apply(p.mem[1] + p.mcomp[1] + ((long long)i * p.sn[1] + yj) * nz + k,
                    cfy[CBH * ny + j], cfy[CAH * ny + j], cfy[CKH * ny + j], dsyydy);
        if (zk >= 0)
          pml_apply(p.mem[2] + p.mcomp[2] + ((long long)i * ny + j) * p.sn[2] + zk,
                    cfz[CB * nz + k], cfz[CA * nz + k], cfz[CK * nz + k], dsyzdz);
      }
      T t = (dsxydx + dsyydy + dsyzdz) * dt;
      t = div_v(t, rhy);
      vy[idx] = vy[idx] + t;
    }

    // ---- vz  (x int, y int, z half) -------------------------------------
    const bool vz_upd = vz_jk && i >= N + 1;
    const bool vz_src = src_col && (i == p.si);
    if (vz_upd || vz_src) {
      T v = vz[idx];
      if (vz_upd) {
        const T r4 = (T)0.25 * (rc0 + rn0 + rn1 + rc1);
        T dsxzdx = 0, dsyzdy = 0, dszzdz = 0;
#pragma unroll
        for (int m = 0; m < N; ++m) dsxzdx += c[m] * (qxz[N + m] - qxz[N - 1 - m]);
#pragma unroll
        for (int m = 0; m < N; ++m)
          dsyzdy += c[m] * (ldg(syz + idx + (long long)m * nz) - ldg(syz + idx - (long long)(m + 1) * nz));
#pragma unroll
        for (int m = 0; m < N; ++m)
          dszzdz += c[m] * (ldg(szz + idx + (m + 1)) - ldg(szz + idx - m));
        dsxzdx = div_c(dsxzdx, dx, p.rd[0], p.fast_div);
        dsyzdy = div_c(dsyzdy, dy, p.rd[1], p.fast_div);
        dszzdz = div_c(dszzdz, dz, p.rd[2], p.fast_div);
        if ((xi >= 0 || yj >= 0 || zk >= 0) && ((fx & 1) || (fy & 1) || (fz & 2))) {
          if (xi >= 0)
            pml_apply(p.mem[0] + 2 * p.mcomp[0] + ((long long)xi * ny + j) * nz + k,
                      cfx[CB * nx + i], cfx[CA * nx + i], cfx[CK * nx + i], dsxzdx);
          if (yj >= 0)
            pml_apply(p.mem[1] + 2 * p.mcomp[1] + ((long long)i * p.sn[1] + yj) * nz + k,
                      cfy[CB * ny + j], cfy[CA * ny + j], cfy[CK * ny + j], dsyzdy);
          if (zk >= 0)
            pml_apply(p.mem[2] + 2 * p.mcomp[2] + ((long long)i * ny + j) * p.sn[2] + zk,
                      cfz[CBH * nz + k], cfz[CAH * nz + k], cfz[CKH * nz + k], dszzdz);
        }
        T s = TENSOR ? (dsxzdx + dsyzdy + dszzdz) : (dszzdz + dsxzdx + dsyzdy);
        T t = s * dt;
        t = div_v(t, r4);
        v = v + t;
      }
      if (vz_src) {
        // Elastic3D_SSG_CPML.py:245 / Elastic3D_SSG_SPML.py:294
        T t = dt * p.wav[it];
        t = div_v(t, rc0);
        v = v + t;
      }
      vz[idx] = v;
    }

    // shift the queues
#pragma unroll
    for (int q = 0; q < 2 * N - 1; ++q) {
      qxx[q] = qxx[q + 1];
      qxy[q] = qxy[q + 1];
      qxz[q] = qxz[q + 1];
    }
    rc0 = rc1;
    rn0 = rn1;
  }
}

// ---------------------------------------------------------------------------
// stress pass
// ---------------------------------------------------------------------------
template <typename T, int N>
__global__ void __launch_bounds__(T3Z * T3Y)
k3_stress(const __grid_constant__ P3<T> p, int it, int inject_next) {
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  // receivers: the velocity fields are final for this step and are not
  // written by this pass (Elastic3D_SSG_Tensor.py:344-345)
  {
    const long long b = blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
    const long long r = b * (T3Z * T3Y) + threadIdx.y * T3Z + threadIdx.x;
    if (r < p.nrec)
      store_rec(p.rec_data, p.rec_f64, (long long)it * p.nrec + r, p.f[p.rec_field][p.rec_idx[r]]);
  }
  const int k = blockIdx.x * T3Z + threadIdx.x;
  const int j = blockIdx.y * T3Y + threadIdx.y;
  if (j < N || j >= ny - N || k < N || k >= nz - N) return;
  const int ib = max((int)blockIdx.z * p.x_chunk, N);
  const int ie = min((int)(blockIdx.z + 1) * p.x_chunk, nx - N);
  if (ib >= ie) return;

  const long long sx = (long long)ny * nz;
  const long long col = (long long)j * nz + k;
  const bool nn_jk = (j >= N + 1) && (k >= N + 1);   // :246
  const bool xy_jk = (j >= N + 1);                   // :268
  const bool xz_jk = (k < nz - N - 1);               // :282
  const bool yz_jk = (j < ny - N - 1) && (k < nz - N - 1);  // :297

  const int yj = slab_index(j, ny, p.lo[1], p.hi[1]);
  const int zk = slab_index(k, nz, p.lo[2], p.hi[2]);
  const uint8_t fy = p.fl[1][j], fz = p.fl[2][k];
  const T* __restrict__ cfx = p.cf[0];
  const T* __restrict__ cfy = p.cf[1];
  const T* __restrict__ cfz = p.cf[2];
  const T dx = p.dx, dy = p.dy, dz = p.dz, dt = p.dt;

  const T* __restrict__ vx = p.f[0];
  const T* __restrict__ vy = p.f[1];
  const T* __restrict__ vz = p.f[2];
  T* __restrict__ sxx = p.f[3];
  T* __restrict__ syy = p.f[4];
  T* __restrict__ szz = p.f[5];
  T* __restrict__ sxy = p.f[6];
  T* __restrict__ sxz = p.f[7];
  T* __restrict__ syz = p.f[8];
  const T* __restrict__ lam = p.lam;
  const T* __restrict__ mu = p.mu;

  T c[N];
#pragma unroll
  for (int m = 0; m < N; ++m) c[m] = p.c[m];

  //   qvx[q] = vx[i-N+q]     (Dx3bm)
  //   qvy[q] = vy[i-N+1+q]   (Dx3fm)
  //   qvz[q] = vz[i-N+1+q]   (Dx3fm)
  T qvx[2 * N], qvy[2 * N], qvz[2 * N];
#pragma unroll
  for (int q = 0; q < 2 * N - 1; ++q) {
    qvx[q] = ldg(vx + (long long)(ib - N + q) * sx + col);
    qvy[q] = ldg(vy + (long long)(ib - N + 1 + q) * sx + col);
    qvz[q] = ldg(vz + (long long)(ib - N + 1 + q) * sx + col);
  }
  T l0 = ldg(lam + (long long)ib * sx + col);
  T u0 = ldg(mu + (long long)ib * sx + col);
  const bool src_col = inject_next && (j == p.sj) && (k == p.sk);
  const T wn = inject_next ? p.wav[it + 1] : (T)0;

  for (int i = ib; i < ie; ++i) {
    const long long pl = (long long)i * sx;
    qvx[2 * N - 1] = ldg(vx + pl + (long long)(N - 1) * sx + col);
    qvy[2 * N - 1] = ldg(vy + pl + (long long)N * sx + col);
    qvz[2 * N - 1] = ldg(vz + pl + (long long)N * sx + col);
    const T l1 = ldg(lam + pl + sx + col);   // lam[i+1, j, k]
    const T u1 = ldg(mu + pl + sx + col);    // mu[i+1, j, k]
    const int xi = slab_index(i, nx, p.lo[0], p.hi[0]);
    const uint8_t fx = p.fl[0][i];
    const long long idx = pl + col;
    const bool src = src_col && (i == p.si);
    const bool any_slab = (xi >= 0 || yj >= 0 || zk >= 0);

    // ---- sxx syy szz  (integer point) :246-266 ---------------------------
    if ((nn_jk && i >= N + 1) || src) {
      T axx = sxx[idx], ayy = syy[idx], azz = szz[idx];
      if (nn_jk && i >= N + 1) {
        const T lhx = (T)0.5 * (l0 + l1);
        const T mhx = (T)0.5 * (u0 + u1);
        const T lpm = lhx + (T)2 * mhx;
        T dvxdx = 0, dvydy = 0, dvzdz = 0;
#pragma unroll
        for (int m = 0; m < N; ++m) dvxdx += c[m] * (qvx[N + m] - qvx[N - 1 - m]);
#pragma unroll
        for (int m = 0; m < N; ++m) {
          const T hi = (m == 0) ? qvy[N - 1] : ldg(vy + idx + (long long)m * nz);
          dvydy += c[m] * (hi - ldg(vy + idx - (long long)(m + 1) * nz));
        }
#pragma unroll
        for (int m = 0; m < N; ++m) {
          const T hi = (m == 0) ? qvz[N - 1] : ldg(vz + idx + m);
          dvzdz += c[m] * (hi - ldg(vz + idx - (m + 1)));
        }
        dvxdx = div_c(dvxdx, dx, p.rd[0], p.fast_div);
        dvydy = div_c(dvydy, dy, p.rd[1], p.fast_div);
        dvzdz = div_c(dvzdz, dz, p.rd[2], p.fast_div);
        if (any_slab && ((fx | fy | fz) & 1)) {
          if (xi >= 0)
            pml_apply(p.mem[0] + 3 * p.mcomp[0] + ((long long)xi * ny + j) * nz + k,
                      cfx[CB * nx + i], cfx[CA * nx + i], cfx[CK * nx + i], dvxdx);
          if (yj >= 0)
            pml_apply(p.mem[1] + 3 * p.mcomp[1] + ((long long)i * p.sn[1] + yj) * nz + k,
                      cfy[CB * ny + j], cfy[CA * ny + j], cfy[CK * ny + j], dvydy);
          if (zk >= 0)
            pml_apply(p.mem[2] + 3 * p.mcomp[2] + ((long long)i * ny + j) * p.sn[2] + zk,
                      cfz[CB * nz + k], cfz[CA * nz + k], cfz[CK * nz + k], dvzdz);
        }
        axx = axx + (lpm * dvxdx + lhx * (dvzdz + dvydy)) * dt;
        ayy = ayy + (lpm * dvydy + lhx * (dvxdx + dvzdz)) * dt;
        azz = azz + (lpm * dvzdz + lhx * (dvxdx + dvydy)) * dt;
      }
      if (src) {
        axx = axx + wn * p.mneg[0];
        ayy = ayy + wn * p.mneg[1];
        azz = azz + wn * p.mneg[2];
      }
      sxx[idx] = axx;
      syy[idx] = ayy;
      szz[idx] = azz;
    }

    // ---- sxy  (x half, y half, z int) :268-280 ---------------------------
    const bool xy_upd = xy_jk && i >= N + 1;
    if (xy_upd || src) {
      T a = sxy[idx];
      if (xy_upd) {
        const T unj = ldg(mu + idx + nz);  // mu[i, j+1, k]
        const T m4 = (T)0.25 * (unj + u0 + u0 + u1);
        T dvydx = 0, dvxdy = 0;
#pragma unroll
        for (int m = 0; m < N; ++m) dvydx += c[m] * (qvy[N + m] - qvy[N - 1 - m]);
#pragma unroll
        for (int m = 0; m < N; ++m) {
          const T lo = (m == 0) ? qvx[N] : ldg(vx + idx - (long long)m * nz);
          dvxdy += c[m] * (ldg(vx + idx + (long long)(m + 1) * nz) - lo);
        }
        dvydx = div_c(dvydx, dx, p.rd[0], p.fast_div);
        dvxdy = div_c(dvxdy, dy, p.rd[1], p.fast_div);
        if (any_slab && ((fx & 2) || (fy & 2) || (fz & 1))) {
          if (xi >= 0)
            pml_apply(p.mem[0] + 4 * p.mcomp[0] + ((long long)xi * ny + j) * nz + k,
                      cfx[CBH * nx + i], cfx[CAH * nx + i], cfx[CKH * nx + i], dvydx);
          if (yj >= 0)
            pml_apply(p.mem[1] + 4 * p.mcomp[1] + ((long long)i * p.sn[1] + yj) * nz + k,
                      cfy[CBH * ny + j], cfy[CAH * ny + j], cfy[CKH * ny + j], dvxdy);
        }
        a = a + m4 * (dvxdy + dvydx) * dt;
      }
      if (src) a = a + wn * p.mneg[3];
      sxy[idx] = a;
    }

    // ---- sxz  (x half, y int, z half) :282-294 ---------------------------
    const bool xz_upd = xz_jk && i < nx - N - 1;
    if (xz_upd || src) {
      T a = sxz[idx];
      if (xz_upd) {
        const T unj = ldg(mu + idx + nz);  // mu[i, j+1, k]
        const T m4 = (T)0.25 * (u0 + u1 + u0 + unj);
        T dvzdx = 0, dvxdz = 0;
#pragma unroll
        for (int m = 0; m < N; ++m) dvzdx += c[m] * (qvz[N + m] - qvz[N - 1 - m]);
#pragma unroll
        for (int m = 0; m < N; ++m) {
          const T lo = (m == 0) ? qvx[N] : ldg(vx + idx - m);
          dvxdz += c[m] * (ldg(vx + idx + (m + 1)) - lo);
        }
        dvzdx = div_c(dvzdx, dx, p.rd[0], p.fast_div);
        dvxdz = div_c(dvxdz, dz, p.rd[2], p.fast_div);
        if (any_slab && ((fx & 2) || (fy & 1) || (fz & 2))) {
          if (xi >= 0)
            pml_apply(p.mem[0] + 5 * p.mcomp[0] + ((long long)xi * ny + j) * nz + k,
                      cfx[CBH * nx + i], cfx[CAH * nx + i], cfx[CKH * nx + i], dvzdx);
          if (zk >= 0)
            pml_apply(p.mem[2] + 4 * p.mcomp[2] + ((long long)i * ny + j) * p.sn[2] + zk,
                      cfz[CBH * nz + k], cfz[CAH * nz + k], cfz[CKH * nz + k], dvxdz);
        }
        a = a + m4 * (dvxdz + dvzdx) * dt;
      }
      if (src) a = a + wn * p.mneg[4];
      sxz[idx] = a;
    }

    // ---- syz  (x int, y half, z half) :297-310 ---------------------------
    if (yz_jk || src) {
      T a = syz[idx];
      if (yz_jk) {
        const T unj = ldg(mu + idx + nz);  // mu[i, j+1, k]
        const T unk = ldg(mu + idx + 1);   // mu[i, j, k+1]
        const T m4 = (T)0.25 * (unj + u0 + unk + u0);
        T dvzdy = 0, dvydz = 0;
#pragma unroll
        for (int m = 0; m < N; ++m) {
          const T lo = (m == 0) ? qvz[N - 1] : ldg(vz + idx - (long long)m * nz);
          dvzdy += c[m] * (ldg(vz + idx + (long long)(m + 1) * nz) - lo);
        }
#pragma unroll
        for (int m = 0; m < N; ++m) {
          const T lo = (m == 0) ? qvy[N - 1] : ldg(vy + idx - m);
          dvydz += c[m] * (ldg(vy + idx + (m + 1)) - lo);
        }
        dvzdy = div_c(dvzdy, dy, p.rd[1], p.fast_div);
        dvydz = div_c(dvydz, dz, p.rd[2], p.fast_div);
        if (any_slab && ((fx & 1) || (fy & 2) || (fz & 2))) {
          if (yj >= 0)
            pml_apply(p.mem[1] + 5 * p.mcomp[1] + ((long long)i * p.sn[1] + yj) * nz + k,
                      cfy[CBH * ny + j], cfy[CAH * ny + j], cfy[CKH * ny + j], dvzdy);
          if (zk >= 0)
            pml_apply(p.mem[2] + 5 * p.mcomp[2] + ((long long)i * ny + j) * p.sn[2] + zk,
                      cfz[CBH * nz + k], cfz[CAH * nz + k], cfz[CKH * nz + k], dvydz);
        }
        a = a + m4 * (dvzdy + dvydz) * dt;
      }
      if (src) a = a + wn * p.mneg[5];
      syz[idx] = a;
    }

#pragma unroll
    for (int q = 0; q < 2 * N - 1; ++q) {
      qvx[q] = qvx[q + 1];
      qvy[q] = qvy[q + 1];
      qvz[q] = qvz[q + 1];
    }
    l0 = l1;
    u0 = u1;
  }
}

// ---------------------------------------------------------------------------
// single-cell source kernels (used when the fused paths cannot cover a step)
// ---------------------------------------------------------------------------
// Elastic3D_SSG_Tensor.py:186-193: sigma_ab[src] += w * (-M_ab)
template <typename T>
__global__ void k3_moment_inject(const __grid_constant__ P3<T> p, int it) {
  const long long s = ((long long)p.si * p.ny + p.sj) * p.nz + p.sk;
  const T w = p.wav[it];
#pragma unroll
  for (int a = 0; a < 6; ++a) p.f[3 + a][s] = p.f[3 + a][s] + w * p.mneg[a];
}

// vz[src] += dt*w/rho[src] for a source cell outside the velocity pass
template <typename T>
__global__ void k3_force_inject(const __grid_constant__ P3<T> p, int it) {
  const long long s = ((long long)p.si * p.ny + p.sj) * p.nz + p.sk;
  T t = p.dt * p.wav[it];
  t = div_v(t, p.rho[s]);
  p.f[2][s] = p.f[2][s] + t;
}

// receivers of a field written by the stress pass
template <typename T>
__global__ void k3_gather(const __grid_constant__ P3<T> p, int it) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < p.nrec) store_rec(p.rec_data, p.rec_f64, (long long)it * p.nrec + r, p.f[p.rec_field][p.rec_idx[r]]);
}

// ---------------------------------------------------------------------------
// host-side launchers
// ---------------------------------------------------------------------------
template <typename T>
static dim3 grid3(const P3<T>& p) {
  return dim3((p.nz + T3Z - 1) / T3Z, (p.ny + T3Y - 1) / T3Y, (p.nx + p.x_chunk - 1) / p.x_chunk);
}

template <typename T, int N>
static void launch3_velocity(const P3<T>& p, int it, bool tensor, bool force_here, cudaStream_t st) {
  if (tensor) k3_velocity<T, N, true><<<grid3(p), dim3(T3Z, T3Y), 0, st>>>(p, it, 0);
  else k3_velocity<T, N, false><<<grid3(p), dim3(T3Z, T3Y), 0, st>>>(p, it, force_here ? 1 : 0);
}

template <typename T, int N>
static void launch3_stress(const P3<T>& p, int it, bool inject_next, cudaStream_t st) {
  k3_stress<T, N><<<grid3(p), dim3(T3Z, T3Y), 0, st>>>(p, it, inject_next ? 1 : 0);
}

#define SW_ORDER_SWITCH(order, CALL)            \
  switch (order) {                              \
    case 1: { constexpr int NN = 1; CALL; break; } \
    case 2: { constexpr int NN = 2; CALL; break; } \
    case 3: { constexpr int NN = 3; CALL; break; } \
    case 4: { constexpr int NN = 4; CALL; break; } \
    case 5: { constexpr int NN = 5; CALL; break; } \
    case 6: { constexpr int NN = 6; CALL; break; } \
    case 7: { constexpr int NN = 7; CALL; break; } \
    case 8: { constexpr int NN = 8; CALL; break; } \
    default: return cudaErrorInvalidValue;      \
  }

// velocity pass of one step (force_here: the point force is added in-kernel)
template <typename T>
cudaError_t sw3_velocity(const P3<T>& p, int order, int it, bool tensor, bool force_here, cudaStream_t st) {
  SW_ORDER_SWITCH(order, (launch3_velocity<T, NN>(p, it, tensor, force_here, st)));
  return cudaGetLastError();
}

// stress pass of one step; p.nrec > 0 gathers receivers of a velocity field,
// inject_next adds the moment-tensor source of step it+1 at the end.
template <typename T>
cudaError_t sw3_stress(const P3<T>& p, int order, int it, bool inject_next, cudaStream_t st) {
  SW_ORDER_SWITCH(order, (launch3_stress<T, NN>(p, it, inject_next, st)));
  return cudaGetLastError();
}

template <typename T>
cudaError_t sw3_moment_inject(const P3<T>& p, int it, cudaStream_t st) {
  k3_moment_inject<T><<<1, 1, 0, st>>>(p, it);
  return cudaGetLastError();
}
template <typename T>
cudaError_t sw3_force_inject(const P3<T>& p, int it, cudaStream_t st) {
  k3_force_inject<T><<<1, 1, 0, st>>>(p, it);
  return cudaGetLastError();
}
// free-surface hook (Elastic3D_SSG_Tensor.py:160-163): szz = 0 on the z layer kz
template <typename T>
__global__ void k3_aea(T* szz, long long nxy, int nz, int kz) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c < nxy) szz[c * nz + kz] = (T)0;
}
template <typename T>
cudaError_t sw3_aea(const P3<T>& p, int kz, cudaStream_t st) {
  const long long nxy = (long long)p.nx * p.ny;
  k3_aea<T><<<(unsigned)((nxy + 255) / 256), 256, 0, st>>>(p.f[5], nxy, p.nz, kz);
  return cudaGetLastError();
}
template <typename T>
cudaError_t sw3_gather(const P3<T>& p, int it, cudaStream_t st) {
  if (p.nrec <= 0) return cudaSuccess;
  k3_gather<T><<<(p.nrec + 255) / 256, 256, 0, st>>>(p, it);
  return cudaGetLastError();
}

template cudaError_t sw3_velocity<float>(const P3<float>&, int, int, bool, bool, cudaStream_t);
template cudaError_t sw3_velocity<double>(const P3<double>&, int, int, bool, bool, cudaStream_t);
template cudaError_t sw3_stress<float>(const P3<float>&, int, int, bool, cudaStream_t);
template cudaError_t sw3_stress<double>(const P3<double>&, int, int, bool, cudaStream_t);
template cudaError_t sw3_moment_inject<float>(const P3<float>&, int, cudaStream_t);
template cudaError_t sw3_moment_inject<double>(const P3<double>&, int, cudaStream_t);
template cudaError_t sw3_force_inject<float>(const P3<float>&, int, cudaStream_t);
template cudaError_t sw3_force_inject<double>(const P3<double>&, int, cudaStream_t);
template cudaError_t sw3_aea<float>(const P3<float>&, int, cudaStream_t);
template cudaError_t sw3_aea<double>(const P3<double>&, int, cudaStream_t);
template cudaError_t sw3_gather<float>(const P3<float>&, int, cudaStream_t);
template cudaError_t sw3_gather<double>(const P3<double>&, int, cudaStream_t);

}  // namespace sw
