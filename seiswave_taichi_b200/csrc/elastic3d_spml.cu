// elastic3d_spml.cu -- 3D staggered-grid kernels with the split-field PML of
// src/Elastic3D_SSG_SPML.py:160-393 (update_SSG_SPML).
//
// Inside the PML predicate each component is advanced as split parts
//   psi_d <- ((1 - dt/2 d) psi_d + dt * term_d) / (1 + dt/2 d)
// and the field is set to their sum; outside it the plain update is used.
// The 24 split fields live only on the PML shell (split[24][scomp], cells
// ordered by shell_index); a cell whose axis predicates are all clear never
// touches them.  One thread per cell, block 32 (z) x 8 (y), one x plane per
// blockIdx.z.
#include "sw_device.cuh"

namespace sw {

constexpr int TSZ = 32;
constexpr int TSY = 8;

template <typename T, int N>
__device__ __forceinline__ T d_fm(const T* f, long long idx, long long s, const T* c) {
  T v = 0;
#pragma unroll
  for (int m = 0; m < N; ++m) v += c[m] * (ldg(f + idx + (m + 1) * s) - ldg(f + idx - m * s));
  return v;
}
template <typename T, int N>
__device__ __forceinline__ T d_bm(const T* f, long long idx, long long s, const T* c) {
  T v = 0;
#pragma unroll
  for (int m = 0; m < N; ++m) v += c[m] * (ldg(f + idx + m * s) - ldg(f + idx - (m + 1) * s));
  return v;
}

template <typename T, int N>
__global__ void __launch_bounds__(TSZ * TSY)
ks_velocity(const __grid_constant__ P3<T> p, int it, int src_here) {
  const int k = blockIdx.x * TSZ + threadIdx.x;
  const int j = blockIdx.y * TSY + threadIdx.y;
  const int i = blockIdx.z;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  if (j >= ny || k >= nz) return;
  const long long sx = (long long)ny * nz, sy = nz;
  const long long idx = (long long)i * sx + (long long)j * nz + k;
  const long long G = p.scomp;
  const T dx = p.dx, dy = p.dy, dz = p.dz, dt = p.dt;
  const T hdt = (T)0.5 * dt;
  T c[N];
#pragma unroll
  for (int m = 0; m < N; ++m) c[m] = p.c[m];
  const T *sxx = p.f[3], *syy = p.f[4], *szz = p.f[5], *sxy = p.f[6], *sxz = p.f[7], *syz = p.f[8];
  T *vx = p.f[0], *vy = p.f[1], *vz = p.f[2];
  T* sp = p.split;
  const T *rho = p.rho, *dpx = p.dmp[0], *dpy = p.dmp[1], *dpz = p.dmp[2];
  const uint8_t fx = p.fl[0][i], fy = p.fl[1][j], fz = p.fl[2][k];
  // every flagged index lies in its axis's slabs (checked when the plan is made)
  const long long sh = (fx | fy | fz) ? shell_index(p, i, j, k) : 0;

  // vx :182-205
  if (i >= N && i < nx - N - 1 && j >= N + 1 && j < ny - N && k >= N + 1 && k < nz - N) {
    T dsxxdx = div_c(d_fm<T, N>(sxx, idx, sx, c), dx, p.rd[0], p.fast_div);
    T dsxydy = div_c(d_bm<T, N>(sxy, idx, sy, c), dy, p.rd[1], p.fast_div);
    T dsxzdz = div_c(d_bm<T, N>(sxz, idx, 1, c), dz, p.rd[2], p.fast_div);
    const T rh = ldg(rho + idx);
    const T ro = (T)1 / rh;
    if ((fx & 2) || (fy & 1) || (fz & 1)) {
      const T xn = (T)1 - hdt * dpx[nx + i], yn = (T)1 - hdt * dpy[j], zn = (T)1 - hdt * dpz[k];
      const T xd = (T)1 + hdt * dpx[nx + i], yd = (T)1 + hdt * dpy[j], zd = (T)1 + hdt * dpz[k];
      T a = div_v((xn * sp[PVX_X * G + sh] + dsxxdx * dt * ro), xd);
      T b = div_v((yn * sp[PVX_Y * G + sh] + dsxydy * dt * ro), yd);
      T cc = div_v((zn * sp[PVX_Z * G + sh] + dsxzdz * dt * ro), zd);
      sp[PVX_X * G + sh] = a;
      sp[PVX_Y * G + sh] = b;
      sp[PVX_Z * G + sh] = cc;
      vx[idx] = a + b + cc;
    } else {
      vx[idx] = vx[idx] + (dsxxdx + dsxydy + dsxzdz) * dt * ro;
    }
  }
  // vy :209-233
  if (i >= N + 1 && i < nx - N && j >= N && j < ny - N - 1 && k >= N + 1 && k < nz - N) {
    const T rhy = (T)0.5 * (ldg(rho + idx) + ldg(rho + idx + sy));
    const T ro = (T)1 / rhy;
    T dsxydx = div_c(d_bm<T, N>(sxy, idx, sx, c), dx, p.rd[0], p.fast_div);
    T dsyydy = div_c(d_fm<T, N>(syy, idx, sy, c), dy, p.rd[1], p.fast_div);
    T dsyzdz = div_c(d_bm<T, N>(syz, idx, 1, c), dz, p.rd[2], p.fast_div);
    if ((fx & 1) || (fy & 2) || (fz & 1)) {
      const T xn = (T)1 - hdt * dpx[i], yn = (T)1 - hdt * dpy[ny + j], zn = (T)1 - hdt * dpz[k];
      const T xd = (T)1 + hdt * dpx[i], yd = (T)1 + hdt * dpy[ny + j], zd = (T)1 + hdt * dpz[k];
      T a = div_v((xn * sp[PVY_X * G + sh] + dt * dsxydx * ro), xd);
      T b = div_v((yn * sp[PVY_Y * G + sh] + dt * dsyydy * ro), yd);
      T cc = div_v((zn * sp[PVY_Z * G + sh] + dt * dsyzdz * ro), zd);
      sp[PVY_X * G + sh] = a;
      sp[PVY_Y * G + sh] = b;
      sp[PVY_Z * G + sh] = cc;
      vy[idx] = a + b + cc;
    } else {
      vy[idx] = vy[idx] + (dsxydx + dsyydy + dsyzdz) * dt * ro;
    }
  }
  // vz :235-259, then the source :294
  const bool upd = i >= N + 1 && i < nx - N && j >= N + 1 && j < ny - N && k >= N && k < nz - N - 1;
  const bool src = src_here && i == p.si && j == p.sj && k == p.sk;
  if (upd || src) {
    T v = vz[idx];
    if (upd) {
      const T r4 = (T)0.25 * (ldg(rho + idx) + ldg(rho + idx + sy) + ldg(rho + idx + sx + sy) + ldg(rho + idx + sx));
      const T ro = (T)1 / r4;
      T dsxzdx = div_c(d_bm<T, N>(sxz, idx, sx, c), dx, p.rd[0], p.fast_div);
      T dsyzdy = div_c(d_bm<T, N>(syz, idx, sy, c), dy, p.rd[1], p.fast_div);
      T dszzdz = div_c(d_fm<T, N>(szz, idx, 1, c), dz, p.rd[2], p.fast_div);
      if ((fx & 1) || (fy & 1) || (fz & 2)) {
        const T xn = (T)1 - hdt * dpx[i], yn = (T)1 - hdt * dpy[j], zn = (T)1 - hdt * dpz[nz + k];
        const T xd = (T)1 + hdt * dpx[i], yd = (T)1 + hdt * dpy[j], zd = (T)1 + hdt * dpz[nz + k];
        T a = div_v((xn * sp[PVZ_X * G + sh] + dt * dsxzdx * ro), xd);
        T b = div_v((yn * sp[PVZ_Y * G + sh] + dt * dsyzdy * ro), yd);
        T cc = div_v((zn * sp[PVZ_Z * G + sh] + dt * dszzdz * ro), zd);
        sp[PVZ_X * G + sh] = a;
        sp[PVZ_Y * G + sh] = b;
        sp[PVZ_Z * G + sh] = cc;
        v = a + b + cc;
      } else {
        v = v + (dsxzdx + dsyzdy + dszzdz) * dt * ro;
      }
    }
    if (src) {
      T t = dt * p.wav[it];
      t = div_v(t, ldg(rho + idx));
      v = v + t;
    }
    vz[idx] = v;
  }
}

template <typename T, int N>
__global__ void __launch_bounds__(TSZ * TSY)
ks_stress(const __grid_constant__ P3<T> p, int it) {
  {
    const long long b = blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
    const long long r = b * (TSZ * TSY) + threadIdx.y * TSZ + threadIdx.x;
    if (r < p.nrec) store_rec(p.rec_data, p.rec_f64, (long long)it * p.nrec + r, p.f[p.rec_field][p.rec_idx[r]]);
  }
  const int k = blockIdx.x * TSZ + threadIdx.x;
  const int j = blockIdx.y * TSY + threadIdx.y;
  const int i = blockIdx.z;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  if (j >= ny || k >= nz) return;
  const long long sx = (long long)ny * nz, sy = nz;
  const long long idx = (long long)i * sx + (long long)j * nz + k;
  const long long G = p.scomp;
  const T dx = p.dx, dy = p.dy, dz = p.dz, dt = p.dt;
  const T hdt = (T)0.5 * dt;
  T c[N];
#pragma unroll
  for (int m = 0; m < N; ++m) c[m] = p.c[m];
  const T *vx = p.f[0], *vy = p.f[1], *vz = p.f[2];
  T *sxx = p.f[3], *syy = p.f[4], *szz = p.f[5], *sxy = p.f[6], *sxz = p.f[7], *syz = p.f[8];
  T* sp = p.split;
  const T *lam = p.lam, *mu = p.mu, *dpx = p.dmp[0], *dpy = p.dmp[1], *dpz = p.dmp[2];
  const uint8_t fx = p.fl[0][i], fy = p.fl[1][j], fz = p.fl[2][k];
  // every flagged index lies in its axis's slabs (checked when the plan is made)
  const long long sh = (fx | fy | fz) ? shell_index(p, i, j, k) : 0;

  // normal stresses :296-333
  if (i >= N + 1 && i < nx - N && j >= N + 1 && j < ny - N && k >= N + 1 && k < nz - N) {
    const T lm = ldg(lam + idx), u = ldg(mu + idx);
    const T l2m = lm + (T)2 * u;
    T dvxdx = div_c(d_bm<T, N>(vx, idx, sx, c), dx, p.rd[0], p.fast_div);
    T dvydy = div_c(d_bm<T, N>(vy, idx, sy, c), dy, p.rd[1], p.fast_div);
    T dvzdz = div_c(d_bm<T, N>(vz, idx, 1, c), dz, p.rd[2], p.fast_div);
    if ((fx | fy | fz) & 1) {
      const T xn = (T)1 - hdt * dpx[i], yn = (T)1 - hdt * dpy[j], zn = (T)1 - hdt * dpz[k];
      const T xd = (T)1 + hdt * dpx[i], yd = (T)1 + hdt * dpy[j], zd = (T)1 + hdt * dpz[k];
      T xx = div_v((xn * sp[PSXX_X * G + sh] + dt * l2m * dvxdx), xd);
      T xy = div_v((yn * sp[PSXX_Y * G + sh] + dt * lm * dvydy), yd);
      T xz = div_v((zn * sp[PSXX_Z * G + sh] + dt * lm * dvzdz), zd);
      T yx = div_v((xn * sp[PSYY_X * G + sh] + dt * lm * dvxdx), xd);
      T yy = div_v((yn * sp[PSYY_Y * G + sh] + dt * l2m * dvydy), yd);
      T yz = div_v((zn * sp[PSYY_Z * G + sh] + dt * lm * dvzdz), zd);
      T zx = div_v((xn * sp[PSZZ_X * G + sh] + dt * lm * dvxdx), xd);
      T zy = div_v((yn * sp[PSZZ_Y * G + sh] + dt * lm * dvydy), yd);
      T zz = div_v((zn * sp[PSZZ_Z * G + sh] + dt * l2m * dvzdz), zd);
      sp[PSXX_X * G + sh] = xx; sp[PSXX_Y * G + sh] = xy; sp[PSXX_Z * G + sh] = xz;
      sp[PSYY_X * G + sh] = yx; sp[PSYY_Y * G + sh] = yy; sp[PSYY_Z * G + sh] = yz;
      sp[PSZZ_X * G + sh] = zx; sp[PSZZ_Y * G + sh] = zy; sp[PSZZ_Z * G + sh] = zz;
      sxx[idx] = xx + xy + xz;
      syy[idx] = yx + yy + yz;
      szz[idx] = zx + zy + zz;
    } else {
      sxx[idx] = sxx[idx] + (l2m * dvxdx + lm * (dvzdz + dvydy)) * dt;
      syy[idx] = syy[idx] + (l2m * dvydy + lm * (dvxdx + dvzdz)) * dt;
      szz[idx] = szz[idx] + (l2m * dvzdz + lm * (dvxdx + dvydy)) * dt;
    }
  }
  // sxy :334-350
  if (i >= N + 1 && i < nx - N && j >= N + 1 && j < ny - N && k >= N && k < nz - N) {
    const T m4 = (T)0.25 * (ldg(mu + idx + sy) + ldg(mu + idx) + ldg(mu + idx) + ldg(mu + idx + sx));
    T dvydx = div_c(d_fm<T, N>(vy, idx, sx, c), dx, p.rd[0], p.fast_div);
    T dvxdy = div_c(d_fm<T, N>(vx, idx, sy, c), dy, p.rd[1], p.fast_div);
    if ((fx & 2) || (fy & 2) || (fz & 1)) {
      const T xn = (T)1 - hdt * dpx[nx + i], yn = (T)1 - hdt * dpy[ny + j];
      const T xd = (T)1 + hdt * dpx[nx + i], yd = (T)1 + hdt * dpy[ny + j];
      T a = div_v((xn * sp[PSXY_X * G + sh] + dt * m4 * dvydx), xd);
      T b = div_v((yn * sp[PSXY_Y * G + sh] + dt * m4 * dvxdy), yd);
      sp[PSXY_X * G + sh] = a;
      sp[PSXY_Y * G + sh] = b;
      sxy[idx] = a + b;
    } else {
      sxy[idx] = sxy[idx] + m4 * (dvxdy + dvydx) * dt;
    }
  }
  // sxz :352-371
  if (i >= N && i < nx - N - 1 && j >= N && j < ny - N && k >= N && k < nz - N - 1) {
    const T m4 = (T)0.25 * (ldg(mu + idx) + ldg(mu + idx + sx) + ldg(mu + idx) + ldg(mu + idx + sy));
    T dvzdx = div_c(d_fm<T, N>(vz, idx, sx, c), dx, p.rd[0], p.fast_div);
    T dvxdz = div_c(d_fm<T, N>(vx, idx, 1, c), dz, p.rd[2], p.fast_div);
    if ((fx & 2) || (fy & 1) || (fz & 2)) {
      const T xn = (T)1 - hdt * dpx[nx + i], zn = (T)1 - hdt * dpz[nz + k];
      const T xd = (T)1 + hdt * dpx[nx + i], zd = (T)1 + hdt * dpz[nz + k];
      T a = div_v((xn * sp[PSXZ_X * G + sh] + dt * m4 * dvzdx), xd);
      T b = div_v((zn * sp[PSXZ_Z * G + sh] + dt * m4 * dvxdz), zd);
      sp[PSXZ_X * G + sh] = a;
      sp[PSXZ_Z * G + sh] = b;
      sxz[idx] = a + b;
    } else {
      sxz[idx] = sxz[idx] + m4 * (dvxdz + dvzdx) * dt;
    }
  }
  // syz :373-391
  if (i >= N && i < nx - N && j >= N && j < ny - N - 1 && k >= N && k < nz - N - 1) {
    const T m4 = (T)0.25 * (ldg(mu + idx + sy) + ldg(mu + idx) + ldg(mu + idx + 1) + ldg(mu + idx));
    T dvzdy = div_c(d_fm<T, N>(vz, idx, sy, c), dy, p.rd[1], p.fast_div);
    T dvydz = div_c(d_fm<T, N>(vy, idx, 1, c), dz, p.rd[2], p.fast_div);
    if ((fx & 1) || (fy & 2) || (fz & 2)) {
      const T yn = (T)1 - hdt * dpy[ny + j], zn = (T)1 - hdt * dpz[nz + k];
      const T yd = (T)1 + hdt * dpy[ny + j], zd = (T)1 + hdt * dpz[nz + k];
      T a = div_v((yn * sp[PSYZ_Y * G + sh] + dt * m4 * dvzdy), yd);
      T b = div_v((zn * sp[PSYZ_Z * G + sh] + dt * m4 * dvydz), zd);
      sp[PSYZ_Y * G + sh] = a;
      sp[PSYZ_Z * G + sh] = b;
      syz[idx] = a + b;
    } else {
      syz[idx] = syz[idx] + m4 * (dvydz + dvzdy) * dt;
    }
  }
}

template <typename T, int N>
static cudaError_t launch_spml(const P3<T>& p, int it, bool gather_in_stress, cudaStream_t st) {
  dim3 block(TSZ, TSY);
  dim3 grid((p.nz + TSZ - 1) / TSZ, (p.ny + TSY - 1) / TSY, p.nx);
  ks_velocity<T, N><<<grid, block, 0, st>>>(p, it, p.src_kind != SW_SRC_NONE ? 1 : 0);
  P3<T> q = p;
  if (!gather_in_stress) q.nrec = 0;
  ks_stress<T, N><<<grid, block, 0, st>>>(q, it);
  return cudaGetLastError();
}

template <typename T>
cudaError_t sw3_spml_step(const P3<T>& p, int order, int it, bool gather_in_stress, cudaStream_t st) {
  switch (order) {
    case 1: return launch_spml<T, 1>(p, it, gather_in_stress, st);
    case 2: return launch_spml<T, 2>(p, it, gather_in_stress, st);
    case 3: return launch_spml<T, 3>(p, it, gather_in_stress, st);
    case 4: return launch_spml<T, 4>(p, it, gather_in_stress, st);
    case 5: return launch_spml<T, 5>(p, it, gather_in_stress, st);
    case 6: return launch_spml<T, 6>(p, it, gather_in_stress, st);
    case 7: return launch_spml<T, 7>(p, it, gather_in_stress, st);
    case 8: return launch_spml<T, 8>(p, it, gather_in_stress, st);
    default: return cudaErrorInvalidValue;
  }
}

template cudaError_t sw3_spml_step<float>(const P3<float>&, int, int, bool, cudaStream_t);
template cudaError_t sw3_spml_step<double>(const P3<double>&, int, int, bool, cudaStream_t);

}  // namespace sw
