// elastic3d_adjoint.cu -- hand-written discrete adjoint of the 3D SSG-CPML
// moment-tensor step (src/Elastic3D_SSG_Tensor.py:166-345) and point-force
// step (src/Elastic3D_SSG_CPML.py:144-309, the same stencils) for gradients of
// a seismogram misfit with respect to rho, lambda and mu.  No reference
// counterpart.
//
// Forward step it (the oracle's velocity3d / stress3d order):
//   inject   sigma_ab[src] += w(it) * (-M_ab)
//   V   vx += dt/rho      (Dx+ sxx' + Dz- sxz' + Dy- sxy')     vx cells
//       vy += dt/rho_y    (Dx- sxy' + Dy+ syy' + Dz- syz')     vy cells
//       vz += dt/rho_4    (Dx- sxz' + Dy- syz' + Dz+ szz')     vz cells
//   S   sxx += dt*(lpm e0 + lhx (e2 + e1)), syy, szz likewise, e = D- v   normal cells
//       sxy += m_xy (Dy+ vx' + Dx+ vy') dt, sxz += m_xz (Dz+ vx' + Dx+ vz') dt,
//       syz += m_yz (Dy+ vz' + Dz+ vy') dt
//   record data[it] = field[rec]
// with D+ f = sum c_m (f[+m+1] - f[-m]), D- f = sum c_m (f[+m] - f[-m-1]) along
// one axis, divided by the spacing, and d' = d/kappa + psi_new on the CPML
// cells.  The adjoint of step it runs the phases in reverse: receivers, the
// stress phase's mids (CPML recursion reversed) and lambda/mu gradients, the
// gather of the transposed stencils into the velocity adjoints, then the same
// for the velocity phase.  Forward values come from sw3d_record snapshots:
// slot k is the state of step it after its source injection, slot k+1 holds
// the velocities after the velocity phase of step it.
#include "sw_device.cuh"

namespace sw {

template <typename T>
struct A3 {
  T* f[9];          // adjoint of vx vy vz sxx syy szz sxy sxz syz
  T* mem[3];        // adjoint memory variables, slab layout of P3::mem
  T* tmp[9];        // mid fields (nx, ny, nz)
  T* grad[8];       // per-cell sums: G_vx G_vy G_vz (densities), G_lpm G_lhx (normal), G_xy G_xz G_yz (shear)
  const T* res;     // receiver residual (nt, nrec)
  const T* snap0;   // slot k
  const T* snap1;   // slot k+1
};

constexpr int B3Z = 32;
constexpr int B3Y = 8;

// stencil along one axis (stride st), forward (D+) or backward (D-)
template <typename T, int N, bool FWD>
__device__ __forceinline__ T d3(const T* f, long long idx, long long st, const T* c) {
  T v = 0;
#pragma unroll
  for (int m = 0; m < N; ++m)
    v += FWD ? c[m] * (f[idx + (m + 1) * st] - f[idx - m * st]) : c[m] * (f[idx + m * st] - f[idx - (m + 1) * st]);
  return v;
}

// transposed stencil of a mid field M along one axis at coordinate x of n
template <typename T, int N, bool FWD>
__device__ __forceinline__ T d3t(const T* M, long long idx, long long st, int x, int n, const T* c) {
  T v = 0;
#pragma unroll
  for (int m = 0; m < N; ++m) {
    const int a = FWD ? x - m - 1 : x - m, b = FWD ? x + m : x + m + 1;
    const T ma = (a >= 0 && a < n) ? M[idx + (long long)(a - x) * st] : (T)0;
    const T mb = (b >= 0 && b < n) ? M[idx + (long long)(b - x) * st] : (T)0;
    v += c[m] * (ma - mb);
  }
  return v;
}

template <typename T>
__device__ __forceinline__ T pml_fwd3(T d, T psi_old, T b, T a, T kk) {
  const T psi = b * psi_old + a * d;
  return div_v(d, kk) + psi;
}
template <typename T>
__device__ __forceinline__ T pml_adj3(T dbar, T* psibar, T b, T a, T kk) {
  const T tot = *psibar + dbar;
  *psibar = b * tot;
  return dbar / kk + a * tot;
}

// CPML of one derivative of component `comp` along axis AX at cell (i, j, k):
// forward value from the snapshot's psi, adjoint through the adjoint psi.
template <typename T, int AX>
struct Cpml3 {
  long long off;  // element offset of psi within the axis's component array
  bool on;
  T b, a, kk;
};

template <typename T, int AX>
__device__ __forceinline__ Cpml3<T, AX> cpml3(const P3<T>& p, int comp, bool half, bool pred, int i, int j, int k) {
  Cpml3<T, AX> r{};
  const int n = AX == 0 ? p.nx : AX == 1 ? p.ny : p.nz;
  const int x = AX == 0 ? i : AX == 1 ? j : k;
  const int s = slab_index(x, n, p.lo[AX], p.hi[AX]);
  r.on = pred && s >= 0;
  if (!r.on) return r;
  const T* cf = p.cf[AX];
  r.b = cf[(half ? CBH : CB) * n + x];
  r.a = cf[(half ? CAH : CA) * n + x];
  r.kk = cf[(half ? CKH : CK) * n + x];
  if (AX == 0) r.off = comp * p.mcomp[0] + ((long long)s * p.ny + j) * p.nz + k;
  else if (AX == 1) r.off = comp * p.mcomp[1] + ((long long)i * p.sn[1] + s) * p.nz + k;
  else r.off = comp * p.mcomp[2] + ((long long)i * p.ny + j) * p.sn[2] + s;
  return r;
}

// snapshot memory variables of axis AX
template <typename T, int AX>
__device__ __forceinline__ const T* snap_mem(const P3<T>& p, const T* snap) {
  const long long nc = (long long)p.nx * p.ny * p.nz;
  const long long base = 9 * nc + (AX >= 1 ? 6 * p.mcomp[0] : 0) + (AX >= 2 ? 6 * p.mcomp[1] : 0);
  return snap + base;
}

#define CELL3                                                   \
  const int k = blockIdx.x * B3Z + threadIdx.x;                 \
  const int j = blockIdx.y * B3Y + threadIdx.y;                 \
  const int i = blockIdx.z;                                     \
  const int nx = p.nx, ny = p.ny, nz = p.nz;                    \
  if (j >= ny || k >= nz) return;                               \
  const long long sx = (long long)ny * nz, sy = nz;             \
  const long long idx = i * sx + (long long)j * nz + k;         \
  T c[N];                                                       \
  _Pragma("unroll") for (int m = 0; m < N; ++m) c[m] = p.c[m];  \
  const uint8_t fx = p.fl[0][i], fy = p.fl[1][j], fz = p.fl[2][k];

template <typename T>
__global__ void k3a_record(const __grid_constant__ P3<T> p, const __grid_constant__ A3<T> a, int it) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < p.nrec) atomicAdd(a.f[p.rec_field] + p.rec_idx[r], a.res[(long long)it * p.nrec + r]);
}

// ---- stress phase ---------------------------------------------------------------
template <typename T, int N>
__global__ void __launch_bounds__(B3Z * B3Y)
k3a_stress_mid(const __grid_constant__ P3<T> p, const __grid_constant__ A3<T> a) {
  CELL3
  const long long nc = (long long)nx * ny * nz;
  const T* vx = a.snap1;
  const T* vy = a.snap1 + nc;
  const T* vz = a.snap1 + 2 * nc;
  const T* m0 = snap_mem<T, 0>(p, a.snap0);
  const T* m1 = snap_mem<T, 1>(p, a.snap0);
  const T* m2 = snap_mem<T, 2>(p, a.snap0);
  const T dx = p.dx, dy = p.dy, dz = p.dz, dt = p.dt;
  T out[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  // normal stresses: i, j, k in [N+1, n-N)
  if (i >= N + 1 && i < nx - N && j >= N + 1 && j < ny - N && k >= N + 1 && k < nz - N) {
    const T lhx = (T)0.5 * (p.lam[idx] + p.lam[idx + sx]);
    const T mhx = (T)0.5 * (p.mu[idx] + p.mu[idx + sx]);
    const T lpm = lhx + (T)2 * mhx;
    const bool P = ((fx | fy | fz) & 1) != 0;
    auto cx = cpml3<T, 0>(p, 3, false, P, i, j, k);
    auto cy = cpml3<T, 1>(p, 3, false, P, i, j, k);
    auto cz = cpml3<T, 2>(p, 3, false, P, i, j, k);
    T e0 = d3<T, N, false>(vx, idx, sx, c) / dx;
    T e1 = d3<T, N, false>(vy, idx, sy, c) / dy;
    T e2 = d3<T, N, false>(vz, idx, 1, c) / dz;
    if (cx.on) e0 = pml_fwd3(e0, m0[cx.off], cx.b, cx.a, cx.kk);
    if (cy.on) e1 = pml_fwd3(e1, m1[cy.off], cy.b, cy.a, cy.kk);
    if (cz.on) e2 = pml_fwd3(e2, m2[cz.off], cz.b, cz.a, cz.kk);
    const T bx = a.f[3][idx], by = a.f[4][idx], bz = a.f[5][idx];
    a.grad[3][idx] += dt * (bx * e0 + by * e1 + bz * e2);
    a.grad[4][idx] += dt * (bx * (e2 + e1) + by * (e0 + e2) + bz * (e0 + e1));
    T g0 = dt * (lpm * bx + lhx * by + lhx * bz);
    T g1 = dt * (lhx * bx + lpm * by + lhx * bz);
    T g2 = dt * (lhx * bx + lhx * by + lpm * bz);
    if (cx.on) g0 = pml_adj3(g0, a.mem[0] + cx.off, cx.b, cx.a, cx.kk);
    if (cy.on) g1 = pml_adj3(g1, a.mem[1] + cy.off, cy.b, cy.a, cy.kk);
    if (cz.on) g2 = pml_adj3(g2, a.mem[2] + cz.off, cz.b, cz.a, cz.kk);
    out[0] = g0 / dx;
    out[1] = g1 / dy;
    out[2] = g2 / dz;
  }
  // sxy: i, j in [N+1, n-N), k in [N, nz-N)
  if (i >= N + 1 && i < nx - N && j >= N + 1 && j < ny - N && k >= N && k < nz - N) {
    const T m4 = (T)0.25 * (p.mu[idx + sy] + p.mu[idx] + p.mu[idx] + p.mu[idx + sx]);
    const bool P = (fx & 2) || (fy & 2) || (fz & 1);
    auto cx = cpml3<T, 0>(p, 4, true, P, i, j, k);
    auto cy = cpml3<T, 1>(p, 4, true, P, i, j, k);
    T f0 = d3<T, N, true>(vy, idx, sx, c) / dx;
    T f1 = d3<T, N, true>(vx, idx, sy, c) / dy;
    if (cx.on) f0 = pml_fwd3(f0, m0[cx.off], cx.b, cx.a, cx.kk);
    if (cy.on) f1 = pml_fwd3(f1, m1[cy.off], cy.b, cy.a, cy.kk);
    const T b = a.f[6][idx];
    a.grad[5][idx] += dt * b * (f1 + f0);
    T g = m4 * dt * b, g0 = g, g1 = g;
    if (cx.on) g0 = pml_adj3(g0, a.mem[0] + cx.off, cx.b, cx.a, cx.kk);
    if (cy.on) g1 = pml_adj3(g1, a.mem[1] + cy.off, cy.b, cy.a, cy.kk);
    out[3] = g0 / dx;
    out[4] = g1 / dy;
  }
  // sxz: i in [N, nx-N-1), j in [N, ny-N), k in [N, nz-N-1)
  if (i >= N && i < nx - N - 1 && j >= N && j < ny - N && k >= N && k < nz - N - 1) {
    const T m4 = (T)0.25 * (p.mu[idx] + p.mu[idx + sx] + p.mu[idx] + p.mu[idx + sy]);
    const bool P = (fx & 2) || (fy & 1) || (fz & 2);
    auto cx = cpml3<T, 0>(p, 5, true, P, i, j, k);
    auto cz = cpml3<T, 2>(p, 4, true, P, i, j, k);
    T h0 = d3<T, N, true>(vz, idx, sx, c) / dx;
    T h1 = d3<T, N, true>(vx, idx, 1, c) / dz;
    if (cx.on) h0 = pml_fwd3(h0, m0[cx.off], cx.b, cx.a, cx.kk);
    if (cz.on) h1 = pml_fwd3(h1, m2[cz.off], cz.b, cz.a, cz.kk);
    const T b = a.f[7][idx];
    a.grad[6][idx] += dt * b * (h1 + h0);
    T g = m4 * dt * b, g0 = g, g1 = g;
    if (cx.on) g0 = pml_adj3(g0, a.mem[0] + cx.off, cx.b, cx.a, cx.kk);
    if (cz.on) g1 = pml_adj3(g1, a.mem[2] + cz.off, cz.b, cz.a, cz.kk);
    out[5] = g0 / dx;
    out[6] = g1 / dz;
  }
  // syz: i in [N, nx-N), j in [N, ny-N-1), k in [N, nz-N-1)
  if (i >= N && i < nx - N && j >= N && j < ny - N - 1 && k >= N && k < nz - N - 1) {
    const T m4 = (T)0.25 * (p.mu[idx + sy] + p.mu[idx] + p.mu[idx + 1] + p.mu[idx]);
    const bool P = (fx & 1) || (fy & 2) || (fz & 2);
    auto cy = cpml3<T, 1>(p, 5, true, P, i, j, k);
    auto cz = cpml3<T, 2>(p, 5, true, P, i, j, k);
    T q0 = d3<T, N, true>(vz, idx, sy, c) / dy;
    T q1 = d3<T, N, true>(vy, idx, 1, c) / dz;
    if (cy.on) q0 = pml_fwd3(q0, m1[cy.off], cy.b, cy.a, cy.kk);
    if (cz.on) q1 = pml_fwd3(q1, m2[cz.off], cz.b, cz.a, cz.kk);
    const T b = a.f[8][idx];
    a.grad[7][idx] += dt * b * (q0 + q1);
    T g = m4 * dt * b, g0 = g, g1 = g;
    if (cy.on) g0 = pml_adj3(g0, a.mem[1] + cy.off, cy.b, cy.a, cy.kk);
    if (cz.on) g1 = pml_adj3(g1, a.mem[2] + cz.off, cz.b, cz.a, cz.kk);
    out[7] = g0 / dy;
    out[8] = g1 / dz;
  }
#pragma unroll
  for (int q = 0; q < 9; ++q) a.tmp[q][idx] = out[q];
}

// vx_bar += D-x^T t0 + D+y^T t4 + D+z^T t6; vy_bar += D-y^T t1 + D+x^T t3 + D+z^T t8;
// vz_bar += D-z^T t2 + D+x^T t5 + D+y^T t7
template <typename T, int N>
__global__ void __launch_bounds__(B3Z * B3Y)
k3a_vel_gather(const __grid_constant__ P3<T> p, const __grid_constant__ A3<T> a) {
  CELL3
  (void)fx; (void)fy; (void)fz;
  a.f[0][idx] += d3t<T, N, false>(a.tmp[0], idx, sx, i, nx, c) + d3t<T, N, true>(a.tmp[4], idx, sy, j, ny, c) +
                 d3t<T, N, true>(a.tmp[6], idx, 1, k, nz, c);
  a.f[1][idx] += d3t<T, N, false>(a.tmp[1], idx, sy, j, ny, c) + d3t<T, N, true>(a.tmp[3], idx, sx, i, nx, c) +
                 d3t<T, N, true>(a.tmp[8], idx, 1, k, nz, c);
  a.f[2][idx] += d3t<T, N, false>(a.tmp[2], idx, 1, k, nz, c) + d3t<T, N, true>(a.tmp[5], idx, sx, i, nx, c) +
                 d3t<T, N, true>(a.tmp[7], idx, sy, j, ny, c);
}

// ---- velocity phase -------------------------------------------------------------
template <typename T, int N>
__global__ void __launch_bounds__(B3Z * B3Y)
k3a_vel_mid(const __grid_constant__ P3<T> p, const __grid_constant__ A3<T> a) {
  CELL3
  const long long nc = (long long)nx * ny * nz;
  const T* sxx = a.snap0 + 3 * nc;
  const T* syy = a.snap0 + 4 * nc;
  const T* szz = a.snap0 + 5 * nc;
  const T* sxy = a.snap0 + 6 * nc;
  const T* sxz = a.snap0 + 7 * nc;
  const T* syz = a.snap0 + 8 * nc;
  const T* m0 = snap_mem<T, 0>(p, a.snap0);
  const T* m1 = snap_mem<T, 1>(p, a.snap0);
  const T* m2 = snap_mem<T, 2>(p, a.snap0);
  const T dx = p.dx, dy = p.dy, dz = p.dz, dt = p.dt;
  const T* rho = p.rho;
  T out[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  // vx: i in [N, nx-N-1), j in [N+1, ny-N), k in [N+1, nz-N)
  if (i >= N && i < nx - N - 1 && j >= N + 1 && j < ny - N && k >= N + 1 && k < nz - N) {
    const bool P = (fx & 2) || (fy & 1) || (fz & 1);
    auto cx = cpml3<T, 0>(p, 0, true, P, i, j, k);
    auto cy = cpml3<T, 1>(p, 0, false, P, i, j, k);
    auto cz = cpml3<T, 2>(p, 0, false, P, i, j, k);
    T d0 = d3<T, N, true>(sxx, idx, sx, c) / dx;
    T d1 = d3<T, N, false>(sxy, idx, sy, c) / dy;
    T d2 = d3<T, N, false>(sxz, idx, 1, c) / dz;
    if (cx.on) d0 = pml_fwd3(d0, m0[cx.off], cx.b, cx.a, cx.kk);
    if (cy.on) d1 = pml_fwd3(d1, m1[cy.off], cy.b, cy.a, cy.kk);
    if (cz.on) d2 = pml_fwd3(d2, m2[cz.off], cz.b, cz.a, cz.kk);
    const T vb = a.f[0][idx];
    a.grad[0][idx] += vb * (d0 + d2 + d1) * dt;
    T g = vb * dt / rho[idx], g0 = g, g1 = g, g2 = g;
    if (cx.on) g0 = pml_adj3(g0, a.mem[0] + cx.off, cx.b, cx.a, cx.kk);
    if (cy.on) g1 = pml_adj3(g1, a.mem[1] + cy.off, cy.b, cy.a, cy.kk);
    if (cz.on) g2 = pml_adj3(g2, a.mem[2] + cz.off, cz.b, cz.a, cz.kk);
    out[0] = g0 / dx;
    out[1] = g1 / dy;
    out[2] = g2 / dz;
  }
  // vy: i in [N+1, nx-N), j in [N, ny-N-1), k in [N+1, nz-N)
  if (i >= N + 1 && i < nx - N && j >= N && j < ny - N - 1 && k >= N + 1 && k < nz - N) {
    const T rhy = (T)0.5 * (rho[idx] + rho[idx + sy]);
    const bool P = (fx & 1) || (fy & 2) || (fz & 1);
    auto cx = cpml3<T, 0>(p, 1, false, P, i, j, k);
    auto cy = cpml3<T, 1>(p, 1, true, P, i, j, k);
    auto cz = cpml3<T, 2>(p, 1, false, P, i, j, k);
    T d0 = d3<T, N, false>(sxy, idx, sx, c) / dx;
    T d1 = d3<T, N, true>(syy, idx, sy, c) / dy;
    T d2 = d3<T, N, false>(syz, idx, 1, c) / dz;
    if (cx.on) d0 = pml_fwd3(d0, m0[cx.off], cx.b, cx.a, cx.kk);
    if (cy.on) d1 = pml_fwd3(d1, m1[cy.off], cy.b, cy.a, cy.kk);
    if (cz.on) d2 = pml_fwd3(d2, m2[cz.off], cz.b, cz.a, cz.kk);
    const T vb = a.f[1][idx];
    a.grad[1][idx] += vb * (d0 + d1 + d2) * dt;
    T g = vb * dt / rhy, g0 = g, g1 = g, g2 = g;
    if (cx.on) g0 = pml_adj3(g0, a.mem[0] + cx.off, cx.b, cx.a, cx.kk);
    if (cy.on) g1 = pml_adj3(g1, a.mem[1] + cy.off, cy.b, cy.a, cy.kk);
    if (cz.on) g2 = pml_adj3(g2, a.mem[2] + cz.off, cz.b, cz.a, cz.kk);
    out[3] = g0 / dx;
    out[4] = g1 / dy;
    out[5] = g2 / dz;
  }
  // vz: i in [N+1, nx-N), j in [N+1, ny-N), k in [N, nz-N-1)
  if (i >= N + 1 && i < nx - N && j >= N + 1 && j < ny - N && k >= N && k < nz - N - 1) {
    const T r4 = (T)0.25 * (rho[idx] + rho[idx + sy] + rho[idx + sx + sy] + rho[idx + sx]);
    const bool P = (fx & 1) || (fy & 1) || (fz & 2);
    auto cx = cpml3<T, 0>(p, 2, false, P, i, j, k);
    auto cy = cpml3<T, 1>(p, 2, false, P, i, j, k);
    auto cz = cpml3<T, 2>(p, 2, true, P, i, j, k);
    T d0 = d3<T, N, false>(sxz, idx, sx, c) / dx;
    T d1 = d3<T, N, false>(syz, idx, sy, c) / dy;
    T d2 = d3<T, N, true>(szz, idx, 1, c) / dz;
    if (cx.on) d0 = pml_fwd3(d0, m0[cx.off], cx.b, cx.a, cx.kk);
    if (cy.on) d1 = pml_fwd3(d1, m1[cy.off], cy.b, cy.a, cy.kk);
    if (cz.on) d2 = pml_fwd3(d2, m2[cz.off], cz.b, cz.a, cz.kk);
    const T vb = a.f[2][idx];
    a.grad[2][idx] += vb * (d0 + d1 + d2) * dt;
    T g = vb * dt / r4, g0 = g, g1 = g, g2 = g;
    if (cx.on) g0 = pml_adj3(g0, a.mem[0] + cx.off, cx.b, cx.a, cx.kk);
    if (cy.on) g1 = pml_adj3(g1, a.mem[1] + cy.off, cy.b, cy.a, cy.kk);
    if (cz.on) g2 = pml_adj3(g2, a.mem[2] + cz.off, cz.b, cz.a, cz.kk);
    out[6] = g0 / dx;
    out[7] = g1 / dy;
    out[8] = g2 / dz;
  }
#pragma unroll
  for (int q = 0; q < 9; ++q) a.tmp[q][idx] = out[q];
}

// sxx_bar += D+x^T t0; syy_bar += D+y^T t4; szz_bar += D+z^T t8;
// sxy_bar += D-y^T t1 + D-x^T t3; sxz_bar += D-z^T t2 + D-x^T t6; syz_bar += D-z^T t5 + D-y^T t7
template <typename T, int N>
__global__ void __launch_bounds__(B3Z * B3Y)
k3a_str_gather(const __grid_constant__ P3<T> p, const __grid_constant__ A3<T> a) {
  CELL3
  (void)fx; (void)fy; (void)fz;
  a.f[3][idx] += d3t<T, N, true>(a.tmp[0], idx, sx, i, nx, c);
  a.f[4][idx] += d3t<T, N, true>(a.tmp[4], idx, sy, j, ny, c);
  a.f[5][idx] += d3t<T, N, true>(a.tmp[8], idx, 1, k, nz, c);
  a.f[6][idx] += d3t<T, N, false>(a.tmp[1], idx, sy, j, ny, c) + d3t<T, N, false>(a.tmp[3], idx, sx, i, nx, c);
  a.f[7][idx] += d3t<T, N, false>(a.tmp[2], idx, 1, k, nz, c) + d3t<T, N, false>(a.tmp[6], idx, sx, i, nx, c);
  a.f[8][idx] += d3t<T, N, false>(a.tmp[5], idx, 1, k, nz, c) + d3t<T, N, false>(a.tmp[7], idx, sy, j, ny, c);
}

#undef CELL3

// The point force (Elastic3D_SSG_CPML.py:245) adds t/rho[src], t = dt*w(it),
// to vz after the velocity phase; its adjoint leaves vz_bar as it is and adds
// -t*vz_bar/rho^2 to d misfit / d rho[src], kept as t*vz_bar in grad[0] (the
// slot whose coefficient is 1/rho of the same cell).  vz_bar here is the
// adjoint after the stress phase's gather.
template <typename T>
__global__ void k3a_force(const __grid_constant__ P3<T> p, const __grid_constant__ A3<T> a, int it) {
  const long long s = ((long long)p.si * p.ny + p.sj) * p.nz + p.sk;
  a.grad[0][s] += (p.dt * p.wav[it]) * a.f[2][s];
}

template <typename T, int N>
static cudaError_t adj3_step(const P3<T>& p, const A3<T>& a, int it, cudaStream_t st) {
  dim3 block(B3Z, B3Y);
  dim3 grid((p.nz + B3Z - 1) / B3Z, (p.ny + B3Y - 1) / B3Y, p.nx);
  if (p.nrec > 0) k3a_record<T><<<(p.nrec + 255) / 256, 256, 0, st>>>(p, a, it);
  k3a_stress_mid<T, N><<<grid, block, 0, st>>>(p, a);
  k3a_vel_gather<T, N><<<grid, block, 0, st>>>(p, a);
  if (p.src_kind == SW_SRC_FORCE) k3a_force<T><<<1, 1, 0, st>>>(p, a, it);
  k3a_vel_mid<T, N><<<grid, block, 0, st>>>(p, a);
  k3a_str_gather<T, N><<<grid, block, 0, st>>>(p, a);
  return cudaGetLastError();
}

template <typename T>
cudaError_t sw3_adjoint_step(const P3<T>& p, const A3<T>& a, int order, int it, cudaStream_t st) {
  switch (order) {
    case 1: return adj3_step<T, 1>(p, a, it, st);
    case 2: return adj3_step<T, 2>(p, a, it, st);
    case 3: return adj3_step<T, 3>(p, a, it, st);
    case 4: return adj3_step<T, 4>(p, a, it, st);
    default: return cudaErrorInvalidValue;
  }
}

template cudaError_t sw3_adjoint_step<float>(const P3<float>&, const A3<float>&, int, int, cudaStream_t);
template cudaError_t sw3_adjoint_step<double>(const P3<double>&, const A3<double>&, int, int, cudaStream_t);

}  // namespace sw
