// elastic2d_adjoint.cu -- hand-written discrete adjoints of the 2D SSG_VS and
// SSG_SV time steps (src/Elastic2D_CPML.py:128-200, :202-275) with a
// moment-tensor source, and the forward recording pass they run on.  No
// reference counterpart.  The VS derivation is written out here; the SV
// kernels below follow it with that scheme's staggering.
//
// Forward step it, as linear maps on the state (v, sigma, psi):
//   inject   sigma[src] += w(it) * (-M)                         (affine)
//   V        vx += dt/rho  * (Dbx sxx' + Dbz sxz')               vx cells
//            vz += dt/rho4 * (Dfx sxz' + Dfz szz')               vz cells
//   S        sxx += dt*(lpm p' + lhx q'),  szz += dt*(lpm q' + lhx p'),
//            p = Dfx vx, q = Dbz vz                              sxx cells
//            sxz += mhz*(u' + r')*dt,  u = Dfz vx, r = Dbx vz    sxz cells
//   record   data[it] = vz[rec]
// where d' = d/kappa + psi_new, psi_new = b psi + a d on the CPML cells.
// The adjoint of step it runs these in reverse: the receiver residual is added
// to vz_bar; each phase computes, per cell, the adjoint of its CPML-corrected
// derivatives ("mid" fields, psi_bar recursion reversed) and the gradient of
// the misfit with respect to the cell's material coefficient, then a gather
// kernel applies the transposed stencils.  The forward values each gradient
// needs come from snapshots recorded by sw2d_record: slot k holds the state of
// step it after its source injection, slot k+1 the velocities after the
// velocity phase of step it.
#include "sw_device.cuh"
#include "sw_stencil2d.cuh"

namespace sw {

template <typename T>
struct A2 {
  T* f[5];          // adjoint of vx vz sxx szz sxz
  T* mem[2];        // adjoint memory variables, slab layout of P2::mem
  T* tmp[4];        // mid fields (nx, nz)
  T* grad[5];       // per-cell sums: G_vx (rho), G_vz (rho4), G_lpm, G_lhx, G_mhz
  const T* res;     // receiver residual (nt, nrec)
  const T* snap0;   // slot k
  const T* snap1;   // slot k+1
};

// Resident blocks per SM the float adjoint kernels are compiled for (a full
// SM): one thread per cell waits on its loads, as in the batched forward.
#define SW_ADJ_MINB (sizeof(T) == 4 ? 2048 / (A2Z * A2X) : 1)
constexpr int A2Z = 32;
constexpr int A2X = 8;

template <typename T>
struct Snap2 {
  const T* s;
  long long ncell, mc0, mc1;
  int nz, sn1;
  __device__ const T* f(int q) const { return s + q * ncell; }
  __device__ T mx(int comp, int xi, int j) const { return s[5 * ncell + comp * mc0 + (long long)xi * nz + j]; }
  __device__ T mz(int comp, int i, int zj) const {
    return s[5 * ncell + 4 * mc0 + comp * mc1 + (long long)i * sn1 + zj];
  }
};

template <typename T>
__device__ __forceinline__ Snap2<T> snap_of(const P2<T>& p, const T* s) {
  return Snap2<T>{s, (long long)p.nx * p.nz, p.mcomp[0], p.mcomp[1], p.nz, p.sn[1]};
}

// forward CPML correction of a derivative d, from the memory variable before
// the step (psi_old): returns d' = d/kappa + (b psi_old + a d)
template <typename T>
__device__ __forceinline__ T pml_fwd(T d, T psi_old, T b, T a, T kk) {
  const T psi = b * psi_old + a * d;
  return div_v(d, kk) + psi;
}
// adjoint of the correction: given dbar' and psi_bar (adjoint of psi after
// this step's update), returns dbar and leaves psi_bar = adjoint of psi_old
template <typename T>
__device__ __forceinline__ T pml_adj(T dbar, T* psibar, T b, T a, T kk) {
  const T tot = *psibar + dbar;
  *psibar = b * tot;
  return dbar / kk + a * tot;
}

// adjoint memory variables, same slab layout as the forward ones
template <typename T>
__device__ __forceinline__ T* amx(const P2<T>& p, const A2<T>& a, int comp, int xi, int j) {
  return a.mem[0] + comp * p.mcomp[0] + (long long)xi * p.nz + j;
}
template <typename T>
__device__ __forceinline__ T* amz(const P2<T>& p, const A2<T>& a, int comp, int i, int zj) {
  return a.mem[1] + comp * p.mcomp[1] + (long long)i * p.sn[1] + zj;
}

template <typename T>
__device__ __forceinline__ T at(const T* f, int i, int j, int nx, int nz) {
  return (i >= 0 && i < nx && j >= 0 && j < nz) ? f[(long long)i * nz + j] : (T)0;
}

// receivers: vz_bar[rec] += residual(it, r)
template <typename T>
__global__ void k2a_record(const __grid_constant__ P2<T> p, const __grid_constant__ A2<T> a, int it) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < p.nrec) atomicAdd(a.f[p.rec_field] + p.rec_idx[r], a.res[(long long)it * p.nrec + r]);
}

// ---- stress phase: mids and lam/mu gradients ---------------------------------
template <typename T, int N>
__global__ void __launch_bounds__(A2Z * A2X, SW_ADJ_MINB)
k2a_stress_mid(const __grid_constant__ P2<T> p, const __grid_constant__ A2<T> a) {
  const int j = blockIdx.x * A2Z + threadIdx.x;
  const int i = blockIdx.y * A2X + threadIdx.y;
  const int nx = p.nx, nz = p.nz;
  if (i >= nx || j >= nz) return;
  const long long idx = (long long)i * nz + j;
  const T dx = p.dx, dz = p.dz, dt = p.dt;
  // quotients by the spacings: the verified constant-divisor route (the
  // forward pass's bits, IEEE division's bits)
  auto qdx = [&](T v) { return div_c(v, dx, p.rd[0], p.fast_div & 1); };
  auto qdz = [&](T v) { return div_c(v, dz, p.rd[1], p.fast_div & 1); };
  T c[N];
#pragma unroll
  for (int m = 0; m < N; ++m) c[m] = p.c[m];
  const Snap2<T> s0 = snap_of(p, a.snap0), s1 = snap_of(p, a.snap1);
  const T* vx = s1.f(0);
  const T* vz = s1.f(1);
  const T* cfx = p.cf[0];
  const T* cfz = p.cf[1];
  const int xi = slab_index(i, nx, p.lo[0], p.hi[0]);
  const int zj = slab_index(j, nz, p.lo[1], p.hi[1]);
  const uint8_t fx = p.fl[0][i], fz = p.fl[1][j];
  T t0 = 0, t1 = 0, t2 = 0, t3 = 0;
  // sxx szz at (i+1/2, j)
  if (i >= N && i < nx - N - 1 && j >= N + 1 && j < nz - N) {
    const T lhx = (T)0.5 * (p.lam[idx] + p.lam[idx + nz]);
    const T mhx = (T)0.5 * (p.mu[idx] + p.mu[idx + nz]);
    const T lpm = lhx + (T)2 * mhx;
    T pv = qdx(dx_fm<T, N>(vx, idx, nz, c));
    T qv = qdz(dz_bm<T, N>(vz, idx, c));
    const bool P = (fx & 2) || (fz & 1);
    const T bxh = cfx[CBH * nx + i], axh = cfx[CAH * nx + i], kxh = cfx[CKH * nx + i];
    const T bz = cfz[CB * nz + j], az = cfz[CA * nz + j], kz = cfz[CK * nz + j];
    if (P && xi >= 0) pv = pml_fwd(pv, s0.mx(2, xi, j), bxh, axh, kxh);
    if (P && zj >= 0) qv = pml_fwd(qv, s0.mz(2, i, zj), bz, az, kz);
    const T sb = a.f[2][idx], zb = a.f[3][idx];
    a.grad[2][idx] += dt * (sb * pv + zb * qv);
    a.grad[3][idx] += dt * (sb * qv + zb * pv);
    T pb = dt * (lpm * sb + lhx * zb);
    T qb = dt * (lhx * sb + lpm * zb);
    if (P && xi >= 0) pb = pml_adj(pb, amx(p, a, 2, xi, j), bxh, axh, kxh);
    if (P && zj >= 0) qb = pml_adj(qb, amz(p, a, 2, i, zj), bz, az, kz);
    t0 = qdx(pb);
    t1 = qdz(qb);
  }
  // sxz at (i, j+1/2)
  if (i >= N + 1 && i < nx - N && j >= N && j < nz - N - 1) {
    const T mhz = (T)0.5 * (p.mu[idx + 1] + p.mu[idx]);
    T rv = qdx(dx_bm<T, N>(vz, idx, nz, c));
    T uv = qdz(dz_fm<T, N>(vx, idx, c));
    const bool P = (fx & 1) || (fz & 2);
    const T bx = cfx[CB * nx + i], ax = cfx[CA * nx + i], kx = cfx[CK * nx + i];
    const T bzh = cfz[CBH * nz + j], azh = cfz[CAH * nz + j], kzh = cfz[CKH * nz + j];
    if (P && xi >= 0) rv = pml_fwd(rv, s0.mx(3, xi, j), bx, ax, kx);
    if (P && zj >= 0) uv = pml_fwd(uv, s0.mz(3, i, zj), bzh, azh, kzh);
    const T xb = a.f[4][idx];
    a.grad[4][idx] += dt * xb * (uv + rv);
    T sb = mhz * dt * xb;
    T ub = sb, rb = sb;
    if (P && xi >= 0) rb = pml_adj(rb, amx(p, a, 3, xi, j), bx, ax, kx);
    if (P && zj >= 0) ub = pml_adj(ub, amz(p, a, 3, i, zj), bzh, azh, kzh);
    t2 = qdz(ub);
    t3 = qdx(rb);
  }
  a.tmp[0][idx] = t0;
  a.tmp[1][idx] = t1;
  a.tmp[2][idx] = t2;
  a.tmp[3][idx] = t3;
}

// vx_bar += Dfx^T t0 + Dfz^T t2;  vz_bar += Dbz^T t1 + Dbx^T t3
template <typename T, int N>
__global__ void __launch_bounds__(A2Z * A2X, SW_ADJ_MINB)
k2a_vel_gather(const __grid_constant__ P2<T> p, const __grid_constant__ A2<T> a) {
  const int j = blockIdx.x * A2Z + threadIdx.x;
  const int i = blockIdx.y * A2X + threadIdx.y;
  const int nx = p.nx, nz = p.nz;
  if (i >= nx || j >= nz) return;
  const long long idx = (long long)i * nz + j;
  T gx = 0, gz = 0;
#pragma unroll
  for (int m = 0; m < N; ++m) {
    const T c = p.c[m];
    gx += c * (at(a.tmp[0], i - m - 1, j, nx, nz) - at(a.tmp[0], i + m, j, nx, nz));
    gx += c * (at(a.tmp[2], i, j - m - 1, nx, nz) - at(a.tmp[2], i, j + m, nx, nz));
    gz += c * (at(a.tmp[1], i, j - m, nx, nz) - at(a.tmp[1], i, j + m + 1, nx, nz));
    gz += c * (at(a.tmp[3], i - m, j, nx, nz) - at(a.tmp[3], i + m + 1, j, nx, nz));
  }
  a.f[0][idx] += gx;
  a.f[1][idx] += gz;
}

// ---- velocity phase: mids and rho gradients ---------------------------------
template <typename T, int N>
__global__ void __launch_bounds__(A2Z * A2X, SW_ADJ_MINB)
k2a_vel_mid(const __grid_constant__ P2<T> p, const __grid_constant__ A2<T> a) {
  const int j = blockIdx.x * A2Z + threadIdx.x;
  const int i = blockIdx.y * A2X + threadIdx.y;
  const int nx = p.nx, nz = p.nz;
  if (i >= nx || j >= nz) return;
  const long long idx = (long long)i * nz + j;
  const T dx = p.dx, dz = p.dz, dt = p.dt;
  // quotients by the spacings: the verified constant-divisor route (the
  // forward pass's bits, IEEE division's bits)
  auto qdx = [&](T v) { return div_c(v, dx, p.rd[0], p.fast_div & 1); };
  auto qdz = [&](T v) { return div_c(v, dz, p.rd[1], p.fast_div & 1); };
  T c[N];
#pragma unroll
  for (int m = 0; m < N; ++m) c[m] = p.c[m];
  const Snap2<T> s0 = snap_of(p, a.snap0);
  const T* sxx = s0.f(2);
  const T* szz = s0.f(3);
  const T* sxz = s0.f(4);
  const T* cfx = p.cf[0];
  const T* cfz = p.cf[1];
  const T* rho = p.rho;
  const int xi = slab_index(i, nx, p.lo[0], p.hi[0]);
  const int zj = slab_index(j, nz, p.lo[1], p.hi[1]);
  const uint8_t fx = p.fl[0][i], fz = p.fl[1][j];
  T t0 = 0, t1 = 0, t2 = 0, t3 = 0;
  // vx at (i, j)
  if (i >= N + 1 && i < nx - N && j >= N + 1 && j < nz - N) {
    T av = qdx(dx_bm<T, N>(sxx, idx, nz, c));
    T bv = qdz(dz_bm<T, N>(sxz, idx, c));
    const bool P = (fx & 1) || (fz & 1);
    const T bx = cfx[CB * nx + i], ax = cfx[CA * nx + i], kx = cfx[CK * nx + i];
    const T bz = cfz[CB * nz + j], az = cfz[CA * nz + j], kz = cfz[CK * nz + j];
    if (P && xi >= 0) av = pml_fwd(av, s0.mx(0, xi, j), bx, ax, kx);
    if (P && zj >= 0) bv = pml_fwd(bv, s0.mz(0, i, zj), bz, az, kz);
    const T vb = a.f[0][idx];
    a.grad[0][idx] += vb * (av + bv) * dt;
    T sb = vb * dt / rho[idx];
    T ab = sb, bb = sb;
    if (P && xi >= 0) ab = pml_adj(ab, amx(p, a, 0, xi, j), bx, ax, kx);
    if (P && zj >= 0) bb = pml_adj(bb, amz(p, a, 0, i, zj), bz, az, kz);
    t0 = qdx(ab);
    t1 = qdz(bb);
  }
  // vz at (i+1/2, j+1/2)
  if (i >= N && i < nx - N - 1 && j >= N && j < nz - N - 1) {
    const T rh = (T)0.25 * (rho[idx] + rho[idx + 1] + rho[idx + nz + 1] + rho[idx + nz]);
    T av = qdx(dx_fm<T, N>(sxz, idx, nz, c));
    T bv = qdz(dz_fm<T, N>(szz, idx, c));
    const bool P = (fx & 2) || (fz & 2);
    const T bxh = cfx[CBH * nx + i], axh = cfx[CAH * nx + i], kxh = cfx[CKH * nx + i];
    const T bzh = cfz[CBH * nz + j], azh = cfz[CAH * nz + j], kzh = cfz[CKH * nz + j];
    if (P && xi >= 0) av = pml_fwd(av, s0.mx(1, xi, j), bxh, axh, kxh);
    if (P && zj >= 0) bv = pml_fwd(bv, s0.mz(1, i, zj), bzh, azh, kzh);
    const T vb = a.f[1][idx];
    a.grad[1][idx] += vb * (av + bv) * dt;
    T sb = vb * dt / rh;
    T ab = sb, bb = sb;
    if (P && xi >= 0) ab = pml_adj(ab, amx(p, a, 1, xi, j), bxh, axh, kxh);
    if (P && zj >= 0) bb = pml_adj(bb, amz(p, a, 1, i, zj), bzh, azh, kzh);
    t2 = qdx(ab);
    t3 = qdz(bb);
  }
  a.tmp[0][idx] = t0;
  a.tmp[1][idx] = t1;
  a.tmp[2][idx] = t2;
  a.tmp[3][idx] = t3;
}

// sxx_bar += Dbx^T t0;  sxz_bar += Dbz^T t1 + Dfx^T t2;  szz_bar += Dfz^T t3
template <typename T, int N>
__global__ void __launch_bounds__(A2Z * A2X, SW_ADJ_MINB)
k2a_str_gather(const __grid_constant__ P2<T> p, const __grid_constant__ A2<T> a) {
  const int j = blockIdx.x * A2Z + threadIdx.x;
  const int i = blockIdx.y * A2X + threadIdx.y;
  const int nx = p.nx, nz = p.nz;
  if (i >= nx || j >= nz) return;
  const long long idx = (long long)i * nz + j;
  T gxx = 0, gxz = 0, gzz = 0;
#pragma unroll
  for (int m = 0; m < N; ++m) {
    const T c = p.c[m];
    gxx += c * (at(a.tmp[0], i - m, j, nx, nz) - at(a.tmp[0], i + m + 1, j, nx, nz));
    gxz += c * (at(a.tmp[1], i, j - m, nx, nz) - at(a.tmp[1], i, j + m + 1, nx, nz));
    gxz += c * (at(a.tmp[2], i - m - 1, j, nx, nz) - at(a.tmp[2], i + m, j, nx, nz));
    gzz += c * (at(a.tmp[3], i, j - m - 1, nx, nz) - at(a.tmp[3], i, j + m, nx, nz));
  }
  a.f[2][idx] += gxx;
  a.f[3][idx] += gzz;
  a.f[4][idx] += gxz;
}

// ============================================================================
// SSG_SV (src/Elastic2D_CPML.py:202-275): vx at (i+1/2, j), vz at (i, j+1/2),
// sxx szz at (i, j), sxz at (i+1/2, j+1/2).
//   V  vx += dt/rho2 * (Dfx sxx' + Dbz sxz'),  rho2 = (rho[i,j] + rho[i+1,j]) / 2
//      vz += dt/rhoz * (Dfz szz' + Dbx sxz'),  rhoz = (rho[i,j] + rho[i,j+1]) / 2
//   S  sxx += dt*(lpm p' + lm q'),  szz += dt*(lpm q' + lm p'),
//      p = Dbx vx, q = Dbz vz, lm = lam[i,j], lpm = lam + 2 mu
//      sxz += m4*(u' + r')*dt,  u = Dfz vx, r = Dfx vz, m4 = mean of mu over
//      (i,j) (i,j+1) (i+1,j+1) (i+1,j)
//   record data[it] = vx[rec]
// The gradient slots hold the same kind of per-cell sums as for VS:
// G_vx (rho2), G_vz (rhoz), G_lpm, G_lm, G_m4.
// ============================================================================
template <typename T, int N>
__global__ void __launch_bounds__(A2Z * A2X, SW_ADJ_MINB)
k2a_sv_stress_mid(const __grid_constant__ P2<T> p, const __grid_constant__ A2<T> a) {
  const int j = blockIdx.x * A2Z + threadIdx.x;
  const int i = blockIdx.y * A2X + threadIdx.y;
  const int nx = p.nx, nz = p.nz;
  if (i >= nx || j >= nz) return;
  const long long idx = (long long)i * nz + j;
  const T dx = p.dx, dz = p.dz, dt = p.dt;
  // quotients by the spacings: the verified constant-divisor route (the
  // forward pass's bits, IEEE division's bits)
  auto qdx = [&](T v) { return div_c(v, dx, p.rd[0], p.fast_div & 1); };
  auto qdz = [&](T v) { return div_c(v, dz, p.rd[1], p.fast_div & 1); };
  T c[N];
#pragma unroll
  for (int m = 0; m < N; ++m) c[m] = p.c[m];
  const Snap2<T> s0 = snap_of(p, a.snap0), s1 = snap_of(p, a.snap1);
  const T* vx = s1.f(0);
  const T* vz = s1.f(1);
  const T* cfx = p.cf[0];
  const T* cfz = p.cf[1];
  const int xi = slab_index(i, nx, p.lo[0], p.hi[0]);
  const int zj = slab_index(j, nz, p.lo[1], p.hi[1]);
  const uint8_t fx = p.fl[0][i], fz = p.fl[1][j];
  T t0 = 0, t1 = 0, t2 = 0, t3 = 0;
  if (i >= N + 1 && i < nx - N && j >= N + 1 && j < nz - N) {
    // sxx szz at (i, j)
    {
      const T lm = p.lam[idx];
      const T lpm = p.lam[idx] + (T)2 * p.mu[idx];
      T pv = qdx(dx_bm<T, N>(vx, idx, nz, c));
      T qv = qdz(dz_bm<T, N>(vz, idx, c));
      const bool P = (fx & 1) || (fz & 1);
      const T bx = cfx[CB * nx + i], ax = cfx[CA * nx + i], kx = cfx[CK * nx + i];
      const T bz = cfz[CB * nz + j], az = cfz[CA * nz + j], kz = cfz[CK * nz + j];
      if (P && xi >= 0) pv = pml_fwd(pv, s0.mx(2, xi, j), bx, ax, kx);
      if (P && zj >= 0) qv = pml_fwd(qv, s0.mz(2, i, zj), bz, az, kz);
      const T sb = a.f[2][idx], zb = a.f[3][idx];
      a.grad[2][idx] += dt * (sb * pv + zb * qv);
      a.grad[3][idx] += dt * (sb * qv + zb * pv);
      T pb = dt * (lpm * sb + lm * zb);
      T qb = dt * (lm * sb + lpm * zb);
      if (P && xi >= 0) pb = pml_adj(pb, amx(p, a, 2, xi, j), bx, ax, kx);
      if (P && zj >= 0) qb = pml_adj(qb, amz(p, a, 2, i, zj), bz, az, kz);
      t0 = qdx(pb);
      t1 = qdz(qb);
    }
    // sxz at (i+1/2, j+1/2)
    {
      const T m4 = (T)0.25 * (p.mu[idx + 1] + p.mu[idx] + p.mu[idx + nz + 1] + p.mu[idx + nz]);
      T rv = qdx(dx_fm<T, N>(vz, idx, nz, c));
      T uv = qdz(dz_fm<T, N>(vx, idx, c));
      const bool P = (fx & 2) || (fz & 2);
      const T bxh = cfx[CBH * nx + i], axh = cfx[CAH * nx + i], kxh = cfx[CKH * nx + i];
      const T bzh = cfz[CBH * nz + j], azh = cfz[CAH * nz + j], kzh = cfz[CKH * nz + j];
      if (P && xi >= 0) rv = pml_fwd(rv, s0.mx(3, xi, j), bxh, axh, kxh);
      if (P && zj >= 0) uv = pml_fwd(uv, s0.mz(3, i, zj), bzh, azh, kzh);
      const T xb = a.f[4][idx];
      a.grad[4][idx] += dt * xb * (uv + rv);
      T sb = m4 * dt * xb;
      T ub = sb, rb = sb;
      if (P && xi >= 0) rb = pml_adj(rb, amx(p, a, 3, xi, j), bxh, axh, kxh);
      if (P && zj >= 0) ub = pml_adj(ub, amz(p, a, 3, i, zj), bzh, azh, kzh);
      t2 = qdz(ub);
      t3 = qdx(rb);
    }
  }
  a.tmp[0][idx] = t0;
  a.tmp[1][idx] = t1;
  a.tmp[2][idx] = t2;
  a.tmp[3][idx] = t3;
}

// vx_bar += Dbx^T t0 + Dfz^T t2;  vz_bar += Dbz^T t1 + Dfx^T t3
template <typename T, int N>
__global__ void __launch_bounds__(A2Z * A2X, SW_ADJ_MINB)
k2a_sv_vel_gather(const __grid_constant__ P2<T> p, const __grid_constant__ A2<T> a) {
  const int j = blockIdx.x * A2Z + threadIdx.x;
  const int i = blockIdx.y * A2X + threadIdx.y;
  const int nx = p.nx, nz = p.nz;
  if (i >= nx || j >= nz) return;
  const long long idx = (long long)i * nz + j;
  T gx = 0, gz = 0;
#pragma unroll
  for (int m = 0; m < N; ++m) {
    const T c = p.c[m];
    gx += c * (at(a.tmp[0], i - m, j, nx, nz) - at(a.tmp[0], i + m + 1, j, nx, nz));
    gx += c * (at(a.tmp[2], i, j - m - 1, nx, nz) - at(a.tmp[2], i, j + m, nx, nz));
    gz += c * (at(a.tmp[1], i, j - m, nx, nz) - at(a.tmp[1], i, j + m + 1, nx, nz));
    gz += c * (at(a.tmp[3], i - m - 1, j, nx, nz) - at(a.tmp[3], i + m, j, nx, nz));
  }
  a.f[0][idx] += gx;
  a.f[1][idx] += gz;
}

template <typename T, int N>
__global__ void __launch_bounds__(A2Z * A2X, SW_ADJ_MINB)
k2a_sv_vel_mid(const __grid_constant__ P2<T> p, const __grid_constant__ A2<T> a) {
  const int j = blockIdx.x * A2Z + threadIdx.x;
  const int i = blockIdx.y * A2X + threadIdx.y;
  const int nx = p.nx, nz = p.nz;
  if (i >= nx || j >= nz) return;
  const long long idx = (long long)i * nz + j;
  const T dx = p.dx, dz = p.dz, dt = p.dt;
  // quotients by the spacings: the verified constant-divisor route (the
  // forward pass's bits, IEEE division's bits)
  auto qdx = [&](T v) { return div_c(v, dx, p.rd[0], p.fast_div & 1); };
  auto qdz = [&](T v) { return div_c(v, dz, p.rd[1], p.fast_div & 1); };
  T c[N];
#pragma unroll
  for (int m = 0; m < N; ++m) c[m] = p.c[m];
  const Snap2<T> s0 = snap_of(p, a.snap0);
  const T* sxx = s0.f(2);
  const T* szz = s0.f(3);
  const T* sxz = s0.f(4);
  const T* cfx = p.cf[0];
  const T* cfz = p.cf[1];
  const T* rho = p.rho;
  const int xi = slab_index(i, nx, p.lo[0], p.hi[0]);
  const int zj = slab_index(j, nz, p.lo[1], p.hi[1]);
  const uint8_t fx = p.fl[0][i], fz = p.fl[1][j];
  T t0 = 0, t1 = 0, t2 = 0, t3 = 0;
  // vx at (i+1/2, j)
  if (i >= N && i < nx - N - 1 && j >= N + 1 && j < nz - N) {
    T av = qdx(dx_fm<T, N>(sxx, idx, nz, c));
    T bv = qdz(dz_bm<T, N>(sxz, idx, c));
    const bool P = (fx & 2) || (fz & 1);
    const T bxh = cfx[CBH * nx + i], axh = cfx[CAH * nx + i], kxh = cfx[CKH * nx + i];
    const T bz = cfz[CB * nz + j], az = cfz[CA * nz + j], kz = cfz[CK * nz + j];
    if (P && xi >= 0) av = pml_fwd(av, s0.mx(0, xi, j), bxh, axh, kxh);
    if (P && zj >= 0) bv = pml_fwd(bv, s0.mz(0, i, zj), bz, az, kz);
    const T vb = a.f[0][idx];
    a.grad[0][idx] += vb * (av + bv) * dt;
    const T rh = (rho[idx] + rho[idx + nz]) / (T)2;
    T sb = vb * dt / rh;
    T ab = sb, bb = sb;
    if (P && xi >= 0) ab = pml_adj(ab, amx(p, a, 0, xi, j), bxh, axh, kxh);
    if (P && zj >= 0) bb = pml_adj(bb, amz(p, a, 0, i, zj), bz, az, kz);
    t0 = qdx(ab);
    t1 = qdz(bb);
  }
  // vz at (i, j+1/2)
  if (i >= N + 1 && i < nx - N && j >= N && j < nz - N - 1) {
    T av = qdx(dx_bm<T, N>(sxz, idx, nz, c));
    T bv = qdz(dz_fm<T, N>(szz, idx, c));
    const bool P = (fx & 1) || (fz & 2);
    const T bx = cfx[CB * nx + i], ax = cfx[CA * nx + i], kx = cfx[CK * nx + i];
    const T bzh = cfz[CBH * nz + j], azh = cfz[CAH * nz + j], kzh = cfz[CKH * nz + j];
    if (P && xi >= 0) av = pml_fwd(av, s0.mx(1, xi, j), bx, ax, kx);
    if (P && zj >= 0) bv = pml_fwd(bv, s0.mz(1, i, zj), bzh, azh, kzh);
    const T vb = a.f[1][idx];
    a.grad[1][idx] += vb * (av + bv) * dt;
    const T rh = (T)0.5 * (rho[idx] + rho[idx + 1]);
    T sb = vb * dt / rh;
    T ab = sb, bb = sb;
    if (P && xi >= 0) ab = pml_adj(ab, amx(p, a, 1, xi, j), bx, ax, kx);
    if (P && zj >= 0) bb = pml_adj(bb, amz(p, a, 1, i, zj), bzh, azh, kzh);
    t2 = qdx(ab);
    t3 = qdz(bb);
  }
  a.tmp[0][idx] = t0;
  a.tmp[1][idx] = t1;
  a.tmp[2][idx] = t2;
  a.tmp[3][idx] = t3;
}

// sxx_bar += Dfx^T t0;  sxz_bar += Dbz^T t1 + Dbx^T t2;  szz_bar += Dfz^T t3
template <typename T, int N>
__global__ void __launch_bounds__(A2Z * A2X, SW_ADJ_MINB)
k2a_sv_str_gather(const __grid_constant__ P2<T> p, const __grid_constant__ A2<T> a) {
  const int j = blockIdx.x * A2Z + threadIdx.x;
  const int i = blockIdx.y * A2X + threadIdx.y;
  const int nx = p.nx, nz = p.nz;
  if (i >= nx || j >= nz) return;
  const long long idx = (long long)i * nz + j;
  T gxx = 0, gxz = 0, gzz = 0;
#pragma unroll
  for (int m = 0; m < N; ++m) {
    const T c = p.c[m];
    gxx += c * (at(a.tmp[0], i - m - 1, j, nx, nz) - at(a.tmp[0], i + m, j, nx, nz));
    gxz += c * (at(a.tmp[1], i, j - m, nx, nz) - at(a.tmp[1], i, j + m + 1, nx, nz));
    gxz += c * (at(a.tmp[2], i - m, j, nx, nz) - at(a.tmp[2], i + m + 1, j, nx, nz));
    gzz += c * (at(a.tmp[3], i, j - m - 1, nx, nz) - at(a.tmp[3], i, j + m, nx, nz));
  }
  a.f[2][idx] += gxx;
  a.f[3][idx] += gzz;
  a.f[4][idx] += gxz;
}

// ---- host side ----------------------------------------------------------------
template <typename T, int N>
static cudaError_t adj_step(const P2<T>& p, const A2<T>& a, int scheme, int it, cudaStream_t st) {
  dim3 block(A2Z, A2X);
  dim3 grid((p.nz + A2Z - 1) / A2Z, (p.nx + A2X - 1) / A2X);
  if (p.nrec > 0) k2a_record<T><<<(p.nrec + 255) / 256, 256, 0, st>>>(p, a, it);
  if (scheme == SW2D_SSG_SV) {
    k2a_sv_stress_mid<T, N><<<grid, block, 0, st>>>(p, a);
    k2a_sv_vel_gather<T, N><<<grid, block, 0, st>>>(p, a);
    k2a_sv_vel_mid<T, N><<<grid, block, 0, st>>>(p, a);
    k2a_sv_str_gather<T, N><<<grid, block, 0, st>>>(p, a);
  } else {
    k2a_stress_mid<T, N><<<grid, block, 0, st>>>(p, a);
    k2a_vel_gather<T, N><<<grid, block, 0, st>>>(p, a);
    k2a_vel_mid<T, N><<<grid, block, 0, st>>>(p, a);
    k2a_str_gather<T, N><<<grid, block, 0, st>>>(p, a);
  }
  return cudaGetLastError();
}

// one adjoint step of the 2D SSG_VS or SSG_SV scheme
template <typename T>
cudaError_t sw2_adjoint_step(const P2<T>& p, const A2<T>& a, int scheme, int order, int it, cudaStream_t st) {
  switch (order) {
    case 1: return adj_step<T, 1>(p, a, scheme, it, st);
    case 2: return adj_step<T, 2>(p, a, scheme, it, st);
    case 3: return adj_step<T, 3>(p, a, scheme, it, st);
    case 4: return adj_step<T, 4>(p, a, scheme, it, st);
    case 5: return adj_step<T, 5>(p, a, scheme, it, st);
    case 6: return adj_step<T, 6>(p, a, scheme, it, st);
    case 7: return adj_step<T, 7>(p, a, scheme, it, st);
    case 8: return adj_step<T, 8>(p, a, scheme, it, st);
    default: return cudaErrorInvalidValue;
  }
}

template cudaError_t sw2_adjoint_step<float>(const P2<float>&, const A2<float>&, int, int, int, cudaStream_t);
template cudaError_t sw2_adjoint_step<double>(const P2<double>&, const A2<double>&, int, int, int, cudaStream_t);

}  // namespace sw
