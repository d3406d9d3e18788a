// sw_oracle.cpp -- CPU restatement of SeisWave_Taichi's elastic staggered-grid
// finite-difference time loop.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path: it is
// linked by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline
// leg, and by nothing else.  The product never calls it.
//
// It restates, loop by loop and expression by expression, the Taichi kernels of
// the reference (paths relative to the reference project):
//   src/Elastic2D_CPML.py        update_SSG_VS 128-200, update_SSG_SV 203-274,
//                                update_RSG 277-353, diff_coff 355-366,
//                                SetADEPML2D 392-528, AEA_init/AEA 113-125
//   src/Elastic3D_SSG_CPML.py    update_SSG 144-309 (point force)
//   src/Elastic3D_SSG_Tensor.py  update_SSG 166-345 (moment tensor)
//   src/Elastic3D_SSG_SPML.py    update_SSG_SPML 160-393 (split-field PML)
//   src/Differential2D.py 4-56, src/Differential3D.py 7-44 (stencils)
//   src/BaseFun.py 4-27 (wavelets)
// Every wavefield and every CPML memory variable is a full-grid array, as in
// the reference.  Phases run in source order; each phase is a pure map, so the
// OpenMP loops inside a phase are order-independent.  Arithmetic follows the
// reference's per-line operation order with true divisions; the build recipe
// (oracle/Makefile) disables floating-point contraction so each operation
// rounds on its own.
//
// Parity unpinned: the reference ships no golden vectors or known-answer
// tests and Taichi cannot run here, so no output of the reference itself
// checks this restatement.  It is held instead by closed-form coefficient
// values, an independent numpy twin (oracle/np_twin.py, bit for bit) and
// physics checks (arrival times, symmetry, reciprocity, convergence, CPML
// reflection energy) in tests/test_oracle.py.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <vector>

#if defined(_OPENMP)
#include <omp.h>
#endif

extern "C" {

// ---------------------------------------------------------------------------
// Descriptors (mirrored by oracle/oracle.py through ctypes)
// ---------------------------------------------------------------------------
struct OAxis {
  // ten profile arrays of the reference's SetADEPML*: integer and half points
  void* pml; void* pml_half; void* alpha; void* alpha_half; void* k; void* k_half;
  void* b; void* b_half; void* a; void* a_half;
  double pml_min, pml_max;   // xmin_pml / xmax_pml (physical coordinates)
};

struct O2Desc {
  int32_t nx, nz, N, dtype;       // dtype 0: float, 1: double
  double dx, dz, dt;
  double c[16];
  void *vx, *vz, *sxx, *szz, *sxz;
  void *rho, *lam, *mu;
  // memory variables, full grid, reference names:
  // 0 sxx_dx 1 sxx_dz 2 sxz_dx 3 sxz_dz 4 szz_dx 5 szz_dz
  // 6 dvx_dx 7 dvx_dz 8 dvz_dx 9 dvz_dz
  void* mem[10];
  OAxis ax[2];
  int32_t isx, isz, rsx, rsz;
  double f0;
  const float* wavelet;           // per-step source value (float), or null
  void* data;                     // receiver trace, length >= it (dtype)
  // moment-tensor source and receiver arrays (no reference counterpart; they
  // follow Elastic3D_SSG_Tensor.py's conventions in two dimensions)
  int32_t src_kind;               // 0: the scheme's point force, 1: moment tensor
  int32_t nrec;                   // 0: one receiver (rsx, rsz); else rec_idx[nrec]
  double mt[3];                   // xx zz xz
  const int64_t* rec_idx;         // linear cell indices; data is (nt, nrec)
};

struct O3Desc {
  int32_t nx, ny, nz, N, dtype, scheme;   // scheme 0 CPML force, 1 tensor, 2 SPML
  double dx, dy, dz, dt;
  double c[16];
  void *vx, *vy, *vz, *sxx, *syy, *szz, *sxy, *sxz, *syz;
  void *rho, *lam, *mu;
  // CPML: 18 memory variables (order below); SPML: 24 split fields
  void* mem[24];
  OAxis ax[3];
  int32_t isx, isy, isz;
  double f0, src_scale, t0;
  double mt[6];                   // xx yy zz xy xz yz
  const float* wavelet;           // per-step source value (float), or null
  int32_t nrec;
  const int32_t *rx, *ry, *rz;
  void* data;                     // float: (nt, nrec) for tensor, (nt,) otherwise
};

}  // extern "C"

namespace {

// Wavelets of src/BaseFun.py, in float as the reference's @ti.func returns ti.f32.
// `pi**2` there is an expression of Python values only, which Taichi's
// frontend folds in double before it meets the float arithmetic, so the
// constant is (float)(pi*pi in double), not pi_f * pi_f.
constexpr double kPiD = 3.14159265358979323846;
// BaseFun.py:4-11
float ricker(int it, float dt, float freq, float scale) {
  const float pi2 = (float)(kPiD * kPiD);
  float t0 = 1.5f / freq;
  float a = pi2 * (freq * freq);
  float t = (float)it * dt;
  float tau = t - t0;
  return ((((-scale) * 2.0f) * a) * tau) * std::exp((-a) * (tau * tau));
}
// BaseFun.py:13-19
float ricker2(int it, float dt, float t0, float freq, float scale) {
  const float pi2 = (float)(kPiD * kPiD);
  float a = pi2 * (freq * freq);
  float t = (float)it * dt;
  float tau = t - t0;
  return (scale * (1.0f - (2.0f * a) * (tau * tau))) * std::exp((-a) * (tau * tau));
}
// BaseFun.py:21-27
float ricker3(int it, float dt, float t0, float freq, float scale) {
  const float pi = 3.14159265358979323846f;
  float ts = 1.0f / freq;
  float t = (float)it * dt;
  float tau = pi * ((t - 1.5f * ts) - t0) / ts;
  return (scale * (1.0f - 2.0f * (tau * tau))) * std::exp(-(tau * tau));
}

template <typename T>
struct G2 {
  T* p; int nz;
  T& operator()(int i, int j) const { return p[(size_t)i * nz + j]; }
};
template <typename T>
struct G3 {
  T* p; int ny, nz;
  T& operator()(int i, int j, int k) const { return p[((size_t)i * ny + j) * nz + k]; }
};

// ---- src/Differential2D.py ------------------------------------------------
template <typename T> inline T Dx2fm(const G2<T>& f, int i, int j, const T* c, int n) {
  T v = 0; for (int m = 0; m < n; ++m) v += c[m] * (f(i + m + 1, j) - f(i - m, j)); return v; }
template <typename T> inline T Dz2fm(const G2<T>& f, int i, int j, const T* c, int n) {
  T v = 0; for (int m = 0; m < n; ++m) v += c[m] * (f(i, j + m + 1) - f(i, j - m)); return v; }
template <typename T> inline T Dx2bm(const G2<T>& f, int i, int j, const T* c, int n) {
  T v = 0; for (int m = 0; m < n; ++m) v += c[m] * (f(i + m, j) - f(i - m - 1, j)); return v; }
template <typename T> inline T Dz2bm(const G2<T>& f, int i, int j, const T* c, int n) {
  T v = 0; for (int m = 0; m < n; ++m) v += c[m] * (f(i, j + m) - f(i, j - m - 1)); return v; }
template <typename T> inline T Drx2fm(const G2<T>& f, int i, int j, const T* c, int n) {
  T v = 0; for (int m = 0; m < n; ++m) v += c[m] * (f(i + m + 1, j + m + 1) - f(i - m, j - m)); return v; }
template <typename T> inline T Drz2fm(const G2<T>& f, int i, int j, const T* c, int n) {
  T v = 0; for (int m = 0; m < n; ++m) v += c[m] * (f(i - m, j + m + 1) - f(i + m + 1, j - m)); return v; }
template <typename T> inline T Drx2bm(const G2<T>& f, int i, int j, const T* c, int n) {
  T v = 0; for (int m = 0; m < n; ++m) v += c[m] * (f(i + m, j + m) - f(i - m - 1, j - m - 1)); return v; }
template <typename T> inline T Drz2bm(const G2<T>& f, int i, int j, const T* c, int n) {
  T v = 0; for (int m = 0; m < n; ++m) v += c[m] * (f(i - m - 1, j + m) - f(i + m, j - m - 1)); return v; }

// ---- src/Differential3D.py ------------------------------------------------
template <typename T> inline T Dx3fm(const G3<T>& f, int i, int j, int k, const T* c, int n) {
  T v = 0; for (int m = 0; m < n; ++m) v += c[m] * (f(i + m + 1, j, k) - f(i - m, j, k)); return v; }
template <typename T> inline T Dy3fm(const G3<T>& f, int i, int j, int k, const T* c, int n) {
  T v = 0; for (int m = 0; m < n; ++m) v += c[m] * (f(i, j + m + 1, k) - f(i, j - m, k)); return v; }
template <typename T> inline T Dz3fm(const G3<T>& f, int i, int j, int k, const T* c, int n) {
  T v = 0; for (int m = 0; m < n; ++m) v += c[m] * (f(i, j, k + m + 1) - f(i, j, k - m)); return v; }
template <typename T> inline T Dx3bm(const G3<T>& f, int i, int j, int k, const T* c, int n) {
  T v = 0; for (int m = 0; m < n; ++m) v += c[m] * (f(i + m, j, k) - f(i - m - 1, j, k)); return v; }
template <typename T> inline T Dy3bm(const G3<T>& f, int i, int j, int k, const T* c, int n) {
  T v = 0; for (int m = 0; m < n; ++m) v += c[m] * (f(i, j + m, k) - f(i, j - m - 1, k)); return v; }
template <typename T> inline T Dz3bm(const G3<T>& f, int i, int j, int k, const T* c, int n) {
  T v = 0; for (int m = 0; m < n; ++m) v += c[m] * (f(i, j, k + m) - f(i, j, k - m - 1)); return v; }

template <typename T>
struct Ax {
  const T *pml, *pml_half, *alpha, *alpha_half, *k, *k_half, *b, *b_half, *a, *a_half;
  T lo, hi;
  explicit Ax(const OAxis& o)
      : pml((const T*)o.pml), pml_half((const T*)o.pml_half), alpha((const T*)o.alpha),
        alpha_half((const T*)o.alpha_half), k((const T*)o.k), k_half((const T*)o.k_half),
        b((const T*)o.b), b_half((const T*)o.b_half), a((const T*)o.a), a_half((const T*)o.a_half),
        lo((T)o.pml_min), hi((T)o.pml_max) {}
  bool in(T x) const { return x <= lo || x >= hi; }
};

// =========================================================================
// 2D  (src/Elastic2D_CPML.py)
// =========================================================================
template <typename T>
struct S2 {
  int nx, nz, N;
  T dx, dz, dt;
  T c[16];
  G2<T> vx, vz, sxx, szz, sxz, rho, lam, mu;
  G2<T> m_sxx_dx, m_sxz_dx, m_sxz_dz, m_szz_dz, m_dvx_dx, m_dvx_dz, m_dvz_dx, m_dvz_dz;
  Ax<T> X, Z;
  explicit S2(const O2Desc& d)
      : nx(d.nx), nz(d.nz), N(d.N), dx((T)d.dx), dz((T)d.dz), dt((T)d.dt),
        vx{(T*)d.vx, d.nz}, vz{(T*)d.vz, d.nz}, sxx{(T*)d.sxx, d.nz}, szz{(T*)d.szz, d.nz},
        sxz{(T*)d.sxz, d.nz}, rho{(T*)d.rho, d.nz}, lam{(T*)d.lam, d.nz}, mu{(T*)d.mu, d.nz},
        m_sxx_dx{(T*)d.mem[0], d.nz}, m_sxz_dx{(T*)d.mem[2], d.nz}, m_sxz_dz{(T*)d.mem[3], d.nz},
        m_szz_dz{(T*)d.mem[5], d.nz}, m_dvx_dx{(T*)d.mem[6], d.nz}, m_dvx_dz{(T*)d.mem[7], d.nz},
        m_dvz_dx{(T*)d.mem[8], d.nz}, m_dvz_dz{(T*)d.mem[9], d.nz}, X(d.ax[0]), Z(d.ax[1]) {
    for (int m = 0; m < 16; ++m) c[m] = (T)d.c[m];
  }
};

// 2D moment-tensor source at the start of the step, in the convention of
// Elastic3D_SSG_Tensor.py:186-193: sigma_ab[src] += w * (-M_ab)
template <typename T>
void inject2d_moment(const O2Desc& d, S2<T>& s, int it) {
  const T w = (T)d.wavelet[it];
  s.sxx(d.isx, d.isz) += w * (-(T)(float)d.mt[0]);
  s.szz(d.isx, d.isz) += w * (-(T)(float)d.mt[1]);
  s.sxz(d.isx, d.isz) += w * (-(T)(float)d.mt[2]);
}

// receivers after the stress phase: one cell (rsx, rsz) or a table
template <typename T>
void record2d(const O2Desc& d, const G2<T>& f, int it) {
  if (!d.data) return;
  if (d.nrec <= 0) {
    ((T*)d.data)[it] = f(d.rsx, d.rsz);
    return;
  }
  for (int r = 0; r < d.nrec; ++r) ((T*)d.data)[(long long)it * d.nrec + r] = f.p[d.rec_idx[r]];
}

// Elastic2D_CPML.py:128-200
template <typename T>
void step2d_vs(const O2Desc& d, int it) {
  S2<T> s(d);
  const int N = s.N, nx = s.nx, nz = s.nz;
  const T dx = s.dx, dz = s.dz, dt = s.dt;
  if (d.src_kind == 1) inject2d_moment(d, s, it);
  // update vx  :144-154
#pragma omp parallel for
  for (int i = N + 1; i < nx - N; ++i)
    for (int j = N + 1; j < nz - N; ++j) {
      T x = (T)(i - N) * dx, z = (T)(j - N) * dz;
      T dsxxdx = Dx2bm(s.sxx, i, j, s.c, N) / dx;
      T dsxzdz = Dz2bm(s.sxz, i, j, s.c, N) / dz;
      if (s.X.in(x) || s.Z.in(z)) {
        s.m_sxx_dx(i, j) = s.X.b[i] * s.m_sxx_dx(i, j) + s.X.a[i] * dsxxdx;
        s.m_sxz_dz(i, j) = s.Z.b[j] * s.m_sxz_dz(i, j) + s.Z.a[j] * dsxzdz;
        dsxxdx = dsxxdx / s.X.k[i] + s.m_sxx_dx(i, j);
        dsxzdz = dsxzdz / s.Z.k[j] + s.m_sxz_dz(i, j);
      }
      s.vx(i, j) += (dsxxdx + dsxzdz) * dt / s.rho(i, j);
    }
  // update vz  :156-167
#pragma omp parallel for
  for (int i = N; i < nx - N - 1; ++i)
    for (int j = N; j < nz - N - 1; ++j) {
      T x = (T)(i - N) * dx + dx / (T)2, z = (T)(j - N) * dz + dz / (T)2;
      T rh = (T)0.25 * (s.rho(i, j) + s.rho(i, j + 1) + s.rho(i + 1, j + 1) + s.rho(i + 1, j));
      T dsxzdx = Dx2fm(s.sxz, i, j, s.c, N) / dx;
      T dszzdz = Dz2fm(s.szz, i, j, s.c, N) / dz;
      if (s.X.in(x) || s.Z.in(z)) {
        s.m_sxz_dx(i, j) = s.X.b_half[i] * s.m_sxz_dx(i, j) + s.X.a_half[i] * dsxzdx;
        s.m_szz_dz(i, j) = s.Z.b_half[j] * s.m_szz_dz(i, j) + s.Z.a_half[j] * dszzdz;
        dsxzdx = dsxzdx / s.X.k_half[i] + s.m_sxz_dx(i, j);
        dszzdz = dszzdz / s.Z.k_half[j] + s.m_szz_dz(i, j);
      }
      s.vz(i, j) += (dszzdz + dsxzdx) * dt / rh;
    }
  // source :170
  if (d.src_kind == 0) {
    float f0 = (float)d.f0;
    float w = d.wavelet ? d.wavelet[it] : ricker2(it, (float)d.dt, 1.5f / f0, f0, 1.0f);
    s.vz(d.isx, d.isz) += dt * (T)w / s.rho(d.isx, d.isz);
  }
  // update sxx szz :172-186
#pragma omp parallel for
  for (int i = N; i < nx - N - 1; ++i)
    for (int j = N + 1; j < nz - N; ++j) {
      T x = (T)(i - N) * dx + dx / (T)2, z = (T)(j - N) * dz;
      T lhx = (T)0.5 * (s.lam(i, j) + s.lam(i + 1, j));
      T mhx = (T)0.5 * (s.mu(i, j) + s.mu(i + 1, j));
      T lpm = lhx + (T)2 * mhx;
      T dvxdx = Dx2fm(s.vx, i, j, s.c, N) / dx;
      T dvzdz = Dz2bm(s.vz, i, j, s.c, N) / dz;
      if (s.X.in(x) || s.Z.in(z)) {
        s.m_dvx_dx(i, j) = s.X.b_half[i] * s.m_dvx_dx(i, j) + s.X.a_half[i] * dvxdx;
        s.m_dvz_dz(i, j) = s.Z.b[j] * s.m_dvz_dz(i, j) + s.Z.a[j] * dvzdz;
        dvxdx = dvxdx / s.X.k_half[i] + s.m_dvx_dx(i, j);
        dvzdz = dvzdz / s.Z.k[j] + s.m_dvz_dz(i, j);
      }
      s.sxx(i, j) += (lpm * dvxdx + lhx * dvzdz) * dt;
      s.szz(i, j) += (lpm * dvzdz + lhx * dvxdx) * dt;
    }
  // update sxz :188-199
#pragma omp parallel for
  for (int i = N + 1; i < nx - N; ++i)
    for (int j = N; j < nz - N - 1; ++j) {
      T x = (T)(i - N) * dx, z = (T)(j - N) * dz + dz / (T)2;
      T mhz = (T)0.5 * (s.mu(i, j + 1) + s.mu(i, j));
      T dvzdx = Dx2bm(s.vz, i, j, s.c, N) / dx;
      T dvxdz = Dz2fm(s.vx, i, j, s.c, N) / dz;
      if (s.X.in(x) || s.Z.in(z)) {
        s.m_dvz_dx(i, j) = s.X.b[i] * s.m_dvz_dx(i, j) + s.X.a[i] * dvzdx;
        s.m_dvx_dz(i, j) = s.Z.b_half[j] * s.m_dvx_dz(i, j) + s.Z.a_half[j] * dvxdz;
        dvzdx = dvzdx / s.X.k[i] + s.m_dvz_dx(i, j);
        dvxdz = dvxdz / s.Z.k_half[j] + s.m_dvx_dz(i, j);
      }
      s.sxz(i, j) += mhz * (dvxdz + dvzdx) * dt;
    }
  // receiver :200
  record2d(d, s.vz, it);
}

// Elastic2D_CPML.py:203-274
template <typename T>
void step2d_sv(const O2Desc& d, int it) {
  S2<T> s(d);
  const int N = s.N, nx = s.nx, nz = s.nz;
  const T dx = s.dx, dz = s.dz, dt = s.dt;
  if (d.src_kind == 1) inject2d_moment(d, s, it);
  // vx :218-229
#pragma omp parallel for
  for (int i = N; i < nx - N - 1; ++i)
    for (int j = N + 1; j < nz - N; ++j) {
      T x = (T)(i - N) * dx + dx / (T)2, z = (T)(j - N) * dz;
      T dsxxdx = Dx2fm(s.sxx, i, j, s.c, N) / dx;
      T dsxzdz = Dz2bm(s.sxz, i, j, s.c, N) / dz;
      T rhx = (s.rho(i, j) + s.rho(i + 1, j)) / (T)2;
      if (s.X.in(x) || s.Z.in(z)) {
        s.m_sxx_dx(i, j) = s.X.b_half[i] * s.m_sxx_dx(i, j) + s.X.a_half[i] * dsxxdx;
        s.m_sxz_dz(i, j) = s.Z.b[j] * s.m_sxz_dz(i, j) + s.Z.a[j] * dsxzdz;
        dsxxdx = dsxxdx / s.X.k_half[i] + s.m_sxx_dx(i, j);
        dsxzdz = dsxzdz / s.Z.k[j] + s.m_sxz_dz(i, j);
      }
      s.vx(i, j) += (dsxxdx + dsxzdz) * dt / rhx;
    }
  // vz :231-242
#pragma omp parallel for
  for (int i = N + 1; i < nx - N; ++i)
    for (int j = N; j < nz - N - 1; ++j) {
      T x = (T)(i - N) * dx, z = (T)(j - N) * dz + dz / (T)2;
      T rhz = (T)0.5 * (s.rho(i, j) + s.rho(i, j + 1));
      T dsxzdx = Dx2bm(s.sxz, i, j, s.c, N) / dx;
      T dszzdz = Dz2fm(s.szz, i, j, s.c, N) / dz;
      if (s.X.in(x) || s.Z.in(z)) {
        s.m_sxz_dx(i, j) = s.X.b[i] * s.m_sxz_dx(i, j) + s.X.a[i] * dsxzdx;
        s.m_szz_dz(i, j) = s.Z.b_half[j] * s.m_szz_dz(i, j) + s.Z.a_half[j] * dszzdz;
        dsxzdx = dsxzdx / s.X.k[i] + s.m_sxz_dx(i, j);
        dszzdz = dszzdz / s.Z.k_half[j] + s.m_szz_dz(i, j);
      }
      s.vz(i, j) += (dszzdz + dsxzdx) * dt / rhz;
    }
  // source :245
  if (d.src_kind == 0) {
    float w = d.wavelet ? d.wavelet[it] : ricker(it, (float)d.dt, (float)d.f0, 1.0f);
    s.vx(d.isx, d.isz) += dt * (T)w / s.rho(d.isx, d.isz);
  }
  // sxx szz :247-260
#pragma omp parallel for
  for (int i = N + 1; i < nx - N; ++i)
    for (int j = N + 1; j < nz - N; ++j) {
      T x = (T)(i - N) * dx, z = (T)(j - N) * dz;
      T lam = s.lam(i, j);
      T lpm = s.lam(i, j) + (T)2 * s.mu(i, j);
      T dvxdx = Dx2bm(s.vx, i, j, s.c, N) / dx;
      T dvzdz = Dz2bm(s.vz, i, j, s.c, N) / dz;
      if (s.X.in(x) || s.Z.in(z)) {
        s.m_dvx_dx(i, j) = s.X.b[i] * s.m_dvx_dx(i, j) + s.X.a[i] * dvxdx;
        s.m_dvz_dz(i, j) = s.Z.b[j] * s.m_dvz_dz(i, j) + s.Z.a[j] * dvzdz;
        dvxdx = dvxdx / s.X.k[i] + s.m_dvx_dx(i, j);
        dvzdz = dvzdz / s.Z.k[j] + s.m_dvz_dz(i, j);
      }
      s.sxx(i, j) += (lpm * dvxdx + lam * dvzdz) * dt;
      s.szz(i, j) += (lpm * dvzdz + lam * dvxdx) * dt;
    }
  // sxz :262-273
#pragma omp parallel for
  for (int i = N + 1; i < nx - N; ++i)
    for (int j = N + 1; j < nz - N; ++j) {
      T x = (T)(i - N) * dx + dx / (T)2, z = (T)(j - N) * dz + dz / (T)2;
      T m4 = (T)0.25 * (s.mu(i, j + 1) + s.mu(i, j) + s.mu(i + 1, j + 1) + s.mu(i + 1, j));
      T dvzdx = Dx2fm(s.vz, i, j, s.c, N) / dx;
      T dvxdz = Dz2fm(s.vx, i, j, s.c, N) / dz;
      if (s.X.in(x) || s.Z.in(z)) {
        s.m_dvz_dx(i, j) = s.X.b_half[i] * s.m_dvz_dx(i, j) + s.X.a_half[i] * dvzdx;
        s.m_dvx_dz(i, j) = s.Z.b_half[j] * s.m_dvx_dz(i, j) + s.Z.a_half[j] * dvxdz;
        dvzdx = dvzdx / s.X.k_half[i] + s.m_dvz_dx(i, j);
        dvxdz = dvxdz / s.Z.k_half[j] + s.m_dvx_dz(i, j);
      }
      s.sxz(i, j) += m4 * (dvxdz + dvzdx) * dt;
    }
  record2d(d, s.vx, it);
}

// Elastic2D_CPML.py:277-353 (source value passed by the caller)
template <typename T>
void step2d_rsg(const O2Desc& d, int it, double source) {
  S2<T> s(d);
  const int N = s.N, nx = s.nx, nz = s.nz;
  const T dx = s.dx, dz = s.dz, dt = s.dt;
  G2<T> m_szz_dz = s.m_szz_dz;
#pragma omp parallel for
  for (int i = N + 1; i < nx - N; ++i)
    for (int j = N + 1; j < nz - N; ++j) {
      T x = (T)(i - N) * dx, z = (T)(j - N) * dz;
      T dsxxrx = Drx2bm(s.sxx, i, j, s.c, N), dsxxrz = Drz2bm(s.sxx, i, j, s.c, N);
      T dszzrx = Drx2bm(s.szz, i, j, s.c, N), dszzrz = Drz2bm(s.szz, i, j, s.c, N);
      T dsxzrx = Drx2bm(s.sxz, i, j, s.c, N), dsxzrz = Drz2bm(s.sxz, i, j, s.c, N);
      T dsxxdx = (dsxxrz - dsxxrx) / ((T)2 * dx);
      T dszzdz = (dszzrz + dszzrx) / ((T)2 * dz);
      T dsxzdx = (dsxzrz - dsxzrx) / ((T)2 * dx);
      T dsxzdz = (dsxzrz + dsxzrx) / ((T)2 * dz);
      T rho = s.rho(i, j);
      if (s.X.in(x) || s.Z.in(z)) {
        s.m_sxx_dx(i, j) = s.X.b[i] * s.m_sxx_dx(i, j) + s.X.a[i] * dsxxdx;
        m_szz_dz(i, j) = s.Z.b[j] * m_szz_dz(i, j) + s.Z.a[j] * dszzdz;
        s.m_sxz_dx(i, j) = s.X.b[i] * s.m_sxz_dx(i, j) + s.X.a[i] * dsxzdx;
        s.m_sxz_dz(i, j) = s.Z.b[j] * s.m_sxz_dz(i, j) + s.Z.a[j] * dsxzdz;
        dsxxdx = dsxxdx / s.X.k[i] + s.m_sxx_dx(i, j);
        dszzdz = dszzdz / s.Z.k[j] + m_szz_dz(i, j);
        dsxzdx = dsxzdx / s.X.k[i] + s.m_sxz_dx(i, j);
        dsxzdz = dsxzdz / s.Z.k[j] + s.m_sxz_dz(i, j);
      }
      s.vx(i, j) += (dsxxdx + dsxzdz) * dt / rho;
      s.vz(i, j) += (dszzdz + dsxzdx) * dt / rho;
    }
  // 2x2 source spread :322-323 (source is ti.f32)
  {
    T src = (T)(float)source;
    for (int a = -1; a < 1; ++a)
      for (int b = -1; b < 1; ++b)
        s.vz(d.isx + a, d.isz + b) += dt * src / ((T)8 * s.rho(d.isx + a, d.isz + b));
  }
#pragma omp parallel for
  for (int i = N; i < nx - N - 1; ++i)
    for (int j = N; j < nz - N - 1; ++j) {
      T x = (T)(i - N) * dx + dx / (T)2, z = (T)(j - N) * dz + dz / (T)2;
      T lam = s.lam(i, j), mu = s.mu(i, j);
      T lpm = lam + (T)2 * mu;
      T dvxrx = Drx2fm(s.vx, i, j, s.c, N), dvxrz = Drz2fm(s.vx, i, j, s.c, N);
      T dvzrx = Drx2fm(s.vz, i, j, s.c, N), dvzrz = Drz2fm(s.vz, i, j, s.c, N);
      T dvxdx = (dvxrz - dvxrx) / ((T)2 * dx);
      T dvxdz = (dvxrz + dvxrx) / ((T)2 * dz);
      T dvzdx = (dvzrz - dvzrx) / ((T)2 * dx);
      T dvzdz = (dvzrz + dvzrx) / ((T)2 * dz);
      if (s.X.in(x) || s.Z.in(z)) {
        s.m_dvx_dx(i, j) = s.X.b_half[i] * s.m_dvx_dx(i, j) + s.X.a_half[i] * dvxdx;
        s.m_dvx_dz(i, j) = s.Z.b_half[j] * s.m_dvx_dz(i, j) + s.Z.a_half[j] * dvxdz;
        s.m_dvz_dx(i, j) = s.X.b_half[i] * s.m_dvz_dx(i, j) + s.X.a_half[i] * dvzdx;
        s.m_dvz_dz(i, j) = s.Z.b_half[j] * s.m_dvz_dz(i, j) + s.Z.a_half[j] * dvzdz;
        dvxdx = dvxdx / s.X.k_half[i] + s.m_dvx_dx(i, j);
        dvxdz = dvxdz / s.Z.k_half[j] + s.m_dvx_dz(i, j);
        dvzdx = dvzdx / s.X.k_half[i] + s.m_dvz_dx(i, j);
        dvzdz = dvzdz / s.Z.k_half[j] + s.m_dvz_dz(i, j);
      }
      s.sxx(i, j) += (lpm * dvxdx + lam * dvzdz) * dt;
      s.szz(i, j) += (lpm * dvzdz + lam * dvxdx) * dt;
      s.sxz(i, j) += (mu * (dvxdz + dvzdx)) * dt;
    }
  (void)it;
}

// =========================================================================
// 3D  (src/Elastic3D_SSG_CPML.py, src/Elastic3D_SSG_Tensor.py)
// =========================================================================
template <typename T>
struct S3 {
  int nx, ny, nz, N;
  T dx, dy, dz, dt;
  T c[16];
  G3<T> vx, vy, vz, sxx, syy, szz, sxy, sxz, syz, rho, lam, mu;
  G3<T> m[24];
  Ax<T> X, Y, Z;
  explicit S3(const O3Desc& d)
      : nx(d.nx), ny(d.ny), nz(d.nz), N(d.N), dx((T)d.dx), dy((T)d.dy), dz((T)d.dz), dt((T)d.dt),
        vx{(T*)d.vx, d.ny, d.nz}, vy{(T*)d.vy, d.ny, d.nz}, vz{(T*)d.vz, d.ny, d.nz},
        sxx{(T*)d.sxx, d.ny, d.nz}, syy{(T*)d.syy, d.ny, d.nz}, szz{(T*)d.szz, d.ny, d.nz},
        sxy{(T*)d.sxy, d.ny, d.nz}, sxz{(T*)d.sxz, d.ny, d.nz}, syz{(T*)d.syz, d.ny, d.nz},
        rho{(T*)d.rho, d.ny, d.nz}, lam{(T*)d.lam, d.ny, d.nz}, mu{(T*)d.mu, d.ny, d.nz},
        X(d.ax[0]), Y(d.ax[1]), Z(d.ax[2]) {
    for (int q = 0; q < 24; ++q) m[q] = G3<T>{(T*)d.mem[q], d.ny, d.nz};
    for (int q = 0; q < 16; ++q) c[q] = (T)d.c[q];
  }
  bool in(T x, T y, T z) const { return X.in(x) || Y.in(y) || Z.in(z); }
};

// CPML memory-variable order used by the 3D descriptors (reference names):
enum {
  M_SXX_DX = 0, M_SXY_DY, M_SXZ_DZ,      // vx  phase
  M_SXY_DX, M_SYY_DY, M_SYZ_DZ,          // vy  phase
  M_SXZ_DX, M_SYZ_DY, M_SZZ_DZ,          // vz  phase
  M_DVX_DX, M_DVY_DY, M_DVZ_DZ,          // normal stresses
  M_DVY_DX, M_DVX_DY,                    // sxy
  M_DVZ_DX, M_DVX_DZ,                    // sxz
  M_DVZ_DY, M_DVY_DZ                     // syz
};

// velocity phase of Elastic3D_SSG_Tensor.py:194-243 and Elastic3D_SSG_CPML.py:163-212.
// `tensor` selects the vz summation order, the only textual difference.
template <typename T>
void velocity3d(S3<T>& s, bool tensor) {
  const int N = s.N, nx = s.nx, ny = s.ny, nz = s.nz;
  const T dx = s.dx, dy = s.dy, dz = s.dz, dt = s.dt;
#pragma omp parallel for collapse(2)
  for (int i = N; i < nx - N - 1; ++i)
    for (int j = N + 1; j < ny - N; ++j)
      for (int k = N + 1; k < nz - N; ++k) {
        T x = (T)(i - N) * dx + dx / (T)2, y = (T)(j - N) * dy, z = (T)(k - N) * dz;
        T dsxxdx = Dx3fm(s.sxx, i, j, k, s.c, N) / dx;
        T dsxydy = Dy3bm(s.sxy, i, j, k, s.c, N) / dy;
        T dsxzdz = Dz3bm(s.sxz, i, j, k, s.c, N) / dz;
        if (s.in(x, y, z)) {
          T& m0 = s.m[M_SXX_DX](i, j, k); T& m1 = s.m[M_SXY_DY](i, j, k); T& m2 = s.m[M_SXZ_DZ](i, j, k);
          m0 = s.X.b_half[i] * m0 + s.X.a_half[i] * dsxxdx;
          m1 = s.Y.b[j] * m1 + s.Y.a[j] * dsxydy;
          m2 = s.Z.b[k] * m2 + s.Z.a[k] * dsxzdz;
          dsxxdx = dsxxdx / s.X.k_half[i] + m0;
          dsxydy = dsxydy / s.Y.k[j] + m1;
          dsxzdz = dsxzdz / s.Z.k[k] + m2;
        }
        s.vx(i, j, k) += (dsxxdx + dsxzdz + dsxydy) * dt / s.rho(i, j, k);
      }
#pragma omp parallel for collapse(2)
  for (int i = N + 1; i < nx - N; ++i)
    for (int j = N; j < ny - N - 1; ++j)
      for (int k = N + 1; k < nz - N; ++k) {
        T x = (T)(i - N) * dx, y = (T)(j - N) * dy + dy / (T)2, z = (T)(k - N) * dz;
        T rhy = (T)0.5 * (s.rho(i, j, k) + s.rho(i, j + 1, k));
        T dsxydx = Dx3bm(s.sxy, i, j, k, s.c, N) / dx;
        T dsyydy = Dy3fm(s.syy, i, j, k, s.c, N) / dy;
        T dsyzdz = Dz3bm(s.syz, i, j, k, s.c, N) / dz;
        if (s.in(x, y, z)) {
          T& m0 = s.m[M_SXY_DX](i, j, k); T& m1 = s.m[M_SYY_DY](i, j, k); T& m2 = s.m[M_SYZ_DZ](i, j, k);
          m0 = s.X.b[i] * m0 + s.X.a[i] * dsxydx;
          m1 = s.Y.b_half[j] * m1 + s.Y.a_half[j] * dsyydy;
          m2 = s.Z.b[k] * m2 + s.Z.a[k] * dsyzdz;
          dsxydx = dsxydx / s.X.k[i] + m0;
          dsyydy = dsyydy / s.Y.k_half[j] + m1;
          dsyzdz = dsyzdz / s.Z.k[k] + m2;
        }
        s.vy(i, j, k) += (dsxydx + dsyydy + dsyzdz) * dt / rhy;
      }
#pragma omp parallel for collapse(2)
  for (int i = N + 1; i < nx - N; ++i)
    for (int j = N + 1; j < ny - N; ++j)
      for (int k = N; k < nz - N - 1; ++k) {
        T x = (T)(i - N) * dx, y = (T)(j - N) * dy, z = (T)(k - N) * dz + dz / (T)2;
        T r4 = (T)0.25 * (s.rho(i, j, k) + s.rho(i, j + 1, k) + s.rho(i + 1, j + 1, k) + s.rho(i + 1, j, k));
        T dsxzdx = Dx3bm(s.sxz, i, j, k, s.c, N) / dx;
        T dsyzdy = Dy3bm(s.syz, i, j, k, s.c, N) / dy;
        T dszzdz = Dz3fm(s.szz, i, j, k, s.c, N) / dz;
        if (s.in(x, y, z)) {
          T& m0 = s.m[M_SXZ_DX](i, j, k); T& m1 = s.m[M_SYZ_DY](i, j, k); T& m2 = s.m[M_SZZ_DZ](i, j, k);
          m0 = s.X.b[i] * m0 + s.X.a[i] * dsxzdx;
          m1 = s.Y.b[j] * m1 + s.Y.a[j] * dsyzdy;
          m2 = s.Z.b_half[k] * m2 + s.Z.a_half[k] * dszzdz;
          dsxzdx = dsxzdx / s.X.k[i] + m0;
          dsyzdy = dsyzdy / s.Y.k[j] + m1;
          dszzdz = dszzdz / s.Z.k_half[k] + m2;
        }
        T sum = tensor ? (dsxzdx + dsyzdy + dszzdz) : (dszzdz + dsxzdx + dsyzdy);
        s.vz(i, j, k) += sum * dt / r4;
      }
}

// stress phase: Elastic3D_SSG_Tensor.py:245-310, Elastic3D_SSG_CPML.py:246-307
template <typename T>
void stress3d(S3<T>& s) {
  const int N = s.N, nx = s.nx, ny = s.ny, nz = s.nz;
  const T dx = s.dx, dy = s.dy, dz = s.dz, dt = s.dt;
#pragma omp parallel for collapse(2)
  for (int i = N + 1; i < nx - N; ++i)
    for (int j = N + 1; j < ny - N; ++j)
      for (int k = N + 1; k < nz - N; ++k) {
        T x = (T)(i - N) * dx, y = (T)(j - N) * dy, z = (T)(k - N) * dz;
        T lhx = (T)0.5 * (s.lam(i, j, k) + s.lam(i + 1, j, k));
        T mhx = (T)0.5 * (s.mu(i, j, k) + s.mu(i + 1, j, k));
        T lpm = lhx + (T)2 * mhx;
        T dvxdx = Dx3bm(s.vx, i, j, k, s.c, N) / dx;
        T dvydy = Dy3bm(s.vy, i, j, k, s.c, N) / dy;
        T dvzdz = Dz3bm(s.vz, i, j, k, s.c, N) / dz;
        if (s.in(x, y, z)) {
          T& m0 = s.m[M_DVX_DX](i, j, k); T& m1 = s.m[M_DVY_DY](i, j, k); T& m2 = s.m[M_DVZ_DZ](i, j, k);
          m0 = s.X.b[i] * m0 + s.X.a[i] * dvxdx;
          m1 = s.Y.b[j] * m1 + s.Y.a[j] * dvydy;
          m2 = s.Z.b[k] * m2 + s.Z.a[k] * dvzdz;
          dvxdx = dvxdx / s.X.k[i] + m0;
          dvydy = dvydy / s.Y.k[j] + m1;
          dvzdz = dvzdz / s.Z.k[k] + m2;
        }
        s.sxx(i, j, k) += (lpm * dvxdx + lhx * (dvzdz + dvydy)) * dt;
        s.syy(i, j, k) += (lpm * dvydy + lhx * (dvxdx + dvzdz)) * dt;
        s.szz(i, j, k) += (lpm * dvzdz + lhx * (dvxdx + dvydy)) * dt;
      }
#pragma omp parallel for collapse(2)
  for (int i = N + 1; i < nx - N; ++i)
    for (int j = N + 1; j < ny - N; ++j)
      for (int k = N; k < nz - N; ++k) {
        T x = (T)(i - N) * dx + dx / (T)2, y = (T)(j - N) * dy + dy / (T)2, z = (T)(k - N) * dz;
        T m4 = (T)0.25 * (s.mu(i, j + 1, k) + s.mu(i, j, k) + s.mu(i, j, k) + s.mu(i + 1, j, k));
        T dvydx = Dx3fm(s.vy, i, j, k, s.c, N) / dx;
        T dvxdy = Dy3fm(s.vx, i, j, k, s.c, N) / dy;
        if (s.in(x, y, z)) {
          T& m0 = s.m[M_DVY_DX](i, j, k); T& m1 = s.m[M_DVX_DY](i, j, k);
          m0 = s.X.b_half[i] * m0 + s.X.a_half[i] * dvydx;
          m1 = s.Y.b_half[j] * m1 + s.Y.a_half[j] * dvxdy;
          dvydx = dvydx / s.X.k_half[i] + m0;
          dvxdy = dvxdy / s.Y.k_half[j] + m1;
        }
        s.sxy(i, j, k) += m4 * (dvxdy + dvydx) * dt;
      }
#pragma omp parallel for collapse(2)
  for (int i = N; i < nx - N - 1; ++i)
    for (int j = N; j < ny - N; ++j)
      for (int k = N; k < nz - N - 1; ++k) {
        T x = (T)(i - N) * dx + dx / (T)2, y = (T)(j - N) * dy, z = (T)(k - N) * dz + dz / (T)2;
        T m4 = (T)0.25 * (s.mu(i, j, k) + s.mu(i + 1, j, k) + s.mu(i, j, k) + s.mu(i, j + 1, k));
        T dvzdx = Dx3fm(s.vz, i, j, k, s.c, N) / dx;
        T dvxdz = Dz3fm(s.vx, i, j, k, s.c, N) / dz;
        if (s.in(x, y, z)) {
          T& m0 = s.m[M_DVZ_DX](i, j, k); T& m1 = s.m[M_DVX_DZ](i, j, k);
          m0 = s.X.b_half[i] * m0 + s.X.a_half[i] * dvzdx;
          m1 = s.Z.b_half[k] * m1 + s.Z.a_half[k] * dvxdz;
          dvzdx = dvzdx / s.X.k_half[i] + m0;
          dvxdz = dvxdz / s.Z.k_half[k] + m1;
        }
        s.sxz(i, j, k) += m4 * (dvxdz + dvzdx) * dt;
      }
#pragma omp parallel for collapse(2)
  for (int i = N; i < nx - N; ++i)
    for (int j = N; j < ny - N - 1; ++j)
      for (int k = N; k < nz - N - 1; ++k) {
        T x = (T)(i - N) * dx, y = (T)(j - N) * dy + dy / (T)2, z = (T)(k - N) * dz + dz / (T)2;
        T m4 = (T)0.25 * (s.mu(i, j + 1, k) + s.mu(i, j, k) + s.mu(i, j, k + 1) + s.mu(i, j, k));
        T dvzdy = Dy3fm(s.vz, i, j, k, s.c, N) / dy;
        T dvydz = Dz3fm(s.vy, i, j, k, s.c, N) / dz;
        if (s.in(x, y, z)) {
          T& m0 = s.m[M_DVZ_DY](i, j, k); T& m1 = s.m[M_DVY_DZ](i, j, k);
          m0 = s.Y.b_half[j] * m0 + s.Y.a_half[j] * dvzdy;
          m1 = s.Z.b_half[k] * m1 + s.Z.a_half[k] * dvydz;
          dvzdy = dvzdy / s.Y.k_half[j] + m0;
          dvydz = dvydz / s.Z.k_half[k] + m1;
        }
        s.syz(i, j, k) += m4 * (dvzdy + dvydz) * dt;
      }
}

// Elastic3D_SSG_Tensor.py:166-345
template <typename T>
void step3d_tensor(const O3Desc& d, int it) {
  S3<T> s(d);
  float f0 = (float)d.f0;
  float w = d.wavelet ? d.wavelet[it]
                      : ricker2(it, (float)d.dt, (float)d.t0, f0, (float)d.src_scale);
  T src = (T)w;
  const int a = d.isx, b = d.isy, c = d.isz;
  s.sxx(a, b, c) += src * (-(T)(float)d.mt[0]);
  s.syy(a, b, c) += src * (-(T)(float)d.mt[1]);
  s.szz(a, b, c) += src * (-(T)(float)d.mt[2]);
  s.sxy(a, b, c) += src * (-(T)(float)d.mt[3]);
  s.sxz(a, b, c) += src * (-(T)(float)d.mt[4]);
  s.syz(a, b, c) += src * (-(T)(float)d.mt[5]);
  velocity3d(s, true);
  stress3d(s);
  if (d.data) {
    float* out = (float*)d.data;
    for (int r = 0; r < d.nrec; ++r) out[(size_t)it * d.nrec + r] = (float)s.vx(d.rx[r], d.ry[r], d.rz[r]);
  }
}

// Elastic3D_SSG_CPML.py:144-309 (the six Dirichlet loops at :215-243 only
// touch cells that no phase ever writes, so on in-range indices they are no-ops)
template <typename T>
void step3d_cpml(const O3Desc& d, int it) {
  S3<T> s(d);
  velocity3d(s, false);
  float w = d.wavelet ? d.wavelet[it] : ricker(it, (float)d.dt, (float)d.f0, 1000.0f);
  const int a = d.isx + 5, b = d.isy + 5, c = d.isz + 5;
  s.vz(a, b, c) += s.dt * (T)w / s.rho(a, b, c);
  stress3d(s);
  if (d.data) ((float*)d.data)[it] = (float)s.vx(d.rx[0], d.ry[0], d.rz[0]);
}

// split-field order used by the SPML descriptor (reference names)
enum {
  P_VX_X = 0, P_VX_Y, P_VX_Z, P_VY_X, P_VY_Y, P_VY_Z, P_VZ_X, P_VZ_Y, P_VZ_Z,
  P_SXX_X, P_SXX_Y, P_SXX_Z, P_SYY_X, P_SYY_Y, P_SYY_Z,
  P_SXY_X, P_SXY_Y, P_SXZ_X, P_SXZ_Z, P_SYZ_Y, P_SYZ_Z,
  P_SZZ_X, P_SZZ_Y, P_SZZ_Z
};

// Elastic3D_SSG_SPML.py:160-393
template <typename T>
void step3d_spml(const O3Desc& d, int it) {
  S3<T> s(d);
  const int N = s.N, nx = s.nx, ny = s.ny, nz = s.nz;
  const T dx = s.dx, dy = s.dy, dz = s.dz, dt = s.dt;
  const T hdt = (T)0.5 * dt;
  auto& m = s.m;
#pragma omp parallel for collapse(2)
  for (int i = N; i < nx - N - 1; ++i)
    for (int j = N + 1; j < ny - N; ++j)
      for (int k = N + 1; k < nz - N; ++k) {
        T x = (T)(i - N) * dx + dx / (T)2, y = (T)(j - N) * dy, z = (T)(k - N) * dz;
        T dsxxdx = Dx3fm(s.sxx, i, j, k, s.c, N) / dx;
        T dsxydy = Dy3bm(s.sxy, i, j, k, s.c, N) / dy;
        T dsxzdz = Dz3bm(s.sxz, i, j, k, s.c, N) / dz;
        T rho = s.rho(i, j, k);
        T ro = (T)1 / rho;
        if (s.in(x, y, z)) {
          T xn = (T)1 - hdt * s.X.pml_half[i], yn = (T)1 - hdt * s.Y.pml[j], zn = (T)1 - hdt * s.Z.pml[k];
          T xd = (T)1 + hdt * s.X.pml_half[i], yd = (T)1 + hdt * s.Y.pml[j], zd = (T)1 + hdt * s.Z.pml[k];
          T& a = m[P_VX_X](i, j, k); T& b = m[P_VX_Y](i, j, k); T& c = m[P_VX_Z](i, j, k);
          a = (xn * a + dsxxdx * dt * ro) / xd;
          b = (yn * b + dsxydy * dt * ro) / yd;
          c = (zn * c + dsxzdz * dt * ro) / zd;
          s.vx(i, j, k) = a + b + c;
        } else {
          s.vx(i, j, k) += (dsxxdx + dsxydy + dsxzdz) * dt * ro;
        }
      }
#pragma omp parallel for collapse(2)
  for (int i = N + 1; i < nx - N; ++i)
    for (int j = N; j < ny - N - 1; ++j)
      for (int k = N + 1; k < nz - N; ++k) {
        T x = (T)(i - N) * dx, y = (T)(j - N) * dy + dy / (T)2, z = (T)(k - N) * dz;
        T rhy = (T)0.5 * (s.rho(i, j, k) + s.rho(i, j + 1, k));
        T ro = (T)1 / rhy;
        T dsxydx = Dx3bm(s.sxy, i, j, k, s.c, N) / dx;
        T dsyydy = Dy3fm(s.syy, i, j, k, s.c, N) / dy;
        T dsyzdz = Dz3bm(s.syz, i, j, k, s.c, N) / dz;
        if (s.in(x, y, z)) {
          T xn = (T)1 - hdt * s.X.pml[i], yn = (T)1 - hdt * s.Y.pml_half[j], zn = (T)1 - hdt * s.Z.pml[k];
          T xd = (T)1 + hdt * s.X.pml[i], yd = (T)1 + hdt * s.Y.pml_half[j], zd = (T)1 + hdt * s.Z.pml[k];
          T& a = m[P_VY_X](i, j, k); T& b = m[P_VY_Y](i, j, k); T& c = m[P_VY_Z](i, j, k);
          a = (xn * a + dt * dsxydx * ro) / xd;
          b = (yn * b + dt * dsyydy * ro) / yd;
          c = (zn * c + dt * dsyzdz * ro) / zd;
          s.vy(i, j, k) = a + b + c;
        } else {
          s.vy(i, j, k) += (dsxydx + dsyydy + dsyzdz) * dt * ro;
        }
      }
#pragma omp parallel for collapse(2)
  for (int i = N + 1; i < nx - N; ++i)
    for (int j = N + 1; j < ny - N; ++j)
      for (int k = N; k < nz - N - 1; ++k) {
        T x = (T)(i - N) * dx, y = (T)(j - N) * dy, z = (T)(k - N) * dz + dz / (T)2;
        T r4 = (T)0.25 * (s.rho(i, j, k) + s.rho(i, j + 1, k) + s.rho(i + 1, j + 1, k) + s.rho(i + 1, j, k));
        T ro = (T)1 / r4;
        T dsxzdx = Dx3bm(s.sxz, i, j, k, s.c, N) / dx;
        T dsyzdy = Dy3bm(s.syz, i, j, k, s.c, N) / dy;
        T dszzdz = Dz3fm(s.szz, i, j, k, s.c, N) / dz;
        if (s.in(x, y, z)) {
          T xn = (T)1 - hdt * s.X.pml[i], yn = (T)1 - hdt * s.Y.pml[j], zn = (T)1 - hdt * s.Z.pml_half[k];
          T xd = (T)1 + hdt * s.X.pml[i], yd = (T)1 + hdt * s.Y.pml[j], zd = (T)1 + hdt * s.Z.pml_half[k];
          T& a = m[P_VZ_X](i, j, k); T& b = m[P_VZ_Y](i, j, k); T& c = m[P_VZ_Z](i, j, k);
          a = (xn * a + dt * dsxzdx * ro) / xd;
          b = (yn * b + dt * dsyzdy * ro) / yd;
          c = (zn * c + dt * dszzdz * ro) / zd;
          s.vz(i, j, k) = a + b + c;
        } else {
          s.vz(i, j, k) += (dsxzdx + dsyzdy + dszzdz) * dt * ro;
        }
      }
  {
    float w = d.wavelet ? d.wavelet[it] : ricker(it, (float)d.dt, (float)d.f0, (float)d.src_scale);
    s.vz(d.isx, d.isy, d.isz) += dt * (T)w / s.rho(d.isx, d.isy, d.isz);
  }
#pragma omp parallel for collapse(2)
  for (int i = N + 1; i < nx - N; ++i)
    for (int j = N + 1; j < ny - N; ++j)
      for (int k = N + 1; k < nz - N; ++k) {
        T x = (T)(i - N) * dx, y = (T)(j - N) * dy, z = (T)(k - N) * dz;
        T lam = s.lam(i, j, k), mu = s.mu(i, j, k);
        T l2m = lam + (T)2 * mu;
        T dvxdx = Dx3bm(s.vx, i, j, k, s.c, N) / dx;
        T dvydy = Dy3bm(s.vy, i, j, k, s.c, N) / dy;
        T dvzdz = Dz3bm(s.vz, i, j, k, s.c, N) / dz;
        if (s.in(x, y, z)) {
          T xn = (T)1 - hdt * s.X.pml[i], yn = (T)1 - hdt * s.Y.pml[j], zn = (T)1 - hdt * s.Z.pml[k];
          T xd = (T)1 + hdt * s.X.pml[i], yd = (T)1 + hdt * s.Y.pml[j], zd = (T)1 + hdt * s.Z.pml[k];
          T& xx = m[P_SXX_X](i, j, k); T& xy = m[P_SXX_Y](i, j, k); T& xz = m[P_SXX_Z](i, j, k);
          T& yx = m[P_SYY_X](i, j, k); T& yy = m[P_SYY_Y](i, j, k); T& yz = m[P_SYY_Z](i, j, k);
          T& zx = m[P_SZZ_X](i, j, k); T& zy = m[P_SZZ_Y](i, j, k); T& zz = m[P_SZZ_Z](i, j, k);
          xx = (xn * xx + dt * l2m * dvxdx) / xd;
          xy = (yn * xy + dt * lam * dvydy) / yd;
          xz = (zn * xz + dt * lam * dvzdz) / zd;
          yx = (xn * yx + dt * lam * dvxdx) / xd;
          yy = (yn * yy + dt * l2m * dvydy) / yd;
          yz = (zn * yz + dt * lam * dvzdz) / zd;
          zx = (xn * zx + dt * lam * dvxdx) / xd;
          zy = (yn * zy + dt * lam * dvydy) / yd;
          zz = (zn * zz + dt * l2m * dvzdz) / zd;
          s.sxx(i, j, k) = xx + xy + xz;
          s.syy(i, j, k) = yx + yy + yz;
          s.szz(i, j, k) = zx + zy + zz;
        } else {
          s.sxx(i, j, k) += (l2m * dvxdx + lam * (dvzdz + dvydy)) * dt;
          s.syy(i, j, k) += (l2m * dvydy + lam * (dvxdx + dvzdz)) * dt;
          s.szz(i, j, k) += (l2m * dvzdz + lam * (dvxdx + dvydy)) * dt;
        }
      }
#pragma omp parallel for collapse(2)
  for (int i = N + 1; i < nx - N; ++i)
    for (int j = N + 1; j < ny - N; ++j)
      for (int k = N; k < nz - N; ++k) {
        T x = (T)(i - N) * dx + dx / (T)2, y = (T)(j - N) * dy + dy / (T)2, z = (T)(k - N) * dz;
        T m4 = (T)0.25 * (s.mu(i, j + 1, k) + s.mu(i, j, k) + s.mu(i, j, k) + s.mu(i + 1, j, k));
        T dvydx = Dx3fm(s.vy, i, j, k, s.c, N) / dx;
        T dvxdy = Dy3fm(s.vx, i, j, k, s.c, N) / dy;
        if (s.in(x, y, z)) {
          T xn = (T)1 - hdt * s.X.pml_half[i], yn = (T)1 - hdt * s.Y.pml_half[j];
          T xd = (T)1 + hdt * s.X.pml_half[i], yd = (T)1 + hdt * s.Y.pml_half[j];
          T& a = m[P_SXY_X](i, j, k); T& b = m[P_SXY_Y](i, j, k);
          a = (xn * a + dt * m4 * dvydx) / xd;
          b = (yn * b + dt * m4 * dvxdy) / yd;
          s.sxy(i, j, k) = a + b;
        } else {
          s.sxy(i, j, k) += m4 * (dvxdy + dvydx) * dt;
        }
      }
#pragma omp parallel for collapse(2)
  for (int i = N; i < nx - N - 1; ++i)
    for (int j = N; j < ny - N; ++j)
      for (int k = N; k < nz - N - 1; ++k) {
        T x = (T)(i - N) * dx + dx / (T)2, y = (T)(j - N) * dy, z = (T)(k - N) * dz + dz / (T)2;
        T m4 = (T)0.25 * (s.mu(i, j, k) + s.mu(i + 1, j, k) + s.mu(i, j, k) + s.mu(i, j + 1, k));
        T dvzdx = Dx3fm(s.vz, i, j, k, s.c, N) / dx;
        T dvxdz = Dz3fm(s.vx, i, j, k, s.c, N) / dz;
        if (s.in(x, y, z)) {
          T xn = (T)1 - hdt * s.X.pml_half[i], zn = (T)1 - hdt * s.Z.pml_half[k];
          T xd = (T)1 + hdt * s.X.pml_half[i], zd = (T)1 + hdt * s.Z.pml_half[k];
          T& a = m[P_SXZ_X](i, j, k); T& b = m[P_SXZ_Z](i, j, k);
          a = (xn * a + dt * m4 * dvzdx) / xd;
          b = (zn * b + dt * m4 * dvxdz) / zd;
          s.sxz(i, j, k) = a + b;
        } else {
          s.sxz(i, j, k) += m4 * (dvxdz + dvzdx) * dt;
        }
      }
#pragma omp parallel for collapse(2)
  for (int i = N; i < nx - N; ++i)
    for (int j = N; j < ny - N - 1; ++j)
      for (int k = N; k < nz - N - 1; ++k) {
        T x = (T)(i - N) * dx, y = (T)(j - N) * dy + dy / (T)2, z = (T)(k - N) * dz + dz / (T)2;
        T m4 = (T)0.25 * (s.mu(i, j + 1, k) + s.mu(i, j, k) + s.mu(i, j, k + 1) + s.mu(i, j, k));
        T dvzdy = Dy3fm(s.vz, i, j, k, s.c, N) / dy;
        T dvydz = Dz3fm(s.vy, i, j, k, s.c, N) / dz;
        if (s.in(x, y, z)) {
          T yn = (T)1 - hdt * s.Y.pml_half[j], zn = (T)1 - hdt * s.Z.pml_half[k];
          T yd = (T)1 + hdt * s.Y.pml_half[j], zd = (T)1 + hdt * s.Z.pml_half[k];
          T& a = m[P_SYZ_Y](i, j, k); T& b = m[P_SYZ_Z](i, j, k);
          a = (yn * a + dt * m4 * dvzdy) / yd;
          b = (zn * b + dt * m4 * dvydz) / zd;
          s.syz(i, j, k) = a + b;
        } else {
          s.syz(i, j, k) += m4 * (dvydz + dvzdy) * dt;
        }
      }
  if (d.data) ((float*)d.data)[it] = (float)s.vx(d.rx[0], d.ry[0], d.rz[0]);
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI of the oracle
// ---------------------------------------------------------------------------
extern "C" {

int oracle_version(void) { return 1; }

int oracle_set_threads(int n) {
#if defined(_OPENMP)
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

// src/BaseFun.py wavelets, float.  kind 0: Ricker(it,dt,f,scale),
// 1: Ricker2(it,dt,t0,f,scale), 2: Ricker3(it,dt,t0,f,scale).
void oracle_wavelet(int kind, int nt, double dt, double t0, double f, double scale, float* out) {
  for (int it = 0; it < nt; ++it) {
    if (kind == 0) out[it] = ricker(it, (float)dt, (float)f, (float)scale);
    else if (kind == 1) out[it] = ricker2(it, (float)dt, (float)t0, (float)f, (float)scale);
    else out[it] = ricker3(it, (float)dt, (float)t0, (float)f, (float)scale);
  }
}

// diff_coff (Elastic2D_CPML.py:355-366): solve A c = e1, A[i][j] = (2j+1)^(2i+1),
// in double with partially pivoted Gaussian elimination; the reference stores
// the result as float.
int oracle_diff_coff(int order, double* out_double, float* out_float) {
  if (order < 1 || order > 16) return -1;
  const int n = order;
  std::vector<double> A((size_t)n * n), b(n, 0.0);
  b[0] = 1.0;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) A[(size_t)i * n + j] = std::pow((double)(2 * j + 1), (double)(2 * i + 1));
  for (int col = 0; col < n; ++col) {
    int piv = col;
    for (int r = col + 1; r < n; ++r)
      if (std::fabs(A[(size_t)r * n + col]) > std::fabs(A[(size_t)piv * n + col])) piv = r;
    if (piv != col) {
      for (int q = 0; q < n; ++q) std::swap(A[(size_t)col * n + q], A[(size_t)piv * n + q]);
      std::swap(b[col], b[piv]);
    }
    for (int r = col + 1; r < n; ++r) {
      double f = A[(size_t)r * n + col] / A[(size_t)col * n + col];
      for (int q = col; q < n; ++q) A[(size_t)r * n + q] -= f * A[(size_t)col * n + q];
      b[r] -= f * b[col];
    }
  }
  for (int r = n - 1; r >= 0; --r) {
    double s = b[r];
    for (int q = r + 1; q < n; ++q) s -= A[(size_t)r * n + q] * b[q];
    b[r] = s / A[(size_t)r * n + r];
  }
  for (int i = 0; i < n; ++i) {
    if (out_double) out_double[i] = b[i];
    if (out_float) out_float[i] = (float)b[i];
  }
  return 0;
}

// One axis of SetADEPML2D/3D (Elastic2D_CPML.py:392-528,
// Elastic3D_SSG_Tensor.py:361-568): profiles evaluated in double, stored in the
// field dtype (dtype 0: float, 1: double), then b and a recomputed in double
// from the stored values.  out: ten arrays of length n in the order
// pml, pml_half, alpha, alpha_half, k, k_half, b, b_half, a, a_half.
int oracle_pml_axis(int n, int star, double d, double thick, int use_lo, int use_hi,
                    double vp_max, double Rcoef, double alpha_max, double kmax, double theta,
                    double dt, int dtype, void** out, double* pml_min_max) {
  const double xmin = 0.0;
  const double xmax = xmin + d * (double)(n - 1 - 2 * star);
  const double lo = xmin + thick, hi = xmax - thick;
  const double d0 = -3.0 * vp_max * std::log(Rcoef) / (2.0 * thick);
  pml_min_max[0] = lo;
  pml_min_max[1] = hi;
  auto store = [&](int which, int i, double v) {
    if (dtype == 0) ((float*)out[which])[i] = (float)v;
    else ((double*)out[which])[i] = v;
  };
  auto load = [&](int which, int i) -> double {
    return dtype == 0 ? (double)((float*)out[which])[i] : ((double*)out[which])[i];
  };
  for (int half = 0; half < 2; ++half) {
    for (int i = 0; i < n; ++i) {
      double x = (double)(i - star) * d;
      if (half) x = (double)(i - star) * d + d / 2;
      double p, al, kk;
      if (x <= lo && use_lo) {
        double s = (lo - x) / thick;
        p = d0 * (s * s);
        al = alpha_max * (1 - s);
        kk = 1 + (kmax - 1) * (s * s);
      } else if (x >= hi && use_hi) {
        double s = (x - hi) / thick;
        p = d0 * (s * s);
        al = alpha_max * (1 - s);
        kk = 1 + (kmax - 1) * (s * s);
      } else {
        p = 0; al = 0; kk = 1;
      }
      store(0 + half, i, p);
      store(2 + half, i, al);
      store(4 + half, i, kk);
      if (load(2 + half, i) < 0) store(2 + half, i, 0.0);
    }
  }
  for (int i = 0; i < n; ++i) {
    for (int half = 0; half < 2; ++half) {
      double p = load(0 + half, i), al = load(2 + half, i), kk = load(4 + half, i);
      double bb = (1 - (1 - theta) * dt * (p / kk + al)) / (1 + theta * dt * (p / kk + al));
      store(6 + half, i, bb);
      if (std::fabs(p) > 1e-6) {
        double aa = -dt * p / (kk * kk) / (1 + theta * dt * (p / kk + al));
        store(8 + half, i, aa);
      } else {
        store(8 + half, i, 0.0);
      }
    }
  }
  return 0;
}

int oracle2d_step(const O2Desc* d, int scheme, int it, double rsg_source) {
  if (!d) return -1;
  if (d->dtype == 0) {
    if (scheme == 0) step2d_vs<float>(*d, it);
    else if (scheme == 1) step2d_sv<float>(*d, it);
    else step2d_rsg<float>(*d, it, rsg_source);
  } else {
    if (scheme == 0) step2d_vs<double>(*d, it);
    else if (scheme == 1) step2d_sv<double>(*d, it);
    else step2d_rsg<double>(*d, it, rsg_source);
  }
  return 0;
}

int oracle2d_run(const O2Desc* d, int scheme, int it0, int nsteps, const double* rsg_sources) {
  for (int s = 0; s < nsteps; ++s)
    oracle2d_step(d, scheme, it0 + s, rsg_sources ? rsg_sources[s] : 0.0);
  return 0;
}

int oracle3d_step(const O3Desc* d, int it) {
  if (!d) return -1;
  if (d->dtype == 0) {
    if (d->scheme == 0) step3d_cpml<float>(*d, it);
    else if (d->scheme == 1) step3d_tensor<float>(*d, it);
    else step3d_spml<float>(*d, it);
  } else {
    if (d->scheme == 0) step3d_cpml<double>(*d, it);
    else if (d->scheme == 1) step3d_tensor<double>(*d, it);
    else step3d_spml<double>(*d, it);
  }
  return 0;
}

int oracle3d_run(const O3Desc* d, int it0, int nsteps) {
  for (int s = 0; s < nsteps; ++s) oracle3d_step(d, it0 + s);
  return 0;
}

}  // extern "C"
