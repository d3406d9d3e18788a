// sw_device.cuh -- kernel parameter blocks and small device helpers shared by
// the 2D and 3D staggered-grid kernels.
//
// Floating-point contract: every kernel is compiled with -fmad=false and IEEE
// division, and evaluates each update in the operation order of the
// reference's Taichi source, so a run is reproducible bit for bit against a
// CPU evaluation of the same expressions.
#pragma once

#include <atomic>
#include <cstdint>
#include <mutex>
#include <cuda_runtime.h>

#include "../../include/seiswave.h"

namespace sw {

// One-time setup per device (kernel attributes such as the dynamic
// shared-memory opt-in are per device): runs f() once for each device the
// calling threads launch on, under a lock; a failed f() is retried next time.
template <class F>
inline cudaError_t once_per_device(std::atomic<unsigned long long>& done, std::mutex& mu, F f) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = 1ull << (dev & 63);
  if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
  std::lock_guard<std::mutex> lock(mu);
  if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
  e = f();
  if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_release);
  return e;
}

// slab-compact index of `i` on an axis of length n whose CPML slabs are
// [0, lo) and [n-hi, n); -1 outside both slabs.
__host__ __device__ __forceinline__ int slab_index(int i, int n, int lo, int hi) {
  return i < lo ? i : (i >= n - hi ? i - (n - hi) + lo : -1);
}

// coefficient table rows (sw_pml_axis.coef): 6 rows of n values
enum { CB = 0, CA = 1, CK = 2, CBH = 3, CAH = 4, CKH = 5 };
// split-PML fields, rows of P3::split in the reference's order
// (vx_x .. szz_z, Elastic3D_SSG_SPML.py:107-138)
enum {
  PVX_X = 0, PVX_Y, PVX_Z, PVY_X, PVY_Y, PVY_Z, PVZ_X, PVZ_Y, PVZ_Z,
  PSXX_X, PSXX_Y, PSXX_Z, PSYY_X, PSYY_Y, PSYY_Z,
  PSXY_X, PSXY_Y, PSXZ_X, PSXZ_Z, PSYZ_Y, PSYZ_Z,
  PSZZ_X, PSZZ_Y, PSZZ_Z
};

// 3D CPML memory-variable components, 6 per direction.
//   x: 0 sxx_dx(vx) 1 sxy_dx(vy) 2 sxz_dx(vz) 3 dvx_dx(normal) 4 dvy_dx(sxy) 5 dvz_dx(sxz)
//   y: 0 sxy_dy(vx) 1 syy_dy(vy) 2 syz_dy(vz) 3 dvy_dy(normal) 4 dvx_dy(sxy) 5 dvz_dy(syz)
//   z: 0 sxz_dz(vx) 1 syz_dz(vy) 2 szz_dz(vz) 3 dvz_dz(normal) 4 dvx_dz(sxz) 5 dvy_dz(syz)
template <typename T>
struct P3 {
  int nx, ny, nz;
  T dx, dy, dz, dt;
  T c[SW_MAX_ORDER];
  T* f[9];  // vx vy vz sxx syy szz sxy sxz syz
  const T* rho;
  const T* lam;
  const T* mu;
  const T* cf[3];
  const T* dmp[3];
  const uint8_t* fl[3];
  int lo[3], hi[3], sn[3];  // slab widths and sn = lo+hi
  T* mem[3];
  long long mcomp[3];       // elements between two components of mem[d]
  T* split;                 // SPML: 24 components over the PML shell (shell_index)
  long long scomp;          // SPML: cells in the shell = elements per component
  // source
  int src_kind, si, sj, sk;
  const T* wav;
  T mneg[6];                // -M_ab (xx yy zz xy xz yz) in the field type
  // receivers
  int nrec, rec_field, rec_f64;
  const long long* rec_idx;
  void* rec_data;
  int x_chunk;              // x planes streamed by one CTA
  T rd[3];                  // RN(1/dx), RN(1/dy), RN(1/dz)
  int fast_div;             // div_c may use the verified constant-divisor path
  T cs[3][SW_MAX_ORDER];    // c_m / dx, c_m / dy, c_m / dz (fast numeric mode)
};

// 2D memory-variable components, 4 per direction, shared by all schemes:
//   x: 0 sxx_dx 1 sxz_dx 2 dvx_dx 3 dvz_dx;  z: 0 sxz_dz 1 szz_dz 2 dvz_dz 3 dvx_dz
template <typename T>
struct P2 {
  int nx, nz;
  T dx, dz, dt;
  T c[SW_MAX_ORDER];
  T* f[5];  // vx vz sxx szz sxz
  const T* rho;
  const T* lam;
  const T* mu;
  const T* cf[2];
  const uint8_t* fl[2];
  int lo[2], hi[2], sn[2];
  T* mem[2];
  long long mcomp[2];
  int src_kind, si, sk;
  const T* wav;
  int nrec, rec_field, rec_f64;
  const long long* rec_idx;
  void* rec_data;
  T rd[2];                  // RN(1/dx), RN(1/dz)
  T rd2[2];                 // RN(1/(2dx)), RN(1/(2dz)) (rotated-grid derivatives)
  int fast_div;             // bit0: dx, dz verified; bit1: 2dx, 2dz verified
  T mneg[3];                // moment-tensor source: -M_xx, -M_zz, -M_xz
};

// A group of at most SW_BATCH_GROUP shots of a 2D batch, passed to the
// batched kernels by value: the shots' parameter blocks live in kernel
// parameter space (read through the constant cache like a single shot's
// parameters, 64 x 368 bytes at most, under the 32 KB parameter limit), and
// work holds the group's work items, one per block: x = shot index in the
// batch, y = tile row (x direction) << 16 | tile column (z direction).
#define SW_BATCH_TILES 4
#define SW_BATCH_GROUP 64
template <typename T>
struct Batch2 {
  P2<T> shots[SW_BATCH_GROUP];
  const int2* work;
  int first, n;  // batch index of shots[0]; shots in the group
};

template <typename T>
__device__ __forceinline__ T ldg(const T* p) { return __ldg(p); }

// Position of cell (i, j, k) in the split-PML shell, the union of the three
// axes' slabs [0, lo) and [n-hi, n): first the x slabs over the whole (y, z)
// plane, then the y slabs of the x interior, then the z slabs of the x-y
// interior, z fastest in each part.  Valid for cells inside some slab.
template <typename T>
__device__ __forceinline__ long long shell_index(const P3<T>& p, int i, int j, int k) {
  const int ix = slab_index(i, p.nx, p.lo[0], p.hi[0]);
  if (ix >= 0) return ((long long)ix * p.ny + j) * p.nz + k;
  const long long a = (long long)p.sn[0] * p.ny * p.nz;
  const long long i2 = i - p.lo[0];
  const int iy = slab_index(j, p.ny, p.lo[1], p.hi[1]);
  if (iy >= 0) return a + (i2 * p.sn[1] + iy) * p.nz + k;
  const long long b = (long long)(p.nx - p.sn[0]) * p.sn[1] * p.nz;
  const int iz = slab_index(k, p.nz, p.lo[2], p.hi[2]);
  return a + b + (i2 * (p.ny - p.sn[1]) + (j - p.lo[1])) * p.sn[2] + iz;
}

// x / d for a positive divisor that varies per cell (density, kappa, split-PML
// denominators).  A zero numerator -- most of the grid ahead of the wavefront
// -- returns x itself, which is exactly +-0/d for d > 0, without entering the
// division routine.
template <typename T>
__device__ __forceinline__ T div_v(T x, T d) {
  return x == (T)0 ? x : x / d;
}

// Division of floats whose numerator may be tiny (the numerical precursor
// ahead of a wavefront holds values down to the denormal range, for which the
// float division routine leaves its fast path).  Such numerators are divided
// in double precision and rounded once to float: with 53 >= 2*24+2 bits the
// double rounding is innocuous (S. Figueroa, "When is double rounding
// innocuous?", SIGNUM Newsletter 30(3), 1995), so the result equals the
// correctly rounded float quotient.  Float inputs are normal doubles, so the
// double division never leaves its own fast path.
// Out of line so the rare path does not bloat every call site.
static __device__ __noinline__ float div_rare(float x, float d) {
  if (x == 0.f) return x;  // +-0/d = +-0 for d > 0
  return __double2float_rn(__ddiv_rn((double)x, (double)d));
}

// The quotient x/d from xs = x*2^64 (exact) and ys = RN(xs/d) for d > 0,
// ys normal: scaled back while normal; in the subnormal range rounded again
// to the 2^-149 grid (2^-85 after the scaling), where only a scaled quotient
// exactly on a midpoint of that grid can round differently from x/d itself;
// the exact residual xs - ys*d (representable because ys is the correctly
// rounded quotient) tells on which side x/d lies.
__device__ __forceinline__ float tiny_finish(float xs, float ys, float d) {
  if (fabsf(ys) >= 0x1p-62f) return __fmul_rn(ys, 0x1p-64f);
  const float t = __fmul_rn(ys, 0x1p85f);  // |t| < 2^23: units of the subnormal grid
  float n = rintf(t);
  if (fabsf(__fadd_rn(t, -truncf(t))) == 0.5f) {
    const float res = __fmaf_rn(-ys, d, xs);
    if (res > 0.f) n = __fadd_rn(floorf(t), 1.f);
    else if (res < 0.f) n = floorf(t);
  }
  return __fmul_rn(n, 0x1p-149f);
}

// x / d for 0 < |x| < 2^-100 and a per-cell divisor: the scaled numerator
// goes through IEEE division's fast path (a tiny numerator sends the float
// division routine to its slow path); divisors outside [2^-60, 2^60] take
// the double-precision quotient.
static __device__ __noinline__ float div_tiny_v(float x, float d) {
  if (!(d >= 0x1p-60f && d <= 0x1p60f)) return div_rare(x, d);
  const float xs = __fmul_rn(x, 0x1p64f);
  return tiny_finish(xs, __fdiv_rn(xs, d), d);
}

template <>
__device__ __forceinline__ float div_v<float>(float x, float d) {
  const unsigned ex = (__float_as_uint(x) >> 23) & 0xffu;  // biased exponent
  if (ex - 27u < 200u) return __fdiv_rn(x, d);                // |x| in [2^-100, 2^100)
  if ((__float_as_uint(x) << 1) == 0u) return x;              // +-0/d = +-0 for d > 0
  if (ex < 27u) return div_tiny_v(x, d);                      // 0 < |x| < 2^-100
  return div_rare(x, d);
}

// Markstein's correction of x * r towards x / d, r = RN(1/d)
__device__ __forceinline__ float mk_core(float x, float d, float r) {
  const float q = __fmul_rn(x, r);
  const float e = __fmaf_rn(-q, d, x);
  return __fmaf_rn(e, r, q);
}

// x / d for 0 < |x| < 2^-100 (the numerical precursor ahead of a wavefront)
// with the constant divisor's correction: the numerator is scaled by 2^64
// (exact) into the corrected range and the quotient scaled back, exact while
// it stays normal.  A quotient below the normal range is rounded again to
// the subnormal grid (2^-149, i.e. 2^-85 after the scaling); that second
// rounding can only differ from rounding x/d directly when the scaled
// quotient lies exactly on a midpoint of the grid, and there the exact
// residual xs - ys*d tells on which side x/d lies.
__device__ __forceinline__ float mk_div_tiny(float x, float d, float r) {
  const float xs = __fmul_rn(x, 0x1p64f);
  return tiny_finish(xs, mk_core(xs, d, r), d);
}

// tiny_finish without branches (both outcomes computed, one selected), for
// groups whose lanes take different routes
__device__ __forceinline__ float tiny_finish_sel(float xs, float ys, float d) {
  const float t = __fmul_rn(ys, 0x1p85f);
  const float fl = floorf(t);
  const bool mid = fabsf(__fadd_rn(t, -truncf(t))) == 0.5f;
  const float res = __fmaf_rn(-ys, d, xs);
  float n = rintf(t);
  n = mid && res > 0.f ? __fadd_rn(fl, 1.f) : n;
  n = mid && res < 0.f ? fl : n;
  return fabsf(ys) >= 0x1p-62f ? __fmul_rn(ys, 0x1p-64f) : __fmul_rn(n, 0x1p-149f);
}

// div_c's result with a verified correction (fast != 0) for any |x| < 2^100
// -- zero, below 2^-100 or in [2^-100, 2^100) -- without a branch
__device__ __forceinline__ float mk_div_any(float x, float d, float r) {
  const unsigned u = __float_as_uint(x) & 0x7fffffffu;
  const bool tiny = u < 0x0D800000u;  // |x| < 2^-100, zero included
  const float xs = tiny ? __fmul_rn(x, 0x1p64f) : x;
  const float q = mk_core(xs, d, r);
  const float y = tiny ? tiny_finish_sel(xs, q, d) : q;
  return u == 0u ? x : y;
}

// div_v's result for |x| < 2^100 and d in [2^-60, 2^60] without a branch (a
// zero numerator divides 1 instead, so the division stays on its fast path,
// and passes through)
__device__ __forceinline__ float dv_div_any(float x, float d) {
  const unsigned u = __float_as_uint(x) & 0x7fffffffu;
  const bool tiny = u < 0x0D800000u;
  const float xs = u == 0u ? 1.f : (tiny ? __fmul_rn(x, 0x1p64f) : x);
  const float q = __fdiv_rn(xs, d);
  const float y = tiny ? tiny_finish_sel(xs, q, d) : q;
  return u == 0u ? x : y;
}

// x / d for a divisor fixed for the run (dx, dy, dz), r = RN(1/d).  With
// fast != 0 (float only) numerators of magnitude in [2^-100, 2^100) use
// Markstein's correction
//   q = RN(x*r), e = fma(-q, d, x), result = fma(e, r, q)
// (P. Markstein, IBM J. Res. Dev. 34(1), 1990), smaller nonzero ones
// mk_div_tiny; zeros pass through and huge values take div_rare.  The plan
// enables the fast path only after checking that the whole function equals
// IEEE division x/d for every finite float x (the 2^32 bit patterns).
__device__ __forceinline__ float div_c(float x, float d, float r, int fast) {
  const unsigned ex = (__float_as_uint(x) >> 23) & 0xffu;  // biased exponent
  if (ex - 27u < 200u) return fast ? mk_core(x, d, r) : __fdiv_rn(x, d);
  if ((__float_as_uint(x) << 1) == 0u) return x;  // +-0/d = +-0 for d > 0
  if (fast && ex < 27u) return mk_div_tiny(x, d, r);
  return div_rare(x, d);
}
__device__ __forceinline__ double div_c(double x, double d, double, int) { return div_v(x, d); }

// ---- groups of exact quotients without a per-lane range branch -------------
// mk_ok: x is zero or of magnitude in [2^-100, 2^100), where div_c's
// Markstein correction and IEEE division are used; mk_div: that correction
// with zeros passed through (the sign of zero kept); dd_div: the quotient
// divided in double precision and rounded once, correctly rounded for every
// finite float x and positive float d (innocuous double rounding).  A group
// tests all its lanes once and then runs one branch-free block, so the
// independent lanes can interleave; every lane gets the bits div_c / div_v
// would give it.
__device__ __forceinline__ bool mk_ok(float x) {
  const unsigned u = __float_as_uint(x) & 0x7fffffffu;
  return (u - 0x0D800000u < 0x64000000u) | (u == 0u);
}
__device__ __forceinline__ float dd_div(float x, float d) {
  const float y = __double2float_rn(__ddiv_rn((double)x, (double)d));
  return x == 0.f ? x : y;
}
__device__ __forceinline__ float mk_div(float x, float d, float r) {
  const float q = __fmul_rn(x, r);
  const float e = __fmaf_rn(-q, d, x);
  const float y = __fmaf_rn(e, r, q);
  return x == 0.f ? x : y;
}
// Three tiers, chosen once per group: every lane zero or in [2^-100, 2^100)
// (the steady state); some lane smaller, none of magnitude 2^100 or more
// (the numerical precursor ahead of a wavefront): every lane runs the scaled
// float route and selects its result (mk_div_any, dv_div_any); otherwise the
// double-precision quotient.  Each tier gives every lane div_c's / div_v's
// bits.
template <int K>
__device__ __forceinline__ void divc_group(float (&x)[K], const float (&d)[K], const float (&r)[K], int fast) {
  bool ok = fast != 0, small = fast != 0;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    ok = ok & mk_ok(x[k]);
    small = small & (fabsf(x[k]) < 0x1p100f);
  }
  if (ok) {
#pragma unroll
    for (int k = 0; k < K; ++k) x[k] = mk_div(x[k], d[k], r[k]);
  } else if (small) {
#pragma unroll
    for (int k = 0; k < K; ++k) x[k] = mk_div_any(x[k], d[k], r[k]);
  } else {
#pragma unroll
    for (int k = 0; k < K; ++k) x[k] = dd_div(x[k], d[k]);
  }
}
template <int K>
__device__ __forceinline__ void divc_group(double (&x)[K], const double (&d)[K], const double (&r)[K], int fast) {
#pragma unroll
  for (int k = 0; k < K; ++k) x[k] = div_c(x[k], d[k], r[k], fast);
}
// quotients by per-cell positive divisors (densities), grouped likewise
template <int K>
__device__ __forceinline__ void divv_group(float (&x)[K], const float (&d)[K]) {
  bool ok = true, small = true;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    ok = ok & mk_ok(x[k]);
    small = small & (fabsf(x[k]) < 0x1p100f) & (d[k] >= 0x1p-60f) & (d[k] <= 0x1p60f);
  }
  if (ok) {
#pragma unroll
    for (int k = 0; k < K; ++k) x[k] = x[k] == 0.f ? x[k] : __fdiv_rn(x[k], d[k]);
  } else if (small) {
#pragma unroll
    for (int k = 0; k < K; ++k) x[k] = dv_div_any(x[k], d[k]);
  } else {
#pragma unroll
    for (int k = 0; k < K; ++k) x[k] = dd_div(x[k], d[k]);
  }
}
template <int K>
__device__ __forceinline__ void divv_group(double (&x)[K], const double (&d)[K]) {
#pragma unroll
  for (int k = 0; k < K; ++k) x[k] = div_v(x[k], d[k]);
}

// receiver sample in the trace's element type
template <typename T>
__device__ __forceinline__ void store_rec(void* data, int f64, long long at, T v) {
  if (f64) ((double*)data)[at] = (double)v;
  else ((float*)data)[at] = (float)v;
}

}  // namespace sw
