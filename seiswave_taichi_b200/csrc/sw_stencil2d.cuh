// sw_stencil2d.cuh -- the staggered and rotated 2D difference operators of
// src/Differential2D.py, the CPML memory-variable update, and slab pointers,
// shared by the forward and adjoint 2D kernels.
#pragma once

#include "sw_device.cuh"

namespace sw {

template <typename T>
__device__ __forceinline__ void pml2(T* __restrict__ m, T b, T a, T kk, T& d) {
  T psi = b * (*m) + a * d;
  *m = psi;
  d = div_v(d, kk) + psi;
}

// ---- 2D stencils of src/Differential2D.py, read through the read-only path --
template <typename T, int N>
__device__ __forceinline__ T dx_fm(const T* f, long long idx, int nz, const T* c) {
  T v = 0;
#pragma unroll
  for (int m = 0; m < N; ++m) v += c[m] * (ldg(f + idx + (long long)(m + 1) * nz) - ldg(f + idx - (long long)m * nz));
  return v;
}
template <typename T, int N>
__device__ __forceinline__ T dz_fm(const T* f, long long idx, const T* c) {
  T v = 0;
#pragma unroll
  for (int m = 0; m < N; ++m) v += c[m] * (ldg(f + idx + (m + 1)) - ldg(f + idx - m));
  return v;
}
template <typename T, int N>
__device__ __forceinline__ T dx_bm(const T* f, long long idx, int nz, const T* c) {
  T v = 0;
#pragma unroll
  for (int m = 0; m < N; ++m) v += c[m] * (ldg(f + idx + (long long)m * nz) - ldg(f + idx - (long long)(m + 1) * nz));
  return v;
}
template <typename T, int N>
__device__ __forceinline__ T dz_bm(const T* f, long long idx, const T* c) {
  T v = 0;
#pragma unroll
  for (int m = 0; m < N; ++m) v += c[m] * (ldg(f + idx + m) - ldg(f + idx - (m + 1)));
  return v;
}
// rotated: Drx2fm f[i+m+1, j+m+1] - f[i-m, j-m]
template <typename T, int N>
__device__ __forceinline__ T drx_fm(const T* f, long long idx, int nz, const T* c) {
  T v = 0;
#pragma unroll
  for (int m = 0; m < N; ++m)
    v += c[m] * (ldg(f + idx + (long long)(m + 1) * nz + (m + 1)) - ldg(f + idx - (long long)m * nz - m));
  return v;
}
// Drz2fm f[i-m, j+m+1] - f[i+m+1, j-m]
template <typename T, int N>
__device__ __forceinline__ T drz_fm(const T* f, long long idx, int nz, const T* c) {
  T v = 0;
#pragma unroll
  for (int m = 0; m < N; ++m)
    v += c[m] * (ldg(f + idx - (long long)m * nz + (m + 1)) - ldg(f + idx + (long long)(m + 1) * nz - m));
  return v;
}
// Drx2bm f[i+m, j+m] - f[i-m-1, j-m-1]
template <typename T, int N>
__device__ __forceinline__ T drx_bm(const T* f, long long idx, int nz, const T* c) {
  T v = 0;
#pragma unroll
  for (int m = 0; m < N; ++m)
    v += c[m] * (ldg(f + idx + (long long)m * nz + m) - ldg(f + idx - (long long)(m + 1) * nz - (m + 1)));
  return v;
}
// Drz2bm f[i-m-1, j+m] - f[i+m, j-m-1]
template <typename T, int N>
__device__ __forceinline__ T drz_bm(const T* f, long long idx, int nz, const T* c) {
  T v = 0;
#pragma unroll
  for (int m = 0; m < N; ++m)
    v += c[m] * (ldg(f + idx - (long long)(m + 1) * nz + m) - ldg(f + idx + (long long)m * nz - (m + 1)));
  return v;
}

// The 2N taps of a staggered difference, loaded before any arithmetic so that
// a thread's loads are all in flight together; rows / columns are clamped to
// the grid (the values of clamped taps only feed cells that are not updated).
// taps_x: f[i0 + q, j], q = 0 .. 2N-1; taps_z: f[i, j0 + q] (row base given).
// Taps wholly inside the grid (every cell away from the edges) skip the clamps.
template <typename T, int N>
__device__ __forceinline__ void taps_x(T (&t)[2 * N], const T* f, int i0, int j, int nx, int nz) {
  if (i0 >= 0 && i0 + 2 * N <= nx) {
    const T* b = f + (long long)i0 * nz + j;
#pragma unroll
    for (int q = 0; q < 2 * N; ++q) t[q] = ldg(b + (long long)q * nz);
  } else {
#pragma unroll
    for (int q = 0; q < 2 * N; ++q) t[q] = ldg(f + (long long)min(max(i0 + q, 0), nx - 1) * nz + j);
  }
}
template <typename T, int N>
__device__ __forceinline__ void taps_z(T (&t)[2 * N], const T* f, long long row, int j0, int nz) {
  if (j0 >= 0 && j0 + 2 * N <= nz) {
    const T* b = f + row + j0;
#pragma unroll
    for (int q = 0; q < 2 * N; ++q) t[q] = ldg(b + q);
  } else {
#pragma unroll
    for (int q = 0; q < 2 * N; ++q) t[q] = ldg(f + row + min(max(j0 + q, 0), nz - 1));
  }
}
// sum_m c_m (t[N+m] - t[N-1-m]) from m = 0: with i0 = i - N this is the
// backward difference at i, with i0 = i - N + 1 the forward one (the order of
// the Dx2bm / Dx2fm sums)
template <typename T, int N>
__device__ __forceinline__ T tapsum(const T (&t)[2 * N], const T* c) {
  T v = 0;
#pragma unroll
  for (int m = 0; m < N; ++m) v += c[m] * (t[N + m] - t[N - 1 - m]);
  return v;
}

// memory-variable pointers
template <typename T>
__device__ __forceinline__ T* mx(const P2<T>& p, int comp, int xi, int j) {
  return p.mem[0] + comp * p.mcomp[0] + (long long)xi * p.nz + j;
}
template <typename T>
__device__ __forceinline__ T* mz(const P2<T>& p, int comp, int i, int zj) {
  return p.mem[1] + comp * p.mcomp[1] + (long long)i * p.sn[1] + zj;
}

}  // namespace sw
