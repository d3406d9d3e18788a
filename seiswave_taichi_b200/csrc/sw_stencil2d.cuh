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
