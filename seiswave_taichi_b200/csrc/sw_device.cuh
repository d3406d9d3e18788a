// sw_device.cuh -- kernel parameter blocks and small device helpers shared by
// the 2D and 3D staggered-grid kernels.
//
// Floating-point contract: every kernel is compiled with -fmad=false and IEEE
// division, and evaluates each update in the operation order of the
// reference's Taichi source, so a run is reproducible bit for bit against a
// CPU evaluation of the same expressions.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/seiswave.h"

namespace sw {

// slab-compact index of `i` on an axis of length n whose CPML slabs are
// [0, lo) and [n-hi, n); -1 outside both slabs.
__host__ __device__ __forceinline__ int slab_index(int i, int n, int lo, int hi) {
  return i < lo ? i : (i >= n - hi ? i - (n - hi) + lo : -1);
}

// coefficient table rows (sw_pml_axis.coef): 6 rows of n values
enum { CB = 0, CA = 1, CK = 2, CBH = 3, CAH = 4, CKH = 5 };

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
  T* split;                 // SPML: 24 full-grid arrays
  // source
  int src_kind, si, sj, sk;
  const T* wav;
  T mneg[6];                // -M_ab (xx yy zz xy xz yz) in the field type
  // receivers
  int nrec, rec_field, rec_f64;
  const long long* rec_idx;
  void* rec_data;
  int x_chunk;              // x planes streamed by one CTA
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
};

template <typename T>
__device__ __forceinline__ T ldg(const T* p) { return __ldg(p); }

// receiver sample in the trace's element type
template <typename T>
__device__ __forceinline__ void store_rec(void* data, int f64, long long at, T v) {
  if (f64) ((double*)data)[at] = (double)v;
  else ((float*)data)[at] = (float)v;
}

}  // namespace sw
