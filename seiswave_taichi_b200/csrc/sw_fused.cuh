// sw_fused.cuh -- host-visible types of the fused single-pass 3D kernel.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "sw_device.cuh"

namespace sw {

// tensor maps: stress [buffer][sxx syy szz sxy sxz syz], velocity [buffer][vx vy vz], density
struct FusedMaps {
  CUtensorMap sig[2][6];
  CUtensorMap vel[2][3];
  CUtensorMap rho;
};

struct FusedExtra {
  float* fB[9];        // second buffer set of the nine wavefields
  float* memB[3];      // second buffer of the velocity memory variables (3 comps per direction)
  int* err;            // error word: bit0 = a TMA wait gave up
  int tiles_y, tiles_z, chunks, chunk_len;
};

struct FusedConfig {
  int N, TY, D;
  size_t smem;
  int tz;
};

// geometry of the instantiation carried for half-stencil length N (false: none)
bool sw3_fused_config(int N, FusedConfig* out);
// tensor maps over both buffer sets and the density
bool sw3_fused_maps(int N, const P3<float>& p, const FusedExtra& x, FusedMaps* m);
// one fused time step: read buffer set `src`, write the other
cudaError_t sw3_fused_step(int N, bool tensor, const P3<float>& p, const FusedMaps& m, const FusedExtra& x,
                           int grid, int it, int src, bool inject_next, int gather_it, cudaStream_t st);
// exhaustive comparison of the constant-divisor path (div_c) with IEEE
// division for every finite float numerator; *h_bad = number of differing results
cudaError_t sw3_check_divisor(float d, float r, unsigned long long* d_bad, unsigned long long* h_bad,
                              cudaStream_t st, int mode = 0);

}  // namespace sw
