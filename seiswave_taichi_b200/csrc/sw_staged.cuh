// sw_staged.cuh -- host-visible types of the TMA-staged two-pass 3D kernels.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "sw_device.cuh"

namespace sw {

// velocity pass maps: sxx sxy sxz syy syz szz rho; stress pass: vx vy vz lam mu
struct StagedMaps {
  CUtensorMap m[7];
};

struct StagedArgs {
  int* err;  // error word: bit0 = a TMA wait gave up
  int tiles_y, tiles_z, chunks, chunk_len;
  int exact;  // 1: IEEE-exact reference order (bit-identical to the CPU oracle)
};

struct StagedConfig {
  int N, TY, D, threads;
  size_t vel_smem, str_smem;
};

bool sw3_staged_config(int N, StagedConfig* out);
bool sw3_staged_maps(int N, const P3<float>& p, StagedMaps* vel, StagedMaps* str);
// velocity pass then stress pass of step it, in place
cudaError_t sw3_staged_step(int N, bool tensor, const P3<float>& p, const StagedMaps& vel, const StagedMaps& str,
                            const StagedArgs& a, int grid, int it, bool force_here, bool inject_next, bool gather,
                            cudaStream_t st);

}  // namespace sw
