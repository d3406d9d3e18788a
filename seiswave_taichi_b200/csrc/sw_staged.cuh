// sw_staged.cuh -- host-visible types of the TMA-staged two-pass 3D kernels.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "sw_device.cuh"

namespace sw {

// velocity pass maps: sxx sxy sxz syy syz szz rho vx vy vz; stress pass:
// vx vy vz lam mu sxx syy szz sxy sxz syz
struct StagedMaps {
  CUtensorMap m[11];
};

struct StagedArgs {
  int* err;  // error word: bit0 = a TMA wait gave up
  int tiles_y, tiles_z, chunks, chunk_len;
  int exact;  // 1: IEEE-exact reference order (bit-identical to the CPU oracle)
};

// tile of TY rows x TZ z cells (TZ 32 or 40), D planes prefetched
struct StagedConfig {
  int N, TY, D, TZ, threads;
  size_t vel_smem, str_smem;
};

bool sw3_staged_config(int N, int tz, StagedConfig* out);
bool sw3_staged_maps(int N, int tz, const P3<float>& p, StagedMaps* vel, StagedMaps* str);
// velocity pass then stress pass of step it, in place; spml: the
// split-field PML scheme (exact numerics), else the CPML schemes.  Each pass
// gets as many CTAs as fit on the device at once (at most one per work unit).
cudaError_t sw3_staged_step(int N, int tz, bool spml, bool tensor, const P3<float>& p, const StagedMaps& vel,
                            const StagedMaps& str, const StagedArgs& a, int it, bool force_here, bool inject_next,
                            bool gather, cudaStream_t st);
// the CTAs sw3_staged_step launches for each pass over `units` work units
cudaError_t sw3_staged_grid(int N, int tz, bool spml, bool tensor, bool exact, int units, int* vel, int* str);

}  // namespace sw
