// learned_abc.cu -- the learned thin absorbing layer of the 2D VS solver and
// the training kernels of its network.  No reference counterpart: it sits
// behind Elastic2D_CPML's thin CPML (SetADEPML2D, Elastic2D_CPML.py:392-528)
// and corrects the fields of the outer L cells after every time step.
//
// Network (one per face: 0 x-low, 1 x-high, 2 z-low, 3 z-high), float32:
//   x (51) = the five fields vx vz sxx szz sxz, each divided by its scale, on
//            the 3x3 stencil around the cell in the face's frame (offset a
//            along the inward normal, b along the face), then a one-hot of
//            the cell's depth 0..L-1 (L = SW_ABC_DEPTH)
//   h1 = tanh(W1 x + b1) (32), h2 = tanh(W2 h1 + b2) (32), y = W3 h2 + b3 (5)
//   field_q += y_q * oscale_q
// Parameter block of one face: W1[32][51] b1[32] W2[32][32] b2[32] W3[5][32] b3[5].
#include <algorithm>
#include <cuda_runtime.h>

#include "sw_device.cuh"

namespace sw {

constexpr int AI = SW_ABC_INPUTS, AH = SW_ABC_HIDDEN, AO = 5;
constexpr int P_W1 = 0, P_B1 = P_W1 + AH * AI, P_W2 = P_B1 + AH, P_B2 = P_W2 + AH * AH, P_W3 = P_B2 + AH,
              P_B3 = P_W3 + AO * AH, P_N = P_B3 + AO;
static_assert(P_N == SW_ABC_PARAMS, "parameter block layout");

struct AbcArgs {
  const int* cell;       // linear cell index of each layer cell
  const int8_t* face;    // its face 0..3
  const int8_t* depth;   // distance to that face 0..L-1
  int ncell;
  int nx, nz;
  const float* f[5];     // vx vz sxx szz sxz
  float* fw[5];
  float scale[5];        // input scales
  float oscale[5];       // output scales
  const float* params;   // 4 faces x SW_ABC_PARAMS
  float* delta;          // ncell x 5 corrections
  float* x_out;          // ncell x SW_ABC_INPUTS (features) or null
};

// the 3x3 face-frame stencil of cell c, clamped to the grid
__device__ __forceinline__ void abc_features(const AbcArgs& a, int c, float* x) {
  const int g = a.cell[c], fc = a.face[c], d = a.depth[c];
  const int i = g / a.nz, j = g - i * a.nz;
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const int an = p - 1, bt = q - 1;  // inward normal, along the face
      int ii, jj;
      if (fc == 0) { ii = i + an; jj = j + bt; }
      else if (fc == 1) { ii = i - an; jj = j + bt; }
      else if (fc == 2) { ii = i + bt; jj = j + an; }
      else { ii = i + bt; jj = j - an; }
      ii = min(max(ii, 0), a.nx - 1);
      jj = min(max(jj, 0), a.nz - 1);
      const long long s = (long long)ii * a.nz + jj;
#pragma unroll
      for (int f = 0; f < 5; ++f) x[f * 9 + p * 3 + q] = a.f[f][s] / a.scale[f];
    }
#pragma unroll
  for (int k = 0; k < SW_ABC_DEPTH; ++k) x[45 + k] = k == d ? 1.f : 0.f;
}

__device__ __forceinline__ void mlp_forward(const float* P, const float* x, float* h1, float* h2, float* y) {
  for (int o = 0; o < AH; ++o) {
    float s = P[P_B1 + o];
    for (int k = 0; k < AI; ++k) s += P[P_W1 + o * AI + k] * x[k];
    h1[o] = tanhf(s);
  }
  for (int o = 0; o < AH; ++o) {
    float s = P[P_B2 + o];
    for (int k = 0; k < AH; ++k) s += P[P_W2 + o * AH + k] * h1[k];
    h2[o] = tanhf(s);
  }
  for (int o = 0; o < AO; ++o) {
    float s = P[P_B3 + o];
    for (int k = 0; k < AH; ++k) s += P[P_W3 + o * AH + k] * h2[k];
    y[o] = s;
  }
}

// corrections of every layer cell from the current fields (no field written)
__global__ void k_abc_delta(const AbcArgs a) {
  __shared__ float P[4 * SW_ABC_PARAMS];
  for (int q = threadIdx.x; q < 4 * SW_ABC_PARAMS; q += blockDim.x) P[q] = a.params[q];
  __syncthreads();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell) return;
  float x[AI], h1[AH], h2[AH], y[AO];
  abc_features(a, c, x);
  mlp_forward(P + a.face[c] * SW_ABC_PARAMS, x, h1, h2, y);
#pragma unroll
  for (int f = 0; f < AO; ++f) a.delta[(long long)c * AO + f] = y[f] * a.oscale[f];
}

__global__ void k_abc_apply(const AbcArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell) return;
  const int g = a.cell[c];
#pragma unroll
  for (int f = 0; f < AO; ++f) a.fw[f][g] += a.delta[(long long)c * AO + f];
}

__global__ void k_abc_features(const AbcArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell) return;
  float x[AI];
  abc_features(a, c, x);
  for (int k = 0; k < AI; ++k) a.x_out[(long long)c * AI + k] = x[k];
}

// ---- adjoint of the correction (training through the time loop) -------------
// The correction maps the fields F to F + D(F).  Given the adjoint L of the
// corrected fields, its adjoint is L + (dD/dF)^T L: ybar = L[cell] * oscale
// is the adjoint of the network outputs, and the network's input gradient,
// divided by the input scales, is added to L on the 3x3 stencil cells.
// Both kernels read the uncorrected fields through a.f.
struct Lam5 {
  float* f[5];
};

__global__ void k_abc_ybar(const AbcArgs a, const Lam5 lam, float* __restrict__ ybar) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell) return;
  const int g = a.cell[c];
#pragma unroll
  for (int f = 0; f < AO; ++f) ybar[(long long)c * AO + f] = lam.f[f][g] * a.oscale[f];
}

__global__ void k_abc_xbar(const AbcArgs a, const Lam5 lam, const float* __restrict__ ybar) {
  __shared__ float P[4 * SW_ABC_PARAMS];
  for (int q = threadIdx.x; q < 4 * SW_ABC_PARAMS; q += blockDim.x) P[q] = a.params[q];
  __syncthreads();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell) return;
  const float* W = P + a.face[c] * SW_ABC_PARAMS;
  float x[AI], h1[AH], h2[AH], y[AO];
  abc_features(a, c, x);
  mlp_forward(W, x, h1, h2, y);
  float g2[AH], g1[AH];
  for (int k = 0; k < AH; ++k) {
    float s = 0.f;
    for (int o = 0; o < AO; ++o) s += W[P_W3 + o * AH + k] * ybar[(long long)c * AO + o];
    g2[k] = s * (1.f - h2[k] * h2[k]);
  }
  for (int k = 0; k < AH; ++k) {
    float s = 0.f;
    for (int o = 0; o < AH; ++o) s += W[P_W2 + o * AH + k] * g2[o];
    g1[k] = s * (1.f - h1[k] * h1[k]);
  }
  const int gc = a.cell[c], fc = a.face[c];
  const int i = gc / a.nz, j = gc - i * a.nz;
  for (int p = 0; p < 3; ++p)
    for (int q = 0; q < 3; ++q) {
      const int an = p - 1, bt = q - 1;
      int ii, jj;
      if (fc == 0) { ii = i + an; jj = j + bt; }
      else if (fc == 1) { ii = i - an; jj = j + bt; }
      else if (fc == 2) { ii = i + bt; jj = j + an; }
      else { ii = i + bt; jj = j - an; }
      ii = min(max(ii, 0), a.nx - 1);
      jj = min(max(jj, 0), a.nz - 1);
      const long long sidx = (long long)ii * a.nz + jj;
      for (int f = 0; f < 5; ++f) {
        const int k = f * 9 + p * 3 + q;
        float xb = 0.f;
        for (int o = 0; o < AH; ++o) xb += W[P_W1 + o * AI + k] * g1[o];
        atomicAdd(lam.f[f] + sidx, xb / a.scale[f]);
      }
    }
}

cudaError_t abc_adjoint(const AbcArgs& a, float* const* lam_host, float* ybar, cudaStream_t st) {
  if (a.ncell == 0) return cudaSuccess;
  Lam5 lam;
  for (int f = 0; f < 5; ++f) lam.f[f] = lam_host[f];
  const int nb = (a.ncell + 127) / 128;
  k_abc_ybar<<<nb, 128, 0, st>>>(a, lam, ybar);
  k_abc_xbar<<<nb, 128, 0, st>>>(a, lam, ybar);
  return cudaGetLastError();
}

// ---- training: MSE loss and its gradient over n samples of one face --------
// Each block takes tiles of MT samples: one thread per sample runs the forward
// and backward passes and leaves x, h1, h2 and the layer gradients in shared
// memory; then each thread adds its own slice of the weight gradient over the
// tile.  The block's sums go to grad with one atomicAdd per parameter.
constexpr int MT = 128;

// dy_given != 0: Y holds d(loss)/dy itself (the adjoint of the outputs) and
// loss is not touched; otherwise loss = mean |y - Y|^2 over the samples.
__global__ void __launch_bounds__(MT) k_mlp_grad(const float* __restrict__ params, const float* __restrict__ X,
                                                 const float* __restrict__ Y, long long n, float inv_n,
                                                 float* __restrict__ grad, float* __restrict__ loss,
                                                 int dy_given) {
  extern __shared__ float sm[];
  float* P = sm;                               // SW_ABC_PARAMS
  float* sx = P + SW_ABC_PARAMS;               // MT x AI
  float* s1 = sx + MT * AI;                    // MT x AH   h1
  float* s2 = s1 + MT * AH;                    // MT x AH   h2
  float* g1 = s2 + MT * AH;                    // MT x AH   d(pre-activation 1)
  float* g2 = g1 + MT * AH;                    // MT x AH   d(pre-activation 2)
  float* gy = g2 + MT * AH;                    // MT x AO   d y
  for (int q = threadIdx.x; q < SW_ABC_PARAMS; q += MT) P[q] = params[q];
  __syncthreads();
  // this thread's slice of the gradient: parameters q = tid, tid + MT, ...
  constexpr int PER = (SW_ABC_PARAMS + MT - 1) / MT;
  float acc[PER];
#pragma unroll
  for (int r = 0; r < PER; ++r) acc[r] = 0.f;
  float lsum = 0.f;
  const long long ntile = (n + MT - 1) / MT;
  for (long long tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    const long long smp = tile * MT + threadIdx.x;
    const int t = threadIdx.x;
    if (smp < n) {
      float* x = sx + t * AI;
      for (int k = 0; k < AI; ++k) x[k] = X[smp * AI + k];
      float h1[AH], h2[AH], y[AO];
      mlp_forward(P, x, h1, h2, y);
      float dy[AO];
      for (int o = 0; o < AO; ++o) {
        if (dy_given) {
          dy[o] = Y[smp * AO + o];
        } else {
          const float e = y[o] - Y[smp * AO + o];
          lsum += e * e;
          dy[o] = 2.f * e * inv_n;
        }
        gy[t * AO + o] = dy[o];
      }
      for (int k = 0; k < AH; ++k) {
        float s = 0.f;
        for (int o = 0; o < AO; ++o) s += P[P_W3 + o * AH + k] * dy[o];
        g2[t * AH + k] = s * (1.f - h2[k] * h2[k]);
        s1[t * AH + k] = h1[k];
        s2[t * AH + k] = h2[k];
      }
      for (int k = 0; k < AH; ++k) {
        float s = 0.f;
        for (int o = 0; o < AH; ++o) s += P[P_W2 + o * AH + k] * g2[t * AH + o];
        g1[t * AH + k] = s * (1.f - h1[k] * h1[k]);
      }
    } else {
      for (int k = 0; k < AI; ++k) sx[t * AI + k] = 0.f;
      for (int k = 0; k < AH; ++k) { s1[t * AH + k] = s2[t * AH + k] = g1[t * AH + k] = g2[t * AH + k] = 0.f; }
      for (int o = 0; o < AO; ++o) gy[t * AO + o] = 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < PER; ++r) {
      const int q = threadIdx.x + r * MT;
      if (q >= SW_ABC_PARAMS) break;
      float s = 0.f;
      if (q < P_B1) {
        const int o = q / AI, k = q - o * AI;
        for (int m = 0; m < MT; ++m) s += g1[m * AH + o] * sx[m * AI + k];
      } else if (q < P_W2) {
        const int o = q - P_B1;
        for (int m = 0; m < MT; ++m) s += g1[m * AH + o];
      } else if (q < P_B2) {
        const int o = (q - P_W2) / AH, k = (q - P_W2) % AH;
        for (int m = 0; m < MT; ++m) s += g2[m * AH + o] * s1[m * AH + k];
      } else if (q < P_W3) {
        const int o = q - P_B2;
        for (int m = 0; m < MT; ++m) s += g2[m * AH + o];
      } else if (q < P_B3) {
        const int o = (q - P_W3) / AH, k = (q - P_W3) % AH;
        for (int m = 0; m < MT; ++m) s += gy[m * AO + o] * s2[m * AH + k];
      } else {
        const int o = q - P_B3;
        for (int m = 0; m < MT; ++m) s += gy[m * AO + o];
      }
      acc[r] += s;
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < PER; ++r) {
    const int q = threadIdx.x + r * MT;
    if (q < SW_ABC_PARAMS) atomicAdd(grad + q, acc[r]);
  }
  // loss: warp sums, then one atomic per warp
  if (dy_given) return;
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, lsum * inv_n);
}

__global__ void k_mlp_forward(const float* __restrict__ params, const float* __restrict__ X, long long n,
                              float* __restrict__ Y) {
  __shared__ float P[SW_ABC_PARAMS];
  for (int q = threadIdx.x; q < SW_ABC_PARAMS; q += blockDim.x) P[q] = params[q];
  __syncthreads();
  const long long smp = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (smp >= n) return;
  float x[AI], h1[AH], h2[AH], y[AO];
  for (int k = 0; k < AI; ++k) x[k] = X[smp * AI + k];
  mlp_forward(P, x, h1, h2, y);
  for (int o = 0; o < AO; ++o) Y[smp * AO + o] = y[o];
}

size_t mlp_grad_smem() { return sizeof(float) * (SW_ABC_PARAMS + MT * AI + 4 * MT * AH + MT * AO); }

cudaError_t abc_correct(const AbcArgs& a, cudaStream_t st) {
  if (a.ncell == 0) return cudaSuccess;
  const int nb = (a.ncell + 127) / 128;
  k_abc_delta<<<nb, 128, 0, st>>>(a);
  k_abc_apply<<<nb, 128, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t abc_features(const AbcArgs& a, cudaStream_t st) {
  if (a.ncell == 0) return cudaSuccess;
  k_abc_features<<<(a.ncell + 127) / 128, 128, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t mlp_grad(const float* params, const float* X, const float* Y, long long n, float* grad, float* loss,
                     int dy_given, cudaStream_t st) {
  static bool init = false;
  const size_t smem = mlp_grad_smem();
  if (!init) {
    cudaError_t e = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    init = true;
  }
  if (n == 0) return cudaSuccess;
  const long long ntile = (n + MT - 1) / MT;
  const int grid = (int)std::min<long long>(ntile, 148 * 2);
  k_mlp_grad<<<grid, MT, smem, st>>>(params, X, Y, n, 1.f / (float)n, grad, loss, dy_given);
  return cudaGetLastError();
}

cudaError_t mlp_forward_batch(const float* params, const float* X, long long n, float* Y, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_mlp_forward<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(params, X, n, Y);
  return cudaGetLastError();
}

}  // namespace sw
