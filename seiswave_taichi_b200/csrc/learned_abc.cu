// learned_abc.cu -- the learned thin absorbing layers of the 2D VS and 3D
// moment-tensor solvers and the training kernels of their networks.  No
// reference counterpart: the layer sits behind a thin CPML built by the
// reference's SetADEPML2D / SetADEPML3D (Elastic2D_CPML.py:392-528,
// Elastic3D_SSG_Tensor.py:361-568) and corrects the fields of the outer
// L = SW_ABC_DEPTH cells after every time step.
//
// Networks (one per face; float32), two tanh layers of SW_ABC_HIDDEN:
//   2D: faces 0 x-low, 1 x-high, 2 z-low, 3 z-high; x (51) = the five fields
//       vx vz sxx szz sxz / scale on the 3x3 stencil around the cell in the
//       face's frame (offset a along the inward normal, b along the face),
//       then a one-hot of the cell's depth; 5 outputs.
//   3D: faces 0 x-low .. 5 z-high; x (33) = the nine fields / scale at the
//       cell and its two neighbours along the inward normal, then the depth
//       one-hot; 9 outputs.
//   h1 = tanh(W1 x + b1), h2 = tanh(W2 h1 + b2), y = W3 h2 + b3,
//   field_q += y_q * oscale_q.
// Parameter block of one face: W1[H][I] b1[H] W2[H][H] b2[H] W3[O][H] b3[O].
#include <algorithm>
#include <cuda_runtime.h>

#include "sw_device.cuh"

namespace sw {

template <int NI_, int NO_>
struct Net {
  static constexpr int NI = NI_, NO = NO_, NH = SW_ABC_HIDDEN;
  static constexpr int W1 = 0, B1 = W1 + NH * NI, W2 = B1 + NH, B2 = W2 + NH * NH, W3 = B2 + NH, B3 = W3 + NO * NH,
                       N = B3 + NO;
};
using Net2 = Net<SW_ABC_INPUTS, 5>;
using Net3 = Net<SW_ABC3_INPUTS, 9>;
static_assert(Net2::N == SW_ABC_PARAMS, "2D parameter block layout");
static_assert(Net3::N == SW_ABC3_PARAMS, "3D parameter block layout");

// The networks' tanh, from tanh(x) = 1 - 2 / (exp(2|x|) + 1) with the sign of
// x put back, on the fast exponential and division intrinsics (absolute error
// below 1e-6; 1 for |x| beyond the float exponential's range).  Training and
// the correction use this one function, and the backward passes take
// 1 - h^2 as its derivative.
__device__ __forceinline__ float act(float s) {
  const float e = __expf(2.f * fabsf(s));
  return copysignf(1.f - __fdividef(2.f, e + 1.f), s);
}

// Every pre-activation is b_o followed by fused multiply-adds over k in
// increasing order, so the generic form below and the transposed
// shared-memory form of the correction kernels give identical bits.
template <class NT>
__device__ __forceinline__ void mlp_forward(const float* P, const float* x, float* h1, float* h2, float* y) {
  for (int o = 0; o < NT::NH; ++o) {
    float s = P[NT::B1 + o];
    for (int k = 0; k < NT::NI; ++k) s = fmaf(P[NT::W1 + o * NT::NI + k], x[k], s);
    h1[o] = act(s);
  }
  for (int o = 0; o < NT::NH; ++o) {
    float s = P[NT::B2 + o];
    for (int k = 0; k < NT::NH; ++k) s = fmaf(P[NT::W2 + o * NT::NH + k], h1[k], s);
    h2[o] = act(s);
  }
  for (int o = 0; o < NT::NO; ++o) {
    float s = P[NT::B3 + o];
    for (int k = 0; k < NT::NH; ++k) s = fmaf(P[NT::W3 + o * NT::NH + k], h2[k], s);
    y[o] = s;
  }
}

// Transposed block of one face in shared memory for the correction kernels:
// W1t[NI][NH] b1[NH] W2t[NH][NH] b2[NH] W3t[NH][NOP] b3[NOP], NOP = NO
// rounded up to 4 (zero padded), so a warp reads four consecutive outputs'
// weights of one input with one 16-byte broadcast load.
template <class NT>
struct TNet {
  static constexpr int NI = NT::NI, NH = NT::NH, NO = NT::NO, NOP = (NO + 3) & ~3;
  static constexpr int W1 = 0, B1 = W1 + NI * NH, W2 = B1 + NH, B2 = W2 + NH * NH, W3 = B2 + NH,
                       B3 = W3 + NH * NOP, N = B3 + NOP;
  static_assert(N % 4 == 0 && NH % 4 == 0, "16-byte rows");
  // parameter of the packed block behind transposed slot q, or -1 (padding)
  __device__ static int src(int q) {
    if (q < B1) { const int k = q / NH, o = q - k * NH; return NT::W1 + o * NI + k; }
    if (q < W2) return NT::B1 + (q - B1);
    if (q < B2) { const int r = q - W2, k = r / NH, o = r - k * NH; return NT::W2 + o * NH + k; }
    if (q < W3) return NT::B2 + (q - B2);
    if (q < B3) { const int r = q - W3, k = r / NOP, o = r - k * NOP; return o < NO ? NT::W3 + o * NH + k : -1; }
    const int o = q - B3;
    return o < NO ? NT::B3 + o : -1;
  }
};

template <class NT>
__device__ void tnet_load(float* T, const float* __restrict__ params, int nface) {
  using TN = TNet<NT>;
  for (int q = threadIdx.x; q < nface * TN::N; q += blockDim.x) {
    const int f = q / TN::N, r = TN::src(q - f * TN::N);
    T[q] = r < 0 ? 0.f : params[f * NT::N + r];
  }
}

// The correction kernels keep each layer's pre-activations as pairs and use
// the packed two-lane FMA (__ffma2_rn, sm_100): each lane is one fmaf with
// the same operands and order as the generic form above, so the bits are the
// same, with half the FMA instructions.

// bias block b[2P] into s
template <int P>
__device__ __forceinline__ void tload(const float* __restrict__ b, float2 (&s)[P]) {
#pragma unroll
  for (int o = 0; o < P; o += 2) {
    const float4 v = *reinterpret_cast<const float4*>(b + 2 * o);
    s[o] = make_float2(v.x, v.y);
    s[o + 1] = make_float2(v.z, v.w);
  }
}

// s += W^T col for a transposed W[nin][2P]; col holds this thread's inputs at
// stride CT (its own column of the block's buffer)
template <int P, int NIN, int U, int CT>
__device__ __forceinline__ void tdense(const float* __restrict__ W, const float* col, float2 (&s)[P]) {
#pragma unroll U
  for (int k = 0; k < NIN; ++k) {
    const float xk = col[k * CT];
    const float2 x2 = make_float2(xk, xk);
#pragma unroll
    for (int o = 0; o < P; o += 2) {
      const float4 v = *reinterpret_cast<const float4*>(W + k * 2 * P + 2 * o);
      s[o] = __ffma2_rn(make_float2(v.x, v.y), x2, s[o]);
      s[o + 1] = __ffma2_rn(make_float2(v.z, v.w), x2, s[o + 1]);
    }
  }
}

// forward pass of one cell from the transposed block T; col holds the NI
// inputs on entry and is reused for the hidden layers
template <class NT, int CT>
__device__ __forceinline__ void mlp_forward_t(const float* __restrict__ T, float* col, float* y) {
  using TN = TNet<NT>;
  float2 s[TN::NH / 2];
  tload(T + TN::B1, s);
  tdense<TN::NH / 2, TN::NI, 3, CT>(T + TN::W1, col, s);
#pragma unroll
  for (int o = 0; o < TN::NH / 2; ++o) {
    col[(2 * o) * CT] = act(s[o].x);
    col[(2 * o + 1) * CT] = act(s[o].y);
  }
  tload(T + TN::B2, s);
  tdense<TN::NH / 2, TN::NH, 4, CT>(T + TN::W2, col, s);
#pragma unroll
  for (int o = 0; o < TN::NH / 2; ++o) {
    col[(2 * o) * CT] = act(s[o].x);
    col[(2 * o + 1) * CT] = act(s[o].y);
  }
  float2 t[TN::NOP / 2];
  tload(T + TN::B3, t);
  tdense<TN::NOP / 2, TN::NH, 4, CT>(T + TN::W3, col, t);
#pragma unroll
  for (int o = 0; o < TN::NO; ++o) y[o] = (o & 1) ? t[o / 2].y : t[o / 2].x;
}

// correction-kernel blocks: the faces' transposed blocks, then one column of
// max(NI, NH) floats per thread
constexpr int CT2 = 256, CT3 = 384;
template <class NT>
constexpr size_t corr_smem(int nface, int ct) {
  return sizeof(float) * ((size_t)nface * TNet<NT>::N + (size_t)ct * (NT::NI > NT::NH ? NT::NI : NT::NH));
}

// correction-kernel grid: the whole layer in a grid-stride loop over two
// blocks per SM, so each block fills its transposed weights once
static int corr_grid(int ncell, int threads) {
  int dev = 0, nsm = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const long long need = ((long long)ncell + threads - 1) / threads;
  return (int)std::max<long long>(1, std::min<long long>(need, 2LL * nsm));
}

// adjoint of the first pre-activation (g1) from the output adjoint ybar
template <class NT>
__device__ __forceinline__ void mlp_input_grad(const float* P, const float* h1, const float* h2, const float* ybar,
                                               float* g1) {
  float g2[NT::NH];
  for (int k = 0; k < NT::NH; ++k) {
    float s = 0.f;
    for (int o = 0; o < NT::NO; ++o) s += P[NT::W3 + o * NT::NH + k] * ybar[o];
    g2[k] = s * (1.f - h2[k] * h2[k]);
  }
  for (int k = 0; k < NT::NH; ++k) {
    float s = 0.f;
    for (int o = 0; o < NT::NH; ++o) s += P[NT::W2 + o * NT::NH + k] * g2[o];
    g1[k] = s * (1.f - h1[k] * h1[k]);
  }
}

template <int K>
struct LamK {
  float* f[K];
};

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

// ======================================================================
// 2D layer: the 3x3 face-frame stencil of cell c, clamped to the grid
// ======================================================================
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

// corrections of every layer cell from the current fields (no field written)
// dynamic shared memory: the four faces' transposed blocks
__global__ void __launch_bounds__(CT2) k_abc_delta(const AbcArgs a) {
  extern __shared__ float4 T2v[];
  float* T = reinterpret_cast<float*>(T2v);
  float* col = T + 4 * TNet<Net2>::N + threadIdx.x;
  tnet_load<Net2>(T, a.params, 4);
  __syncthreads();
  for (int c = blockIdx.x * CT2 + threadIdx.x; c < a.ncell; c += gridDim.x * CT2) {
    float x[Net2::NI], y[Net2::NO];
    abc_features(a, c, x);
#pragma unroll
    for (int k = 0; k < Net2::NI; ++k) col[k * CT2] = x[k];
    mlp_forward_t<Net2, CT2>(T + a.face[c] * TNet<Net2>::N, col, y);
#pragma unroll
    for (int f = 0; f < 5; ++f) a.delta[(long long)c * 5 + f] = y[f] * a.oscale[f];
  }
}

__global__ void k_abc_apply(const AbcArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell) return;
  const int g = a.cell[c];
#pragma unroll
  for (int f = 0; f < 5; ++f) a.fw[f][g] += a.delta[(long long)c * 5 + f];
}

__global__ void k_abc_features(const AbcArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell) return;
  float x[Net2::NI];
  abc_features(a, c, x);
  for (int k = 0; k < Net2::NI; ++k) a.x_out[(long long)c * Net2::NI + k] = x[k];
}

// ---- adjoint of the correction (training through the time loop) -------------
// The correction maps the fields F to F + D(F).  Given the adjoint L of the
// corrected fields, its adjoint is L + (dD/dF)^T L: ybar = L[cell] * oscale
// is the adjoint of the network outputs, and the network's input gradient,
// divided by the input scales, is added to L on the 3x3 stencil cells.
// Both kernels read the uncorrected fields through a.f.
__global__ void k_abc_ybar(const AbcArgs a, const LamK<5> lam, float* __restrict__ ybar) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell) return;
  const int g = a.cell[c];
#pragma unroll
  for (int f = 0; f < 5; ++f) ybar[(long long)c * 5 + f] = lam.f[f][g] * a.oscale[f];
}

__global__ void k_abc_xbar(const AbcArgs a, const LamK<5> lam, const float* __restrict__ ybar) {
  __shared__ float P[4 * SW_ABC_PARAMS];
  for (int q = threadIdx.x; q < 4 * SW_ABC_PARAMS; q += blockDim.x) P[q] = a.params[q];
  __syncthreads();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell) return;
  const float* W = P + a.face[c] * SW_ABC_PARAMS;
  float x[Net2::NI], h1[Net2::NH], h2[Net2::NH], y[Net2::NO];
  abc_features(a, c, x);
  mlp_forward<Net2>(W, x, h1, h2, y);
  float g1[Net2::NH];
  mlp_input_grad<Net2>(W, h1, h2, ybar + (long long)c * 5, g1);
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
        for (int o = 0; o < Net2::NH; ++o) xb += W[Net2::W1 + o * Net2::NI + k] * g1[o];
        atomicAdd(lam.f[f] + sidx, xb / a.scale[f]);
      }
    }
}

cudaError_t abc_adjoint(const AbcArgs& a, float* const* lam_host, float* ybar, cudaStream_t st) {
  if (a.ncell == 0) return cudaSuccess;
  LamK<5> lam;
  for (int f = 0; f < 5; ++f) lam.f[f] = lam_host[f];
  const int nb = (a.ncell + 127) / 128;
  k_abc_ybar<<<nb, 128, 0, st>>>(a, lam, ybar);
  k_abc_xbar<<<nb, 128, 0, st>>>(a, lam, ybar);
  return cudaGetLastError();
}

cudaError_t abc_correct(const AbcArgs& a, cudaStream_t st) {
  if (a.ncell == 0) return cudaSuccess;
  static std::atomic<unsigned long long> done{0};
  static std::mutex mu;
  const int sm = (int)corr_smem<Net2>(4, CT2);
  cudaError_t e = once_per_device(done, mu, [sm] {
    return cudaFuncSetAttribute(k_abc_delta, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  });
  if (e != cudaSuccess) return e;
  k_abc_delta<<<corr_grid(a.ncell, CT2), CT2, sm, st>>>(a);
  k_abc_apply<<<(a.ncell + 127) / 128, 128, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t abc_features(const AbcArgs& a, cudaStream_t st) {
  if (a.ncell == 0) return cudaSuccess;
  k_abc_features<<<(a.ncell + 127) / 128, 128, 0, st>>>(a);
  return cudaGetLastError();
}

// ======================================================================
// 3D layer
// ======================================================================
struct AbcArgs3 {
  const int* cell;       // linear cell index (i*ny + j)*nz + k of each layer cell
  const int8_t* face;    // its face 0..5
  const int8_t* depth;
  int ncell;
  int nx, ny, nz;
  const float* f[9];     // vx vy vz sxx syy szz sxy sxz syz
  float* fw[9];
  float scale[9];
  float oscale[9];
  const float* params;   // 6 faces x SW_ABC3_PARAMS
  float* delta;          // ncell x 9
  float* x_out;          // ncell x SW_ABC3_INPUTS or null
};

// cell at offset an along the inward normal of face fc, clamped to the grid
__device__ __forceinline__ long long abc_cell3(const AbcArgs3& a, int fc, int i, int j, int k, int an) {
  const int ax = fc >> 1, sg = (fc & 1) ? -1 : 1;
  if (ax == 0) i = min(max(i + sg * an, 0), a.nx - 1);
  else if (ax == 1) j = min(max(j + sg * an, 0), a.ny - 1);
  else k = min(max(k + sg * an, 0), a.nz - 1);
  return ((long long)i * a.ny + j) * a.nz + k;
}

__device__ __forceinline__ void abc3_ijk(const AbcArgs3& a, int g, int& i, int& j, int& k) {
  k = g % a.nz;
  const int r = g / a.nz;
  j = r % a.ny;
  i = r / a.ny;
}

__device__ __forceinline__ void abc3_features(const AbcArgs3& a, int c, float* x) {
  int i, j, k;
  abc3_ijk(a, a.cell[c], i, j, k);
  const int fc = a.face[c], d = a.depth[c];
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    const long long s = abc_cell3(a, fc, i, j, k, p - 1);
#pragma unroll
    for (int f = 0; f < 9; ++f) x[f * 3 + p] = a.f[f][s] / a.scale[f];
  }
#pragma unroll
  for (int q = 0; q < SW_ABC_DEPTH; ++q) x[27 + q] = q == d ? 1.f : 0.f;
}

// dynamic shared memory: the six faces' parameter blocks
__global__ void __launch_bounds__(CT3) k_abc3_delta(const AbcArgs3 a) {
  extern __shared__ float4 T3v[];
  float* T = reinterpret_cast<float*>(T3v);
  float* col = T + 6 * TNet<Net3>::N + threadIdx.x;
  tnet_load<Net3>(T, a.params, 6);
  __syncthreads();
  for (int c = blockIdx.x * CT3 + threadIdx.x; c < a.ncell; c += gridDim.x * CT3) {
    float x[Net3::NI], y[Net3::NO];
    abc3_features(a, c, x);
#pragma unroll
    for (int k = 0; k < Net3::NI; ++k) col[k * CT3] = x[k];
    mlp_forward_t<Net3, CT3>(T + a.face[c] * TNet<Net3>::N, col, y);
#pragma unroll
    for (int f = 0; f < 9; ++f) a.delta[(long long)c * 9 + f] = y[f] * a.oscale[f];
  }
}

__global__ void k_abc3_apply(const AbcArgs3 a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell) return;
  const int g = a.cell[c];
#pragma unroll
  for (int f = 0; f < 9; ++f) a.fw[f][g] += a.delta[(long long)c * 9 + f];
}

__global__ void k_abc3_features(const AbcArgs3 a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell) return;
  float x[Net3::NI];
  abc3_features(a, c, x);
  for (int k = 0; k < Net3::NI; ++k) a.x_out[(long long)c * Net3::NI + k] = x[k];
}

__global__ void k_abc3_ybar(const AbcArgs3 a, const LamK<9> lam, float* __restrict__ ybar) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell) return;
  const int g = a.cell[c];
#pragma unroll
  for (int f = 0; f < 9; ++f) ybar[(long long)c * 9 + f] = lam.f[f][g] * a.oscale[f];
}

__global__ void k_abc3_xbar(const AbcArgs3 a, const LamK<9> lam, const float* __restrict__ ybar) {
  extern __shared__ float P3s[];
  for (int q = threadIdx.x; q < 6 * SW_ABC3_PARAMS; q += blockDim.x) P3s[q] = a.params[q];
  __syncthreads();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell) return;
  const float* W = P3s + a.face[c] * SW_ABC3_PARAMS;
  float x[Net3::NI], h1[Net3::NH], h2[Net3::NH], y[Net3::NO], g1[Net3::NH];
  abc3_features(a, c, x);
  mlp_forward<Net3>(W, x, h1, h2, y);
  mlp_input_grad<Net3>(W, h1, h2, ybar + (long long)c * 9, g1);
  int i, j, k;
  abc3_ijk(a, a.cell[c], i, j, k);
  const int fc = a.face[c];
  for (int p = 0; p < 3; ++p) {
    const long long sidx = abc_cell3(a, fc, i, j, k, p - 1);
    for (int f = 0; f < 9; ++f) {
      const int q = f * 3 + p;
      float xb = 0.f;
      for (int o = 0; o < Net3::NH; ++o) xb += W[Net3::W1 + o * Net3::NI + q] * g1[o];
      atomicAdd(lam.f[f] + sidx, xb / a.scale[f]);
    }
  }
}

static size_t abc3_smem() { return sizeof(float) * 6 * SW_ABC3_PARAMS; }
static size_t abc3_tsmem() { return corr_smem<Net3>(6, CT3); }

static cudaError_t abc3_init() {
  static std::atomic<unsigned long long> done{0};
  static std::mutex mu;
  return once_per_device(done, mu, [] {
    cudaError_t e =
        cudaFuncSetAttribute(k_abc3_delta, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)abc3_tsmem());
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_abc3_xbar, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)abc3_smem());
    return e;
  });
}

cudaError_t abc3_correct(const AbcArgs3& a, cudaStream_t st) {
  if (a.ncell == 0) return cudaSuccess;
  cudaError_t e = abc3_init();
  if (e != cudaSuccess) return e;
  k_abc3_delta<<<corr_grid(a.ncell, CT3), CT3, abc3_tsmem(), st>>>(a);
  k_abc3_apply<<<(a.ncell + 127) / 128, 128, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t abc3_features(const AbcArgs3& a, cudaStream_t st) {
  if (a.ncell == 0) return cudaSuccess;
  k_abc3_features<<<(a.ncell + 127) / 128, 128, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t abc3_adjoint(const AbcArgs3& a, float* const* lam_host, float* ybar, cudaStream_t st) {
  if (a.ncell == 0) return cudaSuccess;
  cudaError_t e = abc3_init();
  if (e != cudaSuccess) return e;
  LamK<9> lam;
  for (int f = 0; f < 9; ++f) lam.f[f] = lam_host[f];
  const int nb = (a.ncell + 127) / 128;
  k_abc3_ybar<<<nb, 128, 0, st>>>(a, lam, ybar);
  k_abc3_xbar<<<nb, 128, abc3_smem(), st>>>(a, lam, ybar);
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
template <class NT>
__global__ void __launch_bounds__(MT) k_mlp_grad(const float* __restrict__ params, const float* __restrict__ X,
                                                 const float* __restrict__ Y, long long n, float inv_n,
                                                 float* __restrict__ grad, float* __restrict__ loss,
                                                 int dy_given) {
  constexpr int AI = NT::NI, AH = NT::NH, AO = NT::NO;
  extern __shared__ float sm[];
  float* P = sm;                               // NT::N
  float* sx = P + NT::N;                       // MT x AI
  float* s1 = sx + MT * AI;                    // MT x AH   h1
  float* s2 = s1 + MT * AH;                    // MT x AH   h2
  float* g1 = s2 + MT * AH;                    // MT x AH   d(pre-activation 1)
  float* g2 = g1 + MT * AH;                    // MT x AH   d(pre-activation 2)
  float* gy = g2 + MT * AH;                    // MT x AO   d y
  for (int q = threadIdx.x; q < NT::N; q += MT) P[q] = params[q];
  __syncthreads();
  // this thread's slice of the gradient: parameters q = tid, tid + MT, ...
  constexpr int PER = (NT::N + MT - 1) / MT;
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
      mlp_forward<NT>(P, x, h1, h2, y);
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
        for (int o = 0; o < AO; ++o) s += P[NT::W3 + o * AH + k] * dy[o];
        g2[t * AH + k] = s * (1.f - h2[k] * h2[k]);
        s1[t * AH + k] = h1[k];
        s2[t * AH + k] = h2[k];
      }
      for (int k = 0; k < AH; ++k) {
        float s = 0.f;
        for (int o = 0; o < AH; ++o) s += P[NT::W2 + o * AH + k] * g2[t * AH + o];
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
      if (q >= NT::N) break;
      float s = 0.f;
      if (q < NT::B1) {
        const int o = q / AI, k = q - o * AI;
        for (int m = 0; m < MT; ++m) s += g1[m * AH + o] * sx[m * AI + k];
      } else if (q < NT::W2) {
        const int o = q - NT::B1;
        for (int m = 0; m < MT; ++m) s += g1[m * AH + o];
      } else if (q < NT::B2) {
        const int o = (q - NT::W2) / AH, k = (q - NT::W2) % AH;
        for (int m = 0; m < MT; ++m) s += g2[m * AH + o] * s1[m * AH + k];
      } else if (q < NT::W3) {
        const int o = q - NT::B2;
        for (int m = 0; m < MT; ++m) s += g2[m * AH + o];
      } else if (q < NT::B3) {
        const int o = (q - NT::W3) / AH, k = (q - NT::W3) % AH;
        for (int m = 0; m < MT; ++m) s += gy[m * AO + o] * s2[m * AH + k];
      } else {
        const int o = q - NT::B3;
        for (int m = 0; m < MT; ++m) s += gy[m * AO + o];
      }
      acc[r] += s;
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < PER; ++r) {
    const int q = threadIdx.x + r * MT;
    if (q < NT::N) atomicAdd(grad + q, acc[r]);
  }
  // loss: warp sums, then one atomic per warp
  if (dy_given) return;
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, lsum * inv_n);
}

template <class NT>
__global__ void k_mlp_forward(const float* __restrict__ params, const float* __restrict__ X, long long n,
                              float* __restrict__ Y) {
  __shared__ float P[NT::N];
  for (int q = threadIdx.x; q < NT::N; q += blockDim.x) P[q] = params[q];
  __syncthreads();
  const long long smp = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (smp >= n) return;
  float x[NT::NI], h1[NT::NH], h2[NT::NH], y[NT::NO];
  for (int k = 0; k < NT::NI; ++k) x[k] = X[smp * NT::NI + k];
  mlp_forward<NT>(P, x, h1, h2, y);
  for (int o = 0; o < NT::NO; ++o) Y[smp * NT::NO + o] = y[o];
}

template <class NT>
static size_t mlp_grad_smem() {
  return sizeof(float) * (NT::N + MT * NT::NI + 4 * MT * NT::NH + MT * NT::NO);
}

template <class NT>
static cudaError_t mlp_grad_t(const float* params, const float* X, const float* Y, long long n, float* grad,
                              float* loss, int dy_given, cudaStream_t st) {
  static std::atomic<unsigned long long> done{0};
  static std::mutex mu;
  const size_t smem = mlp_grad_smem<NT>();
  cudaError_t e = once_per_device(done, mu, [smem] {
    return cudaFuncSetAttribute(k_mlp_grad<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  });
  if (e != cudaSuccess) return e;
  if (n == 0) return cudaSuccess;
  const long long ntile = (n + MT - 1) / MT;
  const int grid = (int)std::min<long long>(ntile, 148 * 2);
  k_mlp_grad<NT><<<grid, MT, smem, st>>>(params, X, Y, n, 1.f / (float)n, grad, loss, dy_given);
  return cudaGetLastError();
}

cudaError_t mlp_grad(const float* params, const float* X, const float* Y, long long n, float* grad, float* loss,
                     int dy_given, cudaStream_t st) {
  return mlp_grad_t<Net2>(params, X, Y, n, grad, loss, dy_given, st);
}

cudaError_t mlp3_grad(const float* params, const float* X, const float* Y, long long n, float* grad, float* loss,
                      int dy_given, cudaStream_t st) {
  return mlp_grad_t<Net3>(params, X, Y, n, grad, loss, dy_given, st);
}

cudaError_t mlp_forward_batch(const float* params, const float* X, long long n, float* Y, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_mlp_forward<Net2><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(params, X, n, Y);
  return cudaGetLastError();
}

cudaError_t mlp3_forward_batch(const float* params, const float* X, long long n, float* Y, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_mlp_forward<Net3><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(params, X, n, Y);
  return cudaGetLastError();
}

}  // namespace sw
