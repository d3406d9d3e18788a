// elastic3d_staged.cu -- TMA-staged two-pass 3D SSG-CPML time step (float),
// the default path of the moment-tensor and point-force schemes
// (src/Elastic3D_SSG_Tensor.py:166-345, src/Elastic3D_SSG_CPML.py:144-309).
//
//   k3s_velocity  vx vy vz (+ point force)               reference :194-243
//   k3s_stress    sxx syy szz sxy sxz syz (+ receivers,  reference :245-310
//                 + next step's moment-tensor source)
//
// Each CTA owns a TY x 32 (y x z) column tile and streams x planes.  One
// elected thread issues cp.async.bulk.tensor loads of whole plane tiles (with
// the halo each array needs) into shared-memory rings, D planes ahead,
// completing on mbarriers; x taps come from the ring planes, y and z taps from
// the halo.  Every thread updates Q consecutive z cells (a "quad", Q = 2 or
// 4, moved with 8- or 16-byte shared and global accesses).  A tile plane that lies inside every update range and
// outside every CPML slab takes a branch-free path; the others evaluate the
// update ranges per cell and the CPML memory variables on their slabs.
// Arithmetic follows the reference's operation order with -fmad=false, exact
// division (div_c / div_v), so results equal the CPU oracle bit for bit.
#include <cudaTypedefs.h>

#include "sw_device.cuh"
#include "sw_staged.cuh"
#include "sw_tma.cuh"

namespace sw {

// z cells per thread: 2 in exact mode, 4 in fast mode.  With two cells per
// thread the exact velocity pass is bound to three 256-thread CTAs per SM
// (80 registers, 16/32 bytes of spills: 24 resident warps) and the stress
// pass to two (128 registers, no spills: 16 warps), against 12 warps for
// four cells (three 128-thread CTAs at 160-168 registers); the extra warps
// hide more of the exact arithmetic's dependent chains.  Measured on B200 at
// 200^3 (exact, steps 300-500 / 600-800 us per step): 793 / 601, against
// 835 / 626 with both passes at three CTAs, 823 / 664 with both at two,
// 774 / 691 with one cell per thread and 1215 / 746 with four.  The fast
// kernels, with shorter chains, keep four cells (482 us; 594 with two).
constexpr int staged_q(bool exact) { return exact ? 2 : 4; }

template <int N, int TY, int D, int Q>
struct SG {
  static constexpr int TZ = 32;
  static constexpr int CQ = TZ / Q;            // threads along z: Q cells each
  static constexpr int NT = TY * CQ;
  static constexpr int MINB = 3;              // CTAs per SM the register budget aims at
  static constexpr int MINB_S = Q == 4 ? 3 : 2;  // same for the stress pass
  static constexpr int H4 = ((N + 3) / 4) * 4; // z halo, rounded to 16 bytes
  static constexpr int WZ = TZ + 2 * H4;       // width of boxes with a z halo
  static constexpr int HY = TY + 2 * N;        // height of boxes with a y halo
  // velocity pass boxes
  static constexpr int B_XX = TZ * TY;         // sxx
  static constexpr int B_Y = TZ * HY;          // sxy, syy
  static constexpr int B_Z = WZ * TY;          // sxz, szz
  static constexpr int B_YZ = WZ * HY;         // syz; vx vy vz in the stress pass
  static constexpr int B_R = TZ * (TY + 1);    // rho (j+1)
  // stress pass boxes
  static constexpr int B_L = TZ * TY;          // lam
  static constexpr int WM = TZ + 4;            // mu (k+1 .. k+Q of the last quad)
  static constexpr int B_M = WM * (TY + 1);    // mu (j+1)
  static constexpr int RX = 2 * N + D;         // rings of arrays with x taps
  static constexpr int R1 = 1 + D;             // rings of in-plane arrays
  static constexpr int R2 = 2 + D;             // rings of two-plane arrays
  static constexpr int pad(int x) { return (x + 31) / 32 * 32; }
  // velocity pass layout (floats)
  static constexpr int V_XX = 0;
  static constexpr int V_XY = V_XX + RX * pad(B_XX);
  static constexpr int V_XZ = V_XY + RX * pad(B_Y);
  static constexpr int V_YY = V_XZ + RX * pad(B_Z);
  static constexpr int V_YZ = V_YY + R1 * pad(B_Y);
  static constexpr int V_ZZ = V_YZ + R1 * pad(B_YZ);
  static constexpr int V_R = V_ZZ + R1 * pad(B_Z);
  static constexpr int V_FLOATS = V_R + R2 * pad(B_R);
  // stress pass layout (floats)
  static constexpr int S_VX = 0;
  static constexpr int S_VY = S_VX + RX * pad(B_YZ);
  static constexpr int S_VZ = S_VY + RX * pad(B_YZ);
  static constexpr int S_L = S_VZ + RX * pad(B_YZ);
  static constexpr int S_M = S_L + R2 * pad(B_L);
  static constexpr int S_FLOATS = S_M + R2 * pad(B_M);
  static constexpr size_t V_BYTES = (size_t)V_FLOATS * 4 + 8 * (D + 1) + 128;
  static constexpr size_t S_BYTES = (size_t)S_FLOATS * 4 + 8 * (D + 1) + 128;
  static_assert(N <= 4 || H4 >= N, "z window");
};

// Q consecutive z cells of one thread (Q = 2 or 4): the float2 / float4
// vector type itself, moved with one 8- or 16-byte access
template <int Q>
struct VecOf;
template <>
struct VecOf<4> {
  using type = float4;
};
template <>
struct VecOf<2> {
  using type = float2;
};
template <int Q>
using Vq = typename VecOf<Q>::type;

template <int Q>
__device__ __forceinline__ Vq<Q> ldq(const float* p) {
  return *reinterpret_cast<const Vq<Q>*>(p);
}
template <int Q>
__device__ __forceinline__ void stq(float* p, const Vq<Q>& a) {
  *reinterpret_cast<Vq<Q>*>(p) = a;
}
template <int Q>
__device__ __forceinline__ Vq<Q> ldgq(const float* p) {
  return __ldg(reinterpret_cast<const Vq<Q>*>(p));
}
__device__ __forceinline__ float g4(const float4& v, int e) { return e == 0 ? v.x : e == 1 ? v.y : e == 2 ? v.z : v.w; }
__device__ __forceinline__ void s4(float4& v, int e, float x) {
  if (e == 0) v.x = x; else if (e == 1) v.y = x; else if (e == 2) v.z = x; else v.w = x;
}
__device__ __forceinline__ float g4(const float2& v, int e) { return e == 0 ? v.x : v.y; }
__device__ __forceinline__ void s4(float2& v, int e, float x) {
  if (e == 0) v.x = x; else v.y = x;
}
__device__ __forceinline__ int rslot(int plane, int R) {
  int s = plane % R;
  return s < 0 ? s + R : s;
}

// acc += c * (a - b) lane by lane in the reference's operation order (exact
// mode), or acc = fma(c, a - b, acc) with the spacing folded into c (fast mode)
template <bool EX, int Q>
__device__ __forceinline__ void tapq(Vq<Q>& acc, float c, const Vq<Q>& a, const Vq<Q>& b) {
#pragma unroll
  for (int e = 0; e < Q; ++e)
    s4(acc, e, EX ? g4(acc, e) + c * (g4(a, e) - g4(b, e)) : __fmaf_rn(c, g4(a, e) - g4(b, e), g4(acc, e)));
}

// derivative across ring planes: pl[q] is the plane (centre - N + q + FWD)
template <int N, bool EX, int Q>
__device__ __forceinline__ Vq<Q> dxq(const float* const* pl, int off, const float* c) {
  Vq<Q> v{};
#pragma unroll
  for (int m = 0; m < N; ++m) tapq<EX, Q>(v, c[m], ldq<Q>(pl[N + m] + off), ldq<Q>(pl[N - 1 - m] + off));
  return v;
}
// derivative along a shared-memory stride (y rows): FWD f[+m+1]-f[-m], else f[+m]-f[-m-1]
template <int N, bool FWD, bool EX, int Q>
__device__ __forceinline__ Vq<Q> dyq(const float* s, int off, int stride, const float* c) {
  Vq<Q> v{};
#pragma unroll
  for (int m = 0; m < N; ++m)
    tapq<EX, Q>(v, c[m], ldq<Q>(s + off + (FWD ? m + 1 : m) * stride), ldq<Q>(s + off - (FWD ? m : m + 1) * stride));
  return v;
}
// derivative along z from one window of aligned vectors around the thread's cells
template <int N, bool FWD, bool EX, int Q>
__device__ __forceinline__ Vq<Q> dzq(const float* s, int off, const float* c) {
  constexpr int H = ((N + 3) / 4) * 4;
  constexpr int NW = (2 * H + Q) / Q;
  float w[Q * NW];
#pragma unroll
  for (int t = 0; t < NW; ++t) {
    const Vq<Q> q = ldq<Q>(s + off - H + Q * t);
#pragma unroll
    for (int e = 0; e < Q; ++e) w[Q * t + e] = g4(q, e);
  }
  float r[Q];
#pragma unroll
  for (int e = 0; e < Q; ++e) r[e] = 0.f;
#pragma unroll
  for (int e = 0; e < Q; ++e)
#pragma unroll
    for (int m = 0; m < N; ++m)
    {
      const float df = FWD ? (w[H + e + m + 1] - w[H + e - m]) : (w[H + e + m] - w[H + e - m - 1]);
      r[e] = EX ? r[e] + c[m] * df : __fmaf_rn(c[m], df, r[e]);
    }
  Vq<Q> o;
#pragma unroll
  for (int e = 0; e < Q; ++e) s4(o, e, r[e]);
  return o;
}

// Exact division of a group of stencil sums by the constant spacings.  When
// the spacings' Markstein path is verified (fast != 0) and every lane is zero
// or of magnitude in [2^-100, 2^100), the whole group runs as one branch-free
// block: the same correction div_c applies to such lanes, with zeros passed
// through unchanged (so the sign of zero is kept).  Otherwise every lane is
// divided in double precision and rounded once to float -- the correctly
// rounded float quotient for every finite float input (innocuous double
// rounding, 53 >= 2*24+2), the same result div_c gives -- again without a
// per-lane branch.  Keeping range tests off the per-lane path leaves the
// group's independent lanes free to interleave.
template <int K, int Q>
__device__ __forceinline__ void div_group(Vq<Q> (&v)[K], const float (&d)[K], const float (&r)[K], int fast) {
  bool ok = fast != 0;
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int e = 0; e < Q; ++e) ok = ok & mk_ok(g4(v[k], e));
  if (ok) {
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
      for (int e = 0; e < Q; ++e) s4(v[k], e, mk_div(g4(v[k], e), d[k], r[k]));
  } else {
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
      for (int e = 0; e < Q; ++e) s4(v[k], e, dd_div(g4(v[k], e), d[k]));
  }
}

// division by a per-cell positive value: exact, or __fdividef in fast mode
template <bool EX>
__device__ __forceinline__ float dvv(float x, float d) {
  return EX ? div_v(x, d) : __fdividef(x, d);
}

// CPML on a quad: x and y slabs are per plane / per row, z per cell.
// comp: memory-variable component; h: 0 integer / 1 half point per axis;
// bits: predicate bits of the three axes (fx, fy, fz per cell).
struct QuadPml {
  int xi, yj, i, j, k;
  uint8_t fx, fy;
};

// Memory variables of one quad on the slabs it lies in, components
// c0 .. c0+2 of each axis: x and y slab rows as vectors, z slab per cell.
// quad_mem_load issues every load before any update, so the latencies of the
// up to nine rows overlap instead of forming one load-update-store chain per
// component and axis; quad_mem_store writes them back after the updates.
template <int Q>
struct QuadMem {
  Vq<Q> x[3], y[3];
  float z[3][Q];
  int zk[Q];
};

__device__ __forceinline__ float* memx_ptr(const P3<float>& p, const QuadPml& q, int comp) {
  return p.mem[0] + comp * p.mcomp[0] + ((size_t)q.xi * p.ny + q.j) * p.nz + q.k;
}
__device__ __forceinline__ float* memy_ptr(const P3<float>& p, const QuadPml& q, int comp) {
  return p.mem[1] + comp * p.mcomp[1] + ((size_t)q.i * p.sn[1] + q.yj) * p.nz + q.k;
}
__device__ __forceinline__ float* memz_ptr(const P3<float>& p, const QuadPml& q, int comp, int zk) {
  return p.mem[2] + comp * p.mcomp[2] + ((size_t)q.i * p.ny + q.j) * p.sn[2] + zk;
}

template <int Q>
__device__ __forceinline__ void quad_mem_load(const P3<float>& p, const QuadPml& q, int c0, QuadMem<Q>& m) {
#pragma unroll
  for (int e = 0; e < Q; ++e) m.zk[e] = q.k + e < p.nz ? slab_index(q.k + e, p.nz, p.lo[2], p.hi[2]) : -1;
  if (q.xi >= 0) {
#pragma unroll
    for (int c = 0; c < 3; ++c) m.x[c] = ldq<Q>(memx_ptr(p, q, c0 + c));
  }
  if (q.yj >= 0) {
#pragma unroll
    for (int c = 0; c < 3; ++c) m.y[c] = ldq<Q>(memy_ptr(p, q, c0 + c));
  }
#pragma unroll
  for (int e = 0; e < Q; ++e)
    if (m.zk[e] >= 0) {
#pragma unroll
      for (int c = 0; c < 3; ++c) m.z[c][e] = *memz_ptr(p, q, c0 + c, m.zk[e]);
    }
}

template <int Q>
__device__ __forceinline__ void quad_mem_store(const P3<float>& p, const QuadPml& q, int c0, const QuadMem<Q>& m) {
  if (q.xi >= 0) {
#pragma unroll
    for (int c = 0; c < 3; ++c) stq<Q>(memx_ptr(p, q, c0 + c), m.x[c]);
  }
  if (q.yj >= 0) {
#pragma unroll
    for (int c = 0; c < 3; ++c) stq<Q>(memy_ptr(p, q, c0 + c), m.y[c]);
  }
#pragma unroll
  for (int e = 0; e < Q; ++e)
    if (m.zk[e] >= 0) {
#pragma unroll
      for (int c = 0; c < 3; ++c) *memz_ptr(p, q, c0 + c, m.zk[e]) = m.z[c][e];
    }
}

// CPML of one derivative quad d on axis AX from the preloaded memory
// variables (component c of m), updated in place
template <int AX, bool EX, int Q>
__device__ __forceinline__ void pml_quad_m(const P3<float>& p, const QuadPml& q, int c, int half, const int* pm,
                                           Vq<Q>& d, QuadMem<Q>& m) {
  const float* cf = p.cf[AX];
  const int n = AX == 0 ? p.nx : AX == 1 ? p.ny : p.nz;
  const int ob = half ? CBH : CB, oa = half ? CAH : CA, ok = half ? CKH : CK;
  if (AX == 0 || AX == 1) {
    const int si = AX == 0 ? q.xi : q.yj;
    if (si < 0) return;
    const int idx = AX == 0 ? q.i : q.j;
    const float b = __ldg(cf + ob * n + idx), a = __ldg(cf + oa * n + idx), kk = __ldg(cf + ok * n + idx);
    Vq<Q>& o = AX == 0 ? m.x[c] : m.y[c];
#pragma unroll
    for (int e = 0; e < Q; ++e) {
      if (!pm[e]) continue;
      const float de = g4(d, e);
      const float psi = b * g4(o, e) + a * de;
      s4(o, e, psi);
      s4(d, e, dvv<EX>(de, kk) + psi);
    }
  } else {
#pragma unroll
    for (int e = 0; e < Q; ++e) {
      if (!pm[e] || m.zk[e] < 0) continue;
      const int kk_ = q.k + e;
      const float b = __ldg(cf + ob * n + kk_), a = __ldg(cf + oa * n + kk_), kk = __ldg(cf + ok * n + kk_);
      const float de = g4(d, e);
      const float psi = b * m.z[c][e] + a * de;
      m.z[c][e] = psi;
      s4(d, e, dvv<EX>(de, kk) + psi);
    }
  }
}

// ---------------------------------------------------------------------------
// velocity pass
// ---------------------------------------------------------------------------
template <int N, int TY, int D, bool TENSOR, bool EX, int Q>
__global__ void __launch_bounds__(SG<N, TY, D, Q>::NT, SG<N, TY, D, Q>::MINB)
k3s_velocity(const __grid_constant__ P3<float> p, const __grid_constant__ StagedMaps maps,
             const __grid_constant__ StagedArgs a, int it, int force_here) {
  using G = SG<N, TY, D, Q>;
  extern __shared__ __align__(128) float sm[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + G::V_FLOATS);
  const int tid = threadIdx.x;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const size_t nyz = (size_t)ny * nz;
  if (tid == 0) {
    for (int b = 0; b <= D; ++b) mbar_init(&bars[b], 1);
    mbar_fence_init();
  }
  __syncthreads();

  // exact mode: c_m then / h; fast mode: c_m / h folded on the host
  float cx[N], cy[N], cz[N];
#pragma unroll
  for (int m = 0; m < N; ++m) {
    cx[m] = EX ? p.c[m] : p.cs[0][m];
    cy[m] = EX ? p.c[m] : p.cs[1][m];
    cz[m] = EX ? p.c[m] : p.cs[2][m];
  }
  const float dx = p.dx, dy = p.dy, dz = p.dz, dt = p.dt;
  const int fast = p.fast_div;
  const float rdx = p.rd[0], rdy = p.rd[1], rdz = p.rd[2];
  const float wf = force_here ? p.wav[it] : 0.f;
  const int r = tid / G::CQ, cq = tid % G::CQ;
  constexpr int PXX = G::pad(G::B_XX), PY = G::pad(G::B_Y), PZ = G::pad(G::B_Z), PYZ = G::pad(G::B_YZ),
                PR = G::pad(G::B_R);
  auto sxx_p = [&](int pl) { return sm + G::V_XX + rslot(pl, G::RX) * PXX; };
  auto sxy_p = [&](int pl) { return sm + G::V_XY + rslot(pl, G::RX) * PY; };
  auto sxz_p = [&](int pl) { return sm + G::V_XZ + rslot(pl, G::RX) * PZ; };
  auto syy_p = [&](int pl) { return sm + G::V_YY + rslot(pl, G::R1) * PY; };
  auto syz_p = [&](int pl) { return sm + G::V_YZ + rslot(pl, G::R1) * PYZ; };
  auto szz_p = [&](int pl) { return sm + G::V_ZZ + rslot(pl, G::R1) * PZ; };
  auto rho_p = [&](int pl) { return sm + G::V_R + rslot(pl, G::R2) * PR; };
  const int o_xx = r * G::TZ + Q * cq;                 // sxx, rho boxes
  const int o_y = (r + N) * G::TZ + Q * cq;            // sxy, syy boxes
  const int o_z = r * G::WZ + G::H4 + Q * cq;          // sxz, szz boxes
  const int o_yz = (r + N) * G::WZ + G::H4 + Q * cq;   // syz box

  const int units = a.tiles_y * a.tiles_z * a.chunks;
  uint32_t g = 0;
  bool ok = true;
  for (int u = blockIdx.x; u < units && ok; u += gridDim.x) {
    const int ch = u % a.chunks;
    const int tzi = (u / a.chunks) % a.tiles_z;
    const int tyi = u / (a.chunks * a.tiles_z);
    const int j0 = tyi * TY, k0 = tzi * G::TZ;
    const int x0 = max(ch * a.chunk_len, N), x1 = min(min((ch + 1) * a.chunk_len, nx - N), nx);
    if (x0 >= x1) continue;
    const int j = j0 + r, k = k0 + Q * cq;
    const bool jin = j < ny, kin = k < nz;
    // tile-level interior test (y and z): every cell inside every update
    // range and outside the CPML slabs
    const bool tile_in = j0 >= N + 1 && j0 + TY <= ny - N - 1 && k0 >= N + 1 && k0 + G::TZ <= nz - N - 1 &&
                         j0 >= p.lo[1] && j0 + TY <= ny - p.hi[1] && k0 >= p.lo[2] && k0 + G::TZ <= nz - p.hi[2];
    const int yj = jin ? slab_index(j, ny, p.lo[1], p.hi[1]) : -1;
    const uint8_t fy = jin ? p.fl[1][j] : 0;
    bool zslab = false;
    uint8_t fz[Q];
#pragma unroll
    for (int e = 0; e < Q; ++e) {
      const int kk = k + e;
      fz[e] = kk < nz ? p.fl[2][kk] : 0;
      zslab = zslab || (kk < nz && slab_index(kk, nz, p.lo[2], p.hi[2]) >= 0);
    }

    auto issue = [&](int s, bool first, uint32_t stage) {
      uint64_t* bar = &bars[stage];
      // sxx + sxy + sxz + syy + syz + szz + rho
      uint32_t bytes = (G::B_XX + 2 * G::B_Y + 2 * G::B_Z + G::B_YZ + G::B_R) * 4;
      if (first) bytes += ((2 * N - 1) * (G::B_XX + G::B_Y + G::B_Z) + G::B_R) * 4;
      mbar_expect_tx(bar, bytes);
      const int zh = k0 - G::H4, yh = j0 - N;
      tma_load3(sxx_p(s + N), &maps.m[0], k0, j0, s + N, bar);
      tma_load3(sxy_p(s + N - 1), &maps.m[1], k0, yh, s + N - 1, bar);
      tma_load3(sxz_p(s + N - 1), &maps.m[2], zh, j0, s + N - 1, bar);
      tma_load3(syy_p(s), &maps.m[3], k0, yh, s, bar);
      tma_load3(syz_p(s), &maps.m[4], zh, yh, s, bar);
      tma_load3(szz_p(s), &maps.m[5], zh, j0, s, bar);
      tma_load3(rho_p(s + 1), &maps.m[6], k0, j0, s + 1, bar);
      if (first) {
        for (int q = 1 - N; q < N; ++q) tma_load3(sxx_p(s + q), &maps.m[0], k0, j0, s + q, bar);
        for (int q = -N; q < N - 1; ++q) {
          tma_load3(sxy_p(s + q), &maps.m[1], k0, yh, s + q, bar);
          tma_load3(sxz_p(s + q), &maps.m[2], zh, j0, s + q, bar);
        }
        tma_load3(rho_p(s), &maps.m[6], k0, j0, s, bar);
      }
    };
    if (tid == 0)
      for (int s = x0; s <= min(x0 + D, x1 - 1); ++s) issue(s, s == x0, (g + (s - x0)) % (D + 1));

    for (int i = x0; i < x1; ++i, ++g) {
      const bool landed = mbar_wait(&bars[g % (D + 1)], (g / (D + 1)) & 1);
      if (__syncthreads_or(!landed)) {
        if (tid == 0) atomicOr(a.err, 1);
        ok = false;
        break;
      }
      const int xi = slab_index(i, nx, p.lo[0], p.hi[0]);
      const bool interior = tile_in && i >= N + 1 && i < nx - N - 1 && xi < 0 &&
                            !(force_here && i == p.si && p.sj >= j0 && p.sj < j0 + TY && p.sk >= k0 &&
                              p.sk < k0 + G::TZ);
      if (jin && kin) {
        const float* pxx[2 * N];
        const float* pxy[2 * N];
        const float* pxz[2 * N];
#pragma unroll
        for (int q = 0; q < 2 * N; ++q) {
          pxx[q] = sxx_p(i - N + 1 + q);
          pxy[q] = sxy_p(i - N + q);
          pxz[q] = sxz_p(i - N + q);
        }
        const float* r0 = rho_p(i);
        const float* r1 = rho_p(i + 1);
        const size_t gi = (size_t)i * nyz + (size_t)j * nz + k;
        const Vq<Q> rc = ldq<Q>(r0 + o_xx), rn = ldq<Q>(r0 + o_xx + G::TZ);
        // derivatives of the three components (Dx3fm/Dy3bm/Dz3bm etc.)
        Vq<Q> dv[9] = {dxq<N, EX, Q>(pxx, o_xx, cx),
                        dyq<N, false, EX, Q>(sxy_p(i), o_y, G::TZ, cy),
                        dzq<N, false, EX, Q>(sxz_p(i), o_z, cz),
                        dxq<N, EX, Q>(pxy, o_y, cx),
                        dyq<N, true, EX, Q>(syy_p(i), o_y, G::TZ, cy),
                        dzq<N, false, EX, Q>(syz_p(i), o_yz, cz),
                        dxq<N, EX, Q>(pxz, o_z, cx),
                        dyq<N, false, EX, Q>(syz_p(i), o_yz, G::WZ, cy),
                        dzq<N, true, EX, Q>(szz_p(i), o_z, cz)};
        if (EX) {
          const float hd[9] = {dx, dy, dz, dx, dy, dz, dx, dy, dz};
          const float hr[9] = {rdx, rdy, rdz, rdx, rdy, rdz, rdx, rdy, rdz};
          div_group<9, Q>(dv, hd, hr, fast);
        }
        Vq<Q> a1 = dv[0], a2 = dv[1], a3 = dv[2], b1 = dv[3], b2 = dv[4], b3 = dv[5], c1 = dv[6], c2 = dv[7],
               c3 = dv[8];
        Vq<Q> vx = ldgq<Q>(p.f[0] + gi), vy = ldgq<Q>(p.f[1] + gi), vz = ldgq<Q>(p.f[2] + gi);
        if (interior) {
          const Vq<Q> r1c = ldq<Q>(r1 + o_xx), r1n = ldq<Q>(r1 + o_xx + G::TZ);
          // numerators and densities of the 12 updates, then their quotients
          // as one group (see div_group: no per-lane range branch)
          float tn[3 * Q], td[3 * Q];
#pragma unroll
          for (int e = 0; e < Q; ++e) {
            const float rce = g4(rc, e), rne = g4(rn, e);
            tn[e] = (g4(a1, e) + g4(a3, e) + g4(a2, e)) * dt;
            td[e] = rce;
            tn[Q + e] = (g4(b1, e) + g4(b2, e) + g4(b3, e)) * dt;
            td[Q + e] = 0.5f * (rce + rne);
            const float sum = TENSOR ? (g4(c1, e) + g4(c2, e) + g4(c3, e)) : (g4(c3, e) + g4(c1, e) + g4(c2, e));
            tn[2 * Q + e] = sum * dt;
            td[2 * Q + e] = 0.25f * (rce + rne + g4(r1n, e) + g4(r1c, e));
          }
          if (EX) {
            bool okq = true;
#pragma unroll
            for (int q = 0; q < 3 * Q; ++q) okq = okq & mk_ok(tn[q]);
            if (okq) {
#pragma unroll
              for (int q = 0; q < 3 * Q; ++q) tn[q] = tn[q] == 0.f ? tn[q] : __fdiv_rn(tn[q], td[q]);
            } else {
#pragma unroll
              for (int q = 0; q < 3 * Q; ++q) tn[q] = dd_div(tn[q], td[q]);
            }
          } else {
#pragma unroll
            for (int q = 0; q < 3 * Q; ++q) tn[q] = __fdividef(tn[q], td[q]);
          }
#pragma unroll
          for (int e = 0; e < Q; ++e) {
            s4(vx, e, g4(vx, e) + tn[e]);
            s4(vy, e, g4(vy, e) + tn[Q + e]);
            s4(vz, e, g4(vz, e) + tn[2 * Q + e]);
          }
        } else {
          QuadPml q{xi, yj, i, j, k, p.fl[0][i], fy};
          const bool anyslab = xi >= 0 || yj >= 0 || zslab;
          QuadMem<Q> mm;
          if (anyslab) quad_mem_load(p, q, 0, mm);
          // vx (x half, y int, z int): i in [N, nx-N-1), j in [N+1, ny-N), k in [N+1, nz-N)
          if (i < nx - N - 1 && j >= N + 1 && j < ny - N) {
            int pm[Q], upd[Q];
#pragma unroll
            for (int e = 0; e < Q; ++e) {
              upd[e] = k + e >= N + 1 && k + e < nz - N;
              pm[e] = upd[e] && ((q.fx & 2) || (fy & 1) || (fz[e] & 1));
            }
            if (anyslab) {
              pml_quad_m<0, EX, Q>(p, q, 0, 1, pm, a1, mm);
              pml_quad_m<1, EX, Q>(p, q, 0, 0, pm, a2, mm);
              pml_quad_m<2, EX, Q>(p, q, 0, 0, pm, a3, mm);
            }
#pragma unroll
            for (int e = 0; e < Q; ++e)
              if (upd[e]) {
                const float t = (g4(a1, e) + g4(a3, e) + g4(a2, e)) * dt;
                s4(vx, e, g4(vx, e) + dvv<EX>(t, g4(rc, e)));
              }
          }
          // vy (x int, y half, z int): i in [N+1, nx-N), j in [N, ny-N-1), k in [N+1, nz-N)
          if (i >= N + 1 && j < ny - N - 1 && j >= N) {
            int pm[Q], upd[Q];
#pragma unroll
            for (int e = 0; e < Q; ++e) {
              upd[e] = k + e >= N + 1 && k + e < nz - N;
              pm[e] = upd[e] && ((q.fx & 1) || (fy & 2) || (fz[e] & 1));
            }
            if (anyslab) {
              pml_quad_m<0, EX, Q>(p, q, 1, 0, pm, b1, mm);
              pml_quad_m<1, EX, Q>(p, q, 1, 1, pm, b2, mm);
              pml_quad_m<2, EX, Q>(p, q, 1, 0, pm, b3, mm);
            }
#pragma unroll
            for (int e = 0; e < Q; ++e)
              if (upd[e]) {
                const float rhy = 0.5f * (g4(rc, e) + g4(rn, e));
                const float t = (g4(b1, e) + g4(b2, e) + g4(b3, e)) * dt;
                s4(vy, e, g4(vy, e) + dvv<EX>(t, rhy));
              }
          }
          // vz (x int, y int, z half): i in [N+1, nx-N), j in [N+1, ny-N), k in [N, nz-N-1)
          if (i >= N + 1 && j >= N + 1 && j < ny - N) {
            const Vq<Q> r1c = ldq<Q>(r1 + o_xx), r1n = ldq<Q>(r1 + o_xx + G::TZ);
            int pm[Q], upd[Q];
#pragma unroll
            for (int e = 0; e < Q; ++e) {
              upd[e] = k + e >= N && k + e < nz - N - 1;
              pm[e] = upd[e] && ((q.fx & 1) || (fy & 1) || (fz[e] & 2));
            }
            if (anyslab) {
              pml_quad_m<0, EX, Q>(p, q, 2, 0, pm, c1, mm);
              pml_quad_m<1, EX, Q>(p, q, 2, 0, pm, c2, mm);
              pml_quad_m<2, EX, Q>(p, q, 2, 1, pm, c3, mm);
            }
#pragma unroll
            for (int e = 0; e < Q; ++e)
              if (upd[e]) {
                const float r4 = 0.25f * (g4(rc, e) + g4(rn, e) + g4(r1n, e) + g4(r1c, e));
                const float sum =
                    TENSOR ? (g4(c1, e) + g4(c2, e) + g4(c3, e)) : (g4(c3, e) + g4(c1, e) + g4(c2, e));
                const float t = sum * dt;
                s4(vz, e, g4(vz, e) + dvv<EX>(t, r4));
              }
          }
          if (anyslab) quad_mem_store(p, q, 0, mm);
          // point force (Elastic3D_SSG_CPML.py:245), after the update
          if (force_here && i == p.si && j == p.sj && p.sk >= k && p.sk < k + Q) {
            const int e = p.sk - k;
            const float t = dt * wf;
            s4(vz, e, g4(vz, e) + dvv<EX>(t, g4(rc, e)));
          }
        }
        stq<Q>(p.f[0] + gi, vx);
        stq<Q>(p.f[1] + gi, vy);
        stq<Q>(p.f[2] + gi, vz);
      }
      __syncthreads();
      if (tid == 0 && i + D + 1 < x1) issue(i + D + 1, false, g % (D + 1));
    }
  }
  if (!ok)
    for (int b = 0; b <= D; ++b) mbar_wait(&bars[(g + b) % (D + 1)], ((g + b) / (D + 1)) & 1);
}

// ---------------------------------------------------------------------------
// stress pass
// ---------------------------------------------------------------------------
template <int N, int TY, int D, bool EX, int Q>
__global__ void __launch_bounds__(SG<N, TY, D, Q>::NT, SG<N, TY, D, Q>::MINB_S)
k3s_stress(const __grid_constant__ P3<float> p, const __grid_constant__ StagedMaps maps,
           const __grid_constant__ StagedArgs a, int it, int inject_next, int gather) {
  using G = SG<N, TY, D, Q>;
  extern __shared__ __align__(128) float sm[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + G::S_FLOATS);
  const int tid = threadIdx.x;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const size_t nyz = (size_t)ny * nz;
  // receivers: the velocities are final for this step and not written here
  if (gather && p.nrec > 0)
    for (int rr = blockIdx.x * G::NT + tid; rr < p.nrec; rr += gridDim.x * G::NT)
      store_rec(p.rec_data, p.rec_f64, (long long)it * p.nrec + rr, p.f[p.rec_field][p.rec_idx[rr]]);
  if (tid == 0) {
    for (int b = 0; b <= D; ++b) mbar_init(&bars[b], 1);
    mbar_fence_init();
  }
  __syncthreads();

  // exact mode: c_m then / h; fast mode: c_m / h folded on the host
  float cx[N], cy[N], cz[N];
#pragma unroll
  for (int m = 0; m < N; ++m) {
    cx[m] = EX ? p.c[m] : p.cs[0][m];
    cy[m] = EX ? p.c[m] : p.cs[1][m];
    cz[m] = EX ? p.c[m] : p.cs[2][m];
  }
  const float dx = p.dx, dy = p.dy, dz = p.dz, dt = p.dt;
  const int fast = p.fast_div;
  const float rdx = p.rd[0], rdy = p.rd[1], rdz = p.rd[2];
  const float wn = inject_next ? p.wav[it + 1] : 0.f;
  const int r = tid / G::CQ, cq = tid % G::CQ;
  constexpr int PYZ = G::pad(G::B_YZ), PL = G::pad(G::B_L), PM = G::pad(G::B_M);
  auto vx_p = [&](int pl) { return sm + G::S_VX + rslot(pl, G::RX) * PYZ; };
  auto vy_p = [&](int pl) { return sm + G::S_VY + rslot(pl, G::RX) * PYZ; };
  auto vz_p = [&](int pl) { return sm + G::S_VZ + rslot(pl, G::RX) * PYZ; };
  auto lam_p = [&](int pl) { return sm + G::S_L + rslot(pl, G::R2) * PL; };
  auto mu_p = [&](int pl) { return sm + G::S_M + rslot(pl, G::R2) * PM; };
  const int o_v = (r + N) * G::WZ + G::H4 + Q * cq;
  const int o_l = r * G::TZ + Q * cq;
  const int o_m = r * G::WM + Q * cq;

  const int units = a.tiles_y * a.tiles_z * a.chunks;
  uint32_t g = 0;
  bool ok = true;
  for (int u = blockIdx.x; u < units && ok; u += gridDim.x) {
    const int ch = u % a.chunks;
    const int tzi = (u / a.chunks) % a.tiles_z;
    const int tyi = u / (a.chunks * a.tiles_z);
    const int j0 = tyi * TY, k0 = tzi * G::TZ;
    const int x0 = max(ch * a.chunk_len, N), x1 = min((ch + 1) * a.chunk_len, nx - N);
    if (x0 >= x1) continue;
    const int j = j0 + r, k = k0 + Q * cq;
    const bool jin = j < ny, kin = k < nz;
    const bool tile_in = j0 >= N + 1 && j0 + TY <= ny - N - 1 && k0 >= N + 1 && k0 + G::TZ <= nz - N - 1 &&
                         j0 >= p.lo[1] && j0 + TY <= ny - p.hi[1] && k0 >= p.lo[2] && k0 + G::TZ <= nz - p.hi[2];
    const int yj = jin ? slab_index(j, ny, p.lo[1], p.hi[1]) : -1;
    const uint8_t fy = jin ? p.fl[1][j] : 0;
    bool zslab = false;
    uint8_t fz[Q];
#pragma unroll
    for (int e = 0; e < Q; ++e) {
      const int kk = k + e;
      fz[e] = kk < nz ? p.fl[2][kk] : 0;
      zslab = zslab || (kk < nz && slab_index(kk, nz, p.lo[2], p.hi[2]) >= 0);
    }

    auto issue = [&](int s, bool first, uint32_t stage) {
      uint64_t* bar = &bars[stage];
      uint32_t bytes = (3 * G::B_YZ + G::B_L + G::B_M) * 4;
      if (first) bytes += ((2 * N - 1) * 3 * G::B_YZ + G::B_L + G::B_M) * 4;
      mbar_expect_tx(bar, bytes);
      const int zh = k0 - G::H4, yh = j0 - N;
      // vx planes up to s+N-1 (Dx3bm), vy / vz up to s+N (Dx3fm)
      tma_load3(vx_p(s + N - 1), &maps.m[0], zh, yh, s + N - 1, bar);
      tma_load3(vy_p(s + N), &maps.m[1], zh, yh, s + N, bar);
      tma_load3(vz_p(s + N), &maps.m[2], zh, yh, s + N, bar);
      tma_load3(lam_p(s + 1), &maps.m[3], k0, j0, s + 1, bar);
      tma_load3(mu_p(s + 1), &maps.m[4], k0, j0, s + 1, bar);
      if (first) {
        for (int q = -N; q < N - 1; ++q) tma_load3(vx_p(s + q), &maps.m[0], zh, yh, s + q, bar);
        for (int q = 1 - N; q < N; ++q) {
          tma_load3(vy_p(s + q), &maps.m[1], zh, yh, s + q, bar);
          tma_load3(vz_p(s + q), &maps.m[2], zh, yh, s + q, bar);
        }
        tma_load3(lam_p(s), &maps.m[3], k0, j0, s, bar);
        tma_load3(mu_p(s), &maps.m[4], k0, j0, s, bar);
      }
    };
    if (tid == 0)
      for (int s = x0; s <= min(x0 + D, x1 - 1); ++s) issue(s, s == x0, (g + (s - x0)) % (D + 1));

    for (int i = x0; i < x1; ++i, ++g) {
      const bool landed = mbar_wait(&bars[g % (D + 1)], (g / (D + 1)) & 1);
      if (__syncthreads_or(!landed)) {
        if (tid == 0) atomicOr(a.err, 1);
        ok = false;
        break;
      }
      const int xi = slab_index(i, nx, p.lo[0], p.hi[0]);
      const bool src = inject_next && i == p.si && p.sj == j && p.sk >= k && p.sk < k + Q;
      const bool interior = tile_in && i >= N + 1 && i < nx - N - 1 && xi < 0 &&
                            !(inject_next && i == p.si && p.sj >= j0 && p.sj < j0 + TY && p.sk >= k0 &&
                              p.sk < k0 + G::TZ);
      if (jin && kin) {
        const float* pvx[2 * N];  // vx planes i-N .. i+N-1  (Dx3bm)
        const float* pvy[2 * N];  // vy planes i-N+1 .. i+N  (Dx3fm)
        const float* pvz[2 * N];
#pragma unroll
        for (int q = 0; q < 2 * N; ++q) {
          pvx[q] = vx_p(i - N + q);
          pvy[q] = vy_p(i - N + 1 + q);
          pvz[q] = vz_p(i - N + 1 + q);
        }
        const float* vxi = vx_p(i);
        const float* vyi = vy_p(i);
        const float* vzi = vz_p(i);
        const size_t gi = (size_t)i * nyz + (size_t)j * nz + k;
        Vq<Q> sxx = ldgq<Q>(p.f[3] + gi), syy = ldgq<Q>(p.f[4] + gi), szz = ldgq<Q>(p.f[5] + gi);
        Vq<Q> sxy = ldgq<Q>(p.f[6] + gi), sxz = ldgq<Q>(p.f[7] + gi), syz = ldgq<Q>(p.f[8] + gi);
        const Vq<Q> l0 = ldq<Q>(lam_p(i) + o_l), l1 = ldq<Q>(lam_p(i + 1) + o_l);
        const float* m0p = mu_p(i);
        const Vq<Q> u0 = ldq<Q>(m0p + o_m), u1 = ldq<Q>(mu_p(i + 1) + o_m), unj = ldq<Q>(m0p + o_m + G::WM);
        float unk[Q];  // mu[k+1 .. k+Q] for the k+1 neighbours
#pragma unroll
        for (int e = 0; e + 1 < Q; ++e) unk[e] = g4(u0, e + 1);
        unk[Q - 1] = m0p[o_m + Q];
        // derivatives: dvx/dx dvy/dy dvz/dz dvy/dx dvx/dy dvz/dx dvx/dz dvz/dy dvy/dz
        Vq<Q> dv[9] = {dxq<N, EX, Q>(pvx, o_v, cx),
                        dyq<N, false, EX, Q>(vyi, o_v, G::WZ, cy),
                        dzq<N, false, EX, Q>(vzi, o_v, cz),
                        dxq<N, EX, Q>(pvy, o_v, cx),
                        dyq<N, true, EX, Q>(vxi, o_v, G::WZ, cy),
                        dxq<N, EX, Q>(pvz, o_v, cx),
                        dzq<N, true, EX, Q>(vxi, o_v, cz),
                        dyq<N, true, EX, Q>(vzi, o_v, G::WZ, cy),
                        dzq<N, true, EX, Q>(vyi, o_v, cz)};
        if (EX) {
          const float hd[9] = {dx, dy, dz, dx, dy, dx, dz, dy, dz};
          const float hr[9] = {rdx, rdy, rdz, rdx, rdy, rdx, rdz, rdy, rdz};
          div_group<9, Q>(dv, hd, hr, fast);
        }
        Vq<Q> e1 = dv[0], e2 = dv[1], e3 = dv[2], f1 = dv[3], f2 = dv[4], h1 = dv[5], h2 = dv[6], q1 = dv[7],
               q2 = dv[8];
        if (interior) {
#pragma unroll
          for (int e = 0; e < Q; ++e) {
            const float lhx = 0.5f * (g4(l0, e) + g4(l1, e));
            const float mhx = 0.5f * (g4(u0, e) + g4(u1, e));
            const float lpm = lhx + 2.0f * mhx;
            const float A = g4(e1, e), B = g4(e2, e), Cc = g4(e3, e);
            s4(sxx, e, g4(sxx, e) + (lpm * A + lhx * (Cc + B)) * dt);
            s4(syy, e, g4(syy, e) + (lpm * B + lhx * (A + Cc)) * dt);
            s4(szz, e, g4(szz, e) + (lpm * Cc + lhx * (A + B)) * dt);
            const float u = g4(u0, e);
            const float mxy = 0.25f * (g4(unj, e) + u + u + g4(u1, e));
            s4(sxy, e, g4(sxy, e) + mxy * (g4(f2, e) + g4(f1, e)) * dt);
            const float mxz = 0.25f * (u + g4(u1, e) + u + g4(unj, e));
            s4(sxz, e, g4(sxz, e) + mxz * (g4(h2, e) + g4(h1, e)) * dt);
            const float myz = 0.25f * (g4(unj, e) + u + unk[e] + u);
            s4(syz, e, g4(syz, e) + myz * (g4(q1, e) + g4(q2, e)) * dt);
          }
        } else {
          QuadPml q{xi, yj, i, j, k, p.fl[0][i], fy};
          const bool anyslab = xi >= 0 || yj >= 0 || zslab;
          QuadMem<Q> mm;
          if (anyslab) quad_mem_load(p, q, 3, mm);
          // normal stresses: i, j, k in [N+1, n-N)
          if (i >= N + 1 && j >= N + 1 && j < ny - N) {
            int pm[Q], upd[Q];
#pragma unroll
            for (int e = 0; e < Q; ++e) {
              upd[e] = k + e >= N + 1 && k + e < nz - N;
              pm[e] = upd[e] && ((q.fx | fy | fz[e]) & 1);
            }
            if (anyslab) {
              pml_quad_m<0, EX, Q>(p, q, 0, 0, pm, e1, mm);
              pml_quad_m<1, EX, Q>(p, q, 0, 0, pm, e2, mm);
              pml_quad_m<2, EX, Q>(p, q, 0, 0, pm, e3, mm);
            }
#pragma unroll
            for (int e = 0; e < Q; ++e)
              if (upd[e]) {
                const float lhx = 0.5f * (g4(l0, e) + g4(l1, e));
                const float mhx = 0.5f * (g4(u0, e) + g4(u1, e));
                const float lpm = lhx + 2.0f * mhx;
                const float A = g4(e1, e), B = g4(e2, e), Cc = g4(e3, e);
                s4(sxx, e, g4(sxx, e) + (lpm * A + lhx * (Cc + B)) * dt);
                s4(syy, e, g4(syy, e) + (lpm * B + lhx * (A + Cc)) * dt);
                s4(szz, e, g4(szz, e) + (lpm * Cc + lhx * (A + B)) * dt);
              }
          }
          // sxy (x half, y half, z int): i, j in [N+1, n-N), k in [N, nz-N)
          if (i >= N + 1 && j >= N + 1 && j < ny - N) {
            int pm[Q], upd[Q];
#pragma unroll
            for (int e = 0; e < Q; ++e) {
              upd[e] = k + e >= N && k + e < nz - N;
              pm[e] = upd[e] && ((q.fx & 2) || (fy & 2) || (fz[e] & 1));
            }
            if (anyslab) {
              pml_quad_m<0, EX, Q>(p, q, 1, 1, pm, f1, mm);
              pml_quad_m<1, EX, Q>(p, q, 1, 1, pm, f2, mm);
            }
#pragma unroll
            for (int e = 0; e < Q; ++e)
              if (upd[e]) {
                const float u = g4(u0, e);
                const float m4 = 0.25f * (g4(unj, e) + u + u + g4(u1, e));
                s4(sxy, e, g4(sxy, e) + m4 * (g4(f2, e) + g4(f1, e)) * dt);
              }
          }
          // sxz (x half, y int, z half): i in [N, nx-N-1), j in [N, ny-N), k in [N, nz-N-1)
          if (i < nx - N - 1 && j >= N && j < ny - N) {
            int pm[Q], upd[Q];
#pragma unroll
            for (int e = 0; e < Q; ++e) {
              upd[e] = k + e >= N && k + e < nz - N - 1;
              pm[e] = upd[e] && ((q.fx & 2) || (fy & 1) || (fz[e] & 2));
            }
            if (anyslab) {
              pml_quad_m<0, EX, Q>(p, q, 2, 1, pm, h1, mm);
              pml_quad_m<2, EX, Q>(p, q, 1, 1, pm, h2, mm);
            }
#pragma unroll
            for (int e = 0; e < Q; ++e)
              if (upd[e]) {
                const float u = g4(u0, e);
                const float m4 = 0.25f * (u + g4(u1, e) + u + g4(unj, e));
                s4(sxz, e, g4(sxz, e) + m4 * (g4(h2, e) + g4(h1, e)) * dt);
              }
          }
          // syz (x int, y half, z half): i in [N, nx-N), j in [N, ny-N-1), k in [N, nz-N-1)
          if (j >= N && j < ny - N - 1) {
            int pm[Q], upd[Q];
#pragma unroll
            for (int e = 0; e < Q; ++e) {
              upd[e] = k + e >= N && k + e < nz - N - 1;
              pm[e] = upd[e] && ((q.fx & 1) || (fy & 2) || (fz[e] & 2));
            }
            if (anyslab) {
              pml_quad_m<1, EX, Q>(p, q, 2, 1, pm, q1, mm);
              pml_quad_m<2, EX, Q>(p, q, 2, 1, pm, q2, mm);
            }
#pragma unroll
            for (int e = 0; e < Q; ++e)
              if (upd[e]) {
                const float u = g4(u0, e);
                const float m4 = 0.25f * (g4(unj, e) + u + unk[e] + u);
                s4(syz, e, g4(syz, e) + m4 * (g4(q1, e) + g4(q2, e)) * dt);
              }
          }
          if (anyslab) quad_mem_store(p, q, 3, mm);
          if (src) {
            // next step's moment-tensor source (Elastic3D_SSG_Tensor.py:186-193)
            const int e = p.sk - k;
            s4(sxx, e, g4(sxx, e) + wn * p.mneg[0]);
            s4(syy, e, g4(syy, e) + wn * p.mneg[1]);
            s4(szz, e, g4(szz, e) + wn * p.mneg[2]);
            s4(sxy, e, g4(sxy, e) + wn * p.mneg[3]);
            s4(sxz, e, g4(sxz, e) + wn * p.mneg[4]);
            s4(syz, e, g4(syz, e) + wn * p.mneg[5]);
          }
        }
        stq<Q>(p.f[3] + gi, sxx);
        stq<Q>(p.f[4] + gi, syy);
        stq<Q>(p.f[5] + gi, szz);
        stq<Q>(p.f[6] + gi, sxy);
        stq<Q>(p.f[7] + gi, sxz);
        stq<Q>(p.f[8] + gi, syz);
      }
      __syncthreads();
      if (tid == 0 && i + D + 1 < x1) issue(i + D + 1, false, g % (D + 1));
    }
  }
  if (!ok)
    for (int b = 0; b <= D; ++b) mbar_wait(&bars[(g + b) % (D + 1)], ((g + b) / (D + 1)) & 1);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 staged_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }
  return fn;
}

static bool map3(CUtensorMap* m, const void* base, int nx, int ny, int nz, int bz, int by) {
  auto enc = staged_encoder();
  if (!enc) return false;
  cuuint64_t dims[3] = {(cuuint64_t)nz, (cuuint64_t)ny, (cuuint64_t)nx};
  cuuint64_t strides[2] = {(cuuint64_t)nz * 4, (cuuint64_t)ny * nz * 4};
  cuuint32_t box[3] = {(cuuint32_t)bz, (cuuint32_t)by, 1};
  cuuint32_t es[3] = {1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(base), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int N, int TY, int D>
static bool staged_maps_t(const P3<float>& p, StagedMaps* vm, StagedMaps* sm_) {
  using G = SG<N, TY, D, 4>;  // box shapes do not depend on the cells per thread
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  bool ok = true;
  // velocity pass: sxx sxy sxz syy syz szz rho
  ok = ok && map3(&vm->m[0], p.f[3], nx, ny, nz, G::TZ, TY);
  ok = ok && map3(&vm->m[1], p.f[6], nx, ny, nz, G::TZ, G::HY);
  ok = ok && map3(&vm->m[2], p.f[7], nx, ny, nz, G::WZ, TY);
  ok = ok && map3(&vm->m[3], p.f[4], nx, ny, nz, G::TZ, G::HY);
  ok = ok && map3(&vm->m[4], p.f[8], nx, ny, nz, G::WZ, G::HY);
  ok = ok && map3(&vm->m[5], p.f[5], nx, ny, nz, G::WZ, TY);
  ok = ok && map3(&vm->m[6], p.rho, nx, ny, nz, G::TZ, TY + 1);
  // stress pass: vx vy vz lam mu
  ok = ok && map3(&sm_->m[0], p.f[0], nx, ny, nz, G::WZ, G::HY);
  ok = ok && map3(&sm_->m[1], p.f[1], nx, ny, nz, G::WZ, G::HY);
  ok = ok && map3(&sm_->m[2], p.f[2], nx, ny, nz, G::WZ, G::HY);
  ok = ok && map3(&sm_->m[3], p.lam, nx, ny, nz, G::TZ, TY);
  ok = ok && map3(&sm_->m[4], p.mu, nx, ny, nz, G::WM, TY + 1);
  return ok;
}

template <int N, int TY, int D>
static StagedConfig staged_cfg_t() {
  using G = SG<N, TY, D, staged_q(true)>;
  return StagedConfig{N, TY, D, G::NT, G::V_BYTES, G::S_BYTES};
}

bool sw3_staged_config(int N, StagedConfig* out) {
  switch (N) {
    case 1: *out = staged_cfg_t<1, 16, 2>(); return true;
    case 2: *out = staged_cfg_t<2, 16, 1>(); return true;
    case 3: *out = staged_cfg_t<3, 16, 2>(); return true;
    case 4: *out = staged_cfg_t<4, 16, 1>(); return true;
    default: return false;
  }
}

bool sw3_staged_maps(int N, const P3<float>& p, StagedMaps* vm, StagedMaps* sm_) {
  switch (N) {
    case 1: return staged_maps_t<1, 16, 2>(p, vm, sm_);
    case 2: return staged_maps_t<2, 16, 1>(p, vm, sm_);
    case 3: return staged_maps_t<3, 16, 2>(p, vm, sm_);
    case 4: return staged_maps_t<4, 16, 1>(p, vm, sm_);
    default: return false;
  }
}

template <int N, int TY, int D, bool EX>
static cudaError_t staged_launch(bool tensor, const P3<float>& p, const StagedMaps& vm, const StagedMaps& smp,
                                 const StagedArgs& a, int grid, int it, bool force_here, bool inject_next,
                                 bool gather, cudaStream_t st) {
  constexpr int Q = staged_q(EX);
  using G = SG<N, TY, D, Q>;
  static std::atomic<unsigned long long> done{0};
  static std::mutex mu;
  cudaError_t e0 = once_per_device(done, mu, [] {
    cudaError_t e = cudaFuncSetAttribute(k3s_velocity<N, TY, D, true, EX, Q>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::V_BYTES);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k3s_velocity<N, TY, D, false, EX, Q>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)G::V_BYTES);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k3s_stress<N, TY, D, EX, Q>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)G::S_BYTES);
    return e;
  });
  if (e0 != cudaSuccess) return e0;
  if (tensor) k3s_velocity<N, TY, D, true, EX, Q><<<grid, G::NT, G::V_BYTES, st>>>(p, vm, a, it, 0);
  else k3s_velocity<N, TY, D, false, EX, Q><<<grid, G::NT, G::V_BYTES, st>>>(p, vm, a, it, force_here ? 1 : 0);
  k3s_stress<N, TY, D, EX, Q><<<grid, G::NT, G::S_BYTES, st>>>(p, smp, a, it, inject_next ? 1 : 0, gather ? 1 : 0);
  return cudaGetLastError();
}

template <int N, int TY, int D>
static cudaError_t staged_step_t(bool tensor, const P3<float>& p, const StagedMaps& vm, const StagedMaps& smp,
                                 const StagedArgs& a, int grid, int it, bool force_here, bool inject_next,
                                 bool gather, cudaStream_t st) {
  return a.exact ? staged_launch<N, TY, D, true>(tensor, p, vm, smp, a, grid, it, force_here, inject_next, gather, st)
                 : staged_launch<N, TY, D, false>(tensor, p, vm, smp, a, grid, it, force_here, inject_next, gather,
                                                  st);
}

cudaError_t sw3_staged_step(int N, bool tensor, const P3<float>& p, const StagedMaps& vm, const StagedMaps& smp,
                            const StagedArgs& a, int grid, int it, bool force_here, bool inject_next, bool gather,
                            cudaStream_t st) {
  switch (N) {
    case 1: return staged_step_t<1, 16, 2>(tensor, p, vm, smp, a, grid, it, force_here, inject_next, gather, st);
    case 2: return staged_step_t<2, 16, 1>(tensor, p, vm, smp, a, grid, it, force_here, inject_next, gather, st);
    case 3: return staged_step_t<3, 16, 2>(tensor, p, vm, smp, a, grid, it, force_here, inject_next, gather, st);
    case 4: return staged_step_t<4, 16, 1>(tensor, p, vm, smp, a, grid, it, force_here, inject_next, gather, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace sw
