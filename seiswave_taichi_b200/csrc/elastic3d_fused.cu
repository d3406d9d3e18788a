// elastic3d_fused.cu -- single-pass 3D SSG-CPML time step (velocity + stress),
// TMA-fed, for the moment-tensor and point-force schemes
// (src/Elastic3D_SSG_Tensor.py:166-345, src/Elastic3D_SSG_CPML.py:144-309).
//
// One CTA owns a TY (y) x 32 (z) column tile and streams a chunk of x planes.
// For every plane s it
//   1. waits for the TMA loads of plane s (stress planes with a 2N halo in y
//      and z, old velocities and density with an N halo), issued D planes
//      ahead into shared-memory rings;
//   2. computes the new velocities of plane s on the tile plus an N-cell halo
//      (the halo is recomputed, bit-identically, by the neighbouring tiles)
//      into a shared ring of 2N+1 velocity planes, writing the tile cells to
//      the output buffer;
//   3. computes the new stresses of plane q = s-N on the tile from that ring.
// The step reads one buffer set and writes the other (ping-pong), so the halo
// recompute never sees a neighbour's new values; DRAM traffic per cell is one
// read and one write of each wavefield plus one read of the material.
// Cells are processed in z-pairs (float2).  Division by the constant grid
// spacings uses Markstein's correction q' = q + r*fma(-q, d, x), q = x*RN(1/d),
// which the plan verifies against IEEE division for every float input before
// enabling it; all other operations follow the reference's order with
// -fmad=false, so the result equals the two-pass kernels and the CPU oracle
// bit for bit.
#include <cstdio>
#include <cudaTypedefs.h>

#include "sw_device.cuh"
#include "sw_fused.cuh"
#include "sw_tma.cuh"

namespace sw {

template <int N, int TY, int D>
struct FG {
  static constexpr int TZ = 32;
  static constexpr int NT = 256;
  static constexpr int A4_2N = ((2 * N + 3) / 4) * 4;
  static constexpr int A4_N = ((N + 3) / 4) * 4;
  static constexpr int A2_N = ((N + 1) / 2) * 2;
  static constexpr int SZ0 = A4_2N;            // stress box starts at k0 - SZ0 (16-byte aligned)
  static constexpr int SW = TZ + 2 * SZ0;      // stress box width (z)
  static constexpr int SH = TY + 4 * N;        // stress box height (y), starts at j0 - 2N
  static constexpr int SB = SW * SH;
  static constexpr int VZ0 = A4_N;             // velocity box starts at k0 - VZ0
  static constexpr int VW = TZ + 2 * VZ0;
  static constexpr int VH = TY + 2 * N;        // starts at j0 - N
  static constexpr int VB = VW * VH;
  static constexpr int RH = VH + 1;            // density box, one more row (j+1)
  static constexpr int RB = VW * RH;
  static constexpr int PZ0 = A2_N;             // velocity pairs start at k0 - PZ0
  static constexpr int PV = (TZ + 2 * PZ0) / 2;
  static constexpr int NPV = VH * PV;
  static constexpr int NPS = TY * TZ / 2;
  static constexpr int R1 = 2 * N + D;         // sxx, sxy, sxz rings
  static constexpr int R2 = 1 + D;             // syy, szz, syz rings
  static constexpr int RVO = 1 + D;            // old velocities
  static constexpr int RR = 2 + D;             // density
  static constexpr int RV = 2 * N + 1;         // computed velocities
  static constexpr int pad(int x) { return (x + 31) / 32 * 32; }
  static constexpr int O_S1 = 0;
  static constexpr int O_S2 = O_S1 + 3 * R1 * pad(SB);
  static constexpr int O_VO = O_S2 + 3 * R2 * pad(SB);
  static constexpr int O_R = O_VO + 3 * RVO * pad(VB);
  static constexpr int O_V = O_R + RR * pad(RB);
  static constexpr int FLOATS = O_V + 3 * RV * pad(VB);
  static constexpr size_t BYTES = (size_t)FLOATS * 4 + 8 * (D + 1) + 128;
  static_assert(SZ0 >= 2 * A2_N, "stress box must cover the pair windows of the halo");
  static_assert(SW <= 256 && SH <= 256 && VW <= 256 && RH <= 256, "TMA box too large");
};

__device__ __forceinline__ float2 ld2(const float* p) { return *reinterpret_cast<const float2*>(p); }
__device__ __forceinline__ void st2(float* p, float2 v) { *reinterpret_cast<float2*>(p) = v; }

__device__ __forceinline__ int ring_slot(int plane, int R) {
  int s = plane % R;
  return s < 0 ? s + R : s;
}

// derivative of a pair along a smem stride: FWD: f[+m+1]-f[-m], else f[+m]-f[-m-1]
template <int N, bool FWD>
__device__ __forceinline__ float2 dstride(const float* s, int off, int stride, const float* c) {
  float2 v = make_float2(0.f, 0.f);
#pragma unroll
  for (int m = 0; m < N; ++m) {
    const float2 a = ld2(s + off + (FWD ? (m + 1) : m) * stride);
    const float2 b = ld2(s + off - (FWD ? m : (m + 1)) * stride);
    v.x = v.x + c[m] * (a.x - b.x);
    v.y = v.y + c[m] * (a.y - b.y);
  }
  return v;
}

// derivative of a pair across ring planes: pl[q] = smem base of plane (s - N + FWD + q)
template <int N, bool FWD>
__device__ __forceinline__ float2 dplanes(const float* const* pl, int off, const float* c) {
  float2 v = make_float2(0.f, 0.f);
#pragma unroll
  for (int m = 0; m < N; ++m) {
    const float2 a = ld2(pl[N + m] + off);
    const float2 b = ld2(pl[N - 1 - m] + off);
    v.x = v.x + c[m] * (a.x - b.x);
    v.y = v.y + c[m] * (a.y - b.y);
  }
  return v;
}

// derivative of a pair along z (contiguous) from one window of aligned pairs
template <int N, bool FWD>
__device__ __forceinline__ float2 dzp(const float* s, int off, const float* c) {
  constexpr int A = ((N + 1) / 2) * 2;
  float w[2 * A + 2];
#pragma unroll
  for (int t = 0; t <= A; ++t) {
    const float2 q = ld2(s + off - A + 2 * t);
    w[2 * t] = q.x;
    w[2 * t + 1] = q.y;
  }
  float2 v = make_float2(0.f, 0.f);
#pragma unroll
  for (int m = 0; m < N; ++m) {
    if (FWD) {
      v.x = v.x + c[m] * (w[A + m + 1] - w[A - m]);
      v.y = v.y + c[m] * (w[A + m + 2] - w[A - m + 1]);
    } else {
      v.x = v.x + c[m] * (w[A + m] - w[A - m - 1]);
      v.y = v.y + c[m] * (w[A + m + 1] - w[A - m]);
    }
  }
  return v;
}

__device__ __forceinline__ float pml_step(float* m, float b, float a, float kk, float d) {
  const float psi = b * (*m) + a * d;
  *m = psi;
  return div_v(d, kk) + psi;
}
// velocity memory variables are ping-ponged: read one buffer, write the other
// (only the owner tile writes)
__device__ __forceinline__ float pml_step2(const float* min, float* mout, float b, float a, float kk, float d) {
  const float psi = b * (*min) + a * d;
  if (mout) *mout = psi;
  return div_v(d, kk) + psi;
}

template <int N, int TY, int D, bool TENSOR>
__global__ void __launch_bounds__(256, 1)
k3_fused(const __grid_constant__ P3<float> p, const __grid_constant__ FusedMaps maps,
         const __grid_constant__ FusedExtra x, int it, int src, int inject_next, int gather_it) {
  using G = FG<N, TY, D>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float* sm = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + G::FLOATS);
  const int tid = threadIdx.x;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const size_t nyz = (size_t)ny * nz;

  // input / output buffer sets
  float* fin[9];
  float* fout[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    fin[q] = src == 0 ? p.f[q] : x.fB[q];
    fout[q] = src == 0 ? x.fB[q] : p.f[q];
  }
  const float* vmin[3];
  float* vmout[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    vmin[d] = src == 0 ? p.mem[d] : x.memB[d];
    vmout[d] = src == 0 ? x.memB[d] : p.mem[d];
  }

  // receivers of the previous step, read from this step's input
  if (gather_it >= 0 && p.nrec > 0) {
    for (int r = blockIdx.x * G::NT + tid; r < p.nrec; r += gridDim.x * G::NT)
      store_rec(p.rec_data, p.rec_f64, (long long)gather_it * p.nrec + r, fin[p.rec_field][p.rec_idx[r]]);
  }

  if (tid == 0) {
    for (int b = 0; b <= D; ++b) mbar_init(&bars[b], 1);
    mbar_fence_init();
    for (int a = 0; a < 6; ++a) prefetch_map(&maps.sig[src][a]);
    for (int a = 0; a < 3; ++a) prefetch_map(&maps.vel[src][a]);
    prefetch_map(&maps.rho);
  }
  __syncthreads();

  float c[N];
#pragma unroll
  for (int m = 0; m < N; ++m) c[m] = p.c[m];
  const float dx = p.dx, dy = p.dy, dz = p.dz, dt = p.dt;
  const int fast = p.fast_div;
  const float rdx = p.rd[0], rdy = p.rd[1], rdz = p.rd[2];
  const float wn = inject_next ? p.wav[it + 1] : 0.f;
  const float wf = (!TENSOR && p.src_kind == SW_SRC_FORCE) ? p.wav[it] : 0.f;
  const bool force = !TENSOR && p.src_kind == SW_SRC_FORCE;

  // shared-memory ring bases
  float* S1 = sm + G::O_S1;  // [3][R1][pad(SB)]: sxx, sxy, sxz
  float* S2 = sm + G::O_S2;  // [3][R2][pad(SB)]: syy, szz, syz
  float* VO = sm + G::O_VO;  // [3][RVO][pad(VB)]
  float* RR = sm + G::O_R;   // [RR][pad(RB)]
  float* V = sm + G::O_V;    // [3][RV][pad(VB)]
  constexpr int PSB = G::pad(G::SB), PVB = G::pad(G::VB), PRB = G::pad(G::RB);
  auto s1 = [&](int a, int plane) { return S1 + (a * G::R1 + ring_slot(plane, G::R1)) * PSB; };
  auto s2 = [&](int a, int plane) { return S2 + (a * G::R2 + ring_slot(plane, G::R2)) * PSB; };
  auto vo = [&](int a, int plane) { return VO + (a * G::RVO + ring_slot(plane, G::RVO)) * PVB; };
  auto rr = [&](int plane) { return RR + ring_slot(plane, G::RR) * PRB; };
  auto vv = [&](int a, int plane) { return V + (a * G::RV + ring_slot(plane, G::RV)) * PVB; };

  const int units = x.tiles_y * x.tiles_z * x.chunks;
  uint32_t g = 0;  // steps consumed by this CTA (mbarrier phase bookkeeping)
  bool ok = true;

  for (int u = blockIdx.x; u < units && ok; u += gridDim.x) {
    const int ch = u % x.chunks;
    const int tz = (u / x.chunks) % x.tiles_z;
    const int ty = u / (x.chunks * x.tiles_z);
    const int j0 = ty * TY, k0 = tz * G::TZ;
    const int x0 = ch * x.chunk_len, x1 = min(nx, x0 + x.chunk_len);
    const int i_beg = max(x0 - N, 0), i_end = min(x1 + N - 1, nx - 1);

    // loads of velocity step s (first: also fill the rings)
    auto issue = [&](int s, bool first, uint32_t stage) {
      uint64_t* bar = &bars[stage];
      uint32_t bytes = (6 * G::SB + 3 * G::VB + G::RB) * 4;
      if (first) bytes += ((2 * N - 1) * 3 * G::SB + G::RB) * 4;
      mbar_expect_tx(bar, bytes);
      const int zs = k0 - G::SZ0, ys = j0 - 2 * N, zv = k0 - G::VZ0, yv = j0 - N;
      // sxx planes up to s+N, sxy/sxz up to s+N-1 (the x taps), syy/szz/syz plane s
      tma_load3(s1(0, s + N), &maps.sig[src][0], zs, ys, s + N, bar);
      tma_load3(s1(1, s + N - 1), &maps.sig[src][3], zs, ys, s + N - 1, bar);
      tma_load3(s1(2, s + N - 1), &maps.sig[src][4], zs, ys, s + N - 1, bar);
      tma_load3(s2(0, s), &maps.sig[src][1], zs, ys, s, bar);
      tma_load3(s2(1, s), &maps.sig[src][2], zs, ys, s, bar);
      tma_load3(s2(2, s), &maps.sig[src][5], zs, ys, s, bar);
      for (int a = 0; a < 3; ++a) tma_load3(vo(a, s), &maps.vel[src][a], zv, yv, s, bar);
      tma_load3(rr(s + 1), &maps.rho, zv, yv, s + 1, bar);
      if (first) {
        for (int q = 1 - N; q < N; ++q) tma_load3(s1(0, s + q), &maps.sig[src][0], zs, ys, s + q, bar);
        for (int q = -N; q < N - 1; ++q) {
          tma_load3(s1(1, s + q), &maps.sig[src][3], zs, ys, s + q, bar);
          tma_load3(s1(2, s + q), &maps.sig[src][4], zs, ys, s + q, bar);
        }
        tma_load3(rr(s), &maps.rho, zv, yv, s, bar);
      }
    };

    if (tid == 0) {
      for (int s = i_beg; s <= min(i_beg + D, i_end); ++s) issue(s, s == i_beg, (g + (s - i_beg)) % (D + 1));
    }

    for (int s = i_beg; s <= i_end; ++s, ++g) {
      // every thread waits (bounded); the CTA then agrees on the outcome so no
      // thread is left alone at a later barrier
      const bool landed = mbar_wait(&bars[g % (D + 1)], (g / (D + 1)) & 1);
      if (__syncthreads_or(!landed)) {
        if (tid == 0) atomicOr(x.err, 1);
        ok = false;
        break;
      }
      const int i = s;
      const size_t pl = (size_t)i * nyz;
      const int xi = slab_index(i, nx, p.lo[0], p.hi[0]);
      const uint8_t fx = p.fl[0][i];
      const bool write_v = (i >= x0 && i < x1);

      // plane pointers of the x taps
      const float* pxx[2 * N];
      const float* pxy[2 * N];
      const float* pxz[2 * N];
#pragma unroll
      for (int q = 0; q < 2 * N; ++q) {
        pxx[q] = s1(0, i - N + 1 + q);
        pxy[q] = s1(1, i - N + q);
        pxz[q] = s1(2, i - N + q);
      }
      const float* sxy_i = s1(1, i);
      const float* sxz_i = s1(2, i);
      const float* syy_i = s2(0, i);
      const float* szz_i = s2(1, i);
      const float* syz_i = s2(2, i);
      const float* r0 = rr(i);
      const float* r1 = rr(i + 1);

      // ---------------- velocity phase: plane i on tile + N halo ----------
      for (int pi = tid; pi < G::NPV; pi += G::NT) {
        const int r = pi / G::PV, cc = pi - r * G::PV;
        const int j = j0 - N + r;
        const int k = k0 - G::PZ0 + 2 * cc;
        const int so = (r + N) * G::SW + (G::SZ0 - G::PZ0 + 2 * cc);
        const int vof = r * G::VW + (G::VZ0 - G::PZ0 + 2 * cc);
        const bool jin = j >= 0 && j < ny;
        const bool tile = write_v && j >= j0 && j < j0 + TY && j < ny && k >= k0 && k < k0 + G::TZ && k < nz;
        const int yj = jin ? slab_index(j, ny, p.lo[1], p.hi[1]) : -1;
        const uint8_t fy = jin ? p.fl[1][j] : 0;
        float2 ovx = ld2(vo(0, i) + vof), ovy = ld2(vo(1, i) + vof), ovz = ld2(vo(2, i) + vof);
        float2 nvx = ovx, nvy = ovy, nvz = ovz;
        const float2 rc = ld2(r0 + vof), rn = ld2(r0 + vof + G::VW);
        const size_t rowg = pl + (size_t)j * nz;

        // vx (x half, y int, z int): i in [N, nx-N-1), j in [N+1, ny-N), k in [N+1, nz-N)
        if (i >= N && i < nx - N - 1 && j >= N + 1 && j < ny - N) {
          float2 d1 = dplanes<N, true>(pxx, so, c);
          float2 d2 = dstride<N, false>(sxy_i, so, G::SW, c);
          float2 d3 = dzp<N, false>(sxz_i, so, c);
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int kk = k + e;
            if (kk < N + 1 || kk >= nz - N) continue;
            float a1 = div_c(e ? d1.y : d1.x, dx, rdx, fast);
            float a2 = div_c(e ? d2.y : d2.x, dy, rdy, fast);
            float a3 = div_c(e ? d3.y : d3.x, dz, rdz, fast);
            const int zk = slab_index(kk, nz, p.lo[2], p.hi[2]);
            if ((xi >= 0 || yj >= 0 || zk >= 0) && ((fx & 2) || (fy & 1) || (p.fl[2][kk] & 1))) {
              if (xi >= 0) {
                const size_t o = ((size_t)xi * ny + j) * nz + kk;
                a1 = pml_step2(vmin[0] + o, tile ? vmout[0] + o : nullptr, p.cf[0][CBH * nx + i],
                               p.cf[0][CAH * nx + i], p.cf[0][CKH * nx + i], a1);
              }
              if (yj >= 0) {
                const size_t o = ((size_t)i * p.sn[1] + yj) * nz + kk;
                a2 = pml_step2(vmin[1] + o, tile ? vmout[1] + o : nullptr, p.cf[1][CB * ny + j],
                               p.cf[1][CA * ny + j], p.cf[1][CK * ny + j], a2);
              }
              if (zk >= 0) {
                const size_t o = ((size_t)i * ny + j) * p.sn[2] + zk;
                a3 = pml_step2(vmin[2] + o, tile ? vmout[2] + o : nullptr, p.cf[2][CB * nz + kk],
                               p.cf[2][CA * nz + kk], p.cf[2][CK * nz + kk], a3);
              }
            }
            float t = (a1 + a3 + a2) * dt;
            t = div_v(t, e ? rc.y : rc.x);
            if (e) nvx.y = ovx.y + t; else nvx.x = ovx.x + t;
          }
        }
        // vy (x int, y half, z int): i in [N+1, nx-N), j in [N, ny-N-1), k in [N+1, nz-N)
        if (i >= N + 1 && i < nx - N && j >= N && j < ny - N - 1) {
          float2 d1 = dplanes<N, false>(pxy, so, c);
          float2 d2 = dstride<N, true>(syy_i, so, G::SW, c);
          float2 d3 = dzp<N, false>(syz_i, so, c);
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int kk = k + e;
            if (kk < N + 1 || kk >= nz - N) continue;
            float a1 = div_c(e ? d1.y : d1.x, dx, rdx, fast);
            float a2 = div_c(e ? d2.y : d2.x, dy, rdy, fast);
            float a3 = div_c(e ? d3.y : d3.x, dz, rdz, fast);
            const int zk = slab_index(kk, nz, p.lo[2], p.hi[2]);
            if ((xi >= 0 || yj >= 0 || zk >= 0) && ((fx & 1) || (fy & 2) || (p.fl[2][kk] & 1))) {
              if (xi >= 0) {
                const size_t o = p.mcomp[0] + ((size_t)xi * ny + j) * nz + kk;
                a1 = pml_step2(vmin[0] + o, tile ? vmout[0] + o : nullptr, p.cf[0][CB * nx + i],
                               p.cf[0][CA * nx + i], p.cf[0][CK * nx + i], a1);
              }
              if (yj >= 0) {
                const size_t o = p.mcomp[1] + ((size_t)i * p.sn[1] + yj) * nz + kk;
                a2 = pml_step2(vmin[1] + o, tile ? vmout[1] + o : nullptr, p.cf[1][CBH * ny + j],
                               p.cf[1][CAH * ny + j], p.cf[1][CKH * ny + j], a2);
              }
              if (zk >= 0) {
                const size_t o = p.mcomp[2] + ((size_t)i * ny + j) * p.sn[2] + zk;
                a3 = pml_step2(vmin[2] + o, tile ? vmout[2] + o : nullptr, p.cf[2][CB * nz + kk],
                               p.cf[2][CA * nz + kk], p.cf[2][CK * nz + kk], a3);
              }
            }
            const float rhy = 0.5f * ((e ? rc.y : rc.x) + (e ? rn.y : rn.x));
            float t = (a1 + a2 + a3) * dt;
            t = div_v(t, rhy);
            if (e) nvy.y = ovy.y + t; else nvy.x = ovy.x + t;
          }
        }
        // vz (x int, y int, z half): i in [N+1, nx-N), j in [N+1, ny-N), k in [N, nz-N-1)
        if (i >= N + 1 && i < nx - N && j >= N + 1 && j < ny - N) {
          const float2 r1c = ld2(r1 + vof), r1n = ld2(r1 + vof + G::VW);
          float2 d1 = dplanes<N, false>(pxz, so, c);
          float2 d2 = dstride<N, false>(syz_i, so, G::SW, c);
          float2 d3 = dzp<N, true>(szz_i, so, c);
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int kk = k + e;
            if (kk < N || kk >= nz - N - 1) continue;
            float a1 = div_c(e ? d1.y : d1.x, dx, rdx, fast);
            float a2 = div_c(e ? d2.y : d2.x, dy, rdy, fast);
            float a3 = div_c(e ? d3.y : d3.x, dz, rdz, fast);
            const int zk = slab_index(kk, nz, p.lo[2], p.hi[2]);
            if ((xi >= 0 || yj >= 0 || zk >= 0) && ((fx & 1) || (fy & 1) || (p.fl[2][kk] & 2))) {
              if (xi >= 0) {
                const size_t o = 2 * p.mcomp[0] + ((size_t)xi * ny + j) * nz + kk;
                a1 = pml_step2(vmin[0] + o, tile ? vmout[0] + o : nullptr, p.cf[0][CB * nx + i],
                               p.cf[0][CA * nx + i], p.cf[0][CK * nx + i], a1);
              }
              if (yj >= 0) {
                const size_t o = 2 * p.mcomp[1] + ((size_t)i * p.sn[1] + yj) * nz + kk;
                a2 = pml_step2(vmin[1] + o, tile ? vmout[1] + o : nullptr, p.cf[1][CB * ny + j],
                               p.cf[1][CA * ny + j], p.cf[1][CK * ny + j], a2);
              }
              if (zk >= 0) {
                const size_t o = 2 * p.mcomp[2] + ((size_t)i * ny + j) * p.sn[2] + zk;
                a3 = pml_step2(vmin[2] + o, tile ? vmout[2] + o : nullptr, p.cf[2][CBH * nz + kk],
                               p.cf[2][CAH * nz + kk], p.cf[2][CKH * nz + kk], a3);
              }
            }
            const float r4 = 0.25f * ((e ? rc.y : rc.x) + (e ? rn.y : rn.x) + (e ? r1n.y : r1n.x) +
                                      (e ? r1c.y : r1c.x));
            const float sum = TENSOR ? (a1 + a2 + a3) : (a3 + a1 + a2);
            float t = sum * dt;
            t = div_v(t, r4);
            if (e) nvz.y = ovz.y + t; else nvz.x = ovz.x + t;
          }
        }
        // point force (Elastic3D_SSG_CPML.py:245)
        if (force && i == p.si && j == p.sj && (k == p.sk || k + 1 == p.sk)) {
          float t = dt * wf;
          t = div_v(t, k == p.sk ? rc.x : rc.y);
          if (k == p.sk) nvz.x = nvz.x + t; else nvz.y = nvz.y + t;
        }
        st2(vv(0, i) + vof, nvx);
        st2(vv(1, i) + vof, nvy);
        st2(vv(2, i) + vof, nvz);
        if (tile) {
          st2(fout[0] + rowg + k, nvx);
          st2(fout[1] + rowg + k, nvy);
          st2(fout[2] + rowg + k, nvz);
        }
      }
      named_sync(1, G::NT);

      // ---------------- stress phase: plane q = i - N on the tile ---------
      const int q = i - N;
      if (q >= x0 && q < x1 && q >= 0) {
        const size_t plq = (size_t)q * nyz;
        const int xq = slab_index(q, nx, p.lo[0], p.hi[0]);
        const uint8_t fxq = p.fl[0][q];
        const float* qvx[2 * N];   // vx planes q-N .. q+N-1   (Dx3bm)
        const float* qvy[2 * N];   // vy planes q-N+1 .. q+N   (Dx3fm)
        const float* qvz[2 * N];
#pragma unroll
        for (int t = 0; t < 2 * N; ++t) {
          qvx[t] = vv(0, q - N + t);
          qvy[t] = vv(1, q - N + 1 + t);
          qvz[t] = vv(2, q - N + 1 + t);
        }
        const float* vxq = vv(0, q);
        const float* vyq = vv(1, q);
        const float* vzq = vv(2, q);
        for (int pi = tid; pi < G::NPS; pi += G::NT) {
          const int r = pi / (G::TZ / 2), cc = pi - r * (G::TZ / 2);
          const int j = j0 + r, k = k0 + 2 * cc;
          if (j >= ny || k >= nz) continue;
          const int vof = (r + N) * G::VW + (G::VZ0 + 2 * cc);
          const size_t gi = plq + (size_t)j * nz + k;
          const int yj = slab_index(j, ny, p.lo[1], p.hi[1]);
          const uint8_t fy = p.fl[1][j];
          const bool src = inject_next && q == p.si && j == p.sj && (k == p.sk || k + 1 == p.sk);
          float2 sxx = ld2(fin[3] + gi), syy = ld2(fin[4] + gi), szz = ld2(fin[5] + gi);
          float2 sxy = ld2(fin[6] + gi), sxz = ld2(fin[7] + gi), syz = ld2(fin[8] + gi);
          const float2 l0 = __ldg(reinterpret_cast<const float2*>(p.lam + gi));
          const float2 u0 = __ldg(reinterpret_cast<const float2*>(p.mu + gi));
          const bool jn = j >= N + 1 && j < ny - N;
          // normal stresses: i,j,k in [N+1, n-N)
          if (q >= N + 1 && q < nx - N && jn) {
            const float2 l1 = __ldg(reinterpret_cast<const float2*>(p.lam + gi + nyz));
            const float2 u1 = __ldg(reinterpret_cast<const float2*>(p.mu + gi + nyz));
            float2 d1 = dplanes<N, false>(qvx, vof, c);
            float2 d2 = dstride<N, false>(vyq, vof, G::VW, c);
            float2 d3 = dzp<N, false>(vzq, vof, c);
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int kk = k + e;
              if (kk < N + 1 || kk >= nz - N) continue;
              float a1 = div_c(e ? d1.y : d1.x, dx, rdx, fast);
              float a2 = div_c(e ? d2.y : d2.x, dy, rdy, fast);
              float a3 = div_c(e ? d3.y : d3.x, dz, rdz, fast);
              const int zk = slab_index(kk, nz, p.lo[2], p.hi[2]);
              if ((xq >= 0 || yj >= 0 || zk >= 0) && ((fxq | fy | p.fl[2][kk]) & 1)) {
                if (xq >= 0)
                  a1 = pml_step(p.mem[0] + 3 * p.mcomp[0] + ((size_t)xq * ny + j) * nz + kk,
                                p.cf[0][CB * nx + q], p.cf[0][CA * nx + q], p.cf[0][CK * nx + q], a1);
                if (yj >= 0)
                  a2 = pml_step(p.mem[1] + 3 * p.mcomp[1] + ((size_t)q * p.sn[1] + yj) * nz + kk,
                                p.cf[1][CB * ny + j], p.cf[1][CA * ny + j], p.cf[1][CK * ny + j], a2);
                if (zk >= 0)
                  a3 = pml_step(p.mem[2] + 3 * p.mcomp[2] + ((size_t)q * ny + j) * p.sn[2] + zk,
                                p.cf[2][CB * nz + kk], p.cf[2][CA * nz + kk], p.cf[2][CK * nz + kk], a3);
              }
              const float lhx = 0.5f * ((e ? l0.y : l0.x) + (e ? l1.y : l1.x));
              const float mhx = 0.5f * ((e ? u0.y : u0.x) + (e ? u1.y : u1.x));
              const float lpm = lhx + 2.0f * mhx;
              const float nxx = (e ? sxx.y : sxx.x) + (lpm * a1 + lhx * (a3 + a2)) * dt;
              const float nyy = (e ? syy.y : syy.x) + (lpm * a2 + lhx * (a1 + a3)) * dt;
              const float nzz = (e ? szz.y : szz.x) + (lpm * a3 + lhx * (a1 + a2)) * dt;
              if (e) { sxx.y = nxx; syy.y = nyy; szz.y = nzz; } else { sxx.x = nxx; syy.x = nyy; szz.x = nzz; }
            }
          }
          // sxy (x half, y half, z int): i,j in [N+1, n-N), k in [N, nz-N)
          if (q >= N + 1 && q < nx - N && jn) {
            const float2 u1 = __ldg(reinterpret_cast<const float2*>(p.mu + gi + nyz));
            const float2 unj = __ldg(reinterpret_cast<const float2*>(p.mu + gi + nz));
            float2 d1 = dplanes<N, true>(qvy, vof, c);
            float2 d2 = dstride<N, true>(vxq, vof, G::VW, c);
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int kk = k + e;
              if (kk < N || kk >= nz - N) continue;
              float a1 = div_c(e ? d1.y : d1.x, dx, rdx, fast);
              float a2 = div_c(e ? d2.y : d2.x, dy, rdy, fast);
              const int zk = slab_index(kk, nz, p.lo[2], p.hi[2]);
              if ((xq >= 0 || yj >= 0 || zk >= 0) && ((fxq & 2) || (fy & 2) || (p.fl[2][kk] & 1))) {
                if (xq >= 0)
                  a1 = pml_step(p.mem[0] + 4 * p.mcomp[0] + ((size_t)xq * ny + j) * nz + kk,
                                p.cf[0][CBH * nx + q], p.cf[0][CAH * nx + q], p.cf[0][CKH * nx + q], a1);
                if (yj >= 0)
                  a2 = pml_step(p.mem[1] + 4 * p.mcomp[1] + ((size_t)q * p.sn[1] + yj) * nz + kk,
                                p.cf[1][CBH * ny + j], p.cf[1][CAH * ny + j], p.cf[1][CKH * ny + j], a2);
              }
              const float u = e ? u0.y : u0.x;
              const float m4 = 0.25f * ((e ? unj.y : unj.x) + u + u + (e ? u1.y : u1.x));
              const float v = (e ? sxy.y : sxy.x) + m4 * (a2 + a1) * dt;
              if (e) sxy.y = v; else sxy.x = v;
            }
          }
          // sxz (x half, y int, z half): i in [N, nx-N-1), j in [N, ny-N), k in [N, nz-N-1)
          if (q >= N && q < nx - N - 1 && j >= N && j < ny - N) {
            const float2 u1 = __ldg(reinterpret_cast<const float2*>(p.mu + gi + nyz));
            const float2 unj = __ldg(reinterpret_cast<const float2*>(p.mu + gi + nz));
            float2 d1 = dplanes<N, true>(qvz, vof, c);
            float2 d2 = dzp<N, true>(vxq, vof, c);
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int kk = k + e;
              if (kk < N || kk >= nz - N - 1) continue;
              float a1 = div_c(e ? d1.y : d1.x, dx, rdx, fast);
              float a2 = div_c(e ? d2.y : d2.x, dz, rdz, fast);
              const int zk = slab_index(kk, nz, p.lo[2], p.hi[2]);
              if ((xq >= 0 || yj >= 0 || zk >= 0) && ((fxq & 2) || (fy & 1) || (p.fl[2][kk] & 2))) {
                if (xq >= 0)
                  a1 = pml_step(p.mem[0] + 5 * p.mcomp[0] + ((size_t)xq * ny + j) * nz + kk,
                                p.cf[0][CBH * nx + q], p.cf[0][CAH * nx + q], p.cf[0][CKH * nx + q], a1);
                if (zk >= 0)
                  a2 = pml_step(p.mem[2] + 4 * p.mcomp[2] + ((size_t)q * ny + j) * p.sn[2] + zk,
                                p.cf[2][CBH * nz + kk], p.cf[2][CAH * nz + kk], p.cf[2][CKH * nz + kk], a2);
              }
              const float u = e ? u0.y : u0.x;
              const float m4 = 0.25f * (u + (e ? u1.y : u1.x) + u + (e ? unj.y : unj.x));
              const float v = (e ? sxz.y : sxz.x) + m4 * (a2 + a1) * dt;
              if (e) sxz.y = v; else sxz.x = v;
            }
          }
          // syz (x int, y half, z half): i in [N, nx-N), j in [N, ny-N-1), k in [N, nz-N-1)
          if (q >= N && q < nx - N && j >= N && j < ny - N - 1) {
            const float2 unj = __ldg(reinterpret_cast<const float2*>(p.mu + gi + nz));
            const float unk0 = __ldg(p.mu + gi + 1), unk1 = __ldg(p.mu + gi + 2);
            float2 d1 = dstride<N, true>(vzq, vof, G::VW, c);
            float2 d2 = dzp<N, true>(vyq, vof, c);
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int kk = k + e;
              if (kk < N || kk >= nz - N - 1) continue;
              float a1 = div_c(e ? d1.y : d1.x, dy, rdy, fast);
              float a2 = div_c(e ? d2.y : d2.x, dz, rdz, fast);
              const int zk = slab_index(kk, nz, p.lo[2], p.hi[2]);
              if ((xq >= 0 || yj >= 0 || zk >= 0) && ((fxq & 1) || (fy & 2) || (p.fl[2][kk] & 2))) {
                if (yj >= 0)
                  a1 = pml_step(p.mem[1] + 5 * p.mcomp[1] + ((size_t)q * p.sn[1] + yj) * nz + kk,
                                p.cf[1][CBH * ny + j], p.cf[1][CAH * ny + j], p.cf[1][CKH * ny + j], a1);
                if (zk >= 0)
                  a2 = pml_step(p.mem[2] + 5 * p.mcomp[2] + ((size_t)q * ny + j) * p.sn[2] + zk,
                                p.cf[2][CBH * nz + kk], p.cf[2][CAH * nz + kk], p.cf[2][CKH * nz + kk], a2);
              }
              const float u = e ? u0.y : u0.x;
              const float m4 = 0.25f * ((e ? unj.y : unj.x) + u + (e ? unk1 : unk0) + u);
              const float v = (e ? syz.y : syz.x) + m4 * (a1 + a2) * dt;
              if (e) syz.y = v; else syz.x = v;
            }
          }
          if (src) {
            // next step's moment-tensor source (Elastic3D_SSG_Tensor.py:186-193)
            if (k == p.sk) {
              sxx.x = sxx.x + wn * p.mneg[0]; syy.x = syy.x + wn * p.mneg[1]; szz.x = szz.x + wn * p.mneg[2];
              sxy.x = sxy.x + wn * p.mneg[3]; sxz.x = sxz.x + wn * p.mneg[4]; syz.x = syz.x + wn * p.mneg[5];
            } else {
              sxx.y = sxx.y + wn * p.mneg[0]; syy.y = syy.y + wn * p.mneg[1]; szz.y = szz.y + wn * p.mneg[2];
              sxy.y = sxy.y + wn * p.mneg[3]; sxz.y = sxz.y + wn * p.mneg[4]; syz.y = syz.y + wn * p.mneg[5];
            }
          }
          st2(fout[3] + gi, sxx);
          st2(fout[4] + gi, syy);
          st2(fout[5] + gi, szz);
          st2(fout[6] + gi, sxy);
          st2(fout[7] + gi, sxz);
          st2(fout[8] + gi, syz);
        }
      }
      __syncthreads();
      if (tid == 0 && s + D + 1 <= i_end) issue(s + D + 1, false, g % (D + 1));
    }
    if (!ok) break;

    // stress planes [nx-N, nx) are never updated: carry them over
    if (x1 == nx) {
      for (int q = max(nx - N, x0); q < nx; ++q) {
        const size_t plq = (size_t)q * nyz;
        for (int pi = tid; pi < G::NPS; pi += G::NT) {
          const int r = pi / (G::TZ / 2), cc = pi - r * (G::TZ / 2);
          const int j = j0 + r, k = k0 + 2 * cc;
          if (j >= ny || k >= nz) continue;
          const size_t gi = plq + (size_t)j * nz + k;
#pragma unroll
          for (int a = 3; a < 9; ++a) st2(fout[a] + gi, ld2(fin[a] + gi));
        }
      }
    }
  }
  if (!ok) {
    // drain: give the copies still in flight a bounded chance to land
    for (int b = 0; b <= D; ++b) mbar_wait(&bars[(g + b) % (D + 1)], ((g + b) / (D + 1)) & 1);
  }
}

// ---------------------------------------------------------------------------
// exhaustive check of the constant-divisor path against IEEE division
// ---------------------------------------------------------------------------
// mode 0: the constant-divisor quotient div_c (r = RN(1/d)); mode 1: the
// per-cell quotient div_v; both against IEEE division, every finite float
// numerator
__global__ void k_check_divc(float d, float r, int mode, unsigned long long* bad) {
  unsigned long long local = 0;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long b = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; b < (1ull << 32);
       b += stride) {
    const float xv = __uint_as_float((unsigned)b);
    if (!isfinite(xv)) continue;
    // the branch-free group routes cover numerators below 2^100
    if (mode >= 2 && !(fabsf(xv) < 0x1p100f)) continue;
    const float a = mode == 0   ? div_c(xv, d, r, 1)
                    : mode == 1 ? div_v(xv, d)
                    : mode == 2 ? mk_div_any(xv, d, r)
                                : dv_div_any(xv, d);
    const float e = __fdiv_rn(xv, d);
    if (__float_as_uint(a) != __float_as_uint(e)) ++local;
  }
  if (local) atomicAdd(bad, local);
}

cudaError_t sw3_check_divisor(float d, float r, unsigned long long* d_bad, unsigned long long* h_bad,
                              cudaStream_t st, int mode) {
  cudaError_t e = cudaMemsetAsync(d_bad, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  k_check_divc<<<148 * 16, 256, 0, st>>>(d, r, mode, d_bad);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(h_bad, d_bad, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(st);
}

// ---------------------------------------------------------------------------
// host side: geometry, tensor maps, launch
// ---------------------------------------------------------------------------
template <int N, int TY, int D>
static FusedConfig cfg_of() {
  using G = FG<N, TY, D>;
  return FusedConfig{N, TY, D, G::BYTES, G::TZ};
}

// the instantiations this build carries: (N, TY, D)
bool sw3_fused_config(int N, FusedConfig* out) {
  switch (N) {
    case 1: *out = cfg_of<1, 16, 2>(); return true;
    case 2: *out = cfg_of<2, 16, 1>(); return true;
    case 3: *out = cfg_of<3, 8, 1>(); return true;
    default: return false;
  }
}

static PFN_cuTensorMapEncodeTiled_v12000 encoder() {
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

// 3D map over a (nx, ny, nz) float array, box {bz, by, 1}; zero fill out of bounds
static bool make_map(CUtensorMap* m, const void* base, int nx, int ny, int nz, int bz, int by) {
  auto enc = encoder();
  if (!enc) return false;
  cuuint64_t dims[3] = {(cuuint64_t)nz, (cuuint64_t)ny, (cuuint64_t)nx};
  cuuint64_t strides[2] = {(cuuint64_t)nz * 4, (cuuint64_t)ny * nz * 4};
  cuuint32_t box[3] = {(cuuint32_t)bz, (cuuint32_t)by, 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(base), dims, strides, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <int N, int TY, int D>
static bool build_maps(const P3<float>& p, const FusedExtra& x, FusedMaps* m) {
  using G = FG<N, TY, D>;
  const int sig_field[6] = {3, 4, 5, 6, 7, 8};
  for (int b = 0; b < 2; ++b) {
    for (int a = 0; a < 6; ++a) {
      const float* base = b == 0 ? p.f[sig_field[a]] : x.fB[sig_field[a]];
      if (!make_map(&m->sig[b][a], base, p.nx, p.ny, p.nz, G::SW, G::SH)) return false;
    }
    for (int a = 0; a < 3; ++a) {
      const float* base = b == 0 ? p.f[a] : x.fB[a];
      if (!make_map(&m->vel[b][a], base, p.nx, p.ny, p.nz, G::VW, G::VH)) return false;
    }
  }
  return make_map(&m->rho, p.rho, p.nx, p.ny, p.nz, G::VW, G::RH);
}

bool sw3_fused_maps(int N, const P3<float>& p, const FusedExtra& x, FusedMaps* m) {
  switch (N) {
    case 1: return build_maps<1, 16, 2>(p, x, m);
    case 2: return build_maps<2, 16, 1>(p, x, m);
    case 3: return build_maps<3, 8, 1>(p, x, m);
    default: return false;
  }
}

template <int N, int TY, int D, bool TENSOR>
static cudaError_t launch_fused(const P3<float>& p, const FusedMaps& m, const FusedExtra& x, int grid, int it,
                                int src, bool inject_next, int gather_it, cudaStream_t st) {
  using G = FG<N, TY, D>;
  static std::atomic<unsigned long long> done{0};
  static std::mutex mu;
  cudaError_t e = once_per_device(done, mu, [] {
    return cudaFuncSetAttribute(k3_fused<N, TY, D, TENSOR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)G::BYTES);
  });
  if (e != cudaSuccess) return e;
  k3_fused<N, TY, D, TENSOR><<<grid, G::NT, G::BYTES, st>>>(p, m, x, it, src, inject_next ? 1 : 0, gather_it);
  return cudaGetLastError();
}

cudaError_t sw3_fused_step(int N, bool tensor, const P3<float>& p, const FusedMaps& m, const FusedExtra& x,
                           int grid, int it, int src, bool inject_next, int gather_it, cudaStream_t st) {
  switch (N) {
    case 1: return tensor ? launch_fused<1, 16, 2, true>(p, m, x, grid, it, src, inject_next, gather_it, st)
                          : launch_fused<1, 16, 2, false>(p, m, x, grid, it, src, inject_next, gather_it, st);
    case 2: return tensor ? launch_fused<2, 16, 1, true>(p, m, x, grid, it, src, inject_next, gather_it, st)
                          : launch_fused<2, 16, 1, false>(p, m, x, grid, it, src, inject_next, gather_it, st);
    case 3: return tensor ? launch_fused<3, 8, 1, true>(p, m, x, grid, it, src, inject_next, gather_it, st)
                          : launch_fused<3, 8, 1, false>(p, m, x, grid, it, src, inject_next, gather_it, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace sw
