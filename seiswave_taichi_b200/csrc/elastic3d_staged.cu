// elastic3d_staged.cu -- TMA-staged two-pass 3D SSG-CPML time step (float),
// the default path of the moment-tensor and point-force schemes
// (src/Elastic3D_SSG_Tensor.py:166-345, src/Elastic3D_SSG_CPML.py:144-309).
//
//   k3s_velocity  vx vy vz (+ point force)               reference :194-243
//   k3s_stress    sxx syy szz sxy sxz syz (+ receivers,  reference :245-310
//                 + next step's moment-tensor source)
//
// Each CTA owns a TY x TZ (y x z) column tile (TZ = 32 or 40) and streams x
// planes.  One elected thread issues cp.async.bulk.tensor loads of whole plane
// tiles (with the halo each array needs) into shared-memory rings, D planes
// ahead, completing on mbarriers; x taps come from the ring planes, y and z
// taps from the halo.  Every thread updates Q consecutive z cells (a "quad",
// Q = 2 or 4, moved with 8- or 16-byte shared and global accesses), and
// prefetches the CPML memory variables (split fields, in the split-PML
// scheme) of the planes ahead.  Update ranges are evaluated per cell and the
// CPML memory variables on their slabs; exact quotients run in range-tested
// groups.  Arithmetic follows the reference's operation order with
// -fmad=false and exact division, so results equal the CPU oracle bit for
// bit.
#include <cudaTypedefs.h>

#include "sw_device.cuh"
#include "sw_staged.cuh"
#include "sw_tma.cuh"

namespace sw {

// SW_OWN_TMA: the plane's own cells (the fields a pass updates) arrive by
// TMA with the neighbour planes instead of per-thread global loads.
#ifndef SW_OWN_TMA
#define SW_OWN_TMA 0
#endif

// z cells per thread: 2 in exact mode, 4 in fast mode.  Two cells per thread
// give the exact passes more resident warps to hide the exact arithmetic's
// dependent chains (at 40-cell tiles: two 320-thread CTAs per SM, 96
// registers, 20 warps); when this was chosen on 256-thread CTAs it measured,
// on B200 at 200^3 (exact, steps 300-500 / 600-800 us per step), 793 / 601
// against 774 / 691 with one cell per thread and 1215 / 746 with four.  The
// fast kernels, with shorter chains, keep four cells (482 us; 594 with two).
constexpr int staged_q(bool exact) { return exact ? 2 : 4; }

// TZ: z cells of a tile, 32 or 40 (the plan takes the width that covers nz
// with the fewest idle cells: 40 divides the 200-cell grids of the 3D
// workloads, where 32-wide tiles leave a last tile of 8)
template <int N, int TY, int D, int Q, int TZ_ = 32>
struct SG {
  static constexpr int TZ = TZ_;
  static constexpr int CQ = TZ / Q;            // threads along z: Q cells each
  static constexpr int NT = TY * CQ;
  // CTAs per SM the register budget aims at (velocity pass, stress pass)
  static constexpr int MINB = NT <= 256 ? 3 : 2;
  static constexpr int MINB_S = Q == 4 && TZ == 32 ? 3 : 2;
  static_assert(TZ % 4 == 0 && TZ % Q == 0, "z tile");
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
  static constexpr int V_OWN = V_R + R2 * pad(B_R);        // vx vy vz of the plane (own cells)
  static constexpr int V_TAB = V_OWN + (SW_OWN_TMA ? 3 * R1 * pad(B_XX) : 0);  // CPML tables of the unit
  static constexpr int TAB = pad(6 * (TY + TZ));
  static constexpr int V_FLOATS = V_TAB + TAB;
  // stress pass layout (floats)
  static constexpr int S_VX = 0;
  static constexpr int S_VY = S_VX + RX * pad(B_YZ);
  static constexpr int S_VZ = S_VY + RX * pad(B_YZ);
  static constexpr int S_L = S_VZ + RX * pad(B_YZ);
  static constexpr int S_M = S_L + R2 * pad(B_L);
  static constexpr int S_OWN = S_M + R2 * pad(B_M);         // the six stresses of the plane (own cells)
  static constexpr int S_TAB = S_OWN + (SW_OWN_TMA ? 6 * R1 * pad(B_L) : 0);
  static constexpr int S_FLOATS = S_TAB + TAB;
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
// ring slot of an x plane: planes are never negative here (the loops start
// at x0 >= N and reach back at most N planes), so an unsigned remainder
// needs no sign fix-up
__device__ __forceinline__ int rslot(int plane, int R) { return (int)((unsigned)plane % (unsigned)R); }

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

// Exact division of a group of stencil sums by the constant spacings, in
// three tiers chosen once per group (the lanes of a tier run one branch-free
// block, so the group's independent values interleave):
//  * every lane zero or of magnitude in [2^-100, 2^100), the spacings'
//    correction verified (fast != 0): Markstein's correction, zeros passed
//    through unchanged (so the sign of zero is kept) -- the steady state;
//  * some lane below 2^-100 (the numerical precursor ahead of a wavefront),
//    none huge: mk_div_any, which gives every lane div_c's bits with the
//    scaled-numerator route selected per lane instead of branched to;
//  * otherwise (a huge value, or the correction unverified) each value
//    takes its own route through div_c.
// The group test, the same predicate as mk_ok on every lane, in three
// instructions per value: the smallest of 2*bits - 2 (unsigned; a zero of
// either sign maps to 0xfffffffe, a magnitude below 2^-100 below
// 2*0x0d800000 - 2) and the largest |x| (NaN is ignored by fmaxf; it stays
// NaN on every path).
struct RangeAcc {
  unsigned lo = 0xffffffffu;
  float hi = 0.f;
  __device__ __forceinline__ void add(float x) {
    lo = min(lo, __float_as_uint(x) * 2u - 2u);
    hi = fmaxf(hi, fabsf(x));
  }
  __device__ __forceinline__ bool ok() const { return lo >= 2u * 0x0D800000u - 2u && hi < 0x1p100f; }
  __device__ __forceinline__ bool below_huge() const { return hi < 0x1p100f; }
};

template <int K, int Q>
__device__ __forceinline__ void div_group(Vq<Q> (&v)[K], const float (&d)[K], const float (&r)[K], int fast) {
  RangeAcc acc;
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int e = 0; e < Q; ++e) acc.add(g4(v[k], e));
  if (fast != 0 && acc.ok()) {
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
      for (int e = 0; e < Q; ++e) s4(v[k], e, mk_div(g4(v[k], e), d[k], r[k]));
  } else if (fast != 0 && acc.below_huge()) {
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
      for (int e = 0; e < Q; ++e) s4(v[k], e, mk_div_any(g4(v[k], e), d[k], r[k]));
  } else {
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
      for (int e = 0; e < Q; ++e) s4(v[k], e, div_c(g4(v[k], e), d[k], r[k], fast));
  }
}

// Exact quotients by per-value positive divisors (densities, CPML kappas) in
// the same three tiers: IEEE division when every numerator is zero or in
// [2^-100, 2^100); dv_div_any (div_v's bits, the scaled route selected per
// lane) when some numerator is smaller, none huge and every divisor lies in
// [2^-60, 2^60]; otherwise div_v per value.
template <int K>
__device__ __forceinline__ void dv_group(float (&x)[K], const float (&d)[K]) {
  RangeAcc acc;
#pragma unroll
  for (int k = 0; k < K; ++k) acc.add(x[k]);
  if (acc.ok()) {
#pragma unroll
    for (int k = 0; k < K; ++k) x[k] = x[k] == 0.f ? x[k] : __fdiv_rn(x[k], d[k]);
    return;
  }
  float dlo = d[0], dhi = d[0];
#pragma unroll
  for (int k = 1; k < K; ++k) {
    dlo = fminf(dlo, d[k]);
    dhi = fmaxf(dhi, d[k]);
  }
  if (acc.below_huge() && dlo >= 0x1p-60f && dhi <= 0x1p60f) {
#pragma unroll
    for (int k = 0; k < K; ++k) x[k] = dv_div_any(x[k], d[k]);
  } else {
#pragma unroll
    for (int k = 0; k < K; ++k) x[k] = div_v(x[k], d[k]);
  }
}

// division by a per-cell positive value: exact, or __fdividef in fast mode
template <bool EX>
__device__ __forceinline__ float dvv(float x, float d) {
  return EX ? div_v(x, d) : __fdividef(x, d);
}

// CPML memory variables.  Outside the slab of an axis the reference's update
// of that axis's memory variable, psi = b*psi + a*d and d = d/kappa + psi, is
// an exact no-op (a = 0, b = 1 and kappa = 1 there, and psi stays 0), so only
// slab cells store memory variables (slab-compact layout) and only they run
// the update.  A slab cell lies inside that axis's PML, where the reference's
// CPML predicate holds, so the update is gated by the component's update
// range alone.  x slabs are whole planes (a uniform branch), y slabs whole
// rows of a thread, z slabs single cells.

// psi update of one value: returns the new psi; d becomes d/kappa + psi
template <bool EX>
__device__ __forceinline__ float cpml1(float& d, float psi, float b, float aa, float kk) {
  const float np = b * psi + aa * d;
  d = dvv<EX>(d, kk) + np;
  return np;
}

// one derivative pair d on an axis whose coefficients are the same for the
// pair's cells (x and y), memory variables o, update mask m
template <bool EX, int Q>
__device__ __forceinline__ void cpml_pair(Vq<Q>& d, Vq<Q>& o, const bool (&m)[Q], float b, float aa, float kk) {
  if constexpr (EX) {
    // cpml1's arithmetic with the Q quotients by kappa as one group
    float np[Q], x[Q], kd[Q];
#pragma unroll
    for (int e = 0; e < Q; ++e) {
      const float de = g4(d, e);
      np[e] = b * g4(o, e) + aa * de;
      x[e] = m[e] ? de : 0.f;
      kd[e] = kk;
    }
    dv_group<Q>(x, kd);
#pragma unroll
    for (int e = 0; e < Q; ++e)
      if (m[e]) {
        s4(o, e, np[e]);
        s4(d, e, x[e] + np[e]);
      }
  } else {
#pragma unroll
    for (int e = 0; e < Q; ++e)
      if (m[e]) {
        float de = g4(d, e);
        s4(o, e, cpml1<EX>(de, g4(o, e), b, aa, kk));
        s4(d, e, de);
      }
  }
}

// the z-slab memory variables of one component: the thread's cells e with
// on[e] (in the z slab and inside the component's update range) advance
// psi (at m2[zk[e] + off]) with the unit's z table row set at integer (HALF
// = false) or half points; the quotients by kappa form one group
template <bool EX, bool HALF, int Q, int TZ>
__device__ __forceinline__ void cpml_z(Vq<Q>& d, float* m2, long long off, const int (&zk)[Q], const bool (&m)[Q],
                                       const float* tzt, int kq) {
  float np[Q], x[Q], kd[Q];
  bool on[Q];
#pragma unroll
  for (int e = 0; e < Q; ++e) {
    on[e] = zk[e] >= 0 && m[e];
    const float b = tab(tzt, HALF ? CBH : CB, TZ, kq + e), aa = tab(tzt, HALF ? CAH : CA, TZ, kq + e);
    const float psi = on[e] ? m2[zk[e] + off] : 0.f;
    const float de = g4(d, e);
    np[e] = b * psi + aa * de;
    x[e] = on[e] ? de : 0.f;
    kd[e] = on[e] ? tab(tzt, HALF ? CKH : CK, TZ, kq + e) : 1.f;
  }
  if constexpr (EX) {
    dv_group<Q>(x, kd);
  } else {
#pragma unroll
    for (int e = 0; e < Q; ++e) x[e] = __fdividef(x[e], kd[e]);
  }
#pragma unroll
  for (int e = 0; e < Q; ++e)
    if (on[e]) {
      m2[zk[e] + off] = np[e];
      s4(d, e, x[e] + np[e]);
    }
}

// L2 prefetch of the memory variables (components c0 .. c0+2 of each slab
// axis) that cell quad (j, k) updates in plane i, issued two planes ahead:
// these loads are the slab cells' longest waits (measured at 200^3, steady
// exact / fast us per step: 458 / 392 without, 449 / 401 one plane ahead,
// 448 / 380 two planes ahead)
template <int Q>
__device__ __forceinline__ void prefetch_memvars(const P3<float>& p, int i, int j, int k, int c0, int yj,
                                                 const int (&zk)[Q], bool zany) {
  const int xn = slab_index(i, p.nx, p.lo[0], p.hi[0]);
  if (xn >= 0) {
    const float* b = p.mem[0] + c0 * p.mcomp[0] + ((size_t)xn * p.ny + j) * p.nz + k;
    for (int c = 0; c < 3; ++c) prefetch_l2(b + c * p.mcomp[0]);
  }
  if (yj >= 0) {
    const float* b = p.mem[1] + c0 * p.mcomp[1] + ((size_t)i * p.sn[1] + yj) * p.nz + k;
    for (int c = 0; c < 3; ++c) prefetch_l2(b + c * p.mcomp[1]);
  }
  if (zany) {
    const int ze = zk[0] >= 0 ? zk[0] : zk[Q - 1];
    const float* b = p.mem[2] + c0 * p.mcomp[2] + ((size_t)i * p.ny + j) * p.sn[2] + ze;
    for (int c = 0; c < 3; ++c) prefetch_l2(b + c * p.mcomp[2]);
  }
}

// L1 prefetch of the split fields (components c0 .. c0+nc-1) of cell quad
// (j, k) in plane i, where the quad's first or last cell lies in the PML
// shell, issued one plane ahead (the split-field scheme's counterpart of
// prefetch_memvars; measured at 200^3: 6.37 Gcell/s against 6.03 with an L2
// prefetch two planes ahead and 5.85 without)
template <int Q>
__device__ __forceinline__ void prefetch_split(const P3<float>& p, int i, int j, int k, int c0, int nc, uint8_t fy,
                                               const uint8_t (&fz)[Q]) {
  const uint8_t fx = p.fl[0][i];
  const int e = (fx | fy | fz[0]) ? 0 : Q - 1;
  if (fx | fy | fz[e]) {
    const float* b = p.split + c0 * p.scomp + shell_index(p, i, j, k + e);
    for (int c = 0; c < nc; ++c) prefetch_l1(b + c * p.scomp);
  }
}

// per-unit CPML table of the tile's rows (y) or z cells: row q of the axis
// coefficient table (b, a, kappa at integer points, then at half points)
__device__ __forceinline__ float tab(const float* t, int row, int len, int at) { return t[row * len + at]; }

// fill the unit's y and z tables; the previous unit's readers have passed the
// last barrier of its plane loop, and the first wait of this unit's loop ends
// in a barrier before any read
template <int TY, int TZ, int NT>
__device__ __forceinline__ void fill_tables(const P3<float>& p, float* tyt, float* tzt, int j0, int k0, int tid) {
  for (int q = tid; q < 6 * (TY + TZ); q += NT) {
    if (q < 6 * TY) {
      const int row = q / TY, jj = j0 + q % TY;
      tyt[q] = jj < p.ny ? __ldg(p.cf[1] + row * p.ny + jj) : 0.f;
    } else {
      const int q2 = q - 6 * TY, row = q2 / TZ, kk = k0 + q2 % TZ;
      tzt[q2] = kk < p.nz ? __ldg(p.cf[2] + row * p.nz + kk) : 0.f;
    }
  }
}

// ---------------------------------------------------------------------------
// split-field PML (src/Elastic3D_SSG_SPML.py:160-393) on the same staged
// tiles: inside a component's PML predicate its split parts advance as
//   psi_d = ((1 - dt/2 d) psi_d + term_d) / (1 + dt/2 d)
// and the field is set to their sum; elsewhere the plain update.  The split
// fields live on the PML shell (shell_index); a cell with a predicate bit set
// lies in the shell.
// ---------------------------------------------------------------------------
enum { SCH_CPML = 0, SCH_SPML = 1 };

__device__ __forceinline__ float spml_part(float psi, float term, float damp, float hdt) {
  return div_v((1.f - hdt * damp) * psi + term, 1.f + hdt * damp);
}

template <int Q>
__device__ __forceinline__ void spml_velocity(const P3<float>& p, int i, int j, int k, uint8_t fy,
                                              const uint8_t (&fz)[Q], float dt, const bool (&mx)[Q],
                                              const bool (&my)[Q], const bool (&mz)[Q], const Vq<Q>& a1,
                                              const Vq<Q>& a2, const Vq<Q>& a3, const Vq<Q>& b1, const Vq<Q>& b2,
                                              const Vq<Q>& b3, const Vq<Q>& c1, const Vq<Q>& c2, const Vq<Q>& c3,
                                              const Vq<Q>& rc, const Vq<Q>& rn, const Vq<Q>& r1c, const Vq<Q>& r1n,
                                              Vq<Q>& vx, Vq<Q>& vy, Vq<Q>& vz) {
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const uint8_t fx = p.fl[0][i];
  const float hdt = 0.5f * dt;
  const float *dpx = p.dmp[0], *dpy = p.dmp[1], *dpz = p.dmp[2];
  float* sp = p.split;
  const long long G = p.scomp;
#pragma unroll
  for (int e = 0; e < Q; ++e) {
    const int kk = k + e;
    const uint8_t fze = fz[e];
    const long long sh = (fx | fy | fze) ? shell_index(p, i, j, kk) : 0;
    const float rce = g4(rc, e), rne = g4(rn, e);
    // vx (:182-205): x half, y and z integer; rho unaveraged
    if (mx[e]) {
      const float ro = __fdiv_rn(1.f, rce);
      const float d1 = g4(a1, e), d2 = g4(a2, e), d3 = g4(a3, e);
      if ((fx & 2) || (fy & 1) || (fze & 1)) {
        float* s = sp + PVX_X * G + sh;
        const float A = spml_part(s[0], d1 * dt * ro, __ldg(dpx + nx + i), hdt);
        const float B = spml_part(s[G], d2 * dt * ro, __ldg(dpy + j), hdt);
        const float C = spml_part(s[2 * G], d3 * dt * ro, __ldg(dpz + kk), hdt);
        s[0] = A;
        s[G] = B;
        s[2 * G] = C;
        s4(vx, e, A + B + C);
      } else {
        s4(vx, e, g4(vx, e) + (d1 + d2 + d3) * dt * ro);
      }
    }
    // vy (:209-233): y half; rho averaged over j, j+1
    if (my[e]) {
      const float ro = __fdiv_rn(1.f, 0.5f * (rce + rne));
      const float d1 = g4(b1, e), d2 = g4(b2, e), d3 = g4(b3, e);
      if ((fx & 1) || (fy & 2) || (fze & 1)) {
        float* s = sp + PVY_X * G + sh;
        const float A = spml_part(s[0], dt * d1 * ro, __ldg(dpx + i), hdt);
        const float B = spml_part(s[G], dt * d2 * ro, __ldg(dpy + ny + j), hdt);
        const float C = spml_part(s[2 * G], dt * d3 * ro, __ldg(dpz + kk), hdt);
        s[0] = A;
        s[G] = B;
        s[2 * G] = C;
        s4(vy, e, A + B + C);
      } else {
        s4(vy, e, g4(vy, e) + (d1 + d2 + d3) * dt * ro);
      }
    }
    // vz (:235-259): z half; rho averaged over the x-y quad
    if (mz[e]) {
      const float ro = __fdiv_rn(1.f, 0.25f * (rce + rne + g4(r1n, e) + g4(r1c, e)));
      const float d1 = g4(c1, e), d2 = g4(c2, e), d3 = g4(c3, e);
      if ((fx & 1) || (fy & 1) || (fze & 2)) {
        float* s = sp + PVZ_X * G + sh;
        const float A = spml_part(s[0], dt * d1 * ro, __ldg(dpx + i), hdt);
        const float B = spml_part(s[G], dt * d2 * ro, __ldg(dpy + j), hdt);
        const float C = spml_part(s[2 * G], dt * d3 * ro, __ldg(dpz + nz + kk), hdt);
        s[0] = A;
        s[G] = B;
        s[2 * G] = C;
        s4(vz, e, A + B + C);
      } else {
        s4(vz, e, g4(vz, e) + (d1 + d2 + d3) * dt * ro);
      }
    }
  }
}

template <int Q>
__device__ __forceinline__ void spml_stress(const P3<float>& p, int i, int j, int k, uint8_t fy,
                                            const uint8_t (&fz)[Q], float dt, const bool (&mn)[Q],
                                            const bool (&mxy)[Q], const bool (&mxz)[Q], const bool (&myz)[Q],
                                            const Vq<Q>& e1, const Vq<Q>& e2, const Vq<Q>& e3, const Vq<Q>& f1,
                                            const Vq<Q>& f2, const Vq<Q>& h1, const Vq<Q>& h2, const Vq<Q>& q1,
                                            const Vq<Q>& q2, const Vq<Q>& l0, const Vq<Q>& u0, const Vq<Q>& u1,
                                            const Vq<Q>& unj, const float (&unk)[Q], Vq<Q>& sxx, Vq<Q>& syy,
                                            Vq<Q>& szz, Vq<Q>& sxy, Vq<Q>& sxz, Vq<Q>& syz) {
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const uint8_t fx = p.fl[0][i];
  const float hdt = 0.5f * dt;
  const float *dpx = p.dmp[0], *dpy = p.dmp[1], *dpz = p.dmp[2];
  float* sp = p.split;
  const long long G = p.scomp;
#pragma unroll
  for (int e = 0; e < Q; ++e) {
    const int kk = k + e;
    const uint8_t fze = fz[e];
    const long long sh = (fx | fy | fze) ? shell_index(p, i, j, kk) : 0;
    const float u = g4(u0, e);
    // normal stresses (:296-333): unaveraged lambda and mu
    if (mn[e]) {
      const float lm = g4(l0, e);
      const float l2m = lm + 2.f * u;
      const float A = g4(e1, e), B = g4(e2, e), Cc = g4(e3, e);
      if ((fx | fy | fze) & 1) {
        const float dX = __ldg(dpx + i), dY = __ldg(dpy + j), dZ = __ldg(dpz + kk);
        float* s = sp + sh;
        const float xx = spml_part(s[PSXX_X * G], dt * l2m * A, dX, hdt);
        const float xy = spml_part(s[PSXX_Y * G], dt * lm * B, dY, hdt);
        const float xz = spml_part(s[PSXX_Z * G], dt * lm * Cc, dZ, hdt);
        const float yx = spml_part(s[PSYY_X * G], dt * lm * A, dX, hdt);
        const float yy = spml_part(s[PSYY_Y * G], dt * l2m * B, dY, hdt);
        const float yz = spml_part(s[PSYY_Z * G], dt * lm * Cc, dZ, hdt);
        const float zx = spml_part(s[PSZZ_X * G], dt * lm * A, dX, hdt);
        const float zy = spml_part(s[PSZZ_Y * G], dt * lm * B, dY, hdt);
        const float zz = spml_part(s[PSZZ_Z * G], dt * l2m * Cc, dZ, hdt);
        s[PSXX_X * G] = xx; s[PSXX_Y * G] = xy; s[PSXX_Z * G] = xz;
        s[PSYY_X * G] = yx; s[PSYY_Y * G] = yy; s[PSYY_Z * G] = yz;
        s[PSZZ_X * G] = zx; s[PSZZ_Y * G] = zy; s[PSZZ_Z * G] = zz;
        s4(sxx, e, xx + xy + xz);
        s4(syy, e, yx + yy + yz);
        s4(szz, e, zx + zy + zz);
      } else {
        s4(sxx, e, g4(sxx, e) + (l2m * A + lm * (Cc + B)) * dt);
        s4(syy, e, g4(syy, e) + (l2m * B + lm * (A + Cc)) * dt);
        s4(szz, e, g4(szz, e) + (l2m * Cc + lm * (A + B)) * dt);
      }
    }
    // sxy (:334-350): x half, y half
    if (mxy[e]) {
      const float m4 = 0.25f * (g4(unj, e) + u + u + g4(u1, e));
      if ((fx & 2) || (fy & 2) || (fze & 1)) {
        float* s = sp + PSXY_X * G + sh;
        const float a = spml_part(s[0], dt * m4 * g4(f1, e), __ldg(dpx + nx + i), hdt);
        const float b = spml_part(s[G], dt * m4 * g4(f2, e), __ldg(dpy + ny + j), hdt);
        s[0] = a;
        s[G] = b;
        s4(sxy, e, a + b);
      } else {
        s4(sxy, e, g4(sxy, e) + m4 * (g4(f2, e) + g4(f1, e)) * dt);
      }
    }
    // sxz (:352-371): x half, z half
    if (mxz[e]) {
      const float m4 = 0.25f * (u + g4(u1, e) + u + g4(unj, e));
      if ((fx & 2) || (fy & 1) || (fze & 2)) {
        float* s = sp + PSXZ_X * G + sh;
        const float a = spml_part(s[0], dt * m4 * g4(h1, e), __ldg(dpx + nx + i), hdt);
        const float b = spml_part(s[G], dt * m4 * g4(h2, e), __ldg(dpz + nz + kk), hdt);
        s[0] = a;
        s[G] = b;
        s4(sxz, e, a + b);
      } else {
        s4(sxz, e, g4(sxz, e) + m4 * (g4(h2, e) + g4(h1, e)) * dt);
      }
    }
    // syz (:373-391): y half, z half; its plain update adds dvy/dz + dvz/dy
    if (myz[e]) {
      const float m4 = 0.25f * (g4(unj, e) + u + unk[e] + u);
      if ((fx & 1) || (fy & 2) || (fze & 2)) {
        float* s = sp + PSYZ_Y * G + sh;
        const float a = spml_part(s[0], dt * m4 * g4(q1, e), __ldg(dpy + ny + j), hdt);
        const float b = spml_part(s[G], dt * m4 * g4(q2, e), __ldg(dpz + nz + kk), hdt);
        s[0] = a;
        s[G] = b;
        s4(syz, e, a + b);
      } else {
        s4(syz, e, g4(syz, e) + m4 * (g4(q2, e) + g4(q1, e)) * dt);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// velocity pass
// ---------------------------------------------------------------------------
template <int N, int TY, int D, bool TENSOR, bool EX, int Q, int TZ, int SCH>
__global__ void __launch_bounds__(SG<N, TY, D, Q, TZ>::NT, SG<N, TY, D, Q, TZ>::MINB)
k3s_velocity(const __grid_constant__ P3<float> p, const __grid_constant__ StagedMaps maps,
             const __grid_constant__ StagedArgs a, int it, int force_here) {
  using G = SG<N, TY, D, Q, TZ>;
  extern __shared__ __align__(128) float sm[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + G::V_FLOATS);
  float* tyt = sm + G::V_TAB;   // [6][TY]
  float* tzt = tyt + 6 * TY;    // [6][TZ]
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
  auto own_p = [&](int a, int pl) { return sm + G::V_OWN + (a * G::R1 + rslot(pl, G::R1)) * PXX; };
  const int o_xx = r * G::TZ + Q * cq;                 // sxx, rho, own-cell boxes
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
    if (SCH == SCH_CPML) fill_tables<TY, G::TZ, G::NT>(p, tyt, tzt, j0, k0, tid);
    const int j = j0 + r, k = k0 + Q * cq;
    const bool jin = j < ny, kin = k < nz;
    const int yj = SCH == SCH_CPML && jin ? slab_index(j, ny, p.lo[1], p.hi[1]) : -1;
    int zk[Q];
    bool zany = false;
#pragma unroll
    for (int e = 0; e < Q; ++e) {
      zk[e] = SCH == SCH_CPML && k + e < nz ? slab_index(k + e, nz, p.lo[2], p.hi[2]) : -1;
      zany = zany || zk[e] >= 0;
    }
    // update ranges in y and z (Elastic3D_SSG_Tensor.py:194,210,226):
    // vx and vz rows j in [N+1, ny-N), vy rows j in [N, ny-N-1); vx and vy
    // cells k in [N+1, nz-N), vz cells k in [N, nz-N-1)
    const bool jxz = j >= N + 1 && j < ny - N, jy = j >= N && j < ny - N - 1;
    // split PML: predicate flags of the row and of the z cells
    const uint8_t fy = SCH == SCH_SPML && jin ? p.fl[1][j] : 0;
    uint8_t fz[Q];
#pragma unroll
    for (int e = 0; e < Q; ++e) fz[e] = SCH == SCH_SPML && k + e < nz ? p.fl[2][k + e] : 0;
    bool kxy[Q], kz[Q];
#pragma unroll
    for (int e = 0; e < Q; ++e) {
      kxy[e] = k + e >= N + 1 && k + e < nz - N;
      kz[e] = k + e >= N && k + e < nz - N - 1;
    }

    auto issue = [&](int s, bool first, uint32_t stage) {
      uint64_t* bar = &bars[stage];
      // sxx + sxy + sxz + syy + syz + szz + rho + the plane's own vx vy vz
      uint32_t bytes = ((SW_OWN_TMA ? 4 : 1) * G::B_XX + 2 * G::B_Y + 2 * G::B_Z + G::B_YZ + G::B_R) * 4;
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
      if (SW_OWN_TMA)
        for (int c = 0; c < 3; ++c) tma_load3(own_p(c, s), &maps.m[7 + c], k0, j0, s, bar);
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
      // this plane's data (bounded wait); the CTA agrees on the outcome
      const bool landed = mbar_wait(&bars[g % (D + 1)], (g / (D + 1)) & 1);
      if (__syncthreads_or(!landed)) {
        if (tid == 0) atomicOr(a.err, 1);
        ok = false;
        break;
      }
      const int xi = SCH == SCH_CPML ? slab_index(i, nx, p.lo[0], p.hi[0]) : -1;
      if constexpr (SCH == SCH_CPML)
        if (jin && kin && i + 2 < x1) prefetch_memvars(p, i + 2, j, k, 0, yj, zk, zany);
      if constexpr (SCH == SCH_SPML)
        if (jin && kin && i + 1 < x1) prefetch_split(p, i + 1, j, k, PVX_X, 9, fy, fz);
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
        Vq<Q> vx, vy, vz;
        if (SW_OWN_TMA) {
          vx = ldq<Q>(own_p(0, i) + o_xx), vy = ldq<Q>(own_p(1, i) + o_xx), vz = ldq<Q>(own_p(2, i) + o_xx);
        } else {
          vx = ldgq<Q>(p.f[0] + gi), vy = ldgq<Q>(p.f[1] + gi), vz = ldgq<Q>(p.f[2] + gi);
        }
        // update masks: vx i in [N, nx-N-1), vy and vz i in [N+1, nx-N)
        const bool ix = i < nx - N - 1, iyz = i >= N + 1;
        bool mx[Q], my[Q], mz[Q];
#pragma unroll
        for (int e = 0; e < Q; ++e) {
          mx[e] = ix && jxz && kxy[e];
          my[e] = iyz && jy && kxy[e];
          mz[e] = iyz && jxz && kz[e];
        }
        const Vq<Q> rc = ldq<Q>(r0 + o_xx), rn = ldq<Q>(r0 + o_xx + G::TZ);
        const Vq<Q> r1c = ldq<Q>(r1 + o_xx), r1n = ldq<Q>(r1 + o_xx + G::TZ);
        if constexpr (SCH == SCH_SPML) {
          spml_velocity<Q>(p, i, j, k, fy, fz, dt, mx, my, mz, a1, a2, a3, b1, b2, b3, c1, c2, c3, rc, rn, r1c, r1n,
                           vx, vy, vz);
        } else {
          // CPML: components 0 (vx), 1 (vy), 2 (vz) of each axis; vx is at
          // the x half point, vy at the y half point, vz at the z half point
          if (xi >= 0) {
            const float* cf = p.cf[0];
            const float bi = __ldg(cf + CB * nx + i), ai = __ldg(cf + CA * nx + i), ki = __ldg(cf + CK * nx + i);
            const float bh = __ldg(cf + CBH * nx + i), ah = __ldg(cf + CAH * nx + i),
                        kh = __ldg(cf + CKH * nx + i);
            float* m0 = p.mem[0] + ((size_t)xi * ny + j) * nz + k;
            const long long mc = p.mcomp[0];
            Vq<Q> s0 = ldq<Q>(m0), s1 = ldq<Q>(m0 + mc), s2 = ldq<Q>(m0 + 2 * mc);
            cpml_pair<EX, Q>(a1, s0, mx, bh, ah, kh);
            cpml_pair<EX, Q>(b1, s1, my, bi, ai, ki);
            cpml_pair<EX, Q>(c1, s2, mz, bi, ai, ki);
            stq<Q>(m0, s0);
            stq<Q>(m0 + mc, s1);
            stq<Q>(m0 + 2 * mc, s2);
          }
          if (yj >= 0) {
            const float bi = tab(tyt, CB, TY, r), ai = tab(tyt, CA, TY, r), ki = tab(tyt, CK, TY, r);
            const float bh = tab(tyt, CBH, TY, r), ah = tab(tyt, CAH, TY, r), kh = tab(tyt, CKH, TY, r);
            float* m1 = p.mem[1] + ((size_t)i * p.sn[1] + yj) * nz + k;
            const long long mc = p.mcomp[1];
            Vq<Q> s0 = ldq<Q>(m1), s1 = ldq<Q>(m1 + mc), s2 = ldq<Q>(m1 + 2 * mc);
            cpml_pair<EX, Q>(a2, s0, mx, bi, ai, ki);
            cpml_pair<EX, Q>(b2, s1, my, bh, ah, kh);
            cpml_pair<EX, Q>(c2, s2, mz, bi, ai, ki);
            stq<Q>(m1, s0);
            stq<Q>(m1 + mc, s1);
            stq<Q>(m1 + 2 * mc, s2);
          }
          if (zany) {
            float* m2 = p.mem[2] + ((size_t)i * ny + j) * p.sn[2];
            const long long mc = p.mcomp[2];
            cpml_z<EX, false, Q, G::TZ>(a3, m2, 0, zk, mx, tzt, Q * cq);
            cpml_z<EX, false, Q, G::TZ>(b3, m2, mc, zk, my, tzt, Q * cq);
            cpml_z<EX, true, Q, G::TZ>(c3, m2, 2 * mc, zk, mz, tzt, Q * cq);
          }
          // numerators and densities of the 3Q updates, then their quotients
          // as one group (no per-lane range branch); masked cells keep their value
          float tn[3 * Q], td[3 * Q];
#pragma unroll
          for (int e = 0; e < Q; ++e) {
            const float rce = g4(rc, e), rne = g4(rn, e);
            tn[e] = (g4(a1, e) + g4(a3, e) + g4(a2, e)) * dt;
            td[e] = rce;
            tn[Q + e] = (g4(b1, e) + g4(b2, e) + g4(b3, e)) * dt;
            td[Q + e] = 0.5f * (rce + rne);
            const float sum =
                TENSOR ? (g4(c1, e) + g4(c2, e) + g4(c3, e)) : (g4(c3, e) + g4(c1, e) + g4(c2, e));
            tn[2 * Q + e] = sum * dt;
            td[2 * Q + e] = 0.25f * (rce + rne + g4(r1n, e) + g4(r1c, e));
          }
          if (EX) {
            dv_group<3 * Q>(tn, td);
          } else {
#pragma unroll
            for (int q = 0; q < 3 * Q; ++q) tn[q] = __fdividef(tn[q], td[q]);
          }
#pragma unroll
          for (int e = 0; e < Q; ++e) {
            if (mx[e]) s4(vx, e, g4(vx, e) + tn[e]);
            if (my[e]) s4(vy, e, g4(vy, e) + tn[Q + e]);
            if (mz[e]) s4(vz, e, g4(vz, e) + tn[2 * Q + e]);
          }
        }
        // point force (Elastic3D_SSG_CPML.py:245, Elastic3D_SSG_SPML.py:294),
        // after the update
        if (force_here && i == p.si && j == p.sj && p.sk >= k && p.sk < k + Q) {
          const int e = p.sk - k;
          const float t = dt * wf;
          s4(vz, e, g4(vz, e) + dvv<EX>(t, g4(rc, e)));
        }
        stq<Q>(p.f[0] + gi, vx);
        stq<Q>(p.f[1] + gi, vy);
        stq<Q>(p.f[2] + gi, vz);
      }
      // every thread is done with plane i's ring slots, which plane i+D+1 refills
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
template <int N, int TY, int D, bool EX, int Q, int TZ, int SCH>
__global__ void __launch_bounds__(SG<N, TY, D, Q, TZ>::NT, SG<N, TY, D, Q, TZ>::MINB_S)
k3s_stress(const __grid_constant__ P3<float> p, const __grid_constant__ StagedMaps maps,
           const __grid_constant__ StagedArgs a, int it, int inject_next, int gather) {
  using G = SG<N, TY, D, Q, TZ>;
  extern __shared__ __align__(128) float sm[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + G::S_FLOATS);
  float* tyt = sm + G::S_TAB;   // [6][TY]
  float* tzt = tyt + 6 * TY;    // [6][TZ]
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
  auto own_p = [&](int a, int pl) { return sm + G::S_OWN + (a * G::R1 + rslot(pl, G::R1)) * PL; };
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
    if (SCH == SCH_CPML) fill_tables<TY, G::TZ, G::NT>(p, tyt, tzt, j0, k0, tid);
    const int j = j0 + r, k = k0 + Q * cq;
    const bool jin = j < ny, kin = k < nz;
    const int yj = SCH == SCH_CPML && jin ? slab_index(j, ny, p.lo[1], p.hi[1]) : -1;
    int zk[Q];
    bool zany = false;
#pragma unroll
    for (int e = 0; e < Q; ++e) {
      zk[e] = SCH == SCH_CPML && k + e < nz ? slab_index(k + e, nz, p.lo[2], p.hi[2]) : -1;
      zany = zany || zk[e] >= 0;
    }
    // update ranges in y and z (Elastic3D_SSG_Tensor.py:247,267,281,295):
    // normal stresses j, k in [N+1, n-N); sxy j in [N+1, ny-N), k in [N, nz-N);
    // sxz j in [N, ny-N), k in [N, nz-N-1); syz j in [N, ny-N-1), k in [N, nz-N-1)
    const bool jn = j >= N + 1 && j < ny - N, jxz = j >= N && j < ny - N, jyz = j >= N && j < ny - N - 1;
    const uint8_t fy = SCH == SCH_SPML && jin ? p.fl[1][j] : 0;
    uint8_t fz[Q];
#pragma unroll
    for (int e = 0; e < Q; ++e) fz[e] = SCH == SCH_SPML && k + e < nz ? p.fl[2][k + e] : 0;
    bool kn[Q], kxy[Q], kh[Q];
#pragma unroll
    for (int e = 0; e < Q; ++e) {
      kn[e] = k + e >= N + 1 && k + e < nz - N;
      kxy[e] = k + e >= N && k + e < nz - N;
      kh[e] = k + e >= N && k + e < nz - N - 1;
    }

    auto issue = [&](int s, bool first, uint32_t stage) {
      uint64_t* bar = &bars[stage];
      // vx vy vz + lam + mu + the plane's own six stresses
      uint32_t bytes = (3 * G::B_YZ + (SW_OWN_TMA ? 7 : 1) * G::B_L + G::B_M) * 4;
      if (first) bytes += ((2 * N - 1) * 3 * G::B_YZ + G::B_L + G::B_M) * 4;
      mbar_expect_tx(bar, bytes);
      const int zh = k0 - G::H4, yh = j0 - N;
      // vx planes up to s+N-1 (Dx3bm), vy / vz up to s+N (Dx3fm)
      tma_load3(vx_p(s + N - 1), &maps.m[0], zh, yh, s + N - 1, bar);
      tma_load3(vy_p(s + N), &maps.m[1], zh, yh, s + N, bar);
      tma_load3(vz_p(s + N), &maps.m[2], zh, yh, s + N, bar);
      tma_load3(lam_p(s + 1), &maps.m[3], k0, j0, s + 1, bar);
      tma_load3(mu_p(s + 1), &maps.m[4], k0, j0, s + 1, bar);
      if (SW_OWN_TMA)
        for (int c = 0; c < 6; ++c) tma_load3(own_p(c, s), &maps.m[5 + c], k0, j0, s, bar);
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
      // this plane's data (bounded wait); the CTA agrees on the outcome
      const bool landed = mbar_wait(&bars[g % (D + 1)], (g / (D + 1)) & 1);
      if (__syncthreads_or(!landed)) {
        if (tid == 0) atomicOr(a.err, 1);
        ok = false;
        break;
      }
      const int xi = SCH == SCH_CPML ? slab_index(i, nx, p.lo[0], p.hi[0]) : -1;
      if constexpr (SCH == SCH_CPML)
        if (jin && kin && i + 2 < x1) prefetch_memvars(p, i + 2, j, k, 3, yj, zk, zany);
      if constexpr (SCH == SCH_SPML)
        if (jin && kin && i + 1 < x1) prefetch_split(p, i + 1, j, k, PSXX_X, 15, fy, fz);
      const bool src = inject_next && i == p.si && p.sj == j && p.sk >= k && p.sk < k + Q;
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
        Vq<Q> sxx, syy, szz, sxy, sxz, syz;
        if (SW_OWN_TMA) {
          sxx = ldq<Q>(own_p(0, i) + o_l), syy = ldq<Q>(own_p(1, i) + o_l), szz = ldq<Q>(own_p(2, i) + o_l);
          sxy = ldq<Q>(own_p(3, i) + o_l), sxz = ldq<Q>(own_p(4, i) + o_l), syz = ldq<Q>(own_p(5, i) + o_l);
        } else {
          sxx = ldgq<Q>(p.f[3] + gi), syy = ldgq<Q>(p.f[4] + gi), szz = ldgq<Q>(p.f[5] + gi);
          sxy = ldgq<Q>(p.f[6] + gi), sxz = ldgq<Q>(p.f[7] + gi), syz = ldgq<Q>(p.f[8] + gi);
        }
        // update masks: normal stresses and sxy i in [N+1, nx-N), sxz i in
        // [N, nx-N-1), syz every plane of the loop
        const bool in_ = i >= N + 1, ixz = i < nx - N - 1;
        bool mn[Q], mxy[Q], mxz[Q], myz[Q];
#pragma unroll
        for (int e = 0; e < Q; ++e) {
          mn[e] = in_ && jn && kn[e];
          mxy[e] = in_ && jn && kxy[e];
          mxz[e] = ixz && jxz && kh[e];
          myz[e] = jyz && kh[e];
        }
        const Vq<Q> l0 = ldq<Q>(lam_p(i) + o_l), l1 = ldq<Q>(lam_p(i + 1) + o_l);
        const float* m0p = mu_p(i);
        const Vq<Q> u0 = ldq<Q>(m0p + o_m), u1 = ldq<Q>(mu_p(i + 1) + o_m), unj = ldq<Q>(m0p + o_m + G::WM);
        float unk[Q];  // mu[k+1 .. k+Q] for the k+1 neighbours
#pragma unroll
        for (int e = 0; e + 1 < Q; ++e) unk[e] = g4(u0, e + 1);
        unk[Q - 1] = m0p[o_m + Q];
        if constexpr (SCH == SCH_SPML) {
          spml_stress<Q>(p, i, j, k, fy, fz, dt, mn, mxy, mxz, myz, e1, e2, e3, f1, f2, h1, h2, q1, q2, l0, u0, u1,
                         unj, unk, sxx, syy, szz, sxy, sxz, syz);
        } else {
          // CPML: components 3 (normal), 4, 5 of each axis
          if (xi >= 0) {
            const float* cf = p.cf[0];
            const float bi = __ldg(cf + CB * nx + i), ai = __ldg(cf + CA * nx + i), ki = __ldg(cf + CK * nx + i);
            const float bh = __ldg(cf + CBH * nx + i), ah = __ldg(cf + CAH * nx + i),
                        khx = __ldg(cf + CKH * nx + i);
            const long long mc = p.mcomp[0];
            float* m0 = p.mem[0] + 3 * mc + ((size_t)xi * ny + j) * nz + k;
            Vq<Q> s0 = ldq<Q>(m0), s1 = ldq<Q>(m0 + mc), s2 = ldq<Q>(m0 + 2 * mc);
            cpml_pair<EX, Q>(e1, s0, mn, bi, ai, ki);    // dvx_dx
            cpml_pair<EX, Q>(f1, s1, mxy, bh, ah, khx);  // dvy_dx
            cpml_pair<EX, Q>(h1, s2, mxz, bh, ah, khx);  // dvz_dx
            stq<Q>(m0, s0);
            stq<Q>(m0 + mc, s1);
            stq<Q>(m0 + 2 * mc, s2);
          }
          if (yj >= 0) {
            const float bi = tab(tyt, CB, TY, r), ai = tab(tyt, CA, TY, r), ki = tab(tyt, CK, TY, r);
            const float bh = tab(tyt, CBH, TY, r), ah = tab(tyt, CAH, TY, r), khy = tab(tyt, CKH, TY, r);
            const long long mc = p.mcomp[1];
            float* m1 = p.mem[1] + 3 * mc + ((size_t)i * p.sn[1] + yj) * nz + k;
            Vq<Q> s0 = ldq<Q>(m1), s1 = ldq<Q>(m1 + mc), s2 = ldq<Q>(m1 + 2 * mc);
            cpml_pair<EX, Q>(e2, s0, mn, bi, ai, ki);    // dvy_dy
            cpml_pair<EX, Q>(f2, s1, mxy, bh, ah, khy);  // dvx_dy
            cpml_pair<EX, Q>(q1, s2, myz, bh, ah, khy);  // dvz_dy
            stq<Q>(m1, s0);
            stq<Q>(m1 + mc, s1);
            stq<Q>(m1 + 2 * mc, s2);
          }
          if (zany) {
            const long long mc = p.mcomp[2];
            float* m2 = p.mem[2] + 3 * mc + ((size_t)i * ny + j) * p.sn[2];
            cpml_z<EX, false, Q, G::TZ>(e3, m2, 0, zk, mn, tzt, Q * cq);      // dvz_dz
            cpml_z<EX, true, Q, G::TZ>(h2, m2, mc, zk, mxz, tzt, Q * cq);     // dvx_dz
            cpml_z<EX, true, Q, G::TZ>(q2, m2, 2 * mc, zk, myz, tzt, Q * cq); // dvy_dz
          }
#pragma unroll
          for (int e = 0; e < Q; ++e) {
            const float u = g4(u0, e);
            if (mn[e]) {
              const float lhx = 0.5f * (g4(l0, e) + g4(l1, e));
              const float mhx = 0.5f * (u + g4(u1, e));
              const float lpm = lhx + 2.0f * mhx;
              const float A = g4(e1, e), B = g4(e2, e), Cc = g4(e3, e);
              s4(sxx, e, g4(sxx, e) + (lpm * A + lhx * (Cc + B)) * dt);
              s4(syy, e, g4(syy, e) + (lpm * B + lhx * (A + Cc)) * dt);
              s4(szz, e, g4(szz, e) + (lpm * Cc + lhx * (A + B)) * dt);
            }
            if (mxy[e]) {
              const float m4 = 0.25f * (g4(unj, e) + u + u + g4(u1, e));
              s4(sxy, e, g4(sxy, e) + m4 * (g4(f2, e) + g4(f1, e)) * dt);
            }
            if (mxz[e]) {
              const float m4 = 0.25f * (u + g4(u1, e) + u + g4(unj, e));
              s4(sxz, e, g4(sxz, e) + m4 * (g4(h2, e) + g4(h1, e)) * dt);
            }
            if (myz[e]) {
              const float m4 = 0.25f * (g4(unj, e) + u + unk[e] + u);
              s4(syz, e, g4(syz, e) + m4 * (g4(q1, e) + g4(q2, e)) * dt);
            }
          }
        }
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
        stq<Q>(p.f[3] + gi, sxx);
        stq<Q>(p.f[4] + gi, syy);
        stq<Q>(p.f[5] + gi, szz);
        stq<Q>(p.f[6] + gi, sxy);
        stq<Q>(p.f[7] + gi, sxz);
        stq<Q>(p.f[8] + gi, syz);
      }
      // every thread is done with plane i's ring slots, which plane i+D+1 refills
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

template <int N, int TY, int D, int TZ>
static bool staged_maps_t(const P3<float>& p, StagedMaps* vm, StagedMaps* sm_) {
  using G = SG<N, TY, D, 4, TZ>;  // box shapes do not depend on the cells per thread
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
  for (int c = 0; c < 3; ++c) ok = ok && map3(&vm->m[7 + c], p.f[c], nx, ny, nz, G::TZ, TY);
  // stress pass: vx vy vz lam mu, then the six stresses
  ok = ok && map3(&sm_->m[0], p.f[0], nx, ny, nz, G::WZ, G::HY);
  ok = ok && map3(&sm_->m[1], p.f[1], nx, ny, nz, G::WZ, G::HY);
  ok = ok && map3(&sm_->m[2], p.f[2], nx, ny, nz, G::WZ, G::HY);
  ok = ok && map3(&sm_->m[3], p.lam, nx, ny, nz, G::TZ, TY);
  ok = ok && map3(&sm_->m[4], p.mu, nx, ny, nz, G::WM, TY + 1);
  for (int c = 0; c < 6; ++c) ok = ok && map3(&sm_->m[5 + c], p.f[3 + c], nx, ny, nz, G::TZ, TY);
  return ok;
}

template <int N, int TY, int D, int TZ>
static StagedConfig staged_cfg_t() {
  using G = SG<N, TY, D, staged_q(true), TZ>;
  return StagedConfig{N, TY, D, TZ, G::NT, G::V_BYTES, G::S_BYTES};
}

// tile shapes per order: (TY, D); TZ is 32 or 40
#ifndef SW_TY240
#define SW_TY240 16
#endif
#ifndef SW_D240
#define SW_D240 1
#endif
#define SW_STAGED_SWITCH(N_, TZ_, CALL)                         \
  switch ((N_) * 100 + (TZ_)) {                                 \
    case 132: CALL(1, 16, 2, 32) case 140: CALL(1, 16, 2, 40)   \
    case 232: CALL(2, 16, 1, 32) case 240: CALL(2, SW_TY240, SW_D240, 40)   \
    case 332: CALL(3, 16, 2, 32) case 340: CALL(3, 16, 2, 40)   \
    case 432: CALL(4, 16, 1, 32) case 440: CALL(4, 16, 1, 40)   \
    default: break;                                             \
  }

bool sw3_staged_config(int N, int tz, StagedConfig* out) {
#define SW_CFG(a, b, c, d)           \
  {                                  \
    *out = staged_cfg_t<a, b, c, d>(); \
    return true;                     \
  }
  SW_STAGED_SWITCH(N, tz, SW_CFG)
#undef SW_CFG
  return false;
}

bool sw3_staged_maps(int N, int tz, const P3<float>& p, StagedMaps* vm, StagedMaps* sm_) {
#define SW_MAPS(a, b, c, d) \
  { return staged_maps_t<a, b, c, d>(p, vm, sm_); }
  SW_STAGED_SWITCH(N, tz, SW_MAPS)
#undef SW_MAPS
  return false;
}

// Resident CTAs per SM of each pass (registers, shared memory and threads
// together), queried once per device; each pass is launched with that many
// CTAs per SM (at most one per work unit), so the persistent unit loop runs
// in one wave.
struct StagedOcc {
  int vel = 0, str = 0, sms = 0;
};

template <int N, int TY, int D, int TZ, bool EX, int SCH>
static cudaError_t staged_setup(bool tensor, StagedOcc* occ) {
  constexpr int Q = staged_q(EX);
  using G = SG<N, TY, D, Q, TZ>;
  static std::atomic<unsigned long long> done{0};
  static std::mutex mu;
  static StagedOcc per_dev[64][2];
  int dev = 0;
  cudaError_t e0 = cudaGetDevice(&dev);
  if (e0 != cudaSuccess) return e0;
  e0 = once_per_device(done, mu, [dev] {
    cudaError_t e = cudaFuncSetAttribute(k3s_velocity<N, TY, D, false, EX, Q, TZ, SCH>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::V_BYTES);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k3s_stress<N, TY, D, EX, Q, TZ, SCH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)G::S_BYTES);
    StagedOcc& o0 = per_dev[dev & 63][0];
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o0.vel, k3s_velocity<N, TY, D, false, EX, Q, TZ, SCH>,
                                                        G::NT, G::V_BYTES);
    if constexpr (SCH == SCH_CPML) {
      StagedOcc& o1 = per_dev[dev & 63][1];
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k3s_velocity<N, TY, D, true, EX, Q, TZ, SCH>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::V_BYTES);
      if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o1.vel, k3s_velocity<N, TY, D, true, EX, Q, TZ, SCH>,
                                                          G::NT, G::V_BYTES);
    }
    int str = 0, sms = 0;
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&str, k3s_stress<N, TY, D, EX, Q, TZ, SCH>, G::NT,
                                                        G::S_BYTES);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    for (int t = 0; t < 2; ++t) {
      StagedOcc& o = per_dev[dev & 63][t];
      if (t == 1 && SCH != SCH_CPML) o.vel = per_dev[dev & 63][0].vel;
      o.str = str;
      o.sms = sms;
      if (o.vel < 1) o.vel = 1;
      if (o.str < 1) o.str = 1;
    }
    return e;
  });
  if (e0 != cudaSuccess) return e0;
  *occ = per_dev[dev & 63][tensor ? 1 : 0];
  return cudaSuccess;
}

template <int N, int TY, int D, int TZ, bool EX, int SCH>
static cudaError_t staged_launch(bool tensor, const P3<float>& p, const StagedMaps& vm, const StagedMaps& smp,
                                 const StagedArgs& a, int it, bool force_here, bool inject_next, bool gather,
                                 cudaStream_t st) {
  constexpr int Q = staged_q(EX);
  using G = SG<N, TY, D, Q, TZ>;
  StagedOcc o;
  cudaError_t e0 = staged_setup<N, TY, D, TZ, EX, SCH>(tensor, &o);
  if (e0 != cudaSuccess) return e0;
  const int units = a.tiles_y * a.tiles_z * a.chunks;
  const int gv = units < o.sms * o.vel ? units : o.sms * o.vel;
  const int gs = units < o.sms * o.str ? units : o.sms * o.str;
  if constexpr (SCH == SCH_CPML) {
    if (tensor) k3s_velocity<N, TY, D, true, EX, Q, TZ, SCH><<<gv, G::NT, G::V_BYTES, st>>>(p, vm, a, it, 0);
    else
      k3s_velocity<N, TY, D, false, EX, Q, TZ, SCH><<<gv, G::NT, G::V_BYTES, st>>>(p, vm, a, it, force_here ? 1 : 0);
  } else {
    k3s_velocity<N, TY, D, false, EX, Q, TZ, SCH><<<gv, G::NT, G::V_BYTES, st>>>(p, vm, a, it, force_here ? 1 : 0);
  }
  k3s_stress<N, TY, D, EX, Q, TZ, SCH><<<gs, G::NT, G::S_BYTES, st>>>(p, smp, a, it, inject_next ? 1 : 0,
                                                                       gather ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t sw3_staged_step(int N, int tz, bool spml, bool tensor, const P3<float>& p, const StagedMaps& vm,
                            const StagedMaps& smp, const StagedArgs& a, int it, bool force_here, bool inject_next,
                            bool gather, cudaStream_t st) {
  // the split-field PML runs exact numerics only
#define SW_STEP(a_, b, c, d)                                                                                     \
  {                                                                                                              \
    if (spml)                                                                                                    \
      return staged_launch<a_, b, c, d, true, SCH_SPML>(false, p, vm, smp, a, it, force_here, false, gather, st); \
    return a.exact ? staged_launch<a_, b, c, d, true, SCH_CPML>(tensor, p, vm, smp, a, it, force_here,            \
                                                                inject_next, gather, st)                         \
                   : staged_launch<a_, b, c, d, false, SCH_CPML>(tensor, p, vm, smp, a, it, force_here,           \
                                                                 inject_next, gather, st);                       \
  }
  SW_STAGED_SWITCH(N, tz, SW_STEP)
#undef SW_STEP
  return cudaErrorInvalidValue;
}

template <int N, int TY, int D, int TZ, bool EX, int SCH>
static cudaError_t staged_grid_t(bool tensor, int units, int* vel, int* str) {
  StagedOcc o;
  cudaError_t e = staged_setup<N, TY, D, TZ, EX, SCH>(tensor, &o);
  if (e != cudaSuccess) return e;
  *vel = units < o.sms * o.vel ? units : o.sms * o.vel;
  *str = units < o.sms * o.str ? units : o.sms * o.str;
  return cudaSuccess;
}

cudaError_t sw3_staged_grid(int N, int tz, bool spml, bool tensor, bool exact, int units, int* vel, int* str) {
#define SW_GRID(a_, b, c, d)                                                                \
  {                                                                                         \
    if (spml) return staged_grid_t<a_, b, c, d, true, SCH_SPML>(false, units, vel, str);    \
    return exact ? staged_grid_t<a_, b, c, d, true, SCH_CPML>(tensor, units, vel, str)      \
                 : staged_grid_t<a_, b, c, d, false, SCH_CPML>(tensor, units, vel, str);    \
  }
  SW_STAGED_SWITCH(N, tz, SW_GRID)
#undef SW_GRID
  return cudaErrorInvalidValue;
}

}  // namespace sw
