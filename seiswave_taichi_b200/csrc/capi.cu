// capi.cu -- the extern "C" boundary of libseiswave.so (include/seiswave.h).
//
// A plan validates a descriptor once (shapes, orders, slab extents, source and
// receiver cells) and freezes the kernel parameter blocks; sw_step / sw_run
// then only enqueue kernels.  sw_run replays a cached CUDA graph of the whole
// step sequence so the per-step launch cost of the reference's Python loop
// (test2d_homegenous.py:55-56) disappears.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "sw_device.cuh"
#include <type_traits>

#include "sw_fused.cuh"
#include "sw_staged.cuh"

namespace sw {
template <typename T> cudaError_t sw3_velocity(const P3<T>&, int, int, bool, bool, cudaStream_t);
template <typename T> cudaError_t sw3_stress(const P3<T>&, int, int, bool, cudaStream_t);
template <typename T> cudaError_t sw3_moment_inject(const P3<T>&, int, cudaStream_t);
template <typename T> cudaError_t sw3_force_inject(const P3<T>&, int, cudaStream_t);
template <typename T> cudaError_t sw3_aea(const P3<T>&, int, cudaStream_t);
template <typename T> cudaError_t sw3_gather(const P3<T>&, int, cudaStream_t);
template <typename T> cudaError_t sw3_spml_step(const P3<T>&, int, int, bool, cudaStream_t);
template <typename T> cudaError_t sw2_step(const P2<T>&, int, int, int, T, bool, bool, bool, int, cudaStream_t);
template <typename T> cudaError_t sw2_moment_inject(const P2<T>&, int, cudaStream_t);
cudaError_t segy_decode(const void*, long long, int, int, float*, int32_t*, cudaStream_t);
template <typename T>
cudaError_t sw2_persistent(const P2<T>&, int, int, int, int, bool, bool, unsigned int*, int*, cudaStream_t);
template <typename T>
cudaError_t sw2b_step(const Batch2<T>&, int, int, int, int, int, bool, bool, cudaStream_t);
void sw2b_tile_shape(int cfg, int* bx, int* bz);
template <typename T>
struct A2 {
  T* f[5];
  T* mem[2];
  T* tmp[4];
  T* grad[5];
  const T* res;
  const T* snap0;
  const T* snap1;
};
template <typename T> cudaError_t sw2_adjoint_step(const P2<T>&, const A2<T>&, int, int, int, cudaStream_t);
template <typename T>
struct A3 {
  T* f[9];
  T* mem[3];
  T* tmp[9];
  T* grad[8];
  const T* res;
  const T* snap0;
  const T* snap1;
};
template <typename T> cudaError_t sw3_adjoint_step(const P3<T>&, const A3<T>&, int, int, cudaStream_t);
struct AbcArgs {
  const int* cell;
  const int8_t* face;
  const int8_t* depth;
  int ncell;
  int nx, nz;
  const float* f[5];
  float* fw[5];
  float scale[5];
  float oscale[5];
  const float* params;
  float* delta;
  float* x_out;
};
cudaError_t abc_correct(const AbcArgs&, cudaStream_t);
cudaError_t abc_features(const AbcArgs&, cudaStream_t);
cudaError_t mlp_grad(const float*, const float*, const float*, long long, float*, float*, int, cudaStream_t);
cudaError_t abc_adjoint(const AbcArgs&, float* const*, float*, cudaStream_t);
struct AbcArgs3 {
  const int* cell;
  const int8_t* face;
  const int8_t* depth;
  int ncell;
  int nx, ny, nz;
  const float* f[9];
  float* fw[9];
  float scale[9];
  float oscale[9];
  const float* params;
  float* delta;
  float* x_out;
};
cudaError_t abc3_correct(const AbcArgs3&, cudaStream_t);
cudaError_t abc3_features(const AbcArgs3&, cudaStream_t);
cudaError_t abc3_adjoint(const AbcArgs3&, float* const*, float*, cudaStream_t);
cudaError_t mlp3_grad(const float*, const float*, const float*, long long, float*, float*, int, cudaStream_t);
cudaError_t mlp3_forward_batch(const float*, const float*, long long, float*, cudaStream_t);
cudaError_t mlp_forward_batch(const float*, const float*, long long, float*, cudaStream_t);
}  // namespace sw

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char* where) {
  return fail(SW_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

// count of non-finite values over a set of arrays
template <typename T>
__global__ void k_count_nonfinite(const T* a, long long n, unsigned long long* out) {
  unsigned long long local = 0;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    if (!isfinite(a[q])) ++local;
  if (local) atomicAdd(out, local);
}

}  // namespace

struct sw_plan {
  int dim = 0, scheme = 0, dtype = 0, order = 0, nt_max = 0;
  sw::P2<float> p2f{};
  sw::P2<double> p2d{};
  sw::P3<float> p3f{};
  sw::P3<double> p3d{};
  bool gather_in_stress = true;  // receivers record a velocity field
  bool src_in_kernel = true;     // the source cell is covered by the fused passes
  int src_kind = SW_SRC_NONE;
  long long ncell = 0;
  int nfield = 0;
  void* fields[9] = {};
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t gexec = nullptr;
  int g_it0 = -1, g_n = -1;
  unsigned long long* d_count = nullptr;
  // fused single-pass path (3D float CPML schemes)
  bool fused = false;
  int fused_N = 0, fused_grid = 0;
  sw::FusedMaps fmaps{};
  sw::FusedExtra fx{};
  void* fused_buf = nullptr;
  int* d_err = nullptr;
  // TMA-staged two-pass path (3D float CPML schemes)
  bool staged = false;
  sw::StagedMaps svm{}, ssm{};
  sw::StagedArgs sa{};
  int staged_N = 0, staged_tz = 32;
  // 0: register-queue two-pass kernels (2D: two launches per step), 1: staged
  // two-pass, 2: fused single pass, 3: 2D persistent (one cooperative launch
  // per run)
  int path = 0;
  unsigned int* d_bar = nullptr;  // 2D persistent path: grid-barrier arrival and generation words
  bool aea = false;               // free-surface hook before every step (sw_plan_set_free_surface)
};

namespace {

int dsize(int dtype) { return dtype == SW_F64 ? 8 : 4; }

bool aligned(const void* p, int n) { return ((uintptr_t)p % (uintptr_t)n) == 0; }

int check_axis(const sw_pml_axis& a, int n, const char* name, bool need_damp, int esz) {
  char buf[256];
  if (a.lo < 0 || a.hi < 0 || a.lo + a.hi > n) {
    snprintf(buf, sizeof buf, "pml axis %s: slab widths lo=%d hi=%d do not fit n=%d", name, a.lo, a.hi, n);
    return fail(SW_ERR_ARG, buf);
  }
  if (!a.coef || !aligned(a.coef, esz)) {
    snprintf(buf, sizeof buf, "pml axis %s: coefficient table missing or misaligned", name);
    return fail(SW_ERR_ARG, buf);
  }
  if (!a.flag) {
    snprintf(buf, sizeof buf, "pml axis %s: predicate flags missing", name);
    return fail(SW_ERR_ARG, buf);
  }
  if (need_damp && (!a.damp || !aligned(a.damp, esz))) {
    snprintf(buf, sizeof buf, "pml axis %s: split-PML damping profile missing", name);
    return fail(SW_ERR_ARG, buf);
  }
  return SW_OK;
}

// split PML: the split fields exist only on the shell of the axes' slabs, so
// every index whose predicate flag is set must lie in [0, lo) or [n-hi, n)
int check_shell(const sw_pml_axis& a, int n, const char* name) {
  std::vector<uint8_t> h(n);
  cudaError_t e = cudaMemcpy(h.data(), a.flag, n, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "split PML: reading the predicate flags");
  for (int i = a.lo; i < n - a.hi; ++i)
    if (h[i]) {
      char buf[200];
      snprintf(buf, sizeof buf, "pml axis %s: index %d is inside the split-PML predicate but outside the "
               "slabs lo=%d hi=%d that hold the split fields", name, i, a.lo, a.hi);
      return fail(SW_ERR_ARG, buf);
    }
  return SW_OK;
}

int check_receivers(const sw_receivers& r, int nfield, long long ncell, int nt_max) {
  if (r.nrec < 0) return fail(SW_ERR_ARG, "receivers: nrec < 0");
  if (r.nrec == 0) return SW_OK;
  if (!r.index || !r.data) return fail(SW_ERR_ARG, "receivers: index or data pointer missing");
  if (r.field < 0 || r.field >= nfield) return fail(SW_ERR_ARG, "receivers: field index out of range");
  if (r.dtype != SW_F32 && r.dtype != SW_F64) return fail(SW_ERR_ARG, "receivers: dtype must be SW_F32 or SW_F64");
  if (nt_max <= 0) return fail(SW_ERR_ARG, "receivers: nt_max must be positive");
  std::vector<long long> h(r.nrec);
  cudaError_t e = cudaMemcpy(h.data(), r.index, sizeof(long long) * r.nrec, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "receivers: reading the index table");
  for (int q = 0; q < r.nrec; ++q)
    if (h[q] < 0 || h[q] >= ncell) {
      char buf[160];
      snprintf(buf, sizeof buf, "receivers: index %d = %lld outside the grid of %lld cells", q, h[q], ncell);
      return fail(SW_ERR_ARG, buf);
    }
  return SW_OK;
}

template <typename T>
void fill_axis3(sw::P3<T>& p, int d, const sw_pml_axis& a, int n) {
  p.cf[d] = (const T*)a.coef;
  p.dmp[d] = (const T*)a.damp;
  p.fl[d] = a.flag;
  p.lo[d] = a.lo;
  p.hi[d] = a.hi;
  p.sn[d] = a.lo + a.hi;
  (void)n;
}

int choose_x_chunk(int nx, int ny, int nz) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long tiles = (long long)((nz + 31) / 32) * ((ny + 7) / 8);
  const long long target = (long long)sms * 8;  // ~8 resident-sized CTAs per SM
  long long chunks = (target + tiles - 1) / tiles;
  if (chunks < 1) chunks = 1;
  int xc = (int)((nx + chunks - 1) / chunks);
  if (xc < 4) xc = 4;
  return xc;
}

// ---------------------------------------------------------------------------
// constant divisors: enable div_c's Markstein path only where it equals IEEE
// division for every finite float numerator (checked once per divisor value)
// ---------------------------------------------------------------------------
bool verified_divisor(float d, float r, cudaStream_t st) {
  static std::vector<std::pair<uint32_t, bool>> cache;
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  uint32_t bits;
  memcpy(&bits, &d, 4);
  for (auto& e : cache)
    if (e.first == bits) return e.second;
  unsigned long long* dbad = nullptr;
  unsigned long long hbad = 1;
  bool ok = false;
  if (cudaMalloc(&dbad, sizeof(unsigned long long)) == cudaSuccess) {
    // the per-lane route and the staged kernels' branch-free group route
    ok = sw::sw3_check_divisor(d, r, dbad, &hbad, st, 0) == cudaSuccess && hbad == 0 &&
         sw::sw3_check_divisor(d, r, dbad, &hbad, st, 2) == cudaSuccess && hbad == 0;
    cudaFree(dbad);
  }
  cudaGetLastError();
  cache.push_back({bits, ok});
  return ok;
}

template <typename T>
void set_divisors(T* rd, int* fast, const double* h, int n) {
  int f = 1;
  for (int a = 0; a < n; ++a) {
    rd[a] = (T)1 / (T)h[a];
    if (sizeof(T) == 4) f = f && verified_divisor((float)(T)h[a], (float)rd[a], 0);
    else f = 0;
  }
  *fast = f;
}

template <typename T>
int make_p3(sw_plan* pl, const sw3d_desc* d, sw::P3<T>& p) {
  p.nx = d->nx; p.ny = d->ny; p.nz = d->nz;
  p.dx = (T)d->dx; p.dy = (T)d->dy; p.dz = (T)d->dz; p.dt = (T)d->dt;
  for (int m = 0; m < SW_MAX_ORDER; ++m) p.c[m] = (T)d->coef[m];
  for (int q = 0; q < 9; ++q) p.f[q] = (T*)d->field[q];
  p.rho = (const T*)d->rho; p.lam = (const T*)d->lam; p.mu = (const T*)d->mu;
  const int ns[3] = {d->nx, d->ny, d->nz};
  for (int a = 0; a < 3; ++a) fill_axis3(p, a, d->pml[a], ns[a]);
  for (int a = 0; a < 3; ++a) p.mem[a] = (T*)d->mem[a];
  p.mcomp[0] = (long long)p.sn[0] * d->ny * d->nz;
  p.mcomp[1] = (long long)d->nx * p.sn[1] * d->nz;
  p.mcomp[2] = (long long)d->nx * d->ny * p.sn[2];
  p.split = (T*)d->split;
  p.scomp = (long long)p.sn[0] * d->ny * d->nz + (long long)(d->nx - p.sn[0]) * p.sn[1] * d->nz +
            (long long)(d->nx - p.sn[0]) * (d->ny - p.sn[1]) * p.sn[2];
  p.src_kind = d->src.kind; p.si = d->src.i; p.sj = d->src.j; p.sk = d->src.k;
  p.wav = (const T*)d->src.wavelet;
  for (int q = 0; q < 6; ++q) p.mneg[q] = -(T)(float)d->src.mt[q];
  p.nrec = d->rec.nrec; p.rec_field = d->rec.field;
  p.rec_idx = (const long long*)d->rec.index; p.rec_data = d->rec.data;
  p.rec_f64 = d->rec.dtype == SW_F64;
  p.x_chunk = choose_x_chunk(d->nx, d->ny, d->nz);
  const double hs[3] = {d->dx, d->dy, d->dz};
  set_divisors<T>(p.rd, &p.fast_div, hs, 3);
  for (int a = 0; a < 3; ++a)
    for (int m = 0; m < SW_MAX_ORDER; ++m) p.cs[a][m] = (T)(d->coef[m] / hs[a]);
  (void)pl;
  return SW_OK;
}

template <typename T>
int make_p2(const sw2d_desc* d, sw::P2<T>& p) {
  p.nx = d->nx; p.nz = d->nz;
  p.dx = (T)d->dx; p.dz = (T)d->dz; p.dt = (T)d->dt;
  for (int m = 0; m < SW_MAX_ORDER; ++m) p.c[m] = (T)d->coef[m];
  for (int q = 0; q < 5; ++q) p.f[q] = (T*)d->field[q];
  p.rho = (const T*)d->rho; p.lam = (const T*)d->lam; p.mu = (const T*)d->mu;
  for (int a = 0; a < 2; ++a) {
    p.cf[a] = (const T*)d->pml[a].coef;
    p.fl[a] = d->pml[a].flag;
    p.lo[a] = d->pml[a].lo;
    p.hi[a] = d->pml[a].hi;
    p.sn[a] = d->pml[a].lo + d->pml[a].hi;
    p.mem[a] = (T*)d->mem[a];
  }
  p.mcomp[0] = (long long)p.sn[0] * d->nz;
  p.mcomp[1] = (long long)d->nx * p.sn[1];
  p.src_kind = d->src.kind; p.si = d->src.i; p.sk = d->src.j;
  p.wav = (const T*)d->src.wavelet;
  // 2D moment tensor: xx zz xz in mt[0], mt[2], mt[4], rounded through float
  // like the 3D tensor source
  p.mneg[0] = -(T)(float)d->src.mt[0];
  p.mneg[1] = -(T)(float)d->src.mt[2];
  p.mneg[2] = -(T)(float)d->src.mt[4];
  p.nrec = d->rec.nrec; p.rec_field = d->rec.field;
  p.rec_idx = (const long long*)d->rec.index; p.rec_data = d->rec.data;
  p.rec_f64 = d->rec.dtype == SW_F64;
  const double h1[2] = {d->dx, d->dz}, h2[2] = {2 * d->dx, 2 * d->dz};
  int f1 = 0, f2 = 0;
  set_divisors<T>(p.rd, &f1, h1, 2);
  if (d->scheme == SW2D_RSG) {
    for (int a = 0; a < 2; ++a) p.rd2[a] = (T)1 / ((T)2 * (T)h1[a]);
    const double hh[2] = {(double)((T)2 * (T)h1[0]), (double)((T)2 * (T)h1[1])};
    T tmp[2];
    set_divisors<T>(tmp, &f2, hh, 2);
  }
  p.fast_div = f1 | (f2 << 1);
  return SW_OK;
}

// ---------------------------------------------------------------------------
// one step, enqueued
// ---------------------------------------------------------------------------
template <typename T>
cudaError_t enqueue3(sw_plan* pl, const sw::P3<T>& p, int it, bool first, bool last, cudaStream_t st) {
  cudaError_t e = cudaSuccess;
  sw::P3<T> q = p;
  if (!pl->gather_in_stress) q.nrec = 0;
  // free surface: szz = 0 on the layer k = N before the step, as a driver
  // loop `AEA(); update_SSG(i)` does
  if (pl->aea) {
    e = sw::sw3_aea<T>(p, pl->order, st);
    if (e != cudaSuccess) return e;
  }
  if (pl->scheme == SW3D_SPML) {
    if constexpr (std::is_same<T, float>::value) {
      if (pl->path >= 1 && pl->staged) {
        e = sw::sw3_staged_step(pl->staged_N, pl->staged_tz, true, false, p, pl->svm, pl->ssm, pl->sa, it,
                                pl->src_kind == SW_SRC_FORCE, false, pl->gather_in_stress, st);
        if (e == cudaSuccess && !pl->gather_in_stress) e = sw::sw3_gather<T>(p, it, st);
        return e;
      }
    }
    e = sw::sw3_spml_step<T>(q, pl->order, it, pl->gather_in_stress, st);
    if (e == cudaSuccess && !pl->gather_in_stress) e = sw::sw3_gather<T>(p, it, st);
    return e;
  }
  const bool tensor = pl->scheme == SW3D_CPML_TENSOR;
  const bool moment = pl->src_kind == SW_SRC_MOMENT;
  // a moment source on the free-surface layer must follow that layer's
  // zeroing, so it is not folded into the previous stress pass
  const bool unfold = pl->aea && p.sk == pl->order;
  // moment tensor: the stress pass of step it-1 already added step it's
  // source unless this is the first step of the sequence
  if (moment && (first || !pl->src_in_kernel || unfold)) {
    e = sw::sw3_moment_inject<T>(p, it, st);
    if (e != cudaSuccess) return e;
  }
  const bool force = pl->src_kind == SW_SRC_FORCE;
  if constexpr (std::is_same<T, float>::value) {
    if (pl->path >= 1 && pl->staged) {
      const bool inject_next = moment && !last && !unfold;
      e = sw::sw3_staged_step(pl->staged_N, pl->staged_tz, false, tensor, p, pl->svm, pl->ssm, pl->sa, it, force,
                              inject_next, pl->gather_in_stress, st);
      if (e != cudaSuccess) return e;
      if (!pl->gather_in_stress) e = sw::sw3_gather<T>(p, it, st);
      return e;
    }
  }
  e = sw::sw3_velocity<T>(q, pl->order, it, tensor, force && pl->src_in_kernel, st);
  if (e != cudaSuccess) return e;
  if (force && !pl->src_in_kernel) {
    e = sw::sw3_force_inject<T>(p, it, st);
    if (e != cudaSuccess) return e;
  }
  const bool inject_next = moment && pl->src_in_kernel && !last && !unfold;
  e = sw::sw3_stress<T>(q, pl->order, it, inject_next, st);
  if (e != cudaSuccess) return e;
  if (!pl->gather_in_stress) e = sw::sw3_gather<T>(p, it, st);
  return e;
}

cudaError_t enqueue_step(sw_plan* pl, int it, bool first, bool last, bool has_amp, double amp, cudaStream_t st) {
  if (pl->dim == 3) {
    return pl->dtype == SW_F32 ? enqueue3<float>(pl, pl->p3f, it, first, last, st)
                               : enqueue3<double>(pl, pl->p3d, it, first, last, st);
  }
  // moment tensor: the stress pass of step it-1 adds step it's source, unless
  // this is the first step of the sequence or a receiver records a stress
  const bool moment = pl->src_kind == SW_SRC_MOMENT;
  const bool fold = moment && pl->gather_in_stress;
  const bool pre = moment && (first || !fold), nxt = fold && !last;
  // free surface: the hook of the first step runs on its own, those of the
  // later steps are folded into the previous stress pass
  const int aea = pl->aea ? ((first ? 1 : 0) | (last ? 0 : 2)) : 0;
  if (pl->dtype == SW_F32) {
    float a = has_amp ? (float)amp : 0.f;
    return sw::sw2_step<float>(pl->p2f, pl->scheme, pl->order, it, a, pl->gather_in_stress, pre, nxt, aea, st);
  }
  double a = has_amp ? (double)(float)amp : 0.0;
  return sw::sw2_step<double>(pl->p2d, pl->scheme, pl->order, it, a, pl->gather_in_stress, pre, nxt, aea, st);
}

int check_it(sw_plan* pl, int it0, int n) {
  if (!pl) return fail(SW_ERR_ARG, "null plan");
  if (n < 0 || it0 < 0) return fail(SW_ERR_ARG, "negative step index or count");
  const bool needs_wavelet = pl->src_kind == SW_SRC_FORCE || pl->src_kind == SW_SRC_MOMENT;
  const bool records = pl->dim == 3 ? pl->p3f.nrec + pl->p3d.nrec > 0 : pl->p2f.nrec + pl->p2d.nrec > 0;
  if ((needs_wavelet || records) && (long long)it0 + n > pl->nt_max) {
    char buf[160];
    snprintf(buf, sizeof buf, "steps %d..%d exceed nt_max=%d of the wavelet/receiver arrays", it0,
             it0 + n - 1, pl->nt_max);
    return fail(SW_ERR_ARG, buf);
  }
  return SW_OK;
}


// ---------------------------------------------------------------------------
// fused single-pass path: second buffer set, tensor maps, divisor check
// ---------------------------------------------------------------------------
int choose_fused_grid(sw_plan* pl, const sw::FusedConfig& fc) {
  const auto& p = pl->p3f;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  auto& x = pl->fx;
  x.tiles_y = (p.ny + fc.TY - 1) / fc.TY;
  x.tiles_z = (p.nz + fc.tz - 1) / fc.tz;
  const int tiles = x.tiles_y * x.tiles_z;
  int chunks = (5 * sms + tiles - 1) / tiles;
  if (chunks < 1) chunks = 1;
  int len = (p.nx + chunks - 1) / chunks;
  if (len < 4 * fc.N) len = 4 * fc.N;
  x.chunk_len = len;
  x.chunks = (p.nx + len - 1) / len;
  const int units = tiles * x.chunks;
  return units < sms ? units : sms;
}

void setup_fused(sw_plan* pl) {
  pl->fused = false;
  if (pl->dim != 3 || pl->dtype != SW_F32) return;
  if (pl->scheme != SW3D_CPML_TENSOR && pl->scheme != SW3D_CPML_FORCE) return;
  if (!pl->src_in_kernel) return;
  sw::FusedConfig fc;
  if (!sw::sw3_fused_config(pl->order, &fc)) return;
  auto& p = pl->p3f;
  const int N = pl->order;
  if (p.nz % 4 != 0) return;
  if (pl->src_kind == SW_SRC_MOMENT && p.si >= p.nx - N) return;
  for (int q = 0; q < 9; ++q)
    if (!aligned(p.f[q], 16)) return;
  if (!aligned(p.rho, 16) || !aligned(p.lam, 16) || !aligned(p.mu, 16)) return;
  int dev = 0, maxsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if ((size_t)maxsm < fc.smem) return;
  // second buffer set: nine wavefields + three velocity memory-variable comps per direction
  const size_t ncell = (size_t)p.nx * p.ny * p.nz;
  size_t total = 9 * ncell;
  size_t mv[3];
  for (int d = 0; d < 3; ++d) {
    mv[d] = 3 * (size_t)p.mcomp[d];
    total += (mv[d] + 63) / 64 * 64;
  }
  float* buf = nullptr;
  if (cudaMalloc(&buf, total * sizeof(float)) != cudaSuccess) { cudaGetLastError(); return; }
  if (!pl->d_err) {
    if (cudaMalloc(&pl->d_err, sizeof(int)) != cudaSuccess) { cudaFree(buf); cudaGetLastError(); return; }
    cudaMemset(pl->d_err, 0, sizeof(int));
  }
  cudaMemset(buf, 0, total * sizeof(float));
  auto& x = pl->fx;
  float* cur = buf;
  for (int q = 0; q < 9; ++q) { x.fB[q] = cur; cur += ncell; }
  for (int d = 0; d < 3; ++d) {
    x.memB[d] = mv[d] ? cur : nullptr;
    cur += (mv[d] + 63) / 64 * 64;
  }
  x.err = pl->d_err;
  if (!sw::sw3_fused_maps(N, p, x, &pl->fmaps)) {
    cudaFree(buf);
    return;
  }
  pl->fused_grid = choose_fused_grid(pl, fc);
  pl->fused_buf = buf;
  pl->fused_N = N;
  pl->fused = true;
}

int units_grid(int units, int per_sm) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int cap = sms * per_sm;
  return units < cap ? units : cap;
}

void staged_chunks(sw_plan* pl, int len) {
  const auto& p = pl->p3f;
  sw::StagedConfig sc;
  sw::sw3_staged_config(pl->staged_N, pl->staged_tz, &sc);
  auto& a = pl->sa;
  a.tiles_y = (p.ny + sc.TY - 1) / sc.TY;
  a.tiles_z = (p.nz + sc.TZ - 1) / sc.TZ;
  if (len <= 0) {
    // about five work units per resident CTA
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int tiles = a.tiles_y * a.tiles_z;
    int chunks = (10 * sms + tiles - 1) / tiles;
    len = (p.nx + chunks - 1) / chunks;
  }
  if (len < 2 * pl->staged_N + 2) len = 2 * pl->staged_N + 2;
  a.chunk_len = len;
  a.chunks = (p.nx + len - 1) / len;
}

void setup_staged(sw_plan* pl) {
  pl->staged = false;
  if (pl->dim != 3 || pl->dtype != SW_F32) return;
  if (pl->scheme != SW3D_CPML_TENSOR && pl->scheme != SW3D_CPML_FORCE && pl->scheme != SW3D_SPML) return;
  if (!pl->src_in_kernel) return;
  auto& p = pl->p3f;
  // the staged passes stream planes [N, nx-N): a point force outside them
  // needs the per-cell split-PML kernels
  if (pl->scheme == SW3D_SPML && pl->src_kind != SW_SRC_NONE && (p.si < pl->order || p.si >= p.nx - pl->order))
    return;
  if (p.nz % 4 != 0) return;
  // z tile width: the one leaving fewer idle cells in the last tile (32 on ties)
  const int tz = (p.nz + 39) / 40 * 40 < (p.nz + 31) / 32 * 32 ? 40 : 32;
  sw::StagedConfig sc;
  if (!sw::sw3_staged_config(pl->order, tz, &sc)) return;
  for (int q = 0; q < 9; ++q)
    if (!aligned(p.f[q], 16)) return;
  if (!aligned(p.rho, 16) || !aligned(p.lam, 16) || !aligned(p.mu, 16)) return;
  int dev = 0, maxsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if ((size_t)maxsm < sc.vel_smem || (size_t)maxsm < sc.str_smem) return;
  if (!pl->d_err) {
    if (cudaMalloc(&pl->d_err, sizeof(int)) != cudaSuccess) { cudaGetLastError(); return; }
    cudaMemset(pl->d_err, 0, sizeof(int));
  }
  if (!sw::sw3_staged_maps(pl->order, tz, p, &pl->svm, &pl->ssm)) return;
  pl->staged_N = pl->order;
  pl->staged_tz = tz;
  pl->sa.err = pl->d_err;
  pl->sa.exact = 1;
  staged_chunks(pl, 0);
  pl->staged = true;
  pl->path = 1;
}

// nsteps >= 2 steps through the fused kernel (the last one two-pass when odd)
cudaError_t enqueue_fused_run(sw_plan* pl, int it0, int nsteps, cudaStream_t st) {
  const auto& p = pl->p3f;
  const bool moment = pl->src_kind == SW_SRC_MOMENT;
  const bool tensor = pl->scheme == SW3D_CPML_TENSOR;
  cudaError_t e;
  if (moment) {
    e = sw::sw3_moment_inject<float>(p, it0, st);
    if (e != cudaSuccess) return e;
  }
  const int nf = nsteps & ~1;
  for (int s = 0; s < nf; ++s) {
    const int it = it0 + s;
    e = sw::sw3_fused_step(pl->fused_N, tensor, p, pl->fmaps, pl->fx, pl->fused_grid, it, s & 1,
                           moment && s < nsteps - 1, s > 0 ? it - 1 : -1, st);
    if (e != cudaSuccess) return e;
  }
  // the fused steps end in the caller's buffers; record the last one's receivers
  e = sw::sw3_gather<float>(p, it0 + nf - 1, st);
  if (e != cudaSuccess) return e;
  if (nsteps & 1) return enqueue3<float>(pl, p, it0 + nsteps - 1, false, true, st);
  return cudaSuccess;
}

// 2D persistent path: the barrier words and the error word on first use
cudaError_t persistent_run2(sw_plan* pl, int it0, int nsteps, cudaStream_t st) {
  if (!pl->d_bar) {
    cudaError_t e = cudaMalloc(&pl->d_bar, 2 * sizeof(unsigned int));
    if (e != cudaSuccess) return e;
    e = cudaMemset(pl->d_bar, 0, 2 * sizeof(unsigned int));
    if (e != cudaSuccess) return e;
  }
  if (!pl->d_err) {
    cudaError_t e = cudaMalloc(&pl->d_err, sizeof(int));
    if (e != cudaSuccess) return e;
    e = cudaMemset(pl->d_err, 0, sizeof(int));
    if (e != cudaSuccess) return e;
  }
  if (pl->dtype == SW_F32)
    return sw::sw2_persistent<float>(pl->p2f, pl->scheme, pl->order, it0, nsteps, pl->gather_in_stress,
                                     pl->gather_in_stress, pl->d_bar, pl->d_err, st);
  return sw::sw2_persistent<double>(pl->p2d, pl->scheme, pl->order, it0, nsteps, pl->gather_in_stress,
                                    pl->gather_in_stress, pl->d_bar, pl->d_err, st);
}

cudaError_t enqueue_sequence(sw_plan* pl, int it0, int nsteps, cudaStream_t st) {
  if (pl->fused && pl->path == 2 && nsteps >= 2 && !pl->aea) return enqueue_fused_run(pl, it0, nsteps, st);
  for (int s = 0; s < nsteps; ++s) {
    cudaError_t e = enqueue_step(pl, it0 + s, s == 0, s == nsteps - 1, false, 0.0, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace

extern "C" {

int sw_version(void) { return SW_ABI_VERSION; }

int sw_abi_sizeof(int32_t which) {
  switch (which) {
    case 0: return (int)sizeof(sw_pml_axis);
    case 1: return (int)sizeof(sw_receivers);
    case 2: return (int)sizeof(sw_source);
    case 3: return (int)sizeof(sw2d_desc);
    case 4: return (int)sizeof(sw3d_desc);
    default: return -1;
  }
}

const char* sw_last_error(void) { return g_err.c_str(); }

int sw2d_plan_create(const sw2d_desc* d, sw_plan** out) {
  g_err.clear();
  if (!d || !out) return fail(SW_ERR_ARG, "null descriptor or output pointer");
  *out = nullptr;
  if (d->scheme < SW2D_SSG_VS || d->scheme > SW2D_RSG) return fail(SW_ERR_ARG, "unknown 2D scheme");
  if (d->dtype != SW_F32 && d->dtype != SW_F64) return fail(SW_ERR_ARG, "dtype must be SW_F32 or SW_F64");
  if (d->order < 1 || d->order > SW_MAX_ORDER) return fail(SW_ERR_ARG, "order (accuracy) must be in 1..8");
  const int N = d->order;
  if (d->nx < 2 * N + 3 || d->nz < 2 * N + 3) return fail(SW_ERR_ARG, "grid too small for the stencil order");
  if (!(d->dx > 0) || !(d->dz > 0) || !(d->dt > 0)) return fail(SW_ERR_ARG, "dx, dz and dt must be positive");
  const int esz = dsize(d->dtype);
  for (int q = 0; q < 5; ++q)
    if (!d->field[q] || !aligned(d->field[q], esz)) return fail(SW_ERR_ARG, "wavefield pointer missing or misaligned");
  if (!d->rho || !d->lam || !d->mu) return fail(SW_ERR_ARG, "material pointer missing");
  int rc;
  if ((rc = check_axis(d->pml[0], d->nx, "x", false, esz)) != SW_OK) return rc;
  if ((rc = check_axis(d->pml[1], d->nz, "z", false, esz)) != SW_OK) return rc;
  if (d->pml[0].lo + d->pml[0].hi > 0 && !d->mem[0]) return fail(SW_ERR_ARG, "x memory variables missing");
  if (d->pml[1].lo + d->pml[1].hi > 0 && !d->mem[1]) return fail(SW_ERR_ARG, "z memory variables missing");
  const sw_source& s = d->src;
  if (s.kind != SW_SRC_NONE) {
    if (d->scheme == SW2D_RSG) {
      if (s.kind != SW_SRC_RSG4) return fail(SW_ERR_ARG, "RSG takes the SW_SRC_RSG4 source");
      if (s.i < 1 || s.i >= d->nx || s.j < 1 || s.j >= d->nz) return fail(SW_ERR_ARG, "RSG source block outside the grid");
    } else {
      if (s.kind != SW_SRC_FORCE && s.kind != SW_SRC_MOMENT)
        return fail(SW_ERR_ARG, "2D SSG schemes take a SW_SRC_FORCE or SW_SRC_MOMENT source");
      if (s.i < 0 || s.i >= d->nx || s.j < 0 || s.j >= d->nz) return fail(SW_ERR_ARG, "source cell outside the grid");
      if (!s.wavelet) return fail(SW_ERR_ARG, "source wavelet missing");
    }
  }
  const long long ncell = (long long)d->nx * d->nz;
  if ((rc = check_receivers(d->rec, 5, ncell, d->nt_max)) != SW_OK) return rc;
  sw_plan* pl = new sw_plan();
  pl->dim = 2; pl->scheme = d->scheme; pl->dtype = d->dtype; pl->order = N; pl->nt_max = d->nt_max;
  pl->src_kind = s.kind;
  pl->gather_in_stress = d->rec.nrec == 0 || d->rec.field <= 1;
  pl->ncell = ncell;
  pl->nfield = 5;
  for (int q = 0; q < 5; ++q) pl->fields[q] = d->field[q];
  if (d->dtype == SW_F32) make_p2<float>(d, pl->p2f);
  else make_p2<double>(d, pl->p2d);
  *out = pl;
  return SW_OK;
}

int sw3d_plan_create(const sw3d_desc* d, sw_plan** out) {
  g_err.clear();
  if (!d || !out) return fail(SW_ERR_ARG, "null descriptor or output pointer");
  *out = nullptr;
  if (d->scheme < SW3D_CPML_FORCE || d->scheme > SW3D_SPML) return fail(SW_ERR_ARG, "unknown 3D scheme");
  if (d->dtype != SW_F32 && d->dtype != SW_F64) return fail(SW_ERR_ARG, "dtype must be SW_F32 or SW_F64");
  if (d->order < 1 || d->order > SW_MAX_ORDER) return fail(SW_ERR_ARG, "order (accuracy) must be in 1..8");
  const int N = d->order;
  if (d->nx < 2 * N + 3 || d->ny < 2 * N + 3 || d->nz < 2 * N + 3)
    return fail(SW_ERR_ARG, "grid too small for the stencil order");
  if (!(d->dx > 0) || !(d->dy > 0) || !(d->dz > 0) || !(d->dt > 0))
    return fail(SW_ERR_ARG, "dx, dy, dz and dt must be positive");
  const int esz = dsize(d->dtype);
  for (int q = 0; q < 9; ++q)
    if (!d->field[q] || !aligned(d->field[q], esz)) return fail(SW_ERR_ARG, "wavefield pointer missing or misaligned");
  if (!d->rho || !d->lam || !d->mu) return fail(SW_ERR_ARG, "material pointer missing");
  const bool spml = d->scheme == SW3D_SPML;
  int rc;
  const char* names[3] = {"x", "y", "z"};
  const int ns[3] = {d->nx, d->ny, d->nz};
  for (int a = 0; a < 3; ++a) {
    if ((rc = check_axis(d->pml[a], ns[a], names[a], spml, esz)) != SW_OK) return rc;
    if (spml && (rc = check_shell(d->pml[a], ns[a], names[a])) != SW_OK) return rc;
    if (!spml && d->pml[a].lo + d->pml[a].hi > 0 && !d->mem[a])
      return fail(SW_ERR_ARG, std::string(names[a]) + " memory variables missing");
  }
  if (spml && !d->split) return fail(SW_ERR_ARG, "split-PML fields missing");
  const sw_source& s = d->src;
  bool in_kernel = true;
  if (s.kind != SW_SRC_NONE) {
    if (s.i < 0 || s.i >= d->nx || s.j < 0 || s.j >= d->ny || s.k < 0 || s.k >= d->nz)
      return fail(SW_ERR_ARG, "source cell outside the grid");
    if (!s.wavelet) return fail(SW_ERR_ARG, "source wavelet missing");
    if (d->scheme == SW3D_CPML_TENSOR && s.kind != SW_SRC_MOMENT)
      return fail(SW_ERR_ARG, "the tensor scheme takes a SW_SRC_MOMENT source");
    if (d->scheme != SW3D_CPML_TENSOR && s.kind != SW_SRC_FORCE)
      return fail(SW_ERR_ARG, "the point-force schemes take a SW_SRC_FORCE source");
    // the fused passes cover cells [N, n-N) on every axis
    in_kernel = s.i >= N && s.i < d->nx - N && s.j >= N && s.j < d->ny - N && s.k >= N && s.k < d->nz - N;
    if (spml) in_kernel = true;
  }
  const long long ncell = (long long)d->nx * d->ny * d->nz;
  if ((rc = check_receivers(d->rec, 9, ncell, d->nt_max)) != SW_OK) return rc;
  sw_plan* pl = new sw_plan();
  pl->dim = 3; pl->scheme = d->scheme; pl->dtype = d->dtype; pl->order = N; pl->nt_max = d->nt_max;
  pl->src_kind = s.kind;
  pl->src_in_kernel = in_kernel;
  pl->gather_in_stress = d->rec.nrec == 0 || d->rec.field <= 2;
  pl->ncell = ncell;
  pl->nfield = 9;
  for (int q = 0; q < 9; ++q) pl->fields[q] = d->field[q];
  if (d->dtype == SW_F32) make_p3<float>(pl, d, pl->p3f);
  else make_p3<double>(pl, d, pl->p3d);
  setup_staged(pl);
  *out = pl;
  return SW_OK;
}

int sw_plan_set_tile(sw_plan* pl, int32_t x_chunk) {
  if (!pl) return fail(SW_ERR_ARG, "null plan");
  if (pl->dim != 3) return fail(SW_ERR_UNSUPPORTED, "tile choice applies to 3D plans");
  if (x_chunk < 1) return fail(SW_ERR_ARG, "x_chunk must be >= 1");
  pl->p3f.x_chunk = x_chunk;
  pl->p3d.x_chunk = x_chunk;
  if (pl->gexec) { cudaGraphExecDestroy(pl->gexec); pl->gexec = nullptr; pl->g_it0 = pl->g_n = -1; }
  return SW_OK;
}

int sw_check_division(float divisor, int32_t mode, uint64_t* mismatches, void* stream) {
  if (!mismatches || mode < 0 || mode > 3) return fail(SW_ERR_ARG, "sw_check_division: mode 0..3 and an output");
  if (!(divisor > 0.f) || !std::isfinite(divisor)) return fail(SW_ERR_ARG, "sw_check_division: positive finite divisor");
  if (mode == 3 && !(divisor >= 0x1p-60f && divisor <= 0x1p60f))
    return fail(SW_ERR_ARG, "sw_check_division: mode 3 needs a divisor in [2^-60, 2^60]");
  unsigned long long* d_bad = nullptr;
  unsigned long long h_bad = 0;
  cudaError_t e = cudaMalloc(&d_bad, sizeof(unsigned long long));
  if (e != cudaSuccess) return cuda_fail(e, "sw_check_division");
  e = sw::sw3_check_divisor(divisor, 1.f / divisor, d_bad, &h_bad, (cudaStream_t)stream, mode);
  cudaFree(d_bad);
  if (e != cudaSuccess) return cuda_fail(e, "sw_check_division");
  *mismatches = h_bad;
  return SW_OK;
}

int sw_plan_status(sw_plan* pl, void* stream) {
  if (!pl) return fail(SW_ERR_ARG, "null plan");
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "sw_plan_status");
  if (pl->d_err) {
    int h = 0;
    e = cudaMemcpy(&h, pl->d_err, sizeof h, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "sw_plan_status");
    if (h != 0) {
      // reported once: clear the word so that a retry after a transient
      // timeout reads the status of the runs since this read
      e = cudaMemset(pl->d_err, 0, sizeof(int));
      if (e != cudaSuccess) return cuda_fail(e, "sw_plan_status");
    }
    if (h & 1) return fail(SW_ERR_TIMEOUT, "a bounded device wait gave up (TMA data never arrived)");
    if (h & 2) return fail(SW_ERR_TIMEOUT, "a bounded device wait gave up (grid barrier of the persistent run)");
  }
  return SW_OK;
}

int sw_plan_info(sw_plan* pl, int32_t* info) {
  if (!pl || !info) return fail(SW_ERR_ARG, "null plan or output");
  info[0] = pl->path;
  info[1] = pl->dim == 3 ? (pl->dtype == SW_F32 ? pl->p3f.fast_div : 0) : (pl->dtype == SW_F32 ? pl->p2f.fast_div : 0);
  info[2] = pl->staged ? 1 : 0;
  info[3] = 0;
  if (pl->staged) {
    // the velocity pass's grid (the occupancy of the numerics in use)
    int gv = 0, gs = 0;
    const bool spml = pl->scheme == SW3D_SPML, tensor = pl->scheme == SW3D_CPML_TENSOR;
    if (sw::sw3_staged_grid(pl->staged_N, pl->staged_tz, spml, tensor, pl->sa.exact != 0,
                            pl->sa.tiles_y * pl->sa.tiles_z * pl->sa.chunks, &gv, &gs) == cudaSuccess)
      info[3] = gv;
    cudaGetLastError();
  }
  info[4] = pl->staged ? pl->sa.chunk_len : 0;
  info[5] = pl->fused ? 1 : 0;
  info[6] = pl->fused ? pl->fused_grid : 0;
  info[7] = pl->fused ? pl->fx.chunk_len : 0;
  info[8] = pl->staged ? pl->sa.exact : 1;
  return SW_OK;
}

int sw_plan_set_path(sw_plan* pl, int32_t path, int32_t chunk_len) {
  if (!pl) return fail(SW_ERR_ARG, "null plan");
  if (path < 0 || path > 3) return fail(SW_ERR_ARG, "path must be 0, 1, 2 or 3");
  if (path == 3) {
    if (pl->dim != 2) return fail(SW_ERR_UNSUPPORTED, "the persistent path is for 2D plans");
    int dev = 0, coop = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    cudaGetLastError();
    if (!coop) return fail(SW_ERR_UNSUPPORTED, "this device has no cooperative launch");
  }
  if (path == 1 && !pl->staged) return fail(SW_ERR_UNSUPPORTED, "this plan has no staged path");
  if (path == 2 && !pl->fused) setup_fused(pl);  // allocates the second buffer set on first use
  if (path == 2 && !pl->fused) return fail(SW_ERR_UNSUPPORTED, "this plan has no fused path");
  pl->path = path;
  if (chunk_len > 0 && path == 1) staged_chunks(pl, chunk_len);
  if (chunk_len > 0 && path == 2) {
    sw::FusedConfig fc;
    sw::sw3_fused_config(pl->fused_N, &fc);
    int len = chunk_len < 2 * fc.N ? 2 * fc.N : chunk_len;
    pl->fx.chunk_len = len;
    pl->fx.chunks = (pl->p3f.nx + len - 1) / len;
    pl->fused_grid = units_grid(pl->fx.tiles_y * pl->fx.tiles_z * pl->fx.chunks, 1);
  }
  if (pl->gexec) { cudaGraphExecDestroy(pl->gexec); pl->gexec = nullptr; pl->g_it0 = pl->g_n = -1; }
  return SW_OK;
}

int sw_plan_set_free_surface(sw_plan* pl, int32_t on) {
  if (!pl) return fail(SW_ERR_ARG, "null plan");
  const bool v = on != 0;
  if (v != pl->aea && pl->gexec) { cudaGraphExecDestroy(pl->gexec); pl->gexec = nullptr; pl->g_it0 = pl->g_n = -1; }
  pl->aea = v;
  return SW_OK;
}

int sw_plan_set_exact(sw_plan* pl, int32_t exact) {
  if (!pl) return fail(SW_ERR_ARG, "null plan");
  pl->sa.exact = exact ? 1 : 0;
  if (pl->gexec) { cudaGraphExecDestroy(pl->gexec); pl->gexec = nullptr; pl->g_it0 = pl->g_n = -1; }
  return SW_OK;
}

int sw_plan_destroy(sw_plan* pl) {
  if (!pl) return SW_OK;
  if (pl->gexec) cudaGraphExecDestroy(pl->gexec);
  if (pl->cap_stream) cudaStreamDestroy(pl->cap_stream);
  if (pl->d_count) cudaFree(pl->d_count);
  if (pl->fused_buf) cudaFree(pl->fused_buf);
  if (pl->d_err) cudaFree(pl->d_err);
  if (pl->d_bar) cudaFree(pl->d_bar);
  delete pl;
  return SW_OK;
}

int sw_step(sw_plan* pl, int32_t it, void* stream) {
  int rc = check_it(pl, it, 1);
  if (rc != SW_OK) return rc;
  cudaError_t e = enqueue_step(pl, it, true, true, false, 0.0, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "sw_step");
  return SW_OK;
}

int sw_step_amp(sw_plan* pl, int32_t it, double amplitude, void* stream) {
  if (!pl) return fail(SW_ERR_ARG, "null plan");
  if (!(pl->dim == 2 && pl->scheme == SW2D_RSG))
    return fail(SW_ERR_UNSUPPORTED, "a per-call source amplitude applies to the 2D RSG scheme");
  int rc = check_it(pl, it, 1);
  if (rc != SW_OK) return rc;
  cudaError_t e = enqueue_step(pl, it, true, true, true, amplitude, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "sw_step_amp");
  return SW_OK;
}

int sw_run(sw_plan* pl, int32_t it0, int32_t nsteps, int32_t use_graph, void* stream) {
  int rc = check_it(pl, it0, nsteps);
  if (rc != SW_OK) return rc;
  if (nsteps == 0) return SW_OK;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  if (pl->dim == 2 && pl->path == 3 && !pl->aea) {
    // one launch for the whole run: nothing to capture
    e = persistent_run2(pl, it0, nsteps, st);
    if (e != cudaSuccess) return cuda_fail(e, "sw_run: persistent launch");
    return SW_OK;
  }
  if (!use_graph) {
    e = enqueue_sequence(pl, it0, nsteps, st);
    if (e != cudaSuccess) return cuda_fail(e, "sw_run");
    return SW_OK;
  }
  if (!(pl->gexec && pl->g_it0 == it0 && pl->g_n == nsteps)) {
    if (pl->gexec) { cudaGraphExecDestroy(pl->gexec); pl->gexec = nullptr; }
    if (!pl->cap_stream) {
      e = cudaStreamCreateWithFlags(&pl->cap_stream, cudaStreamNonBlocking);
      if (e != cudaSuccess) return cuda_fail(e, "sw_run: capture stream");
    }
    e = cudaStreamBeginCapture(pl->cap_stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_fail(e, "sw_run: begin capture");
    cudaError_t le = enqueue_sequence(pl, it0, nsteps, pl->cap_stream);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(pl->cap_stream, &g);
    if (le != cudaSuccess) { if (g) cudaGraphDestroy(g); return cuda_fail(le, "sw_run: capture"); }
    if (e != cudaSuccess) return cuda_fail(e, "sw_run: end capture");
    e = cudaGraphInstantiate(&pl->gexec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { pl->gexec = nullptr; return cuda_fail(e, "sw_run: instantiate"); }
    pl->g_it0 = it0;
    pl->g_n = nsteps;
  }
  e = cudaGraphLaunch(pl->gexec, st);
  if (e != cudaSuccess) return cuda_fail(e, "sw_run: graph launch");
  return SW_OK;
}

int sw_check_finite(sw_plan* pl, void* stream, int64_t* nonfinite) {
  if (!pl || !nonfinite) return fail(SW_ERR_ARG, "null plan or output");
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  if (!pl->d_count) {
    e = cudaMalloc(&pl->d_count, sizeof(unsigned long long));
    if (e != cudaSuccess) return cuda_fail(e, "sw_check_finite: counter");
  }
  e = cudaMemsetAsync(pl->d_count, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return cuda_fail(e, "sw_check_finite: reset");
  for (int q = 0; q < pl->nfield; ++q) {
    if (pl->dtype == SW_F32) k_count_nonfinite<float><<<1184, 256, 0, st>>>((const float*)pl->fields[q], pl->ncell, pl->d_count);
    else k_count_nonfinite<double><<<1184, 256, 0, st>>>((const double*)pl->fields[q], pl->ncell, pl->d_count);
  }
  unsigned long long h = 0;
  e = cudaMemcpyAsync(&h, pl->d_count, sizeof h, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "sw_check_finite");
  *nonfinite = (int64_t)h;
  if (h) return fail(SW_ERR_NONFINITE, "wavefield holds " + std::to_string(h) + " non-finite values");
  return SW_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// 2D adjoint: forward recording and the reverse sweep
// ---------------------------------------------------------------------------
namespace {

int adjoint_plan_ok(sw_plan* pl, const char* who) {
  if (!pl) return fail(SW_ERR_ARG, std::string(who) + ": null plan");
  if (pl->dim != 2 || (pl->scheme != SW2D_SSG_VS && pl->scheme != SW2D_SSG_SV))
    return fail(SW_ERR_UNSUPPORTED, std::string(who) + ": the adjoint covers the 2D SSG_VS and SSG_SV schemes");
  if (pl->src_kind != SW_SRC_MOMENT && pl->src_kind != SW_SRC_NONE)
    return fail(SW_ERR_UNSUPPORTED, std::string(who) + ": the adjoint covers moment-tensor sources");
  if (pl->aea) return fail(SW_ERR_UNSUPPORTED, std::string(who) + ": the adjoint does not cover the free-surface mode");
  const int nrec = pl->dtype == SW_F32 ? pl->p2f.nrec : pl->p2d.nrec;
  const int rf = pl->dtype == SW_F32 ? pl->p2f.rec_field : pl->p2d.rec_field;
  if (nrec > 0 && rf != (pl->scheme == SW2D_SSG_VS ? 1 : 0))
    return fail(SW_ERR_UNSUPPORTED,
                std::string(who) + ": the adjoint covers receivers of the scheme's own component (VS: vz, SV: vx)");
  return SW_OK;
}

template <typename T>
long long snap_elems(const sw::P2<T>& p) {
  return 5LL * p.nx * p.nz + 4 * p.mcomp[0] + 4 * p.mcomp[1];
}

template <typename T>
cudaError_t snap_store(const sw::P2<T>& p, T* slot, cudaStream_t st) {
  const long long nc = (long long)p.nx * p.nz;
  cudaError_t e = cudaSuccess;
  for (int q = 0; q < 5 && e == cudaSuccess; ++q)
    e = cudaMemcpyAsync(slot + q * nc, p.f[q], nc * sizeof(T), cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess && p.mcomp[0] > 0)
    e = cudaMemcpyAsync(slot + 5 * nc, p.mem[0], 4 * p.mcomp[0] * sizeof(T), cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess && p.mcomp[1] > 0)
    e = cudaMemcpyAsync(slot + 5 * nc + 4 * p.mcomp[0], p.mem[1], 4 * p.mcomp[1] * sizeof(T),
                        cudaMemcpyDeviceToDevice, st);
  return e;
}

template <typename T>
cudaError_t record2(sw_plan* pl, const sw::P2<T>& p, int it0, int n, T* snap, cudaStream_t st) {
  const long long se = snap_elems(p);
  for (int k = 0; k < n; ++k) {
    const int it = it0 + k;
    cudaError_t e = cudaSuccess;
    if (pl->src_kind == SW_SRC_MOMENT) e = sw::sw2_moment_inject<T>(p, it, st);
    if (e == cudaSuccess) e = snap_store(p, snap + k * se, st);
    if (e == cudaSuccess) e = sw::sw2_step<T>(p, pl->scheme, pl->order, it, (T)0, pl->gather_in_stress, false, false, 0, st);
    if (e != cudaSuccess) return e;
  }
  return snap_store(p, snap + (long long)n * se, st);
}

template <typename T>
cudaError_t adjoint2(sw_plan* pl, const sw::P2<T>& p, const sw2d_adjoint_desc* d, int it0, int n, const T* snap,
                     cudaStream_t st) {
  sw::A2<T> a{};
  for (int q = 0; q < 5; ++q) a.f[q] = (T*)d->field[q];
  for (int q = 0; q < 2; ++q) a.mem[q] = (T*)d->mem[q];
  for (int q = 0; q < 4; ++q) a.tmp[q] = (T*)d->tmp[q];
  for (int q = 0; q < 5; ++q) a.grad[q] = (T*)d->grad[q];
  a.res = (const T*)d->residual;
  const long long se = snap_elems(p);
  for (int k = n - 1; k >= 0; --k) {
    a.snap0 = snap + k * se;
    a.snap1 = snap + (k + 1) * se;
    cudaError_t e = sw::sw2_adjoint_step<T>(p, a, pl->scheme, pl->order, it0 + k, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

int adjoint3_plan_ok(sw_plan* pl, const char* who) {
  if (!pl) return fail(SW_ERR_ARG, std::string(who) + ": null plan");
  if (pl->dim != 3 || (pl->scheme != SW3D_CPML_TENSOR && pl->scheme != SW3D_CPML_FORCE))
    return fail(SW_ERR_UNSUPPORTED,
                std::string(who) + ": the 3D adjoint covers the CPML moment-tensor and point-force schemes");
  if (pl->order > 4) return fail(SW_ERR_UNSUPPORTED, std::string(who) + ": the 3D adjoint covers orders 1..4");
  if (pl->aea) return fail(SW_ERR_UNSUPPORTED, std::string(who) + ": the adjoint does not cover the free-surface mode");
  return SW_OK;
}

template <typename T>
long long snap3_elems(const sw::P3<T>& p) {
  return 9LL * p.nx * p.ny * p.nz + 6 * (p.mcomp[0] + p.mcomp[1] + p.mcomp[2]);
}

template <typename T>
cudaError_t snap3_store(const sw::P3<T>& p, T* slot, cudaStream_t st) {
  const long long nc = (long long)p.nx * p.ny * p.nz;
  cudaError_t e = cudaSuccess;
  for (int q = 0; q < 9 && e == cudaSuccess; ++q)
    e = cudaMemcpyAsync(slot + q * nc, p.f[q], nc * sizeof(T), cudaMemcpyDeviceToDevice, st);
  long long off = 9 * nc;
  for (int a = 0; a < 3 && e == cudaSuccess; ++a) {
    if (p.mcomp[a] > 0)
      e = cudaMemcpyAsync(slot + off, p.mem[a], 6 * p.mcomp[a] * sizeof(T), cudaMemcpyDeviceToDevice, st);
    off += 6 * p.mcomp[a];
  }
  return e;
}

template <typename T>
cudaError_t record3(sw_plan* pl, const sw::P3<T>& p, int it0, int n, T* snap, cudaStream_t st) {
  const long long se = snap3_elems(p);
  sw::P3<T> q = p;
  if (!pl->gather_in_stress) q.nrec = 0;
  const bool tensor = pl->scheme == SW3D_CPML_TENSOR;
  const bool moment = pl->src_kind == SW_SRC_MOMENT, force = pl->src_kind == SW_SRC_FORCE;
  for (int k = 0; k < n; ++k) {
    const int it = it0 + k;
    cudaError_t e = moment ? sw::sw3_moment_inject<T>(p, it, st) : cudaSuccess;
    if (e == cudaSuccess) e = snap3_store(p, snap + k * se, st);
    if (e == cudaSuccess) e = sw::sw3_velocity<T>(q, pl->order, it, tensor, force && pl->src_in_kernel, st);
    if (e == cudaSuccess && force && !pl->src_in_kernel) e = sw::sw3_force_inject<T>(p, it, st);
    if (e == cudaSuccess) e = sw::sw3_stress<T>(q, pl->order, it, false, st);
    if (e == cudaSuccess && !pl->gather_in_stress) e = sw::sw3_gather<T>(p, it, st);
    if (e != cudaSuccess) return e;
  }
  return snap3_store(p, snap + (long long)n * se, st);
}

template <typename T>
cudaError_t adjoint3(sw_plan* pl, const sw::P3<T>& p, const sw3d_adjoint_desc* d, int it0, int n, const T* snap,
                     cudaStream_t st) {
  sw::A3<T> a{};
  for (int q = 0; q < 9; ++q) a.f[q] = (T*)d->field[q];
  for (int q = 0; q < 3; ++q) a.mem[q] = (T*)d->mem[q];
  for (int q = 0; q < 9; ++q) a.tmp[q] = (T*)d->tmp[q];
  for (int q = 0; q < 8; ++q) a.grad[q] = (T*)d->grad[q];
  a.res = (const T*)d->residual;
  const long long se = snap3_elems(p);
  for (int k = n - 1; k >= 0; --k) {
    a.snap0 = snap + k * se;
    a.snap1 = snap + (k + 1) * se;
    cudaError_t e = sw::sw3_adjoint_step<T>(p, a, pl->order, it0 + k, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace

extern "C" {

int sw3d_snapshot_elems(sw_plan* pl, int64_t* elems) {
  int rc = adjoint3_plan_ok(pl, "sw3d_snapshot_elems");
  if (rc != SW_OK) return rc;
  if (!elems) return fail(SW_ERR_ARG, "sw3d_snapshot_elems: null output");
  *elems = pl->dtype == SW_F32 ? snap3_elems(pl->p3f) : snap3_elems(pl->p3d);
  return SW_OK;
}

int sw3d_record(sw_plan* pl, int32_t it0, int32_t nsteps, void* snap, void* stream) {
  int rc = adjoint3_plan_ok(pl, "sw3d_record");
  if (rc != SW_OK) return rc;
  if ((rc = check_it(pl, it0, nsteps)) != SW_OK) return rc;
  if (!snap || !aligned(snap, dsize(pl->dtype))) return fail(SW_ERR_ARG, "sw3d_record: snapshot buffer");
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = pl->dtype == SW_F32 ? record3<float>(pl, pl->p3f, it0, nsteps, (float*)snap, st)
                                      : record3<double>(pl, pl->p3d, it0, nsteps, (double*)snap, st);
  return e == cudaSuccess ? SW_OK : cuda_fail(e, "sw3d_record");
}

int sw3d_adjoint_run(sw_plan* pl, const sw3d_adjoint_desc* d, int32_t it0, int32_t nsteps, const void* snap,
                     void* stream) {
  int rc = adjoint3_plan_ok(pl, "sw3d_adjoint_run");
  if (rc != SW_OK) return rc;
  if ((rc = check_it(pl, it0, nsteps)) != SW_OK) return rc;
  const int esz = dsize(pl->dtype);
  if (!d || !snap || !aligned(snap, esz)) return fail(SW_ERR_ARG, "sw3d_adjoint_run: descriptor or snapshots");
  for (int q = 0; q < 9; ++q)
    if (!d->field[q] || !aligned(d->field[q], esz) || !d->tmp[q] || !aligned(d->tmp[q], esz))
      return fail(SW_ERR_ARG, "sw3d_adjoint_run: adjoint field or scratch pointer");
  for (int q = 0; q < 8; ++q)
    if (!d->grad[q] || !aligned(d->grad[q], esz)) return fail(SW_ERR_ARG, "sw3d_adjoint_run: gradient pointer");
  for (int a = 0; a < 3; ++a) {
    const long long mc = pl->dtype == SW_F32 ? pl->p3f.mcomp[a] : pl->p3d.mcomp[a];
    if (mc > 0 && !d->mem[a]) return fail(SW_ERR_ARG, "sw3d_adjoint_run: adjoint memory variables missing");
  }
  const int nrec = pl->dtype == SW_F32 ? pl->p3f.nrec : pl->p3d.nrec;
  if (nrec > 0 && !d->residual) return fail(SW_ERR_ARG, "sw3d_adjoint_run: residual missing");
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = pl->dtype == SW_F32 ? adjoint3<float>(pl, pl->p3f, d, it0, nsteps, (const float*)snap, st)
                                      : adjoint3<double>(pl, pl->p3d, d, it0, nsteps, (const double*)snap, st);
  return e == cudaSuccess ? SW_OK : cuda_fail(e, "sw3d_adjoint_run");
}

int sw2d_snapshot_elems(sw_plan* pl, int64_t* elems) {
  int rc = adjoint_plan_ok(pl, "sw2d_snapshot_elems");
  if (rc != SW_OK) return rc;
  if (!elems) return fail(SW_ERR_ARG, "sw2d_snapshot_elems: null output");
  *elems = pl->dtype == SW_F32 ? snap_elems(pl->p2f) : snap_elems(pl->p2d);
  return SW_OK;
}

int sw2d_record(sw_plan* pl, int32_t it0, int32_t nsteps, void* snap, void* stream) {
  int rc = adjoint_plan_ok(pl, "sw2d_record");
  if (rc != SW_OK) return rc;
  if ((rc = check_it(pl, it0, nsteps)) != SW_OK) return rc;
  if (!snap || !aligned(snap, dsize(pl->dtype))) return fail(SW_ERR_ARG, "sw2d_record: snapshot buffer");
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = pl->dtype == SW_F32 ? record2<float>(pl, pl->p2f, it0, nsteps, (float*)snap, st)
                                      : record2<double>(pl, pl->p2d, it0, nsteps, (double*)snap, st);
  if (e != cudaSuccess) return cuda_fail(e, "sw2d_record");
  return SW_OK;
}

int sw2d_adjoint_run(sw_plan* pl, const sw2d_adjoint_desc* d, int32_t it0, int32_t nsteps, const void* snap,
                     void* stream) {
  int rc = adjoint_plan_ok(pl, "sw2d_adjoint_run");
  if (rc != SW_OK) return rc;
  if ((rc = check_it(pl, it0, nsteps)) != SW_OK) return rc;
  const int esz = dsize(pl->dtype);
  if (!d || !snap || !aligned(snap, esz)) return fail(SW_ERR_ARG, "sw2d_adjoint_run: descriptor or snapshots");
  for (int q = 0; q < 5; ++q)
    if (!d->field[q] || !aligned(d->field[q], esz) || !d->grad[q] || !aligned(d->grad[q], esz))
      return fail(SW_ERR_ARG, "sw2d_adjoint_run: adjoint field or gradient pointer");
  for (int q = 0; q < 4; ++q)
    if (!d->tmp[q] || !aligned(d->tmp[q], esz)) return fail(SW_ERR_ARG, "sw2d_adjoint_run: scratch pointer");
  const long long mc0 = pl->dtype == SW_F32 ? pl->p2f.mcomp[0] : pl->p2d.mcomp[0];
  const long long mc1 = pl->dtype == SW_F32 ? pl->p2f.mcomp[1] : pl->p2d.mcomp[1];
  if ((mc0 > 0 && !d->mem[0]) || (mc1 > 0 && !d->mem[1]))
    return fail(SW_ERR_ARG, "sw2d_adjoint_run: adjoint memory variables missing");
  const int nrec = pl->dtype == SW_F32 ? pl->p2f.nrec : pl->p2d.nrec;
  if (nrec > 0 && !d->residual) return fail(SW_ERR_ARG, "sw2d_adjoint_run: residual missing");
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = pl->dtype == SW_F32 ? adjoint2<float>(pl, pl->p2f, d, it0, nsteps, (const float*)snap, st)
                                      : adjoint2<double>(pl, pl->p2d, d, it0, nsteps, (const double*)snap, st);
  if (e != cudaSuccess) return cuda_fail(e, "sw2d_adjoint_run");
  return SW_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// learned thin absorbing layer (2D)
// ---------------------------------------------------------------------------
namespace {

int abc_args(sw_plan* pl, const sw_abc_desc* d, const char* who, sw::AbcArgs* a) {
  if (!pl || !d) return fail(SW_ERR_ARG, std::string(who) + ": null plan or descriptor");
  if (pl->dim != 2 || pl->dtype != SW_F32)
    return fail(SW_ERR_UNSUPPORTED, std::string(who) + ": the learned layer runs on float32 2D plans");
  if (d->ncell < 0 || (d->ncell > 0 && (!d->cell || !d->face || !d->depth || !d->params || !d->delta)))
    return fail(SW_ERR_ARG, std::string(who) + ": layer tables, parameters or scratch missing");
  for (int f = 0; f < 5; ++f)
    if (!(d->scale[f] > 0.f) || !(d->oscale[f] >= 0.f))
      return fail(SW_ERR_ARG, std::string(who) + ": field scales must be positive");
  *a = sw::AbcArgs{};
  a->cell = d->cell; a->face = d->face; a->depth = d->depth; a->ncell = d->ncell;
  a->nx = pl->p2f.nx; a->nz = pl->p2f.nz;
  for (int f = 0; f < 5; ++f) {
    a->f[f] = pl->p2f.f[f];
    a->fw[f] = pl->p2f.f[f];
    a->scale[f] = d->scale[f];
    a->oscale[f] = d->oscale[f];
  }
  a->params = d->params;
  a->delta = d->delta;
  return SW_OK;
}

}  // namespace

extern "C" {

int sw2d_abc_correct(sw_plan* pl, const sw_abc_desc* d, void* stream) {
  sw::AbcArgs a;
  int rc = abc_args(pl, d, "sw2d_abc_correct", &a);
  if (rc != SW_OK) return rc;
  cudaError_t e = sw::abc_correct(a, (cudaStream_t)stream);
  return e == cudaSuccess ? SW_OK : cuda_fail(e, "sw2d_abc_correct");
}

int sw2d_abc_features(sw_plan* pl, const sw_abc_desc* d, float* x, void* stream) {
  sw::AbcArgs a;
  int rc = abc_args(pl, d, "sw2d_abc_features", &a);
  if (rc != SW_OK) return rc;
  if (d->ncell > 0 && !x) return fail(SW_ERR_ARG, "sw2d_abc_features: null output");
  a.x_out = x;
  cudaError_t e = sw::abc_features(a, (cudaStream_t)stream);
  return e == cudaSuccess ? SW_OK : cuda_fail(e, "sw2d_abc_features");
}

int sw_mlp_grad(const float* params, const float* x, const float* y, int64_t n, float* grad, float* loss,
                void* stream) {
  if (n < 0 || (n > 0 && (!params || !x || !y || !grad || !loss))) return fail(SW_ERR_ARG, "sw_mlp_grad: arguments");
  cudaError_t e = sw::mlp_grad(params, x, y, n, grad, loss, 0, (cudaStream_t)stream);
  return e == cudaSuccess ? SW_OK : cuda_fail(e, "sw_mlp_grad");
}

}  // extern "C"

namespace {

int abc3_args(sw_plan* pl, const sw_abc3_desc* d, const char* who, sw::AbcArgs3* a) {
  if (!pl || !d) return fail(SW_ERR_ARG, std::string(who) + ": null plan or descriptor");
  if (pl->dim != 3 || pl->dtype != SW_F32 || pl->scheme != SW3D_CPML_TENSOR)
    return fail(SW_ERR_UNSUPPORTED, std::string(who) + ": the 3D learned layer runs on float32 moment-tensor plans");
  if (d->ncell < 0 || (d->ncell > 0 && (!d->cell || !d->face || !d->depth || !d->params || !d->delta)))
    return fail(SW_ERR_ARG, std::string(who) + ": layer tables, parameters or scratch missing");
  for (int f = 0; f < 9; ++f)
    if (!(d->scale[f] > 0.f) || !(d->oscale[f] >= 0.f))
      return fail(SW_ERR_ARG, std::string(who) + ": field scales must be positive");
  *a = sw::AbcArgs3{};
  a->cell = d->cell; a->face = d->face; a->depth = d->depth; a->ncell = d->ncell;
  a->nx = pl->p3f.nx; a->ny = pl->p3f.ny; a->nz = pl->p3f.nz;
  for (int f = 0; f < 9; ++f) {
    a->f[f] = pl->p3f.f[f];
    a->fw[f] = pl->p3f.f[f];
    a->scale[f] = d->scale[f];
    a->oscale[f] = d->oscale[f];
  }
  a->params = d->params;
  a->delta = d->delta;
  return SW_OK;
}

}  // namespace

extern "C" {

int sw3d_abc_correct(sw_plan* pl, const sw_abc3_desc* d, void* stream) {
  sw::AbcArgs3 a;
  int rc = abc3_args(pl, d, "sw3d_abc_correct", &a);
  if (rc != SW_OK) return rc;
  cudaError_t e = sw::abc3_correct(a, (cudaStream_t)stream);
  return e == cudaSuccess ? SW_OK : cuda_fail(e, "sw3d_abc_correct");
}

int sw3d_abc_features(sw_plan* pl, const sw_abc3_desc* d, float* x, void* stream) {
  sw::AbcArgs3 a;
  int rc = abc3_args(pl, d, "sw3d_abc_features", &a);
  if (rc != SW_OK) return rc;
  if (d->ncell > 0 && !x) return fail(SW_ERR_ARG, "sw3d_abc_features: null output");
  a.x_out = x;
  cudaError_t e = sw::abc3_features(a, (cudaStream_t)stream);
  return e == cudaSuccess ? SW_OK : cuda_fail(e, "sw3d_abc_features");
}

int sw3d_abc_adjoint(sw_plan* pl, const sw_abc3_desc* d, const float* fields, float* const* adj, float* ybar,
                     void* stream) {
  sw::AbcArgs3 a;
  int rc = abc3_args(pl, d, "sw3d_abc_adjoint", &a);
  if (rc != SW_OK) return rc;
  if (d->ncell > 0 && (!fields || !adj || !ybar)) return fail(SW_ERR_ARG, "sw3d_abc_adjoint: null argument");
  const long long nc = (long long)a.nx * a.ny * a.nz;
  for (int f = 0; f < 9; ++f) {
    if (d->ncell > 0 && !adj[f]) return fail(SW_ERR_ARG, "sw3d_abc_adjoint: adjoint field missing");
    a.f[f] = fields + f * nc;
  }
  cudaError_t e = sw::abc3_adjoint(a, adj, ybar, (cudaStream_t)stream);
  return e == cudaSuccess ? SW_OK : cuda_fail(e, "sw3d_abc_adjoint");
}

int sw3d_mlp_grad(const float* params, const float* x, const float* y, int64_t n, float* grad, float* loss,
                  void* stream) {
  if (n < 0 || (n > 0 && (!params || !x || !y || !grad || !loss))) return fail(SW_ERR_ARG, "sw3d_mlp_grad: arguments");
  cudaError_t e = sw::mlp3_grad(params, x, y, n, grad, loss, 0, (cudaStream_t)stream);
  return e == cudaSuccess ? SW_OK : cuda_fail(e, "sw3d_mlp_grad");
}

int sw3d_mlp_forward(const float* params, const float* x, int64_t n, float* y, void* stream) {
  if (n < 0 || (n > 0 && (!params || !x || !y))) return fail(SW_ERR_ARG, "sw3d_mlp_forward: arguments");
  cudaError_t e = sw::mlp3_forward_batch(params, x, n, y, (cudaStream_t)stream);
  return e == cudaSuccess ? SW_OK : cuda_fail(e, "sw3d_mlp_forward");
}

int sw3d_mlp_backward(const float* params, const float* x, const float* dy, int64_t n, float* grad, void* stream) {
  if (n < 0 || (n > 0 && (!params || !x || !dy || !grad))) return fail(SW_ERR_ARG, "sw3d_mlp_backward: arguments");
  cudaError_t e = sw::mlp3_grad(params, x, dy, n, grad, nullptr, 1, (cudaStream_t)stream);
  return e == cudaSuccess ? SW_OK : cuda_fail(e, "sw3d_mlp_backward");
}

int sw_mlp_backward(const float* params, const float* x, const float* dy, int64_t n, float* grad, void* stream) {
  if (n < 0 || (n > 0 && (!params || !x || !dy || !grad))) return fail(SW_ERR_ARG, "sw_mlp_backward: arguments");
  cudaError_t e = sw::mlp_grad(params, x, dy, n, grad, nullptr, 1, (cudaStream_t)stream);
  return e == cudaSuccess ? SW_OK : cuda_fail(e, "sw_mlp_backward");
}

int sw2d_abc_adjoint(sw_plan* pl, const sw_abc_desc* d, const float* fields, float* const* adj, float* ybar,
                     void* stream) {
  sw::AbcArgs a;
  int rc = abc_args(pl, d, "sw2d_abc_adjoint", &a);
  if (rc != SW_OK) return rc;
  if (d->ncell > 0 && (!fields || !adj || !ybar)) return fail(SW_ERR_ARG, "sw2d_abc_adjoint: null argument");
  const long long nc = (long long)a.nx * a.nz;
  for (int f = 0; f < 5; ++f) {
    if (d->ncell > 0 && !adj[f]) return fail(SW_ERR_ARG, "sw2d_abc_adjoint: adjoint field missing");
    a.f[f] = fields + f * nc;
  }
  cudaError_t e = sw::abc_adjoint(a, adj, ybar, (cudaStream_t)stream);
  return e == cudaSuccess ? SW_OK : cuda_fail(e, "sw2d_abc_adjoint");
}

int sw_mlp_forward(const float* params, const float* x, int64_t n, float* y, void* stream) {
  if (n < 0 || (n > 0 && (!params || !x || !y))) return fail(SW_ERR_ARG, "sw_mlp_forward: arguments");
  cudaError_t e = sw::mlp_forward_batch(params, x, n, y, (cudaStream_t)stream);
  return e == cudaSuccess ? SW_OK : cuda_fail(e, "sw_mlp_forward");
}

}  // extern "C"

// ---------------------------------------------------------------------------
// batches of 2D shots of uneven sizes
// ---------------------------------------------------------------------------
struct sw_batch {
  int nshots = 0, scheme = 0, dtype = 0, order = 0, nt_max = 0;
  bool fold = true;                       // next-step moment source folded into the stress pass
  std::vector<sw_plan*> plans;            // per-shot validated plans
  std::vector<char> shots;                // host P2<T>[nshots], passed to the kernels by value
  int2* d_work = nullptr;                 // device, per tile shape: one work item per block
  long long work_off[SW_BATCH_TILES] = {};
  int total[SW_BATCH_TILES] = {};
  // per tile shape and group of SW_BATCH_GROUP shots: first work item and count
  std::vector<long long> grp_off[SW_BATCH_TILES];
  std::vector<int> grp_n[SW_BATCH_TILES];
  int cfg = 0;
  long long cells = 0;
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t gexec = nullptr;
  int g_it0 = -1, g_n = -1, g_cfg = -1;
};

namespace {

// group g of the batch (shots g*SW_BATCH_GROUP ..) for the current tile shape
template <typename T>
sw::Batch2<T> batch_group(const sw_batch* b, int g) {
  sw::Batch2<T> v{};
  v.first = g * SW_BATCH_GROUP;
  v.n = std::min(SW_BATCH_GROUP, b->nshots - v.first);
  memcpy(v.shots, b->shots.data() + sizeof(sw::P2<T>) * v.first, sizeof(sw::P2<T>) * v.n);
  v.work = b->d_work + b->grp_off[b->cfg][g];
  return v;
}

template <typename T>
cudaError_t batch_sequence_t(sw_batch* b, int it0, int n, cudaStream_t st) {
  const int groups = (b->nshots + SW_BATCH_GROUP - 1) / SW_BATCH_GROUP;
  std::vector<sw::Batch2<T>> views;
  for (int g = 0; g < groups; ++g) views.push_back(batch_group<T>(b, g));
  for (int s = 0; s < n; ++s) {
    const int it = it0 + s;
    const bool pre = s == 0 || !b->fold, nxt = b->fold && s != n - 1;
    for (int g = 0; g < groups; ++g) {
      cudaError_t e = sw::sw2b_step<T>(views[g], b->scheme, b->order, b->cfg, b->grp_n[b->cfg][g], it, pre, nxt, st);
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

cudaError_t batch_sequence(sw_batch* b, int it0, int n, cudaStream_t st) {
  return b->dtype == SW_F32 ? batch_sequence_t<float>(b, it0, n, st) : batch_sequence_t<double>(b, it0, n, st);
}

void batch_free(sw_batch* b) {
  if (!b) return;
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  if (b->d_work) cudaFree(b->d_work);
  for (sw_plan* p : b->plans) sw_plan_destroy(p);
  delete b;
}

}  // namespace

extern "C" {

int sw2d_batch_create(const sw2d_desc* shots, int32_t nshots, sw_batch** out) {
  g_err.clear();
  if (!shots || !out || nshots <= 0) return fail(SW_ERR_ARG, "sw2d_batch_create: empty batch or null output");
  *out = nullptr;
  const sw2d_desc& d0 = shots[0];
  if (d0.scheme != SW2D_SSG_VS && d0.scheme != SW2D_SSG_SV)
    return fail(SW_ERR_UNSUPPORTED, "sw2d_batch_create: batches run the SSG_VS or SSG_SV scheme");
  sw_batch* b = new sw_batch();
  b->nshots = nshots; b->scheme = d0.scheme; b->dtype = d0.dtype; b->order = d0.order; b->nt_max = d0.nt_max;
  for (int s = 0; s < nshots; ++s) {
    const sw2d_desc& d = shots[s];
    if (d.scheme != d0.scheme || d.dtype != d0.dtype || d.order != d0.order || d.nt_max != d0.nt_max) {
      batch_free(b);
      return fail(SW_ERR_ARG, "sw2d_batch_create: shot " + std::to_string(s) +
                                  " differs from shot 0 in scheme, dtype, order or nt_max");
    }
    sw_plan* pl = nullptr;
    int rc = sw2d_plan_create(&d, &pl);
    if (rc != SW_OK) {
      std::string m = g_err;
      batch_free(b);
      return fail(rc, "sw2d_batch_create: shot " + std::to_string(s) + ": " + m);
    }
    b->plans.push_back(pl);
    if (!pl->gather_in_stress || (long long)d.rec.nrec > (long long)d.nx * d.nz) {
      batch_free(b);
      return fail(SW_ERR_UNSUPPORTED, "sw2d_batch_create: shot " + std::to_string(s) +
                                          ": batch receivers record a velocity field, at most one per cell");
    }
    b->cells += (long long)d.nx * d.nz;
  }
  const size_t psz = b->dtype == SW_F32 ? sizeof(sw::P2<float>) : sizeof(sw::P2<double>);
  b->shots.resize(psz * nshots);
  for (int s = 0; s < nshots; ++s) {
    if (b->dtype == SW_F32) memcpy(b->shots.data() + psz * s, &b->plans[s]->p2f, psz);
    else memcpy(b->shots.data() + psz * s, &b->plans[s]->p2d, psz);
  }
  // work items, shot by shot, tile rows (x) outer, tile columns (z) inner
  std::vector<int2> work;
  for (int c = 0; c < SW_BATCH_TILES; ++c) {
    int bx, bz;
    sw::sw2b_tile_shape(c, &bx, &bz);
    b->work_off[c] = (long long)work.size();
    for (int s = 0; s < nshots; ++s) {
      if (s % SW_BATCH_GROUP == 0) {
        b->grp_off[c].push_back((long long)work.size());
        b->grp_n[c].push_back(0);
      }
      const int tx = (shots[s].nx + bx - 1) / bx, tz = (shots[s].nz + bz - 1) / bz;
      if (tx > 0xffff || tz > 0xffff) {
        batch_free(b);
        return fail(SW_ERR_ARG, "sw2d_batch_create: shot " + std::to_string(s) + " has too many tiles");
      }
      for (int x = 0; x < tx; ++x)
        for (int z = 0; z < tz; ++z) work.push_back(make_int2(s, (x << 16) | z));
      const long long gn = (long long)work.size() - b->grp_off[c].back();
      if (gn > 0x7fffffffLL) {
        batch_free(b);
        return fail(SW_ERR_ARG, "sw2d_batch_create: batch too large for one launch");
      }
      b->grp_n[c].back() = (int)gn;
    }
    const long long tot = (long long)work.size() - b->work_off[c];
    if (tot > 0x7fffffffLL) {
      batch_free(b);
      return fail(SW_ERR_ARG, "sw2d_batch_create: batch too large for one launch");
    }
    b->total[c] = (int)tot;
  }
  cudaError_t e = cudaMalloc((void**)&b->d_work, work.size() * sizeof(int2));
  if (e == cudaSuccess) e = cudaMemcpy(b->d_work, work.data(), work.size() * sizeof(int2), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    batch_free(b);
    return cuda_fail(e, "sw2d_batch_create");
  }
  *out = b;
  return SW_OK;
}

int sw_batch_set_tile(sw_batch* b, int32_t cfg) {
  if (!b) return fail(SW_ERR_ARG, "null batch");
  if (cfg < 0 || cfg >= SW_BATCH_TILES) return fail(SW_ERR_ARG, "sw_batch_set_tile: tile shape index out of range");
  b->cfg = cfg;
  return SW_OK;
}

int sw_batch_info(sw_batch* b, int32_t* info) {
  if (!b || !info) return fail(SW_ERR_ARG, "null batch or output");
  int bx, bz;
  sw::sw2b_tile_shape(b->cfg, &bx, &bz);
  info[0] = b->cfg;
  info[1] = SW_BATCH_TILES;
  info[2] = b->total[b->cfg];
  info[3] = bx;
  info[4] = bz;
  info[5] = b->nshots;
  return SW_OK;
}

int sw_batch_run(sw_batch* b, int32_t it0, int32_t nsteps, int32_t use_graph, void* stream) {
  if (!b) return fail(SW_ERR_ARG, "null batch");
  if (it0 < 0 || nsteps < 0 || (long long)it0 + nsteps > b->nt_max)
    return fail(SW_ERR_ARG, "sw_batch_run: steps outside 0..nt_max-1");
  if (nsteps == 0) return SW_OK;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  if (!use_graph) {
    e = batch_sequence(b, it0, nsteps, st);
    return e == cudaSuccess ? SW_OK : cuda_fail(e, "sw_batch_run");
  }
  if (!(b->gexec && b->g_it0 == it0 && b->g_n == nsteps && b->g_cfg == b->cfg)) {
    if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
    if (!b->cap_stream) {
      e = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking);
      if (e != cudaSuccess) return cuda_fail(e, "sw_batch_run: capture stream");
    }
    e = cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_fail(e, "sw_batch_run: begin capture");
    cudaError_t le = batch_sequence(b, it0, nsteps, b->cap_stream);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(b->cap_stream, &g);
    if (le != cudaSuccess) { if (g) cudaGraphDestroy(g); return cuda_fail(le, "sw_batch_run: capture"); }
    if (e != cudaSuccess) return cuda_fail(e, "sw_batch_run: end capture");
    e = cudaGraphInstantiate(&b->gexec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { b->gexec = nullptr; return cuda_fail(e, "sw_batch_run: instantiate"); }
    b->g_it0 = it0; b->g_n = nsteps; b->g_cfg = b->cfg;
  }
  e = cudaGraphLaunch(b->gexec, st);
  return e == cudaSuccess ? SW_OK : cuda_fail(e, "sw_batch_run: graph launch");
}

int sw_batch_destroy(sw_batch* b) {
  batch_free(b);
  return SW_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// sw_count_nonfinite_noalloc: the NaN/Inf scan of sw_check_finite over arrays
// the caller names, with its counters in a static device array instead of
// plan memory, so that the call allocates nothing.
// ---------------------------------------------------------------------------
namespace {

// One 64-bit counter per scanned array (SW_NOALLOC_MAX_ARRAYS * 8 = 512
// bytes).  Every call zeroes the counters it uses on its stream before the
// scan, so nothing has to be zero on entry.
static __device__ __align__(256) unsigned long long g_noalloc_count[SW_NOALLOC_MAX_ARRAYS];

constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned long long* g_noalloc_ptr[kNoallocMaxDevices] = {};

// Address of the counters on the current device, resolved once per device.
int noalloc_scratch(unsigned long long** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "sw_count_nonfinite_noalloc: current device");
  if (dev < 0 || dev >= kNoallocMaxDevices)
    return fail(SW_ERR_UNSUPPORTED, "sw_count_nonfinite_noalloc: device ordinal " + std::to_string(dev) +
                                        " is beyond the " + std::to_string(kNoallocMaxDevices) + " this build tracks");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    unsigned long long* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, g_noalloc_count);
    if (e != cudaSuccess) return cuda_fail(e, "sw_count_nonfinite_noalloc: scratch address");
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return SW_OK;
}

}  // namespace

extern "C" {

int sw_segy_decode(const void* traces, int64_t ntraces, int32_t nsamples, int32_t format, float* out,
                   int32_t* srcx, void* stream) {
  if (ntraces < 0 || nsamples < 0) return fail(SW_ERR_ARG, "sw_segy_decode: negative trace or sample count");
  if (format != 1 && format != 2 && format != 3 && format != 5 && format != 8)
    return fail(SW_ERR_UNSUPPORTED, "sw_segy_decode: sample format " + std::to_string(format) +
                                        " (supported: 1 IBM float, 2 int32, 3 int16, 5 IEEE float, 8 int8)");
  if (ntraces == 0 || nsamples == 0) return SW_OK;
  if (!traces || !out) return fail(SW_ERR_ARG, "sw_segy_decode: null traces or output");
  if (!aligned(traces, 4) || !aligned(out, 4) || (srcx && !aligned(srcx, 4)))
    return fail(SW_ERR_ARG, "sw_segy_decode: traces, out and srcx must be 4-byte aligned");
  cudaError_t e = sw::segy_decode(traces, ntraces, nsamples, format, out, srcx, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "sw_segy_decode");
  return SW_OK;
}

int sw_count_nonfinite_noalloc(const void* const* arrays, const int64_t* lengths, int32_t narrays, int32_t dtype,
                               void* stream, int64_t* counts) {
  if (narrays < 0 || narrays > SW_NOALLOC_MAX_ARRAYS)
    return fail(SW_ERR_ARG, "sw_count_nonfinite_noalloc: " + std::to_string(narrays) +
                                " arrays requested; the static scratch holds counters for at most " +
                                std::to_string(SW_NOALLOC_MAX_ARRAYS));
  if (narrays > 0 && (!arrays || !lengths || !counts))
    return fail(SW_ERR_ARG, "sw_count_nonfinite_noalloc: null arrays, lengths or counts");
  if (dtype != SW_F32 && dtype != SW_F64) return fail(SW_ERR_ARG, "sw_count_nonfinite_noalloc: dtype");
  for (int a = 0; a < narrays; ++a) {
    if (lengths[a] < 0) return fail(SW_ERR_ARG, "sw_count_nonfinite_noalloc: negative length");
    if (lengths[a] > 0 && !arrays[a]) return fail(SW_ERR_ARG, "sw_count_nonfinite_noalloc: null array");
  }
  if (narrays == 0) return SW_OK;
  unsigned long long* cnt = nullptr;
  int rc = noalloc_scratch(&cnt);
  if (rc != SW_OK) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * narrays, st);
  if (e != cudaSuccess) return cuda_fail(e, "sw_count_nonfinite_noalloc: reset");
  for (int a = 0; a < narrays; ++a) {
    if (lengths[a] == 0) continue;
    if (dtype == SW_F32)
      k_count_nonfinite<float><<<1184, 256, 0, st>>>((const float*)arrays[a], lengths[a], cnt + a);
    else
      k_count_nonfinite<double><<<1184, 256, 0, st>>>((const double*)arrays[a], lengths[a], cnt + a);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "sw_count_nonfinite_noalloc: launch");
  unsigned long long h[SW_NOALLOC_MAX_ARRAYS];
  e = cudaMemcpyAsync(h, cnt, sizeof(unsigned long long) * narrays, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "sw_count_nonfinite_noalloc");
  unsigned long long total = 0;
  for (int a = 0; a < narrays; ++a) {
    counts[a] = (int64_t)h[a];
    total += h[a];
  }
  if (total) return fail(SW_ERR_NONFINITE, "arrays hold " + std::to_string(total) + " non-finite values");
  return SW_OK;
}

}  // extern "C"
