/*
 * seiswave.h -- C ABI of libseiswave.so, the B200 (sm_100a) elastic
 * staggered-grid finite-difference time loop.
 *
 * The reference (SeisWave_Taichi) is pure Python/Taichi and has no FFI of its
 * own; each entry point below replaces one Taichi kernel or host routine of
 * the reference's ElasticWAVE classes (paths relative to the reference
 * project), and the Python package seiswave_taichi_b200 binds them through
 * ctypes with the reference's class names and signatures.
 *
 * Ownership: every array is allocated by the caller (PyTorch in the Python
 * package) and borrowed by the plan; nothing here frees caller memory.  A plan
 * owns only its small internal scratch (step counters, CUDA graphs), released
 * by sw_plan_destroy.  Device arrays are C-contiguous, last index fastest:
 * (nx, nz) in 2D, (nx, ny, nz) in 3D.
 *
 * Errors: every call returns SW_OK (0) or a negative SW_ERR_* code; the
 * message of the last failure on the calling thread is sw_last_error().
 * Nothing calls exit() or traps on the device.
 *
 * Threading: work is enqueued on the caller's stream (a cudaStream_t passed as
 * void*, NULL = legacy default stream).  A plan is not thread-safe; use one plan
 * per stream.  No call blocks the host except sw_check_finite,
 * sw_count_nonfinite_noalloc, sw_check_division and sw_plan_status.
 */
#ifndef SEISWAVE_H
#define SEISWAVE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define SW_API __attribute__((visibility("default")))
#else
#define SW_API
#endif

#define SW_ABI_VERSION 1
#define SW_MAX_ORDER 8 /* largest half-stencil length N (accuracy) */

/* status codes */
#define SW_OK 0
#define SW_ERR_ARG (-1)          /* invalid descriptor or argument */
#define SW_ERR_CUDA (-2)         /* a CUDA runtime call failed */
#define SW_ERR_NONFINITE (-3)    /* a wavefield holds NaN or Inf */
#define SW_ERR_UNSUPPORTED (-4)  /* valid request this build does not implement */
#define SW_ERR_TIMEOUT (-5)      /* a bounded device wait gave up */

/* element types */
#define SW_F32 0
#define SW_F64 1

/* 2D schemes: Elastic2D_CPML.py update_SSG_VS :128, update_SSG_SV :203, update_RSG :277 */
#define SW2D_SSG_VS 0
#define SW2D_SSG_SV 1
#define SW2D_RSG 2

/* 3D schemes: Elastic3D_SSG_CPML.py update_SSG :144 (point force),
 * Elastic3D_SSG_Tensor.py update_SSG :166 (moment tensor),
 * Elastic3D_SSG_SPML.py update_SSG_SPML :160 (split-field PML) */
#define SW3D_CPML_FORCE 0
#define SW3D_CPML_TENSOR 1
#define SW3D_SPML 2

/* source kinds */
#define SW_SRC_NONE 0
#define SW_SRC_FORCE 1  /* v[src] += dt*w/rho[src] after the velocity phase */
#define SW_SRC_MOMENT 2 /* sigma_ab[src] += w*(-M_ab) before the velocity phase */
#define SW_SRC_RSG4 3   /* 2D RSG: vz[isx+a,isz+b] += dt*w/(8 rho), a,b in {-1,0} */

/* One axis of the absorbing boundary, built on the host exactly as the
 * reference's SetADEPML2D/SetADEPML3D (Elastic2D_CPML.py:392-528,
 * Elastic3D_SSG_Tensor.py:361-568) builds it. */
typedef struct sw_pml_axis {
  int32_t lo;          /* memory-variable slab: indices [0, lo) ...            */
  int32_t hi;          /* ... and [n-hi, n) of this axis; elsewhere the CPML
                          correction is the identity and is not stored (split
                          PML: the slabs of the split-field shell)            */
  const void* coef;    /* 6*n values (field type): b, a, k at integer points,
                          then b_half, a_half, k_half                          */
  const void* damp;    /* 2*n values: d, d_half (split PML only, else NULL)    */
  const uint8_t* flag; /* n bytes: bit0 = integer point lies inside the PML
                          predicate (x<=xmin_pml or x>=xmax_pml), bit1 = half  */
} sw_pml_axis;

/* Receivers: data[it*nrec + r] = field[rec_index[r]] after step it. */
typedef struct sw_receivers {
  int32_t nrec;
  int32_t field;             /* index into the descriptor's field[] array      */
  const int64_t* index;      /* device, nrec linear cell indices               */
  void* data;                /* device, (nt_max, nrec) traces (reference .data) */
  int32_t dtype;             /* element type of data: SW_F32 or SW_F64         */
} sw_receivers;

typedef struct sw_source {
  int32_t kind;              /* SW_SRC_*                                       */
  int32_t i, j, k;           /* cell (k unused in 2D)                          */
  const void* wavelet;       /* device, nt_max values (field type)             */
  double mt[6];              /* moment tensor: xx yy zz xy xz yz (2D: xx zz xz in 0,2,4) */
} sw_source;

/* 2D: fields are vx vz sxx szz sxz; memory variables slab-compact:
 * mem[0] = x direction, (4, lo+hi, nz): sxx_dx sxz_dx dvx_dx dvz_dx;
 * mem[1] = z direction, (4, nx, lo+hi): sxz_dz szz_dz dvz_dz dvx_dz.
 * The same arrays serve the VS, SV and RSG schemes, as in the reference. */
typedef struct sw2d_desc {
  int32_t scheme, dtype, nx, nz, order;
  int32_t nt_max;
  double dx, dz, dt;
  double coef[SW_MAX_ORDER];
  void* field[5];            /* vx vz sxx szz sxz */
  const void* rho;
  const void* lam;
  const void* mu;
  sw_pml_axis pml[2];        /* x, z */
  void* mem[2];
  sw_source src;
  sw_receivers rec;
} sw2d_desc;

/* 3D: fields are vx vy vz sxx syy szz sxy sxz syz.
 * CPML memory variables slab-compact: mem[0] = x, (6, lo+hi, ny, nz):
 *   sxx_dx sxy_dx sxz_dx dvx_dx dvy_dx dvz_dx;
 * mem[1] = y, (6, nx, lo+hi, nz): sxy_dy syy_dy syz_dy dvy_dy dvx_dy dvz_dy;
 * mem[2] = z, (6, nx, ny, lo+hi): sxz_dz syz_dz szz_dz dvz_dz dvx_dz dvy_dz.
 * Split PML: the 24 split fields (vx_x vx_y vx_z vy_x vy_y vy_z vz_x vz_y vz_z
 * sxx_x sxx_y sxx_z syy_x syy_y syy_z sxy_x sxy_y sxz_x sxz_z syz_y syz_z szz_x
 * szz_y szz_z) are stored only on the PML shell: split = (24, S), where the
 * shell is the union of the axes' slabs [0, lo) and [n-hi, n) and its S cells
 * are ordered as the x slabs (sx, ny, nz), then the y slabs of the x interior
 * (nx-sx, sy, nz), then the z slabs of the x-y interior (nx-sx, ny-sy, sz),
 * with s_d = lo_d + hi_d and S = sx*ny*nz + (nx-sx)*sy*nz + (nx-sx)*(ny-sy)*sz.
 * For the split PML, lo and hi of each axis must cover every index whose
 * predicate flag is set (sw_plan_create checks it). */
typedef struct sw3d_desc {
  int32_t scheme, dtype, nx, ny, nz, order;
  int32_t nt_max;
  double dx, dy, dz, dt;
  double coef[SW_MAX_ORDER];
  void* field[9];            /* vx vy vz sxx syy szz sxy sxz syz */
  const void* rho;
  const void* lam;
  const void* mu;
  sw_pml_axis pml[3];        /* x, y, z */
  void* mem[3];
  void* split;
  sw_source src;
  sw_receivers rec;
} sw3d_desc;

typedef struct sw_plan sw_plan;

/* Version of this ABI (SW_ABI_VERSION). */
SW_API int sw_version(void);

/* Message of the last failed call on this thread ("" if none). */
SW_API const char* sw_last_error(void);

/* Validate a 2D descriptor and build a plan.  Replaces the state set-up of
 * Elastic2D_CPML.ElasticWAVE.__init__ (Elastic2D_CPML.py:11-91) and the
 * profile upload of SetADEPML2D (:392-528); the caller keeps the arrays. */
SW_API int sw2d_plan_create(const sw2d_desc* desc, sw_plan** plan);

/* Same for 3D: Elastic3D_SSG_CPML.py:9-122, Elastic3D_SSG_Tensor.py:9-130,
 * Elastic3D_SSG_SPML.py:8-138 and their SetADEPML3D. */
SW_API int sw3d_plan_create(const sw3d_desc* desc, sw_plan** plan);

/* Override the number of x planes one CTA streams in the 3D CPML passes
 * (the autotuner's knob; the plan picks a default from the grid and SM count). */
SW_API int sw_plan_set_tile(sw_plan* plan, int32_t x_chunk);

/* No reference counterpart (a self-check of this library's exact division).
 * Counts the finite float numerators x (all 2^32 bit patterns) for which the
 * kernels' quotient by `divisor` differs from IEEE division x/divisor: mode 0
 * the constant-spacing quotient (Markstein's correction with r = RN(1/d), its
 * scaled form below 2^-100), which a plan enables for a spacing only when
 * this count is zero; mode 1 the per-cell quotient (density, kappa) with its
 * scaled route for numerators below 2^-100; modes 2 and 3 the branch-free
 * forms of modes 0 and 1 that quotient groups holding numerators below
 * 2^-100 use, over the numerators of magnitude below 2^100 (mode 2 is also
 * checked before a plan enables a spacing; mode 3 takes divisors in
 * [2^-60, 2^60]).  Blocks on the stream; about a millisecond on a B200.
 * Allocates one 8-byte counter. */
SW_API int sw_check_division(float divisor, int32_t mode, uint64_t* mismatches, void* stream);

/* Block until the stream is idle and report a device-side failure recorded
 * by the plan's kernels since the previous status read (SW_ERR_TIMEOUT: a
 * bounded wait for TMA data, or a grid barrier of the 2D persistent run, gave
 * up); a failure is reported once and then cleared, so a caller may retry.  No reference counterpart (the reference has no error
 * path); it is the status read the drivers' loops can add after run(). */
SW_API int sw_plan_status(sw_plan* plan, void* stream);

/* Describe the plan's execution path: info[0] current path of sw_step/sw_run
 * (0 register-queue two-pass kernels, 2D: two launches per step, 1 TMA-staged
 * two-pass kernels, 2 fused single-pass kernel, 3 2D persistent: sw_run is
 * one cooperative launch for all its steps, the phases separated by a
 * bounded grid barrier; opt-in, as the two launches per step replayed from
 * a CUDA graph are faster on B200 at every grid size measured; sw_step
 * keeps the two launches), [1] constant-divisor fast path verified, [2] staged
 * path available, [3] its grid, [4] its x-chunk length, [5] fused path set
 * up, [6] its grid, [7] its x-chunk length, [8] exact numerics (see
 * sw_plan_set_exact).  info must hold 9 int32. */
SW_API int sw_plan_info(sw_plan* plan, int32_t* info);

/* Choose the execution path (values of info[0]); the fused path allocates a
 * second buffer set of the wavefields on first use.  chunk_len > 0 sets the
 * x planes per work unit of the staged or fused path (the autotuner's knob).
 * Every path gives the same result bit for bit. */
SW_API int sw_plan_set_path(sw_plan* plan, int32_t path, int32_t chunk_len);

/* Free-surface mode: when on != 0 every step first applies the reference's
 * free-surface hook AEA, as a driver loop `AEA(); update_SSG_VS(i)` does
 * (Relay_wave.py:55-59).  2D: sxx = 0 on the x layer N (Elastic2D_CPML.py:
 * 122-125); inside sw_run the hooks of all but the first step are folded into
 * the previous stress pass.  3D: szz = 0 on the z layer N
 * (Elastic3D_SSG_Tensor.py:160-163), one small kernel at the start of each
 * step (the two-step fused path is not used in this mode).  Pair it with
 * AEA_init (lambda = 0 and rho halved on the first N layers), which the
 * Python classes apply to the material arrays.  The adjoint entry points
 * refuse plans in this mode (SW_ERR_UNSUPPORTED). */
SW_API int sw_plan_set_free_surface(sw_plan* plan, int32_t on);

/* Numeric mode of the staged path.  exact != 0: every operation rounds in
 * the reference's order with IEEE division (default; results bit-identical
 * to a CPU evaluation of the reference's expressions).  exact == 0: spacings
 * folded into the stencil coefficients, fused multiply-adds and approximate
 * division by the material (receiver traces within relative L2 1e-5 of the
 * exact mode, final wavefields within 1e-4).  The other paths are always
 * exact. */
SW_API int sw_plan_set_exact(sw_plan* plan, int32_t exact);

/* sizeof of the ABI structs as this library was compiled: which = 0
 * sw_pml_axis, 1 sw_receivers, 2 sw_source, 3 sw2d_desc, 4 sw3d_desc; -1 else.
 * Lets a binding check its struct layout without touching a GPU. */
SW_API int sw_abi_sizeof(int32_t which);

/* Release the plan's own scratch and graphs. */
SW_API int sw_plan_destroy(sw_plan* plan);

/* One time step `it`: the reference's update_SSG_VS(it) / update_SSG_SV(it) /
 * update_SSG(it) / update_SSG_SPML(it) (Elastic2D_CPML.py:128,203;
 * Elastic3D_SSG_CPML.py:144; Elastic3D_SSG_Tensor.py:166;
 * Elastic3D_SSG_SPML.py:160). */
SW_API int sw_step(sw_plan* plan, int32_t it, void* stream);

/* One time step with the source amplitude given by the caller instead of the
 * plan's wavelet: update_RSG(it, source) (Elastic2D_CPML.py:277). */
SW_API int sw_step_amp(sw_plan* plan, int32_t it, double amplitude, void* stream);

/* Steps it0 .. it0+nsteps-1 back to back, the reference driver loop
 * `for i in range(nt): obj.update_*(i)` (e.g. test2d_homegenous.py:55-56),
 * replayed from a cached CUDA graph when use_graph != 0. */
SW_API int sw_run(sw_plan* plan, int32_t it0, int32_t nsteps, int32_t use_graph, void* stream);

/* ---- batches of 2D shots (no reference counterpart) -------------------------
 * Many shots of uneven grid sizes (one sw2d_desc each, sharing scheme VS or
 * SV, dtype, order and nt_max; velocity receivers) stepped together: per time
 * step one launch of the velocity phase and one of the stress phase cover
 * every tile of every shot, and sw_batch_run replays the whole step sequence
 * from one cached CUDA graph.  It replaces a Python loop over the reference's
 * ElasticWAVE objects, each running `for i in range(nt): update_SSG_VS(i)`
 * (Elastic2D_CPML.py:128-200).  Each shot's result equals its own sw_run. */
typedef struct sw_batch sw_batch;
#define SW_BATCH_TILES 4 /* tile shapes the autotuner picks from (sw_batch_info) */
SW_API int sw2d_batch_create(const sw2d_desc* shots, int32_t nshots, sw_batch** batch);
/* Tile shape index 0..SW_BATCH_TILES-1: (x rows, z columns) 8x32, 4x32, 16x32, 4x64. */
SW_API int sw_batch_set_tile(sw_batch* batch, int32_t tile);
/* info[0] tile index, [1] SW_BATCH_TILES, [2] tiles per launch, [3] rows, [4] columns,
 * [5] shots.  info must hold 6 int32. */
SW_API int sw_batch_info(sw_batch* batch, int32_t* info);
SW_API int sw_batch_run(sw_batch* batch, int32_t it0, int32_t nsteps, int32_t use_graph, void* stream);
SW_API int sw_batch_destroy(sw_batch* batch);

/* ---- learned thin absorbing layer, 2D (no reference counterpart) ------------
 * A network corrects the five fields of the outer SW_ABC_DEPTH cells of a 2D
 * VS solver after each time step; it runs on top of a thin CPML built by the
 * reference's SetADEPML2D (Elastic2D_CPML.py:392-528), which stays the
 * fallback.  One network per face (0 x-low, 1 x-high, 2 z-low, 3 z-high):
 * inputs are the fields / scale on the 3x3 stencil around the cell in the
 * face's frame plus a one-hot of the cell's depth; two tanh layers of
 * SW_ABC_HIDDEN; five outputs times oscale are added to the fields.  Parameter
 * block per face: W1[H][I] b1[H] W2[H][H] b2[H] W3[5][H] b3[5] (float32). */
#define SW_ABC_DEPTH 6
#define SW_ABC_INPUTS (45 + SW_ABC_DEPTH)
#define SW_ABC_HIDDEN 32
#define SW_ABC_PARAMS (SW_ABC_HIDDEN * SW_ABC_INPUTS + SW_ABC_HIDDEN + SW_ABC_HIDDEN * SW_ABC_HIDDEN + \
                       SW_ABC_HIDDEN + 5 * SW_ABC_HIDDEN + 5)
typedef struct sw_abc_desc {
  int32_t ncell;             /* layer cells                                     */
  const int32_t* cell;       /* device, linear index of each layer cell         */
  const int8_t* face;        /* device, its face 0..3                           */
  const int8_t* depth;       /* device, its distance to the face 0..DEPTH-1     */
  const float* params;       /* device, 4 x SW_ABC_PARAMS                       */
  float scale[5];            /* input scales of the fields vx vz sxx szz sxz    */
  float oscale[5];           /* output scales: field_q += y_q * oscale_q        */
  float* delta;              /* device scratch, ncell x 5                       */
} sw_abc_desc;
/* Add the network's corrections to the plan's fields (float32 2D plans). */
SW_API int sw2d_abc_correct(sw_plan* plan, const sw_abc_desc* abc, void* stream);
/* Network inputs of every layer cell from the plan's fields: x is ncell x SW_ABC_INPUTS. */
SW_API int sw2d_abc_features(sw_plan* plan, const sw_abc_desc* abc, float* x, void* stream);
/* Training: loss += mean over n samples of |net(x) - y|^2 (sum over the 5
 * outputs) and grad += its gradient with respect to one face's parameters. */
SW_API int sw_mlp_grad(const float* params, const float* x, const float* y, int64_t n, float* grad, float* loss,
                       void* stream);
/* y = net(x) for n samples of one face. */
SW_API int sw_mlp_forward(const float* params, const float* x, int64_t n, float* y, void* stream);
/* grad += sum over n samples of (d net(x_s) / d params)^T dy_s: the
 * parameter gradient for given output adjoints dy (n x 5). */
SW_API int sw_mlp_backward(const float* params, const float* x, const float* dy, int64_t n, float* grad,
                           void* stream);
/* Adjoint of one sw2d_abc_correct for training through the time loop.
 * fields: the uncorrected state (five (nx, nz) arrays packed back to back, as
 * the first five of a sw2d_record snapshot slot); adj: the five adjoint field
 * arrays, which hold the adjoint of the corrected state on entry and of the
 * uncorrected state on return; ybar (ncell x 5) receives the adjoint of the
 * network outputs (feed it with the layer's inputs to sw_mlp_backward). */
SW_API int sw2d_abc_adjoint(sw_plan* plan, const sw_abc_desc* abc, const float* fields, float* const* adj,
                            float* ybar, void* stream);

/* 3D layer: the same on the six faces of a SW3D_CPML_TENSOR solver; inputs
 * are the nine fields / scale at the cell and its two neighbours along the
 * face's inward normal plus the depth one-hot; nine outputs. */
#define SW_ABC3_INPUTS (27 + SW_ABC_DEPTH)
#define SW_ABC3_PARAMS (SW_ABC_HIDDEN * SW_ABC3_INPUTS + SW_ABC_HIDDEN + SW_ABC_HIDDEN * SW_ABC_HIDDEN + \
                        SW_ABC_HIDDEN + 9 * SW_ABC_HIDDEN + 9)
typedef struct sw_abc3_desc {
  int32_t ncell;
  const int32_t* cell;       /* device, linear index (i*ny + j)*nz + k          */
  const int8_t* face;        /* device, face 0..5 (x-low, x-high, y-low, ...)   */
  const int8_t* depth;       /* device, distance to the face 0..DEPTH-1         */
  const float* params;       /* device, 6 x SW_ABC3_PARAMS                      */
  float scale[9];            /* input scales: vx vy vz sxx syy szz sxy sxz syz  */
  float oscale[9];           /* output scales                                   */
  float* delta;              /* device scratch, ncell x 9                       */
} sw_abc3_desc;
SW_API int sw3d_abc_correct(sw_plan* plan, const sw_abc3_desc* abc, void* stream);
SW_API int sw3d_abc_features(sw_plan* plan, const sw_abc3_desc* abc, float* x, void* stream);
/* fields: nine (nx, ny, nz) arrays packed back to back (a sw3d_record slot's
 * first part); adj: the nine adjoint field arrays, updated in place. */
SW_API int sw3d_abc_adjoint(sw_plan* plan, const sw_abc3_desc* abc, const float* fields, float* const* adj,
                            float* ybar, void* stream);
SW_API int sw3d_mlp_grad(const float* params, const float* x, const float* y, int64_t n, float* grad, float* loss,
                         void* stream);
SW_API int sw3d_mlp_forward(const float* params, const float* x, int64_t n, float* y, void* stream);
SW_API int sw3d_mlp_backward(const float* params, const float* x, const float* dy, int64_t n, float* grad,
                             void* stream);

/* ---- 2D adjoint (no reference counterpart) --------------------------------
 * Hand-written discrete adjoint of the SW2D_SSG_VS or SW2D_SSG_SV time loop
 * (the plan's scheme) with a SW_SRC_MOMENT (or no) source and the scheme's
 * receivers (vz for VS, vx for SV; plans recording another field are
 * refused with SW_ERR_UNSUPPORTED), for gradients of a seismogram
 * misfit with respect to the material.  sw2d_record runs forward steps
 * it0..it0+nsteps-1 from the plan's current state and stores nsteps+1
 * snapshots of sw2d_snapshot_elems() elements each; sw2d_adjoint_run then
 * steps the adjoint state from it0+nsteps-1 down to it0 using them.  Together
 * they replace one checkpoint segment of the reference loop
 * (Elastic2D_CPML.py:128-200, :202-275) run backwards. */
typedef struct sw2d_adjoint_desc {
  void* field[5];            /* adjoint of vx vz sxx szz sxz, (nx, nz) each    */
  void* mem[2];              /* adjoint memory variables, layout of sw2d_desc.mem */
  void* tmp[4];              /* scratch, (nx, nz) each                          */
  void* grad[5];             /* per-cell sums, added to: G_vx (coefficient
                                dt/rho of vx), G_vz (dt/rho of vz, rho the
                                scheme's average), G_lpm (lambda+2mu at sxx),
                                G_lhx (lambda at sxx), G_mhz (mu at sxz); see
                                the Python wrapper for the chain to rho,
                                lambda, mu                                      */
  const void* residual;      /* (nt_max, nrec): d misfit / d data              */
} sw2d_adjoint_desc;

/* Elements (of the plan's dtype) in one snapshot slot. */
SW_API int sw2d_snapshot_elems(sw_plan* plan, int64_t* elems);
/* Forward steps with snapshots: snap holds (nsteps+1) slots. */
SW_API int sw2d_record(sw_plan* plan, int32_t it0, int32_t nsteps, void* snap, void* stream);
/* Adjoint steps it0+nsteps-1 .. it0 over the snapshots of sw2d_record(it0, nsteps). */
SW_API int sw2d_adjoint_run(sw_plan* plan, const sw2d_adjoint_desc* adj, int32_t it0, int32_t nsteps,
                            const void* snap, void* stream);

/* ---- 3D adjoint (no reference counterpart) --------------------------------
 * The same for the SW3D_CPML_TENSOR scheme (Elastic3D_SSG_Tensor.py:166-345)
 * and the SW3D_CPML_FORCE scheme (Elastic3D_SSG_CPML.py:144-309, whose point
 * force adds its rho term to grad[0] at the source cell), orders 1..4: sw3d_record runs forward steps it0..it0+nsteps-1 with the
 * exact register-queue kernels and stores nsteps+1 snapshots of
 * sw3d_snapshot_elems() elements; sw3d_adjoint_run steps the adjoint state
 * back over them. */
typedef struct sw3d_adjoint_desc {
  void* field[9];            /* adjoint of vx vy vz sxx syy szz sxy sxz syz    */
  void* mem[3];              /* adjoint memory variables, layout of sw3d_desc.mem */
  void* tmp[9];              /* scratch, (nx, ny, nz) each                      */
  void* grad[8];             /* per-cell sums, added to: G_vx (coefficient dt/rho
                                of vx), G_vy (dt/rho_y), G_vz (dt/rho_4), G_lpm,
                                G_lhx (normal stresses), G_xy, G_xz, G_yz (the
                                shear stresses' averaged mu)                    */
  const void* residual;      /* (nt_max, nrec): d misfit / d data              */
} sw3d_adjoint_desc;
SW_API int sw3d_snapshot_elems(sw_plan* plan, int64_t* elems);
SW_API int sw3d_record(sw_plan* plan, int32_t it0, int32_t nsteps, void* snap, void* stream);
SW_API int sw3d_adjoint_run(sw_plan* plan, const sw3d_adjoint_desc* adj, int32_t it0, int32_t nsteps,
                            const void* snap, void* stream);

/* Scan every wavefield for NaN/Inf; blocks on the stream.  *nonfinite is set
 * to the number of non-finite values found (0 when the state is finite);
 * returns SW_ERR_NONFINITE when it is non-zero. */
SW_API int sw_check_finite(sw_plan* plan, void* stream, int64_t* nonfinite);

/* No reference counterpart.  The scan of sw_check_finite over caller-named
 * device arrays (arrays[a] holds lengths[a] elements of dtype SW_F32 or
 * SW_F64), allocating no device memory: its counters live in a static device
 * array of SW_NOALLOC_MAX_ARRAYS 64-bit words inside this library, and
 * narrays above that limit is rejected with SW_ERR_ARG.  For hosts that may
 * not allocate at this point: device memory owned by another allocator (a
 * framework's memory pool), or a loop where cudaFree's device-wide
 * synchronisation would stall other streams; sw_check_finite allocates its
 * counter on first use and needs a plan.
 * counts[a] receives array a's NaN/Inf count; returns SW_ERR_NONFINITE when
 * any is non-zero.  Blocks on the stream.  Each call zeroes the counters it
 * uses before its scan, so nothing must be zero on entry.  The first call on
 * each device (that device current) resolves the counters' address with
 * cudaGetSymbolAddress, and with lazy module loading (CUDA_MODULE_LOADING=LAZY,
 * the default) that first use may load this library's device code, which the
 * driver backs with device memory: make the first call on each device before
 * any stream capture and before any region where allocation is forbidden.  The counters are
 * shared by every caller on a device: calls that overlap in time on one device
 * (several host threads) race and return mixed counts, so serialise them. */
#define SW_NOALLOC_MAX_ARRAYS 64
SW_API int sw_count_nonfinite_noalloc(const void* const* arrays, const int64_t* lengths, int32_t narrays,
                                      int32_t dtype, void* stream, int64_t* counts);

/* ---- SEG-Y ingestion -------------------------------------------------------
 * Decode SEG-Y traces on the device, replacing the segyio trace reads of
 * ReadSegy.py:3-18 (read_segy).  traces: the file's bytes from the first trace
 * header on (after the 3600-byte header and any extended textual headers),
 * in device memory, 4-byte aligned: ntraces records of a 240-byte trace
 * header and nsamples big-endian samples in `format` (1 IBM float, 2 int32,
 * 3 int16, 5 IEEE float, 8 int8).  out: (ntraces, nsamples) float32; IBM
 * values are exact in double and rounded once to float.  srcx (optional,
 * ntraces int32): the SourceX header word (bytes 73-76) of each trace, which
 * read_segy groups shots by.  Enqueued on stream; nothing is allocated. */
SW_API int sw_segy_decode(const void* traces, int64_t ntraces, int32_t nsamples, int32_t format, float* out,
                          int32_t* srcx, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SEISWAVE_H */
