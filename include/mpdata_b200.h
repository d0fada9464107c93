/* mpdata_b200 -- MPDATA transport step on NVIDIA B200 (sm_100a).
 *
 * C ABI.  Plain pointers and sizes only.  Two groups of entry points:
 *
 *  1. Drop-in replacements for the reference library's public API
 *     (apc-llc/mpdata smolar.h).  Same names, argument meaning, host-memory
 *     arrays and pointer-swap behaviour; `real` is float, as in the
 *     reference's default build (CMakeLists.txt:5 adds -DSINGLE).  The
 *     double-precision build of the reference corresponds to the *_f64
 *     twins.  Each call stages its inputs to the GPU and the results back.
 *
 *  2. A device-resident handle API (mpdata_*) for stepping without host
 *     round trips: fields stay in HBM between steps, advective faces are
 *     computed once per velocity update, and every step is a fixed sequence
 *     of kernel launches on the handle's stream.
 *
 * Memory layout of every full-grid array (both groups): nx*ny*ns elements,
 * x fastest, a[(k*ny + j)*nx + i]; the outer one-cell shell is the fixed
 * boundary and only cells 1..n-2 of each axis are updated
 * (reference core/src/smolar_pass.c:30-34, core/src/smolar.c:5-31).
 *
 * Return values: 0 on success, a negative MPDATA_ERR_* code otherwise; the
 * text of the last error on the calling thread is in mpdata_last_error().
 * (The reference always returns 0, core/src/smolar.c:62.)
 */
#ifndef MPDATA_B200_H
#define MPDATA_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Flow-type values accepted (and, as in the reference, not used). smolar.h:3-4 */
#define SOLENOIDAL 0
#define DIVERGENT 1

/* msmolar execution modes (accepted and ignored, as in the reference). smolar.h:53-63 */
#define MSMOLAR_SERIAL 0
#define MSMOLAR_PTHREADS 1
#define MSMOLAR_OPENMP 2

#define MPDATA_OK 0
#define MPDATA_ERR_ARG (-1)      /* bad dimensions, order, pointer or option */
#define MPDATA_ERR_CUDA (-2)     /* a CUDA runtime call failed */
#define MPDATA_ERR_NOMEM (-3)    /* device or host allocation failed */
#define MPDATA_ERR_COURANT (-4)  /* |face Courant number| > 1 (when checking is on) */
#define MPDATA_ERR_STATE (-5)    /* call out of order (e.g. step before set_field) */
#define MPDATA_ERR_INT_DIV0 (-6) /* integer mode: a division by zero (the reference traps) */

/* ---- 1. Reference-compatible entry points --------------------------------
 *
 * One MPDATA step: `order` passes (1 = donor cell only, each further pass an
 * antidiffusive correction).  On return *c1 points to the newest field and
 * *c0 to the field before the last pass; the two pointers are exchanged iff
 * `order` is even, and both buffers are written (reference
 * core/src/smolar.c:44-58).  dx has nx entries (0..nx-2 used), dy ny, ds ns.
 * u0/u1 (v, w alike) are the cell velocities at the previous and current time
 * level; the same array may be passed twice.
 *
 * Replaces smolar() declared at reference smolar.h:45-48. */
int smolar(int nx, int ny, int ns, float* dx, float* dy, float* ds, const float dt,
           float* u0, float* u1, float* v0, float* v1, float* w0, float* w1,
           float** c0, float** c1, int flow_type, int order);

/* Double-precision twin: the reference's smolar() built with -DDOUBLE
 * (smolar.h:10-12). */
int smolar_f64(int nx, int ny, int ns, double* dx, double* dy, double* ds,
               const double dt, double* u0, double* u1, double* v0, double* v1,
               double* w0, double* w1, double** c0, double** c1, int flow_type,
               int order);

/* Integer twin: the reference's smolar() built with -DINTEGER (real = long,
 * smolar.h:14-16; ONE 4, HALF 2, QUAT 1, MINVAL 1, smolar_int.h:27-31), an
 * exact-arithmetic mode.  Results equal that build's bit for bit while no
 * value overflows 64 bits.  Where the reference would divide by zero (and
 * trap) the call returns MPDATA_ERR_INT_DIV0 and leaves *c0, *c1 untouched.
 * No limiter, no options; calls from several threads take turns. */
int smolar_i64(int nx, int ny, int ns, long* dx, long* dy, long* ds, const long dt,
               long* u0, long* u1, long* v0, long* v1, long* w0, long* w1, long** c0,
               long** c1, int flow_type, int order);

/* Decomposed step over an sx*sy*ss block grid.  *desc is created on the
 * first call (pass a NULL-initialised void*), holds the per-block device
 * state between calls and is released by msmolar_free().  Every step
 * exchanges block halos deep enough for all `order` passes, so the result
 * equals smolar() on the whole grid (the reference's intent; its own 1-cell
 * halo does not achieve that).  The caller's *c0 and *c1 pointers are exchanged
 * the way smolar() exchanges them, and the caller's arrays are brought up to
 * date only by msmolar_gather().  flow_type and mode are ignored.
 *
 * Replaces msmolar() declared at reference smolar.h:95-99. */
int msmolar(void** desc, int nx, int ny, int ns, float* dx, float* dy, float* ds,
            const float dt, float* u0, float* u1, float* v0, float* v1, float* w0,
            float* w1, float** c0, float** c1, int flow_type, int order, int sx, int sy,
            int ss, int mode);

/* Copy the decomposed state's newest field into *c1 (and the field before
 * the last pass into *c0).  Replaces msmolar_gather() declared at reference
 * smolar.h:132-136. */
int msmolar_gather(void** desc, int nx, int ny, int ns, float* dx, float* dy, float* ds,
                   const float dt, float* u0, float* u1, float* v0, float* v1,
                   float* w0, float* w1, float** c0, float** c1, int flow_type,
                   int order, int sx, int sy, int ss, int mode);

/* Release the state created by msmolar() and set *desc to NULL.  No reference
 * counterpart (the reference never frees it, core/src/msmolar.c:25-32). */
int msmolar_free(void** desc);

/* Text of the last error raised on the calling thread ("" if none). */
const char* mpdata_last_error(void);

struct mpdata_options;
/* Options used by smolar(), smolar_f64() and msmolar() on the calling thread
 * (NULL restores the defaults: reference behaviour, fused kernels).  Each
 * thread starts from the environment variable MPDATA_B200_OPTIONS, a
 * comma-separated list of limiter, precision_form, strict, unfused, single,
 * pair, vv_fix, div_off, approx_div, check_courant, so programs written against the
 * reference API can select options without code changes.  No reference
 * counterpart: the reference has no run-time options. */
int mpdata_set_default_options(const struct mpdata_options* opts);

/* smolar() / smolar_f64() on the calling thread: z planes per chunk of the
 * pipelined host step (0: automatic, the default; < 0: no pipelining).  The
 * pipelined step overlaps the uploads of the velocities and the field, the
 * kernels and the downloads of both outputs chunk by chunk (with pinned host
 * memory all copies are asynchronous); its results are the same bits as the
 * unpipelined step.  Not with kernel=1 or check_courant (those step whole).
 * No reference counterpart. */
int mpdata_set_pipeline(int chunk_planes);

/* ---- 2. Device-resident handle API ---------------------------------------- */

typedef struct mpdata_solver* mpdata_handle;

#define MPDATA_F32 0
#define MPDATA_F64 1

/* Where a pointer argument lives.  A DEVICE array is read or written by a
 * copy queued on the handle's stream: the caller orders the work that makes
 * or reuses it with that stream (mpdata_set_stream to share one stream, or
 * synchronise both sides). */
#define MPDATA_HOST 0
#define MPDATA_DEVICE 1
/* Host memory (pinned: mpdata_host_alloc) written by a copy that is only
 * queued: mpdata_get_planes() returns a ticket for mpdata_wait(). */
#define MPDATA_HOST_ASYNC 2
/* mpdata_set_velocity only: device arrays the handle reads in place instead
 * of copying them, until the next mpdata_step has run on the handle's stream
 * (the caller leaves them unchanged until then).  Taken in place when they
 * have the handle's row pitch (nx a multiple of 32) and 16-byte alignment,
 * copied as MPDATA_DEVICE otherwise. */
#define MPDATA_DEVICE_BORROW 3

/* Divergent-flow term of the antidiffusive velocity. */
#define MPDATA_DIV_REFERENCE 0 /* as the reference codes it (uu.c:81-84, vv.c:85-89, ww.c:88-92) */
#define MPDATA_DIV_OFF 1

typedef struct mpdata_options {
    int limiter;        /* 1: nonoscillatory (FCT) limiter on every corrective pass */
    int precision_form; /* 1 (F32 only): limiter ratios in FP64 (FP32 storage form) */
    int div_mode;       /* MPDATA_DIV_* */
    int vv_fix;         /* 1: compute the y-face column i=1 the reference leaves
                           unwritten (vv.c:81-82) instead of its buffer rule */
    int strict;         /* 1: no FMA contraction; bit-identical to a strict-IEEE
                           CPU build of the reference arithmetic */
    int kernel;         /* 0: fused per-pass kernels, the faster of the two forms
                           below for the options (default); 1: one kernel per
                           reference function (slower; cross-check path);
                           2: fused, one cell per thread; 3: fused, two cells per
                           thread (F32 without strict) */
    int check_courant;  /* 1: reject advective faces with |Courant| > 1 */
    int approx_div;     /* 1 (F32, fused kernels, not strict): the ratios of the
                           antidiffusive velocity and of the limiter use the
                           hardware reciprocal (<= 2 ulp) instead of IEEE division */
} mpdata_options;

/* Fill *o with the defaults (all zero: reference behaviour, fused kernels). */
void mpdata_default_options(mpdata_options* o);

int mpdata_create(mpdata_handle* h, int nx, int ny, int ns, int dtype, int order,
                  const mpdata_options* opts);
int mpdata_destroy(mpdata_handle h);

/* Use the given cudaStream_t (NULL = the legacy default stream) for all work
 * of this handle.  The handle creates its own non-blocking stream otherwise. */
int mpdata_set_stream(mpdata_handle h, void* stream);

/* Velocities as in smolar() (six full-grid arrays of the handle's dtype plus
 * dx, dy, ds and dt); the advective faces are computed on the GPU, by the
 * next step's donor pass in the same kernel (at once when check_courant is
 * set or kernel = 1).  The arrays are copied into the handle's own buffers
 * in stream order: pageable host arrays may be reused when the call returns,
 * pinned host or device arrays once the handle's stream has passed the copy
 * (mpdata_sync).  `where` tells whether the pointers are host or device
 * memory; MPDATA_DEVICE_BORROW lends device arrays without the copy. */
int mpdata_set_velocity(mpdata_handle h, const void* dx, const void* dy, const void* ds,
                        double dt, const void* u0, const void* u1, const void* v0,
                        const void* v1, const void* w0, const void* w1, int where);

/* Advective face Courant numbers directly, each a full-grid array where the
 * entry (i,j,k) is the face on the high side of cell (i,j,k) along the axis:
 * U between cells i and i+1 (used for i 0..nx-2, j and k interior), V between
 * j and j+1 (j 0..ny-2), W between k and k+1 (k 0..ns-2). */
int mpdata_set_faces(mpdata_handle h, const void* U, const void* V, const void* W,
                     int where);

/* Concentration field (full grid, shell included). */
int mpdata_set_field(mpdata_handle h, const void* c, int where);
int mpdata_get_field(mpdata_handle h, void* c, int where);
/* The field before the last pass of the latest step (what smolar() leaves in *c0). */
int mpdata_get_previous(mpdata_handle h, void* c, int where);

/* z-planes [k0, k0+nk) of the newest field as dense nx*ny planes (halo
 * exchange of z-slab decompositions, output frames).  get: host copies
 * synchronise, device copies are queued on the handle's stream, and
 * MPDATA_HOST_ASYNC copies are queued too and return a ticket (>= 0): the
 * caller may step on and write out the planes after mpdata_wait(h, ticket),
 * so frame output overlaps the next steps.  set: the planes are written into
 * every field level (planes on the grid's own z boundary are shell). */
int mpdata_get_planes(mpdata_handle h, int k0, int nk, void* dst, int where);
int mpdata_set_planes(mpdata_handle h, int k0, int nk, const void* src, int where);

/* Wait until the MPDATA_HOST_ASYNC copy with this ticket has landed. */
int mpdata_wait(mpdata_handle h, int ticket);

/* Advance nsteps steps on the handle's stream (asynchronous). */
int mpdata_step(mpdata_handle h, int nsteps);

/* Wait for the handle's stream. */
int mpdata_sync(mpdata_handle h);

/* Interior mass in FP64 with compensated summation (synchronous). */
int mpdata_mass(mpdata_handle h, double* mass);

/* Minimum over the interior cells and the number of negative cells (synchronous). */
int mpdata_min(mpdata_handle h, double* minval, long long* nneg);

/* Kernel launches a single mpdata_step(h, 1) issues. */
int mpdata_launches_per_step(mpdata_handle h);

/* z-march depth of the fused kernels: each CTA marches a chunk of `depth`
 * interior planes (after a 2-3 plane warm-up that keeps results identical);
 * 0 = the whole column.  A default is chosen at creation from the grid size;
 * mpdata_autotune times the candidates (whole, 128, 64, 32, 16, 8) over
 * trial_steps steps on the handle's own field, keeps the fastest and puts
 * the field back as it was. */
int mpdata_set_march_depth(mpdata_handle h, int depth);
int mpdata_march_depth(mpdata_handle h);
int mpdata_autotune(mpdata_handle h, int trial_steps, int* depth, double* ms_per_step);

/* Per-pass kernel timing with CUDA events on the handle's stream (for the
 * roofline report).  While enabled, every mpdata_step records an event pair
 * around the donor pass and around each corrective pass.  mpdata_pass_times
 * synchronises and returns the accumulated milliseconds and launch counts
 * since the last reset: [0] donor pass, [1] corrective passes that also write
 * faces, [2] the last corrective pass. */
int mpdata_enable_pass_timing(mpdata_handle h, int on);
int mpdata_pass_times(mpdata_handle h, double ms[3], long long launches[3], int reset);

/* ---- Batched ensemble of independent 2D problems --------------------------
 *
 * No reference counterpart (the reference steps one grid per smolar() call).
 * n instances of uneven size nx[q] x ny[q] (each the 2D form: the reference's
 * nx x ny x 3 grid with w = 0, fixed one-cell shell), float storage, one
 * common order and option set.  Every pass covers all instances in one
 * launch; mpdata_ensemble_step replays a CUDA graph of nsteps steps (captured
 * on first use per step count).  2D arrays are ny x nx, x fastest; U is the
 * face between cells i and i+1, V between rows j and j+1 (as in
 * mpdata_set_faces). */
typedef struct mpdata_ensemble* mpdata_ensemble_handle;

int mpdata_ensemble_create(mpdata_ensemble_handle* e, int n, const int* nx, const int* ny,
                           int order, const struct mpdata_options* opts);
int mpdata_ensemble_destroy(mpdata_ensemble_handle e);
int mpdata_ensemble_set_stream(mpdata_ensemble_handle e, void* stream);
int mpdata_ensemble_set_faces(mpdata_ensemble_handle e, int q, const void* U, const void* V,
                              int where);
int mpdata_ensemble_set_field(mpdata_ensemble_handle e, int q, const void* c, int where);
int mpdata_ensemble_get_field(mpdata_ensemble_handle e, int q, void* c, int where);
/* nsteps steps of every instance, as one CUDA graph launch (asynchronous). */
int mpdata_ensemble_step(mpdata_ensemble_handle e, int nsteps);
/* The same steps as individual kernel launches (no graph). */
int mpdata_ensemble_step_direct(mpdata_ensemble_handle e, int nsteps);
int mpdata_ensemble_sync(mpdata_ensemble_handle e);
/* Time every tile-shape candidate over trial_steps steps on the ensemble
 * itself and keep the fastest (*chosen = its index, *ms_per_step = its time).
 * The trials advance the instances: set the fields again afterwards. */
int mpdata_ensemble_autotune(mpdata_ensemble_handle e, int trial_steps, int* chosen,
                             double* ms_per_step);
/* Force a candidate: tile shapes 0: 32x8, 1: 32x16, 2: 64x8 threads; 3: the
 * first corrective pass as a y-march (one warp per strip of 32 columns and 64
 * rows, no shared memory or barriers), the other passes with shape 1. */
int mpdata_ensemble_tile(mpdata_ensemble_handle e, int tile);

/* ---- Adjoint of a window of steps ------------------------------------------
 *
 * No reference counterpart.  Hand-written reverse mode of the full step
 * (donor pass, antidiffusive passes, limiter) with every branch frozen at its
 * forward choice (sign of each face value in |U|, the limiter's min
 * selections and the argmax/argmin of its bounds).  Steady faces; the
 * adjoint is taken with respect to the field.
 *
 * mpdata_adjoint_forward steps c0 through nsteps steps (cN receives the
 * result if non-NULL), storing a checkpoint every `checkpoint_every` steps;
 * mpdata_adjoint_backward maps the adjoint of the window's output (lamN) to
 * the adjoint of its input (lam0), recomputing each checkpoint segment.
 * Arrays as in mpdata_set_field (full grids, dense, host or device). */
typedef struct mpdata_adjoint* mpdata_adjoint_handle;

int mpdata_adjoint_create(mpdata_adjoint_handle* h, int nx, int ny, int ns, int dtype, int order,
                          const struct mpdata_options* opts, int checkpoint_every);
int mpdata_adjoint_destroy(mpdata_adjoint_handle h);
int mpdata_adjoint_set_stream(mpdata_adjoint_handle h, void* stream);
int mpdata_adjoint_set_faces(mpdata_adjoint_handle h, const void* U, const void* V,
                             const void* W, int where);
int mpdata_adjoint_forward(mpdata_adjoint_handle h, const void* c0, int nsteps, void* cN,
                           int where);
int mpdata_adjoint_backward(mpdata_adjoint_handle h, const void* lamN, void* lam0, int where);

/* ---- 3. Allocation-free step --------------------------------------------
 *
 * No counterpart in the reference.  One FP32 step (`order` passes, optional
 * limiter, reference arithmetic, default FMA contraction) from advective faces
 * U, V, W and the field c_in to c_out, all caller-owned DEVICE arrays in the
 * dense full-grid layout (faces as for mpdata_set_faces), queued on `stream`
 * (a cudaStream_t; NULL = legacy default stream).  For callers that cannot
 * allocate device memory while they run (inside stream capture, under a
 * fixed memory budget, inside a host framework that owns the allocator): it
 * calls no cudaMalloc/cudaFree and no allocating library routine.  Its
 * intermediate levels, pseudo-velocity faces and limiter ratios live in one
 * static device array of MPDATA_NOALLOC_MAX_FLOATS floats (32 MiB, held by
 * every GPU that loads the library until exit); grids needing more
 * (10 * nx*ny*ns floats, i.e. more than 838860 cells) are rejected with
 * MPDATA_ERR_ARG.  All calls share that array: calls that overlap on the GPU
 * race, so keep them on one stream.  The first call on each device looks up
 * the array's address (and may load the module): make it before any stream
 * capture.  c_out must not alias c_in. */
#define MPDATA_NOALLOC_MAX_FLOATS (8u << 20)
int mpdata_step_noalloc(int nx, int ny, int ns, int order, int limiter, const float* U,
                        const float* V, const float* W, const float* c_in, float* c_out,
                        void* stream);

/* Page-locked host memory for fast staging (cudaMallocHost / cudaFreeHost). */
/* Self-check of the two-cell pass's division (no counterpart in the
 * reference): n seeded random operand pairs of the ranges the pass divides,
 * the division it uses without the library's slow path against IEEE
 * round-to-nearest division; *mismatches = results that differ in any bit
 * (0 expected).  Runs on the current device. */
int mpdata_check_division(long long n, unsigned long long seed, long long* mismatches);

void* mpdata_host_alloc(size_t bytes);
void mpdata_host_free(void* p);

#ifdef __cplusplus
}
#endif

#endif /* MPDATA_B200_H */
