/* CPU oracle for the MPDATA transport step -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference solver's hot path (apc-llc/mpdata,
 * smolar() in core/src/smolar.c:33-63 and the kernels it calls), used by the
 * tests, smoke() and the bench's CPU-baseline leg as the checker.  The shipped
 * library never links or calls it.
 *
 * Parity pin: built with strict IEEE flags (no FMA contraction, no
 * fast-math), oracle_smolar_f32/_f64 reproduce the reference compiled with
 * the same flags bit for bit (tests/test_oracle_pin.py, against
 * oracle/_ref/ built from the reference sources, and tests/golden/ fixtures
 * generated from it).  The nonoscillatory limiter has no counterpart in the
 * reference: its parity is unpinned (checked by property tests only).
 *
 * Layout: every array is a full nx*ny*ns grid, x fastest,
 * a[(k*ny + j)*nx + i].  Face arrays use the same shape; the face stored at
 * (i,j,k) is the one on the high side of cell (i,j,k) along its axis:
 *   U[k][j][i]  between cells i and i+1   (used: i 0..nx-2, j,k interior)
 *   V[k][j][i]  between cells j and j+1   (used: j 0..ny-2, i,k interior)
 *   W[k][j][i]  between cells k and k+1   (used: k 0..ns-2, i,j interior)
 * Entries outside the used ranges are never read and are left at zero.
 */
#pragma once
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_opts {
    int limiter;   /* 1: nonoscillatory (FCT) limiting of every corrective pass */
    int vv_fix;    /* 0: y-face column i=1 follows the reference's buffer rule
                          (0 on odd corrective passes, advective face on even);
                      1: that column is computed, out-of-grid x-faces read as 0 */
    int div_mode;  /* 0: divergent-flow term as the reference codes it; 1: off */
    int wide_beta; /* 1: limiter ratios evaluated in double (FP32-storage form) */
} oracle_opts;

/* Advective face Courant numbers from two time levels of cell velocities
 * (reference uu.c:104-141, vv.c:109-152, ww.c:115-158). */
void oracle_courant_f32(int nx, int ny, int ns, const float* dx, const float* dy,
                        const float* ds, float dt, const float* u0, const float* u1,
                        const float* v0, const float* v1, const float* w0,
                        const float* w1, float* U, float* V, float* W);
void oracle_courant_f64(int nx, int ny, int ns, const double* dx, const double* dy,
                        const double* ds, double dt, const double* u0, const double* u1,
                        const double* v0, const double* v1, const double* w0,
                        const double* w1, double* U, double* V, double* W);

/* One full step from given advective faces.  c0 is the input field, c1
 * receives the result; both are full grids and are never swapped here.
 * If inter is non-NULL it receives the field before the last pass (what the
 * reference leaves behind in *c0). */
int oracle_step_faces_f32(int nx, int ny, int ns, const float* U, const float* V,
                          const float* W, const float* c0, float* c1, float* inter,
                          int order, const oracle_opts* opts);
int oracle_step_faces_f64(int nx, int ny, int ns, const double* U, const double* V,
                          const double* W, const double* c0, double* c1, double* inter,
                          int order, const oracle_opts* opts);

/* The reference's smolar() signature and pointer-swap behaviour
 * (smolar.h:45-48, smolar.c:58), plus an options pointer (NULL = reference). */
int oracle_smolar_f32(int nx, int ny, int ns, float* dx, float* dy, float* ds,
                      const float dt, float* u0, float* u1, float* v0, float* v1,
                      float* w0, float* w1, float** c0, float** c1, int flow_type,
                      int order, const oracle_opts* opts);
int oracle_smolar_f64(int nx, int ny, int ns, double* dx, double* dy, double* ds,
                      const double dt, double* u0, double* u1, double* v0, double* v1,
                      double* w0, double* w1, double** c0, double** c1, int flow_type,
                      int order, const oracle_opts* opts);

/* Single pieces, for kernel-level checks. */
void oracle_antidiff_f32(int nx, int ny, int ns, const float* c, const float* Uo,
                         const float* Vo, const float* Wo, const float* Vadv, int pass,
                         float* Un, float* Vn, float* Wn, const oracle_opts* opts);
void oracle_antidiff_f64(int nx, int ny, int ns, const double* c, const double* Uo,
                         const double* Vo, const double* Wo, const double* Vadv, int pass,
                         double* Un, double* Vn, double* Wn, const oracle_opts* opts);
void oracle_donor_f32(int nx, int ny, int ns, const float* c0, const float* U,
                      const float* V, const float* W, float* c1);
void oracle_donor_f64(int nx, int ny, int ns, const double* c0, const double* U,
                      const double* V, const double* W, double* c1);

/* Compensated (Neumaier) sum of the interior cells, in double. */
double oracle_mass_f32(int nx, int ny, int ns, const float* c);
double oracle_mass_f64(int nx, int ny, int ns, const double* c);

/* The reference's INTEGER build (smolar.h:14-16: real = long; ONE 4, HALF 2,
 * QUAT 1, MINVAL 1, core/include/smolar_int.h:27-31).  Same functions, C's
 * truncating division; oracle_smolar_i64 returns -2 where the reference would
 * divide by zero (and trap), -1 for the limiter (the mode has none). */
void oracle_courant_i64(int nx, int ny, int ns, const long* dx, const long* dy,
                        const long* ds, long dt, const long* u0, const long* u1,
                        const long* v0, const long* v1, const long* w0, const long* w1,
                        long* U, long* V, long* W);
int oracle_step_faces_i64(int nx, int ny, int ns, const long* U, const long* V,
                          const long* W, const long* c0, long* c1, long* inter, int order,
                          const oracle_opts* opts);
int oracle_smolar_i64(int nx, int ny, int ns, long* dx, long* dy, long* ds, const long dt,
                      long* u0, long* u1, long* v0, long* v1, long* w0, long* w1,
                      long** c0, long** c1, int flow_type, int order,
                      const oracle_opts* opts);
void oracle_antidiff_i64(int nx, int ny, int ns, const long* c, const long* Uo,
                         const long* Vo, const long* Wo, const long* Vadv, int pass,
                         long* Un, long* Vn, long* Wn, const oracle_opts* opts);
void oracle_donor_i64(int nx, int ny, int ns, const long* c0, const long* U, const long* V,
                      const long* W, long* c1);
double oracle_mass_i64(int nx, int ny, int ns, const long* c);

#ifdef __cplusplus
}
#endif
