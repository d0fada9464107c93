// Host-side launchers of the MPDATA kernels.  kernels_all.cuh is compiled
// twice: namespace mpd::fast (nvcc's default FMA contraction) and
// mpd::strict (-fmad=false: bit-identical to a strict-IEEE CPU build of the
// reference arithmetic).  Both expose the same launcher set.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "common.cuh"

namespace mpd {

// TMA descriptors of the arrays a fused pass stages (host-side copies; the
// launcher passes them to the kernel by value).
struct PassMaps {
    const CUtensorMap* c;
    const CUtensorMap* cn;
    const CUtensorMap* uo;
    const CUtensorMap* vo;
    const CUtensorMap* wo;
};

// Box staged per plane by the fused kernels: 40 x 19 elements (x: two halo
// columns below, up to three columns of 16-byte alignment slack, 32 + 1
// above; y: two halo rows below, 16 + 1 above).
constexpr int kBoxX = 40, kBoxY = 19;

// Two-cells-per-thread fast pass (kernels_pair.cuh): CTAs of 32 x kPairCY
// cells staged as 40 x (kPairCY + 2) boxes (x: two columns below plus up to
// two of alignment slack, y: one row below and one above).  16 rows: two
// CTAs of 256 threads per SM (measured faster than one CTA of 32 rows).
#ifndef MPD_PAIR_CY
#define MPD_PAIR_CY 16
#endif
constexpr int kPairCY = MPD_PAIR_CY;
constexpr int kPairBoxX = 40, kPairBoxY = kPairCY + 2;

// Per-pass description for the corrective-pass launchers.
template <typename T> struct PassArgs {
    PassMaps maps;     // fused path: descriptors of c, cn, Uo, Vo, Wo
    PassMaps maps2;    // the same arrays with the two-cell pass's boxes
    int* err;          // device error word (bounded-wait timeouts); may be null
    const T* c;        // this pass's input field (level o)
    const T* cn;       // the step's input field (limiter bounds); may be null without limiter
    const T* Uo;       // previous pass's faces (advective on pass 1)
    const T* Vo;
    const T* Wo;
    const T* Vadv;     // advective y faces (column rule of vv.c:81-82)
    T* Un;             // this pass's (limited) faces
    T* Vn;
    T* Wn;
    T* c_out;          // level o+1
    int pass;          // o >= 1
    int use_div;       // divergent-flow term on
    int vv_fix;        // compute the y-face column i=1
    int limiter;       // FCT on
    int wide;          // FP64 limiter ratios (float storage only)
    int write_faces;   // the next pass reads Un/Vn/Wn
    int approx;        // fused FP32 path: hardware-reciprocal ratios (approx_div form)
    int zdepth;        // fused path: planes per CTA z chunk (0 = the whole range)
    int zbase, zend;   // fused path: update planes [zbase, zend) only (0, 0: all interior planes)
};

// Ensemble (batched 2D instances): per-instance descriptor with the element
// offsets of its arrays inside the ensemble's arena.
struct EnsInst {
    int nx, ny, px, pad;
    long long c[3];     // field levels
    long long f[3][2];  // face sets: [0] advective, [1..2] Jacobi ping-pong; [axis] U, V
};

// One work item: a tile of an instance, given by its first interior cell.
struct EnsItem {
    int inst, i0, j0, pad;
};

// Which levels / face sets a pass reads and writes (the same for every instance).
struct EnsPass {
    int in, out, cn;   // field levels
    int rs, ws;        // face sets read / written
    int pass, use_div, vv_fix, write_faces;
    int fuse_donor;    // pass 1 forms c^(1) from c^n itself (no pass-0 launch)
};

// Adjoint of one pass o of a step (kernels_adjoint.cuh).
template <typename T> struct AdjPassArgs {
    int pass, limiter, wide, use_div, vv_fix;
    int accum_F;                   // lFU.. hold a later pass's contributions (o < P-1)
    const T *c, *cn;               // level c_o, step input c_0
    const T *FU, *FV, *FW;         // faces of this pass's donor update (advective for o = 0)
    const T *RU, *RV, *RW;         // raw antidiffusive faces of pass o
    const T *bup, *bdn;            // limiter ratios of pass o
    const T *Uo, *Vo, *Wo;         // previous faces (the pattern's inputs)
    const T* lam_out;              // adjoint of c_{o+1}
    T* lam_in;                     // adjoint of c_o (written by the donor part; += for o = 0)
    T* lam_cn;                     // adjoint of c_0 (+=, limiter bounds)
    T *lFU, *lFV, *lFW;            // adjoint of this pass's donor faces (null for o = 0)
    T *lRU, *lRV, *lRW;            // adjoint of the raw faces (limiter only)
    T *lbup, *lbdn;                // adjoint of the ratios (+=)
    T *lUo, *lVo, *lWo;            // adjoint of the previous faces (+=; null if advective)
};

#define MPD_DECLARE_LAUNCHERS                                                              \
    template <typename T> void launch_adj_pass(const Dims& d, const AdjPassArgs<T>& a,      \
                                               cudaStream_t s);                            \
    /* Corrective pass keeping its intermediates: raw faces R, limited faces L (= R         \
       without limiter, may alias), ratios bup/bdn. */                                     \
    template <typename T>                                                                  \
    void launch_pass_record(const Dims& d, const PassArgs<T>& a, T* RU, T* RV, T* RW,       \
                            T* bup, T* bdn, cudaStream_t s);                               \
    template <typename T>                                                                  \
    int launch_ens_pass(int tile, T* arena, const EnsInst* insts, const EnsItem* items,    \
                        int nitems, int grid, const EnsPass& p, int limiter, int wide,     \
                        int approx, cudaStream_t s);                                       \
    template <typename T>                                                                  \
    int launch_ens_march(T* arena, const EnsInst* insts, const EnsItem* items, int nitems, \
                         const EnsPass& p, int limiter, int approx, cudaStream_t s);       \
    template <typename T>                                                                  \
    int launch_ens_donor(int tile, T* arena, const EnsInst* insts, const EnsItem* items,   \
                         int nitems, int grid, const EnsPass& p, cudaStream_t s);          \
    /* Faces of planes [k0, k0 + nk). */                                                   \
    template <typename T>                                                                  \
    void launch_courant(const Dims& d, const T* dx, const T* dy, const T* ds, T dt,        \
                        const T* u0, const T* u1, const T* v0, const T* v1, const T* w0,   \
                        const T* w1, T* U, T* V, T* W, int k0, int nk, cudaStream_t s);    \
    /* Pass 0 over interior planes [zb, ze) (0, 0: all); copy_shell: every plane. */       \
    template <typename T>                                                                  \
    void launch_donor(const Dims& d, const T* c0, const T* U, const T* V, const T* W,      \
                      T* c1, int copy_shell, int zb, int ze, cudaStream_t s);              \
    /* Faces of the interior rows of planes [zb, ze) and pass 0 there, one kernel. */      \
    template <typename T>                                                                  \
    void launch_courant_donor(const Dims& d, const T* dx, const T* dy, const T* ds, T dt,  \
                              const T* u0, const T* u1, const T* v0, const T* v1,          \
                              const T* w0, const T* w1, const T* c0, T* U, T* V, T* W,     \
                              T* c1, int zb, int ze, cudaStream_t s);                      \
    /* Corrective pass, one kernel per reference routine; bup/bdn scratch (limiter). */    \
    template <typename T>                                                                  \
    int launch_pass_unfused(const Dims& d, const PassArgs<T>& a, T* bup, T* bdn,           \
                            cudaStream_t s);                                               \
    /* Corrective pass as one fused kernel; returns launches issued. */                    \
    template <typename T>                                                                  \
    int launch_pass_fused(const Dims& d, const PassArgs<T>& a, cudaStream_t s);

namespace fast {
MPD_DECLARE_LAUNCHERS
/* Corrective pass, two cells per thread (FP32, regrouped arithmetic: fast mode only). */
int launch_pass_pair(const Dims& d, const PassArgs<float>& a, cudaStream_t s);
}
namespace strict { MPD_DECLARE_LAUNCHERS }

// Mode-independent utility kernels (reductions, fills), in solver.cu.
template <typename T> void launch_mass(const Dims& d, const T* c, double* partial, int nblk,
                                       double* out, cudaStream_t s);

}  // namespace mpd
