// Kernel set of one arithmetic mode.  Included by kernels_fast.cu and
// kernels_strict.cu with MPD_NS defined as the mode's namespace.
#include <algorithm>

#include "launch.h"
#include "tma.cuh"

namespace mpd {
namespace MPD_NS {

#include "kernels_unfused.cuh"
#include "kernels_fused.cuh"
#include "kernels_ensemble.cuh"
#include "kernels_adjoint.cuh"

// Corrective pass with its intermediates kept for the adjoint: the raw faces
// go to R, the limited faces to a.Un/Vn/Wn (copied from R and limited in place).
template <typename T>
void launch_pass_record(const Dims& d, const PassArgs<T>& a, T* RU, T* RV, T* RW, T* bup, T* bdn,
                        cudaStream_t s)
{
    dim3 g((d.nx + 31) / 32, (d.ny + 7) / 8, d.ns), b(32, 8);
    k_antidiff<T><<<g, b, 0, s>>>(d, a.c, a.Uo, a.Vo, a.Wo, a.Vadv, RU, RV, RW, a.pass, a.use_div,
                                  a.vv_fix);
    if (a.limiter) {
        if (a.wide)
            k_fct_beta<T, double><<<g, b, 0, s>>>(d, a.c, a.cn, RU, RV, RW, bup, bdn);
        else
            k_fct_beta<T, T><<<g, b, 0, s>>>(d, a.c, a.cn, RU, RV, RW, bup, bdn);
        // raw faces stay in R, the limited ones go to Un/Vn/Wn (every used face is written)
        k_fct_apply<T><<<g, b, 0, s>>>(d, bup, bdn, RU, RV, RW, a.Un, a.Vn, a.Wn);
        k_donor<T><<<g, b, 0, s>>>(d, a.c, a.Un, a.Vn, a.Wn, a.c_out, 1);
    } else {
        k_donor<T><<<g, b, 0, s>>>(d, a.c, RU, RV, RW, a.c_out, 1);
    }
}

template void launch_pass_record<float>(const Dims&, const PassArgs<float>&, float*, float*, float*,
                                        float*, float*, cudaStream_t);
template void launch_pass_record<double>(const Dims&, const PassArgs<double>&, double*, double*,
                                         double*, double*, double*, cudaStream_t);
template void launch_adj_pass<float>(const Dims&, const AdjPassArgs<float>&, cudaStream_t);
template void launch_adj_pass<double>(const Dims&, const AdjPassArgs<double>&, cudaStream_t);

template int launch_ens_pass<float>(int, float*, const EnsInst*, const EnsItem*, int, int,
                                    const EnsPass&, int, int, int, cudaStream_t);
template int launch_ens_donor<float>(int, float*, const EnsInst*, const EnsItem*, int, int,
                                     const EnsPass&, cudaStream_t);
template int launch_ens_march<float>(float*, const EnsInst*, const EnsItem*, int, const EnsPass&,
                                     int, int, cudaStream_t);

namespace {
constexpr int kBX = 32, kBY = 8;
inline dim3 full_grid(const Dims& d) { return dim3((d.nx + kBX - 1) / kBX, (d.ny + kBY - 1) / kBY, d.ns); }
}  // namespace

// z-chunk depth of a vector march over `planes` planes with `cols` CTAs per
// plane and `per_sm` CTAs resident on each of the 148 SMs: the depth that
// minimises whole waves x (planes per CTA + one plane of setup loads), so
// that no nearly empty last wave costs a full CTA's march.
inline int vector_march_depth(long long cols, int planes, int per_sm)
{
    const long long slots = 148LL * std::max(per_sm, 1);
    int best_d = planes;
    long long best = -1;
    for (int dep = planes; dep >= std::min(planes, 4); dep--) {
        const long long nch = (planes + dep - 1) / dep;
        const long long waves = (cols * nch + slots - 1) / slots;
        const long long t = waves * (dep + 1);
        if (best < 0 || t < best) { best = t; best_d = dep; }
    }
    return best_d;
}

// CTAs of `kern` (256 threads, no dynamic shared memory) resident per SM.
template <typename K> int resident_per_sm(K kern)
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, 256, 0) != cudaSuccess || n < 1) n = 1;
    return n;
}

template <typename T>
void launch_courant(const Dims& d, const T* dx, const T* dy, const T* ds, T dt, const T* u0,
                    const T* u1, const T* v0, const T* v1, const T* w0, const T* w1, T* U,
                    T* V, T* W, int k0, int nk, cudaStream_t s)
{
    if (nk <= 0) return;
    // vector march (k_courant_v): 32 x 8 threads of 16 bytes each, z chunks in whole waves
    constexpr int N = 16 / (int)sizeof(T);
    const bool one = u0 == u1 && v0 == v1 && w0 == w1;
    auto kern = one ? k_courant_v<T, true> : k_courant_v<T, false>;
    static const int per_sm[2] = {resident_per_sm(k_courant_v<T, false>),
                                  resident_per_sm(k_courant_v<T, true>)};
    const int gx = (d.nx + 32 * N - 1) / (32 * N), gy = (d.ny + 7) / 8;
    const int depth = vector_march_depth((long long)gx * gy, nk, per_sm[one]);
    dim3 g(gx, gy, (nk + depth - 1) / depth);
    kern<<<g, dim3(32, 8), 0, s>>>(d, dx, dy, ds, dt, u0, u1, v0, v1, w0, w1, U, V, W, depth, k0,
                                   k0 + nk);
}

template <typename T>
void launch_donor(const Dims& d, const T* c0, const T* U, const T* V, const T* W, T* c1,
                  int copy_shell, int zb, int ze, cudaStream_t s)
{
    if (copy_shell) {
        k_donor<T><<<full_grid(d), dim3(kBX, kBY), 0, s>>>(d, c0, U, V, W, c1, copy_shell);
        return;
    }
    if (zb <= 0) zb = 1;
    if (ze <= 0) ze = d.ns - 1;
    if (ze <= zb) return;
    // vector march: 32 x 8 threads of 16 bytes each, z chunks in whole waves
    constexpr int N = 16 / (int)sizeof(T);
    static const int per_sm = resident_per_sm(k_donor_v<T>);
    const int gx = (int)((d.px / N + 31) / 32), gy = (d.ny - 2 + 7) / 8;
    const int depth = vector_march_depth((long long)gx * gy, ze - zb, per_sm);
    dim3 g(gx, gy, (ze - zb + depth - 1) / depth);
    k_donor_v<T><<<g, dim3(32, 8), 0, s>>>(d, c0, U, V, W, c1, depth, zb, ze);
}

// Advective faces and pass 0 of planes [zb, ze) in one z march (k_courant_donor_v).
template <typename T>
void launch_courant_donor(const Dims& d, const T* dx, const T* dy, const T* ds, T dt,
                          const T* u0, const T* u1, const T* v0, const T* v1, const T* w0,
                          const T* w1, const T* c0, T* U, T* V, T* W, T* c1, int zb, int ze,
                          cudaStream_t s)
{
    if (zb <= 0) zb = 1;
    if (ze <= 0) ze = d.ns - 1;
    if (ze <= zb) return;
    constexpr int N = 16 / (int)sizeof(T);
    const bool one = u0 == u1 && v0 == v1 && w0 == w1;
    auto kern = one ? k_courant_donor_v<T, true> : k_courant_donor_v<T, false>;
    static const int per_sm[2] = {resident_per_sm(k_courant_donor_v<T, false>),
                                  resident_per_sm(k_courant_donor_v<T, true>)};
    const int gx = (int)((d.px / N + 31) / 32), gy = (d.ny - 2 + 7) / 8;
    const int depth = vector_march_depth((long long)gx * gy, ze - zb, per_sm[one]);
    dim3 g(gx, gy, (ze - zb + depth - 1) / depth);
    kern<<<g, dim3(32, 8), 0, s>>>(d, dx, dy, ds, dt, u0, u1, v0, v1, w0, w1, c0, U, V, W, c1, depth,
                                   zb, ze);
}

template <typename T>
int launch_pass_unfused(const Dims& d, const PassArgs<T>& a, T* bup, T* bdn, cudaStream_t s)
{
    dim3 g = full_grid(d), b(kBX, kBY);
    k_antidiff<T><<<g, b, 0, s>>>(d, a.c, a.Uo, a.Vo, a.Wo, a.Vadv, a.Un, a.Vn, a.Wn, a.pass,
                                  a.use_div, a.vv_fix);
    int n = 1;
    if (a.limiter) {
        if (a.wide)
            k_fct_beta<T, double><<<g, b, 0, s>>>(d, a.c, a.cn, a.Un, a.Vn, a.Wn, bup, bdn);
        else
            k_fct_beta<T, T><<<g, b, 0, s>>>(d, a.c, a.cn, a.Un, a.Vn, a.Wn, bup, bdn);
        k_fct_apply<T><<<g, b, 0, s>>>(d, bup, bdn, a.Un, a.Vn, a.Wn, a.Un, a.Vn, a.Wn);
        n += 2;
    }
    k_donor<T><<<g, b, 0, s>>>(d, a.c, a.Un, a.Vn, a.Wn, a.c_out, 1);
    return n + 1;
}

#define MPD_INSTANTIATE(T)                                                                  \
    template void launch_courant<T>(const Dims&, const T*, const T*, const T*, T, const T*, \
                                    const T*, const T*, const T*, const T*, const T*, T*,   \
                                    T*, T*, int, int, cudaStream_t);                        \
    template void launch_donor<T>(const Dims&, const T*, const T*, const T*, const T*, T*,  \
                                  int, int, int, cudaStream_t);                             \
    template void launch_courant_donor<T>(const Dims&, const T*, const T*, const T*, T,     \
                                          const T*, const T*, const T*, const T*, const T*, \
                                          const T*, const T*, T*, T*, T*, T*, int, int,     \
                                          cudaStream_t);                                    \
    template int launch_pass_unfused<T>(const Dims&, const PassArgs<T>&, T*, T*,            \
                                        cudaStream_t);                                      \
    template int launch_pass_fused<T>(const Dims&, const PassArgs<T>&, cudaStream_t);
MPD_INSTANTIATE(float)
MPD_INSTANTIATE(double)
#undef MPD_INSTANTIATE

}  // namespace MPD_NS
}  // namespace mpd
