// The reference's INTEGER build as smolar_i64().
//
// Compiled with -DINTEGER the reference runs its whole step on `long`
// (smolar.h:14-16) with ONE 4, HALF 2, QUAT 1 and MINVAL 1
// (core/include/smolar_int.h:27-31): an exact-arithmetic mode whose results
// depend on nothing but the order of the integer operations.  Here the
// per-routine kernels of kernels_unfused.cuh run on long long: every formula
// keeps the reference's evaluation order and C's truncating division, so the
// results equal the reference's bit for bit while no value leaves the 64-bit
// range (past it the reference's behaviour is undefined).  Where the
// reference would divide by zero and trap (c_hi + c_lo + MINVAL is 0 once a
// field turns negative; a zero dx, dy or ds), the kernels record it and the
// call fails with MPDATA_ERR_INT_DIV0, leaving the caller's arrays untouched.
//
// The step is core/src/smolar.c:33-63 on two device levels that mirror the
// caller's arrays: pass 0 writes c1 from c0, every corrective pass writes the
// other level from the newest one with faces computed Jacobi-style from the
// previous pass's (pvelocity.c:22-36), the shell copied along (bndcpy,
// smolar.c:5-31).  Both levels go back, and the two pointers trade places iff
// order is even (smolar.c:58).  The mode has no limiter, as the reference.
#include <cuda_runtime.h>

#include <mutex>

#include "launch.h"
#include "mpdata_b200.h"
#include "solver.h"

namespace mpd {
namespace i64 {
#include "kernels_unfused.cuh"
}  // namespace i64
}  // namespace mpd

static_assert(sizeof(long) == sizeof(long long), "the reference's long is 64-bit here");

namespace {

using T = long long;

// The zero-divisor flag lives once per process: calls take turns.
std::mutex g_mutex;
cudaStream_t g_stream = nullptr;

struct Arena {
    T* p = nullptr;
    ~Arena()
    {
        if (p) cudaFree(p);
    }
};

#define I64_TRY(expr)                                                                       \
    do {                                                                                    \
        cudaError_t e_ = (expr);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return mpd::fail(MPDATA_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(e_)); \
    } while (0)

int step_i64(int nx, int ny, int ns, const T* dx, const T* dy, const T* ds, T dt,
             const T* const vel[6], T* c0, T* c1, int order)
{
    mpd::Dims d;
    d.nx = nx;
    d.ny = ny;
    d.ns = ns;
    d.px = (nx + 31) / 32 * 32;  // rows start 256-byte aligned
    d.pp = d.px * ny;
    const size_t n = (size_t)d.pp * ns;

    // distinct velocity arrays (drivers pass each time level twice, ring2d/test.c:47-49)
    int slot[6], nvel = 0;
    for (int a = 0; a < 6; a++) {
        slot[a] = -1;
        for (int b = 0; b < a; b++)
            if (vel[b] == vel[a]) slot[a] = slot[b];
        if (slot[a] < 0) slot[a] = nvel++;
    }
    // arena: levels A, B; face sets 0 (advective), 1, 2; velocities; dx, dy, ds
    const size_t n_elems = (2 + 9 + (size_t)nvel) * n + (size_t)nx + ny + ns;
    Arena ar;
    I64_TRY(cudaMalloc(&ar.p, n_elems * sizeof(T)));
    T* A = ar.p;
    T* B = A + n;
    T* F[3][3];
    for (int s = 0; s < 3; s++)
        for (int x = 0; x < 3; x++) F[s][x] = B + n + (size_t)(3 * s + x) * n;
    T* V0 = F[2][2] + n;
    T* ddx = V0 + (size_t)nvel * n;
    T* ddy = ddx + nx;
    T* dds = ddy + ny;
    cudaStream_t s = g_stream;

    // unused face entries read as 0, as in the reference's fresh buffers
    I64_TRY(cudaMemsetAsync(F[0][0], 0, 9 * n * sizeof(T), s));
    const size_t row = (size_t)nx * sizeof(T), pitch = (size_t)d.px * sizeof(T);
    const size_t rows = (size_t)ny * ns;
    I64_TRY(cudaMemcpy2DAsync(A, pitch, c0, row, row, rows, cudaMemcpyHostToDevice, s));
    for (int a = 0; a < 6; a++) {
        bool first = true;
        for (int b = 0; b < a; b++) first = first && slot[b] != slot[a];
        if (first)
            I64_TRY(cudaMemcpy2DAsync(V0 + (size_t)slot[a] * n, pitch, vel[a], row, row, rows,
                                      cudaMemcpyHostToDevice, s));
    }
    I64_TRY(cudaMemcpyAsync(ddx, dx, nx * sizeof(T), cudaMemcpyHostToDevice, s));
    I64_TRY(cudaMemcpyAsync(ddy, dy, ny * sizeof(T), cudaMemcpyHostToDevice, s));
    I64_TRY(cudaMemcpyAsync(dds, ds, ns * sizeof(T), cudaMemcpyHostToDevice, s));
    const int zero = 0;
    I64_TRY(cudaMemcpyToSymbolAsync(mpd::g_int_div_zero, &zero, sizeof(int), 0,
                                    cudaMemcpyHostToDevice, s));

    const dim3 g((nx + 31) / 32, (ny + 7) / 8, ns), b(32, 8);
    auto v = [&](int a) { return V0 + (size_t)slot[a] * n; };
    mpd::i64::k_courant<T><<<g, b, 0, s>>>(d, ddx, ddy, dds, dt, v(0), v(1), v(2), v(3), v(4),
                                            v(5), F[0][0], F[0][1], F[0][2], 0);
    // pass 0: donor cell with the advective faces, c0 -> c1 (the shell copied along)
    mpd::i64::k_donor<T><<<g, b, 0, s>>>(d, A, F[0][0], F[0][1], F[0][2], B, 1);
    for (int o = 1; o < order; o++) {
        T* cur = (o & 1) ? B : A;
        T* nxt = (o & 1) ? A : B;
        // faces of pass o: set 1 (odd o), set 2 (even o); pass 1 reads the advective set 0
        const int fn = (o & 1) ? 1 : 2;
        const int fo = (o == 1) ? 0 : 3 - fn;
        mpd::i64::k_antidiff<T><<<g, b, 0, s>>>(d, cur, F[fo][0], F[fo][1], F[fo][2], F[0][1],
                                                 F[fn][0], F[fn][1], F[fn][2], o, 1, 0);
        mpd::i64::k_donor<T><<<g, b, 0, s>>>(d, cur, F[fn][0], F[fn][1], F[fn][2], nxt, 1);
    }
    I64_TRY(cudaGetLastError());
    int div0 = 0;
    I64_TRY(cudaMemcpyFromSymbolAsync(&div0, mpd::g_int_div_zero, sizeof(int), 0,
                                      cudaMemcpyDeviceToHost, s));
    I64_TRY(cudaStreamSynchronize(s));
    if (div0)
        return mpd::fail(MPDATA_ERR_INT_DIV0,
                         "integer mode: a division by zero (the reference would trap)");
    I64_TRY(cudaMemcpy2DAsync(c0, row, A, pitch, row, rows, cudaMemcpyDeviceToHost, s));
    I64_TRY(cudaMemcpy2DAsync(c1, row, B, pitch, row, rows, cudaMemcpyDeviceToHost, s));
    I64_TRY(cudaStreamSynchronize(s));
    return 0;
}

}  // namespace

extern "C" int smolar_i64(int nx, int ny, int ns, long* dx, long* dy, long* ds, const long dt,
                          long* u0, long* u1, long* v0, long* v1, long* w0, long* w1, long** c0,
                          long** c1, int flow_type, int order)
{
    (void)flow_type;  // stored but never read by the reference (uu.c:111)
    if (nx < 3 || ny < 3 || ns < 3 || order < 0)
        return mpd::fail(MPDATA_ERR_ARG, "bad grid %dx%dx%d or order %d", nx, ny, ns, order);
    if (!dx || !dy || !ds || !u0 || !u1 || !v0 || !v1 || !w0 || !w1 || !c0 || !c1 || !*c0 || !*c1)
        return mpd::fail(MPDATA_ERR_ARG, "null pointer");
    if (order == 0) {  // no pass runs; the reference still exchanges the pointers
        long* t = *c0;
        *c0 = *c1;
        *c1 = t;
        return 0;
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_stream) {
        cudaError_t e = cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            g_stream = nullptr;
            return mpd::fail(MPDATA_ERR_CUDA, "stream: %s", cudaGetErrorString(e));
        }
    }
    const T* vel[6] = {reinterpret_cast<const T*>(u0), reinterpret_cast<const T*>(u1),
                       reinterpret_cast<const T*>(v0), reinterpret_cast<const T*>(v1),
                       reinterpret_cast<const T*>(w0), reinterpret_cast<const T*>(w1)};
    int rc = step_i64(nx, ny, ns, reinterpret_cast<const T*>(dx), reinterpret_cast<const T*>(dy),
                      reinterpret_cast<const T*>(ds), (T)dt, vel, reinterpret_cast<T*>(*c0),
                      reinterpret_cast<T*>(*c1), order);
    if (rc) return rc;
    if ((order & 1) == 0) {  // the newest level is in *c0's array
        long* t = *c0;
        *c0 = *c1;
        *c1 = t;
    }
    return 0;
}
