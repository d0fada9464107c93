// Host side of the C ABI: the device-resident solver handle and the
// reference-compatible smolar()/smolar_f64() entry points built on it.
//
// Step driver (reference core/src/smolar.c:33-63, re-designed for the GPU):
//   * three field buffers rotate so the step's input c^n stays intact for the
//     limiter bounds while passes ping-pong between the other two;
//   * the advective faces are computed once per velocity update (the
//     reference recomputes them on every call, smolar.c:40-42); the
//     pipelined host-array step behind smolar() forms them per call, fused
//     with pass 0 chunk by chunk, overlapping the uploads and downloads;
//   * pseudo-velocities are Jacobi-updated between two face sets
//     (pvelocity.c:22-36), the advective set staying untouched;
//   * the fixed boundary shell is written into all three buffers once, when
//     the field is set, and never changes afterwards (bndcpy, smolar.c:5-31,
//     only ever copies it forward).
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>

#include "launch.h"
#include "mpdata_b200.h"
#include "solver.h"

using mpd::Dims;

// ---------------------------------------------------------------------------
// errors
namespace {
thread_local std::string g_last_error;
}  // namespace

int mpd::fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

extern "C" const char* mpdata_last_error(void) { return g_last_error.c_str(); }

#define CUDA_TRY(expr)                                                                      \
    do {                                                                                    \
        cudaError_t e_ = (expr);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return mpd::fail(MPDATA_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(e_)); \
    } while (0)

// ---------------------------------------------------------------------------
// reductions (mode independent)
namespace mpd {
namespace {

constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 592;  // 4 x 148 SMs

// Neumaier two-sum accumulate.
__device__ __forceinline__ void neu_add(double& s, double& comp, double x)
{
    double t = s + x;
    comp += (fabs(s) >= fabs(x)) ? (s - t) + x : (x - t) + s;
    s = t;
}

// Merge the partial (S, C, M, N) in slot b of a 4 x kRedThreads shared
// array into slot a: Neumaier sum of the sums, compensations added, min,
// count.
__device__ __forceinline__ void stats_merge(double (*sh)[kRedThreads], int a, int b)
{
    neu_add(sh[0][a], sh[1][a], sh[0][b]);
    sh[1][a] += sh[1][b];
    sh[2][a] = sh[2][b] < sh[2][a] ? sh[2][b] : sh[2][a];
    sh[3][a] += sh[3][b];
}

// Fixed-order tree over the block's kRedThreads slots (deterministic); slot 0
// holds the result.
__device__ __forceinline__ void stats_tree(double (*sh)[kRedThreads])
{
    __syncthreads();
    for (int w = kRedThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) stats_merge(sh, threadIdx.x, threadIdx.x + w);
        __syncthreads();
    }
}

// Per-block partials over the interior cells: compensated sum, min, count < 0.
// One warp per interior row (rows spread over the blocks in a fixed order),
// lanes along x with four loads in flight; no per-element index arithmetic.
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_stats(Dims d, const T* __restrict__ c,
                                                       double* __restrict__ part)
{
    constexpr int NW = kRedThreads / 32;
    const int nxi = d.nx - 2, nyi = d.ny - 2;
    const long long rows = (long long)nyi * (d.ns - 2);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // four independent compensated sums per thread (the loads of one group
    // of four feed four dependency chains), merged in a fixed order
    double s[4] = {0, 0, 0, 0}, comp[4] = {0, 0, 0, 0}, mn = 1e308;
    long long neg = 0;
    auto acc = [&](int a, double x) {
        neu_add(s[a], comp[a], x);
        mn = x < mn ? x : mn;
        neg += x < 0 ? 1 : 0;
    };
    for (long long r = (long long)blockIdx.x * NW + warp; r < rows; r += (long long)gridDim.x * NW) {
        const int j = 1 + (int)(r % nyi), k = 1 + (int)(r / nyi);
        const T* row = c + cell(d, 1, j, k);
        int i = lane;
        for (; i + 96 < nxi; i += 128) {
            const double x0 = (double)row[i], x1 = (double)row[i + 32], x2 = (double)row[i + 64],
                         x3 = (double)row[i + 96];
            acc(0, x0);
            acc(1, x1);
            acc(2, x2);
            acc(3, x3);
        }
        for (; i < nxi; i += 32) acc(0, (double)row[i]);
    }
#pragma unroll
    for (int a = 1; a < 4; a++) {
        neu_add(s[0], comp[0], s[a]);
        comp[0] += comp[a];
    }
    __shared__ double sh[4][kRedThreads];
    sh[0][threadIdx.x] = s[0];
    sh[1][threadIdx.x] = comp[0];
    sh[2][threadIdx.x] = mn;
    sh[3][threadIdx.x] = (double)neg;
    stats_tree(sh);
    if (threadIdx.x < 4) part[4 * blockIdx.x + threadIdx.x] = sh[threadIdx.x][0];
}

// One block of kRedThreads: thread t merges the partials t, t + kRedThreads,
// ... in order, then the fixed-order tree (deterministic).
__global__ void __launch_bounds__(kRedThreads) k_stats_final(const double* __restrict__ part,
                                                             int nblk, double* __restrict__ out)
{
    __shared__ double sh[4][kRedThreads];
    const int t = threadIdx.x;
    double S = 0, Cp = 0, M = 1e308, N = 0;
    for (int b = t; b < nblk; b += kRedThreads) {
        neu_add(S, Cp, part[4 * b + 0]);
        Cp += part[4 * b + 1];
        M = part[4 * b + 2] < M ? part[4 * b + 2] : M;
        N += part[4 * b + 3];
    }
    sh[0][t] = S;
    sh[1][t] = Cp;
    sh[2][t] = M;
    sh[3][t] = N;
    stats_tree(sh);
    if (t == 0) {
        out[0] = sh[0][0] + sh[1][0];
        out[1] = sh[2][0];
        out[2] = sh[3][0];
    }
}

// max |face| over the three face arrays, whole (unused entries hold 0):
// 16-byte loads (every array is a multiple of 32 elements, 256-byte
// aligned), three independent maxima per thread.
template <typename T> struct Vec16Of;
template <> struct Vec16Of<float> { using type = float4; };
template <> struct Vec16Of<double> { using type = double2; };
__device__ __forceinline__ double vabsmax(float4 v)
{
    return fmax(fmax(fabs((double)v.x), fabs((double)v.y)), fmax(fabs((double)v.z), fabs((double)v.w)));
}
__device__ __forceinline__ double vabsmax(double2 v) { return fmax(fabs(v.x), fabs(v.y)); }

template <typename T>
__global__ void k_facemax(Dims d, const T* __restrict__ U, const T* __restrict__ V,
                          const T* __restrict__ W, double* __restrict__ part)
{
    using VT = typename Vec16Of<T>::type;
    const long long n = (long long)d.pp * d.ns / (long long)(16 / sizeof(T));
    const VT* u = reinterpret_cast<const VT*>(U);
    const VT* v = reinterpret_cast<const VT*>(V);
    const VT* w = reinterpret_cast<const VT*>(W);
    double ma = 0, mb = 0, mc = 0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        ma = fmax(ma, vabsmax(u[t]));
        mb = fmax(mb, vabsmax(v[t]));
        mc = fmax(mc, vabsmax(w[t]));
    }
    __shared__ double sh[kRedThreads];
    sh[threadIdx.x] = fmax(ma, fmax(mb, mc));
    __syncthreads();
    for (int k = kRedThreads / 2; k > 0; k >>= 1) {
        if ((int)threadIdx.x < k) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + k]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void __launch_bounds__(kRedThreads) k_max_final(const double* __restrict__ part,
                                                           int nblk, double* __restrict__ out)
{
    __shared__ double sh[kRedThreads];
    double m = 0;
    for (int b = threadIdx.x; b < nblk; b += kRedThreads) m = fmax(m, part[b]);
    sh[threadIdx.x] = m;
    __syncthreads();
    for (int w = kRedThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sh[0];
}

}  // namespace
}  // namespace mpd

// ---------------------------------------------------------------------------
// solver
using mpd::Solver;

namespace {

// Default z-chunk depth of the fused kernels: enough CTAs for at least six
// waves (two CTAs per SM for either pass), deep chunks rounded up to whole
// 16-plane blocks, never chunks thinner than 8 planes.  Measured on B200 at
// 512x512x256 (Gcell-steps/s, limiter approx / IEEE one-cell / plain):
// depth 96 (this rule) 24.99 / 12.94 / 28.06 against 24.46 / 12.42 / 27.15 for
// four waves (127, 127, 85 planes).
int default_zdepth(const mpd::Solver* h)
{
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
    const bool lim = h->opts.limiter != 0;
    int sx, sy, per_sm;
    if (h->pair) {
        sx = lim ? 28 : 30;
        sy = lim ? mpd::kPairCY - 3 : mpd::kPairCY - 1;
        per_sm = mpd::kPairCY >= 32 ? 1 : 2;
    } else {
        sx = lim ? 30 : 32;
        sy = lim ? 14 : 16;
        per_sm = 2;
    }
    const long long bx = (h->d.nx - 2 + sx - 1) / sx;
    const long long by = (h->d.ny - 2 + sy - 1) / sy;
    const long long want = 6LL * per_sm * sms;
    const int interior = h->d.ns - 2;
    long long chunks = (want + bx * by - 1) / (bx * by);
    if (chunks < 1) chunks = 1;
    int depth = (int)((interior + chunks - 1) / chunks);
    if (depth >= 32) depth = (depth + 15) / 16 * 16;
    if (depth < 8) depth = 8;
    return depth >= interior ? 0 : depth;
}

int check_dims(int nx, int ny, int ns)
{
    if (nx < 3 || ny < 3 || ns < 3)
        return mpd::fail(MPDATA_ERR_ARG, "grid %dx%dx%d: every dimension must be >= 3", nx, ny, ns);
    if ((long long)nx * ny * ns > (1LL << 40))
        return mpd::fail(MPDATA_ERR_ARG, "grid %dx%dx%d too large", nx, ny, ns);
    return 0;
}

size_t field_bytes(const Solver* h) { return (size_t)h->d.pp * h->d.ns * h->esz; }

template <typename T> T* F(Solver* h, int set, int axis) { return (T*)h->faces[set][axis]; }
template <typename T> T* Cb(Solver* h, int b) { return (T*)h->c[b]; }

int ensure_device(const Solver* h)
{
    int cur = -1;
    CUDA_TRY(cudaGetDevice(&cur));
    if (cur != h->device) CUDA_TRY(cudaSetDevice(h->device));
    return 0;
}

// Copy a dense host/device full grid (row pitch nx) into a pitched device array.
int put_grid(Solver* h, void* dst, const void* src, int where)
{
    if (where != MPDATA_HOST && where != MPDATA_DEVICE) return mpd::fail(MPDATA_ERR_ARG, "bad where %d", where);
    size_t w = (size_t)h->d.nx * h->esz;
    CUDA_TRY(cudaMemcpy2DAsync(dst, (size_t)h->d.px * h->esz, src, w, w,
                               (size_t)h->d.ny * h->d.ns,
                               where == MPDATA_HOST ? cudaMemcpyHostToDevice
                                                    : cudaMemcpyDeviceToDevice,
                               h->stream));
    return 0;
}

int get_grid(Solver* h, void* dst, const void* src, int where)
{
    if (where != MPDATA_HOST && where != MPDATA_DEVICE) return mpd::fail(MPDATA_ERR_ARG, "bad where %d", where);
    size_t w = (size_t)h->d.nx * h->esz;
    CUDA_TRY(cudaMemcpy2DAsync(dst, w, src, (size_t)h->d.px * h->esz, w,
                               (size_t)h->d.ny * h->d.ns,
                               where == MPDATA_HOST ? cudaMemcpyDeviceToHost
                                                    : cudaMemcpyDeviceToDevice,
                               h->stream));
    return 0;
}

template <typename T> struct ModeOps {
    decltype(&mpd::fast::launch_courant<T>) courant;
    decltype(&mpd::fast::launch_donor<T>) donor;
    decltype(&mpd::fast::launch_courant_donor<T>) courant_donor;
    decltype(&mpd::fast::launch_pass_unfused<T>) pass_unfused;
    decltype(&mpd::fast::launch_pass_fused<T>) pass_fused;
};

template <typename T> ModeOps<T> ops(const Solver* h)
{
    if (h->opts.strict)
        return {mpd::strict::launch_courant<T>, mpd::strict::launch_donor<T>,
                mpd::strict::launch_courant_donor<T>, mpd::strict::launch_pass_unfused<T>,
                mpd::strict::launch_pass_fused<T>};
    return {mpd::fast::launch_courant<T>, mpd::fast::launch_donor<T>,
            mpd::fast::launch_courant_donor<T>, mpd::fast::launch_pass_unfused<T>,
            mpd::fast::launch_pass_fused<T>};
}

template <typename T> int check_courant(Solver* h)
{
    mpd::k_facemax<T><<<mpd::kRedBlocks, mpd::kRedThreads, 0, h->stream>>>(
        h->d, F<T>(h, 0, 0), F<T>(h, 0, 1), F<T>(h, 0, 2), h->red);
    mpd::k_max_final<<<1, mpd::kRedThreads, 0, h->stream>>>(h->red, mpd::kRedBlocks,
                                                            h->red + 4 * mpd::kRedBlocks);
    double m = 0;
    CUDA_TRY(cudaMemcpyAsync(&m, h->red + 4 * mpd::kRedBlocks, sizeof m, cudaMemcpyDeviceToHost,
                             h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (!(m <= 1.0))
        return mpd::fail(MPDATA_ERR_COURANT, "max |face Courant number| = %g exceeds 1", m);
    return 0;
}

// Event pair around one pass launch when per-pass timing is on.
struct PassTimer {
    Solver* h;
    int cls;
    cudaEvent_t a = nullptr, b = nullptr;
    PassTimer(Solver* h_, int cls_) : h(h_), cls(cls_)
    {
        if (!h->timing) return;
        a = take();
        b = take();
        cudaEventRecord(a, h->stream);
    }
    ~PassTimer()
    {
        if (!h->timing) return;
        cudaEventRecord(b, h->stream);
        h->pending[cls].push_back({a, b});
    }
    cudaEvent_t take()
    {
        cudaEvent_t e = nullptr;
        if (!h->event_pool.empty()) {
            e = h->event_pool.back();
            h->event_pool.pop_back();
        } else {
            cudaEventCreate(&e);
        }
        return e;
    }
};

// Arguments of corrective pass o: input level `in`, output level `out`, step
// input level b0 (limiter bounds); every interior plane unless narrowed.
template <typename T> mpd::PassArgs<T> pass_args(Solver* h, int o, int in, int out, int b0)
{
    const int P = h->order;
    const int rs = (o == 1) ? 0 : 1 + ((o - 2) & 1);  // face set read
    const int ws = 1 + ((o - 1) & 1);                  // face set written
    mpd::PassArgs<T> a{};
    a.maps = {&h->tm_c[in], &h->tm_c[b0], &h->tm_f[rs][0], &h->tm_f[rs][1], &h->tm_f[rs][2]};
    a.maps2 = {&h->tm2_c[in], &h->tm2_c[b0], &h->tm2_f[rs][0], &h->tm2_f[rs][1], &h->tm2_f[rs][2]};
    a.err = h->dev_err;
    a.c = Cb<T>(h, in);
    a.cn = Cb<T>(h, b0);
    a.Uo = F<T>(h, rs, 0);
    a.Vo = F<T>(h, rs, 1);
    a.Wo = F<T>(h, rs, 2);
    a.Vadv = F<T>(h, 0, 1);
    a.Un = F<T>(h, ws, 0);
    a.Vn = F<T>(h, ws, 1);
    a.Wn = F<T>(h, ws, 2);
    a.c_out = Cb<T>(h, out);
    a.pass = o;
    a.use_div = h->opts.div_mode != MPDATA_DIV_OFF;
    a.vv_fix = h->opts.vv_fix;
    a.limiter = h->opts.limiter;
    a.wide = h->opts.precision_form;
    a.write_faces = o < P - 1;
    a.approx = h->opts.approx_div;
    a.zdepth = h->zdepth;
    a.zbase = a.zend = 0;  // every interior plane
    return a;
}

// Launch one corrective pass with the solver's kernel choice.
template <typename T> void launch_pass(Solver* h, const mpd::PassArgs<T>& a, cudaStream_t s)
{
    if constexpr (std::is_same<T, float>::value) {
        if (h->pair) {
            mpd::fast::launch_pass_pair(h->d, a, s);
            return;
        }
    }
    ModeOps<T> op = ops<T>(h);
    if (h->opts.kernel != 1) op.pass_fused(h->d, a, s);
    else op.pass_unfused(h->d, a, (T*)h->bup, (T*)h->bdn, s);
}

template <typename T> int step_impl(Solver* h, int nsteps)
{
    ModeOps<T> op = ops<T>(h);
    const Dims& d = h->d;
    const int P = h->order;
    for (int s = 0; s < nsteps; s++) {
        const int b0 = h->cur, b1 = (b0 + 1) % 3, b2 = (b0 + 2) % 3;
        // pass 0: donor cell with the advective faces (formed in the same march
        // when a velocity update left them pending)
        {
            PassTimer t(h, 0);
            if (h->vel_pending) {
                const T* m = (const T*)h->metric;
                const T* const* v = reinterpret_cast<const T* const*>(h->vel_dev);
                op.courant_donor(d, m, m + d.nx, m + d.nx + d.ny, (T)h->vel_dt, v[0], v[1], v[2],
                                 v[3], v[4], v[5], Cb<T>(h, b0), F<T>(h, 0, 0), F<T>(h, 0, 1),
                                 F<T>(h, 0, 2), Cb<T>(h, b1), 0, 0, h->stream);
                h->vel_pending = false;
            } else {
                op.donor(d, Cb<T>(h, b0), F<T>(h, 0, 0), F<T>(h, 0, 1), F<T>(h, 0, 2),
                         Cb<T>(h, b1), 0, 0, 0, h->stream);
            }
        }
        int in = b1, out = b2;
        for (int o = 1; o < P; o++) {
            const mpd::PassArgs<T> a = pass_args<T>(h, o, in, out, b0);
            {
                PassTimer timer(h, a.write_faces ? 1 : 2);
                launch_pass<T>(h, a, h->stream);
            }
            int t = in; in = out; out = t;
        }
        if (P == 1) { h->cur = b1; h->prev = b0; }
        else { h->cur = in; h->prev = out; }
    }
    CUDA_TRY(cudaGetLastError());
    return 0;
}

// One step of the host-array entry point, pipelined over z chunks.
//
// smolar() is bound by PCIe, not by the GPU: every call uploads the velocity
// arrays and the field and downloads two fields.  Here the interior planes
// are cut into chunks of D planes and three streams overlap the work:
// the upload stream copies chunk i (velocities, field, one plane past the
// chunk) and records an event; the compute stream, once it has arrived,
// copies its planes of the input level into the other two levels (their
// shell), forms the faces and runs pass 0 on chunk i, then every corrective
// pass on the chunk's planes, pass o shifted down by 4 o planes (it reads
// pass o-1 from 3 planes below its range to 1 above); the download stream
// then copies the last pass's planes of the chunk, newest and previous
// level, to the host.  Downloads overlap the later uploads (PCIe is full
// duplex) and the kernels overlap both; after the last upload only one
// chunk's passes and download remain.  The kernels and their plane order are those of
// the unchunked step (z-chunked marches give the same bits), so the result
// equals step() on the whole grid bit for bit.  Pinned host memory lets every
// copy run asynchronously; pageable memory gives the same result with less
// overlap.
template <typename T>
int host_step_pipelined_impl(Solver* h, const void* dx, const void* dy, const void* ds,
                             double dt, const void* const vel[6], const void* c_in, void* newest,
                             void* prev, int chunk)
{
    ModeOps<T> op = ops<T>(h);
    const Dims& d = h->d;
    const int ns = d.ns, P = h->order;
    const size_t esz = h->esz, fb = field_bytes(h);
    const int interior = ns - 2;
    // 12 planes: measured best on B200 for a 512 x 512 plane at IORD 3
    // (16: -0.7 %, 24: -4 %, 32: -5 %, 48: -6 %)
    int D = chunk > 0 ? chunk : 12;
    // Pass o runs on chunk i's planes shifted down by o * S: it reads the
    // previous pass's output from 3 planes below its range to 1 above, so it
    // needs nothing from chunk i+1, and the level it reads is overwritten by
    // pass o+1 only below that (every pass of a chunk runs once the chunk has
    // arrived).  A chunk keeps at least 4 planes for the last pass.
    constexpr int S = 4;
    D = std::max(std::max(4, S * (P - 1) + 4), std::min(D, interior));
    const int NC = (interior + D - 1) / D;
    auto cb = [&](int i) { return 1 + i * D; };
    auto ce = [&](int i) { return std::min(ns - 1, 1 + (i + 1) * D); };
    // upload range: through plane ce(i), the one the chunk's last plane reads
    // above it, so chunk i's compute waits for its own upload only
    auto ul = [&](int i) { return i == 0 ? 0 : ce(i - 1) + 1; };
    auto uh = [&](int i) { return i == NC - 1 ? ns : ce(i) + 1; };
    // planes [pb, pe) of pass o on chunk i
    auto pb = [&](int o, int i) { return i == 0 ? 1 : cb(i) - S * o; };
    auto pe = [&](int o, int i) { return i == NC - 1 ? ns - 1 : ce(i) - S * o; };
    // download range: the last pass's planes of the chunk (and the shell planes)
    auto dl = [&](int i) { return i == 0 ? 0 : pb(P - 1, i); };
    auto dh = [&](int i) { return i == NC - 1 ? ns : pe(P - 1, i); };

    if (!h->s_up) CUDA_TRY(cudaStreamCreateWithFlags(&h->s_up, cudaStreamNonBlocking));
    if (!h->s_down) CUDA_TRY(cudaStreamCreateWithFlags(&h->s_down, cudaStreamNonBlocking));
    while ((int)h->pipe_ev.size() < 2 * NC + 1) {
        cudaEvent_t e;
        CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        h->pipe_ev.push_back(e);
    }
    cudaEvent_t* ev_up = h->pipe_ev.data();
    cudaEvent_t* ev_done = ev_up + NC;
    cudaEvent_t ev_start = ev_up[2 * NC];

    // distinct velocity arrays (drivers pass the same array twice)
    int src_of[6];
    for (int v = 0; v < 6; v++) {
        src_of[v] = v;
        for (int w = 0; w < v; w++)
            if (vel[w] == vel[v]) { src_of[v] = src_of[w]; break; }
        if (src_of[v] == v && !h->vel[v]) CUDA_TRY(cudaMalloc(&h->vel[v], fb));
    }
    const T* dev[6];
    for (int v = 0; v < 6; v++) dev[v] = (const T*)h->vel[src_of[v]];

    h->vel_pending = false;  // this step forms its own faces from its own velocities
    // the fused face+donor kernel writes only the face entries the passes read
    if (!h->faces0_clean) {
        for (int a = 0; a < 3; a++) CUDA_TRY(cudaMemsetAsync(h->faces[0][a], 0, fb, h->stream));
        h->faces0_clean = true;
    }
    // the upload stream may overwrite buffers only after earlier work on them
    CUDA_TRY(cudaEventRecord(ev_start, h->stream));
    CUDA_TRY(cudaStreamWaitEvent(h->s_up, ev_start, 0));
    CUDA_TRY(cudaStreamWaitEvent(h->s_down, ev_start, 0));
    char* met = (char*)h->metric;
    CUDA_TRY(cudaMemcpyAsync(met, dx, d.nx * esz, cudaMemcpyHostToDevice, h->s_up));
    CUDA_TRY(cudaMemcpyAsync(met + d.nx * esz, dy, d.ny * esz, cudaMemcpyHostToDevice, h->s_up));
    CUDA_TRY(cudaMemcpyAsync(met + (d.nx + d.ny) * esz, ds, d.ns * esz, cudaMemcpyHostToDevice,
                             h->s_up));
    const size_t w = (size_t)d.nx * esz, plane_host = (size_t)d.nx * d.ny * esz;
    const size_t plane_dev = (size_t)d.pp * esz;
    auto up = [&](void* dst, const void* src, int k0, int k1) -> int {
        CUDA_TRY(cudaMemcpy2DAsync((char*)dst + k0 * plane_dev, (size_t)d.px * esz,
                                   (const char*)src + k0 * plane_host, w, w,
                                   (size_t)d.ny * (k1 - k0), cudaMemcpyHostToDevice, h->s_up));
        return 0;
    };
    auto down = [&](void* dst, const void* src, int k0, int k1) -> int {
        CUDA_TRY(cudaMemcpy2DAsync((char*)dst + k0 * plane_host, w,
                                   (const char*)src + k0 * plane_dev, (size_t)d.px * esz, w,
                                   (size_t)d.ny * (k1 - k0), cudaMemcpyDeviceToHost, h->s_down));
        return 0;
    };
    auto upload = [&](int i) -> int {
        for (int v = 0; v < 6; v++)
            if (src_of[v] == v)
                if (int rc = up(h->vel[v], vel[v], ul(i), uh(i))) return rc;
        if (int rc = up(h->c[0], c_in, ul(i), uh(i))) return rc;
        CUDA_TRY(cudaEventRecord(ev_up[i], h->s_up));
        return 0;
    };

    // levels: input 0; pass 0 writes 1, then the corrective passes alternate
    const int b0 = 0, b1 = 1;
    std::vector<int> lin(P), lout(P);
    lout[0] = b1;
    for (int o = 1; o < P; o++) {
        lin[o] = lout[o - 1];
        lout[o] = (o == 1) ? 2 : lin[o - 1];
    }
    const int cur = lout[P - 1], prv = (P == 1) ? b0 : lin[P - 1];
    const T* m = (const T*)h->metric;

    if (int rc = upload(0)) return rc;
    if (NC > 1)
        if (int rc = upload(1)) return rc;
    for (int i = 0; i < NC; i++) {
        if (i + 2 < NC)
            if (int rc = upload(i + 2)) return rc;
        {
            CUDA_TRY(cudaStreamWaitEvent(h->stream, ev_up[i], 0));
            const size_t off = (size_t)ul(i) * plane_dev, len = (size_t)(uh(i) - ul(i)) * plane_dev;
            for (int b = 1; b < 3; b++)
                CUDA_TRY(cudaMemcpyAsync((char*)h->c[b] + off, (const char*)h->c[0] + off, len,
                                         cudaMemcpyDeviceToDevice, h->stream));
            // advective faces and pass 0 of the chunk in one march
            op.courant_donor(d, m, m + d.nx, m + d.nx + d.ny, (T)dt, dev[0], dev[1], dev[2],
                             dev[3], dev[4], dev[5], Cb<T>(h, b0), F<T>(h, 0, 0), F<T>(h, 0, 1),
                             F<T>(h, 0, 2), Cb<T>(h, b1), cb(i), ce(i), h->stream);
        }
        for (int o = 1; o < P; o++) {
            mpd::PassArgs<T> a = pass_args<T>(h, o, lin[o], lout[o], b0);
            a.zbase = pb(o, i);
            a.zend = pe(o, i);
            if (a.zdepth >= a.zend - a.zbase) a.zdepth = 0;  // one march per column
            launch_pass<T>(h, a, h->stream);
        }
        CUDA_TRY(cudaEventRecord(ev_done[i], h->stream));
        CUDA_TRY(cudaStreamWaitEvent(h->s_down, ev_done[i], 0));
        if (int rc = down(newest, h->c[cur], dl(i), dh(i))) return rc;
        if (int rc = down(prev, h->c[prv], dl(i), dh(i))) return rc;
    }
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(h->s_down));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->cur = cur;
    h->prev = prv;
    h->have_field = h->have_faces = true;
    return mpd::check_device_error(h);
}

template <typename T> int launches_per_step(const Solver* h)
{
    int n = 1;  // donor pass
    for (int o = 1; o < h->order; o++) {
        if (h->opts.kernel != 1) n += 1;
        else n += h->opts.limiter ? 4 : 2;
    }
    return n;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no -lcuda).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// Descriptor of one full-grid array for the fused kernels' per-plane boxes.
int make_map(const Solver* h, void* ptr, CUtensorMap* map, int box_x = mpd::kBoxX,
             int box_y = mpd::kBoxY)
{
    EncodeTiledFn enc = encode_fn();
    if (!enc) return mpd::fail(MPDATA_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[3] = {(cuuint64_t)h->d.nx, (cuuint64_t)h->d.ny, (cuuint64_t)h->d.ns};
    cuuint64_t strides[2] = {(cuuint64_t)(h->d.px * h->esz), (cuuint64_t)(h->d.pp * h->esz)};
    cuuint32_t box[3] = {(cuuint32_t)box_x, (cuuint32_t)box_y, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(map, h->dtype == MPDATA_F32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                                 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                     3, ptr, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return mpd::fail(MPDATA_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return 0;
}

int alloc_solver(Solver* h)
{
    size_t fb = field_bytes(h);
    for (int b = 0; b < 3; b++) CUDA_TRY(cudaMalloc(&h->c[b], fb));
    for (int s = 0; s < 3; s++)
        for (int a = 0; a < 3; a++) CUDA_TRY(cudaMalloc(&h->faces[s][a], fb));
    CUDA_TRY(cudaMalloc(&h->dev_err, sizeof(int)));
    CUDA_TRY(cudaMemsetAsync(h->dev_err, 0, sizeof(int), h->stream));
    if (h->opts.kernel != 1) {
        for (int b = 0; b < 3; b++)
            if (int rc = make_map(h, h->c[b], &h->tm_c[b])) return rc;
        for (int s = 0; s < 3; s++)
            for (int a = 0; a < 3; a++)
                if (int rc = make_map(h, h->faces[s][a], &h->tm_f[s][a])) return rc;
    }
    if (h->pair) {
        for (int b = 0; b < 3; b++)
            if (int rc = make_map(h, h->c[b], &h->tm2_c[b], mpd::kPairBoxX, mpd::kPairBoxY)) return rc;
        for (int s = 0; s < 3; s++)
            for (int a = 0; a < 3; a++)
                if (int rc = make_map(h, h->faces[s][a], &h->tm2_f[s][a], mpd::kPairBoxX,
                                      mpd::kPairBoxY))
                    return rc;
    }
    if (h->opts.kernel == 1 && h->opts.limiter) {
        CUDA_TRY(cudaMalloc(&h->bup, fb));
        CUDA_TRY(cudaMalloc(&h->bdn, fb));
    }
    CUDA_TRY(cudaMalloc(&h->red, sizeof(double) * (4 * mpd::kRedBlocks + 8)));
    size_t nmet = (size_t)h->d.nx + h->d.ny + h->d.ns;
    CUDA_TRY(cudaMalloc(&h->metric, nmet * h->esz));
    for (int b = 0; b < 3; b++) CUDA_TRY(cudaMemsetAsync(h->c[b], 0, fb, h->stream));
    for (int s = 0; s < 3; s++)
        for (int a = 0; a < 3; a++) CUDA_TRY(cudaMemsetAsync(h->faces[s][a], 0, fb, h->stream));
    return 0;
}

void free_solver(Solver* h)
{
    for (auto& v : h->pending)
        for (auto& p : v) {
            cudaEventDestroy(p.first);
            cudaEventDestroy(p.second);
        }
    for (cudaEvent_t e : h->event_pool) cudaEventDestroy(e);
    for (cudaEvent_t e : h->pipe_ev) cudaEventDestroy(e);
    for (cudaEvent_t e : h->fence_ev)
        if (e) cudaEventDestroy(e);
    if (h->s_up) cudaStreamDestroy(h->s_up);
    if (h->s_down) cudaStreamDestroy(h->s_down);
    for (int b = 0; b < 3; b++) cudaFree(h->c[b]);
    for (int s = 0; s < 3; s++)
        for (int a = 0; a < 3; a++) cudaFree(h->faces[s][a]);
    for (int v = 0; v < 6; v++) cudaFree(h->vel[v]);
    cudaFree(h->bup);
    cudaFree(h->bdn);
    cudaFree(h->red);
    cudaFree(h->metric);
    cudaFree(h->dev_err);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
}

}  // namespace

int mpd::create_solver(Solver** out, int nx, int ny, int ns, int dtype, int order,
                       const mpdata_options* opts)
{
    if (!out) return fail(MPDATA_ERR_ARG, "null handle pointer");
    *out = nullptr;
    if (int rc = check_dims(nx, ny, ns)) return rc;
    if (dtype != MPDATA_F32 && dtype != MPDATA_F64) return fail(MPDATA_ERR_ARG, "bad dtype %d", dtype);
    if (order < 1 || order > 64) return fail(MPDATA_ERR_ARG, "order %d outside 1..64", order);
    mpdata_options o;
    mpdata_default_options(&o);
    if (opts) o = *opts;
    if (o.precision_form && dtype != MPDATA_F32)
        return fail(MPDATA_ERR_ARG, "precision_form applies to float storage only");
    if (o.kernel < 0 || o.kernel > 3) return fail(MPDATA_ERR_ARG, "bad kernel option %d", o.kernel);
    if (o.kernel == 3 && (dtype != MPDATA_F32 || o.strict))
        return fail(MPDATA_ERR_ARG, "the two-cell pass needs float storage without strict mode");
    if (o.approx_div && (dtype != MPDATA_F32 || o.strict || o.kernel == 1))
        return fail(MPDATA_ERR_ARG, "approx_div needs float storage, fused kernels and no strict mode");
    std::unique_ptr<Solver> h(new Solver());
    h->dtype = dtype;
    h->esz = dtype == MPDATA_F32 ? 4 : 8;
    h->order = order;
    h->opts = o;
    h->d.nx = nx;
    h->d.ny = ny;
    h->d.ns = ns;
    h->d.px = ((long long)nx + 31) / 32 * 32;
    h->d.pp = h->d.px * ny;
    CUDA_TRY(cudaGetDevice(&h->device));
    CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
    // The two-cell pass: FP32, fast arithmetic, fused kernels by default.  Its IEEE
    // form divides by div_nearest (round-to-nearest results without the slow-path
    // call that made the compiled division cost it registers); with precision_form
    // it takes FP64 only for near-zero limiter sums, which needs approx_div -- the
    // precision form with IEEE division (all limiter sums and ratios in FP64) stays
    // on the one-cell pass.
    h->pair = o.kernel == 3 || (dtype == MPDATA_F32 && !o.strict && o.kernel == 0 &&
                                !(o.precision_form && !o.approx_div));
    h->zdepth = default_zdepth(h.get());
    if (int rc = alloc_solver(h.get())) {
        free_solver(h.get());
        return rc == MPDATA_ERR_CUDA ? fail(MPDATA_ERR_NOMEM, "device allocation failed: %s",
                                            mpdata_last_error())
                                     : rc;
    }
    *out = h.release();
    return 0;
}

void mpd::destroy_solver(Solver* h)
{
    if (!h) return;
    ensure_device(h);
    cudaStreamSynchronize(h->stream);
    free_solver(h);
    delete h;
}

int mpd::set_velocity(Solver* h, const void* dx, const void* dy, const void* ds, double dt,
                      const void* const vel[6], int where)
{
    if (!h || !dx || !dy || !ds) return fail(MPDATA_ERR_ARG, "null argument");
    for (int v = 0; v < 6; v++)
        if (!vel[v]) return fail(MPDATA_ERR_ARG, "null velocity array");
    if (where != MPDATA_HOST && where != MPDATA_DEVICE && where != MPDATA_DEVICE_BORROW)
        return fail(MPDATA_ERR_ARG, "bad where %d", where);
    if (int rc = ensure_device(h)) return rc;
    const size_t fb = field_bytes(h);
    // Lent device arrays are read in place when their layout is the handle's
    // (dense rows of pitch nx == px, 16-byte aligned for the vector loads).
    bool in_place = where == MPDATA_DEVICE_BORROW && h->d.px == h->d.nx;
    for (int v = 0; v < 6 && in_place; v++) in_place = (uintptr_t)vel[v] % 16 == 0;
    if (where == MPDATA_DEVICE_BORROW) where = MPDATA_DEVICE;
    // Stage the distinct velocity arrays (drivers pass the same array for both
    // time levels, reference tests/ring2d/test.c:89-91).
    const void* dev[6];
    for (int v = 0; v < 6; v++) {
        if (in_place) { dev[v] = vel[v]; continue; }
        int same = -1;
        for (int w = 0; w < v; w++)
            if (vel[w] == vel[v]) same = w;
        if (same >= 0) { dev[v] = dev[same]; continue; }
        if (!h->vel[v]) CUDA_TRY(cudaMalloc(&h->vel[v], fb));
        if (int rc = put_grid(h, h->vel[v], vel[v], where)) return rc;
        dev[v] = h->vel[v];
    }
    const cudaMemcpyKind kind = where == MPDATA_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    char* met = (char*)h->metric;
    CUDA_TRY(cudaMemcpyAsync(met, dx, h->d.nx * h->esz, kind, h->stream));
    CUDA_TRY(cudaMemcpyAsync(met + h->d.nx * h->esz, dy, h->d.ny * h->esz, kind, h->stream));
    CUDA_TRY(cudaMemcpyAsync(met + (h->d.nx + h->d.ny) * h->esz, ds, h->d.ns * h->esz, kind, h->stream));
    for (int v = 0; v < 6; v++) h->vel_dev[v] = dev[v];
    h->vel_dt = dt;
    h->vel_pending = true;
    h->have_faces = true;
    // The next step forms the faces in its pass 0 (one march with the donor
    // update); the Courant check and the one-kernel-per-routine path need
    // them now.
    if (!h->opts.check_courant && h->opts.kernel != 1) {
        if (!h->faces0_clean) {  // the fused march writes only the used entries
            for (int a = 0; a < 3; a++) CUDA_TRY(cudaMemsetAsync(h->faces[0][a], 0, fb, h->stream));
            h->faces0_clean = true;
        }
        return 0;
    }
    if (int rc = materialize_faces(h)) return rc;
    if (h->opts.check_courant)
        return h->dtype == MPDATA_F32 ? check_courant<float>(h) : check_courant<double>(h);
    return 0;
}

// The advective faces of a pending velocity update, formed now (k_courant
// writes every entry, unused ones as 0).
int mpd::materialize_faces(Solver* h)
{
    if (!h->vel_pending) return 0;
    if (int rc = ensure_device(h)) return rc;
    if (h->dtype == MPDATA_F32) {
        const float* m = (const float*)h->metric;
        const float* const* v = reinterpret_cast<const float* const*>(h->vel_dev);
        ops<float>(h).courant(h->d, m, m + h->d.nx, m + h->d.nx + h->d.ny, (float)h->vel_dt, v[0],
                              v[1], v[2], v[3], v[4], v[5], F<float>(h, 0, 0), F<float>(h, 0, 1),
                              F<float>(h, 0, 2), 0, h->d.ns, h->stream);
    } else {
        const double* m = (const double*)h->metric;
        const double* const* v = reinterpret_cast<const double* const*>(h->vel_dev);
        ops<double>(h).courant(h->d, m, m + h->d.nx, m + h->d.nx + h->d.ny, h->vel_dt, v[0], v[1],
                               v[2], v[3], v[4], v[5], F<double>(h, 0, 0), F<double>(h, 0, 1),
                               F<double>(h, 0, 2), 0, h->d.ns, h->stream);
    }
    CUDA_TRY(cudaGetLastError());
    h->vel_pending = false;
    h->faces0_clean = true;
    return 0;
}

int mpd::set_faces(Solver* h, const void* U, const void* V, const void* W, int where)
{
    if (!h || !U || !V || !W) return fail(MPDATA_ERR_ARG, "null argument");
    if (int rc = ensure_device(h)) return rc;
    const void* src[3] = {U, V, W};
    for (int a = 0; a < 3; a++)
        if (int rc = put_grid(h, h->faces[0][a], src[a], where)) return rc;
    h->have_faces = true;
    h->faces0_clean = false;
    h->vel_pending = false;  // these faces supersede a pending velocity update
    if (h->opts.check_courant)
        return h->dtype == MPDATA_F32 ? check_courant<float>(h) : check_courant<double>(h);
    return 0;
}

int mpd::set_field(Solver* h, const void* c, int where)
{
    if (!h || !c) return fail(MPDATA_ERR_ARG, "null argument");
    if (int rc = ensure_device(h)) return rc;
    h->cur = 0;
    h->prev = 0;
    if (int rc = put_grid(h, h->c[0], c, where)) return rc;
    // The shell is constant from here on: give every buffer the same one.
    const size_t fb = field_bytes(h);
    CUDA_TRY(cudaMemcpyAsync(h->c[1], h->c[0], fb, cudaMemcpyDeviceToDevice, h->stream));
    CUDA_TRY(cudaMemcpyAsync(h->c[2], h->c[0], fb, cudaMemcpyDeviceToDevice, h->stream));
    h->have_field = true;
    return 0;
}

int mpd::get_field(Solver* h, void* c, int where, bool previous)
{
    if (!h || !c) return fail(MPDATA_ERR_ARG, "null argument");
    if (!h->have_field) return fail(MPDATA_ERR_STATE, "no field set");
    if (int rc = ensure_device(h)) return rc;
    return get_grid(h, c, h->c[previous ? h->prev : h->cur], where);
}

int mpd::host_step_pipelined(Solver* h, const void* dx, const void* dy, const void* ds, double dt,
                             const void* const vel[6], const void* c_in, void* newest, void* prev,
                             int chunk)
{
    if (!h || !dx || !dy || !ds || !c_in || !newest || !prev) return fail(MPDATA_ERR_ARG, "null argument");
    for (int v = 0; v < 6; v++)
        if (!vel[v]) return fail(MPDATA_ERR_ARG, "null velocity array");
    if (h->opts.kernel == 1) return fail(MPDATA_ERR_ARG, "the pipelined step needs the fused kernels");
    if (int rc = ensure_device(h)) return rc;
    return h->dtype == MPDATA_F32
               ? host_step_pipelined_impl<float>(h, dx, dy, ds, dt, vel, c_in, newest, prev, chunk)
               : host_step_pipelined_impl<double>(h, dx, dy, ds, dt, vel, c_in, newest, prev, chunk);
}

int mpd::step(Solver* h, int nsteps)
{
    if (!h) return fail(MPDATA_ERR_ARG, "null handle");
    if (nsteps < 0) return fail(MPDATA_ERR_ARG, "negative step count");
    if (!h->have_field || !h->have_faces)
        return fail(MPDATA_ERR_STATE, "field and velocity/faces must be set before stepping");
    if (int rc = ensure_device(h)) return rc;
    return h->dtype == MPDATA_F32 ? step_impl<float>(h, nsteps) : step_impl<double>(h, nsteps);
}

int mpd::stats(Solver* h, double out[3])
{
    if (!h) return fail(MPDATA_ERR_ARG, "null handle");
    if (!h->have_field) return fail(MPDATA_ERR_STATE, "no field set");
    if (int rc = ensure_device(h)) return rc;
    if (h->d.nx < 3 || h->d.ny < 3 || h->d.ns < 3) return fail(MPDATA_ERR_ARG, "no interior");
    if (h->dtype == MPDATA_F32)
        mpd::k_stats<float><<<mpd::kRedBlocks, mpd::kRedThreads, 0, h->stream>>>(
            h->d, (const float*)h->c[h->cur], h->red);
    else
        mpd::k_stats<double><<<mpd::kRedBlocks, mpd::kRedThreads, 0, h->stream>>>(
            h->d, (const double*)h->c[h->cur], h->red);
    mpd::k_stats_final<<<1, mpd::kRedThreads, 0, h->stream>>>(h->red, mpd::kRedBlocks,
                                                              h->red + 4 * mpd::kRedBlocks);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(out, h->red + 4 * mpd::kRedBlocks, 3 * sizeof(double),
                             cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return check_device_error(h);
}

int mpd::check_device_error(Solver* h)
{
    int flag = 0;
    CUDA_TRY(cudaMemcpyAsync(&flag, h->dev_err, sizeof flag, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (flag) {
        CUDA_TRY(cudaMemsetAsync(h->dev_err, 0, sizeof(int), h->stream));
        return fail(MPDATA_ERR_CUDA, "fused pass: a staged-plane wait timed out (results invalid)");
    }
    return 0;
}

int mpd::launches(const Solver* h)
{
    return h->dtype == MPDATA_F32 ? launches_per_step<float>(h) : launches_per_step<double>(h);
}

// ---------------------------------------------------------------------------
// C ABI: handle API

extern "C" {

void mpdata_default_options(mpdata_options* o)
{
    if (o) memset(o, 0, sizeof *o);
}

int mpdata_create(mpdata_handle* h, int nx, int ny, int ns, int dtype, int order,
                  const mpdata_options* opts)
{
    return mpd::create_solver(reinterpret_cast<Solver**>(h), nx, ny, ns, dtype, order, opts);
}

int mpdata_destroy(mpdata_handle h)
{
    mpd::destroy_solver(reinterpret_cast<Solver*>(h));
    return 0;
}

int mpdata_set_stream(mpdata_handle hh, void* stream)
{
    Solver* h = reinterpret_cast<Solver*>(hh);
    if (!h) return mpd::fail(MPDATA_ERR_ARG, "null handle");
    if (int rc = ensure_device(h)) return rc;
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (h->own_stream) cudaStreamDestroy(h->stream);
    h->stream = (cudaStream_t)stream;
    h->own_stream = false;
    return 0;
}

int mpdata_set_velocity(mpdata_handle h, const void* dx, const void* dy, const void* ds,
                        double dt, const void* u0, const void* u1, const void* v0,
                        const void* v1, const void* w0, const void* w1, int where)
{
    const void* vel[6] = {u0, u1, v0, v1, w0, w1};
    return mpd::set_velocity(reinterpret_cast<Solver*>(h), dx, dy, ds, dt, vel, where);
}

int mpdata_set_faces(mpdata_handle h, const void* U, const void* V, const void* W, int where)
{
    return mpd::set_faces(reinterpret_cast<Solver*>(h), U, V, W, where);
}

int mpdata_set_field(mpdata_handle h, const void* c, int where)
{
    return mpd::set_field(reinterpret_cast<Solver*>(h), c, where);
}

int mpdata_get_field(mpdata_handle h, void* c, int where)
{
    int rc = mpd::get_field(reinterpret_cast<Solver*>(h), c, where, false);
    if (rc) return rc;
    return mpdata_sync(h);
}

int mpdata_get_previous(mpdata_handle h, void* c, int where)
{
    int rc = mpd::get_field(reinterpret_cast<Solver*>(h), c, where, true);
    if (rc) return rc;
    return mpdata_sync(h);
}

int mpdata_step(mpdata_handle h, int nsteps)
{
    return mpd::step(reinterpret_cast<Solver*>(h), nsteps);
}

// z-planes [k0, k0 + nk) of the newest field, dense (nx x ny per plane).
int mpdata_get_planes(mpdata_handle hh, int k0, int nk, void* dst, int where)
{
    Solver* h = reinterpret_cast<Solver*>(hh);
    if (!h || !dst || nk < 0 || k0 < 0 || k0 + nk > (h ? h->d.ns : 0))
        return mpd::fail(MPDATA_ERR_ARG, "bad plane range");
    if (where != MPDATA_HOST && where != MPDATA_DEVICE && where != MPDATA_HOST_ASYNC)
        return mpd::fail(MPDATA_ERR_ARG, "bad where %d", where);
    if (!h->have_field) return mpd::fail(MPDATA_ERR_STATE, "no field set");
    if (nk == 0 && where != MPDATA_HOST_ASYNC) return 0;
    if (int rc = ensure_device(h)) return rc;
    const size_t w = (size_t)h->d.nx * h->esz;
    const char* src = (const char*)h->c[h->cur] + (size_t)k0 * h->d.pp * h->esz;
    if (nk > 0)
        CUDA_TRY(cudaMemcpy2DAsync(dst, w, src, (size_t)h->d.px * h->esz, w,
                                   (size_t)h->d.ny * nk,
                                   where == MPDATA_DEVICE ? cudaMemcpyDeviceToDevice
                                                          : cudaMemcpyDeviceToHost,
                                   h->stream));
    if (where == MPDATA_HOST) return mpdata_sync(hh);
    if (where != MPDATA_HOST_ASYNC) return 0;
    // queued host copy: fence it and hand out its ticket
    const int slot = h->fence_n % Solver::kFences;
    if (!h->fence_ev[slot])
        CUDA_TRY(cudaEventCreateWithFlags(&h->fence_ev[slot], cudaEventDisableTiming));
    CUDA_TRY(cudaEventRecord(h->fence_ev[slot], h->stream));
    const int ticket = h->fence_n;
    h->fence_n = (h->fence_n + 1) & 0x3fffffff;
    return ticket;
}

// Wait for a queued host copy.  A ticket older than the fence ring waits on
// the fence of a later copy, which completes after it (in stream order).
int mpdata_wait(mpdata_handle hh, int ticket)
{
    Solver* h = reinterpret_cast<Solver*>(hh);
    if (!h || ticket < 0) return mpd::fail(MPDATA_ERR_ARG, "bad ticket");
    cudaEvent_t e = h->fence_ev[ticket % Solver::kFences];
    if (!e) return mpd::fail(MPDATA_ERR_ARG, "no copy with ticket %d", ticket);
    if (int rc = ensure_device(h)) return rc;
    CUDA_TRY(cudaEventSynchronize(e));
    return 0;
}

// Overwrite z-planes [k0, k0 + nk) in every field level (a plane on the
// solver's own z boundary is shell, which every level carries; interior
// planes of the other levels are rewritten by the passes before they are read).
int mpdata_set_planes(mpdata_handle hh, int k0, int nk, const void* src, int where)
{
    Solver* h = reinterpret_cast<Solver*>(hh);
    if (!h || !src || nk < 0 || k0 < 0 || k0 + nk > (h ? h->d.ns : 0))
        return mpd::fail(MPDATA_ERR_ARG, "bad plane range");
    if (!h->have_field) return mpd::fail(MPDATA_ERR_STATE, "no field set");
    if (where != MPDATA_HOST && where != MPDATA_DEVICE)
        return mpd::fail(MPDATA_ERR_ARG, "bad where %d", where);
    if (nk == 0) return 0;
    if (int rc = ensure_device(h)) return rc;
    const size_t w = (size_t)h->d.nx * h->esz;
    for (int b = 0; b < 3; b++) {
        char* dst = (char*)h->c[b] + (size_t)k0 * h->d.pp * h->esz;
        CUDA_TRY(cudaMemcpy2DAsync(dst, (size_t)h->d.px * h->esz, src, w, w, (size_t)h->d.ny * nk,
                                   where == MPDATA_HOST ? cudaMemcpyHostToDevice
                                                        : cudaMemcpyDeviceToDevice,
                                   h->stream));
    }
    return where == MPDATA_HOST ? mpdata_sync(hh) : 0;
}

int mpdata_sync(mpdata_handle hh)
{
    Solver* h = reinterpret_cast<Solver*>(hh);
    if (!h) return mpd::fail(MPDATA_ERR_ARG, "null handle");
    if (int rc = ensure_device(h)) return rc;
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    CUDA_TRY(cudaGetLastError());
    return mpd::check_device_error(h);
}

int mpdata_mass(mpdata_handle h, double* mass)
{
    if (!mass) return mpd::fail(MPDATA_ERR_ARG, "null output");
    double s[3];
    if (int rc = mpd::stats(reinterpret_cast<Solver*>(h), s)) return rc;
    *mass = s[0];
    return 0;
}

int mpdata_min(mpdata_handle h, double* minval, long long* nneg)
{
    double s[3];
    if (int rc = mpd::stats(reinterpret_cast<Solver*>(h), s)) return rc;
    if (minval) *minval = s[1];
    if (nneg) *nneg = (long long)s[2];
    return 0;
}

int mpdata_launches_per_step(mpdata_handle h)
{
    if (!h) return mpd::fail(MPDATA_ERR_ARG, "null handle");
    return mpd::launches(reinterpret_cast<Solver*>(h));
}

int mpdata_set_march_depth(mpdata_handle hh, int depth)
{
    Solver* h = reinterpret_cast<Solver*>(hh);
    if (!h || depth < 0) return mpd::fail(MPDATA_ERR_ARG, "bad arguments");
    h->zdepth = depth >= h->d.ns - 2 ? 0 : depth;
    return 0;
}

int mpdata_march_depth(mpdata_handle hh)
{
    Solver* h = reinterpret_cast<Solver*>(hh);
    if (!h) return mpd::fail(MPDATA_ERR_ARG, "null handle");
    return h->zdepth;
}

int mpdata_autotune(mpdata_handle hh, int trial_steps, int* depth_out, double* ms_out)
{
    Solver* h = reinterpret_cast<Solver*>(hh);
    if (!h || trial_steps < 1) return mpd::fail(MPDATA_ERR_ARG, "bad arguments");
    if (!h->have_field || !h->have_faces) return mpd::fail(MPDATA_ERR_STATE, "field and faces first");
    if (int rc = ensure_device(h)) return rc;
    const size_t fb = field_bytes(h);
    void* saved = nullptr;
    CUDA_TRY(cudaMalloc(&saved, fb));
    CUDA_TRY(cudaMemcpyAsync(saved, h->c[h->cur], fb, cudaMemcpyDeviceToDevice, h->stream));
    const int interior = h->d.ns - 2;
    const int cand[] = {0, 128, 96, 64, 48, 32, 24, 16, 8};
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    int best = h->zdepth;
    double best_ms = 1e300;
    for (int c : cand) {
        if (c != 0 && c >= interior) continue;
        h->zdepth = c;
        if (int rc = mpd::step(h, 1)) { cudaFree(saved); return rc; }
        CUDA_TRY(cudaEventRecord(e0, h->stream));
        if (int rc = mpd::step(h, trial_steps)) { cudaFree(saved); return rc; }
        CUDA_TRY(cudaEventRecord(e1, h->stream));
        CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0;
        CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best_ms) { best_ms = ms; best = c; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    h->zdepth = best;
    // put the field back as it was (all three levels, as set_field does)
    for (int b = 0; b < 3; b++)
        CUDA_TRY(cudaMemcpyAsync(h->c[b], saved, fb, cudaMemcpyDeviceToDevice, h->stream));
    h->cur = 0;
    h->prev = 0;
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    cudaFree(saved);
    if (depth_out) *depth_out = best;
    if (ms_out) *ms_out = best_ms / trial_steps;
    return mpd::check_device_error(h);
}

int mpdata_enable_pass_timing(mpdata_handle hh, int on)
{
    Solver* h = reinterpret_cast<Solver*>(hh);
    if (!h) return mpd::fail(MPDATA_ERR_ARG, "null handle");
    h->timing = on != 0;
    return 0;
}

int mpdata_pass_times(mpdata_handle hh, double ms[3], long long launches[3], int reset)
{
    Solver* h = reinterpret_cast<Solver*>(hh);
    if (!h) return mpd::fail(MPDATA_ERR_ARG, "null handle");
    if (int rc = ensure_device(h)) return rc;
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (int c = 0; c < 3; c++) {
        for (auto& p : h->pending[c]) {
            float t = 0;
            CUDA_TRY(cudaEventElapsedTime(&t, p.first, p.second));
            h->pass_ms[c] += t;
            h->pass_n[c] += 1;
            h->event_pool.push_back(p.first);
            h->event_pool.push_back(p.second);
        }
        h->pending[c].clear();
        if (ms) ms[c] = h->pass_ms[c];
        if (launches) launches[c] = h->pass_n[c];
        if (reset) {
            h->pass_ms[c] = 0;
            h->pass_n[c] = 0;
        }
    }
    return 0;
}

void* mpdata_host_alloc(size_t bytes)
{
    void* p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) {
        mpd::fail(MPDATA_ERR_NOMEM, "cudaMallocHost(%zu) failed", bytes);
        return nullptr;
    }
    return p;
}

void mpdata_host_free(void* p)
{
    if (p) cudaFreeHost(p);
}

}  // extern "C"
