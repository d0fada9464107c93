// Reference-compatible entry points: smolar(), smolar_f64(), msmolar(),
// msmolar_gather(), msmolar_free().
//
// smolar() keeps the reference's host-memory contract (smolar.h:45-48): each
// call stages the distinct velocity arrays and the input field to the GPU,
// runs one step on a per-thread cached solver and copies back both the
// newest field and the level before the last pass, then exchanges the
// caller's pointers exactly as core/src/smolar.c:58 does.
//
// msmolar() is the decomposed step (reference core/src/msmolar.c:13-188) as
// device blocks: the grid is split into sx*sy*ss blocks with the reference's
// sizing rule (multigrid/src/grid.c:68-144: n/s cells each, the first n%s
// blocks one more); each block is a solver over its owned cells plus a halo
// of depth P + L(P-1) (P passes, L = limiter) clipped at the grid edge.  Per
// step every block pulls its halo from the global field, steps, and pushes
// its owned cells back.  With that halo the owned cells are bit-identical to
// the single-domain step (the reference's 1-cell halo is not, so its mring
// tests compare a buffer with itself, tests/init.c:114-115).
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "mpdata_b200.h"
#include "solver.h"

using mpd::Dims;
using mpd::Solver;

#define CUDA_TRY(expr)                                                                      \
    do {                                                                                    \
        cudaError_t e_ = (expr);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return mpd::fail(MPDATA_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(e_)); \
    } while (0)

namespace {

// ---------------------------------------------------------------------------
// smolar()

struct HostCache {
    Solver* h[2] = {nullptr, nullptr};
    ~HostCache()
    {
        for (Solver* s : h) mpd::destroy_solver(s);
    }
};
thread_local HostCache g_cache;
// Options of smolar()/msmolar() on this thread.  Start from the environment
// variable MPDATA_B200_OPTIONS (comma-separated: limiter, precision_form,
// strict, unfused, vv_fix, div_off, approx_div, check_courant), so programs
// written against the reference API, which has no options call, can still
// select them.
mpdata_options env_options()
{
    mpdata_options o;
    memset(&o, 0, sizeof o);
    const char* s = getenv("MPDATA_B200_OPTIONS");
    if (!s) return o;
    std::string v(s);
    auto has = [&](const char* w) {
        size_t p = 0, n = strlen(w);
        while ((p = v.find(w, p)) != std::string::npos) {
            bool start = p == 0 || v[p - 1] == ',';
            bool end = p + n == v.size() || v[p + n] == ',';
            if (start && end) return true;
            p += n;
        }
        return false;
    };
    o.limiter = has("limiter");
    o.precision_form = has("precision_form");
    o.strict = has("strict");
    o.kernel = has("unfused") ? 1 : has("single") ? 2 : has("pair") ? 3 : 0;
    o.vv_fix = has("vv_fix");
    o.div_mode = has("div_off") ? MPDATA_DIV_OFF : MPDATA_DIV_REFERENCE;
    o.approx_div = has("approx_div");
    o.check_courant = has("check_courant");
    return o;
}

thread_local mpdata_options g_opts = env_options();
// smolar(): planes per chunk of the pipelined host step (0 automatic, < 0 off).
thread_local int g_pipe_chunk = 0;

bool same_options(const mpdata_options& a, const mpdata_options& b)
{
    return memcmp(&a, &b, sizeof a) == 0;
}

template <typename T> int smolar_host(int nx, int ny, int ns, T* dx, T* dy, T* ds, T dt,
                                      T* u0, T* u1, T* v0, T* v1, T* w0, T* w1, T** c0,
                                      T** c1, int order)
{
    if (!c0 || !c1 || !*c0 || !*c1) return mpd::fail(MPDATA_ERR_ARG, "null field pointer");
    if (nx < 3 || ny < 3 || ns < 3)
        return mpd::fail(MPDATA_ERR_ARG, "grid %dx%dx%d: every dimension must be >= 3", nx, ny, ns);
    if (order < 0) return mpd::fail(MPDATA_ERR_ARG, "negative order %d", order);
    if (order == 0) {  // no pass runs; the reference still exchanges the pointers
        T* t = *c0; *c0 = *c1; *c1 = t;
        return 0;
    }
    const int dtype = sizeof(T) == 4 ? MPDATA_F32 : MPDATA_F64;
    Solver*& h = g_cache.h[dtype];
    if (h && (h->d.nx != nx || h->d.ny != ny || h->d.ns != ns || !same_options(h->opts, g_opts))) {
        mpd::destroy_solver(h);
        h = nullptr;
    }
    if (!h) {
        if (int rc = mpd::create_solver(&h, nx, ny, ns, dtype, order, &g_opts)) return rc;
    }
    h->order = order;
    const void* vel[6] = {u0, u1, v0, v1, w0, w1};
    // Pipelined over z chunks (the default): the input *c0 is also an output
    // buffer, which is safe because a chunk's planes come back only after the
    // same planes have been uploaded and consumed.
    if (g_pipe_chunk >= 0 && h->opts.kernel != 1 && !h->opts.check_courant) {
        // the last pass writes the caller's c1 buffer when order is odd, c0 otherwise
        T* newest = (order & 1) ? *c1 : *c0;
        T* other = (order & 1) ? *c0 : *c1;
        if (int rc = mpd::host_step_pipelined(h, dx, dy, ds, (double)dt, vel, *c0, newest, other,
                                              g_pipe_chunk))
            return rc;
        *c1 = newest;
        *c0 = other;
        return 0;
    }
    if (int rc = mpd::set_velocity(h, dx, dy, ds, (double)dt, vel, MPDATA_HOST)) return rc;
    if (int rc = mpd::set_field(h, *c0, MPDATA_HOST)) return rc;
    if (int rc = mpd::step(h, 1)) return rc;
    // The last pass writes the caller's c1 buffer when order is odd, c0 otherwise.
    T* newest = (order & 1) ? *c1 : *c0;
    T* other = (order & 1) ? *c0 : *c1;
    if (int rc = mpd::get_field(h, newest, MPDATA_HOST, false)) return rc;
    if (int rc = mpd::get_field(h, other, MPDATA_HOST, true)) return rc;
    if (int rc = mpd::check_device_error(h)) return rc;
    *c1 = newest;
    *c0 = other;
    return 0;
}

// ---------------------------------------------------------------------------
// msmolar()

// Box copy between two pitched grids (the device form of the reference's
// subcpy, multigrid/src/subcpy.c:6-19, and of its scatter/gather block copies,
// multigrid/src/scatter.c:6-153, gather.c:6-139).
template <typename T>
__global__ void k_box_copy(T* __restrict__ dst, long long dpx, long long dpp,
                           const T* __restrict__ src, long long spx, long long spp, int bx,
                           int by, int bz)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    int k = blockIdx.z;
    if (i >= bx || j >= by || k >= bz) return;
    dst[k * dpp + j * dpx + i] = src[k * spp + j * spx + i];
}

template <typename T>
int box_copy(void* dst, const Dims& dd, int dx0, int dy0, int dz0, const void* src,
             const Dims& sd, int sx0, int sy0, int sz0, int bx, int by, int bz, cudaStream_t s)
{
    if (bx <= 0 || by <= 0 || bz <= 0) return 0;
    T* d = (T*)dst + mpd::cell(dd, dx0, dy0, dz0);
    const T* r = (const T*)src + mpd::cell(sd, sx0, sy0, sz0);
    dim3 b(32, 8), g((bx + 31) / 32, (by + 7) / 8, bz);
    k_box_copy<T><<<g, b, 0, s>>>(d, dd.px, dd.pp, r, sd.px, sd.pp, bx, by, bz);
    CUDA_TRY(cudaGetLastError());
    return 0;
}

struct Block {
    int lo[3], hi[3];    // owned cells (global indices)
    int elo[3], ehi[3];  // owned + halo, clipped to the grid
    Solver* s = nullptr; // null when the extended box is thinner than 3 (shell-only block)
};

struct Decomp {
    int n[3], split[3], order = 1, halo = 1, dtype = MPDATA_F32;
    Solver* global = nullptr;  // global field levels, advective faces, stream
    int cur = 0, prev = 1;     // global levels live in global->c[]
    std::vector<Block> blocks;
    ~Decomp()
    {
        for (Block& b : blocks) mpd::destroy_solver(b.s);
        mpd::destroy_solver(global);
    }
};

// Reference block sizing: n/s cells per block, the first n%s blocks one more.
void split_axis(int n, int s, std::vector<int>& start)
{
    start.assign(s + 1, 0);
    int base = n / s, rem = n % s;
    for (int b = 0; b < s; b++) start[b + 1] = start[b] + base + (b < rem ? 1 : 0);
}

template <typename T>
int decomp_create(Decomp** out, int nx, int ny, int ns, T* dx, T* dy, T* ds, T dt, T* u0,
                  T* u1, T* v0, T* v1, T* w0, T* w1, T* c0, int order, int sx, int sy, int ss)
{
    std::unique_ptr<Decomp> D(new Decomp());
    D->dtype = sizeof(T) == 4 ? MPDATA_F32 : MPDATA_F64;
    D->n[0] = nx; D->n[1] = ny; D->n[2] = ns;
    // Same clamping as multigrid/src/grid.c:34-36.
    D->split[0] = sx > nx ? nx : sx;
    D->split[1] = sy > ny ? ny : sy;
    D->split[2] = ss > ns ? ns : ss;
    D->order = order;
    // Exact-equality halo: P cells, plus P-1 more with the limiter.
    D->halo = order + (g_opts.limiter ? order - 1 : 0);
    if (int rc = mpd::create_solver(&D->global, nx, ny, ns, D->dtype, order, &g_opts)) return rc;
    Solver* g = D->global;
    const void* vel[6] = {u0, u1, v0, v1, w0, w1};
    if (int rc = mpd::set_velocity(g, dx, dy, ds, (double)dt, vel, MPDATA_HOST)) return rc;
    if (int rc = mpd::materialize_faces(g)) return rc;  // the blocks copy them below
    if (int rc = mpd::set_field(g, c0, MPDATA_HOST)) return rc;
    std::vector<int> st[3];
    for (int a = 0; a < 3; a++) split_axis(D->n[a], D->split[a], st[a]);
    for (int bz = 0; bz < D->split[2]; bz++)
        for (int by = 0; by < D->split[1]; by++)
            for (int bx = 0; bx < D->split[0]; bx++) {
                Block b;
                int idx[3] = {bx, by, bz};
                bool thin = false;
                for (int a = 0; a < 3; a++) {
                    b.lo[a] = st[a][idx[a]];
                    b.hi[a] = st[a][idx[a] + 1];
                    b.elo[a] = b.lo[a] - D->halo < 0 ? 0 : b.lo[a] - D->halo;
                    b.ehi[a] = b.hi[a] + D->halo > D->n[a] ? D->n[a] : b.hi[a] + D->halo;
                    if (b.ehi[a] - b.elo[a] < 3) thin = true;  // owns shell cells only
                }
                if (!thin) {
                    int e[3] = {b.ehi[0] - b.elo[0], b.ehi[1] - b.elo[1], b.ehi[2] - b.elo[2]};
                    if (int rc = mpd::create_solver(&b.s, e[0], e[1], e[2], D->dtype, order, &g_opts)) {
                        D->blocks.push_back(b);
                        return rc;
                    }
                    // Share the global stream so the whole step is one ordered queue.
                    cudaStreamDestroy(b.s->stream);
                    b.s->stream = g->stream;
                    b.s->own_stream = false;
                    for (int a = 0; a < 3; a++)
                        if (int rc = box_copy<T>(b.s->faces[0][a], b.s->d, 0, 0, 0, g->faces[0][a],
                                                 g->d, b.elo[0], b.elo[1], b.elo[2], e[0], e[1],
                                                 e[2], g->stream))
                            return rc;
                    b.s->have_faces = true;
                    b.s->have_field = true;
                }
                D->blocks.push_back(b);
            }
    // Global previous level = the input until a step runs.
    const size_t fb = (size_t)g->d.pp * g->d.ns * g->esz;
    CUDA_TRY(cudaMemcpyAsync(g->c[1], g->c[0], fb, cudaMemcpyDeviceToDevice, g->stream));
    D->cur = 0;
    D->prev = 1;
    *out = D.release();
    return 0;
}

template <typename T> int decomp_step(Decomp* D)
{
    Solver* g = D->global;
    const int nxt = 3 - D->cur - D->prev;  // the free global level
    const size_t fb = (size_t)g->d.pp * g->d.ns * g->esz;
    // The shell of the whole grid never changes; carry it into the new level.
    CUDA_TRY(cudaMemcpyAsync(g->c[nxt], g->c[D->cur], fb, cudaMemcpyDeviceToDevice, g->stream));
    for (Block& b : D->blocks) {
        if (!b.s) continue;
        Solver* s = b.s;
        int e[3] = {b.ehi[0] - b.elo[0], b.ehi[1] - b.elo[1], b.ehi[2] - b.elo[2]};
        // Halo exchange: pull owned + halo into all three block levels (the
        // block's outer layer is its fixed shell for this step).
        for (int l = 0; l < 3; l++)
            if (int rc = box_copy<T>(s->c[l], s->d, 0, 0, 0, g->c[D->cur], g->d, b.elo[0],
                                     b.elo[1], b.elo[2], e[0], e[1], e[2], g->stream))
                return rc;
        s->cur = 0;
        if (int rc = mpd::step(s, 1)) return rc;
        int o[3] = {b.lo[0] - b.elo[0], b.lo[1] - b.elo[1], b.lo[2] - b.elo[2]};
        int w[3] = {b.hi[0] - b.lo[0], b.hi[1] - b.lo[1], b.hi[2] - b.lo[2]};
        if (int rc = box_copy<T>(g->c[nxt], g->d, b.lo[0], b.lo[1], b.lo[2], s->c[s->cur], s->d,
                                 o[0], o[1], o[2], w[0], w[1], w[2], g->stream))
            return rc;
        if (int rc = box_copy<T>(g->c[D->prev], g->d, b.lo[0], b.lo[1], b.lo[2], s->c[s->prev],
                                 s->d, o[0], o[1], o[2], w[0], w[1], w[2], g->stream))
            return rc;
    }
    D->cur = nxt;
    // D->prev keeps the level before the last pass (written above).
    return 0;
}

template <typename T>
int msmolar_host(void** desc, int nx, int ny, int ns, T* dx, T* dy, T* ds, T dt, T* u0, T* u1,
                 T* v0, T* v1, T* w0, T* w1, T** c0, T** c1, int order, int sx, int sy, int ss)
{
    if (!desc || !c0 || !c1 || !*c0 || !*c1) return mpd::fail(MPDATA_ERR_ARG, "null pointer");
    if (sx < 1 || sy < 1 || ss < 1) return mpd::fail(MPDATA_ERR_ARG, "bad block grid %dx%dx%d", sx, sy, ss);
    if (order < 1) return mpd::fail(MPDATA_ERR_ARG, "order %d < 1", order);
    Decomp* D = (Decomp*)*desc;
    if (!D) {
        // First call: scatter the inputs (msmolar.c:25-32 -> msmolar_scatter.c).
        if (int rc = decomp_create<T>(&D, nx, ny, ns, dx, dy, ds, dt, u0, u1, v0, v1, w0, w1,
                                      *c0, order, sx, sy, ss))
            return rc;
        *desc = D;
    } else if (D->n[0] != nx || D->n[1] != ny || D->n[2] != ns || D->order != order ||
               D->dtype != (sizeof(T) == 4 ? MPDATA_F32 : MPDATA_F64)) {
        return mpd::fail(MPDATA_ERR_STATE, "msmolar state was created for another grid/order");
    }
    if (int rc = decomp_step<T>(D)) return rc;
    // Exchange the caller's pointers the way smolar() would (msmolar.c:182-187).
    if (!(order & 1)) {
        T* t = *c0; *c0 = *c1; *c1 = t;
    }
    return 0;
}

template <typename T> int msmolar_gather_host(void** desc, T** c0, T** c1)
{
    if (!desc || !*desc || !c0 || !c1 || !*c0 || !*c1)
        return mpd::fail(MPDATA_ERR_STATE, "msmolar_gather before msmolar");
    Decomp* D = (Decomp*)*desc;
    Solver* g = D->global;
    const size_t w = (size_t)g->d.nx * g->esz;
    CUDA_TRY(cudaMemcpy2DAsync(*c1, w, g->c[D->cur], (size_t)g->d.px * g->esz, w,
                               (size_t)g->d.ny * g->d.ns, cudaMemcpyDeviceToHost, g->stream));
    CUDA_TRY(cudaMemcpy2DAsync(*c0, w, g->c[D->prev], (size_t)g->d.px * g->esz, w,
                               (size_t)g->d.ny * g->d.ns, cudaMemcpyDeviceToHost, g->stream));
    for (Block& b : D->blocks)
        if (b.s)
            if (int rc = mpd::check_device_error(b.s)) return rc;
    return mpd::check_device_error(g);
}

}  // namespace

extern "C" {

int mpdata_set_pipeline(int chunk_planes)
{
    g_pipe_chunk = chunk_planes;
    return 0;
}

int mpdata_set_default_options(const mpdata_options* opts)
{
    if (!opts) {
        memset(&g_opts, 0, sizeof g_opts);
        return 0;
    }
    if (opts->kernel < 0 || opts->kernel > 3 || opts->div_mode < 0 || opts->div_mode > 1)
        return mpd::fail(MPDATA_ERR_ARG, "bad option value");
    g_opts = *opts;
    return 0;
}

int smolar(int nx, int ny, int ns, float* dx, float* dy, float* ds, const float dt, float* u0,
           float* u1, float* v0, float* v1, float* w0, float* w1, float** c0, float** c1,
           int flow_type, int order)
{
    (void)flow_type;  // stored but never read by the reference (uu.c:111)
    return smolar_host<float>(nx, ny, ns, dx, dy, ds, dt, u0, u1, v0, v1, w0, w1, c0, c1, order);
}

int smolar_f64(int nx, int ny, int ns, double* dx, double* dy, double* ds, const double dt,
               double* u0, double* u1, double* v0, double* v1, double* w0, double* w1,
               double** c0, double** c1, int flow_type, int order)
{
    (void)flow_type;
    return smolar_host<double>(nx, ny, ns, dx, dy, ds, dt, u0, u1, v0, v1, w0, w1, c0, c1, order);
}

int msmolar(void** desc, int nx, int ny, int ns, float* dx, float* dy, float* ds, const float dt,
            float* u0, float* u1, float* v0, float* v1, float* w0, float* w1, float** c0,
            float** c1, int flow_type, int order, int sx, int sy, int ss, int mode)
{
    (void)flow_type;
    (void)mode;  // the reference ignores it as well (msmolar.c:13-188)
    return msmolar_host<float>(desc, nx, ny, ns, dx, dy, ds, dt, u0, u1, v0, v1, w0, w1, c0, c1,
                               order, sx, sy, ss);
}

int msmolar_gather(void** desc, int nx, int ny, int ns, float* dx, float* dy, float* ds,
                   const float dt, float* u0, float* u1, float* v0, float* v1, float* w0,
                   float* w1, float** c0, float** c1, int flow_type, int order, int sx, int sy,
                   int ss, int mode)
{
    (void)nx; (void)ny; (void)ns; (void)dx; (void)dy; (void)ds; (void)dt; (void)u0; (void)u1;
    (void)v0; (void)v1; (void)w0; (void)w1; (void)flow_type; (void)order; (void)sx; (void)sy;
    (void)ss; (void)mode;
    return msmolar_gather_host<float>(desc, c0, c1);
}

int msmolar_free(void** desc)
{
    if (!desc) return mpd::fail(MPDATA_ERR_ARG, "null pointer");
    delete (Decomp*)*desc;
    *desc = nullptr;
    return 0;
}

}  // extern "C"
