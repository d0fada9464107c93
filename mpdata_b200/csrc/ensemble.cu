// Batched ensemble of independent 2D MPDATA problems of uneven sizes.
//
// All instances step in lockstep: one launch per pass covers every instance
// (kernels_ensemble.cuh), a multi-step sequence is captured once into a CUDA
// graph and replayed, and the tile shape is chosen by timing the candidates
// on the ensemble itself (mpdata_ensemble_autotune).  Instance arrays live
// in one device arena; each instance has its own row pitch (a multiple of 32).
// The level rotation is the solver's (three field levels, advective + two
// Jacobi face sets), shared by every instance.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <memory>
#include <vector>

#include "launch.h"
#include "mpdata_b200.h"
#include "solver.h"

using mpd::Dims;

#define CUDA_TRY(expr)                                                                      \
    do {                                                                                    \
        cudaError_t e_ = (expr);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return mpd::fail(MPDATA_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(e_)); \
    } while (0)

namespace {

// Tile shapes of the tile kernels.  Candidate kMarch runs the first
// corrective pass as a y-march (one warp per strip of 32 columns x kMarchRows
// rows, k_ens_march) and every other pass with tile kMarchTile.
constexpr int kTiles = 3;
const int kTileX[kTiles] = {32, 32, 64};
const int kTileY[kTiles] = {8, 16, 8};
constexpr int kMarch = kTiles, kMarchTile = 1, kCandidates = kTiles + 1;
#ifndef MPD_MARCH_ROWS
#define MPD_MARCH_ROWS 48
#endif
constexpr int kMarchRows = MPD_MARCH_ROWS;

struct GraphKey {
    int nsteps, cur;
    bool operator<(const GraphKey& o) const { return nsteps != o.nsteps ? nsteps < o.nsteps : cur < o.cur; }
};

}  // namespace

struct mpdata_ensemble {
    int n = 0, order = 2;
    mpdata_options opts{};
    std::vector<int> nx, ny, px;
    std::vector<mpd::EnsInst> host_insts;
    float* arena = nullptr;
    mpd::EnsInst* insts = nullptr;
    // work lists per tile shape: [tile][0] donor items, [tile][1] pass items
    mpd::EnsItem* items[kTiles][2] = {{nullptr}};
    int nitems[kTiles][2] = {{0}};
    mpd::EnsItem* march_items = nullptr;  // (instance, first owned column, rows [j0, pad))
    int nmarch = 0;
    int tile = 0;  // candidate 0 .. kCandidates-1
    int grid_donor = 0, grid_pass = 0;
    int cur = 0, prev = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::map<GraphKey, cudaGraphExec_t> graphs;
    std::vector<bool> have_field, have_faces;
};

namespace {

void drop_graphs(mpdata_ensemble* e)
{
    for (auto& kv : e->graphs) cudaGraphExecDestroy(kv.second);
    e->graphs.clear();
}

int build_items(mpdata_ensemble* e)
{
    for (int t = 0; t < kTiles; t++)
        for (int kind = 0; kind < 2; kind++) {
            // cells a pass item owns: the tile less 2 low + 1 high halo cells
            // with the limiter, 1 low without (k_ens_pass LO / HI); donor: all
            const int halo = kind == 0 ? 0 : (e->opts.limiter ? 3 : 1);
            const int sx = kTileX[t] - halo, sy = kTileY[t] - halo;
            std::vector<mpd::EnsItem> v;
            for (int q = 0; q < e->n; q++)
                for (int j0 = 1; j0 <= e->ny[q] - 2; j0 += sy)
                    for (int i0 = 1; i0 <= e->nx[q] - 2; i0 += sx) v.push_back({q, i0, j0, 0});
            // largest instances first: the persistent grid's stride then mixes sizes
            std::stable_sort(v.begin(), v.end(), [&](const mpd::EnsItem& a, const mpd::EnsItem& b) {
                return (long long)e->nx[a.inst] * e->ny[a.inst] > (long long)e->nx[b.inst] * e->ny[b.inst];
            });
            CUDA_TRY(cudaMalloc(&e->items[t][kind], std::max<size_t>(1, v.size()) * sizeof(mpd::EnsItem)));
            CUDA_TRY(cudaMemcpy(e->items[t][kind], v.data(), v.size() * sizeof(mpd::EnsItem),
                                cudaMemcpyHostToDevice));
            e->nitems[t][kind] = (int)v.size();
        }
    // march strips: 26 owned columns of 32 lanes with the limiter (3 halo lanes
    // each side), 28 without; chunks of kMarchRows owned rows
    {
        const int w = e->opts.limiter ? 26 : 28;
        std::vector<mpd::EnsItem> v;
        for (int q = 0; q < e->n; q++)
            for (int j0 = 1; j0 <= e->ny[q] - 2; j0 += kMarchRows)
                for (int i0 = 1; i0 <= e->nx[q] - 2; i0 += w)
                    v.push_back({q, i0, j0, std::min(j0 + kMarchRows, e->ny[q] - 1)});
        std::stable_sort(v.begin(), v.end(), [&](const mpd::EnsItem& a, const mpd::EnsItem& b) {
            return (long long)e->nx[a.inst] * e->ny[a.inst] > (long long)e->nx[b.inst] * e->ny[b.inst];
        });
        CUDA_TRY(cudaMalloc(&e->march_items, std::max<size_t>(1, v.size()) * sizeof(mpd::EnsItem)));
        CUDA_TRY(cudaMemcpy(e->march_items, v.data(), v.size() * sizeof(mpd::EnsItem),
                            cudaMemcpyHostToDevice));
        e->nmarch = (int)v.size();
    }
    return 0;
}

// The tile kernels' shape for the current candidate.
int tile_shape(const mpdata_ensemble* e) { return e->tile == kMarch ? kMarchTile : e->tile; }

void set_grid(mpdata_ensemble* e)
{
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device);
    // persistent grids: a few CTAs per SM, never more than there are items
    const int t = tile_shape(e);
    e->grid_donor = std::max(1, std::min(e->nitems[t][0], sms * 8));
    e->grid_pass = std::max(1, std::min(e->nitems[t][1], sms * 4));
}

template <bool STRICT>
void launch_step_passes(mpdata_ensemble* e, int& cur, int& prev)
{
    const int P = e->order;
    const int b0 = cur, b1 = (b0 + 1) % 3, b2 = (b0 + 2) % 3;
    mpd::EnsPass p{};
    p.in = b0; p.out = b1; p.cn = b0; p.rs = 0; p.ws = 0; p.pass = 0;
    p.use_div = e->opts.div_mode != MPDATA_DIV_OFF;
    p.vv_fix = e->opts.vv_fix;
    p.fuse_donor = 0;
    const int t = tile_shape(e);
    // With corrective passes, pass 1 forms c^(1) itself (level b1 is then not written)
    if (P == 1) {
        if (STRICT)
            mpd::strict::launch_ens_donor<float>(t, e->arena, e->insts, e->items[t][0],
                                                 e->nitems[t][0], e->grid_donor, p, e->stream);
        else
            mpd::fast::launch_ens_donor<float>(t, e->arena, e->insts, e->items[t][0],
                                               e->nitems[t][0], e->grid_donor, p, e->stream);
    }
    int in = b1, out = b2;
    for (int o = 1; o < P; o++) {
        p.in = in; p.out = out; p.cn = b0;
        p.rs = (o == 1) ? 0 : 1 + ((o - 2) & 1);
        p.ws = 1 + ((o - 1) & 1);
        p.pass = o;
        p.write_faces = o < P - 1;
        p.fuse_donor = o == 1;
        // the march candidate runs the (fused) first pass as a y-march; the march
        // has FP32 limiter ratios only, so the precision form keeps the tile kernel
        if (o == 1 && e->tile == kMarch && !e->opts.precision_form) {
            if (STRICT)
                mpd::strict::launch_ens_march<float>(e->arena, e->insts, e->march_items, e->nmarch, p,
                                                     e->opts.limiter, 0, e->stream);
            else
                mpd::fast::launch_ens_march<float>(e->arena, e->insts, e->march_items, e->nmarch, p,
                                                   e->opts.limiter, e->opts.approx_div, e->stream);
        } else if (STRICT) {
            mpd::strict::launch_ens_pass<float>(t, e->arena, e->insts, e->items[t][1], e->nitems[t][1],
                                                e->grid_pass, p, e->opts.limiter,
                                                e->opts.precision_form, 0, e->stream);
        } else {
            mpd::fast::launch_ens_pass<float>(t, e->arena, e->insts, e->items[t][1], e->nitems[t][1],
                                              e->grid_pass, p, e->opts.limiter, e->opts.precision_form,
                                              e->opts.approx_div, e->stream);
        }
        std::swap(in, out);
    }
    if (P == 1) { cur = b1; prev = b0; }
    else { cur = in; prev = out; }
}

int run_steps_direct(mpdata_ensemble* e, int nsteps)
{
    for (int s = 0; s < nsteps; s++) {
        if (e->opts.strict) launch_step_passes<true>(e, e->cur, e->prev);
        else launch_step_passes<false>(e, e->cur, e->prev);
    }
    CUDA_TRY(cudaGetLastError());
    return 0;
}

int ensure_device(const mpdata_ensemble* e)
{
    int cur = -1;
    CUDA_TRY(cudaGetDevice(&cur));
    if (cur != e->device) CUDA_TRY(cudaSetDevice(e->device));
    return 0;
}

int copy_2d(mpdata_ensemble* e, int q, long long off, const void* src, void* dst, int where, bool put)
{
    const size_t w = (size_t)e->nx[q] * sizeof(float), dp = (size_t)e->px[q] * sizeof(float);
    cudaMemcpyKind kind = where == MPDATA_HOST ? (put ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost)
                                               : cudaMemcpyDeviceToDevice;
    if (put)
        CUDA_TRY(cudaMemcpy2DAsync(e->arena + off, dp, src, w, w, e->ny[q], kind, e->stream));
    else
        CUDA_TRY(cudaMemcpy2DAsync(dst, w, e->arena + off, dp, w, e->ny[q], kind, e->stream));
    return 0;
}

void destroy_ensemble(mpdata_ensemble* e)
{
    if (!e) return;
    cudaStreamSynchronize(e->stream);
    drop_graphs(e);
    for (int t = 0; t < kTiles; t++)
        for (int k = 0; k < 2; k++) cudaFree(e->items[t][k]);
    cudaFree(e->march_items);
    cudaFree(e->insts);
    cudaFree(e->arena);
    if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

}  // namespace

extern "C" {

int mpdata_ensemble_create(mpdata_ensemble_handle* out, int n, const int* nx, const int* ny,
                           int order, const mpdata_options* opts)
{
    if (!out || !nx || !ny || n < 1) return mpd::fail(MPDATA_ERR_ARG, "bad ensemble arguments");
    *out = nullptr;
    if (order < 1 || order > 64) return mpd::fail(MPDATA_ERR_ARG, "order %d outside 1..64", order);
    mpdata_options o;
    mpdata_default_options(&o);
    if (opts) o = *opts;
    if (o.approx_div && o.strict) return mpd::fail(MPDATA_ERR_ARG, "approx_div excludes strict");
    for (int q = 0; q < n; q++)
        if (nx[q] < 3 || ny[q] < 3)
            return mpd::fail(MPDATA_ERR_ARG, "instance %d: grid %dx%d, every dimension must be >= 3", q,
                             nx[q], ny[q]);
    std::unique_ptr<mpdata_ensemble> e(new mpdata_ensemble());
    e->n = n;
    e->order = order;
    e->opts = o;
    e->nx.assign(nx, nx + n);
    e->ny.assign(ny, ny + n);
    e->px.resize(n);
    e->have_field.assign(n, false);
    e->have_faces.assign(n, false);
    CUDA_TRY(cudaGetDevice(&e->device));
    CUDA_TRY(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    e->own_stream = true;
    long long total = 0;
    e->host_insts.resize(n);
    for (int q = 0; q < n; q++) {
        e->px[q] = (nx[q] + 31) / 32 * 32;
        const long long sz = (long long)e->px[q] * ny[q];
        mpd::EnsInst& I = e->host_insts[q];
        I.nx = nx[q]; I.ny = ny[q]; I.px = e->px[q]; I.pad = 0;
        for (int l = 0; l < 3; l++) { I.c[l] = total; total += sz; }
        for (int s = 0; s < 3; s++)
            for (int a = 0; a < 2; a++) { I.f[s][a] = total; total += sz; }
    }
    mpdata_ensemble* E = e.get();
    auto fail_destroy = [&](int rc) {
        destroy_ensemble(e.release());
        return rc;
    };
    if (cudaMalloc(&E->arena, (size_t)total * sizeof(float)) != cudaSuccess)
        return fail_destroy(mpd::fail(MPDATA_ERR_NOMEM, "ensemble arena of %lld floats", total));
    if (cudaMemsetAsync(E->arena, 0, (size_t)total * sizeof(float), E->stream) != cudaSuccess ||
        cudaMalloc(&E->insts, n * sizeof(mpd::EnsInst)) != cudaSuccess ||
        cudaMemcpy(E->insts, E->host_insts.data(), n * sizeof(mpd::EnsInst), cudaMemcpyHostToDevice) !=
            cudaSuccess)
        return fail_destroy(mpd::fail(MPDATA_ERR_CUDA, "ensemble set-up failed"));
    if (int rc = build_items(E)) return fail_destroy(rc);
    E->tile = 0;
    set_grid(E);
    *out = e.release();
    return 0;
}

int mpdata_ensemble_destroy(mpdata_ensemble_handle e)
{
    destroy_ensemble(e);
    return 0;
}

int mpdata_ensemble_set_stream(mpdata_ensemble_handle e, void* stream)
{
    if (!e) return mpd::fail(MPDATA_ERR_ARG, "null ensemble");
    if (int rc = ensure_device(e)) return rc;
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    if (e->own_stream) cudaStreamDestroy(e->stream);
    e->stream = (cudaStream_t)stream;
    e->own_stream = false;
    drop_graphs(e);
    return 0;
}

int mpdata_ensemble_set_faces(mpdata_ensemble_handle e, int q, const void* U, const void* V, int where)
{
    if (!e || q < 0 || q >= e->n || !U || !V) return mpd::fail(MPDATA_ERR_ARG, "bad arguments");
    if (int rc = ensure_device(e)) return rc;
    if (int rc = copy_2d(e, q, e->host_insts[q].f[0][0], U, nullptr, where, true)) return rc;
    if (int rc = copy_2d(e, q, e->host_insts[q].f[0][1], V, nullptr, where, true)) return rc;
    e->have_faces[q] = true;
    return 0;
}

int mpdata_ensemble_set_field(mpdata_ensemble_handle e, int q, const void* c, int where)
{
    if (!e || q < 0 || q >= e->n || !c) return mpd::fail(MPDATA_ERR_ARG, "bad arguments");
    if (int rc = ensure_device(e)) return rc;
    // Every instance's levels follow the ensemble's rotation: write all three
    // (the fixed shell must be in each of them).
    for (int l = 0; l < 3; l++)
        if (int rc = copy_2d(e, q, e->host_insts[q].c[l], c, nullptr, where, true)) return rc;
    e->have_field[q] = true;
    return 0;
}

int mpdata_ensemble_get_field(mpdata_ensemble_handle e, int q, void* c, int where)
{
    if (!e || q < 0 || q >= e->n || !c) return mpd::fail(MPDATA_ERR_ARG, "bad arguments");
    if (int rc = ensure_device(e)) return rc;
    if (int rc = copy_2d(e, q, e->host_insts[q].c[e->cur], nullptr, c, where, false)) return rc;
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return 0;
}

int mpdata_ensemble_step(mpdata_ensemble_handle e, int nsteps)
{
    if (!e || nsteps < 0) return mpd::fail(MPDATA_ERR_ARG, "bad arguments");
    for (int q = 0; q < e->n; q++)
        if (!e->have_field[q] || !e->have_faces[q])
            return mpd::fail(MPDATA_ERR_STATE, "instance %d has no field or faces", q);
    if (int rc = ensure_device(e)) return rc;
    if (nsteps == 0) return 0;
    // The legacy default stream cannot be captured: launch directly there.
    if (e->stream == nullptr) return run_steps_direct(e, nsteps);
    // One graph per (nsteps, starting level): the level rotation is baked in.
    GraphKey key{nsteps, e->cur};
    auto it = e->graphs.find(key);
    int cur = e->cur, prev = e->prev;
    if (it == e->graphs.end()) {
        cudaGraph_t g = nullptr;
        CUDA_TRY(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        for (int s = 0; s < nsteps; s++) {
            if (e->opts.strict) launch_step_passes<true>(e, cur, prev);
            else launch_step_passes<false>(e, cur, prev);
        }
        cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
        if (ce != cudaSuccess) return mpd::fail(MPDATA_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
        cudaGraphExec_t ex = nullptr;
        ce = cudaGraphInstantiate(&ex, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) return mpd::fail(MPDATA_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ce));
        it = e->graphs.emplace(key, ex).first;
    } else {
        for (int s = 0; s < nsteps; s++) {  // advance the rotation without launching
            const int P = e->order, b0 = cur, b1 = (b0 + 1) % 3, b2 = (b0 + 2) % 3;
            if (P == 1) { prev = b0; cur = b1; }
            else {
                int in = b1, out = b2;
                for (int o = 1; o < P; o++) std::swap(in, out);
                cur = in; prev = out;
            }
        }
    }
    CUDA_TRY(cudaGraphLaunch(it->second, e->stream));
    e->cur = cur;
    e->prev = prev;
    return 0;
}

int mpdata_ensemble_step_direct(mpdata_ensemble_handle e, int nsteps)
{
    if (!e || nsteps < 0) return mpd::fail(MPDATA_ERR_ARG, "bad arguments");
    if (int rc = ensure_device(e)) return rc;
    return run_steps_direct(e, nsteps);
}

int mpdata_ensemble_sync(mpdata_ensemble_handle e)
{
    if (!e) return mpd::fail(MPDATA_ERR_ARG, "null ensemble");
    if (int rc = ensure_device(e)) return rc;
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    CUDA_TRY(cudaGetLastError());
    return 0;
}

int mpdata_ensemble_autotune(mpdata_ensemble_handle e, int trial_steps, int* chosen, double* ms_per_step)
{
    if (!e || trial_steps < 1) return mpd::fail(MPDATA_ERR_ARG, "bad arguments");
    if (int rc = ensure_device(e)) return rc;
    // The trials step the instances: the fields must be set again afterwards.
    int cur0 = e->cur, prev0 = e->prev, best = e->tile;
    double best_ms = 1e300;
    cudaEvent_t a, b;
    CUDA_TRY(cudaEventCreate(&a));
    CUDA_TRY(cudaEventCreate(&b));
    for (int t = 0; t < kCandidates; t++) {
        e->tile = t;
        set_grid(e);
        run_steps_direct(e, 1);  // warm-up
        CUDA_TRY(cudaEventRecord(a, e->stream));
        run_steps_direct(e, trial_steps);
        CUDA_TRY(cudaEventRecord(b, e->stream));
        CUDA_TRY(cudaEventSynchronize(b));
        float ms = 0;
        CUDA_TRY(cudaEventElapsedTime(&ms, a, b));
        if (ms < best_ms) { best_ms = ms; best = t; }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    e->tile = best;
    set_grid(e);
    drop_graphs(e);
    // the trials stepped the instances; the caller re-sets the fields
    e->cur = cur0;
    e->prev = prev0;
    for (int q = 0; q < e->n; q++) e->have_field[q] = false;
    if (chosen) *chosen = best;
    if (ms_per_step) *ms_per_step = best_ms / trial_steps;
    return 0;
}

int mpdata_ensemble_tile(mpdata_ensemble_handle e, int tile)
{
    if (!e || tile < 0 || tile >= kCandidates) return mpd::fail(MPDATA_ERR_ARG, "bad tile %d", tile);
    e->tile = tile;
    set_grid(e);
    drop_graphs(e);
    return 0;
}

}  // extern "C"
