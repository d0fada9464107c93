// Adjoint of a window of MPDATA steps with step checkpointing.
//
// Forward: steps c^0 -> c^N with the kernels of kernels_unfused.cuh, storing
// the field every `every` steps.  Backward: for each checkpoint segment, last
// first, the segment's steps are recomputed from its checkpoint with every
// intermediate kept (levels, raw and limited faces, limiter ratios), then the
// adjoint of each step is applied in reverse (kernels_adjoint.cuh), pass by
// pass, last pass first.  Memory: N/every checkpoints + one segment of step
// records, so long windows fit in HBM.  A full segment's launches (replay and
// reverse steps, on fixed buffers) are captured once as a CUDA graph and
// replayed for every full segment.
//
// The faces are steady (set once); the adjoint is with respect to the field.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
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

struct mpdata_adjoint {
    int dtype = MPDATA_F32, order = 2, every = 20, device = 0;
    size_t esz = 4;
    mpdata_options opts{};
    Dims d{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::vector<void*> blocks;  // every device allocation
    void* adv[3] = {nullptr, nullptr, nullptr};
    std::vector<void*> ckpt;    // checkpoint fields
    int nsteps = 0;             // length of the last forward window
    // Step records of one segment: per step, levels 0..P-1 and, per corrective
    // pass o = 1..P-1, raw faces R[o][3], limited faces L[o][3], ratios B[o][2].
    struct Record {
        std::vector<void*> lev;
        std::vector<std::array<void*, 3>> R, L;
        std::vector<std::array<void*, 2>> B;
    };
    std::vector<Record> rec;
    // Forward scratch: intermediate levels (work) and step outputs (tmp).
    void* work[2] = {nullptr, nullptr};
    void* tmp[2] = {nullptr, nullptr};
    // Adjoint buffers: levels 0..P, limited-face adjoints per pass, raw-face
    // adjoints, ratio adjoints.
    std::vector<void*> lam_lev;
    std::vector<std::array<void*, 3>> lam_L;
    void* lam_R[3] = {nullptr, nullptr, nullptr};
    void* lam_B[2] = {nullptr, nullptr};
    // The accumulators every adjoint step starts from zero share one
    // allocation, cleared by one memset per step: lam_L of the passes before
    // the last (later passes scatter into them) and, at its end, lam_B (the
    // ratio adjoints, scattered into by every pass and cleared again before
    // each earlier pass).  lam_lev[1..P-1], lam_L of the last pass and lam_R
    // are written (=) by each pass's first kernel and need no clearing.
    void* zblock = nullptr;
    size_t zblock_bytes = 0, zB_bytes = 0;
    bool have_faces = false;
    // A full segment of the backward sweep (replay + adjoint steps) as a CUDA
    // graph, captured on first use; one per parity of the adjoint buffers at
    // the segment's start (an odd interval swaps them segment by segment).
    cudaGraphExec_t seg_graph[2] = {nullptr, nullptr};
    cudaStream_t cap_stream = nullptr;  // private stream the capture records on
};

namespace {

size_t field_bytes(const mpdata_adjoint* h) { return (size_t)h->d.pp * h->d.ns * h->esz; }

int alloc_field(mpdata_adjoint* h, void** p)
{
    CUDA_TRY(cudaMalloc(p, field_bytes(h)));
    CUDA_TRY(cudaMemsetAsync(*p, 0, field_bytes(h), h->stream));
    h->blocks.push_back(*p);
    return 0;
}

int put(mpdata_adjoint* h, void* dst, const void* src, int where)
{
    const size_t w = (size_t)h->d.nx * h->esz;
    CUDA_TRY(cudaMemcpy2DAsync(dst, (size_t)h->d.px * h->esz, src, w, w, (size_t)h->d.ny * h->d.ns,
                               where == MPDATA_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                               h->stream));
    return 0;
}

int get(mpdata_adjoint* h, void* dst, const void* src, int where)
{
    const size_t w = (size_t)h->d.nx * h->esz;
    CUDA_TRY(cudaMemcpy2DAsync(dst, w, src, (size_t)h->d.px * h->esz, w, (size_t)h->d.ny * h->d.ns,
                               where == MPDATA_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                               h->stream));
    return 0;
}

// One forward step from `in` to `out`.  With a record, every intermediate
// is kept there (rec.lev[0] must already hold `in`); without one, the two
// work buffers and the record-0 face slots serve as scratch.
template <typename T>
void step_fwd(mpdata_adjoint* h, const T* in, T* out, mpdata_adjoint::Record* r)
{
    const Dims& d = h->d;
    const int P = h->order;
    mpdata_adjoint::Record& R = r ? *r : h->rec[0];
    const T* Fu = (const T*)h->adv[0];
    const T* Fv = (const T*)h->adv[1];
    const T* Fw = (const T*)h->adv[2];
    T* lev_prev = (T*)in;
    for (int o = 0; o < P; o++) {
        T* dst = (o == P - 1) ? out : (r ? (T*)R.lev[o + 1] : (T*)h->work[o & 1]);
        if (o == 0) {
            mpd::fast::launch_donor<T>(d, lev_prev, Fu, Fv, Fw, dst, 1, 0, 0, h->stream);
        } else {
            mpd::PassArgs<T> a{};
            a.c = lev_prev;
            a.cn = (const T*)in;
            a.Uo = Fu; a.Vo = Fv; a.Wo = Fw;
            a.Vadv = (const T*)h->adv[1];
            a.Un = (T*)R.L[o][0]; a.Vn = (T*)R.L[o][1]; a.Wn = (T*)R.L[o][2];
            a.c_out = dst;
            a.pass = o;
            a.use_div = h->opts.div_mode != MPDATA_DIV_OFF;
            a.vv_fix = h->opts.vv_fix;
            a.limiter = h->opts.limiter;
            a.wide = h->opts.precision_form;
            a.write_faces = 1;
            mpd::fast::launch_pass_record<T>(d, a, (T*)R.R[o][0], (T*)R.R[o][1], (T*)R.R[o][2],
                                             (T*)R.B[o][0], (T*)R.B[o][1], h->stream);
            Fu = (const T*)R.L[o][0]; Fv = (const T*)R.L[o][1]; Fw = (const T*)R.L[o][2];
        }
        lev_prev = dst;
    }
}

// Adjoint of one recorded step: lam_next (adjoint of its output) -> lam_prev.
template <typename T>
int step_adj(mpdata_adjoint* h, mpdata_adjoint::Record& R, const T* lam_next, T* lam_prev)
{
    const Dims& d = h->d;
    const int P = h->order;
    const size_t fb = field_bytes(h);
    // adjoint levels: lam_lev[P] = lam_next, lam_lev[0] = lam_prev (zeroed)
    std::vector<T*> L(P + 1);
    for (int o = 1; o < P; o++) L[o] = (T*)h->lam_lev[o];
    L[P] = (T*)lam_next;
    L[0] = lam_prev;
    CUDA_TRY(cudaMemsetAsync(L[0], 0, fb, h->stream));
    if (h->zblock) CUDA_TRY(cudaMemsetAsync(h->zblock, 0, h->zblock_bytes, h->stream));
    for (int o = P - 1; o >= 0; o--) {
        mpd::AdjPassArgs<T> a{};
        a.pass = o;
        a.accum_F = o < P - 1;
        a.limiter = h->opts.limiter;
        a.wide = h->opts.precision_form;
        a.use_div = h->opts.div_mode != MPDATA_DIV_OFF;
        a.vv_fix = h->opts.vv_fix;
        a.c = (const T*)R.lev[o];
        a.cn = (const T*)R.lev[0];
        a.lam_out = L[o + 1];
        a.lam_in = L[o];
        a.lam_cn = L[0];
        if (o == 0) {
            a.FU = (const T*)h->adv[0]; a.FV = (const T*)h->adv[1]; a.FW = (const T*)h->adv[2];
        } else {
            const auto& F = h->opts.limiter ? R.L[o] : R.R[o];
            a.FU = (const T*)F[0]; a.FV = (const T*)F[1]; a.FW = (const T*)F[2];
            a.lFU = (T*)h->lam_L[o][0]; a.lFV = (T*)h->lam_L[o][1]; a.lFW = (T*)h->lam_L[o][2];
            a.RU = (const T*)R.R[o][0]; a.RV = (const T*)R.R[o][1]; a.RW = (const T*)R.R[o][2];
            a.bup = (const T*)R.B[o][0]; a.bdn = (const T*)R.B[o][1];
            if (h->opts.limiter) {
                // cleared with the block for the step's last pass; again for earlier passes
                if (o != P - 1) CUDA_TRY(cudaMemsetAsync(h->lam_B[0], 0, h->zB_bytes, h->stream));
                a.lRU = (T*)h->lam_R[0]; a.lRV = (T*)h->lam_R[1]; a.lRW = (T*)h->lam_R[2];
                a.lbup = (T*)h->lam_B[0]; a.lbdn = (T*)h->lam_B[1];
            }
            if (o == 1) {
                a.Uo = (const T*)h->adv[0]; a.Vo = (const T*)h->adv[1]; a.Wo = (const T*)h->adv[2];
            } else {
                const auto& Fp = h->opts.limiter ? R.L[o - 1] : R.R[o - 1];
                a.Uo = (const T*)Fp[0]; a.Vo = (const T*)Fp[1]; a.Wo = (const T*)Fp[2];
                a.lUo = (T*)h->lam_L[o - 1][0]; a.lVo = (T*)h->lam_L[o - 1][1]; a.lWo = (T*)h->lam_L[o - 1][2];
            }
        }
        mpd::fast::launch_adj_pass<T>(d, a, h->stream);
    }
    CUDA_TRY(cudaGetLastError());
    return 0;
}

template <typename T> int forward_impl(mpdata_adjoint* h, const void* c0, int nsteps, void* cN, int where)
{
    // checkpoint seg = the input of step seg * every
    const int nseg = (nsteps + h->every - 1) / h->every;
    while ((int)h->ckpt.size() < nseg) {
        void* p;
        if (int rc = alloc_field(h, &p)) return rc;
        h->ckpt.push_back(p);
    }
    if (int rc = put(h, h->ckpt[0], c0, where)) return rc;
    T* cur = (T*)h->ckpt[0];
    for (int s = 0; s < nsteps; s++) {
        const int next = s + 1;
        T* out;
        if (next < nsteps && next % h->every == 0) out = (T*)h->ckpt[next / h->every];
        else out = (cur == (T*)h->tmp[0]) ? (T*)h->tmp[1] : (T*)h->tmp[0];
        step_fwd<T>(h, cur, out, nullptr);
        cur = out;
    }
    h->nsteps = nsteps;
    if (cN) {
        if (int rc = get(h, cN, cur, where)) return rc;
    }
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    CUDA_TRY(cudaGetLastError());
    return 0;
}

template <typename T> int backward_impl(mpdata_adjoint* h, const void* lamN, void* lam0, int where)
{
    const int N = h->nsteps, P = h->order;
    const size_t fb = field_bytes(h);
    T* lam_a = (T*)h->lam_lev[P];      // adjoint of the current step's output
    T* lam_b = (T*)h->lam_lev[P + 1];  // adjoint of its input
    if (int rc = put(h, lam_a, lamN, where)) return rc;
    const int nseg = (N + h->every - 1) / h->every;
    // recompute a segment from its checkpoint (staged in rec[0].lev[0]),
    // keeping every intermediate, then apply its adjoint, last step first
    auto segment = [&](int len) -> int {
        for (int t = 0; t < len; t++) {
            T* out = (t + 1 < len) ? (T*)h->rec[t + 1].lev[0] : (T*)h->tmp[0];
            step_fwd<T>(h, (const T*)h->rec[t].lev[0], out, &h->rec[t]);
        }
        for (int t = len - 1; t >= 0; t--) {
            if (int rc = step_adj<T>(h, h->rec[t], lam_a, lam_b)) return rc;
            std::swap(lam_a, lam_b);
        }
        return 0;
    };
    for (int seg = nseg - 1; seg >= 0; seg--) {
        const int len = std::min(h->every, N - seg * h->every);
        CUDA_TRY(cudaMemcpyAsync(h->rec[0].lev[0], h->ckpt[seg], fb, cudaMemcpyDeviceToDevice, h->stream));
        if (len < h->every) {  // a short last segment: launched directly
            if (int rc = segment(len)) return rc;
            continue;
        }
        // full segments: the same launches on the same buffers every time,
        // replayed from one captured graph (hundreds of launches -> one)
        const int par = (lam_a == (T*)h->lam_lev[P]) ? 0 : 1;
        if (!h->seg_graph[par]) {
            // recorded on a private stream (the caller's may be the legacy
            // default stream, which cannot be captured), launched on the caller's
            if (!h->cap_stream)
                CUDA_TRY(cudaStreamCreateWithFlags(&h->cap_stream, cudaStreamNonBlocking));
            cudaStream_t user = h->stream;
            h->stream = h->cap_stream;
            cudaError_t eb = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
            if (eb != cudaSuccess) {
                h->stream = user;
                return mpd::fail(MPDATA_ERR_CUDA, "segment capture: %s", cudaGetErrorString(eb));
            }
            const int rc = segment(len);  // swaps lam_a / lam_b as the graph will
            cudaGraph_t g = nullptr;
            const cudaError_t ec = cudaStreamEndCapture(h->stream, &g);
            h->stream = user;
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            if (ec != cudaSuccess)
                return mpd::fail(MPDATA_ERR_CUDA, "segment capture: %s", cudaGetErrorString(ec));
            const cudaError_t ei = cudaGraphInstantiate(&h->seg_graph[par], g, 0);
            cudaGraphDestroy(g);
            if (ei != cudaSuccess) {
                h->seg_graph[par] = nullptr;
                return mpd::fail(MPDATA_ERR_CUDA, "segment graph: %s", cudaGetErrorString(ei));
            }
        } else if (len & 1) {
            std::swap(lam_a, lam_b);
        }
        CUDA_TRY(cudaGraphLaunch(h->seg_graph[par], h->stream));
    }
    if (int rc = get(h, lam0, lam_a, where)) return rc;
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    CUDA_TRY(cudaGetLastError());
    return 0;
}

void destroy(mpdata_adjoint* h)
{
    if (!h) return;
    cudaStreamSynchronize(h->stream);
    for (cudaGraphExec_t g : h->seg_graph)
        if (g) cudaGraphExecDestroy(g);
    if (h->cap_stream) cudaStreamDestroy(h->cap_stream);
    for (void* p : h->blocks) cudaFree(p);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

}  // namespace

extern "C" {

int mpdata_adjoint_create(mpdata_adjoint_handle* out, int nx, int ny, int ns, int dtype, int order,
                          const mpdata_options* opts, int checkpoint_every)
{
    if (!out) return mpd::fail(MPDATA_ERR_ARG, "null handle pointer");
    *out = nullptr;
    if (nx < 3 || ny < 3 || ns < 3) return mpd::fail(MPDATA_ERR_ARG, "every dimension must be >= 3");
    if (dtype != MPDATA_F32 && dtype != MPDATA_F64) return mpd::fail(MPDATA_ERR_ARG, "bad dtype");
    if (order < 1 || order > 16) return mpd::fail(MPDATA_ERR_ARG, "order %d outside 1..16", order);
    if (checkpoint_every < 1) return mpd::fail(MPDATA_ERR_ARG, "checkpoint interval must be >= 1");
    std::unique_ptr<mpdata_adjoint> h(new mpdata_adjoint());
    h->dtype = dtype;
    h->esz = dtype == MPDATA_F32 ? 4 : 8;
    h->order = order;
    h->every = checkpoint_every;
    if (opts) h->opts = *opts;
    if (h->opts.precision_form && dtype != MPDATA_F32)
        return mpd::fail(MPDATA_ERR_ARG, "precision_form applies to float storage only");
    h->d.nx = nx; h->d.ny = ny; h->d.ns = ns;
    h->d.px = ((long long)nx + 31) / 32 * 32;
    h->d.pp = h->d.px * ny;
    CUDA_TRY(cudaGetDevice(&h->device));
    CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
    mpdata_adjoint* H = h.get();
    auto A = [&](void** p) { return alloc_field(H, p); };
    int rc = 0;
    for (int a = 0; a < 3 && !rc; a++) rc = A(&H->adv[a]);
    for (int a = 0; a < 2 && !rc; a++) rc = A(&H->work[a]);
    for (int a = 0; a < 2 && !rc; a++) rc = A(&H->tmp[a]);
    H->rec.resize(checkpoint_every);
    for (auto& R : H->rec) {
        R.lev.resize(order);
        R.R.resize(order);
        R.L.resize(order);
        R.B.resize(order);
        for (int l = 0; l < order && !rc; l++) rc = A(&R.lev[l]);
        for (int o = 1; o < order && !rc; o++) {
            for (int a = 0; a < 3 && !rc; a++) rc = A(&R.R[o][a]);
            if (H->opts.limiter) {
                for (int a = 0; a < 3 && !rc; a++) rc = A(&R.L[o][a]);
                for (int a = 0; a < 2 && !rc; a++) rc = A(&R.B[o][a]);
            } else {
                R.L[o] = R.R[o];
                R.B[o] = {nullptr, nullptr};
            }
        }
    }
    H->lam_lev.resize(order + 2);
    H->lam_L.resize(order);
    const size_t fb = field_bytes(H);
    for (int o = 1; o < order && !rc; o++) rc = A(&H->lam_lev[o]);
    if (order > 1)
        for (int a = 0; a < 3 && !rc; a++) rc = A(&H->lam_L[order - 1][a]);
    if (H->opts.limiter)
        for (int a = 0; a < 3 && !rc; a++) rc = A(&H->lam_R[a]);
    const int nz = 3 * std::max(order - 2, 0) + (H->opts.limiter ? 2 : 0);
    if (!rc && nz > 0) {
        if (cudaMalloc(&H->zblock, nz * fb) != cudaSuccess) {
            rc = mpd::fail(MPDATA_ERR_CUDA, "adjoint allocation failed");
        } else {
            H->blocks.push_back(H->zblock);
            H->zblock_bytes = nz * fb;
            char* z = (char*)H->zblock;
            for (int o = 1; o < order - 1; o++)
                for (int a = 0; a < 3; a++) { H->lam_L[o][a] = z; z += fb; }
            if (H->opts.limiter) {
                H->zB_bytes = 2 * fb;
                for (int a = 0; a < 2; a++) { H->lam_B[a] = z; z += fb; }
            }
        }
    }
    if (!rc) rc = A(&H->lam_lev[0]);
    if (!rc) rc = A(&H->lam_lev[order]);
    if (!rc) rc = A(&H->lam_lev[order + 1]);
    if (rc) {
        destroy(h.release());
        return rc == MPDATA_ERR_CUDA ? mpd::fail(MPDATA_ERR_NOMEM, "adjoint allocation failed") : rc;
    }
    *out = h.release();
    return 0;
}

int mpdata_adjoint_destroy(mpdata_adjoint_handle h)
{
    destroy(h);
    return 0;
}

int mpdata_adjoint_set_faces(mpdata_adjoint_handle h, const void* U, const void* V, const void* W,
                             int where)
{
    if (!h || !U || !V || !W) return mpd::fail(MPDATA_ERR_ARG, "null argument");
    const void* src[3] = {U, V, W};
    for (int a = 0; a < 3; a++)
        if (int rc = put(h, h->adv[a], src[a], where)) return rc;
    h->have_faces = true;
    return 0;
}

int mpdata_adjoint_forward(mpdata_adjoint_handle h, const void* c0, int nsteps, void* cN, int where)
{
    if (!h || !c0 || nsteps < 1) return mpd::fail(MPDATA_ERR_ARG, "bad arguments");
    if (!h->have_faces) return mpd::fail(MPDATA_ERR_STATE, "faces not set");
    return h->dtype == MPDATA_F32 ? forward_impl<float>(h, c0, nsteps, cN, where)
                                  : forward_impl<double>(h, c0, nsteps, cN, where);
}

int mpdata_adjoint_backward(mpdata_adjoint_handle h, const void* lamN, void* lam0, int where)
{
    if (!h || !lamN || !lam0) return mpd::fail(MPDATA_ERR_ARG, "bad arguments");
    if (h->nsteps < 1) return mpd::fail(MPDATA_ERR_STATE, "no forward window to differentiate");
    return h->dtype == MPDATA_F32 ? backward_impl<float>(h, lamN, lam0, where)
                                  : backward_impl<double>(h, lamN, lam0, where);
}

int mpdata_adjoint_set_stream(mpdata_adjoint_handle h, void* stream)
{
    if (!h) return mpd::fail(MPDATA_ERR_ARG, "null handle");
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (h->own_stream) cudaStreamDestroy(h->stream);
    h->stream = (cudaStream_t)stream;
    h->own_stream = false;
    return 0;
}

}  // extern "C"
