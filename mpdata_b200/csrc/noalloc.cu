// mpdata_step_noalloc(): one MPDATA step on caller-provided device arrays
// that allocates no memory at all.
//
// Who needs it: callers that must not (or cannot) call cudaMalloc/cudaFree
// while they run -- code inside a CUDA stream capture, real-time loops whose
// memory is budgeted up front, plug-ins living in a host framework that owns
// the device allocator, and anything running after the device heap is full.
// The regular entry points allocate their buffers (solver handles, smolar()'s
// per-thread cache); this one keeps every intermediate field level, both
// pseudo-velocity face sets and the limiter ratios in the static device array
// below, which exists from the moment the library's device code is loaded.
//
// Limits and sharing:
//  * the scratch array holds kNoallocMaxFloats floats (32 MiB); a grid needs
//    10 * nx * ny * ns of them, so nx * ny * ns <= 838860 cells (for example
//    96 x 96 x 91, or 512 x 512 x 3); larger grids are rejected with
//    MPDATA_ERR_ARG and a message;
//  * every GPU that loads the library holds the 32 MiB until the process exits;
//  * every call on a device uses the same array and leaves its contents
//    behind; each call writes every scratch element it later reads, so nothing
//    has to start at zero, but calls that overlap on the GPU (different
//    streams, or host threads on the same device) race on the array: order
//    them on one stream or synchronise between them;
//  * the first call on each device looks up the array's device address
//    (cudaGetSymbolAddress, which may load the module); make that first call
//    outside any stream capture.
#include <cuda_runtime.h>

#include <mutex>

#include "launch.h"
#include "mpdata_b200.h"
#include "solver.h"

namespace {

constexpr size_t kNoallocMaxFloats = MPDATA_NOALLOC_MAX_FLOATS;
constexpr int kNoallocFields = 10;  // 2 field levels + 2 x 3 face arrays + 2 limiter ratios

// The scratch.  In host code this name is only a stand-in for the symbol;
// its device address comes from cudaGetSymbolAddress (see scratch_address).
static __device__ __align__(256) float g_noalloc_scratch[kNoallocMaxFloats];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
float* g_addr[kMaxDevices] = {nullptr};

int scratch_address(float** out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return mpd::fail(MPDATA_ERR_CUDA, "mpdata_step_noalloc: no usable current device");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return mpd::fail(MPDATA_ERR_CUDA, "mpdata_step_noalloc: cudaGetSymbolAddress: %s",
                             cudaGetErrorString(e));
        g_addr[dev] = static_cast<float*>(p);
    }
    *out = g_addr[dev];
    return 0;
}

}  // namespace

extern "C" int mpdata_step_noalloc(int nx, int ny, int ns, int order, int limiter,
                                   const float* U, const float* V, const float* W,
                                   const float* c_in, float* c_out, void* stream)
{
    if (nx < 3 || ny < 3 || ns < 3)
        return mpd::fail(MPDATA_ERR_ARG, "mpdata_step_noalloc: grid %dx%dx%d: every dimension must be >= 3",
                         nx, ny, ns);
    if (order < 1 || order > 64)
        return mpd::fail(MPDATA_ERR_ARG, "mpdata_step_noalloc: order %d outside 1..64", order);
    if (!U || !V || !W || !c_in || !c_out)
        return mpd::fail(MPDATA_ERR_ARG, "mpdata_step_noalloc: null array");
    if (c_out == c_in)
        return mpd::fail(MPDATA_ERR_ARG, "mpdata_step_noalloc: c_out must not alias c_in");
    const size_t cells = (size_t)nx * ny * ns;
    if (cells * kNoallocFields > kNoallocMaxFloats)
        return mpd::fail(MPDATA_ERR_ARG,
                         "mpdata_step_noalloc: grid %dx%dx%d needs %zu scratch floats, the static "
                         "scratch holds %zu (at most %zu cells)",
                         nx, ny, ns, cells * kNoallocFields, kNoallocMaxFloats,
                         kNoallocMaxFloats / kNoallocFields);
    float* base = nullptr;
    if (int rc = scratch_address(&base)) return rc;

    // Dense arrays (row pitch nx): the same layout as the caller's.
    mpd::Dims d{nx, ny, ns, nx, (long long)nx * ny};
    float* lvl[2] = {base, base + cells};
    float* fset[2][3] = {{base + 2 * cells, base + 3 * cells, base + 4 * cells},
                         {base + 5 * cells, base + 6 * cells, base + 7 * cells}};
    float* bup = base + 8 * cells;
    float* bdn = base + 9 * cells;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    // Pass o writes c_out when it is the last pass, else the level buffers in turn.
    auto dst = [&](int o) { return o == order - 1 ? c_out : lvl[o & 1]; };
    mpd::fast::launch_donor<float>(d, c_in, U, V, W, dst(0), 1, 0, 0, s);
    const float* in = dst(0);
    for (int o = 1; o < order; o++) {
        mpd::PassArgs<float> a{};
        a.c = in;
        a.cn = c_in;
        const float* const* prev = (o == 1) ? nullptr : fset[(o - 2) & 1];
        a.Uo = prev ? prev[0] : U;
        a.Vo = prev ? prev[1] : V;
        a.Wo = prev ? prev[2] : W;
        a.Vadv = V;
        a.Un = fset[(o - 1) & 1][0];
        a.Vn = fset[(o - 1) & 1][1];
        a.Wn = fset[(o - 1) & 1][2];
        a.c_out = dst(o);
        a.pass = o;
        a.use_div = 1;
        a.vv_fix = 0;
        a.limiter = limiter != 0;
        a.wide = 0;
        a.write_faces = 1;
        mpd::fast::launch_pass_unfused<float>(d, a, bup, bdn, s);
        in = dst(o);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return mpd::fail(MPDATA_ERR_CUDA, "mpdata_step_noalloc: launch failed: %s", cudaGetErrorString(e));
    return 0;
}
