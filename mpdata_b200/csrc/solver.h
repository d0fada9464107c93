// Internal solver state shared by the C-ABI translation units.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <utility>
#include <vector>

#include "common.cuh"
#include "mpdata_b200.h"

namespace mpd {

struct Solver {
    int dtype = MPDATA_F32;
    size_t esz = 4;
    int order = 1;
    mpdata_options opts{};
    Dims d{};
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // Field levels: c[cur] is the newest, c[prev] the level before the last pass.
    void* c[3] = {nullptr, nullptr, nullptr};
    int cur = 0, prev = 0;
    // faces[0] = advective (constant between velocity updates), faces[1..2]
    // the Jacobi ping-pong of the antidiffusive passes; [axis] = U, V, W.
    void* faces[3][3] = {{nullptr}};
    void* bup = nullptr;  // limiter ratios (one-kernel-per-routine path only)
    void* bdn = nullptr;
    void* vel[6] = {nullptr};  // velocity staging for set_velocity
    void* metric = nullptr;    // dx | dy | ds
    double* red = nullptr;     // reduction partials
    int* dev_err = nullptr;    // device error word (bounded-wait timeouts in the fused pass)
    // TMA descriptors of the three field levels and the nine face arrays.
    CUtensorMap tm_c[3];
    CUtensorMap tm_f[3][3];
    // Two-cells-per-thread pass (FP32 fast arithmetic): its own descriptors (larger boxes).
    bool pair = false;
    CUtensorMap tm2_c[3];
    CUtensorMap tm2_f[3][3];
    bool have_field = false, have_faces = false;
    // faces[0] entries no pass reads (shell rows and planes) hold 0, as
    // k_courant writes them; set_faces may leave the caller's values there.
    bool faces0_clean = true;
    // A velocity update whose advective faces the next step's pass 0 forms
    // (fused with the donor update); materialize_faces() forms them earlier.
    bool vel_pending = false;
    double vel_dt = 0;
    const void* vel_dev[6] = {nullptr};  // staged velocity arrays (vel[]) or lent ones
    int zdepth = 0;  // fused kernels: planes per z chunk (set by the default heuristic / autotuner)
    // Pipelined host-array step: upload and download streams, chunk events.
    cudaStream_t s_up = nullptr, s_down = nullptr;
    std::vector<cudaEvent_t> pipe_ev;
    // Queued host copies (MPDATA_HOST_ASYNC): ticket t is fenced by fence_ev[t % kFences].
    static constexpr int kFences = 8;
    cudaEvent_t fence_ev[kFences] = {};
    int fence_n = 0;  // tickets issued
    // Optional per-pass event timing: pending event pairs per pass class.
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending[3];
    std::vector<cudaEvent_t> event_pool;
    double pass_ms[3] = {0, 0, 0};
    long long pass_n[3] = {0, 0, 0};
};

int fail(int code, const char* fmt, ...);

int create_solver(Solver** out, int nx, int ny, int ns, int dtype, int order,
                  const mpdata_options* opts);
void destroy_solver(Solver* h);
int set_velocity(Solver* h, const void* dx, const void* dy, const void* ds, double dt,
                 const void* const vel[6], int where);
int set_faces(Solver* h, const void* U, const void* V, const void* W, int where);
// Forms the advective faces of a pending velocity update now (no-op otherwise).
int materialize_faces(Solver* h);
int set_field(Solver* h, const void* c, int where);
int get_field(Solver* h, void* c, int where, bool previous);
int step(Solver* h, int nsteps);
// One step from host arrays (velocities vel[6], field c_in) to host arrays
// (newest, prev: the field before the last pass), pipelined over z chunks of
// `chunk` planes (0: automatic).  Fused kernels only.
int host_step_pipelined(Solver* h, const void* dx, const void* dy, const void* ds, double dt,
                        const void* const vel[6], const void* c_in, void* newest, void* prev,
                        int chunk);
int stats(Solver* h, double out[3]);
int check_device_error(Solver* h);  // synchronises; reports a kernel's recorded error
int launches(const Solver* h);

}  // namespace mpd
