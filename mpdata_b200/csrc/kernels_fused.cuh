// Fused corrective pass: antidiffusive faces (+ nonoscillatory limiter) and
// the donor-cell update of one MPDATA pass in one kernel, z-marching.
//
// Work decomposition.  A CTA of 32 x 16 threads covers a 32 x 16 column of
// cells and marches it through z.  Each thread owns one cell of the column:
// per plane it forms the cell's three high faces (x, y and the z face above)
// and, with the limiter, the cell's in/out ratios; then it applies the
// donor-cell update.  Without the limiter every cell of the CTA is updated;
// with it the outer ring of the CTA is a halo (30 x 14 cells updated) whose
// faces and ratios the limited faces of the updated cells need.  The first
// warps also form the faces just below the column (x face at local x = -1, y
// face at local y = -1), which the lowest cells read.
//
// Staging.  The pass input c, the step input c^n (limiter bounds) and the
// previous pass's faces U, V, W are brought in one plane at a time by TMA
// (cp.async.bulk.tensor, 40 x 19 element boxes, zero-filled outside the grid)
// into a four-deep ring of shared-memory stages, two planes ahead of the
// plane being computed; one mbarrier per stage.  The box starts on a 16-byte
// boundary in x (its low edge is rounded down and the slack is skipped).
//
// z dependence.  The cell's own c values of the neighbouring planes and its
// own z faces live in registers from one plane to the next.  With the
// limiter, the limited z face above a cell needs the ratios of the cell
// above, so the update trails the face computation by one plane; the limited
// x and y faces of a plane are kept (registers + a two-plane ring in shared
// memory for the neighbours) until the update of that plane.
//
// Arithmetic: identical formulas and evaluation order as kernels_unfused.cuh
// (the reference's, see there for file:line citations).
//
// Included by kernels_all.cuh inside namespace mpd::MPD_NS.

namespace fused {

constexpr int BX = 32, BY = 16, NT = BX * BY;
constexpr int SBX = kBoxX, SBY = kBoxY;      // staged plane box
constexpr int NSTAGE = 4;
constexpr int WX = BX + 2, WY = BY + 2, WPL = WX * WY;  // work planes: local [-1,32] x [-1,16]

template <typename T> __host__ __device__ constexpr int stage_bytes()
{
    return (SBX * SBY * (int)sizeof(T) + 127) / 128 * 128;
}
template <bool LIM> __host__ __device__ constexpr int n_arrays() { return LIM ? 5 : 4; }
template <bool LIM> __host__ __device__ constexpr int n_work() { return LIM ? 8 : 2; }
template <typename T, bool LIM> __host__ __device__ constexpr size_t smem_bytes()
{
    return (size_t)NSTAGE * n_arrays<LIM>() * stage_bytes<T>() + (size_t)n_work<LIM>() * WPL * sizeof(T) +
           NSTAGE * sizeof(uint64_t);
}

// The staged planes one face computation reads (pointers into stage slots).
template <typename T> struct Planes {
    const T *c_m, *c_0, *c_p;     // c at planes k-1, k, k+1
    const T *uo_0, *uo_p;         // previous x faces, planes k, k+1
    const T *vo_0, *vo_p;         // previous y faces, planes k, k+1
    const T *wo_m, *wo_0, *wo_p;  // previous z faces, face-planes k-1, k, k+1
};

struct FaceCtx {
    int nx, ny, ns, use_div, vv_fix, pass;
};

// x face between cells i and i+1 (row j, plane k); o = staged offset of cell i.
template <typename T>
__device__ __forceinline__ T face_u(const Planes<T>& P, int o, int i, const FaceCtx& f)
{
    constexpr int Y = SBX;
    T vb, wb, neg_div = T(0);
    if (i == 0 || i == f.nx - 2) {
        const int a = (i == 0) ? o + 1 : o;
        vb = T(0.5) * (P.vo_0[a - Y] + P.vo_0[a]);
        wb = T(0.5) * (P.wo_m[a] + P.wo_0[a]);
    } else {
        vb = T(0.25) * (((P.vo_0[o + 1 - Y] + P.vo_0[o + 1]) + P.vo_0[o]) + P.vo_0[o - Y]);
        wb = T(0.25) * (((P.wo_m[o + 1] + P.wo_0[o + 1]) + P.wo_0[o]) + P.wo_m[o]);
        if (f.use_div) {
            T s = P.uo_0[o + 1] - P.uo_0[o - 1];
            s = s + P.vo_0[o + 1 - Y];
            s = s - P.vo_0[o + 1];
            s = s - P.vo_0[o];
            s = s + P.vo_0[o - Y];
            s = s + P.wo_m[o + 1];
            s = s - P.wo_0[o + 1];
            s = s - P.wo_0[o];
            s = s + P.wo_m[o];
            neg_div = -((T(0.25) * P.uo_0[o]) * s);
        } else {
            neg_div = -T(0);
        }
    }
    T n1, d1, n2, d2;
    grad_pair(P.c_0[o + 1 + Y], P.c_0[o + Y], P.c_0[o - Y], P.c_0[o + 1 - Y], n1, d1);
    grad_pair(P.c_p[o + 1], P.c_p[o], P.c_m[o], P.c_m[o + 1], n2, d2);
    return face_pattern(neg_div, P.uo_0[o], P.c_0[o], P.c_0[o + 1], vb, n1, d1, wb, n2, d2);
}

// y face between rows j and j+1 (column i, plane k).
template <typename T>
__device__ __forceinline__ T face_v(const Planes<T>& P, int o, int i, int j, int k,
                                   const FaceCtx& f, const Dims& d, const T* __restrict__ Vadv)
{
    constexpr int Y = SBX;
    T ub, wb, neg_div = T(0);
    if (j == 0 || j == f.ny - 2) {
        const int a = (j == 0) ? o + Y : o;
        ub = T(0.5) * (P.uo_0[a - 1] + P.uo_0[a]);
        wb = T(0.5) * (P.wo_m[a] + P.wo_0[a]);
    } else {
        if (i == 1 && !f.vv_fix)  // the column vv_pass never writes (vv.c:81-82)
            return (f.pass & 1) ? T(0) : Vadv[cell(d, 1, j, k)];
        ub = T(0.25) * (((P.uo_0[o - 1 + Y] + P.uo_0[o + Y]) + P.uo_0[o]) + P.uo_0[o - 1]);
        wb = T(0.25) * (((P.wo_m[o + Y] + P.wo_0[o + Y]) + P.wo_0[o]) + P.wo_m[o]);
        if (f.use_div) {
            const T ul2u = (i >= 2) ? P.uo_0[o - 2 + Y] : T(0);
            const T ul2 = (i >= 2) ? P.uo_0[o - 2] : T(0);
            T s = P.vo_0[o + Y] - P.vo_0[o - Y];
            s = s + P.wo_m[o + Y];
            s = s - P.wo_0[o + Y];
            s = s - P.wo_0[o];
            s = s + P.wo_m[o];
            s = s + P.uo_0[o - 1 + Y];
            s = s - ul2u;
            s = s - ul2;
            s = s + P.uo_0[o - 1];
            neg_div = -((T(0.25) * P.vo_0[o]) * s);
        } else {
            neg_div = -T(0);
        }
    }
    T n1, d1, n2, d2;
    grad_pair(P.c_0[o + 1 + Y], P.c_0[o + 1], P.c_0[o - 1], P.c_0[o - 1 + Y], n1, d1);
    grad_pair(P.c_p[o + Y], P.c_p[o], P.c_m[o], P.c_m[o + Y], n2, d2);
    return face_pattern(neg_div, P.vo_0[o], P.c_0[o], P.c_0[o + Y], ub, n1, d1, wb, n2, d2);
}

// z face between planes k and k+1 (cell column i, j).
template <typename T>
__device__ __forceinline__ T face_w(const Planes<T>& P, int o, int k, const FaceCtx& f)
{
    constexpr int Y = SBX;
    T ub, vb, neg_div = T(0);
    if (k == 0 || k == f.ns - 2) {
        const T* U = (k == 0) ? P.uo_p : P.uo_0;  // the interior plane next to the face
        const T* V = (k == 0) ? P.vo_p : P.vo_0;
        ub = T(0.5) * (U[o - 1] + U[o]);
        vb = T(0.5) * (V[o - Y] + V[o]);
    } else {
        ub = T(0.25) * (((P.uo_0[o] + P.uo_p[o]) + P.uo_p[o - 1]) + P.uo_0[o - 1]);
        vb = T(0.25) * (((P.vo_p[o - Y] + P.vo_p[o]) + P.vo_0[o]) + P.vo_0[o - Y]);
        if (f.use_div) {
            T s = P.wo_p[o] - P.wo_m[o];
            s = s + P.uo_p[o - 1];
            s = s - P.uo_p[o];
            s = s - P.uo_0[o];
            s = s + P.uo_0[o - 1];
            s = s + P.vo_p[o - Y];
            s = s - P.vo_p[o];
            s = s - P.vo_0[o];
            s = s + P.vo_0[o - Y];
            neg_div = -((T(0.25) * P.wo_0[o]) * s);
        } else {
            neg_div = -T(0);
        }
    }
    T n1, d1, n2, d2;
    grad_pair(P.c_p[o + 1], P.c_0[o + 1], P.c_0[o - 1], P.c_p[o - 1], n1, d1);
    grad_pair(P.c_p[o + Y], P.c_0[o + Y], P.c_0[o - Y], P.c_p[o - Y], n2, d2);
    return face_pattern(neg_div, P.wo_0[o], P.c_0[o], P.c_p[o], ub, n1, d1, vb, n2, d2);
}

}  // namespace fused

template <typename T, bool LIM, typename A>
__global__ void __launch_bounds__(fused::NT, sizeof(T) == 4 ? 2 : 1)
    k_pass_tma(Dims d, PassArgs<T> a, const __grid_constant__ CUtensorMap map_c,
               const __grid_constant__ CUtensorMap map_cn, const __grid_constant__ CUtensorMap map_uo,
               const __grid_constant__ CUtensorMap map_vo, const __grid_constant__ CUtensorMap map_wo)
{
    using namespace fused;
    constexpr int NARR = n_arrays<LIM>();
    constexpr int SB = stage_bytes<T>();
    constexpr int Y = SBX;
    extern __shared__ __align__(128) unsigned char smem[];
    T* work = reinterpret_cast<T*>(smem + (size_t)NSTAGE * NARR * SB);
    T* sRU = work;              // raw x faces of plane k
    T* sRV = sRU + WPL;         // raw y faces of plane k
    T* sBU = sRV + WPL;         // limiter ratios of plane k
    T* sBD = sBU + WPL;
    T* sLU = sBD + WPL;         // limited x faces, planes k-1 / k (two slots)
    T* sLV = sLU + 2 * WPL;     // limited y faces, two slots
    uint64_t* bars = reinterpret_cast<uint64_t*>(work + n_work<LIM>() * WPL);
    auto box = [&](int p, int arr) -> const T* {
        return reinterpret_cast<const T*>(smem + (size_t)((p & (NSTAGE - 1)) * NARR + arr) * SB);
    };

    const int nx = d.nx, ny = d.ny, ns = d.ns;
    const int x = threadIdx.x, y = threadIdx.y, tid = y * BX + x;
    constexpr int OW = LIM ? 1 : 0;  // halo ring width
    const int i0 = 1 + (int)blockIdx.x * (BX - 2 * OW) - OW;  // global i of local x = 0
    const int j0 = 1 + (int)blockIdx.y * (BY - 2 * OW) - OW;
    constexpr int ALIGN = 16 / (int)sizeof(T);                // TMA: x * size multiple of 16 B
    const int gx0 = (i0 - 2) & ~(ALIGN - 1);
    const int gy0 = j0 - 2;
    const int rx = (i0 - 2) - gx0;
    const int o = (y + 2) * Y + (x + 2 + rx);   // own cell in a staged plane
    const int w = (y + 1) * WX + (x + 1);       // own cell in a work plane
    const int i = i0 + x, j = j0 + y;
    const FaceCtx fc{nx, ny, ns, a.use_div, a.vv_fix, a.pass};
    const bool cell_in = i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2;
    const bool owned = cell_in && (!LIM || (x >= 1 && x <= BX - 2 && y >= 1 && y <= BY - 2));

    if (tid == 0) {
        for (int s = 0; s < NSTAGE; s++) tma::mbar_init(&bars[s], 1);
        tma::fence_barrier_init();
        tma::prefetch_map(&map_c);
        tma::prefetch_map(&map_uo);
        tma::prefetch_map(&map_vo);
        tma::prefetch_map(&map_wo);
        if (LIM) tma::prefetch_map(&map_cn);
    }
    __syncthreads();

    auto issue = [&](int p) {  // one elected thread: stage plane p of every array
        uint64_t* bar = &bars[p & (NSTAGE - 1)];
        tma::fence_proxy_async_shared();
        tma::mbar_arrive_expect_tx(bar, (uint32_t)(NARR * SBX * SBY * sizeof(T)));
        T* dst = const_cast<T*>(box(p, 0));
        tma::load_3d(dst, &map_c, gx0, gy0, p, bar);
        tma::load_3d(const_cast<T*>(box(p, 1)), &map_uo, gx0, gy0, p, bar);
        tma::load_3d(const_cast<T*>(box(p, 2)), &map_vo, gx0, gy0, p, bar);
        tma::load_3d(const_cast<T*>(box(p, 3)), &map_wo, gx0, gy0, p, bar);
        if (LIM) tma::load_3d(const_cast<T*>(box(p, 4)), &map_cn, gx0, gy0, p, bar);
    };
    auto planes = [&](int k) {
        Planes<T> P;
        P.c_m = box(k - 1, 0); P.c_0 = box(k, 0); P.c_p = box(k + 1, 0);
        P.uo_0 = box(k, 1); P.uo_p = box(k + 1, 1);
        P.vo_0 = box(k, 2); P.vo_p = box(k + 1, 2);
        P.wo_m = box(k - 1, 3); P.wo_0 = box(k, 3); P.wo_p = box(k + 1, 3);
        return P;
    };

    bool ok = true;
    int confirmed = 0;  // planes whose stage thread 0 has seen complete
    if (tid == 0) {
        issue(0);
        issue(1);
    }
    ok = tma::mbar_wait(&bars[0], 0);
    if (tid == 0 && ok) confirmed = 1;

    // Register state carried between planes.
    T cq0 = T(0), cq1 = T(0), cq2 = ok ? box(0, 0)[o] : T(0), cq3 = T(0);  // own c, planes k-2..k+1
    T rw_prev = T(0);                      // raw z face below (face-plane k-1)
    T bu_prev = T(1), bd_prev = T(1);      // own ratios of plane k-1
    T lu_prev = T(0), lv_prev = T(0), lw_prev = T(0);  // limited faces of plane k-1 / face-plane k-2

    const int last = LIM ? ns - 1 : ns - 2;
    for (int k = 0; k <= last; k++) {
        __syncthreads();  // every read of the slot plane k+2 reuses is done
        if (tid == 0 && k + 2 <= ns - 1) issue(k + 2);
        if (k + 1 <= ns - 1) {
            if (ok) ok = tma::mbar_wait(&bars[(k + 1) & (NSTAGE - 1)], ((k + 1) / NSTAGE) & 1);
            if (tid == 0 && ok) confirmed = k + 2;
            cq3 = box(k + 1, 0)[o];
        }
        const bool kin = k >= 1 && k <= ns - 2;

        // ---- raw faces of plane k (z face: face-plane k) ----
        T ru = T(0), rv = T(0), rw = T(0);
        if (k <= ns - 2) {
            const Planes<T> P = planes(k);
            if (kin && i >= 0 && i <= nx - 2 && j >= 1 && j <= ny - 2) ru = face_u(P, o, i, fc);
            if (kin && i >= 1 && i <= nx - 2 && j >= 0 && j <= ny - 2)
                rv = face_v(P, o, i, j, k, fc, d, a.Vadv);
            if (cell_in) rw = face_w(P, o, k, fc);
            sRU[w] = ru;
            sRV[w] = rv;
            if (tid < BY) {  // x faces just left of the column
                const int ye = tid, ie = i0 - 1, je = j0 + ye;
                T v = T(0);
                if (kin && ie >= 0 && ie <= nx - 2 && je >= 1 && je <= ny - 2)
                    v = face_u(P, (ye + 2) * Y + (1 + rx), ie, fc);
                sRU[(ye + 1) * WX] = v;
            } else if (tid < BY + BX) {  // y faces just below the column
                const int xe = tid - BY, ie = i0 + xe, je = j0 - 1;
                T v = T(0);
                if (kin && ie >= 1 && ie <= nx - 2 && je >= 0 && je <= ny - 2)
                    v = face_v(P, Y + (xe + 2 + rx), ie, je, k, fc, d, a.Vadv);
                sRV[xe + 1] = v;
            }
        }
        __syncthreads();

        if (LIM) {
            // ---- limiter ratios of plane k ----
            T bu = T(1), bd = T(1);
            if (kin && cell_in) {
                const T* c0 = box(k, 0);
                const T* n0 = box(k, 4);
                const T psi = cq2;
                T mx = psi, mn = psi, t;
#define MPD_BOUND(v) do { t = (v); mx = t > mx ? t : mx; mn = t < mn ? t : mn; } while (0)
                MPD_BOUND(n0[o]);
                MPD_BOUND(c0[o - 1]); MPD_BOUND(n0[o - 1]);
                MPD_BOUND(c0[o + 1]); MPD_BOUND(n0[o + 1]);
                MPD_BOUND(c0[o - Y]); MPD_BOUND(n0[o - Y]);
                MPD_BOUND(c0[o + Y]); MPD_BOUND(n0[o + Y]);
                if (ns > 3) {
                    MPD_BOUND(cq1); MPD_BOUND(box(k - 1, 4)[o]);
                    MPD_BOUND(cq3); MPD_BOUND(box(k + 1, 4)[o]);
                }
#undef MPD_BOUND
                A fin = A(0), fout = A(0);
                lim_acc(lim_flux<T, A>(sRU[w - 1], c0[o - 1], psi), false, fin, fout);
                lim_acc(lim_flux<T, A>(ru, psi, c0[o + 1]), true, fin, fout);
                lim_acc(lim_flux<T, A>(sRV[w - WX], c0[o - Y], psi), false, fin, fout);
                lim_acc(lim_flux<T, A>(rv, psi, c0[o + Y]), true, fin, fout);
                lim_acc(lim_flux<T, A>(rw_prev, cq1, psi), false, fin, fout);
                lim_acc(lim_flux<T, A>(rw, psi, cq3), true, fin, fout);
                bu = T((A(mx) - A(psi)) / (fin + lim_tiny<A>()));
                bd = T((A(psi) - A(mn)) / (fout + lim_tiny<A>()));
            }
            sBU[w] = bu;
            sBD[w] = bd;
            __syncthreads();

            // ---- limited faces: x, y of plane k; z of face-plane k-1 ----
            T lu = ru, lv = rv;
            if (x < BX - 1) lu = limit_face(ru, bu, bd, sBU[w + 1], sBD[w + 1]);
            if (y < BY - 1) lv = limit_face(rv, bu, bd, sBU[w + WX], sBD[w + WX]);
            const T lw = limit_face(rw_prev, bu_prev, bd_prev, bu, bd);
            sLU[(k & 1) * WPL + w] = lu;
            sLV[(k & 1) * WPL + w] = lv;
            if (a.write_faces) {
                const bool ox = x >= 1 && x <= BX - 2, oy = y >= 1 && y <= BY - 2;
                const long long q = cell(d, i, j, k);
                if (kin && i >= 0 && i <= nx - 2 && j >= 1 && j <= ny - 2 && oy && (ox || i == 0))
                    a.Un[q] = lu;
                if (kin && i >= 1 && i <= nx - 2 && j >= 0 && j <= ny - 2 && ox && (oy || j == 0))
                    a.Vn[q] = lv;
                if (k >= 1 && owned) a.Wn[q - d.pp] = lw;
            }

            // ---- donor update of plane k-1 ----
            const int u = k - 1;
            if (u >= 1 && u <= ns - 2 && owned) {
                const T* cu = box(u, 0);
                const T ul = sLU[(u & 1) * WPL + w - 1];
                const T vb = sLV[(u & 1) * WPL + w - WX];
                a.c_out[cell(d, i, j, u)] =
                    donor_update(cu[o], cu[o - 1], cu[o + 1], cu[o - Y], cu[o + Y], cq0, cq2, lu_prev,
                                 ul, lv_prev, vb, lw, lw_prev);
            }
            lu_prev = lu;
            lv_prev = lv;
            lw_prev = lw;
            bu_prev = bu;
            bd_prev = bd;
        } else {
            // ---- donor update of plane k ----
            if (kin && owned) {
                const T* c0 = box(k, 0);
                const T ul = sRU[w - 1], vb = sRV[w - WX];
                const long long q = cell(d, i, j, k);
                a.c_out[q] = donor_update(c0[o], c0[o - 1], c0[o + 1], c0[o - Y], c0[o + Y], cq1,
                                          cq3, ru, ul, rv, vb, rw, rw_prev);
                if (a.write_faces) {
                    a.Un[q] = ru;
                    a.Vn[q] = rv;
                    a.Wn[q] = rw;
                    if (i == 1) a.Un[q - 1] = ul;
                    if (j == 1) a.Vn[q - d.px] = vb;
                    if (k == 1) a.Wn[q - d.pp] = rw_prev;
                }
            }
        }
        rw_prev = rw;
        cq0 = cq1;
        cq1 = cq2;
        cq2 = cq3;
    }

    if (!ok && a.err) atomicOr(a.err, 1);
    if (tid == 0) {  // never leave with a copy in flight
        for (int p = confirmed; p <= ns - 1 && p <= last + 1; p++)
            if (!tma::mbar_wait(&bars[p & (NSTAGE - 1)], (p / NSTAGE) & 1)) break;
    }
}

template <typename T, bool LIM, typename A>
int launch_fused_variant(const Dims& d, const PassArgs<T>& a, cudaStream_t s)
{
    using namespace fused;
    constexpr size_t smem = smem_bytes<T, LIM>();
    static bool configured = false;  // the attribute is per device function
    if (!configured) {
        cudaFuncSetAttribute(k_pass_tma<T, LIM, A>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        configured = true;
    }
    constexpr int OW = LIM ? 1 : 0;
    dim3 g((d.nx - 2 + BX - 2 * OW - 1) / (BX - 2 * OW), (d.ny - 2 + BY - 2 * OW - 1) / (BY - 2 * OW));
    dim3 b(BX, BY);
    const CUtensorMap& cn = LIM ? *a.maps.cn : *a.maps.c;
    k_pass_tma<T, LIM, A><<<g, b, smem, s>>>(d, a, *a.maps.c, cn, *a.maps.uo, *a.maps.vo,
                                             *a.maps.wo);
    return 1;
}

template <typename T>
int launch_pass_fused(const Dims& d, const PassArgs<T>& a, cudaStream_t s)
{
    if (!a.limiter) return launch_fused_variant<T, false, T>(d, a, s);
    if (a.wide) return launch_fused_variant<T, true, double>(d, a, s);
    return launch_fused_variant<T, true, T>(d, a, s);
}
