// Fused corrective pass: antidiffusive faces (+ nonoscillatory limiter) and
// the donor-cell update of one MPDATA pass in one kernel, z-marching.
//
// Work decomposition.  A CTA of 32 x 16 threads covers a 32 x 16 column of
// cells and marches it through z.  Each thread owns one cell of the column:
// per plane it forms the cell's three high faces (x, y and the z face above)
// and, with the limiter, the cell's in/out ratios; then it applies the
// donor-cell update.  Without the limiter every cell of the CTA is updated;
// with it the outer ring of the CTA is a halo (30 x 14 cells updated) whose
// faces and ratios the limited faces of the updated cells need.  Warps 2 and
// 3 also form the faces just below the column (x faces at local x = -1 by
// half of warp 2, y faces at local y = -1 by warp 3), which the lowest cells
// read.
//
// Staging.  The pass input c, the step input c^n (limiter bounds) and the
// previous pass's faces U, V, W are brought in one plane at a time by TMA
// (cp.async.bulk.tensor, 40 x 19 element boxes, zero-filled outside the grid)
// into a four-deep ring of shared-memory stages, two planes ahead of the
// plane being computed; one mbarrier per stage.  The box starts on a 16-byte
// boundary in x (its low edge is rounded down and the slack is skipped).
//
// Per plane each thread reads the 39 staged values its three faces use once
// into registers (struct Nb) and evaluates every formula from them.  The
// cell's own c values of the neighbouring planes and its own z faces live in
// registers from one plane to the next.  With the limiter, the limited z face
// above a cell needs the ratios of the cell above, so the update trails the
// face computation by one plane; the limited x and y faces of a plane are
// kept (registers + a two-plane ring in shared memory for the neighbours)
// until the update of that plane.
//
// Arithmetic: the formulas and evaluation order of kernels_unfused.cuh (the
// reference's, see there for file:line citations).  APPROX replaces the
// ratios' IEEE divisions by the hardware reciprocal (the "approx_div" form).
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

// Every staged value the three high faces of one cell read.  Names: plane
// prefix (none = plane k, P = k+1, M = k-1 for c; u/v/w = previous faces,
// p = plane k+1, m = face-plane k-1) then the offset (L/R = x -+ 1, D/U =
// y -+ 1, L2 = x - 2).
template <typename T> struct Nb {
    T C, L, R, D, Uu, RU, RD, LU;   // c, plane k
    T P, PL, PR, PD, PU;            // c, plane k+1
    T M, MR, MU;                    // c, plane k-1
    T u, uL, uR, uL2, uLU, uU, uL2U;  // x faces, plane k
    T up, upL;                      // x faces, plane k+1
    T v, vD, vU, vR, vRD;           // y faces, plane k
    T vp, vpD;                      // y faces, plane k+1
    T wm, wmR, wmU;                 // z faces, face-plane k-1
    T w, wR, wU;                    // z faces, face-plane k
    T wp;                           // z faces, face-plane k+1
};

template <typename T>
__device__ __forceinline__ Nb<T> gather(const Planes<T>& S, int o, T own_m, T own_p)
{
    constexpr int Y = SBX;
    Nb<T> n;
    n.C = S.c_0[o]; n.L = S.c_0[o - 1]; n.R = S.c_0[o + 1]; n.D = S.c_0[o - Y];
    n.Uu = S.c_0[o + Y]; n.RU = S.c_0[o + 1 + Y]; n.RD = S.c_0[o + 1 - Y]; n.LU = S.c_0[o - 1 + Y];
    n.P = own_p; n.PL = S.c_p[o - 1]; n.PR = S.c_p[o + 1]; n.PD = S.c_p[o - Y]; n.PU = S.c_p[o + Y];
    n.M = own_m; n.MR = S.c_m[o + 1]; n.MU = S.c_m[o + Y];
    n.u = S.uo_0[o]; n.uL = S.uo_0[o - 1]; n.uR = S.uo_0[o + 1]; n.uL2 = S.uo_0[o - 2];
    n.uLU = S.uo_0[o - 1 + Y]; n.uU = S.uo_0[o + Y]; n.uL2U = S.uo_0[o - 2 + Y];
    n.up = S.uo_p[o]; n.upL = S.uo_p[o - 1];
    n.v = S.vo_0[o]; n.vD = S.vo_0[o - Y]; n.vU = S.vo_0[o + Y]; n.vR = S.vo_0[o + 1];
    n.vRD = S.vo_0[o + 1 - Y];
    n.vp = S.vo_p[o]; n.vpD = S.vo_p[o - Y];
    n.wm = S.wo_m[o]; n.wmR = S.wo_m[o + 1]; n.wmU = S.wo_m[o + Y];
    n.w = S.wo_0[o]; n.wR = S.wo_0[o + 1]; n.wU = S.wo_0[o + Y];
    n.wp = S.wo_p[o];
    return n;
}

struct FaceCtx {
    int nx, ny, ns, use_div, vv_fix, pass;
};

template <int V> struct IC {
    static constexpr int value = V;
};

// x face between cells i and i+1.
template <bool AP, typename T> __device__ __forceinline__ T face_u(const Nb<T>& n, int i, const FaceCtx& f)
{
    T vb, wb, neg_div = T(0);
    if (i == 0) {
        vb = T(0.5) * (n.vRD + n.vR);
        wb = T(0.5) * (n.wmR + n.wR);
    } else if (i == f.nx - 2) {
        vb = T(0.5) * (n.vD + n.v);
        wb = T(0.5) * (n.wm + n.w);
    } else {
        vb = T(0.25) * (((n.vRD + n.vR) + n.v) + n.vD);
        wb = T(0.25) * (((n.wmR + n.wR) + n.w) + n.wm);
        if (f.use_div) {
            T s = n.uR - n.uL;
            s = s + n.vRD;
            s = s - n.vR;
            s = s - n.v;
            s = s + n.vD;
            s = s + n.wmR;
            s = s - n.wR;
            s = s - n.w;
            s = s + n.wm;
            neg_div = -((T(0.25) * n.u) * s);
        } else {
            neg_div = -T(0);
        }
    }
    T n1, d1, n2, d2;
    grad_pair(n.RU, n.Uu, n.D, n.RD, n1, d1);
    grad_pair(n.PR, n.P, n.M, n.MR, n2, d2);
    return face_pattern<T, AP>(neg_div, n.u, n.C, n.R, vb, n1, d1, wb, n2, d2);
}

// y face between rows j and j+1 (column i, plane k).
template <bool AP, typename T>
__device__ __forceinline__ T face_v(const Nb<T>& n, int i, int j, int k, const FaceCtx& f,
                                   const Dims& d, const T* __restrict__ Vadv)
{
    T ub, wb, neg_div = T(0);
    if (j == 0) {
        ub = T(0.5) * (n.uLU + n.uU);
        wb = T(0.5) * (n.wmU + n.wU);
    } else if (j == f.ny - 2) {
        ub = T(0.5) * (n.uL + n.u);
        wb = T(0.5) * (n.wm + n.w);
    } else {
        if (i == 1 && !f.vv_fix)  // the column vv_pass never writes (vv.c:81-82)
            return (f.pass & 1) ? T(0) : Vadv[cell(d, 1, j, k)];
        ub = T(0.25) * (((n.uLU + n.uU) + n.u) + n.uL);
        wb = T(0.25) * (((n.wmU + n.wU) + n.w) + n.wm);
        if (f.use_div) {
            const T ul2u = (i >= 2) ? n.uL2U : T(0);
            const T ul2 = (i >= 2) ? n.uL2 : T(0);
            T s = n.vU - n.vD;
            s = s + n.wmU;
            s = s - n.wU;
            s = s - n.w;
            s = s + n.wm;
            s = s + n.uLU;
            s = s - ul2u;
            s = s - ul2;
            s = s + n.uL;
            neg_div = -((T(0.25) * n.v) * s);
        } else {
            neg_div = -T(0);
        }
    }
    T n1, d1, n2, d2;
    grad_pair(n.RU, n.R, n.L, n.LU, n1, d1);
    grad_pair(n.PU, n.P, n.M, n.MU, n2, d2);
    return face_pattern<T, AP>(neg_div, n.v, n.C, n.Uu, ub, n1, d1, wb, n2, d2);
}

// z face between planes k and k+1.
template <bool AP, typename T> __device__ __forceinline__ T face_w(const Nb<T>& n, int k, const FaceCtx& f)
{
    T ub, vb, neg_div = T(0);
    if (k == 0) {
        ub = T(0.5) * (n.upL + n.up);
        vb = T(0.5) * (n.vpD + n.vp);
    } else if (k == f.ns - 2) {
        ub = T(0.5) * (n.uL + n.u);
        vb = T(0.5) * (n.vD + n.v);
    } else {
        ub = T(0.25) * (((n.u + n.up) + n.upL) + n.uL);
        vb = T(0.25) * (((n.vpD + n.vp) + n.v) + n.vD);
        if (f.use_div) {
            T s = n.wp - n.wm;
            s = s + n.upL;
            s = s - n.up;
            s = s - n.u;
            s = s + n.uL;
            s = s + n.vpD;
            s = s - n.vp;
            s = s - n.v;
            s = s + n.vD;
            neg_div = -((T(0.25) * n.w) * s);
        } else {
            neg_div = -T(0);
        }
    }
    T n1, d1, n2, d2;
    grad_pair(n.PR, n.R, n.L, n.PL, n1, d1);
    grad_pair(n.PU, n.Uu, n.D, n.PD, n2, d2);
    return face_pattern<T, AP>(neg_div, n.w, n.C, n.P, ub, n1, d1, vb, n2, d2);
}

}  // namespace fused

template <typename T, bool LIM, typename A, bool AP>
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
    const bool u_ok = i >= 0 && i <= nx - 2 && j >= 1 && j <= ny - 2;  // own x face exists
    const bool v_ok = i >= 1 && i <= nx - 2 && j >= 0 && j <= ny - 2;  // own y face exists
    // Extra faces below the column: the x faces at local x = -1 by half of warp
    // 2, the y faces at local y = -1 by warp 3, so no warp runs both face
    // paths one after the other (measured faster than warps 0-1 doing both).
    constexpr int EXU0 = 2 * 32, EXV0 = 3 * 32;
    static_assert(EXU0 + BY <= EXV0 && EXV0 + BX <= NT, "extra-face threads out of the CTA");
    const int tu = tid - EXU0, tv = tid - EXV0;  // index along the tile's low edge
    const bool ex_u = tu >= 0 && tu < BY, ex_v = tv >= 0 && tv < BX;
    const int ex_i = ex_u ? i0 - 1 : i0 + tv;
    const int ex_j = ex_u ? j0 + tu : j0 - 1;
    const int ex_o = ex_u ? (tu + 2) * Y + (1 + rx) : Y + (tv + 2 + rx);
    const int ex_w = ex_u ? (tu + 1) * WX : (tv + 1);
    const bool ex_ok = ex_u ? (ex_i >= 0 && ex_i <= nx - 2 && ex_j >= 1 && ex_j <= ny - 2)
                            : (ex_v && ex_i >= 1 && ex_i <= nx - 2 && ex_j >= 0 && ex_j <= ny - 2);

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
        tma::load_3d(const_cast<T*>(box(p, 0)), &map_c, gx0, gy0, p, bar);
        tma::load_3d(const_cast<T*>(box(p, 1)), &map_uo, gx0, gy0, p, bar);
        tma::load_3d(const_cast<T*>(box(p, 2)), &map_vo, gx0, gy0, p, bar);
        tma::load_3d(const_cast<T*>(box(p, 3)), &map_wo, gx0, gy0, p, bar);
        if (LIM) tma::load_3d(const_cast<T*>(box(p, 4)), &map_cn, gx0, gy0, p, bar);
    };
    // Stage slot s of array arr (s is a compile-time constant at every use:
    // the march below is unrolled by the ring depth).
    auto slot = [&](int s, int arr) -> const T* {
        return reinterpret_cast<const T*>(smem + (size_t)(s * NARR + arr) * SB);
    };

    // z chunk: this CTA updates planes [z0, z1); the march starts a few planes
    // earlier so every value the first updated plane reads is formed exactly
    // as an unchunked march would form it (2 planes of warm-up without the
    // limiter, 3 with it: the z faces below, then the ratios below).
    const int zb = a.zbase > 0 ? a.zbase : 1, ze = a.zend > 0 ? a.zend : ns - 1;
    const int depth = a.zdepth > 0 ? a.zdepth : ze - zb;
    const int z0 = zb + (int)blockIdx.z * depth;
    const int z1 = min(ze, z0 + depth);
    const int kstart = max(0, z0 - (LIM ? 3 : 2));
    const int last = LIM ? z1 : z1 - 1;  // iteration of the last update

    bool ok = true;
    int confirmed = kstart;  // planes below this one: thread 0 has seen their stage complete
    if (tid == 0) {
        issue(kstart);
        issue(kstart + 1);
    }
    ok = tma::mbar_wait(&bars[kstart & (NSTAGE - 1)], 0);
    if (tid == 0 && ok) confirmed = kstart + 1;

    // Register state carried between planes.
    T cq0 = T(0), cq1 = T(0), cq2 = ok ? box(kstart, 0)[o] : T(0), cq3 = T(0);  // own c, planes k-2..k+1
    T rw_prev = T(0);                      // raw z face below (face-plane k-1)
    T bu_prev = T(1), bd_prev = T(1);      // own ratios of plane k-1
    T lu_prev = T(0), lv_prev = T(0), lw_prev = T(0);  // limited faces of plane k-1 / face-plane k-2

    // One plane of the march; S = k mod NSTAGE (compile-time).
    auto plane = [&](auto Sc, const int k) {
        constexpr int S = decltype(Sc)::value;
        constexpr int SM1 = (S + NSTAGE - 1) % NSTAGE, SP1 = (S + 1) % NSTAGE, SP2 = (S + 2) % NSTAGE;
        __syncthreads();  // every read of the slot plane k+2 reuses is done
        if (tid == 0 && k + 2 <= min(ns - 1, last + 1)) issue(k + 2);
        if (k + 1 <= ns - 1) {
            if (ok) ok = tma::mbar_wait(&bars[SP1], ((k + 1 - kstart) / NSTAGE) & 1);
            if (tid == 0 && ok) confirmed = k + 2;
            cq3 = slot(SP1, 0)[o];
        }
        (void)SP2;
        const bool kin = k >= 1 && k <= ns - 2;

        // ---- raw faces of plane k (z face: face-plane k) ----
        T ru = T(0), rv = T(0), rw = T(0);
        if (k <= ns - 2) {
            Planes<T> SP;
            SP.c_m = slot(SM1, 0); SP.c_0 = slot(S, 0); SP.c_p = slot(SP1, 0);
            SP.uo_0 = slot(S, 1); SP.uo_p = slot(SP1, 1);
            SP.vo_0 = slot(S, 2); SP.vo_p = slot(SP1, 2);
            SP.wo_m = slot(SM1, 3); SP.wo_0 = slot(S, 3); SP.wo_p = slot(SP1, 3);
            {
                const Nb<T> nb = gather(SP, o, cq1, cq3);
                if (kin && u_ok) ru = face_u<AP>(nb, i, fc);
                if (kin && v_ok) rv = face_v<AP>(nb, i, j, k, fc, d, a.Vadv);
                if (cell_in) rw = face_w<AP>(nb, k, fc);
            }
            sRU[w] = ru;
            sRV[w] = rv;
            if (ex_u || ex_v) {
                T ev = T(0);
                if (kin && ex_ok) {
                    const Nb<T> nb = gather(SP, ex_o, SP.c_m[ex_o], SP.c_p[ex_o]);
                    ev = ex_u ? face_u<AP>(nb, ex_i, fc)
                              : face_v<AP>(nb, ex_i, ex_j, k, fc, d, a.Vadv);
                }
                (ex_u ? sRU : sRV)[ex_w] = ev;
            }
        }
        __syncthreads();

        if (LIM) {
            // ---- limiter ratios of plane k ----
            T bu = T(1), bd = T(1);
            if (kin && cell_in) {
                const T* c0 = slot(S, 0);
                const T* n0 = slot(S, 4);
                const T psi = cq2;
                const T cl = c0[o - 1], cr = c0[o + 1], cd = c0[o - Y], cu = c0[o + Y];
                T mx = vmax(psi, n0[o]), mn = vmin(psi, n0[o]);
                mx = vmax(vmax(cl, n0[o - 1]), mx); mn = vmin(vmin(cl, n0[o - 1]), mn);
                mx = vmax(vmax(cr, n0[o + 1]), mx); mn = vmin(vmin(cr, n0[o + 1]), mn);
                mx = vmax(vmax(cd, n0[o - Y]), mx); mn = vmin(vmin(cd, n0[o - Y]), mn);
                mx = vmax(vmax(cu, n0[o + Y]), mx); mn = vmin(vmin(cu, n0[o + Y]), mn);
                if (ns > 3) {
                    const T nm = slot(SM1, 4)[o], np = slot(SP1, 4)[o];
                    mx = vmax(vmax(cq1, nm), mx); mn = vmin(vmin(cq1, nm), mn);
                    mx = vmax(vmax(cq3, np), mx); mn = vmin(vmin(cq3, np), mn);
                }
                A fin = A(0), fout = A(0);
                lim_acc(lim_flux<T, A>(sRU[w - 1], cl, psi), false, fin, fout);
                lim_acc(lim_flux<T, A>(ru, psi, cr), true, fin, fout);
                lim_acc(lim_flux<T, A>(sRV[w - WX], cd, psi), false, fin, fout);
                lim_acc(lim_flux<T, A>(rv, psi, cu), true, fin, fout);
                lim_acc(lim_flux<T, A>(rw_prev, cq1, psi), false, fin, fout);
                lim_acc(lim_flux<T, A>(rw, psi, cq3), true, fin, fout);
                bu = T(ratio<AP>(A(mx) - A(psi), fin + lim_tiny<A>()));
                bd = T(ratio<AP>(A(psi) - A(mn), fout + lim_tiny<A>()));
            }
            sBU[w] = bu;
            sBD[w] = bd;
            __syncthreads();

            // ---- limited faces: x, y of plane k; z of face-plane k-1 ----
            T lu = ru, lv = rv;
            if (x < BX - 1) lu = limit_face(ru, bu, bd, sBU[w + 1], sBD[w + 1]);
            if (y < BY - 1) lv = limit_face(rv, bu, bd, sBU[w + WX], sBD[w + WX]);
            const T lw = limit_face(rw_prev, bu_prev, bd_prev, bu, bd);
            sLU[(S & 1) * WPL + w] = lu;
            sLV[(S & 1) * WPL + w] = lv;
            if (a.write_faces) {
                const bool ox = x >= 1 && x <= BX - 2, oy = y >= 1 && y <= BY - 2;
                const long long q = cell(d, i, j, k);
                const bool mine_k = k >= z0 && k < z1;  // this chunk's planes
                if (kin && mine_k && u_ok && oy && (ox || i == 0)) a.Un[q] = lu;
                if (kin && mine_k && v_ok && ox && (oy || j == 0)) a.Vn[q] = lv;
                // face-plane k-1: the high face of plane k-1, and face-plane 0 in the first chunk
                // (face-plane 0 only from the chunk that starts at plane 1: a later
                // chunk's warm-up does not form it)
                if (k >= 1 && owned && k - 1 < z1 && (k - 1 >= z0 || (k - 1 == 0 && z0 == 1)))
                    a.Wn[q - d.pp] = lw;
            }

            // ---- donor update of plane k-1 ----
            const int u = k - 1;
            if (u >= z0 && u < z1 && owned) {
                const T* cu = slot(SM1, 0);
                const T ul = sLU[(SM1 & 1) * WPL + w - 1];
                const T vb = sLV[(SM1 & 1) * WPL + w - WX];
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
            if (k >= z0 && k < z1 && owned) {
                const T* c0 = slot(S, 0);
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
    };
    for (int kb = kstart & ~(NSTAGE - 1); kb <= last; kb += NSTAGE) {
        if (kb >= kstart) plane(IC<0>{}, kb);
        if (kb + 1 >= kstart && kb + 1 <= last) plane(IC<1>{}, kb + 1);
        if (kb + 2 >= kstart && kb + 2 <= last) plane(IC<2>{}, kb + 2);
        if (kb + 3 >= kstart && kb + 3 <= last) plane(IC<3>{}, kb + 3);
    }

    if (!ok && a.err) atomicOr(a.err, 1);
    if (tid == 0) {  // never leave with a copy in flight
        const int issued_last = min(ns - 1, last + 1);
        for (int p = confirmed; p <= issued_last; p++)
            if (!tma::mbar_wait(&bars[p & (NSTAGE - 1)], ((p - kstart) / NSTAGE) & 1)) break;
    }
}

template <typename T, bool LIM, typename A, bool AP>
int launch_fused_variant(const Dims& d, const PassArgs<T>& a, cudaStream_t s)
{
    using namespace fused;
    constexpr size_t smem = smem_bytes<T, LIM>();
    static bool configured = false;  // the attribute is per device function
    if (!configured) {
        cudaFuncSetAttribute(k_pass_tma<T, LIM, A, AP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        configured = true;
    }
    constexpr int OW = LIM ? 1 : 0;
    const int zb = a.zbase > 0 ? a.zbase : 1, ze = a.zend > 0 ? a.zend : d.ns - 1;
    if (ze <= zb) return 0;
    const int depth = a.zdepth > 0 ? a.zdepth : ze - zb;
    dim3 g((d.nx - 2 + BX - 2 * OW - 1) / (BX - 2 * OW), (d.ny - 2 + BY - 2 * OW - 1) / (BY - 2 * OW),
           (ze - zb + depth - 1) / depth);
    dim3 b(BX, BY);
    const CUtensorMap& cn = LIM ? *a.maps.cn : *a.maps.c;
    k_pass_tma<T, LIM, A, AP><<<g, b, smem, s>>>(d, a, *a.maps.c, cn, *a.maps.uo, *a.maps.vo,
                                                 *a.maps.wo);
    return 1;
}

template <typename T, bool AP> int launch_fused_mode(const Dims& d, const PassArgs<T>& a, cudaStream_t s)
{
    if (!a.limiter) return launch_fused_variant<T, false, T, AP>(d, a, s);
    if (a.wide) return launch_fused_variant<T, true, double, AP>(d, a, s);
    return launch_fused_variant<T, true, T, AP>(d, a, s);
}

template <typename T>
int launch_pass_fused(const Dims& d, const PassArgs<T>& a, cudaStream_t s)
{
    if (a.approx && sizeof(T) == 4) return launch_fused_mode<T, true>(d, a, s);
    return launch_fused_mode<T, false>(d, a, s);
}
