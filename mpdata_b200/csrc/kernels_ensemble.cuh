// Batched ensemble of independent 2D problems: one launch per pass covers
// every instance.
//
// An instance is a 2D grid nx x ny with a fixed one-cell shell: the
// reference's 2D form is the 3D grid nx x ny x 3 with w = 0 (tests/init.c:64-68,
// ring2d calls test_init(n, 3)); every z term there is an exact zero, so these
// 2D formulas (the 3D ones with the z terms dropped, same evaluation order
// otherwise) give the same values as the 3D kernels on the 3-plane form.
//
// Work list: (instance, tile) items over the instances' interior cells.  A
// persistent grid of CTAs walks the list (item = blockIdx.x + n * gridDim.x).
// The corrective pass stages each item's tile with a halo of 3 into shared
// memory by 16-byte cp.async chunks (rows rounded down to a 16-byte
// boundary), double-buffered (the next item's copies run while the current
// item computes; four barriers per item).  The first corrective pass forms
// c^(1) itself from c^n and the advective faces (FUSE0, no pass-0 launch).
// Each pass forms the faces of every cell of the tile (and, with the limiter,
// their ratios) and updates the cells it owns: all but the first column and
// row (the first two and the last with the limiter), so every face an owned
// cell reads is the high face of a tile cell.  Tiles away from the instance's
// boundary run a copy without the boundary cases.  Tile shape
// TX x TY is a template parameter chosen by the host-side autotuner.
//
// Included by kernels_all.cuh inside namespace mpd::MPD_NS.

namespace ens {

constexpr int H = 3;  // staged halo (the y faces' divergent term reaches two x faces back)

// The staged values the two high faces of one cell read (2D subset of Nb).
template <typename T> struct Nb2 {
    T C, L, R, D, Uu, RU, RD, LU;
    T u, uL, uR, uL2, uLU, uU, uL2U;
    T v, vD, vU, vR, vRD;
};

template <typename T> __device__ __forceinline__ Nb2<T> gather2(const T* c, const T* uo, const T* vo, int o, int Y)
{
    Nb2<T> n;
    n.C = c[o]; n.L = c[o - 1]; n.R = c[o + 1]; n.D = c[o - Y]; n.Uu = c[o + Y];
    n.RU = c[o + 1 + Y]; n.RD = c[o + 1 - Y]; n.LU = c[o - 1 + Y];
    n.u = uo[o]; n.uL = uo[o - 1]; n.uR = uo[o + 1]; n.uL2 = uo[o - 2]; n.uLU = uo[o - 1 + Y];
    n.uU = uo[o + Y]; n.uL2U = uo[o - 2 + Y];
    n.v = vo[o]; n.vD = vo[o - Y]; n.vU = vo[o + Y]; n.vR = vo[o + 1]; n.vRD = vo[o + 1 - Y];
    return n;
}

// x face between i and i+1 (uu.c:18-102 with the z terms, all zero here, dropped).
// BORDER = false: the caller knows the face takes the interior pattern.
template <bool AP, bool BORDER, typename T>
__device__ __forceinline__ T face_u2(const Nb2<T>& n, int i, int nx, int use_div)
{
    T vb, neg_div = T(0);
    if (BORDER && i == 0) {
        vb = T(0.5) * (n.vRD + n.vR);
    } else if (BORDER && i == nx - 2) {
        vb = T(0.5) * (n.vD + n.v);
    } else {
        vb = T(0.25) * (((n.vRD + n.vR) + n.v) + n.vD);
        if (use_div) {
            T s = n.uR - n.uL;
            s = s + n.vRD;
            s = s - n.vR;
            s = s - n.v;
            s = s + n.vD;
            neg_div = -((T(0.25) * n.u) * s);
        } else {
            neg_div = -T(0);
        }
    }
    T n1, d1;
    grad_pair(n.RU, n.Uu, n.D, n.RD, n1, d1);
    const T ma = mag(n.u);
    const T t = neg_div + ratio<AP>((ma * (T(1) - ma)) * (n.R - n.C), (n.R + n.C) + tiny<T>());
    return t - T(0.5) * (n.u * ratio<AP>(vb * n1, d1));
}

// y face between j and j+1 (vv.c:21-107, z terms dropped, column rule kept).
template <bool AP, bool BORDER, typename T>
__device__ __forceinline__ T face_v2(const Nb2<T>& n, int i, int j, int ny, int use_div, int vv_fix,
                                    int pass, T vadv)
{
    T ub, neg_div = T(0);
    if (BORDER && j == 0) {
        ub = T(0.5) * (n.uLU + n.uU);
    } else if (BORDER && j == ny - 2) {
        ub = T(0.5) * (n.uL + n.u);
    } else {
        if (BORDER && i == 1 && !vv_fix) return (pass & 1) ? T(0) : vadv;  // vv.c:81-82
        ub = T(0.25) * (((n.uLU + n.uU) + n.u) + n.uL);
        if (use_div) {
            const T ul2u = (!BORDER || i >= 2) ? n.uL2U : T(0);
            const T ul2 = (!BORDER || i >= 2) ? n.uL2 : T(0);
            T s = n.vU - n.vD;
            s = s + n.uLU;
            s = s - ul2u;
            s = s - ul2;
            s = s + n.uL;
            neg_div = -((T(0.25) * n.v) * s);
        } else {
            neg_div = -T(0);
        }
    }
    T n1, d1;
    grad_pair(n.RU, n.R, n.L, n.LU, n1, d1);
    const T ma = mag(n.v);
    const T t = neg_div + ratio<AP>((ma * (T(1) - ma)) * (n.Uu - n.C), (n.Uu + n.C) + tiny<T>());
    return t - T(0.5) * (n.v * ratio<AP>(ub * n1, d1));
}

// Asynchronous 16-byte copy global -> shared (cp.async.cg, bypassing
// registers and L1); valid = false copies nothing and fills the 16 bytes with
// zeros.  Both addresses must be 16-byte aligned.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid)
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(src),
                 "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

}  // namespace ens

// Donor-cell pass (smolar_pass.c:30-57, 2D), one thread per cell of a tile.
template <typename T, int TX, int TY>
__global__ void __launch_bounds__(TX * TY)
    k_ens_donor(T* __restrict__ arena, const EnsInst* __restrict__ insts,
                const EnsItem* __restrict__ items, int nitems, EnsPass p)
{
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const EnsItem item = items[it];
        const EnsInst& in = insts[item.inst];  // fields read in place (no local copy)
        const int i = item.i0 + threadIdx.x, j = item.j0 + threadIdx.y;
        if (i > in.nx - 2 || j > in.ny - 2) continue;
        const long long q = (long long)j * in.px + i;
        const T* c0 = arena + in.c[p.in];
        const T* U = arena + in.f[p.rs][0];
        const T* V = arena + in.f[p.rs][1];
        const T cc = c0[q];
        const T fx = upwind(cc, c0[q + 1], U[q]) - upwind(c0[q - 1], cc, U[q - 1]);
        const T fy = upwind(cc, c0[q + in.px], V[q]) - upwind(c0[q - in.px], cc, V[q - in.px]);
        arena[in.c[p.out] + q] = cc - T(0.5) * (fx + fy);
    }
}

// Corrective pass (antidiffusive faces + optional limiter + donor update), 2D.
// FUSE0 (first corrective pass only): the tile's c^(1) is formed here from the
// staged c^n and advective faces by the donor update (k_ens_donor's
// arithmetic, same order), so pass 0 needs no launch of its own and c^(1)
// never goes through global memory.
template <typename T, bool LIM, typename A, bool AP, int TX, int TY, bool FUSE0>
__global__ void __launch_bounds__(TX * TY)
    k_ens_pass(T* __restrict__ arena, const EnsInst* __restrict__ insts,
               const EnsItem* __restrict__ items, int nitems, EnsPass p)
{
    using namespace ens;
    // Staged rows start on a 16-byte boundary (x rounded down by rx < V
    // elements) and hold whole 16-byte chunks: TX + 2H cells plus the
    // alignment slack, rounded up to V elements.
    constexpr int V = 16 / (int)sizeof(T);
    constexpr int SX = (TX + 2 * H + V - 1 + V - 1) / V * V, SY = TY + 2 * H, PL = SX * SY;
    constexpr int CH = SX / V;  // 16-byte chunks per staged row
    constexpr int NT = TX * TY;
    // Owned cells: local x in [LO, TX-1-HI] (likewise y).  The halo cells are
    // the ones whose high faces (and, with the limiter, ratios) the owned
    // cells read, so every face needed is formed by a thread of the tile.
    constexpr int LO = LIM ? 2 : 1, HI = LIM ? 1 : 0;
    constexpr int WX = TX + 2, WPL = WX * (TY + 2);  // work planes: local [-1, TX] x [-1, TY]
    // Stage buffers, double-buffered: the next item's tile is copied in
    // (cp.async) while the current one is computed.
    // (fused: c^n is staged in bN, c^(1) formed into bC[0])
    constexpr bool STAGE_N = LIM || FUSE0;
    __shared__ __align__(16) T bC[FUSE0 ? 1 : 2][PL];
    __shared__ __align__(16) T bU[2][PL];
    __shared__ __align__(16) T bV[2][PL];
    __shared__ __align__(16) T bN[2][STAGE_N ? PL : V];
    __shared__ T sRU[WPL], sRV[WPL], sBU[LIM ? WPL : 1], sBD[LIM ? WPL : 1];
    const int x = threadIdx.x, y = threadIdx.y, tid = y * TX + x;
    const int w = (y + 1) * WX + (x + 1);

    // Queue the copies of item `it`'s tile.  Rows of every instance array start
    // 128-byte aligned and are padded to px (a multiple of 32) with zeros that
    // no kernel writes, so a chunk is either inside a row (cells past nx read
    // 0) or wholly outside the instance (zero-filled): every cell outside the
    // instance reads 0.
    auto stage = [&](int it, int b) {
        const EnsItem item = items[it];
        const EnsInst& in = insts[item.inst];  // fields read in place (no local copy)
        const int gx0 = (item.i0 - LO - H) & ~(V - 1), gy0 = item.j0 - LO - H;
        const T* gc = arena + in.c[p.in];
        const T* gn = arena + in.c[p.cn];
        const T* gu = arena + in.f[p.rs][0];
        const T* gv = arena + in.f[p.rs][1];
        for (int e = tid; e < CH * SY; e += NT) {
            const int sy = e / CH, cx = e - sy * CH;
            const int gi = gx0 + cx * V, gj = gy0 + sy;
            const bool inside = gi >= 0 && gi < in.px && gj >= 0 && gj < in.ny;
            const long long q = inside ? (long long)gj * in.px + gi : 0;
            const int d = sy * SX + cx * V;
            if (!FUSE0) cp_async16(&bC[b][d], gc + q, inside);
            cp_async16(&bU[b][d], gu + q, inside);
            cp_async16(&bV[b][d], gv + q, inside);
            if (STAGE_N) cp_async16(&bN[b][d], gn + q, inside);
        }
        cp_async_commit();
    };

    int b = 0;
    if ((int)blockIdx.x < nitems) stage(blockIdx.x, 0);
    for (int it = blockIdx.x; it < nitems; it += gridDim.x, b ^= 1) {
        cp_async_wait<0>();  // this item's tile (the only copy group in flight)
        // ...has landed for every thread, and every thread is done with the
        // previous item, so its buffers (the other stage, c^(1), the work
        // planes) may be refilled
        __syncthreads();
        if (it + (int)gridDim.x < nitems) stage(it + gridDim.x, b ^ 1);  // overlaps this item
        const T* sC = bC[FUSE0 ? 0 : b];
        const T* sU = bU[b];
        const T* sV = bV[b];
        const T* sN = bN[b];
        const EnsItem item = items[it];
        const EnsInst& in = insts[item.inst];  // fields read in place (no local copy)
        const int nx = in.nx, ny = in.ny, px = in.px;
        const int i0 = item.i0 - LO, j0 = item.j0 - LO;  // global cell of local (0, 0)
        const T* vadv = arena + in.f[0][1];
        const int rx = (i0 - H) - ((i0 - H) & ~(V - 1));  // alignment slack of this tile
        const int o = (y + H) * SX + (x + H) + rx;
        // Tiles whose every cell, face and c^(1) cell takes the interior forms
        // run a copy without the boundary cases (uniform over the CTA).
        auto item_body = [&](auto border_tag) {
            constexpr bool BORDER = decltype(border_tag)::value;
            if constexpr (FUSE0) {
                // c^(1) over local [-1, TX] x [-1, TY] (every cell the pass reads):
                // the donor update of interior cells, the fixed shell copied, 0 outside
                T* c1 = bC[0];
                for (int e = tid; e < (TX + 2) * (TY + 2); e += NT) {
                    const int ly = e / (TX + 2) - 1, lx = e - (ly + 1) * (TX + 2) - 1;
                    const int q = (ly + H) * SX + (lx + H) + rx;
                    const int gi = i0 + lx, gj = j0 + ly;
                    T v = sN[q];
                    if (!BORDER || (gi >= 1 && gi <= nx - 2 && gj >= 1 && gj <= ny - 2)) {
                        const T cc = sN[q];
                        const T fx = upwind(cc, sN[q + 1], sU[q]) - upwind(sN[q - 1], cc, sU[q - 1]);
                        const T fy = upwind(cc, sN[q + SX], sV[q]) - upwind(sN[q - SX], cc, sV[q - SX]);
                        v = cc - T(0.5) * (fx + fy);
                    }
                    c1[q] = v;
                }
                __syncthreads();
            }

            const int i = i0 + x, j = j0 + y;
            const bool cell_in = !BORDER || (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2);
            const bool owned = cell_in && x >= LO && x <= TX - 1 - HI && y >= LO && y <= TY - 1 - HI;
            T ru = T(0), rv = T(0);
            {
                const Nb2<T> nb = gather2(sC, sU, sV, o, SX);
                if (!BORDER || (i >= 0 && i <= nx - 2 && j >= 1 && j <= ny - 2))
                    ru = face_u2<AP, BORDER>(nb, i, nx, p.use_div);
                if (!BORDER || (i >= 1 && i <= nx - 2 && j >= 0 && j <= ny - 2)) {
                    const T va = (BORDER && i == 1) ? vadv[(long long)j * px + 1] : T(0);
                    rv = face_v2<AP, BORDER>(nb, i, j, ny, p.use_div, p.vv_fix, p.pass, va);
                }
            }
            sRU[w] = ru;
            sRV[w] = rv;
            __syncthreads();

            T ur = ru, ul = sRU[w - 1], vt = rv, vb = sRV[w - WX];
            if (LIM) {
                T bu = T(1), bd = T(1);
                if (cell_in) {
                    const T psi = sC[o], cl = sC[o - 1], cr = sC[o + 1], cd = sC[o - SX], cu = sC[o + SX];
                    T mx = vmax(psi, sN[o]), mn = vmin(psi, sN[o]);
                    mx = vmax(vmax(cl, sN[o - 1]), mx); mn = vmin(vmin(cl, sN[o - 1]), mn);
                    mx = vmax(vmax(cr, sN[o + 1]), mx); mn = vmin(vmin(cr, sN[o + 1]), mn);
                    mx = vmax(vmax(cd, sN[o - SX]), mx); mn = vmin(vmin(cd, sN[o - SX]), mn);
                    mx = vmax(vmax(cu, sN[o + SX]), mx); mn = vmin(vmin(cu, sN[o + SX]), mn);
                    A fin = A(0), fout = A(0);
                    lim_acc(lim_flux<T, A>(ul, cl, psi), false, fin, fout);
                    lim_acc(lim_flux<T, A>(ru, psi, cr), true, fin, fout);
                    lim_acc(lim_flux<T, A>(vb, cd, psi), false, fin, fout);
                    lim_acc(lim_flux<T, A>(rv, psi, cu), true, fin, fout);
                    bu = T(ratio<AP>(A(mx) - A(psi), fin + lim_tiny<A>()));
                    bd = T(ratio<AP>(A(psi) - A(mn), fout + lim_tiny<A>()));
                }
                sBU[w] = bu;
                sBD[w] = bd;
                __syncthreads();
                auto BU = [&](int q2) { return sBU[q2]; };
                auto BD = [&](int q2) { return sBD[q2]; };
                if (owned) {
                    ur = limit_face(ru, BU(w), BD(w), BU(w + 1), BD(w + 1));
                    ul = limit_face(ul, BU(w - 1), BD(w - 1), BU(w), BD(w));
                    vt = limit_face(rv, BU(w), BD(w), BU(w + WX), BD(w + WX));
                    vb = limit_face(vb, BU(w - WX), BD(w - WX), BU(w), BD(w));
                }
            }
            if (owned) {
                const long long q = (long long)j * px + i;
                const T cc = sC[o];
                const T fx = upwind(cc, sC[o + 1], ur) - upwind(sC[o - 1], cc, ul);
                const T fy = upwind(cc, sC[o + SX], vt) - upwind(sC[o - SX], cc, vb);
                arena[in.c[p.out] + q] = cc - T(0.5) * (fx + fy);
                if (p.write_faces) {
                    arena[in.f[p.ws][0] + q] = ur;
                    arena[in.f[p.ws][1] + q] = vt;
                    if (BORDER && i == 1) arena[in.f[p.ws][0] + q - 1] = ul;
                    if (BORDER && j == 1) arena[in.f[p.ws][1] + q - px] = vb;
                }
            }
        };
        if (i0 >= 2 && i0 + TX <= nx - 2 && j0 >= 2 && j0 + TY <= ny - 2)
            item_body(std::false_type{});
        else
            item_body(std::true_type{});
    }
}

// ---- the first corrective pass as a y-march, one warp per item -------------
//
// An item is a strip of an instance: 32 consecutive columns (lane l holds
// column x0 - LO + l) and a chunk of owned rows [ya, yb).  The warp marches
// the rows upwards; every value a cell needs from a column to its left or
// right comes from the neighbouring lane by a warp shuffle, every value of a
// row below from registers carried by the march, so the pass uses no shared
// memory and no barrier.  Iteration j: c^(1) of row j+1 (the donor update,
// pass 0 fused as in k_ens_pass), the raw faces of row j (x face and the y
// face above), with the limiter the ratios of row j and the limited faces
// that need them, and the update of row j-1.  The arithmetic is k_ens_pass's
// (the same face, limiter and donor functions on the same operands), so both
// give the same bits.  Lanes whose columns lack a neighbour's operands only
// feed their neighbours: owned lanes are LO .. 31 - HI (limiter: 3 .. 28).
//
// The items' i0 is the first owned column, j0 the first owned row, pad the
// end of the owned rows.
template <typename T, bool LIM, bool AP>
__global__ void __launch_bounds__(128)
    k_ens_march(T* __restrict__ arena, const EnsInst* __restrict__ insts,
                const EnsItem* __restrict__ items, int nitems, EnsPass p)
{
    using namespace ens;
    constexpr int LO = LIM ? 3 : 2, HI = LIM ? 3 : 2;
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int it = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (it >= nitems) return;  // whole warps only: every lane of a warp takes this branch alike
    const EnsItem item = items[it];
    const EnsInst& in = insts[item.inst];
    const int nx = in.nx, ny = in.ny, px = in.px;
    const int i = item.i0 - LO + lane;  // this lane's column
    const int ya = item.j0, yb = item.pad;
    const T* gn = arena + in.c[p.cn];
    const T* gu = arena + in.f[0][0];
    const T* gv = arena + in.f[0][1];
    T* gout = arena + in.c[p.out];
    const bool col_ok = i >= 0 && i < px;
    const bool own_lane = lane >= LO && lane <= 31 - HI;
    auto ld = [&](const T* a, int row) -> T {
        return (col_ok && row >= 0 && row < ny) ? a[(long long)row * px + i] : T(0);
    };
    auto left = [&](T v) { return __shfl_up_sync(FULL, v, 1); };
    auto right = [&](T v) { return __shfl_down_sync(FULL, v, 1); };
    auto left2 = [&](T v) { return __shfl_up_sync(FULL, v, 2); };
    // c^(1) of row r from c^n rows r-1 (nm), r (nc, its left / right
    // neighbours nl, nr), r+1 (np), the advective x faces of row r (ur, and
    // ul of the column to the left) and the y faces below (vm) and above (vc)
    // the row: k_ens_pass's fused donor update for interior cells, the fixed
    // shell copied, 0 outside the instance
    auto c1_of = [&](bool border, int r, T nm, T nc, T np, T nl, T nr, T ur, T ul, T vm,
                     T vc) -> T {
        if (!border || (i >= 1 && i <= nx - 2 && r >= 1 && r <= ny - 2)) {
            const T fx = upwind(nc, nr, ur) - upwind(nl, nc, ul);
            const T fy = upwind(nc, np, vc) - upwind(nm, nc, vm);
            return nc - T(0.5) * (fx + fy);
        }
        return nc;
    };
    // The march starts two rows below the first owned row: the ratios of row
    // ya-1 need the raw y face below it.  Registers by row relative to j; the
    // neighbours' values a later iteration needs again are carried (suffix
    // L / R / L2: the lane to the left / right / two to the left).
    const int j_first = ya - 2;
    T nm1 = ld(gn, j_first - 1), n0 = ld(gn, j_first), np1 = ld(gn, j_first + 1);
    T np2 = ld(gn, j_first + 2);
    T u0 = ld(gu, j_first), up1 = ld(gu, j_first + 1);
    T vm1 = ld(gv, j_first - 1), v0 = ld(gv, j_first), vp1 = ld(gv, j_first + 1);
    T cm2, cm1, c0;  // c^(1) of rows j-2, j-1, j
    {
        const T n_m3 = ld(gn, j_first - 3), n_m2 = ld(gn, j_first - 2);
        const T v_m3 = ld(gv, j_first - 3), v_m2 = ld(gv, j_first - 2);
        const T u_m2 = ld(gu, j_first - 2), u_m1 = ld(gu, j_first - 1);
        cm2 = c1_of(true, j_first - 2, n_m3, n_m2, nm1, left(n_m2), right(n_m2), u_m2, left(u_m2),
                    v_m3, v_m2);
        cm1 = c1_of(true, j_first - 1, n_m2, nm1, n0, left(nm1), right(nm1), u_m1, left(u_m1),
                    v_m2, vm1);
        c0 = c1_of(true, j_first, nm1, n0, np1, left(n0), right(n0), u0, left(u0), vm1, v0);
    }
    T cL0 = left(c0), cR0 = right(c0), cLm1 = left(cm1), cRm1 = right(cm1);
    T nL0 = left(n0), nR0 = right(n0);
    T uL0 = left(u0), uR0 = right(u0), uL20 = left2(u0);
    T vR0 = right(v0), vRm1 = right(vm1);
    // Carried faces: the raw y face below row j (rv_prev), the x face of row
    // j-1 and the y face (j-2|j-1) in the form the update uses (limited with
    // the limiter), the ratios of row j-1.
    T rv_prev = T(0), fx_prev = T(0), fy_pp = T(0);
    T bu_prev = T(1), bd_prev = T(1);
    // Strips whose every column takes the interior forms run rows 1 .. ny-3
    // through a copy without the boundary cases (uniform over the warp).
    const bool strip_in = item.i0 - LO >= 2 && item.i0 - LO + 31 <= nx - 3;

    auto iteration = [&](auto border_tag, const int j) {
        constexpr bool BORDER = decltype(border_tag)::value;
        // operands of the next iteration (latency overlaps this one)
        const T n_next = ld(gn, j + 3), u_next = ld(gu, j + 2), v_next = ld(gv, j + 2);
        const T npL = left(np1), npR = right(np1);
        const T upL = left(up1), upR = right(up1), upL2 = left2(up1);
        const T vpR = right(vp1);
        const T cp1 = c1_of(BORDER, j + 1, n0, np1, np2, npL, npR, up1, upL, v0, vp1);
        const T cpL = left(cp1), cpR = right(cp1);
        // ---- raw faces of row j ----
        Nb2<T> nb;
        nb.C = c0; nb.L = cL0; nb.R = cR0; nb.D = cm1; nb.Uu = cp1;
        nb.RU = cpR; nb.RD = cRm1; nb.LU = cpL;
        nb.u = u0; nb.uL = uL0; nb.uR = uR0; nb.uL2 = uL20;
        nb.uLU = upL; nb.uU = up1; nb.uL2U = upL2;
        nb.v = v0; nb.vD = vm1; nb.vU = vp1; nb.vR = vR0; nb.vRD = vRm1;
        T ru = T(0), rv = T(0);
        if (!BORDER || (i >= 0 && i <= nx - 2 && j >= 1 && j <= ny - 2))
            ru = face_u2<AP, BORDER>(nb, i, nx, p.use_div);
        if (!BORDER || (i >= 1 && i <= nx - 2 && j >= 0 && j <= ny - 2))
            rv = face_v2<AP, BORDER>(nb, i, j, ny, p.use_div, p.vv_fix, p.pass, v0);
        const T ru_l = left(ru);
        // ---- the faces the update of row j-1 uses ----
        T fx_cur, fy_cur;  // x face of row j, y face (j-1|j)
        T bu = T(1), bd = T(1);
        if (LIM) {
            const T psi = c0, cl = cL0, cr = cR0, cd = cm1, cu = cp1;
            if (!BORDER || (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2)) {
                T mx = vmax(psi, n0), mn = vmin(psi, n0);
                mx = vmax(vmax(cl, nL0), mx); mn = vmin(vmin(cl, nL0), mn);
                mx = vmax(vmax(cr, nR0), mx); mn = vmin(vmin(cr, nR0), mn);
                mx = vmax(vmax(cd, nm1), mx); mn = vmin(vmin(cd, nm1), mn);
                mx = vmax(vmax(cu, np1), mx); mn = vmin(vmin(cu, np1), mn);
                T fin = T(0), fout = T(0);
                lim_acc(lim_flux<T, T>(ru_l, cl, psi), false, fin, fout);
                lim_acc(lim_flux<T, T>(ru, psi, cr), true, fin, fout);
                lim_acc(lim_flux<T, T>(rv_prev, cd, psi), false, fin, fout);
                lim_acc(lim_flux<T, T>(rv, psi, cu), true, fin, fout);
                bu = ratio<AP>(mx - psi, fin + lim_tiny<T>());
                bd = ratio<AP>(psi - mn, fout + lim_tiny<T>());
            }
            fx_cur = limit_face(ru, bu, bd, right(bu), right(bd));
            fy_cur = limit_face(rv_prev, bu_prev, bd_prev, bu, bd);
        } else {
            fx_cur = ru;
            fy_cur = rv_prev;
        }
        // ---- update of row r = j-1 ----
        const int r = j - 1;
        {
            const T ul = left(fx_prev);
            const T fxx = upwind(cm1, cRm1, fx_prev) - upwind(cLm1, cm1, ul);
            const T fyy = upwind(cm1, c0, fy_cur) - upwind(cm2, cm1, fy_pp);
            const T out = cm1 - T(0.5) * (fxx + fyy);
            const bool owned = own_lane && r >= ya && r < yb && i >= 1 && i <= nx - 2 &&
                               r >= 1 && r <= ny - 2;
            if (owned) {
                const long long q = (long long)r * px + i;
                gout[q] = out;
                if (p.write_faces) {
                    arena[in.f[p.ws][0] + q] = fx_prev;
                    arena[in.f[p.ws][1] + q] = fy_cur;
                    if (i == 1) arena[in.f[p.ws][0] + q - 1] = ul;
                    if (r == 1) arena[in.f[p.ws][1] + q - px] = fy_pp;
                }
            }
        }
        // ---- rotate ----
        fy_pp = fy_cur;
        fx_prev = fx_cur;
        rv_prev = rv;
        bu_prev = bu;
        bd_prev = bd;
        cm2 = cm1; cm1 = c0; c0 = cp1;
        cLm1 = cL0; cRm1 = cR0; cL0 = cpL; cR0 = cpR;
        nm1 = n0; n0 = np1; np1 = np2; np2 = n_next;
        nL0 = npL; nR0 = npR;
        u0 = up1; up1 = u_next;
        uL0 = upL; uR0 = upR; uL20 = upL2;
        vm1 = v0; v0 = vp1; vp1 = v_next;
        vRm1 = vR0; vR0 = vpR;
    };
    for (int j = j_first; j <= yb; j++) {
        if (strip_in && j >= 1 && j <= ny - 3) iteration(std::false_type{}, j);
        else iteration(std::true_type{}, j);
    }
}

template <typename T, bool LIM, bool AP>
void ens_launch_march(T* arena, const EnsInst* insts, const EnsItem* items, int nitems,
                      const EnsPass& p, cudaStream_t s)
{
    const int grid = (nitems + 3) / 4;
    if (grid > 0) k_ens_march<T, LIM, AP><<<grid, 128, 0, s>>>(arena, insts, items, nitems, p);
}

template <typename T, bool LIM, typename A, bool AP, int TX, int TY>
void ens_launch_pass(T* arena, const EnsInst* insts, const EnsItem* items, int nitems, int grid,
                     const EnsPass& p, cudaStream_t s)
{
    if (p.fuse_donor)
        k_ens_pass<T, LIM, A, AP, TX, TY, true><<<grid, dim3(TX, TY), 0, s>>>(arena, insts, items,
                                                                              nitems, p);
    else
        k_ens_pass<T, LIM, A, AP, TX, TY, false><<<grid, dim3(TX, TY), 0, s>>>(arena, insts, items,
                                                                               nitems, p);
}

template <typename T, int TX, int TY>
void ens_launch_donor_t(T* arena, const EnsInst* insts, const EnsItem* items, int nitems, int grid,
                        const EnsPass& p, cudaStream_t s)
{
    k_ens_donor<T, TX, TY><<<grid, dim3(TX, TY), 0, s>>>(arena, insts, items, nitems, p);
}

// Dispatch on the runtime tile index (the autotuner's candidates) and options.
template <typename T, int TX, int TY>
void ens_pass_tile(T* arena, const EnsInst* insts, const EnsItem* items, int nitems, int grid,
                   const EnsPass& p, int limiter, int wide, int approx, cudaStream_t s)
{
    if (!limiter) {
        if (approx) ens_launch_pass<T, false, T, true, TX, TY>(arena, insts, items, nitems, grid, p, s);
        else ens_launch_pass<T, false, T, false, TX, TY>(arena, insts, items, nitems, grid, p, s);
    } else if (wide) {
        if (approx) ens_launch_pass<T, true, double, true, TX, TY>(arena, insts, items, nitems, grid, p, s);
        else ens_launch_pass<T, true, double, false, TX, TY>(arena, insts, items, nitems, grid, p, s);
    } else {
        if (approx) ens_launch_pass<T, true, T, true, TX, TY>(arena, insts, items, nitems, grid, p, s);
        else ens_launch_pass<T, true, T, false, TX, TY>(arena, insts, items, nitems, grid, p, s);
    }
}

template <typename T>
int launch_ens_pass(int tile, T* arena, const EnsInst* insts, const EnsItem* items, int nitems,
                    int grid, const EnsPass& p, int limiter, int wide, int approx, cudaStream_t s)
{
    switch (tile) {
    case 0: ens_pass_tile<T, 32, 8>(arena, insts, items, nitems, grid, p, limiter, wide, approx, s); break;
    case 1: ens_pass_tile<T, 32, 16>(arena, insts, items, nitems, grid, p, limiter, wide, approx, s); break;
    case 2: ens_pass_tile<T, 64, 8>(arena, insts, items, nitems, grid, p, limiter, wide, approx, s); break;
    default: return -1;
    }
    return 0;
}

// The first corrective pass as a y-march (k_ens_march; FP32 limiter ratios only).
template <typename T>
int launch_ens_march(T* arena, const EnsInst* insts, const EnsItem* items, int nitems,
                     const EnsPass& p, int limiter, int approx, cudaStream_t s)
{
    if (limiter) {
        if (approx) ens_launch_march<T, true, true>(arena, insts, items, nitems, p, s);
        else ens_launch_march<T, true, false>(arena, insts, items, nitems, p, s);
    } else {
        if (approx) ens_launch_march<T, false, true>(arena, insts, items, nitems, p, s);
        else ens_launch_march<T, false, false>(arena, insts, items, nitems, p, s);
    }
    return 0;
}

template <typename T>
int launch_ens_donor(int tile, T* arena, const EnsInst* insts, const EnsItem* items, int nitems,
                     int grid, const EnsPass& p, cudaStream_t s)
{
    switch (tile) {
    case 0: ens_launch_donor_t<T, 32, 8>(arena, insts, items, nitems, grid, p, s); break;
    case 1: ens_launch_donor_t<T, 32, 16>(arena, insts, items, nitems, grid, p, s); break;
    case 2: ens_launch_donor_t<T, 64, 8>(arena, insts, items, nitems, grid, p, s); break;
    default: return -1;
    }
    return 0;
}
