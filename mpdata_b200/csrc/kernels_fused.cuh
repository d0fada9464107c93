// Fused corrective pass: antidiffusive faces (+ nonoscillatory limiter) and
// the donor-cell update of one MPDATA pass in a single kernel.
//
// Decomposition: each CTA owns a TX x TY column of interior cells and marches
// it through z.  Per plane it stages the pass input c, the step input c^n
// (limiter bounds) and the previous pass's faces into shared-memory rings
// (halo 3 in x and y: the divergent term of the y faces reaches two x faces
// back, vv.c:89, and the limiter needs the faces of the halo cells), then
//   1. computes the new faces over the tile (+ the cells' low edge faces;
//      with the limiter, over the tile plus a one-cell halo),
//   2. with the limiter: the in/out ratios of every tile+halo cell,
//   3. limits the faces of the cell it updates and applies the donor update.
// The limiter needs the ratios of the z neighbour above, so with it the
// update trails the face computation by one plane.
//
// Included by kernels_all.cuh inside namespace mpd::MPD_NS.

namespace fused {

constexpr int TX = 32, TY = 8, NT = TX * TY;
constexpr int H = 3;                  // halo of every staged plane
constexpr int SX = TX + 2 * H, SY = TY + 2 * H, PL = SX * SY;

// Ring slots per staged array.
constexpr int RC = 4, RCN = 4, RUO = 2, RVO = 2, RWO = 4, RRU = 2, RRV = 2, RRW = 4, RB = 4;

template <bool LIM> constexpr int planes()
{
    return RC + RUO + RVO + RWO + RRU + RRV + RRW + (LIM ? RCN + 2 * RB : 0);
}

}  // namespace fused

template <typename T, bool LIM, typename A>
__global__ void __launch_bounds__(fused::NT) k_pass_fused(Dims d, PassArgs<T> a)
{
    using namespace fused;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sC = reinterpret_cast<T*>(smem_raw);
    T* sUO = sC + RC * PL;
    T* sVO = sUO + RUO * PL;
    T* sWO = sVO + RVO * PL;
    T* sRU = sWO + RWO * PL;
    T* sRV = sRU + RRU * PL;
    T* sRW = sRV + RRV * PL;
    T* sCN = sRW + RRW * PL;  // limiter only
    T* sBU = sCN + RCN * PL;
    T* sBD = sBU + RB * PL;

    const int nx = d.nx, ny = d.ny, ns = d.ns;
    const int tid = threadIdx.y * TX + threadIdx.x;
    const int i0 = 1 + blockIdx.x * TX, j0 = 1 + blockIdx.y * TY;
    const int gx0 = i0 - H, gy0 = j0 - H;

    // Shared-memory offset of global (i, j) within a plane.
    auto S = [&](int i, int j) { return (j - gy0) * SX + (i - gx0); };
    auto c = [&](int p, int i, int j) { return sC[(p & (RC - 1)) * PL + S(i, j)]; };
    auto cn = [&](int p, int i, int j) { return sCN[(p & (RCN - 1)) * PL + S(i, j)]; };
    auto uo = [&](int p, int i, int j) { return sUO[(p & (RUO - 1)) * PL + S(i, j)]; };
    auto vo = [&](int p, int i, int j) { return sVO[(p & (RVO - 1)) * PL + S(i, j)]; };
    auto wo = [&](int p, int i, int j) { return sWO[(p & (RWO - 1)) * PL + S(i, j)]; };
    auto ru = [&](int p, int i, int j) -> T& { return sRU[(p & (RRU - 1)) * PL + S(i, j)]; };
    auto rv = [&](int p, int i, int j) -> T& { return sRV[(p & (RRV - 1)) * PL + S(i, j)]; };
    auto rw = [&](int p, int i, int j) -> T& { return sRW[(p & (RRW - 1)) * PL + S(i, j)]; };
    auto bu = [&](int p, int i, int j) -> T& { return sBU[(p & (RB - 1)) * PL + S(i, j)]; };
    auto bd = [&](int p, int i, int j) -> T& { return sBD[(p & (RB - 1)) * PL + S(i, j)]; };
    auto interior = [&](int i, int j, int p) {
        return i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2 && p >= 1 && p <= ns - 2;
    };

    // Stage plane p of a full-grid array into a ring slot (zero outside the grid).
    auto load = [&](T* ring, int slots, const T* __restrict__ src, int p) {
        T* dst = ring + (p & (slots - 1)) * PL;
        const T* base = src + (long long)p * d.pp;
        for (int e = tid; e < PL; e += NT) {
            int y = e / SX, x = e - y * SX;
            int gi = gx0 + x, gj = gy0 + y;
            T v = T(0);
            if (gi >= 0 && gi < nx && gj >= 0 && gj < ny) v = base[(long long)gj * d.px + gi];
            dst[e] = v;
        }
    };

    // ---- face formulas (the reference's, see kernels_unfused.cuh) ----
    auto face_u = [&](int m, int f, int j) -> T {  // x face between f and f+1, row j, plane m
        T vb, wb, neg_div = T(0);
        if (f == 0 || f == nx - 2) {
            int ic = (f == 0) ? 1 : nx - 2;
            vb = T(0.5) * (vo(m, ic, j - 1) + vo(m, ic, j));
            wb = T(0.5) * (wo(m - 1, ic, j) + wo(m, ic, j));
        } else {
            vb = T(0.25) * (((vo(m, f + 1, j - 1) + vo(m, f + 1, j)) + vo(m, f, j)) + vo(m, f, j - 1));
            wb = T(0.25) * (((wo(m - 1, f + 1, j) + wo(m, f + 1, j)) + wo(m, f, j)) + wo(m - 1, f, j));
            if (a.use_div) {
                T s = uo(m, f + 1, j) - uo(m, f - 1, j);
                s = s + vo(m, f + 1, j - 1);
                s = s - vo(m, f + 1, j);
                s = s - vo(m, f, j);
                s = s + vo(m, f, j - 1);
                s = s + wo(m - 1, f + 1, j);
                s = s - wo(m, f + 1, j);
                s = s - wo(m, f, j);
                s = s + wo(m - 1, f, j);
                neg_div = -((T(0.25) * uo(m, f, j)) * s);
            } else {
                neg_div = -T(0);
            }
        }
        T n1, d1, n2, d2;
        grad_pair(c(m, f + 1, j + 1), c(m, f, j + 1), c(m, f, j - 1), c(m, f + 1, j - 1), n1, d1);
        grad_pair(c(m + 1, f + 1, j), c(m + 1, f, j), c(m - 1, f, j), c(m - 1, f + 1, j), n2, d2);
        return face_pattern(neg_div, uo(m, f, j), c(m, f, j), c(m, f + 1, j), vb, n1, d1, wb, n2, d2);
    };
    auto face_v = [&](int m, int i, int g) -> T {  // y face between g and g+1, column i
        T ub, wb, neg_div = T(0);
        if (g == 0 || g == ny - 2) {
            int jc = (g == 0) ? 1 : ny - 2;
            ub = T(0.5) * (uo(m, i - 1, jc) + uo(m, i, jc));
            wb = T(0.5) * (wo(m - 1, i, jc) + wo(m, i, jc));
        } else {
            if (i == 1 && !a.vv_fix)  // column vv_pass never writes (vv.c:81-82)
                return (a.pass & 1) ? T(0) : a.Vadv[cell(d, 1, g, m)];
            ub = T(0.25) * (((uo(m, i - 1, g + 1) + uo(m, i, g + 1)) + uo(m, i, g)) + uo(m, i - 1, g));
            wb = T(0.25) * (((wo(m - 1, i, g + 1) + wo(m, i, g + 1)) + wo(m, i, g)) + wo(m - 1, i, g));
            if (a.use_div) {
                T ul2u = (i >= 2) ? uo(m, i - 2, g + 1) : T(0);
                T ul2 = (i >= 2) ? uo(m, i - 2, g) : T(0);
                T s = vo(m, i, g + 1) - vo(m, i, g - 1);
                s = s + wo(m - 1, i, g + 1);
                s = s - wo(m, i, g + 1);
                s = s - wo(m, i, g);
                s = s + wo(m - 1, i, g);
                s = s + uo(m, i - 1, g + 1);
                s = s - ul2u;
                s = s - ul2;
                s = s + uo(m, i - 1, g);
                neg_div = -((T(0.25) * vo(m, i, g)) * s);
            } else {
                neg_div = -T(0);
            }
        }
        T n1, d1, n2, d2;
        grad_pair(c(m, i + 1, g + 1), c(m, i + 1, g), c(m, i - 1, g), c(m, i - 1, g + 1), n1, d1);
        grad_pair(c(m + 1, i, g + 1), c(m + 1, i, g), c(m - 1, i, g), c(m - 1, i, g + 1), n2, d2);
        return face_pattern(neg_div, vo(m, i, g), c(m, i, g), c(m, i, g + 1), ub, n1, d1, wb, n2, d2);
    };
    auto face_w = [&](int m, int i, int j) -> T {  // z face between planes m and m+1
        T ub, vb, neg_div = T(0);
        if (m == 0 || m == ns - 2) {
            int kc = (m == 0) ? 1 : ns - 2;
            ub = T(0.5) * (uo(kc, i - 1, j) + uo(kc, i, j));
            vb = T(0.5) * (vo(kc, i, j - 1) + vo(kc, i, j));
        } else {
            ub = T(0.25) * (((uo(m, i, j) + uo(m + 1, i, j)) + uo(m + 1, i - 1, j)) + uo(m, i - 1, j));
            vb = T(0.25) * (((vo(m + 1, i, j - 1) + vo(m + 1, i, j)) + vo(m, i, j)) + vo(m, i, j - 1));
            if (a.use_div) {
                T s = wo(m + 1, i, j) - wo(m - 1, i, j);
                s = s + uo(m + 1, i - 1, j);
                s = s - uo(m + 1, i, j);
                s = s - uo(m, i, j);
                s = s + uo(m, i - 1, j);
                s = s + vo(m + 1, i, j - 1);
                s = s - vo(m + 1, i, j);
                s = s - vo(m, i, j);
                s = s + vo(m, i, j - 1);
                neg_div = -((T(0.25) * wo(m, i, j)) * s);
            } else {
                neg_div = -T(0);
            }
        }
        T n1, d1, n2, d2;
        grad_pair(c(m + 1, i + 1, j), c(m, i + 1, j), c(m, i - 1, j), c(m + 1, i - 1, j), n1, d1);
        grad_pair(c(m + 1, i, j + 1), c(m, i, j + 1), c(m, i, j - 1), c(m + 1, i, j - 1), n2, d2);
        return face_pattern(neg_div, wo(m, i, j), c(m, i, j), c(m + 1, i, j), ub, n1, d1, vb, n2, d2);
    };

    // Regions (global coordinates, inclusive) over which faces are formed.
    // Without the limiter: the tile's cells and their low edge faces; with it,
    // every face of the tile cells and of their one-cell halo.
    const int e = LIM ? 1 : 0;
    const int ux0 = i0 - 1 - e, ux1 = i0 + TX - 1 + e, uy0 = j0 - e, uy1 = j0 + TY - 1 + e;
    const int vx0 = i0 - e, vx1 = i0 + TX - 1 + e, vy0 = j0 - 1 - e, vy1 = j0 + TY - 1 + e;
    const int wx0 = i0 - e, wx1 = i0 + TX - 1 + e, wy0 = j0 - e, wy1 = j0 + TY - 1 + e;

    auto make_w = [&](int m) {  // raw z faces of face-plane m
        const int w = wx1 - wx0 + 1, n = w * (wy1 - wy0 + 1);
        for (int q = tid; q < n; q += NT) {
            int y = q / w, x = q - y * w;
            int i = wx0 + x, j = wy0 + y;
            bool ok = i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2 && m >= 0 && m <= ns - 2;
            rw(m, i, j) = ok ? face_w(m, i, j) : T(0);
        }
    };
    auto make_uv = [&](int m) {  // raw x and y faces of plane m
        {
            const int w = ux1 - ux0 + 1, n = w * (uy1 - uy0 + 1);
            for (int q = tid; q < n; q += NT) {
                int y = q / w, x = q - y * w;
                int f = ux0 + x, j = uy0 + y;
                bool ok = f >= 0 && f <= nx - 2 && j >= 1 && j <= ny - 2;
                ru(m, f, j) = ok ? face_u(m, f, j) : T(0);
            }
        }
        {
            const int w = vx1 - vx0 + 1, n = w * (vy1 - vy0 + 1);
            for (int q = tid; q < n; q += NT) {
                int y = q / w, x = q - y * w;
                int i = vx0 + x, g = vy0 + y;
                bool ok = i >= 1 && i <= nx - 2 && g >= 0 && g <= ny - 2;
                rv(m, i, g) = ok ? face_v(m, i, g) : T(0);
            }
        }
    };
    auto make_beta = [&](int m) {  // limiter ratios of the tile + halo cells of plane m
        const int w = TX + 2, n = w * (TY + 2);
        for (int q = tid; q < n; q += NT) {
            int y = q / w, x = q - y * w;
            int i = i0 - 1 + x, j = j0 - 1 + y;
            if (!interior(i, j, m)) { bu(m, i, j) = T(1); bd(m, i, j) = T(1); continue; }
            T psi = c(m, i, j), mx = psi, mn = psi, t;
#define MPD_BOUND(v) do { t = (v); mx = t > mx ? t : mx; mn = t < mn ? t : mn; } while (0)
            MPD_BOUND(cn(m, i, j));
            MPD_BOUND(c(m, i - 1, j)); MPD_BOUND(cn(m, i - 1, j));
            MPD_BOUND(c(m, i + 1, j)); MPD_BOUND(cn(m, i + 1, j));
            MPD_BOUND(c(m, i, j - 1)); MPD_BOUND(cn(m, i, j - 1));
            MPD_BOUND(c(m, i, j + 1)); MPD_BOUND(cn(m, i, j + 1));
            if (ns > 3) {
                MPD_BOUND(c(m - 1, i, j)); MPD_BOUND(cn(m - 1, i, j));
                MPD_BOUND(c(m + 1, i, j)); MPD_BOUND(cn(m + 1, i, j));
            }
#undef MPD_BOUND
            A fin = A(0), fout = A(0);
            lim_acc(lim_flux<T, A>(ru(m, i - 1, j), c(m, i - 1, j), psi), false, fin, fout);
            lim_acc(lim_flux<T, A>(ru(m, i, j), psi, c(m, i + 1, j)), true, fin, fout);
            lim_acc(lim_flux<T, A>(rv(m, i, j - 1), c(m, i, j - 1), psi), false, fin, fout);
            lim_acc(lim_flux<T, A>(rv(m, i, j), psi, c(m, i, j + 1)), true, fin, fout);
            lim_acc(lim_flux<T, A>(rw(m - 1, i, j), c(m - 1, i, j), psi), false, fin, fout);
            lim_acc(lim_flux<T, A>(rw(m, i, j), psi, c(m + 1, i, j)), true, fin, fout);
            bu(m, i, j) = T((A(mx) - A(psi)) / (fin + lim_tiny<A>()));
            bd(m, i, j) = T((A(psi) - A(mn)) / (fout + lim_tiny<A>()));
        }
    };
    // Ratio of cell (i, j, p), 1 for the fixed shell.
    auto BU = [&](int p, int i, int j) { return interior(i, j, p) ? bu(p, i, j) : T(1); };
    auto BD = [&](int p, int i, int j) { return interior(i, j, p) ? bd(p, i, j) : T(1); };
    auto FU = [&](int p, int f, int j) {
        T r = ru(p, f, j);
        if (!LIM) return r;
        return limit_face(r, BU(p, f, j), BD(p, f, j), BU(p, f + 1, j), BD(p, f + 1, j));
    };
    auto FV = [&](int p, int i, int g) {
        T r = rv(p, i, g);
        if (!LIM) return r;
        return limit_face(r, BU(p, i, g), BD(p, i, g), BU(p, i, g + 1), BD(p, i, g + 1));
    };
    auto FW = [&](int q, int i, int j) {  // face-plane q
        T r = rw(q, i, j);
        if (!LIM) return r;
        return limit_face(r, BU(q, i, j), BD(q, i, j), BU(q + 1, i, j), BD(q + 1, i, j));
    };

    // ---- prologue: planes 0 and 1, z faces of face-plane 0 ----
    load(sC, RC, a.c, 0);
    load(sC, RC, a.c, 1);
    if (LIM) {
        load(sCN, RCN, a.cn, 0);
        load(sCN, RCN, a.cn, 1);
    }
    load(sUO, RUO, a.Uo, 1);
    load(sVO, RVO, a.Vo, 1);
    load(sWO, RWO, a.Wo, 0);
    load(sWO, RWO, a.Wo, 1);
    __syncthreads();
    make_w(0);

    const int my_i = i0 + threadIdx.x, my_j = j0 + threadIdx.y;
    const bool mine = my_i <= nx - 2 && my_j <= ny - 2;
    const int last = LIM ? ns - 1 : ns - 2;
    for (int m = 1; m <= last; m++) {
        __syncthreads();  // ring slots of plane m+1 are free again
        if (m + 1 <= ns - 1) {
            load(sC, RC, a.c, m + 1);
            if (LIM) load(sCN, RCN, a.cn, m + 1);
        }
        if (m + 1 <= ns - 2) {
            load(sUO, RUO, a.Uo, m + 1);
            load(sVO, RVO, a.Vo, m + 1);
            load(sWO, RWO, a.Wo, m + 1);
        }
        __syncthreads();
        if (m <= ns - 2) {
            make_uv(m);
            make_w(m);
            if (LIM) {
                __syncthreads();
                make_beta(m);
            }
        }
        __syncthreads();
        const int u = LIM ? m - 1 : m;  // plane updated this iteration
        if (u >= 1 && mine) {
            const int i = my_i, j = my_j;
            T ur = FU(u, i, j), ul = FU(u, i - 1, j);
            T vt = FV(u, i, j), vb = FV(u, i, j - 1);
            T wf = FW(u, i, j), wb = FW(u - 1, i, j);
            T out = donor_update(c(u, i, j), c(u, i - 1, j), c(u, i + 1, j), c(u, i, j - 1),
                                 c(u, i, j + 1), c(u - 1, i, j), c(u + 1, i, j), ur, ul, vt, vb,
                                 wf, wb);
            const long long q = cell(d, i, j, u);
            a.c_out[q] = out;
            if (a.write_faces) {
                a.Un[q] = ur;
                a.Vn[q] = vt;
                a.Wn[q] = wf;
                if (i == 1) a.Un[q - 1] = ul;
                if (j == 1) a.Vn[q - d.px] = vb;
                if (u == 1) a.Wn[q - d.pp] = wb;
            }
        }
    }
}

template <typename T, bool LIM, typename A>
int launch_fused_variant(const Dims& d, const PassArgs<T>& a, cudaStream_t s)
{
    using namespace fused;
    const size_t smem = (size_t)planes<LIM>() * PL * sizeof(T);
    static bool configured = false;  // per instantiation; attribute is per device function
    if (!configured) {
        cudaFuncSetAttribute(k_pass_fused<T, LIM, A>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        configured = true;
    }
    dim3 g((d.nx - 2 + TX - 1) / TX, (d.ny - 2 + TY - 1) / TY), b(TX, TY);
    k_pass_fused<T, LIM, A><<<g, b, smem, s>>>(d, a);
    return 1;
}

template <typename T>
int launch_pass_fused(const Dims& d, const PassArgs<T>& a, cudaStream_t s)
{
    if (!a.limiter) return launch_fused_variant<T, false, T>(d, a, s);
    if (a.wide) return launch_fused_variant<T, true, double>(d, a, s);
    return launch_fused_variant<T, true, T>(d, a, s);
}
