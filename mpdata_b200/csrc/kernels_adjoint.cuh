// Adjoint (reverse mode) of one MPDATA step, one kernel per forward routine.
//
// The forward routines are those of kernels_unfused.cuh (donor pass
// smolar_pass.c:30-57, antidiffusive faces uu.c/vv.c/ww.c, the limiter).  The
// adjoint differentiates every formula with each branch frozen at its
// forward choice: the sign of a face value in |a| (a > 0 ? a : -a), the
// boundary/interior pattern, the limiter's min selections and the argmax /
// argmin of its bounds.  Contributions to neighbouring cells and faces are
// accumulated with atomicAdd into arrays the host zeroes first.
//
// Array roles for corrective pass o (forward: c_o --faces F_o--> c_{o+1}):
//   c      level c_o;  cn  the step input c_0 (limiter bounds)
//   Fp     faces of the previous pass (advective for o = 1): the pattern's inputs
//   R      raw antidiffusive faces of pass o;  L  limited faces (= R without limiter)
//   bup/bdn limiter ratios of pass o
//   lam_*  adjoint of the same arrays
//
// Included by kernels_all.cuh inside namespace mpd::MPD_NS.

namespace adj {

template <typename T> __device__ __forceinline__ void acc(T* a, long long i, T v)
{
    if (a && v != T(0)) atomicAdd(a + i, v);
}

__device__ __forceinline__ bool interior(const Dims& d, int i, int j, int k)
{
    return i >= 1 && i <= d.nx - 2 && j >= 1 && j <= d.ny - 2 && k >= 1 && k <= d.ns - 2;
}

// Adjoint of the face pattern (common.cuh face_pattern):
//   out = (neg_div + (m(1-m)(hi-lo)) / ((hi+lo)+eps)) - 1/2 a ((b1 n1)/d1 + (b2 n2)/d2),
//   m = |a| (sign frozen), neg_div = -(a/4) s (when use_div), n = ((p+q)-r)-s,
//   d = (((p+q)+r)+s)+eps.
// Returns the adjoints of a, lo, hi, b1, b2, s and of the two gradient
// quadruples' shared parts: ln (for the +,+,-,- numerator) and ld (all +).
template <typename T> struct PatAdj {
    T a, lo, hi, b1, b2, s, n1, d1, n2, d2;
};

template <typename T>
__device__ __forceinline__ PatAdj<T> pattern_adj(T lam, T a, T lo, T hi, T b1, T n1, T d1, T b2,
                                                 T n2, T d2, bool has_div, T sdiv)
{
    // Three reciprocals (of d1, d2 and the first term's denominator) stand
    // for the dozen quotients of the derivative.
    PatAdj<T> g;
    const T id1 = T(1) / d1, id2 = T(1) / d2;
    const T r1 = (b1 * n1) * id1, r2 = (b2 * n2) * id2;
    const T sg = a > T(0) ? T(1) : T(-1);
    const T m = a > T(0) ? a : -a;
    const T num = (m * (T(1) - m)) * (hi - lo);
    const T iden = T(1) / ((hi + lo) + tiny<T>());
    // out = t - 0.5 a (r1 + r2)
    const T lr = T(-0.5) * a * lam;
    const T lr1 = lr * id1, lr2 = lr * id2;
    g.a = T(-0.5) * (r1 + r2) * lam;
    g.b1 = lr1 * n1;
    g.n1 = lr1 * b1;
    g.d1 = -lr1 * r1;
    g.b2 = lr2 * n2;
    g.n2 = lr2 * b2;
    g.d2 = -lr2 * r2;
    // t = neg_div + num / den
    const T lnum = lam * iden;
    const T lden = -lnum * (num * iden);
    const T lm = lnum * (T(1) - T(2) * m) * (hi - lo);
    g.hi = lnum * (m * (T(1) - m)) + lden;
    g.lo = -lnum * (m * (T(1) - m)) + lden;
    g.a += lm * sg;
    g.s = T(0);
    if (has_div) {  // neg_div = -(0.25 a) s
        g.a += T(-0.25) * sdiv * lam;
        g.s = T(-0.25) * a * lam;
    }
    return g;
}

// Limiter application adjoint of one face (forward: k_fct_apply, L = R g,
// g = the frozen min of 1 and the two ratios): lR = g l, and a l to the
// ratio the min selected.  q / hq: the face's low / high cell, lo_in / hi_in:
// whether they are interior (shell cells have no ratio: 1).
template <typename T>
__device__ __forceinline__ void limit_face_adj(T a, T l, long long q, long long hq, bool lo_in,
                                               bool hi_in, const T* bup, const T* bdn, T* lR,
                                               T* lbup, T* lbdn)
{
    const T bu_lo = lo_in ? bup[q] : T(1), bd_lo = lo_in ? bdn[q] : T(1);
    const T bu_hi = hi_in ? bup[hq] : T(1), bd_hi = hi_in ? bdn[hq] : T(1);
    T x, y;
    T *lx, *ly;  // adjoint slots of the two candidate ratios (null for the shell)
    if (a > T(0)) { x = bd_lo; y = bu_hi; lx = lo_in ? lbdn : nullptr; ly = hi_in ? lbup : nullptr; }
    else { x = bu_lo; y = bd_hi; lx = lo_in ? lbup : nullptr; ly = hi_in ? lbdn : nullptr; }
    const bool pick_x = x < y;
    const T g1 = pick_x ? x : y;
    const bool ratio_sel = g1 < T(1);
    const T g = ratio_sel ? g1 : T(1);
    lR[q] = g * l;  // the first contribution of the step (the ratio adjoint adds later)
    if (ratio_sel) {
        if (pick_x) acc(lx, q, a * l);
        else acc(ly, hq, a * l);
    }
}

// Arrays of the limiter-application adjoint, fused into the donor adjoint of
// a corrective pass (all null without the limiter and for pass 0).
template <typename T> struct LimAdj {
    const T *RU, *RV, *RW, *bup, *bdn;
    T *lRU, *lRV, *lRW, *lbup, *lbdn;
};

}  // namespace adj

// Donor pass adjoint (forward: k_donor).  One thread per cell of the full grid:
// gathers the cell's adjoint (identity for every cell, shell included, plus
// the flux terms of its six faces) and, when lamF is given, the adjoint of
// its three high faces.  lam_in accumulates (+=) when add_in is set and is
// written (=) otherwise (the first kernel of the step to touch it); lamF
// adds to what earlier kernels accumulated there when add_F is set.  With
// the limiter (lim.lRU set) the adjoint of each high face goes on at once
// through the limiter application (the faces the donor update read are
// L = R g) to the raw face and the ratios, in place of a kernel of its own,
// and lamF is not written; without it lamF is written (=).
template <typename T>
__global__ void k_adj_donor(Dims d, const T* __restrict__ c, const T* __restrict__ U,
                            const T* __restrict__ V, const T* __restrict__ W,
                            const T* __restrict__ lam_out, T* __restrict__ lam_in, T* lamU, T* lamV,
                            T* lamW, adj::LimAdj<T> lim, int add_in, int add_F)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= d.nx || j >= d.ny) return;
    const long long q = cell(d, i, j, k);
    const long long S[3] = {1, d.px, d.pp};
    const T* F[3] = {U, V, W};
    T* lF[3] = {lamU, lamV, lamW};
    const int idx[3] = {i, j, k};
    const int ext[3] = {d.nx, d.ny, d.ns};
    auto inner = [&](int a, int off) {  // is the neighbour along axis a (offset off) interior?
        int ii = i + (a == 0 ? off : 0), jj = j + (a == 1 ? off : 0), kk = k + (a == 2 ? off : 0);
        return adj::interior(d, ii, jj, kk);
    };
    // face along axis a between cell (idx - 1 + hi) and (idx + hi): used iff the
    // two transverse indices are interior and the face index is 0..ext-2
    auto face_used = [&](int a, int f) {
        if (f < 0 || f > ext[a] - 2) return false;
        for (int b = 0; b < 3; b++)
            if (b != a && (idx[b] < 1 || idx[b] > ext[b] - 2)) return false;
        return true;
    };
    const bool me_in = adj::interior(d, i, j, k);
    T lam = lam_out[q];
    const T lq = me_in ? lam_out[q] : T(0);
    for (int a = 0; a < 3; a++) {
        if (face_used(a, idx[a])) {  // high face: this cell is lo
            const T A = F[a][q];
            const T sg = A > T(0) ? T(1) : T(-1);
            const T dF = T(0.5) * ((inner(a, 1) ? lam_out[q + S[a]] : T(0)) - lq);
            lam += dF * (A * (T(1) + sg));
            if (lF[a]) {
                const T lf = dF * (c[q] * (T(1) + sg) + c[q + S[a]] * (T(1) - sg));
                const T l = add_F ? lF[a][q] + lf : lf;
                if (lim.lRU) {
                    const T* R[3] = {lim.RU, lim.RV, lim.RW};
                    T* lR[3] = {lim.lRU, lim.lRV, lim.lRW};
                    adj::limit_face_adj(R[a][q], l, q, q + S[a], me_in, inner(a, 1), lim.bup,
                                        lim.bdn, lR[a], lim.lbup, lim.lbdn);
                } else {
                    lF[a][q] = l;
                }
            }
        }
        if (face_used(a, idx[a] - 1)) {  // low face: this cell is hi
            const T A = F[a][q - S[a]];
            const T sg = A > T(0) ? T(1) : T(-1);
            const T dF = T(0.5) * (lq - (inner(a, -1) ? lam_out[q - S[a]] : T(0)));
            lam += dF * (A * (T(1) - sg));
        }
    }
    lam_in[q] = add_in ? lam_in[q] + lam : lam;
}

// Limiter ratio adjoint (forward: k_fct_beta), one thread per interior cell.
template <typename T, typename A>
__global__ void k_adj_beta(Dims d, const T* __restrict__ c, const T* __restrict__ cn,
                           const T* __restrict__ RU, const T* __restrict__ RV,
                           const T* __restrict__ RW, const T* __restrict__ lbup,
                           const T* __restrict__ lbdn, T* lam_c, T* lam_cn, T* lRU, T* lRV, T* lRW)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (!adj::interior(d, i, j, k)) return;
    const long long q = cell(d, i, j, k);
    const T lu = lbup[q], ld = lbdn[q];
    if (lu == T(0) && ld == T(0)) return;
    const long long X = 1, Y = d.px, Z = d.pp;
    // bound candidates in the forward order (kernels_unfused.cuh k_fct_beta)
    const bool zact = d.ns > 3;
    const int ncand = zact ? 14 : 10;
    const T* arr[14] = {c, cn, c, cn, c, cn, c, cn, c, cn, c, cn, c, cn};
    const long long off[14] = {0, 0, -X, -X, X, X, -Y, -Y, Y, Y, -Z, -Z, Z, Z};
    T mx = c[q], mn = c[q];
    for (int n = 1; n < ncand; n++) {
        const T t = arr[n][q + off[n]];
        mx = vmax(t, mx);
        mn = vmin(t, mn);
    }
    int imx = 0, imn = 0;
    for (int n = ncand - 1; n >= 0; n--) {
        if (arr[n][q + off[n]] == mx) imx = n;
        if (arr[n][q + off[n]] == mn) imn = n;
    }
    const T psi = c[q];
    // face fluxes: low x, high x, low y, high y, low z, high z
    const T* R[6] = {RU, RU, RV, RV, RW, RW};
    T* lR[6] = {lRU, lRU, lRV, lRV, lRW, lRW};
    const long long fq[6] = {q - X, q, q - Y, q, q - Z, q};
    const long long lo[6] = {q - X, q, q - Y, q, q - Z, q};
    const long long hi[6] = {q, q + X, q, q + Y, q, q + Z};
    A fin = A(0), fout = A(0);
    A fl[6];
    for (int f = 0; f < 6; f++) {
        const T a = R[f][fq[f]];
        fl[f] = lim_flux<T, A>(a, c[lo[f]], c[hi[f]]);
        lim_acc(fl[f], (f & 1) != 0, fin, fout);
    }
    // two reciprocals for the eight quotients of the derivative
    const A idin = A(1) / (fin + lim_tiny<A>()), idout = A(1) / (fout + lim_tiny<A>());
    const A bu = (A(mx) - A(psi)) * idin, bd = (A(psi) - A(mn)) * idout;
    const A l_mx = A(lu) * idin, l_mn = -A(ld) * idout;
    const A l_psi = -l_mx - l_mn;
    const A l_fin = -l_mx * bu, l_fout = l_mn * bd;
    adj::acc(arr[imx] == c ? lam_c : lam_cn, q + off[imx], T(l_mx));
    adj::acc(arr[imn] == c ? lam_c : lam_cn, q + off[imn], T(l_mn));
    adj::acc(lam_c, q, T(l_psi));
    for (int f = 0; f < 6; f++) {
        const bool high = (f & 1) != 0;
        const A lfl = high ? (fl[f] > A(0) ? l_fout : -l_fin) : (fl[f] > A(0) ? l_fin : -l_fout);
        if (lfl == A(0)) continue;
        const T a = R[f][fq[f]];
        if (a > T(0)) {
            adj::acc(lR[f], fq[f], T(lfl * A(c[lo[f]])));
            adj::acc(lam_c, lo[f], T(lfl * A(a)));
        } else {
            adj::acc(lR[f], fq[f], T(lfl * A(c[hi[f]])));
            adj::acc(lam_c, hi[f], T(lfl * A(a)));
        }
    }
}

// Antidiffusive-face adjoint (forward: k_antidiff): one thread per cell for
// its three high faces; scatters into the pass input's adjoint and, when
// given, the previous faces' adjoints.
template <typename T>
__global__ void k_adj_pattern(Dims d, const T* __restrict__ c, const T* __restrict__ Uo,
                              const T* __restrict__ Vo, const T* __restrict__ Wo,
                              const T* __restrict__ lRU, const T* __restrict__ lRV,
                              const T* __restrict__ lRW, T* lam_c, T* lUo, T* lVo, T* lWo,
                              int use_div, int vv_fix)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= d.nx || j >= d.ny) return;
    const long long X = 1, Y = d.px, Z = d.pp;
    const long long q = cell(d, i, j, k);
    const int nx = d.nx, ny = d.ny, ns = d.ns;
    const bool kin = k >= 1 && k <= ns - 2, jin = j >= 1 && j <= ny - 2, iin = i >= 1 && i <= nx - 2;
    using adj::acc;
    auto grads = [&](long long p, long long qq, long long r, long long s, T& n, T& dd) {
        grad_pair(c[p], c[qq], c[r], c[s], n, dd);
    };
    auto scatter_grad = [&](long long p, long long qq, long long r, long long s, T ln, T ld) {
        acc(lam_c, p, ln + ld);
        acc(lam_c, qq, ln + ld);
        acc(lam_c, r, -ln + ld);
        acc(lam_c, s, -ln + ld);
    };

    // ---- x face between i and i+1 ----
    if (kin && jin && i <= nx - 2 && lRU[q] != T(0)) {
        const T lam = lRU[q];
        const bool bnd = (i == 0 || i == nx - 2);
        const long long a_c = (i == 0) ? q + X : q;
        T vb, wb, sdiv = T(0);
        if (bnd) {
            vb = T(0.5) * (Vo[a_c - Y] + Vo[a_c]);
            wb = T(0.5) * (Wo[a_c - Z] + Wo[a_c]);
        } else {
            vb = T(0.25) * (((Vo[q + X - Y] + Vo[q + X]) + Vo[q]) + Vo[q - Y]);
            wb = T(0.25) * (((Wo[q + X - Z] + Wo[q + X]) + Wo[q]) + Wo[q - Z]);
            sdiv = Uo[q + X] - Uo[q - X];
            sdiv = sdiv + Vo[q + X - Y]; sdiv = sdiv - Vo[q + X]; sdiv = sdiv - Vo[q]; sdiv = sdiv + Vo[q - Y];
            sdiv = sdiv + Wo[q + X - Z]; sdiv = sdiv - Wo[q + X]; sdiv = sdiv - Wo[q]; sdiv = sdiv + Wo[q - Z];
        }
        T n1, d1, n2, d2;
        grads(q + X + Y, q + Y, q - Y, q + X - Y, n1, d1);
        grads(q + X + Z, q + Z, q - Z, q + X - Z, n2, d2);
        const auto g = adj::pattern_adj(lam, Uo[q], c[q], c[q + X], vb, n1, d1, wb, n2, d2,
                                        !bnd && use_div, sdiv);
        acc(lam_c, q, g.lo);
        acc(lam_c, q + X, g.hi);
        scatter_grad(q + X + Y, q + Y, q - Y, q + X - Y, g.n1, g.d1);
        scatter_grad(q + X + Z, q + Z, q - Z, q + X - Z, g.n2, g.d2);
        acc(lUo, q, g.a);
        if (bnd) {
            acc(lVo, a_c - Y, T(0.5) * g.b1); acc(lVo, a_c, T(0.5) * g.b1);
            acc(lWo, a_c - Z, T(0.5) * g.b2); acc(lWo, a_c, T(0.5) * g.b2);
        } else {
            const T qb1 = T(0.25) * g.b1, qb2 = T(0.25) * g.b2, s = g.s;
            acc(lVo, q + X - Y, qb1 + s); acc(lVo, q + X, qb1 - s); acc(lVo, q, qb1 - s); acc(lVo, q - Y, qb1 + s);
            acc(lWo, q + X - Z, qb2 + s); acc(lWo, q + X, qb2 - s); acc(lWo, q, qb2 - s); acc(lWo, q - Z, qb2 + s);
            acc(lUo, q + X, s); acc(lUo, q - X, -s);
        }
    }

    // ---- y face between j and j+1 ----
    if (kin && iin && j <= ny - 2 && lRV[q] != T(0)) {
        const bool bnd = (j == 0 || j == ny - 2);
        const bool frozen_col = !bnd && i == 1 && !vv_fix;  // constant in the forward
        if (!frozen_col) {
            const T lam = lRV[q];
            const long long a_c = (j == 0) ? q + Y : q;
            const bool l2 = i >= 2;
            T ub, wb, sdiv = T(0);
            if (bnd) {
                ub = T(0.5) * (Uo[a_c - X] + Uo[a_c]);
                wb = T(0.5) * (Wo[a_c - Z] + Wo[a_c]);
            } else {
                ub = T(0.25) * (((Uo[q - X + Y] + Uo[q + Y]) + Uo[q]) + Uo[q - X]);
                wb = T(0.25) * (((Wo[q + Y - Z] + Wo[q + Y]) + Wo[q]) + Wo[q - Z]);
                sdiv = Vo[q + Y] - Vo[q - Y];
                sdiv = sdiv + Wo[q + Y - Z]; sdiv = sdiv - Wo[q + Y]; sdiv = sdiv - Wo[q]; sdiv = sdiv + Wo[q - Z];
                sdiv = sdiv + Uo[q - X + Y];
                sdiv = sdiv - (l2 ? Uo[q - 2 * X + Y] : T(0));
                sdiv = sdiv - (l2 ? Uo[q - 2 * X] : T(0));
                sdiv = sdiv + Uo[q - X];
            }
            T n1, d1, n2, d2;
            grads(q + X + Y, q + X, q - X, q - X + Y, n1, d1);
            grads(q + Y + Z, q + Z, q - Z, q + Y - Z, n2, d2);
            const auto g = adj::pattern_adj(lam, Vo[q], c[q], c[q + Y], ub, n1, d1, wb, n2, d2,
                                            !bnd && use_div, sdiv);
            acc(lam_c, q, g.lo);
            acc(lam_c, q + Y, g.hi);
            scatter_grad(q + X + Y, q + X, q - X, q - X + Y, g.n1, g.d1);
            scatter_grad(q + Y + Z, q + Z, q - Z, q + Y - Z, g.n2, g.d2);
            acc(lVo, q, g.a);
            if (bnd) {
                acc(lUo, a_c - X, T(0.5) * g.b1); acc(lUo, a_c, T(0.5) * g.b1);
                acc(lWo, a_c - Z, T(0.5) * g.b2); acc(lWo, a_c, T(0.5) * g.b2);
            } else {
                const T qb1 = T(0.25) * g.b1, qb2 = T(0.25) * g.b2, s = g.s;
                acc(lUo, q - X + Y, qb1 + s); acc(lUo, q + Y, qb1); acc(lUo, q, qb1); acc(lUo, q - X, qb1 + s);
                if (l2) { acc(lUo, q - 2 * X + Y, -s); acc(lUo, q - 2 * X, -s); }
                acc(lWo, q + Y - Z, qb2 + s); acc(lWo, q + Y, qb2 - s); acc(lWo, q, qb2 - s); acc(lWo, q - Z, qb2 + s);
                acc(lVo, q + Y, s); acc(lVo, q - Y, -s);
            }
        }
    }

    // ---- z face between k and k+1 ----
    if (jin && iin && k <= ns - 2 && lRW[q] != T(0)) {
        const T lam = lRW[q];
        const bool bnd = (k == 0 || k == ns - 2);
        const long long a_c = (k == 0) ? q + Z : q;
        T ub, vb, sdiv = T(0);
        if (bnd) {
            ub = T(0.5) * (Uo[a_c - X] + Uo[a_c]);
            vb = T(0.5) * (Vo[a_c - Y] + Vo[a_c]);
        } else {
            ub = T(0.25) * (((Uo[q] + Uo[q + Z]) + Uo[q - X + Z]) + Uo[q - X]);
            vb = T(0.25) * (((Vo[q - Y + Z] + Vo[q + Z]) + Vo[q]) + Vo[q - Y]);
            sdiv = Wo[q + Z] - Wo[q - Z];
            sdiv = sdiv + Uo[q - X + Z]; sdiv = sdiv - Uo[q + Z]; sdiv = sdiv - Uo[q]; sdiv = sdiv + Uo[q - X];
            sdiv = sdiv + Vo[q - Y + Z]; sdiv = sdiv - Vo[q + Z]; sdiv = sdiv - Vo[q]; sdiv = sdiv + Vo[q - Y];
        }
        T n1, d1, n2, d2;
        grads(q + X + Z, q + X, q - X, q - X + Z, n1, d1);
        grads(q + Y + Z, q + Y, q - Y, q - Y + Z, n2, d2);
        const auto g = adj::pattern_adj(lam, Wo[q], c[q], c[q + Z], ub, n1, d1, vb, n2, d2,
                                        !bnd && use_div, sdiv);
        acc(lam_c, q, g.lo);
        acc(lam_c, q + Z, g.hi);
        scatter_grad(q + X + Z, q + X, q - X, q - X + Z, g.n1, g.d1);
        scatter_grad(q + Y + Z, q + Y, q - Y, q - Y + Z, g.n2, g.d2);
        acc(lWo, q, g.a);
        if (bnd) {
            acc(lUo, a_c - X, T(0.5) * g.b1); acc(lUo, a_c, T(0.5) * g.b1);
            acc(lVo, a_c - Y, T(0.5) * g.b2); acc(lVo, a_c, T(0.5) * g.b2);
        } else {
            const T qb1 = T(0.25) * g.b1, qb2 = T(0.25) * g.b2, s = g.s;
            acc(lUo, q, qb1 - s); acc(lUo, q + Z, qb1 - s); acc(lUo, q - X + Z, qb1 + s); acc(lUo, q - X, qb1 + s);
            acc(lVo, q - Y + Z, qb2 + s); acc(lVo, q + Z, qb2 - s); acc(lVo, q, qb2 - s); acc(lVo, q - Y, qb2 + s);
            acc(lWo, q + Z, s); acc(lWo, q - Z, -s);
        }
    }
}

template <typename T>
void launch_adj_pass(const Dims& d, const AdjPassArgs<T>& a, cudaStream_t s)
{
    dim3 b(32, 8), g((d.nx + 31) / 32, (d.ny + 7) / 8, d.ns);
    // donor part of this pass (faces F = limited faces, or advective for pass 0),
    // with the limiter application's adjoint fused in
    adj::LimAdj<T> lim{};
    if (a.pass > 0 && a.limiter)
        lim = adj::LimAdj<T>{a.RU, a.RV, a.RW, a.bup, a.bdn, a.lRU, a.lRV, a.lRW, a.lbup, a.lbdn};
    k_adj_donor<T><<<g, b, 0, s>>>(d, a.c, a.FU, a.FV, a.FW, a.lam_out, a.lam_in, a.lFU, a.lFV, a.lFW,
                                   lim, a.pass == 0, a.accum_F);
    if (a.pass == 0) return;
    const T* lRU = a.lFU; const T* lRV = a.lFV; const T* lRW = a.lFW;
    if (a.limiter) {
        if (a.wide)
            k_adj_beta<T, double><<<g, b, 0, s>>>(d, a.c, a.cn, a.RU, a.RV, a.RW, a.lbup, a.lbdn,
                                                  a.lam_in, a.lam_cn, a.lRU, a.lRV, a.lRW);
        else
            k_adj_beta<T, T><<<g, b, 0, s>>>(d, a.c, a.cn, a.RU, a.RV, a.RW, a.lbup, a.lbdn, a.lam_in,
                                             a.lam_cn, a.lRU, a.lRV, a.lRW);
        lRU = a.lRU; lRV = a.lRV; lRW = a.lRW;
    }
    k_adj_pattern<T><<<g, b, 0, s>>>(d, a.c, a.Uo, a.Vo, a.Wo, lRU, lRV, lRW, a.lam_in, a.lUo, a.lVo,
                                     a.lWo, a.use_div, a.vv_fix);
}
