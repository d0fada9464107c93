// Fast-mode fused corrective pass, two cells per thread (FP32 only).
//
// The same pass as k_pass_tma (kernels_fused.cuh): antidiffusive faces, the
// optional nonoscillatory limiter and the donor-cell update in one kernel
// that marches a column of cells through z over TMA-staged planes.  What
// differs is how the work is laid out, to cut the instructions per cell of
// an issue-bound kernel:
//
//  * Each thread owns two x-adjacent cells (A = local x 2*tx, B = 2*tx + 1)
//    and evaluates both with the paired FP32 instructions of sm_100
//    (add/mul/fma .f32x2); the pair also shares the staged values the two
//    stencils have in common and is read with 64-bit shared-memory loads.
//  * The face formulas are regrouped around sums both faces of a pair (and
//    the faces of one cell) share: face sums C = c_hi + c_lo, whose
//    differences across the face are the transverse gradients
//    ((RU + U) - D - RD = Cx(j+1) - Cx(j-1)), per-cell face sums
//    (SV = v + vD: the 4-face averages are SV(i) + SV(i+1)), and the
//    divergence term as a sum of two per-cell terms (e(i) + e(i+1) with
//    e = du - dv - dw; f and g likewise for the y and z faces).  Values
//    equal the reference's formulas up to rounding (not bit for bit), so
//    strict mode keeps k_pass_tma.
//  * Neighbours exchange fluxes, not raw values: the limiter's in/out
//    fluxes of each cell's high faces, the cells' bound extrema, the ratios
//    (clamped to <= 1) and the donor fluxes F = a (a > 0 ? c_lo : c_hi),
//    so the donor update needs no neighbour c values.
//  * No extra low faces are formed: the CTA's cells overlap their
//    neighbours' (x: cell 0,1 and 31, y: row 0 and 31 with the limiter;
//    x: 0 and 31, y: 0 without), so every face a kept cell needs is the high
//    face of a cell of the same CTA.
//
// Per plane k (limiter): raw faces of plane k and z face k+1/2 -> sync ->
// ratios of plane k -> sync -> limited x/y faces of plane k, limited z face
// k-1/2, donor fluxes -> donor update of plane k-1.  Without the limiter the
// update of plane k follows the raw faces after one sync.
//
// The step input c^n (limiter bounds) is read with one 64-bit global load
// per pair and plane, one plane ahead.  Every wait is bounded (tma.cuh).
//
// Included by kernels_pair.cu inside namespace mpd::fast.

namespace pair {

template <int V> struct IC {  // compile-time stage slot of one unrolled plane
    static constexpr int value = V;
};

constexpr int TX = 16, CX = 2 * TX, CY = kPairCY, NT = TX * CY;
constexpr int SBX = kPairBoxX, SBY = kPairBoxY;  // staged box: x [-2-rx, 37-rx], y [-1, CY]
constexpr int NSTAGE = 4;
constexpr int WX = 36, WY = CY + 1, WPL = WX * WY;  // work planes: x [-2, 33], y [-1, CY-1]

__host__ __device__ constexpr int stage_bytes() { return (SBX * SBY * 4 + 127) / 128 * 128; }
template <bool LIM> __host__ __device__ constexpr int n_work() { return LIM ? 10 : 2; }
template <bool LIM> __host__ __device__ constexpr size_t smem_bytes()
{
    return (size_t)NSTAGE * 4 * stage_bytes() + (size_t)n_work<LIM>() * WPL * 4 + NSTAGE * 8;
}
// Tile strides: cells of a CTA that are updated (x: 3..30 / 1..30, y: 2..CY-2 / 1..CY-1).
template <bool LIM> __host__ __device__ constexpr int stride_x() { return LIM ? CX - 4 : CX - 2; }
template <bool LIM> __host__ __device__ constexpr int stride_y() { return LIM ? CY - 3 : CY - 1; }

// ---- paired arithmetic -----------------------------------------------------
__device__ __forceinline__ float2 bc(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 operator+(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 operator-(float2 a, float2 b)
{
    return __fadd2_rn(a, make_float2(-b.x, -b.y));
}
__device__ __forceinline__ float2 operator*(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 abs2(float2 a) { return make_float2(fabsf(a.x), fabsf(a.y)); }
__device__ __forceinline__ float2 max2(float2 a, float2 b) { return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
__device__ __forceinline__ float2 min2(float2 a, float2 b) { return make_float2(fminf(a.x, b.x), fminf(a.y, b.y)); }
// (a.y, b) and (a, b.x): the pair shifted by one cell to the right / left.
__device__ __forceinline__ float2 sh(float2 a, float b) { return make_float2(a.y, b); }
__device__ __forceinline__ float2 shl(float a, float2 b) { return make_float2(a, b.x); }
__device__ __forceinline__ float2 pick(bool px, bool py, float2 a, float2 b)
{
    return make_float2(px ? a.x : b.x, py ? a.y : b.y);
}
__device__ __forceinline__ float2 ld2(const float* p) { return *reinterpret_cast<const float2*>(p); }
__device__ __forceinline__ void st2(float* p, float2 v) { *reinterpret_cast<float2*>(p) = v; }

template <bool AP> __device__ __forceinline__ float2 rat2(float2 n, float2 d)
{
    if constexpr (AP) return n * make_float2(rcp_approx(d.x), rcp_approx(d.y));
    else return make_float2(n.x / d.x, n.y / d.y);
}
// Lane-wise sums with the pair's right neighbour: (a.x + a.y, a.y + b) and
// differences (a.y - a.x, b - a.y).  Written as scalar operations: a paired
// instruction would first need (a.y, b) moved into an aligned register pair.
__device__ __forceinline__ float2 sum_r(float2 a, float b) { return make_float2(a.x + a.y, a.y + b); }
__device__ __forceinline__ float2 dif_r(float2 a, float b) { return make_float2(a.y - a.x, b - a.y); }
// With the left neighbour: (b + a.x, a.x + a.y) and (a.x - b, a.y - a.x).
__device__ __forceinline__ float2 sum_l(float b, float2 a) { return make_float2(b + a.x, a.x + a.y); }
__device__ __forceinline__ float2 dif_l(float b, float2 a) { return make_float2(a.x - b, a.y - a.x); }

// Flux through a face with Courant number a between cells lo and hi, upwind
// value: a (a > 0 ? lo : hi).  It is the limiter's in/out flux with the raw
// face and, with the limited face, half the donor-cell flux of
// smolar_pass.c:104 (L(a+|a|) + R(a-|a|) = 2 a (a > 0 ? L : R)).
__device__ __forceinline__ float flux(float a, float lo, float hi) { return a * (a > 0.f ? lo : hi); }
__device__ __forceinline__ float2 flux2(float2 a, float2 lo, float2 hi)
{
    return a * make_float2(a.x > 0.f ? lo.x : hi.x, a.y > 0.f ? lo.y : hi.y);
}

// Antidiffusive face from regrouped parts (the face_pattern of common.cuh):
//   |a|(1-|a|) D / (C + MINVAL) - a (s/4 + (b1 n1 / (d1 + MINVAL) + b2 n2 / (d2 + MINVAL)) / 8)
// with b1, b2 the four-face velocity sums (4 x the reference's averages) and
// s the divergence sum (-(a s)/4 is the reference's -DIV).
template <bool AP>
__device__ __forceinline__ float2 pattern2(float2 a, float2 D, float2 C, float2 b1, float2 n1,
                                           float2 d1, float2 b2, float2 n2, float2 d2, float2 s)
{
    const float2 eps = bc(FLT_MIN);
    const float2 ma = abs2(a);
    const float2 A = rat2<AP>((ma * (bc(1.f) - ma)) * D, C + eps);
    const float2 X = rat2<AP>(b1 * n1, d1 + eps);
    const float2 Z = rat2<AP>(b2 * n2, d2 + eps);
    const float2 inner = fma2(bc(0.125f), X + Z, bc(0.25f) * s);
    return fma2(make_float2(-a.x, -a.y), inner, A);
}

// Staged values the three high faces of a pair read (plane k unless noted;
// suffix _m1/_2 = x - 1 / x + 2 of cell A, pairs are (A, B) columns).
struct PairNb {
    float2 c, cU, cD;            // c rows y, y+1, y-1
    float c_m1, c_2, cU_m1, cU_2, cD_2;
    float2 P, PD, PU;            // c plane k+1 rows y, y-1, y+1
    float P_m1, P_2;
    float2 M, MU;                // c plane k-1 rows y, y+1
    float M_2;
    float2 u, um, uU, uUm;       // x faces: (u0,u1), (u-2,u-1), row y+1 likewise
    float u_2;
    float2 up;                   // x faces plane k+1
    float up_m1;
    float2 v, vD, vU, vp, vpD;   // y faces: rows y, y-1, y+1; plane k+1 rows y, y-1
    float v_2, vD_2;
    float2 wm, wmU, w, wU, wp;   // z faces: face-planes k-1 (rows y, y+1), k (rows y, y+1), k+1
    float wm_2, w_2;
};

__device__ __forceinline__ PairNb gather(const float* c_m, const float* c_0, const float* c_p,
                                         const float* u_0, const float* u_p, const float* v_0,
                                         const float* v_p, const float* w_m, const float* w_0,
                                         const float* w_p, int o, float2 own_c, float2 own_m,
                                         float2 own_p)
{
    constexpr int Y = SBX;
    PairNb n;
    n.c = own_c; n.c_m1 = c_0[o - 1]; n.c_2 = c_0[o + 2];
    n.cU = ld2(c_0 + o + Y); n.cU_m1 = c_0[o + Y - 1]; n.cU_2 = c_0[o + Y + 2];
    n.cD = ld2(c_0 + o - Y); n.cD_2 = c_0[o - Y + 2];
    n.P = own_p; n.P_m1 = c_p[o - 1]; n.P_2 = c_p[o + 2];
    n.PD = ld2(c_p + o - Y); n.PU = ld2(c_p + o + Y);
    n.M = own_m; n.M_2 = c_m[o + 2]; n.MU = ld2(c_m + o + Y);
    n.u = ld2(u_0 + o); n.um = ld2(u_0 + o - 2); n.u_2 = u_0[o + 2];
    n.uU = ld2(u_0 + o + Y); n.uUm = ld2(u_0 + o + Y - 2);
    n.up = ld2(u_p + o); n.up_m1 = u_p[o - 1];
    n.v = ld2(v_0 + o); n.v_2 = v_0[o + 2];
    n.vD = ld2(v_0 + o - Y); n.vD_2 = v_0[o - Y + 2];
    n.vU = ld2(v_0 + o + Y);
    n.vp = ld2(v_p + o); n.vpD = ld2(v_p + o - Y);
    n.wm = ld2(w_m + o); n.wm_2 = w_m[o + 2]; n.wmU = ld2(w_m + o + Y);
    n.w = ld2(w_0 + o); n.w_2 = w_0[o + 2]; n.wU = ld2(w_0 + o + Y);
    n.wp = ld2(w_p + o);
    return n;
}

// Per-thread geometry of the pair: which faces exist and which take the
// boundary forms (only evaluated by CTAs that touch the domain boundary).
struct PairGeo {
    bool ux, uy;        // x face of A / B exists (0 <= i <= nx-2, j interior)
    bool xlo_x, xlo_y;  // x face is the low boundary face (i == 0)
    bool xhi_x, xhi_y;  // x face is the high boundary face (i == nx-2)
    bool vx, vy;        // y face exists (i interior, 0 <= j <= ny-2)
    bool ylo, yhi;      // y face is a boundary face (j == 0 / j == ny-2)
    bool qx, qy;        // y face is the column the reference leaves unwritten (vv.c:81-82)
    bool cx, cy;        // cell interior (z face exists)
};

__device__ __forceinline__ PairGeo pair_geo(const Dims& d, int iA, int j, int vv_fix)
{
    const int iB = iA + 1, nx = d.nx, ny = d.ny;
    const bool jin = j >= 1 && j <= ny - 2;
    PairGeo g;
    g.ux = iA >= 0 && iA <= nx - 2 && jin;
    g.uy = iB >= 0 && iB <= nx - 2 && jin;
    g.xlo_x = iA == 0; g.xlo_y = iB == 0;
    g.xhi_x = iA == nx - 2; g.xhi_y = iB == nx - 2;
    const bool jv = j >= 0 && j <= ny - 2;
    g.vx = iA >= 1 && iA <= nx - 2 && jv;
    g.vy = iB >= 1 && iB <= nx - 2 && jv;
    g.ylo = j == 0; g.yhi = j == ny - 2;
    const bool jq = !vv_fix && j >= 1 && j <= ny - 3;
    g.qx = jq && iA == 1; g.qy = jq && iB == 1;
    g.cx = iA >= 1 && iA <= nx - 2 && jin;
    g.cy = iB >= 1 && iB <= nx - 2 && jin;
    return g;
}

// Shared per-pair sums of the previous faces (plane k).
struct PairSums {
    float2 SV, SW, SU, dv, dw, du, e;
    float SV2, SW2, e2;
};

__device__ __forceinline__ PairSums pair_sums(const PairNb& n)
{
    PairSums q;
    q.SV = n.v + n.vD; q.SV2 = n.v_2 + n.vD_2;
    q.SW = n.w + n.wm; q.SW2 = n.w_2 + n.wm_2;
    q.SU = sum_l(n.um.y, n.u);   // u + (the cell's low x face)
    q.du = dif_l(n.um.y, n.u);
    q.dv = n.v - n.vD;
    q.dw = n.w - n.wm;
    q.e = (q.du - q.dv) - q.dw;
    q.e2 = ((n.u_2 - n.u.y) - (n.v_2 - n.vD_2)) - (n.w_2 - n.wm_2);
    return q;
}

// x faces of A and B (A's is the face between A and B).
template <bool AP, bool BORDER>
__device__ __forceinline__ float2 face_x(const PairNb& n, const PairSums& q, const PairGeo& g,
                                         bool use_div)
{
    const float2 C = sum_r(n.c, n.c_2), D = dif_r(n.c, n.c_2);
    const float2 CU = sum_r(n.cU, n.cU_2), CD = sum_r(n.cD, n.cD_2);
    const float2 CP = sum_r(n.P, n.P_2), CM = sum_r(n.M, n.M_2);
    float2 vb = sum_r(q.SV, q.SV2), wb = sum_r(q.SW, q.SW2), s = sum_r(q.e, q.e2);
    if (!use_div) s = bc(0.f);
    if constexpr (BORDER) {  // boundary faces: the inner cell's pair sum doubled, no divergence
        const float2 vlo = make_float2(q.SV.y + q.SV.y, q.SV2 + q.SV2);
        const float2 wlo = make_float2(q.SW.y + q.SW.y, q.SW2 + q.SW2);
        vb = pick(g.xlo_x, g.xlo_y, vlo, pick(g.xhi_x, g.xhi_y, q.SV + q.SV, vb));
        wb = pick(g.xlo_x, g.xlo_y, wlo, pick(g.xhi_x, g.xhi_y, q.SW + q.SW, wb));
        s = pick(g.xlo_x || g.xhi_x, g.xlo_y || g.xhi_y, bc(0.f), s);
    }
    const float2 r = pattern2<AP>(n.u, D, C, vb, CU - CD, CU + CD, wb, CP - CM, CP + CM, s);
    if constexpr (BORDER) return pick(g.ux, g.uy, r, bc(0.f));
    return r;
}

// y faces of A and B (between rows y and y+1).
template <bool AP, bool BORDER>
__device__ __forceinline__ float2 face_y(const PairNb& n, const PairSums& q, const PairGeo& g,
                                         const Dims& d, const float* __restrict__ Vadv, int j,
                                         int k, int pass, bool use_div)
{
    const float2 C = n.c + n.cU, D = n.cU - n.c;
    // x-gradient across the face: C(x+1) - C(x-1), lane-wise
    const float sl = n.c_m1 + n.cU_m1, sr = n.c_2 + n.cU_2;
    const float2 n1 = make_float2(C.y - sl, sr - C.x), d1 = make_float2(C.y + sl, sr + C.x);
    const float2 CP = n.P + n.PU, CM = n.M + n.MU;
    const float2 SUu = sum_l(n.uUm.y, n.uU), SWu = n.wU + n.wmU;
    float2 ub = q.SU + SUu, wb = q.SW + SWu;
    const float2 fy = q.dv - q.dw, fu = (n.vU - n.v) - (n.wU - n.wmU);
    // du of the column to the left (the reference's uL - uL2 terms, vv.c:85-89)
    const float dulA = (n.um.y - n.um.x) + (n.uUm.y - n.uUm.x);
    const float dulB = q.du.x + (n.uU.x - n.uUm.y);
    float2 s = (fy + fu) + make_float2(dulA, dulB);
    if (!use_div) s = bc(0.f);
    if constexpr (BORDER) {
        if (g.ylo) { ub = SUu + SUu; wb = SWu + SWu; s = bc(0.f); }
        if (g.yhi) { ub = q.SU + q.SU; wb = q.SW + q.SW; s = bc(0.f); }
    }
    float2 r = pattern2<AP>(n.v, D, C, ub, n1, d1, wb, CP - CM, CP + CM, s);
    if constexpr (BORDER) {
        if (g.qx || g.qy) {  // column i = 1: 0 on odd passes, the advective face on even ones
            const float qv = (pass & 1) ? 0.f : Vadv[cell(d, 1, j, k)];
            r = pick(g.qx, g.qy, bc(qv), r);
        }
        r = pick(g.vx, g.vy, r, bc(0.f));
    }
    return r;
}

// z faces of A and B (between planes k and k+1).
template <bool AP, bool BORDER>
__device__ __forceinline__ float2 face_z(const PairNb& n, const PairSums& q, const PairGeo& g,
                                         bool zlo, bool zhi, bool use_div)
{
    const float2 C = n.c + n.P, D = n.P - n.c;
    const float sl = n.c_m1 + n.P_m1, sr = n.c_2 + n.P_2;
    const float2 n1 = make_float2(C.y - sl, sr - C.x), d1 = make_float2(C.y + sl, sr + C.x);
    const float2 CU = n.cU + n.PU, CD = n.cD + n.PD;
    const float2 SUp = sum_l(n.up_m1, n.up), SVp = n.vp + n.vpD;
    float2 ub = q.SU + SUp, vb = q.SV + SVp;
    const float2 g0 = (q.dw - q.du) - q.dv;
    const float2 gp = ((n.wp - n.w) - dif_l(n.up_m1, n.up)) - (n.vp - n.vpD);
    float2 s = g0 + gp;
    if (!use_div) s = bc(0.f);
    if (zlo) { ub = SUp + SUp; vb = SVp + SVp; s = bc(0.f); }
    if (zhi) { ub = q.SU + q.SU; vb = q.SV + q.SV; s = bc(0.f); }
    const float2 r = pattern2<AP>(n.w, D, C, ub, n1, d1, vb, CU - CD, CU + CD, s);
    if constexpr (BORDER) return pick(g.cx, g.cy, r, bc(0.f));
    return r;
}

// Limited face: a min(1, beta_out(lo), beta_in(hi)) for a > 0, a min(1, beta_in(lo),
// beta_out(hi)) otherwise; the ratios are stored already clamped to <= 1.
__device__ __forceinline__ float limit(float a, float bu_lo, float bd_lo, float bu_hi, float bd_hi)
{
    return a * (a > 0.f ? fminf(bd_lo, bu_hi) : fminf(bu_lo, bd_hi));
}

}  // namespace pair

template <bool LIM, bool AP, bool BORDER>
__device__ __forceinline__ void pair_march(const Dims& d, const PassArgs<float>& a,
                                           const CUtensorMap* map_c, const CUtensorMap* map_uo,
                                           const CUtensorMap* map_vo, const CUtensorMap* map_wo,
                                           unsigned char* smem, int i0, int j0)
{
    using namespace pair;
    constexpr int SB = stage_bytes();
    constexpr int Y = SBX;
    float* work = reinterpret_cast<float*>(smem + (size_t)NSTAGE * 4 * SB);
    // limiter: fluxes of the raw high faces, bound extrema, ratios, donor fluxes (two slots)
    float* sFX = work;
    float* sFY = sFX + WPL;
    float* sMX = sFY + WPL;
    float* sMN = sMX + WPL;
    float* sBU = sMN + WPL;
    float* sBD = sBU + WPL;
    float* sDX = LIM ? sBD + WPL : work;          // donor x fluxes (LIM: slots at +0 / +WPL)
    float* sDY = LIM ? sDX + 2 * WPL : work + WPL;
    uint64_t* bars = reinterpret_cast<uint64_t*>(work + n_work<LIM>() * WPL);

    const int ny = d.ny, ns = d.ns;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int gx0 = (i0 - 2) & ~3, gy0 = j0 - 1, rx = (i0 - 2) - gx0;
    const int o = (ty + 1) * Y + 2 * tx + 2 + rx;  // cell A in a staged plane (even: 8-byte pairs)
    const int w = (ty + 1) * WX + 2 * tx + 2;      // cell A in a work plane (even)
    const int xA = 2 * tx;
    const int iA = i0 + xA, j = j0 + ty;
    const PairGeo g = pair_geo(d, iA, j, a.vv_fix);
    // cells this CTA updates (and whose faces it writes)
    const int ox0 = LIM ? 3 : 1, ox1 = CX - 2, oy0 = LIM ? 2 : 1, oy1 = LIM ? CY - 2 : CY - 1;
    const bool own_y = ty >= oy0 && ty <= oy1;
    const bool ownA = own_y && xA >= ox0 && xA <= ox1 && (!BORDER || g.cx);
    const bool ownB = own_y && xA + 1 >= ox0 && xA + 1 <= ox1 && (!BORDER || g.cy);
    // faces on the low domain boundary are written by the CTA holding the shell cell
    const bool wxA = own_y && ((xA >= ox0 && xA <= ox1) || iA == 0) && g.ux;
    const bool wxB = own_y && ((xA + 1 >= ox0 && xA + 1 <= ox1) || iA + 1 == 0) && g.uy;
    const bool wy_row = own_y || j == 0;
    const bool wyA = wy_row && xA >= ox0 && xA <= ox1 && g.vx;
    const bool wyB = wy_row && xA + 1 >= ox0 && xA + 1 <= ox1 && g.vy;
    // The step input c^n: 64-bit loads of the pair (rows inside the grid,
    // columns inside the pitch).  The ring cells on the high sides (x = 31,
    // y = CY-1) bound over a neighbour outside the CTA, whose c^n the edge
    // threads read as well (x + 2 / the row above).
    const bool cn_ok = LIM && j >= 0 && j < ny && iA >= 0 && iA < d.px;
    const bool edge_x = LIM && tx == TX - 1, edge_y = LIM && ty == CY - 1;
    const bool cnR_ok = edge_x && j >= 0 && j < ny && iA + 2 < d.px;
    const bool cnU_ok = edge_y && j + 1 >= 0 && j + 1 < ny && iA >= 0 && iA < d.px;

    if (tid == 0) {
        for (int s = 0; s < NSTAGE; s++) tma::mbar_init(&bars[s], 1);
        tma::fence_barrier_init();
        tma::prefetch_map(map_c);
        tma::prefetch_map(map_uo);
        tma::prefetch_map(map_vo);
        tma::prefetch_map(map_wo);
    }
    __syncthreads();

    auto slot = [&](int s, int arr) -> const float* {
        return reinterpret_cast<const float*>(smem + (size_t)(s * 4 + arr) * SB);
    };
    auto issue = [&](int p) {
        const int s = p & (NSTAGE - 1);
        uint64_t* bar = &bars[s];
        tma::fence_proxy_async_shared();
        tma::mbar_arrive_expect_tx(bar, (uint32_t)(4 * SBX * SBY * sizeof(float)));
        tma::load_3d(const_cast<float*>(slot(s, 0)), map_c, gx0, gy0, p, bar);
        tma::load_3d(const_cast<float*>(slot(s, 1)), map_uo, gx0, gy0, p, bar);
        tma::load_3d(const_cast<float*>(slot(s, 2)), map_vo, gx0, gy0, p, bar);
        tma::load_3d(const_cast<float*>(slot(s, 3)), map_wo, gx0, gy0, p, bar);
    };
    // global element offsets: the pair's column (plane 0) and one plane
    const long long col = (long long)j * d.px + iA, pp = d.pp;
    const float* cn_col = a.cn + col;
    auto ldcn = [&](int k, long long kp) -> float2 {
        if (!cn_ok || k > ns - 1) return bc(0.f);
        return *reinterpret_cast<const float2*>(cn_col + kp);
    };
    auto ldcnR = [&](int k, long long kp) -> float {
        if (!cnR_ok || k > ns - 1) return 0.f;
        return cn_col[kp + 2];
    };
    auto ldcnU = [&](int k, long long kp) -> float2 {
        if (!cnU_ok || k > ns - 1) return bc(0.f);
        return *reinterpret_cast<const float2*>(cn_col + kp + d.px);
    };

    // z chunk (see k_pass_tma): warm-up planes so the first updated plane sees
    // exactly what an unchunked march would form.
    const int depth = a.zdepth > 0 ? a.zdepth : ns - 2;
    const int z0 = 1 + (int)blockIdx.z * depth;
    const int z1 = min(ns - 1, z0 + depth);
    const int kstart = max(0, z0 - (LIM ? 3 : 2));
    const int last = LIM ? z1 : z1 - 1;

    bool ok = true;
    int confirmed = kstart;
    if (tid == 0) {
        issue(kstart);
        issue(kstart + 1);
    }
    ok = tma::mbar_wait(&bars[kstart & (NSTAGE - 1)], 0);
    if (tid == 0 && ok) confirmed = kstart + 1;

    // state carried between planes (pairs of the own cells)
    float2 cq1 = bc(0.f), cq2 = ok ? ld2(slot(kstart & (NSTAGE - 1), 0) + o) : bc(0.f), cq3 = bc(0.f);
    const long long kp0 = (long long)kstart * pp;
    float2 cn_next = LIM ? ldcn(kstart + 1, kp0 + pp) : bc(0.f);  // c^n of plane k+1
    float cnR_cur = LIM ? ldcnR(kstart, kp0) : 0.f;  // edge threads: c^n of plane k at x+2 / y+1
    float2 cnU_cur = LIM ? ldcnU(kstart, kp0) : bc(0.f);
    float2 mx_m = bc(0.f), mn_m = bc(0.f);               // own bounds of plane k-1
    float2 mx_0 = bc(0.f), mn_0 = bc(0.f);               // own bounds of plane k
    if (LIM) {
        const float2 cn0 = ldcn(kstart, kp0);
        mx_0 = max2(cq2, cn0);
        mn_0 = min2(cq2, cn0);
    }
    float2 bu_prev = bc(1.f), bd_prev = bc(1.f);  // own ratios of plane k-1
    float2 rw_prev = bc(0.f), fz_prev = bc(0.f);  // raw z face k-1/2 and its limiter flux
    float2 dx_prev = bc(0.f), dy_prev = bc(0.f);  // own donor fluxes (x: A|B, B|x+2; y) of plane k-1
    float2 dz_prev = bc(0.f);                     // donor flux of the z face below

    auto plane = [&](auto Sc, const int k) {
        constexpr int S = decltype(Sc)::value;
        constexpr int SM1 = (S + NSTAGE - 1) % NSTAGE, SP1 = (S + 1) % NSTAGE;
        __syncthreads();
        if (tid == 0 && k + 2 <= min(ns - 1, last + 1)) issue(k + 2);
        const long long kp = (long long)k * pp;  // element offset of plane k
        float2 cn_next2 = bc(0.f), cnU_next = bc(0.f);
        float cnR_next = 0.f;
        if (LIM) {
            cn_next2 = ldcn(k + 2, kp + 2 * pp);
            cnR_next = ldcnR(k + 1, kp + pp);
            cnU_next = ldcnU(k + 1, kp + pp);
        }
        if (k + 1 <= ns - 1) {
            if (ok) ok = tma::mbar_wait(&bars[SP1], ((k + 1 - kstart) / NSTAGE) & 1);
            if (tid == 0 && ok) confirmed = k + 2;
            cq3 = ld2(slot(SP1, 0) + o);
        }
        const bool kin = k >= 1 && k <= ns - 2;

        // ---- raw faces of plane k (z: face-plane k) ----
        float2 ru = bc(0.f), rv = bc(0.f), rw = bc(0.f);
        float c2 = 0.f;      // c at x+2 (row y, plane k)
        float2 cU = bc(0.f); // c at y+1
        if (k <= ns - 2) {
            const PairNb nb = gather(slot(SM1, 0), slot(S, 0), slot(SP1, 0), slot(S, 1),
                                     slot(SP1, 1), slot(S, 2), slot(SP1, 2), slot(SM1, 3),
                                     slot(S, 3), slot(SP1, 3), o, cq2, cq1, cq3);
            const PairSums qs = pair_sums(nb);
            if (kin) {
                ru = face_x<AP, BORDER>(nb, qs, g, a.use_div);
                rv = face_y<AP, BORDER>(nb, qs, g, d, a.Vadv, j, k, a.pass, a.use_div);
            }
            rw = face_z<AP, BORDER>(nb, qs, g, k == 0, k == ns - 2, a.use_div);
            c2 = nb.c_2; cU = nb.cU;
        }

        if constexpr (LIM) {
            // own bounds of plane k+1 (c^(o) and c^n)
            const float2 mx_p = max2(cq3, cn_next), mn_p = min2(cq3, cn_next);
            // limiter fluxes of the own high faces
            const float fxI = flux(ru.x, cq2.x, cq2.y), fxH = flux(ru.y, cq2.y, c2);
            const float2 fyH = flux2(rv, cq2, cU), fzH = flux2(rw, cq2, cq3);
            st2(sFX + w, make_float2(fxI, fxH));
            st2(sFY + w, fyH);
            st2(sMX + w, mx_0);
            st2(sMN + w, mn_0);
            __syncthreads();

            // ---- ratios of plane k ----
            float2 bu = bc(1.f), bd = bc(1.f);
            if (kin) {
                const float fxL = sFX[w - 1];
                const float2 fyL = ld2(sFY + w - WX);
                // in: positive low-face and negative high-face fluxes; out: the rest
                // (max(f,0) - f = max(-f,0)).  x lane-wise: A's faces are L|A and
                // A|B, B's are A|B and B|x+2.
                const float pL = fmaxf(fxL, 0.f), pI = fmaxf(fxI, 0.f), pH = fmaxf(fxH, 0.f);
                const float2 finx = make_float2(pL + (pI - fxI), pI + (pH - fxH));
                const float2 foutx = make_float2((pL - fxL) + pI, (pI - fxI) + pH);
                const float2 z0v = bc(0.f);
                const float2 py = max2(fyL, z0v), pz = max2(fz_prev, z0v);
                const float2 hy = max2(fyH, z0v), hz = max2(fzH, z0v);
                const float2 fin = finx + ((py + pz) + ((hy - fyH) + (hz - fzH)));
                const float2 fout = foutx + (((py - fyL) + (pz - fz_prev)) + (hy + hz));
                // bounds over the cell and its face neighbours (z only in 3D)
                const float mAB = fmaxf(mx_0.x, mx_0.y), nAB = fminf(mn_0.x, mn_0.y);
                const float2 mD = ld2(sMX + w - WX), nD = ld2(sMN + w - WX);
                float2 mU, nU;
                float mR, nR;
                if (edge_y) { mU = max2(cU, cnU_cur); nU = min2(cU, cnU_cur); }
                else { mU = ld2(sMX + w + WX); nU = ld2(sMN + w + WX); }
                if (edge_x) { mR = fmaxf(c2, cnR_cur); nR = fminf(c2, cnR_cur); }
                else { mR = sMX[w + 2]; nR = sMN[w + 2]; }
                float2 mx = make_float2(fmaxf(mAB, sMX[w - 1]), fmaxf(mAB, mR));
                float2 mn = make_float2(fminf(nAB, sMN[w - 1]), fminf(nAB, nR));
                mx = max2(mx, max2(mD, mU));
                mn = min2(mn, min2(nD, nU));
                if (ns > 3) {
                    mx = max2(mx, max2(mx_m, mx_p));
                    mn = min2(mn, min2(mn_m, mn_p));
                }
                const float2 eps = bc(FLT_MIN);
                bu = min2(rat2<AP>(mx - cq2, fin + eps), bc(1.f));
                bd = min2(rat2<AP>(cq2 - mn, fout + eps), bc(1.f));
                if constexpr (BORDER) {
                    bu = pick(g.cx, g.cy, bu, bc(1.f));
                    bd = pick(g.cx, g.cy, bd, bc(1.f));
                }
            }
            st2(sBU + w, bu);
            st2(sBD + w, bd);
            __syncthreads();

            // ---- limited faces: x, y of plane k; z of face-plane k-1 ----
            float2 lu = ru, lv = rv;
            lu.x = limit(ru.x, bu.x, bd.x, bu.y, bd.y);
            if (tx < TX - 1) lu.y = limit(ru.y, bu.y, bd.y, sBU[w + 2], sBD[w + 2]);
            if (ty < CY - 1) {
                const float2 buU = ld2(sBU + w + WX), bdU = ld2(sBD + w + WX);
                lv = make_float2(limit(rv.x, bu.x, bd.x, buU.x, bdU.x),
                                 limit(rv.y, bu.y, bd.y, buU.y, bdU.y));
            }
            const float2 lw = make_float2(limit(rw_prev.x, bu_prev.x, bd_prev.x, bu.x, bd.x),
                                          limit(rw_prev.y, bu_prev.y, bd_prev.y, bu.y, bd.y));
            // donor fluxes of plane k (read by the neighbours' update one plane later)
            const float2 dx_cur = make_float2(flux(lu.x, cq2.x, cq2.y), flux(lu.y, cq2.y, c2));
            const float2 dy_cur = flux2(lv, cq2, cU);
            const float2 dz = flux2(lw, cq1, cq2);  // face k-1/2
            float* sDXk = sDX + (S & 1) * WPL;
            float* sDYk = sDY + (S & 1) * WPL;
            st2(sDXk + w, dx_cur);
            st2(sDYk + w, dy_cur);
            if (a.write_faces) {
                const long long q = col + kp;
                const bool mine_k = kin && k >= z0 && k < z1;
                if (mine_k) {
                    if (wxA) a.Un[q] = lu.x;
                    if (wxB) a.Un[q + 1] = lu.y;
                    if (wyA) a.Vn[q] = lv.x;
                    if (wyB) a.Vn[q + 1] = lv.y;
                }
                if (k >= 1 && k - 1 < z1 && (k - 1 >= z0 || k - 1 == 0)) {
                    if (ownA) a.Wn[q - pp] = lw.x;
                    if (ownB) a.Wn[q - pp + 1] = lw.y;
                }
            }

            // ---- donor update of plane k-1 ----
            const int u = k - 1;
            if (u >= z0 && u < z1 && (ownA || ownB)) {
                const float* sDXp = sDX + (SM1 & 1) * WPL;
                const float* sDYp = sDY + (SM1 & 1) * WPL;
                const float2 netx = make_float2(dx_prev.x - sDXp[w - 1], dx_prev.y - dx_prev.x);
                const float2 lowy = ld2(sDYp + w - WX);
                const float2 cnew = cq1 - ((netx + (dy_prev - lowy)) + (dz - dz_prev));
                float* out = a.c_out + (col + kp - pp);
                if (ownA && ownB) st2(out, cnew);
                else if (ownA) out[0] = cnew.x;
                else out[1] = cnew.y;
            }
            mx_m = mx_0; mn_m = mn_0;
            mx_0 = mx_p; mn_0 = mn_p;
            bu_prev = bu; bd_prev = bd;
            fz_prev = fzH;
            dx_prev = dx_cur; dy_prev = dy_cur;
            dz_prev = dz;
        } else {
            // donor fluxes of the raw faces of plane k
            const float2 dx_cur = make_float2(flux(ru.x, cq2.x, cq2.y), flux(ru.y, cq2.y, c2));
            const float2 dy_cur = flux2(rv, cq2, cU);
            const float2 dz = flux2(rw, cq2, cq3);  // face k+1/2
            st2(sDX + w, dx_cur);
            st2(sDY + w, dy_cur);
            __syncthreads();
            if (k >= z0 && k < z1) {
                const long long q = col + kp;
                if (ownA || ownB) {
                    const float2 netx = make_float2(dx_cur.x - sDX[w - 1], dx_cur.y - dx_cur.x);
                    const float2 lowy = ld2(sDY + w - WX);
                    const float2 cnew = cq2 - ((netx + (dy_cur - lowy)) + (dz - dz_prev));
                    float* out = a.c_out + q;
                    if (ownA && ownB) st2(out, cnew);
                    else if (ownA) out[0] = cnew.x;
                    else out[1] = cnew.y;
                }
                if (a.write_faces) {
                    if (wxA) a.Un[q] = ru.x;
                    if (wxB) a.Un[q + 1] = ru.y;
                    if (wyA) a.Vn[q] = rv.x;
                    if (wyB) a.Vn[q + 1] = rv.y;
                    if (ownA) a.Wn[q] = rw.x;
                    if (ownB) a.Wn[q + 1] = rw.y;
                }
            } else if (k == 0 && z0 == 1 && a.write_faces) {  // face-plane 0 (below plane 1)
                if (ownA) a.Wn[col] = rw.x;
                if (ownB) a.Wn[col + 1] = rw.y;
            }
            dz_prev = dz;
        }
        rw_prev = rw;
        cq1 = cq2;
        cq2 = cq3;
        if (LIM) {
            cn_next = cn_next2;
            cnR_cur = cnR_next;
            cnU_cur = cnU_next;
        }
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

template <bool LIM, bool AP>
__global__ void __launch_bounds__(pair::NT, pair::NT >= 512 ? 1 : 2)
    k_pass_pair(Dims d, PassArgs<float> a, const __grid_constant__ CUtensorMap map_c,
                const __grid_constant__ CUtensorMap map_uo, const __grid_constant__ CUtensorMap map_vo,
                const __grid_constant__ CUtensorMap map_wo)
{
    using namespace pair;
    extern __shared__ __align__(128) unsigned char smem[];
    const int i0 = LIM ? stride_x<LIM>() * (int)blockIdx.x - 2 : stride_x<LIM>() * (int)blockIdx.x;
    const int j0 = LIM ? stride_y<LIM>() * (int)blockIdx.y - 1 : stride_y<LIM>() * (int)blockIdx.y;
    // CTAs whose every face is an interior face of the interior pattern take
    // the branch-free path (no boundary forms, no existence masks, no i = 1 column).
    const bool interior = i0 >= 2 && i0 + CX - 1 <= d.nx - 3 && j0 >= 1 && j0 + CY - 1 <= d.ny - 3;
    if (interior)
        pair_march<LIM, AP, false>(d, a, &map_c, &map_uo, &map_vo, &map_wo, smem, i0, j0);
    else
        pair_march<LIM, AP, true>(d, a, &map_c, &map_uo, &map_vo, &map_wo, smem, i0, j0);
}

template <bool LIM, bool AP>
int launch_pair_variant(const Dims& d, const PassArgs<float>& a, cudaStream_t s)
{
    using namespace pair;
    constexpr size_t smem = smem_bytes<LIM>();
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_pass_pair<LIM, AP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        configured = true;
    }
    const int depth = a.zdepth > 0 ? a.zdepth : d.ns - 2;
    dim3 g((d.nx - 2 + stride_x<LIM>() - 1) / stride_x<LIM>(),
           (d.ny - 2 + stride_y<LIM>() - 1) / stride_y<LIM>(), (d.ns - 2 + depth - 1) / depth);
    dim3 b(TX, CY);
    k_pass_pair<LIM, AP><<<g, b, smem, s>>>(d, a, *a.maps2.c, *a.maps2.uo, *a.maps2.vo, *a.maps2.wo);
    return 1;
}

int launch_pass_pair(const Dims& d, const PassArgs<float>& a, cudaStream_t s)
{
    if (a.limiter) return a.approx ? launch_pair_variant<true, true>(d, a, s) : launch_pair_variant<true, false>(d, a, s);
    return a.approx ? launch_pair_variant<false, true>(d, a, s) : launch_pair_variant<false, false>(d, a, s);
}
