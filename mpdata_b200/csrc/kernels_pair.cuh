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
//    fluxes of each cell's high faces, the ratios (clamped to <= 1) and the
//    donor fluxes F = a (a > 0 ? c_lo : c_hi), so the donor update needs no
//    neighbour c values.  A donor flux is the raw face's limiter flux,
//    carried from the plane before, times the limiter factor.
//  * The limiter's bounds come from the staged planes and the values the
//    faces read, with three-input min / max.
//  * No extra low faces are formed: the CTA's cells overlap their
//    neighbours' (with the limiter x 0..2 and 31, rows 0, 1 and CY-1 are not
//    updated; without it x 0 and 31 and row 0), so every face a kept cell
//    needs is the high face of a cell of the same CTA.
//  * No divergent branches in the plane body: tile-edge threads select, and
//    owned lanes are written by predicated scalar stores.
//  * The precision form (WIDE): a non-zero limiter in/out sum near zero is
//    formed again in FP64 from its flux parts and its ratio divided in FP64;
//    every ratio is shrunk by 2^-20 so rounding cannot break positivity.
//
// Per plane k (limiter): [limited x/y faces of plane k-1, limited z face
// k-3/2, donor fluxes, update of plane k-2; raw faces of plane k and z face
// k+1/2] -> sync -> [ratios of plane k] -> sync.  Without the limiter the
// update of plane k follows the raw faces after one sync.
//
// The planes of c, the previous faces and (with the limiter) the step input
// c^n are staged by TMA, four planes deep.  Every wait is bounded (tma.cuh).
//
// Included by kernels_pair.cu inside namespace mpd::fast.

namespace pair {

template <int V> struct IC {  // compile-time stage slot of one unrolled plane
    static constexpr int value = V;
};
struct RC {  // stage slot of a plane of a rolled loop
    int value;
};

constexpr int TX = 16, CX = 2 * TX, CY = kPairCY, NT = TX * CY;
constexpr int SBX = kPairBoxX, SBY = kPairBoxY;  // staged box: x [-2-rx, 37-rx], y [-1, CY]
constexpr int NSTAGE = 4;
constexpr int WX = 36, WY = CY + 1, WPL = WX * WY;  // work planes: x [-2, 33], y [-1, CY-1]

__host__ __device__ constexpr int stage_bytes() { return (SBX * SBY * 4 + 127) / 128 * 128; }
// staged arrays: c, Uo, Vo, Wo (+ c^n with the limiter)
template <bool LIM> __host__ __device__ constexpr int n_arrays() { return LIM ? 5 : 4; }
template <bool LIM> __host__ __device__ constexpr int n_work() { return LIM ? 10 : 2; }
template <bool LIM> __host__ __device__ constexpr size_t smem_bytes()
{
    return (size_t)NSTAGE * n_arrays<LIM>() * stage_bytes() + (size_t)n_work<LIM>() * WPL * 4 +
           NSTAGE * 8;
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
// Three-input max / min (PTX max.f32 / min.f32 with three operands, sm_100).
__device__ __forceinline__ float max3f(float a, float b, float c)
{
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float min3f(float a, float b, float c)
{
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
// (a.y, b) and (a, b.x): the pair shifted by one cell to the right / left.
__device__ __forceinline__ float2 sh(float2 a, float b) { return make_float2(a.y, b); }
__device__ __forceinline__ float2 shl(float a, float2 b) { return make_float2(a, b.x); }
__device__ __forceinline__ float2 pick(bool px, bool py, float2 a, float2 b)
{
    return make_float2(px ? a.x : b.x, py ? a.y : b.y);
}
__device__ __forceinline__ float2 ld2(const float* p) { return *reinterpret_cast<const float2*>(p); }
__device__ __forceinline__ void st2(float* p, float2 v) { *reinterpret_cast<float2*>(p) = v; }

// Lane-wise n / d: hardware reciprocal (approx_div) or round-to-nearest
// division without the slow-path call (div_nearest, IEEE results).
template <bool AP> __device__ __forceinline__ float2 rat2(float2 n, float2 d)
{
    if constexpr (AP) return n * make_float2(rcp_approx(d.x), rcp_approx(d.y));
    else return make_float2(div_nearest(n.x, d.x), div_nearest(n.y, d.y));
}
// min(n / d, 1) lane-wise for n >= 0 (the limiter's clamped ratios).
template <bool AP> __device__ __forceinline__ float2 rat2_min1(float2 n, float2 d)
{
    if constexpr (AP) return min2(rat2<true>(n, d), bc(1.f));
    else return make_float2(div_nearest<true>(n.x, d.x), div_nearest<true>(n.y, d.y));
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

// Limiter factor of a face: min(1, beta_out(lo), beta_in(hi)) for a > 0,
// min(1, beta_in(lo), beta_out(hi)) otherwise; the ratios are stored already
// clamped to <= 1.  The limited face is a times it, and its flux (upwind
// value from the same c) the raw face's flux times it.
__device__ __forceinline__ float lim_factor(float a, float bu_lo, float bd_lo, float bu_hi,
                                            float bd_hi)
{
    return a > 0.f ? fminf(bd_lo, bu_hi) : fminf(bu_lo, bd_hi);
}

}  // namespace pair

// Per-thread placement shared by both marches.
struct PairSetup {
    int gx0, gy0;       // box origin of the staged planes (x 16-byte aligned)
    int o, w;           // cell A in a staged plane / a work plane (both even: 8-byte pairs)
    int xA, iA, j;      // local x of A, global i of A, global j
    pair::PairGeo g;
    bool ownA, ownB;    // cells this CTA updates
    bool wxA, wxB, wyA, wyB;  // x / y faces this CTA writes (incl. the low domain faces)
    long long col;      // element offset of (iA, j, 0)
};

template <bool LIM, bool BORDER>
__device__ __forceinline__ PairSetup pair_setup(const Dims& d, const PassArgs<float>& a, int i0, int j0)
{
    using namespace pair;
    PairSetup p;
    const int tx = threadIdx.x, ty = threadIdx.y;
    p.gx0 = (i0 - 2) & ~3;
    p.gy0 = j0 - 1;
    const int rx = (i0 - 2) - p.gx0;
    p.o = (ty + 1) * SBX + 2 * tx + 2 + rx;
    p.w = (ty + 1) * WX + 2 * tx + 2;
    p.xA = 2 * tx;
    p.iA = i0 + p.xA;
    p.j = j0 + ty;
    p.g = pair_geo(d, p.iA, p.j, a.vv_fix);
    const int ox0 = LIM ? 3 : 1, ox1 = CX - 2, oy0 = LIM ? 2 : 1, oy1 = LIM ? CY - 2 : CY - 1;
    const bool own_y = ty >= oy0 && ty <= oy1;
    const bool inA = p.xA >= ox0 && p.xA <= ox1, inB = p.xA + 1 >= ox0 && p.xA + 1 <= ox1;
    p.ownA = own_y && inA && (!BORDER || p.g.cx);
    p.ownB = own_y && inB && (!BORDER || p.g.cy);
    // faces on the low domain boundary are written by the CTA holding the shell cell
    p.wxA = own_y && (inA || p.iA == 0) && p.g.ux;
    p.wxB = own_y && (inB || p.iA + 1 == 0) && p.g.uy;
    const bool wy_row = own_y || p.j == 0;
    p.wyA = wy_row && inA && p.g.vx;
    p.wyB = wy_row && inB && p.g.vy;
    p.col = (long long)p.j * d.px + p.iA;
    return p;
}

// Store the lanes of a pair this CTA owns, each as its own predicated scalar
// store.  Measured faster than one 8-byte store behind a branch on ownership
// (tile-edge pairs own one lane, so that branch diverges).
__device__ __forceinline__ void store_lanes(float* out, float2 v, bool a, bool b)
{
    if (a) out[0] = v.x;
    if (b) out[1] = v.y;
}

// ---- without the limiter: faces of plane k -> sync -> update of plane k ----
template <bool AP, bool BORDER>
__device__ __forceinline__ void pair_march_plain(const Dims& d, const PassArgs<float>& a,
                                                 const CUtensorMap* map_c, const CUtensorMap* map_uo,
                                                 const CUtensorMap* map_vo, const CUtensorMap* map_wo,
                                                 unsigned char* smem, int i0, int j0)
{
    using namespace pair;
    constexpr int NARR = n_arrays<false>();
    constexpr int SB = stage_bytes();
    float* work = reinterpret_cast<float*>(smem + (size_t)NSTAGE * NARR * SB);
    float* sDX = work;        // donor fluxes through the x faces of plane k (A|B, B|x+2)
    float* sDY = work + WPL;  // through the y faces
    uint64_t* bars = reinterpret_cast<uint64_t*>(work + n_work<false>() * WPL);
    const PairSetup p = pair_setup<false, BORDER>(d, a, i0, j0);
    const int ns = d.ns;
    const int tid = threadIdx.y * TX + threadIdx.x;
    const long long pp = d.pp;

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
        return reinterpret_cast<const float*>(smem + (size_t)(s * NARR + arr) * SB);
    };
    auto issue = [&](int pl) {
        const int s = pl & (NSTAGE - 1);
        uint64_t* bar = &bars[s];
        tma::fence_proxy_async_shared();
        tma::mbar_arrive_expect_tx(bar, (uint32_t)(NARR * SBX * SBY * sizeof(float)));
        tma::load_3d(const_cast<float*>(slot(s, 0)), map_c, p.gx0, p.gy0, pl, bar);
        tma::load_3d(const_cast<float*>(slot(s, 1)), map_uo, p.gx0, p.gy0, pl, bar);
        tma::load_3d(const_cast<float*>(slot(s, 2)), map_vo, p.gx0, p.gy0, pl, bar);
        tma::load_3d(const_cast<float*>(slot(s, 3)), map_wo, p.gx0, p.gy0, pl, bar);
    };

    // z chunk (see k_pass_tma): two warm-up planes, the first for the z face below
    const int zb = a.zbase > 0 ? a.zbase : 1, ze = a.zend > 0 ? a.zend : ns - 1;
    const int depth = a.zdepth > 0 ? a.zdepth : ze - zb;
    const int z0 = zb + (int)blockIdx.z * depth;
    const int z1 = min(ze, z0 + depth);
    const int kstart = max(0, z0 - 2);
    const int last = z1 - 1;
    const int issue_max = min(ns - 1, last + 1);

    bool ok = true;
    int confirmed = kstart;
    if (tid == 0) {
        issue(kstart);
        issue(kstart + 1);
    }
    ok = tma::mbar_wait(&bars[kstart & (NSTAGE - 1)], 0);
    if (tid == 0 && ok) confirmed = kstart + 1;
    float2 cq1 = bc(0.f), cq2 = ok ? ld2(slot(kstart & (NSTAGE - 1), 0) + p.o) : bc(0.f), cq3 = bc(0.f);
    float2 dz_prev = bc(0.f);  // donor flux through the z face below plane k

    auto plane = [&](auto Sc, const int k) {
        constexpr int S = decltype(Sc)::value;
        constexpr int SM1 = (S + NSTAGE - 1) % NSTAGE, SP1 = (S + 1) % NSTAGE;
        __syncthreads();  // every read of the slot plane k+2 reuses is done
        if (tid == 0 && k + 2 <= issue_max) issue(k + 2);
        if (k + 1 <= ns - 1) {
            if (ok) ok = tma::mbar_wait(&bars[SP1], ((k + 1 - kstart) / NSTAGE) & 1);
            if (tid == 0 && ok) confirmed = k + 2;
            cq3 = ld2(slot(SP1, 0) + p.o);
        }
        const bool kin = k >= 1 && k <= ns - 2;
        float2 ru = bc(0.f), rv = bc(0.f), rw = bc(0.f), cU;
        float c2;
        {
            const PairNb nb = gather(slot(SM1, 0), slot(S, 0), slot(SP1, 0), slot(S, 1),
                                     slot(SP1, 1), slot(S, 2), slot(SP1, 2), slot(SM1, 3),
                                     slot(S, 3), slot(SP1, 3), p.o, cq2, cq1, cq3);
            const PairSums qs = pair_sums(nb);
            if (kin) {
                ru = face_x<AP, BORDER>(nb, qs, p.g, a.use_div);
                rv = face_y<AP, BORDER>(nb, qs, p.g, d, a.Vadv, p.j, k, a.pass, a.use_div);
            }
            rw = face_z<AP, BORDER>(nb, qs, p.g, k == 0, k == ns - 2, a.use_div);
            c2 = nb.c_2;
            cU = nb.cU;
        }
        const float2 dx = make_float2(flux(ru.x, cq2.x, cq2.y), flux(ru.y, cq2.y, c2));
        const float2 dy = flux2(rv, cq2, cU);
        const float2 dz = flux2(rw, cq2, cq3);  // face k+1/2
        st2(sDX + p.w, dx);
        st2(sDY + p.w, dy);
        __syncthreads();
        if (k >= z0 && k < z1) {
            const long long q = p.col + (long long)k * pp;
            {  // every thread forms its pair's update; owned lanes are stored
                const float2 netx = make_float2(dx.x - sDX[p.w - 1], dx.y - dx.x);
                const float2 nety = dy - ld2(sDY + p.w - WX);
                store_lanes(a.c_out + q, cq2 - ((netx + nety) + (dz - dz_prev)), p.ownA, p.ownB);
            }
            if (a.write_faces) {
                if (p.wxA) a.Un[q] = ru.x;
                if (p.wxB) a.Un[q + 1] = ru.y;
                if (p.wyA) a.Vn[q] = rv.x;
                if (p.wyB) a.Vn[q + 1] = rv.y;
                store_lanes(a.Wn + q, rw, p.ownA, p.ownB);
            }
        } else if (k == 0 && z0 == 1 && a.write_faces) {  // face-plane 0 (below plane 1)
            store_lanes(a.Wn + p.col, rw, p.ownA, p.ownB);
        }
        dz_prev = dz;
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
        for (int pl = confirmed; pl <= issue_max; pl++)
            if (!tma::mbar_wait(&bars[pl & (NSTAGE - 1)], ((pl - kstart) / NSTAGE) & 1)) break;
    }
}

// ---- with the limiter ----
// Iteration k: [limited faces of plane k-1 and z face k-3/2, donor fluxes,
// update of plane k-2; raw faces of plane k and z face k+1/2 with their
// limiter fluxes and the bound extrema of plane k] -> sync -> [ratios of
// plane k] -> sync.  Ratios and donor fluxes live in two-slot rings (plane
// parity), so two barriers per plane suffice.
template <bool AP, bool WIDE, bool BORDER>
__device__ __forceinline__ void pair_march_lim(const Dims& d, const PassArgs<float>& a,
                                               const CUtensorMap* map_c, const CUtensorMap* map_cn,
                                               const CUtensorMap* map_uo, const CUtensorMap* map_vo,
                                               const CUtensorMap* map_wo, unsigned char* smem,
                                               int i0, int j0)
{
    using namespace pair;
    constexpr int NARR = n_arrays<true>();  // c, Uo, Vo, Wo, c^n
    constexpr int SB = stage_bytes();
    constexpr int Y = SBX;
    float* work = reinterpret_cast<float*>(smem + (size_t)NSTAGE * NARR * SB);
    float* sFX = work;           // limiter fluxes through the raw x faces of plane k (A|B, B|x+2)
    float* sFY = sFX + WPL;      // through the raw y faces
    float* sBU = sFY + WPL;      // ratios (clamped to <= 1), two slots by plane parity
    float* sBD = sBU + 2 * WPL;
    float* sDX = sBD + 2 * WPL;  // donor fluxes through the limited faces, two slots
    float* sDY = sDX + 2 * WPL;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sDY + 2 * WPL);
    const PairSetup p = pair_setup<true, BORDER>(d, a, i0, j0);
    const int ns = d.ns;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    // The ring cells at x = 31 and y = CY-1 bound over a neighbour outside the
    // CTA: the edge threads take its c and c^n from the staged planes.
    const bool edge_x = tx == TX - 1, edge_y = ty == CY - 1;
    const long long pp = d.pp;

    if (tid == 0) {
        for (int s = 0; s < NSTAGE; s++) tma::mbar_init(&bars[s], 1);
        tma::fence_barrier_init();
        tma::prefetch_map(map_c);
        tma::prefetch_map(map_cn);
        tma::prefetch_map(map_uo);
        tma::prefetch_map(map_vo);
        tma::prefetch_map(map_wo);
    }
    __syncthreads();
    auto slot = [&](int s, int arr) -> const float* {
        return reinterpret_cast<const float*>(smem + (size_t)(s * NARR + arr) * SB);
    };
    auto issue = [&](int pl) {
        const int s = pl & (NSTAGE - 1);
        uint64_t* bar = &bars[s];
        tma::fence_proxy_async_shared();
        tma::mbar_arrive_expect_tx(bar, (uint32_t)(NARR * SBX * SBY * sizeof(float)));
        tma::load_3d(const_cast<float*>(slot(s, 0)), map_c, p.gx0, p.gy0, pl, bar);
        tma::load_3d(const_cast<float*>(slot(s, 1)), map_uo, p.gx0, p.gy0, pl, bar);
        tma::load_3d(const_cast<float*>(slot(s, 2)), map_vo, p.gx0, p.gy0, pl, bar);
        tma::load_3d(const_cast<float*>(slot(s, 3)), map_wo, p.gx0, p.gy0, pl, bar);
        tma::load_3d(const_cast<float*>(slot(s, 4)), map_cn, p.gx0, p.gy0, pl, bar);
    };

    // z chunk: the update of plane u comes two iterations after its raw faces
    // (the limited z face above u needs the ratios of u+1).  Three warm-up
    // planes: the z face below, then the ratios below, then their limited face.
    const int zb = a.zbase > 0 ? a.zbase : 1, ze = a.zend > 0 ? a.zend : ns - 1;
    const int depth = a.zdepth > 0 ? a.zdepth : ze - zb;
    const int z0 = zb + (int)blockIdx.z * depth;
    const int z1 = min(ze, z0 + depth);
    const int kstart = max(0, z0 - 3);
    const int last_a = z1;      // last plane whose raw faces and ratios are formed
    const int last = z1 + 1;    // last iteration (update of plane z1 - 1)
    const int issue_max = min(ns - 1, last_a + 1);

    bool ok = true;
    int confirmed = kstart;
    if (tid == 0) {
        issue(kstart);
        issue(kstart + 1);
    }
    ok = tma::mbar_wait(&bars[kstart & (NSTAGE - 1)], 0);
    if (tid == 0 && ok) confirmed = kstart + 1;

    // state carried between planes (pairs of the own cells)
    float2 cq0 = bc(0.f), cq1 = bc(0.f);  // c of planes k-2, k-1
    float2 cq2 = ok ? ld2(slot(kstart & (NSTAGE - 1), 0) + p.o) : bc(0.f), cq3 = bc(0.f);
    float2 ru_prev = bc(0.f), rv_prev = bc(0.f);  // raw x / y faces of plane k-1
    float2 rw_prev = bc(0.f), rw_pp = bc(0.f);    // raw z faces k-1/2 and k-3/2
    float2 fx_prev = bc(0.f), fy_prev = bc(0.f);  // their limiter fluxes (x: A|B, B|x+2)
    float2 fz_prev = bc(0.f), fz_pp = bc(0.f);
    float2 dz_prev = bc(0.f);                     // donor flux through the limited z face k-5/2
    long long qk = p.col + (long long)kstart * pp;  // element offset of the pair in plane k

    // One iteration.  The last one (k = last_a + 1) only limits the faces of
    // plane k-1 and updates plane k-2, and needs no barrier.  It runs the
    // same compiled copy as every plane with the same stage slot (a separate
    // copy could contract multiply-adds differently, and a z chunk updates
    // its first plane in the last iteration), so chunked marches stay
    // bit-identical to unchunked ones; a rolled loop has one copy.
    auto plane = [&](auto Sc, const int k) {
        const int S = Sc.value;  // a constant in the unrolled loop
        const bool HA = k <= last_a;  // uniform over the CTA
        const int SM1 = (S + NSTAGE - 1) & (NSTAGE - 1), SP1 = (S + 1) & (NSTAGE - 1);
        const int PK = S & 1, PM = (S + 1) & 1;  // ring slots of planes k (and k-2) / k-1
        // (the previous iteration ended with a barrier: the slot plane k+2 reuses is free)
        if (HA && tid == 0 && k + 2 <= issue_max) issue(k + 2);

        // ---- limited faces of plane k-1 and z face k-3/2; update of plane k-2 ----
        {
            const float* bu1 = sBU + PM * WPL;  // ratios of plane k-1
            const float* bd1 = sBD + PM * WPL;
            const float2 bu = ld2(bu1 + p.w), bd = ld2(bd1 + p.w);
            const float2 bu2 = ld2(sBU + PK * WPL + p.w), bd2 = ld2(sBD + PK * WPL + p.w);
            // Limiter factors; the donor fluxes through the limited faces are the
            // raw faces' fluxes (formed with the same c) times them.  The edge
            // threads' outer faces (x = 31|32, y = CY-1|CY) have no ratio on the far
            // side in this CTA and stay raw (factor 1; no kept cell uses them); both
            // forms are evaluated and selected, without a divergent branch (the far
            // reads stay inside shared memory: x + 2 <= 33 < WX, and row CY + 1 of
            // a ratio plane is the first row of the next work array).
            const float buR = bu1[p.w + 2], bdR = bd1[p.w + 2];
            const float2 buU = ld2(bu1 + p.w + WX), bdU = ld2(bd1 + p.w + WX);
            const float myB = lim_factor(ru_prev.y, bu.y, bd.y, buR, bdR);
            const float2 gx = make_float2(lim_factor(ru_prev.x, bu.x, bd.x, bu.y, bd.y),
                                          edge_x ? 1.f : myB);
            float2 gy = make_float2(lim_factor(rv_prev.x, bu.x, bd.x, buU.x, bdU.x),
                                    lim_factor(rv_prev.y, bu.y, bd.y, buU.y, bdU.y));
            if (edge_y) gy = bc(1.f);
            const float2 gz = make_float2(lim_factor(rw_pp.x, bu2.x, bd2.x, bu.x, bd.x),
                                          lim_factor(rw_pp.y, bu2.y, bd2.y, bu.y, bd.y));
            const float2 dx = gx * fx_prev, dy = gy * fy_prev;
            const float2 dz = gz * fz_pp;  // face k-3/2
            st2(sDX + PM * WPL + p.w, dx);
            st2(sDY + PM * WPL + p.w, dy);
            const long long q1 = qk - pp;  // plane k-1
            if (a.write_faces) {
                const float2 lu = gx * ru_prev, lv = gy * rv_prev, lw = gz * rw_pp;
                if (k - 1 >= z0 && k - 1 < z1) {
                    if (p.wxA) a.Un[q1] = lu.x;
                    if (p.wxB) a.Un[q1 + 1] = lu.y;
                    if (p.wyA) a.Vn[q1] = lv.x;
                    if (p.wyB) a.Vn[q1 + 1] = lv.y;
                }
                // face-plane k-2: the high face of plane k-2, and face-plane 0 only in
                // the chunk that starts at plane 1 (a later chunk's warm-up does not form it)
                if (k >= 2 && k - 2 < z1 && (k - 2 >= z0 || (k - 2 == 0 && z0 == 1)))
                    store_lanes(a.Wn + (q1 - pp), lw, p.ownA, p.ownB);
            }
            const int u = k - 2;
            if (u >= z0 && u < z1) {  // uniform; every thread forms its pair's update
                const float* dxp = sDX + PK * WPL;  // donor fluxes of plane k-2
                const float* dyp = sDY + PK * WPL;
                const float2 dxo = ld2(dxp + p.w);
                const float2 netx = make_float2(dxo.x - dxp[p.w - 1], dxo.y - dxo.x);
                const float2 nety = ld2(dyp + p.w) - ld2(dyp + p.w - WX);
                store_lanes(a.c_out + (q1 - pp), cq0 - ((netx + nety) + (dz - dz_prev)), p.ownA,
                            p.ownB);
            }
            dz_prev = dz;
        }

        if (!HA) return;
        // ---- raw faces of plane k (z: face k+1/2), limiter fluxes, bound extrema ----
        const bool kin = k >= 1 && k <= ns - 2;
        float2 ru, rv, rw, cU, cD, fyH, fzH;
        float c2, cL, fxI, fxH;
        {
            if (k + 1 <= ns - 1) {
                if (ok) ok = tma::mbar_wait(&bars[SP1], ((k + 1 - kstart) / NSTAGE) & 1);
                if (tid == 0 && ok) confirmed = k + 2;
                cq3 = ld2(slot(SP1, 0) + p.o);
            }
            if (k <= ns - 2) {
                const PairNb nb = gather(slot(SM1, 0), slot(S, 0), slot(SP1, 0), slot(S, 1),
                                         slot(SP1, 1), slot(S, 2), slot(SP1, 2), slot(SM1, 3),
                                         slot(S, 3), slot(SP1, 3), p.o, cq2, cq1, cq3);
                const PairSums qs = pair_sums(nb);
                if (kin) {
                    ru = face_x<AP, BORDER>(nb, qs, p.g, a.use_div);
                    rv = face_y<AP, BORDER>(nb, qs, p.g, d, a.Vadv, p.j, k, a.pass, a.use_div);
                } else {
                    ru = rv = bc(0.f);
                }
                rw = face_z<AP, BORDER>(nb, qs, p.g, k == 0, k == ns - 2, a.use_div);
                c2 = nb.c_2;
                cL = nb.c_m1;
                cU = nb.cU;
                cD = nb.cD;
            } else {  // the top shell plane: no faces
                ru = rv = rw = cU = cD = bc(0.f);
                c2 = cL = 0.f;
            }
            fxI = flux(ru.x, cq2.x, cq2.y);
            fxH = flux(ru.y, cq2.y, c2);
            fyH = flux2(rv, cq2, cU);
            fzH = flux2(rw, cq2, cq3);
            st2(sFX + p.w, make_float2(fxI, fxH));
            st2(sFY + p.w, fyH);
        }
        __syncthreads();

        // ---- ratios of plane k ----
        {
            float2 bu = bc(1.f), bd = bc(1.f);
            if (kin) {
                const float fxL = sFX[p.w - 1];
                const float2 fyL = ld2(sFY + p.w - WX);
                const float2 fzL = fz_prev;  // raw z face k-1/2
                // in: positive low-face and negative high-face fluxes; out: the rest
                // (max(f,0) - f = max(-f,0)).  x lane-wise: A's faces are L|A and
                // A|B, B's are A|B and B|x+2.
                const float pL = fmaxf(fxL, 0.f), pI = fmaxf(fxI, 0.f), pH = fmaxf(fxH, 0.f);
                const float2 finx = make_float2(pL + (pI - fxI), pI + (pH - fxH));
                const float2 foutx = make_float2((pL - fxL) + pI, (pI - fxI) + pH);
                const float2 z0v = bc(0.f);
                const float2 py = max2(fyL, z0v), pz = max2(fzL, z0v);
                const float2 hy = max2(fyH, z0v), hz = max2(fzH, z0v);

                // bounds over the cell and its face neighbours (z only in 3D): max /
                // min of c and c^n over the seven cells, every value from the staged
                // planes or registers (the pair's own two cells are shared by both
                // lanes), with three-input min / max
                const float* cnS = slot(S, 4);
                const float2 cn0 = ld2(cnS + p.o), cnD = ld2(cnS + p.o - Y), cnU = ld2(cnS + p.o + Y);
                const float cnL = cnS[p.o - 1], cnR = cnS[p.o + 2];
                const float mAB = max3f(cq2.x, cq2.y, fmaxf(cn0.x, cn0.y));
                const float nAB = min3f(cq2.x, cq2.y, fminf(cn0.x, cn0.y));
                float2 mx = make_float2(max3f(max3f(mAB, cL, cnL), max3f(cD.x, cnD.x, cU.x), cnU.x),
                                        max3f(max3f(mAB, c2, cnR), max3f(cD.y, cnD.y, cU.y), cnU.y));
                float2 mn = make_float2(min3f(min3f(nAB, cL, cnL), min3f(cD.x, cnD.x, cU.x), cnU.x),
                                        min3f(min3f(nAB, c2, cnR), min3f(cD.y, cnD.y, cU.y), cnU.y));
                if (ns > 3) {
                    const float2 cnm = ld2(slot(SM1, 4) + p.o), cnp = ld2(slot(SP1, 4) + p.o);
                    mx = make_float2(max3f(mx.x, max3f(cq1.x, cnm.x, cq3.x), cnp.x),
                                     max3f(mx.y, max3f(cq1.y, cnm.y, cq3.y), cnp.y));
                    mn = make_float2(min3f(mn.x, min3f(cq1.x, cnm.x, cq3.x), cnp.x),
                                     min3f(mn.y, min3f(cq1.y, cnm.y, cq3.y), cnp.y));
                }
                const float2 fin = finx + ((py + pz) + ((hy - fyH) + (hz - fzH)));
                const float2 fout = foutx + (((py - fyL) + (pz - fzL)) + (hy + hz));
                const float2 eps = bc(FLT_MIN);
                // The precision form shrinks every ratio by 2^-20 before the clamp:
                // the rounding of the ratio (<= 2 ulp with rcp.approx), of the
                // limited fluxes and of their sums then never lets a cell's
                // limited out-fluxes exceed its margin above its lower bound, so a
                // field with zeros stays non-negative.
                if constexpr (WIDE) {
                    const float2 rup = rat2<AP>(mx - cq2, fin + eps) * bc(1.f - 0x1p-20f);
                    const float2 rdn = rat2<AP>(cq2 - mn, fout + eps) * bc(1.f - 0x1p-20f);
                    bu = min2(rup, bc(1.f));
                    bd = min2(rdn, bc(1.f));
                } else {
                    bu = rat2_min1<AP>(mx - cq2, fin + eps);
                    bd = rat2_min1<AP>(cq2 - mn, fout + eps);
                }
                if constexpr (WIDE) {
                    // A non-zero sum near zero (below 2^-100, where FLT_MIN and
                    // subnormal flux parts stop being negligible) is formed again in
                    // FP64 from its exact non-negative parts and its ratio divided in
                    // FP64.  A zero sum needs nothing: no flux of that direction is
                    // limited by it.  Such sums are rare, so the branch costs nothing
                    // where the field stays away from zero.
                    constexpr float kNearZero = 0x1p-100f;
                    auto near0 = [&](float v) { return v > 0.f && v < kNearZero; };
                    if (near0(fin.x) || near0(fin.y) || near0(fout.x) || near0(fout.y)) {
                        const double finA = (((double)pL + (double)(pI - fxI)) +
                                             ((double)py.x + (double)pz.x)) +
                                            ((double)(hy.x - fyH.x) + (double)(hz.x - fzH.x));
                        const double finB = (((double)pI + (double)(pH - fxH)) +
                                             ((double)py.y + (double)pz.y)) +
                                            ((double)(hy.y - fyH.y) + (double)(hz.y - fzH.y));
                        const double foutA = (((double)(pL - fxL) + (double)pI) +
                                              ((double)(py.x - fyL.x) + (double)(pz.x - fzL.x))) +
                                             ((double)hy.x + (double)hz.x);
                        const double foutB = (((double)(pI - fxI) + (double)pH) +
                                              ((double)(py.y - fyL.y) + (double)(pz.y - fzL.y))) +
                                             ((double)hy.y + (double)hz.y);
                        auto r64 = [](double n, double den) {
                            return (float)fmin(n / (den + DBL_MIN) * (1.0 - 0x1p-20), 1.0);
                        };
                        if (near0(fin.x)) bu.x = r64((double)mx.x - (double)cq2.x, finA);
                        if (near0(fin.y)) bu.y = r64((double)mx.y - (double)cq2.y, finB);
                        if (near0(fout.x)) bd.x = r64((double)cq2.x - (double)mn.x, foutA);
                        if (near0(fout.y)) bd.y = r64((double)cq2.y - (double)mn.y, foutB);
                    }
                }
                if constexpr (BORDER) {
                    bu = pick(p.g.cx, p.g.cy, bu, bc(1.f));
                    bd = pick(p.g.cx, p.g.cy, bd, bc(1.f));
                }
            }
            st2(sBU + PK * WPL + p.w, bu);
            st2(sBD + PK * WPL + p.w, bd);
        }
        __syncthreads();
        cq0 = cq1;
        cq1 = cq2;
        cq2 = cq3;
        ru_prev = ru;
        rv_prev = rv;
        rw_pp = rw_prev;
        rw_prev = rw;
        fx_prev = make_float2(fxI, fxH);
        fy_prev = fyH;
        fz_pp = fz_prev;
        fz_prev = fzH;
        qk += pp;
    };
    // The IEEE and precision forms run the plane body as a rolled loop (stage
    // slots computed per plane): their larger bodies unrolled four times miss
    // the instruction cache (measured: 11 % / 2 % faster rolled); approx_div's
    // unrolled copy, with every shared-memory address a constant offset, is
    // 2 % faster than its rolled one.
    if constexpr (!AP || WIDE) {
#pragma unroll 1
        for (int k = kstart; k <= last; k++) plane(RC{k & (NSTAGE - 1)}, k);
    } else {
        for (int kb = kstart & ~(NSTAGE - 1); kb <= last; kb += NSTAGE) {
            if (kb >= kstart) plane(IC<0>{}, kb);
            if (kb + 1 >= kstart && kb + 1 <= last) plane(IC<1>{}, kb + 1);
            if (kb + 2 >= kstart && kb + 2 <= last) plane(IC<2>{}, kb + 2);
            if (kb + 3 >= kstart && kb + 3 <= last) plane(IC<3>{}, kb + 3);
        }
    }

    if (!ok && a.err) atomicOr(a.err, 1);
    if (tid == 0) {  // never leave with a copy in flight
        for (int pl = confirmed; pl <= issue_max; pl++)
            if (!tma::mbar_wait(&bars[pl & (NSTAGE - 1)], ((pl - kstart) / NSTAGE) & 1)) break;
    }
}

template <bool LIM, bool AP, bool WIDE>
__global__ void __launch_bounds__(pair::NT, pair::NT >= 512 ? 1 : 2)
    k_pass_pair(Dims d, PassArgs<float> a, const __grid_constant__ CUtensorMap map_c,
                const __grid_constant__ CUtensorMap map_cn, const __grid_constant__ CUtensorMap map_uo,
                const __grid_constant__ CUtensorMap map_vo, const __grid_constant__ CUtensorMap map_wo)
{
    using namespace pair;
    extern __shared__ __align__(128) unsigned char smem[];
    const int i0 = LIM ? stride_x<LIM>() * (int)blockIdx.x - 2 : stride_x<LIM>() * (int)blockIdx.x;
    const int j0 = LIM ? stride_y<LIM>() * (int)blockIdx.y - 1 : stride_y<LIM>() * (int)blockIdx.y;
    // CTAs whose every face is an interior face of the interior pattern take
    // the branch-free path (no boundary forms, no existence masks, no i = 1 column).
    const bool interior = i0 >= 2 && i0 + CX - 1 <= d.nx - 3 && j0 >= 1 && j0 + CY - 1 <= d.ny - 3;
    if constexpr (LIM) {
        if (interior)
            pair_march_lim<AP, WIDE, false>(d, a, &map_c, &map_cn, &map_uo, &map_vo, &map_wo, smem,
                                            i0, j0);
        else
            pair_march_lim<AP, WIDE, true>(d, a, &map_c, &map_cn, &map_uo, &map_vo, &map_wo, smem,
                                           i0, j0);
    } else {
        if (interior)
            pair_march_plain<AP, false>(d, a, &map_c, &map_uo, &map_vo, &map_wo, smem, i0, j0);
        else
            pair_march_plain<AP, true>(d, a, &map_c, &map_uo, &map_vo, &map_wo, smem, i0, j0);
    }
}

template <bool LIM, bool AP, bool WIDE>
int launch_pair_variant(const Dims& d, const PassArgs<float>& a, cudaStream_t s)
{
    using namespace pair;
    constexpr size_t smem = smem_bytes<LIM>();
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_pass_pair<LIM, AP, WIDE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        configured = true;
    }
    const int zb = a.zbase > 0 ? a.zbase : 1, ze = a.zend > 0 ? a.zend : d.ns - 1;
    if (ze <= zb) return 0;
    const int depth = a.zdepth > 0 ? a.zdepth : ze - zb;
    dim3 g((d.nx - 2 + stride_x<LIM>() - 1) / stride_x<LIM>(),
           (d.ny - 2 + stride_y<LIM>() - 1) / stride_y<LIM>(), (ze - zb + depth - 1) / depth);
    dim3 b(TX, CY);
    const CUtensorMap& cn = LIM ? *a.maps2.cn : *a.maps2.c;
    k_pass_pair<LIM, AP, WIDE><<<g, b, smem, s>>>(d, a, *a.maps2.c, cn, *a.maps2.uo, *a.maps2.vo,
                                                  *a.maps2.wo);
    return 1;
}

int launch_pass_pair(const Dims& d, const PassArgs<float>& a, cudaStream_t s)
{
    if (a.limiter && a.wide)
        return a.approx ? launch_pair_variant<true, true, true>(d, a, s)
                        : launch_pair_variant<true, false, true>(d, a, s);
    if (a.limiter)
        return a.approx ? launch_pair_variant<true, true, false>(d, a, s)
                        : launch_pair_variant<true, false, false>(d, a, s);
    return a.approx ? launch_pair_variant<false, true, false>(d, a, s)
                    : launch_pair_variant<false, false, false>(d, a, s);
}
