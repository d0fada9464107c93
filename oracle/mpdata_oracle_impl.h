/* Precision-generic body of the CPU oracle -- TEST INFRASTRUCTURE ONLY.
 * Included by mpdata_oracle.c with R = float / double / long, SFX() adding the
 * _f32 / _f64 / _i64 suffix, TINY = the reference's MINVAL and R_ONE, R_HALF,
 * R_QUAT its ONE, HALF, QUAT (core/include/smolar_int.h:12-31), R_DIV its
 * division (C's truncating one, with a zero-divisor record, for long).
 *
 * Every expression keeps the reference's evaluation order (C's left-to-right
 * association of its macro expansions), so a strict-IEEE build reproduces
 * the strict-IEEE reference build bit for bit.  Citations are to files of
 * the reference project. */

#define AT(a, i, j, k) (a)[((size_t)(k) * (size_t)ny + (size_t)(j)) * (size_t)nx + (size_t)(i)]

static inline R SFX(mag)(R a) { return a > 0 ? a : -a; }  /* smolar_int.h:8 */

/* Advective face Courant numbers.
 * x: uu.c:126-138, y: vv.c:137-149, z: ww.c:143-155. */
void SFX(oracle_courant)(int nx, int ny, int ns, const R* dx, const R* dy, const R* ds,
                         R dt, const R* u0, const R* u1, const R* v0, const R* v1,
                         const R* w0, const R* w1, R* U, R* V, R* W)
{
    size_t n = (size_t)nx * ny * ns;
    memset(U, 0, n * sizeof(R));
    memset(V, 0, n * sizeof(R));
    memset(W, 0, n * sizeof(R));
    const R quarter_dt = R_QUAT * dt;
    for (int k = 1; k < ns - 1; k++)
        for (int j = 1; j < ny - 1; j++)
            for (int i = 0; i < nx - 1; i++) {
                R q = R_DIV(quarter_dt, dx[i]);
                AT(U, i, j, k) = q * (((AT(u0, i, j, k) + AT(u0, i + 1, j, k)) +
                                       AT(u1, i, j, k)) + AT(u1, i + 1, j, k));
            }
    for (int k = 1; k < ns - 1; k++)
        for (int j = 0; j < ny - 1; j++) {
            R q = R_DIV(quarter_dt, dy[j]);
            for (int i = 1; i < nx - 1; i++)
                AT(V, i, j, k) = q * (((AT(v0, i, j, k) + AT(v0, i, j + 1, k)) +
                                       AT(v1, i, j, k)) + AT(v1, i, j + 1, k));
        }
    for (int k = 0; k < ns - 1; k++) {
        R q = R_DIV(quarter_dt, ds[k]);
        for (int j = 1; j < ny - 1; j++)
            for (int i = 1; i < nx - 1; i++)
                AT(W, i, j, k) = q * (((AT(w0, i, j, k) + AT(w0, i, j, k + 1)) +
                                       AT(w1, i, j, k)) + AT(w1, i, j, k + 1));
    }
}

/* The antidiffusive pseudo-velocity of one face (uu.c:18-32, vv.c:21-35,
 * ww.c:20-34 share this shape):
 *   ((-DIV) + (|a|(1-|a|) (c_hi - c_lo)) / ((c_hi + c_lo) + TINY))
 *     - 1/2 a ((b1 n1) / d1 + (b2 n2) / d2)
 * neg_div is -DIV on interior faces and exactly +0 on boundary faces (the
 * reference passes the integer literal 0 there).  `one` is ONE for the x and
 * y faces (uu.c:20, vv.c:23) and the literal 1 for the z faces (ww.c:22):
 * equal except in the INTEGER build. */
static inline R SFX(face_pattern)(R neg_div, R a, R c_lo, R c_hi,
                                  R b1, R n1, R d1, R b2, R n2, R d2, R one)
{
    R ma = SFX(mag)(a);
    R t = neg_div + R_DIV((ma * (one - ma)) * (c_hi - c_lo), (c_hi + c_lo) + TINY);
    return t - R_HALF * (a * (R_DIV(b1 * n1, d1) + R_DIV(b2 * n2, d2)));
}

/* Sum-difference pair of a transverse gradient ratio:
 * n = ((p + q) - r) - s,  d = (((p + q) + r) + s) + TINY. */
#define GRAD_PAIR(p, q, r, s, n, d)                      \
    do {                                                 \
        R p_ = (p), q_ = (q), r_ = (r), s_ = (s);        \
        n = ((p_ + q_) - r_) - s_;                       \
        d = (((p_ + q_) + r_) + s_) + TINY;              \
    } while (0)

/* x-faces of one corrective pass: uu.c:34-102 (boundary faces i=0 and
 * i=nx-2 use the reduced transverse averages of the adjacent interior cell,
 * uu.c:60-70,92-97; interior faces the 4-point averages and the divergent
 * term with the reference's signs, uu.c:78-89). */
static void SFX(antidiff_x)(int nx, int ny, int ns, const R* c, const R* U,
                            const R* V, const R* W, R* Un, int use_div)
{
    for (int k = 1; k < ns - 1; k++)
        for (int j = 1; j < ny - 1; j++)
            for (int i = 0; i < nx - 1; i++) {
                R vb, wb, neg_div = 0;
                if (i == 0 || i == nx - 2) {
                    int ic = (i == 0) ? 1 : nx - 2;   /* adjacent interior cell */
                    vb = R_HALF * (AT(V, ic, j - 1, k) + AT(V, ic, j, k));
                    wb = R_HALF * (AT(W, ic, j, k - 1) + AT(W, ic, j, k));
                } else {
                    vb = R_QUAT * (((AT(V, i + 1, j - 1, k) + AT(V, i + 1, j, k)) +
                                     AT(V, i, j, k)) + AT(V, i, j - 1, k));
                    wb = R_QUAT * (((AT(W, i + 1, j, k - 1) + AT(W, i + 1, j, k)) +
                                     AT(W, i, j, k)) + AT(W, i, j, k - 1));
                    if (use_div) {
                        R s = AT(U, i + 1, j, k) - AT(U, i - 1, j, k);
                        s = s + AT(V, i + 1, j - 1, k);
                        s = s - AT(V, i + 1, j, k);
                        s = s - AT(V, i, j, k);
                        s = s + AT(V, i, j - 1, k);
                        s = s + AT(W, i + 1, j, k - 1);
                        s = s - AT(W, i + 1, j, k);
                        s = s - AT(W, i, j, k);
                        s = s + AT(W, i, j, k - 1);
                        neg_div = -((R_QUAT * AT(U, i, j, k)) * s);
                    } else {
                        neg_div = -(R)0;
                    }
                }
                R n1, d1, n2, d2;
                GRAD_PAIR(AT(c, i + 1, j + 1, k), AT(c, i, j + 1, k),
                          AT(c, i, j - 1, k), AT(c, i + 1, j - 1, k), n1, d1);
                GRAD_PAIR(AT(c, i + 1, j, k + 1), AT(c, i, j, k + 1),
                          AT(c, i, j, k - 1), AT(c, i + 1, j, k - 1), n2, d2);
                AT(Un, i, j, k) = SFX(face_pattern)(neg_div, AT(U, i, j, k),
                                                    AT(c, i, j, k), AT(c, i + 1, j, k),
                                                    vb, n1, d1, wb, n2, d2, R_ONE);
            }
}

/* y-faces: vv.c:37-107.  Interior rows run i=2..nx-2 only (vv.c:81-82); the
 * column i=1 is then whatever the swapped buffer held (see vv_col_rule).
 * The x part of the divergent term is taken one face to the left
 * (vv.c:89), exactly as coded. */
static void SFX(antidiff_y)(int nx, int ny, int ns, const R* c, const R* U,
                            const R* V, const R* W, const R* Vadv, int pass,
                            R* Vn, int use_div, int vv_fix)
{
    for (int k = 1; k < ns - 1; k++)
        for (int j = 0; j < ny - 1; j++)
            for (int i = 1; i < nx - 1; i++) {
                R ub, wb, neg_div = 0;
                if (j == 0 || j == ny - 2) {
                    int jc = (j == 0) ? 1 : ny - 2;
                    ub = R_HALF * (AT(U, i - 1, jc, k) + AT(U, i, jc, k));
                    wb = R_HALF * (AT(W, i, jc, k - 1) + AT(W, i, jc, k));
                } else {
                    if (i == 1 && !vv_fix) {
                        /* Never written by the reference: odd corrective passes
                         * see the zero-filled spare buffer, even passes the
                         * advective faces still held by the other buffer. */
                        AT(Vn, i, j, k) = (pass & 1) ? (R)0 : AT(Vadv, i, j, k);
                        continue;
                    }
                    ub = R_QUAT * (((AT(U, i - 1, j + 1, k) + AT(U, i, j + 1, k)) +
                                     AT(U, i, j, k)) + AT(U, i - 1, j, k));
                    wb = R_QUAT * (((AT(W, i, j + 1, k - 1) + AT(W, i, j + 1, k)) +
                                     AT(W, i, j, k)) + AT(W, i, j, k - 1));
                    if (use_div) {
                        R u_l2_up = (i >= 2) ? AT(U, i - 2, j + 1, k) : (R)0;
                        R u_l2 = (i >= 2) ? AT(U, i - 2, j, k) : (R)0;
                        R s = AT(V, i, j + 1, k) - AT(V, i, j - 1, k);
                        s = s + AT(W, i, j + 1, k - 1);
                        s = s - AT(W, i, j + 1, k);
                        s = s - AT(W, i, j, k);
                        s = s + AT(W, i, j, k - 1);
                        s = s + AT(U, i - 1, j + 1, k);
                        s = s - u_l2_up;
                        s = s - u_l2;
                        s = s + AT(U, i - 1, j, k);
                        neg_div = -((R_QUAT * AT(V, i, j, k)) * s);
                    } else {
                        neg_div = -(R)0;
                    }
                }
                R n1, d1, n2, d2;
                GRAD_PAIR(AT(c, i + 1, j + 1, k), AT(c, i + 1, j, k),
                          AT(c, i - 1, j, k), AT(c, i - 1, j + 1, k), n1, d1);
                GRAD_PAIR(AT(c, i, j + 1, k + 1), AT(c, i, j, k + 1),
                          AT(c, i, j, k - 1), AT(c, i, j + 1, k - 1), n2, d2);
                AT(Vn, i, j, k) = SFX(face_pattern)(neg_div, AT(V, i, j, k),
                                                    AT(c, i, j, k), AT(c, i, j + 1, k),
                                                    ub, n1, d1, wb, n2, d2, R_ONE);
            }
}

/* z-faces: ww.c:36-113 (boundary planes k=0, k=ns-2 reduced, ww.c:62-73,
 * 101-110; interior ww.c:81-99). */
static void SFX(antidiff_z)(int nx, int ny, int ns, const R* c, const R* U,
                            const R* V, const R* W, R* Wn, int use_div)
{
    for (int k = 0; k < ns - 1; k++)
        for (int j = 1; j < ny - 1; j++)
            for (int i = 1; i < nx - 1; i++) {
                R ub, vb, neg_div = 0;
                if (k == 0 || k == ns - 2) {
                    int kc = (k == 0) ? 1 : ns - 2;
                    ub = R_HALF * (AT(U, i - 1, j, kc) + AT(U, i, j, kc));
                    vb = R_HALF * (AT(V, i, j - 1, kc) + AT(V, i, j, kc));
                } else {
                    ub = R_QUAT * (((AT(U, i, j, k) + AT(U, i, j, k + 1)) +
                                     AT(U, i - 1, j, k + 1)) + AT(U, i - 1, j, k));
                    vb = R_QUAT * (((AT(V, i, j - 1, k + 1) + AT(V, i, j, k + 1)) +
                                     AT(V, i, j, k)) + AT(V, i, j - 1, k));
                    if (use_div) {
                        R s = AT(W, i, j, k + 1) - AT(W, i, j, k - 1);
                        s = s + AT(U, i - 1, j, k + 1);
                        s = s - AT(U, i, j, k + 1);
                        s = s - AT(U, i, j, k);
                        s = s + AT(U, i - 1, j, k);
                        s = s + AT(V, i, j - 1, k + 1);
                        s = s - AT(V, i, j, k + 1);
                        s = s - AT(V, i, j, k);
                        s = s + AT(V, i, j - 1, k);
                        neg_div = -((R_QUAT * AT(W, i, j, k)) * s);
                    } else {
                        neg_div = -(R)0;
                    }
                }
                R n1, d1, n2, d2;
                GRAD_PAIR(AT(c, i + 1, j, k + 1), AT(c, i + 1, j, k),
                          AT(c, i - 1, j, k), AT(c, i - 1, j, k + 1), n1, d1);
                GRAD_PAIR(AT(c, i, j + 1, k + 1), AT(c, i, j + 1, k),
                          AT(c, i, j - 1, k), AT(c, i, j - 1, k + 1), n2, d2);
                AT(Wn, i, j, k) = SFX(face_pattern)(neg_div, AT(W, i, j, k),
                                                    AT(c, i, j, k), AT(c, i, j, k + 1),
                                                    ub, n1, d1, vb, n2, d2, (R)1);
            }
}

void SFX(oracle_antidiff)(int nx, int ny, int ns, const R* c, const R* Uo, const R* Vo,
                          const R* Wo, const R* Vadv, int pass, R* Un, R* Vn, R* Wn,
                          const oracle_opts* opts)
{
    int use_div = !(opts && opts->div_mode == 1);
    int vv_fix = opts && opts->vv_fix;
    /* Jacobi update: all three read the previous pass's faces
     * (pvelocity.c:22-36). */
    SFX(antidiff_x)(nx, ny, ns, c, Uo, Vo, Wo, Un, use_div);
    SFX(antidiff_y)(nx, ny, ns, c, Uo, Vo, Wo, Vadv, pass, Vn, use_div, vv_fix);
    SFX(antidiff_z)(nx, ny, ns, c, Uo, Vo, Wo, Wn, use_div);
}

/* Upwind flux form of smolar_pass.c:104: F = L(a+|a|) + R(a-|a|). */
static inline R SFX(upwind)(R l, R r, R a)
{
    R ma = SFX(mag)(a);
    return (l * (a + ma)) + (r * (a - ma));
}

/* Donor-cell update of the interior cells: smolar_pass.c:30-57. */
void SFX(oracle_donor)(int nx, int ny, int ns, const R* c0, const R* U, const R* V,
                       const R* W, R* c1)
{
    for (int k = 1; k < ns - 1; k++)
        for (int j = 1; j < ny - 1; j++)
            for (int i = 1; i < nx - 1; i++) {
                R cc = AT(c0, i, j, k);
                R fx = SFX(upwind)(cc, AT(c0, i + 1, j, k), AT(U, i, j, k)) -
                       SFX(upwind)(AT(c0, i - 1, j, k), cc, AT(U, i - 1, j, k));
                R fy = SFX(upwind)(cc, AT(c0, i, j + 1, k), AT(V, i, j, k)) -
                       SFX(upwind)(AT(c0, i, j - 1, k), cc, AT(V, i, j - 1, k));
                R fz = SFX(upwind)(cc, AT(c0, i, j, k + 1), AT(W, i, j, k)) -
                       SFX(upwind)(AT(c0, i, j, k - 1), cc, AT(W, i, j, k - 1));
                AT(c1, i, j, k) = cc - R_HALF * ((fx + fy) + fz);
            }
}

/* Copy of the fixed one-cell boundary shell: smolar.c:5-31. */
static void SFX(shell_copy)(int nx, int ny, int ns, R* to, const R* from)
{
    for (int k = 0; k < ns; k++)
        for (int j = 0; j < ny; j++) {
            if (k == 0 || k == ns - 1 || j == 0 || j == ny - 1) {
                memcpy(&AT(to, 0, j, k), &AT(from, 0, j, k), (size_t)nx * sizeof(R));
            } else {
                AT(to, 0, j, k) = AT(from, 0, j, k);
                AT(to, nx - 1, j, k) = AT(from, nx - 1, j, k);
            }
        }
}

/* Nonoscillatory limiting of the raw antidiffusive faces (no reference
 * counterpart; Smolarkiewicz & Grabowski 1990, J. Comput. Phys. 86).
 *   bounds  : max/min of psi (= c, this pass's input) and psi^n (= cn, the
 *             step's input) over the cell and its face neighbours (the z
 *             neighbours only when ns > 3, so the 3-plane 2D form matches a
 *             native 2D grid);
 *   fluxes  : f = max(a,0) c_lo + min(a,0) c_hi on every face of the cell;
 *   beta_up = (max - psi) / (sum of incoming f + TINY),
 *   beta_dn = (psi - min) / (sum of outgoing f + TINY), for interior cells;
 *             the fixed shell cells take 1 (no constraint from that side);
 *   a_lim   = a * min(1, beta_dn(lo), beta_up(hi))  if a > 0,
 *             a * min(1, beta_up(lo), beta_dn(hi))  otherwise.
 * With wide != 0 the in/out sums and the ratios are formed in double (the
 * FP32-storage form). */
static void SFX(fct_limit)(int nx, int ny, int ns, const R* c, const R* cn, R* U, R* V,
                           R* W, int wide)
{
    size_t n = (size_t)nx * ny * ns;
    R* bup = (R*)malloc(n * sizeof(R));
    R* bdn = (R*)malloc(n * sizeof(R));
    for (size_t q = 0; q < n; q++) { bup[q] = (R)1; bdn[q] = (R)1; }
    int zact = ns > 3;
    for (int k = 1; k < ns - 1; k++)
        for (int j = 1; j < ny - 1; j++)
            for (int i = 1; i < nx - 1; i++) {
                R psi = AT(c, i, j, k);
                R mx = psi, mn = psi, t;
#define BOUND(a) do { t = (a); mx = RMAX(t, mx); mn = RMIN(t, mn); } while (0)
                BOUND(AT(cn, i, j, k));
                BOUND(AT(c, i - 1, j, k)); BOUND(AT(cn, i - 1, j, k));
                BOUND(AT(c, i + 1, j, k)); BOUND(AT(cn, i + 1, j, k));
                BOUND(AT(c, i, j - 1, k)); BOUND(AT(cn, i, j - 1, k));
                BOUND(AT(c, i, j + 1, k)); BOUND(AT(cn, i, j + 1, k));
                if (zact) {
                    BOUND(AT(c, i, j, k - 1)); BOUND(AT(cn, i, j, k - 1));
                    BOUND(AT(c, i, j, k + 1)); BOUND(AT(cn, i, j, k + 1));
                }
#undef BOUND
                /* Face fluxes, low side then high side of the cell per axis. */
                R ax[6] = {AT(U, i - 1, j, k), AT(U, i, j, k), AT(V, i, j - 1, k),
                           AT(V, i, j, k), AT(W, i, j, k - 1), AT(W, i, j, k)};
                R lo[6] = {AT(c, i - 1, j, k), psi, AT(c, i, j - 1, k), psi,
                           AT(c, i, j, k - 1), psi};
                R hi[6] = {psi, AT(c, i + 1, j, k), psi, AT(c, i, j + 1, k), psi,
                           AT(c, i, j, k + 1)};
                if (wide) {
                    double fin = 0, fout = 0;
                    for (int f = 0; f < 6; f++) {
                        double a = ax[f];
                        double fl = a > 0 ? a * (double)lo[f] : a * (double)hi[f];
                        if (f & 1) { /* high face: positive flux leaves */
                            if (fl > 0) fout += fl; else fin -= fl;
                        } else {     /* low face: positive flux enters */
                            if (fl > 0) fin += fl; else fout -= fl;
                        }
                    }
                    AT(bup, i, j, k) = (R)(((double)mx - (double)psi) / (fin + DBL_MIN));
                    AT(bdn, i, j, k) = (R)(((double)psi - (double)mn) / (fout + DBL_MIN));
                } else {
                    R fin = 0, fout = 0;
                    for (int f = 0; f < 6; f++) {
                        R a = ax[f];
                        R fl = a > 0 ? a * lo[f] : a * hi[f];
                        if (f & 1) {
                            if (fl > 0) fout += fl; else fin -= fl;
                        } else {
                            if (fl > 0) fin += fl; else fout -= fl;
                        }
                    }
                    AT(bup, i, j, k) = (mx - psi) / (fin + TINY);
                    AT(bdn, i, j, k) = (psi - mn) / (fout + TINY);
                }
            }
#define LIMIT(face, lo_q, hi_q)                                                  \
    do {                                                                         \
        R a = (face);                                                            \
        R g;                                                                     \
        if (a > 0) { g = bdn[lo_q] < bup[hi_q] ? bdn[lo_q] : bup[hi_q]; }        \
        else       { g = bup[lo_q] < bdn[hi_q] ? bup[lo_q] : bdn[hi_q]; }        \
        g = g < (R)1 ? g : (R)1;                                                 \
        (face) = a * g;                                                          \
    } while (0)
#define Q(i, j, k) (((size_t)(k) * (size_t)ny + (size_t)(j)) * (size_t)nx + (size_t)(i))
    for (int k = 1; k < ns - 1; k++)
        for (int j = 1; j < ny - 1; j++)
            for (int i = 0; i < nx - 1; i++) LIMIT(AT(U, i, j, k), Q(i, j, k), Q(i + 1, j, k));
    for (int k = 1; k < ns - 1; k++)
        for (int j = 0; j < ny - 1; j++)
            for (int i = 1; i < nx - 1; i++) LIMIT(AT(V, i, j, k), Q(i, j, k), Q(i, j + 1, k));
    for (int k = 0; k < ns - 1; k++)
        for (int j = 1; j < ny - 1; j++)
            for (int i = 1; i < nx - 1; i++) LIMIT(AT(W, i, j, k), Q(i, j, k), Q(i, j, k + 1));
#undef Q
#undef LIMIT
    free(bup);
    free(bdn);
}

/* The pass loop of smolar.c:44-58 on caller-owned buffers.
 * cold/cnew alternate exactly as in the reference; on return *pold holds the
 * newest level and *pnew the one before it. */
static int SFX(pass_loop)(int nx, int ny, int ns, const R* Uadv, const R* Vadv,
                          const R* Wadv, R** pold, R** pnew, int order,
                          const oracle_opts* opts)
{
    size_t n = (size_t)nx * ny * ns;
    int lim = opts && opts->limiter;
    int wide = opts && opts->wide_beta;
    R* Uc = (R*)malloc(n * sizeof(R)); R* Vc = (R*)malloc(n * sizeof(R));
    R* Wc = (R*)malloc(n * sizeof(R)); R* Un = (R*)calloc(n, sizeof(R));
    R* Vn = (R*)calloc(n, sizeof(R)); R* Wn = (R*)calloc(n, sizeof(R));
    R* cn = NULL;
    if (!Uc || !Vc || !Wc || !Un || !Vn || !Wn) return -1;
    memcpy(Uc, Uadv, n * sizeof(R));
    memcpy(Vc, Vadv, n * sizeof(R));
    memcpy(Wc, Wadv, n * sizeof(R));
    if (lim) {
        cn = (R*)malloc(n * sizeof(R));
        memcpy(cn, *pold, n * sizeof(R));
    }
    R* cold = *pold;
    R* cnew = *pnew;
    for (int o = 0; o < order; o++) {
        if (o) {
            SFX(oracle_antidiff)(nx, ny, ns, cold, Uc, Vc, Wc, Vadv, o, Un, Vn, Wn, opts);
            if (lim) SFX(fct_limit)(nx, ny, ns, cold, cn, Un, Vn, Wn, wide);
            R* s;
            s = Uc; Uc = Un; Un = s;
            s = Vc; Vc = Vn; Vn = s;
            s = Wc; Wc = Wn; Wn = s;
        }
        SFX(shell_copy)(nx, ny, ns, cnew, cold);
        SFX(oracle_donor)(nx, ny, ns, cold, Uc, Vc, Wc, cnew);
        R* s = cnew; cnew = cold; cold = s;
    }
    *pold = cold;
    *pnew = cnew;
    free(Uc); free(Vc); free(Wc); free(Un); free(Vn); free(Wn); free(cn);
    return 0;
}

int SFX(oracle_step_faces)(int nx, int ny, int ns, const R* U, const R* V, const R* W,
                           const R* c0, R* c1, R* inter, int order,
                           const oracle_opts* opts)
{
    if (nx < 3 || ny < 3 || ns < 3 || order < 1) return -1;
    size_t n = (size_t)nx * ny * ns;
    R* a = (R*)malloc(n * sizeof(R));
    R* b = (R*)calloc(n, sizeof(R));
    if (!a || !b) return -1;
    memcpy(a, c0, n * sizeof(R));
    R* pold = a;
    R* pnew = b;
    int rc = SFX(pass_loop)(nx, ny, ns, U, V, W, &pold, &pnew, order, opts);
    memcpy(c1, pold, n * sizeof(R));
    if (inter) memcpy(inter, pnew, n * sizeof(R));
    free(a);
    free(b);
    return rc;
}

/* smolar(): smolar.c:33-63, including the returned pointer order. */
int SFX(oracle_smolar)(int nx, int ny, int ns, R* dx, R* dy, R* ds, const R dt, R* u0,
                       R* u1, R* v0, R* v1, R* w0, R* w1, R** c0, R** c1, int flow_type,
                       int order, const oracle_opts* opts)
{
    (void)flow_type; /* stored but never read by the reference (uu.c:111) */
    if (nx < 3 || ny < 3 || ns < 3 || order < 0) return -1;
    if (R_IS_INTEGER && opts && opts->limiter) return -1; /* no limiter in the integer mode */
    R* cold = *c0;
    R* cnew = *c1;
    if (order > 0) {
        size_t n = (size_t)nx * ny * ns;
        R* U = (R*)malloc(n * sizeof(R));
        R* V = (R*)malloc(n * sizeof(R));
        R* W = (R*)malloc(n * sizeof(R));
        if (!U || !V || !W) return -1;
        R_DIV_RESET();
        SFX(oracle_courant)(nx, ny, ns, dx, dy, ds, dt, u0, u1, v0, v1, w0, w1, U, V, W);
        int rc = SFX(pass_loop)(nx, ny, ns, U, V, W, &cold, &cnew, order, opts);
        free(U); free(V); free(W);
        if (rc) return rc;
        if (R_DIV_FAILED()) return -2; /* a zero divisor: the reference traps there */
    }
    *c1 = cold;
    *c0 = cnew;
    return 0;
}

double SFX(oracle_mass)(int nx, int ny, int ns, const R* c)
{
    double s = 0, comp = 0;
    for (int k = 1; k < ns - 1; k++)
        for (int j = 1; j < ny - 1; j++)
            for (int i = 1; i < nx - 1; i++) {
                double x = AT(c, i, j, k);
                double t = s + x;
                if (fabs(s) >= fabs(x)) comp += (s - t) + x;
                else comp += (x - t) + s;
                s = t;
            }
    return s + comp;
}

#undef AT
#undef GRAD_PAIR
