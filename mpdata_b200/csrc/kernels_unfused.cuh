// One kernel per reference routine, one thread per grid point.
//
// This is the cross-check path (mpdata_options.kernel = 1): simple enough to
// read against the reference line by line, it runs every formula exactly as
// the fused kernels do but through global memory, one routine at a time.
// Included by kernels_fast.cu / kernels_strict.cu inside namespace
// mpd::MPD_NS, and by smolar_i64.cu (the reference's INTEGER build: the
// same kernels on long long, constants from RealConst, truncating division).

// Advective face Courant numbers (uu.c:126-138, vv.c:137-149, ww.c:143-155):
//   U(i+1/2) = ((dt/4)/dx[i]) (((u0_i + u0_{i+1}) + u1_i) + u1_{i+1})
// Unused face entries are written as 0.
template <typename T>
__global__ void k_courant(Dims d, const T* __restrict__ dx, const T* __restrict__ dy,
                          const T* __restrict__ ds, T dt, const T* __restrict__ u0,
                          const T* __restrict__ u1, const T* __restrict__ v0,
                          const T* __restrict__ v1, const T* __restrict__ w0,
                          const T* __restrict__ w1, T* __restrict__ U, T* __restrict__ V,
                          T* __restrict__ W, int k0)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    int k = k0 + (int)blockIdx.z;
    if (i >= d.nx || j >= d.ny) return;
    long long q = cell(d, i, j, k);
    const T quarter_dt = RealConst<T>::quat * dt;
    bool kin = k >= 1 && k <= d.ns - 2, jin = j >= 1 && j <= d.ny - 2, iin = i >= 1 && i <= d.nx - 2;
    T uf = T(0), vf = T(0), wf = T(0);
    if (kin && jin && i <= d.nx - 2)
        uf = ratio<false>(quarter_dt, dx[i]) * (((u0[q] + u0[q + 1]) + u1[q]) + u1[q + 1]);
    if (kin && iin && j <= d.ny - 2)
        vf = ratio<false>(quarter_dt, dy[j]) * (((v0[q] + v0[q + d.px]) + v1[q]) + v1[q + d.px]);
    if (jin && iin && k <= d.ns - 2)
        wf = ratio<false>(quarter_dt, ds[k]) * (((w0[q] + w0[q + d.pp]) + w1[q]) + w1[q + d.pp]);
    U[q] = uf;
    V[q] = vf;
    W[q] = wf;
}

// Antidiffusive faces of one corrective pass, Jacobi style (pvelocity.c:22-36):
// every new face reads the previous pass's faces Uo/Vo/Wo and the pass input c.
//   x faces: uu.c:34-102, y faces: vv.c:37-107, z faces: ww.c:36-113.
// Vadv holds the advective y faces, for the column i=1 that vv_pass leaves
// unwritten (vv.c:81-82): it reads 0 on odd passes and Vadv on even ones
// unless vv_fix is set.
template <typename T>
__global__ void k_antidiff(Dims d, const T* __restrict__ c, const T* __restrict__ Uo,
                           const T* __restrict__ Vo, const T* __restrict__ Wo,
                           const T* __restrict__ Vadv, T* __restrict__ Un, T* __restrict__ Vn,
                           T* __restrict__ Wn, int pass, int use_div, int vv_fix)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    int k = blockIdx.z;
    if (i >= d.nx || j >= d.ny) return;
    const long long X = 1, Y = d.px, Z = d.pp;
    const long long q = cell(d, i, j, k);
    const int nx = d.nx, ny = d.ny, ns = d.ns;
    const bool kin = k >= 1 && k <= ns - 2, jin = j >= 1 && j <= ny - 2, iin = i >= 1 && i <= nx - 2;

    // ---- x face between i and i+1 ----
    if (kin && jin && i <= nx - 2) {
        T vb, wb, neg_div = T(0);
        if (i == 0 || i == nx - 2) {
            long long a = (i == 0) ? q + X : q;  // adjacent interior cell
            vb = RealConst<T>::half * (Vo[a - Y] + Vo[a]);
            wb = RealConst<T>::half * (Wo[a - Z] + Wo[a]);
        } else {
            vb = RealConst<T>::quat * (((Vo[q + X - Y] + Vo[q + X]) + Vo[q]) + Vo[q - Y]);
            wb = RealConst<T>::quat * (((Wo[q + X - Z] + Wo[q + X]) + Wo[q]) + Wo[q - Z]);
            if (use_div) {
                T s = Uo[q + X] - Uo[q - X];
                s = s + Vo[q + X - Y];
                s = s - Vo[q + X];
                s = s - Vo[q];
                s = s + Vo[q - Y];
                s = s + Wo[q + X - Z];
                s = s - Wo[q + X];
                s = s - Wo[q];
                s = s + Wo[q - Z];
                neg_div = -((RealConst<T>::quat * Uo[q]) * s);
            } else {
                neg_div = -T(0);
            }
        }
        T n1, d1, n2, d2;
        grad_pair(c[q + X + Y], c[q + Y], c[q - Y], c[q + X - Y], n1, d1);
        grad_pair(c[q + X + Z], c[q + Z], c[q - Z], c[q + X - Z], n2, d2);
        Un[q] = face_pattern(neg_div, Uo[q], c[q], c[q + X], vb, n1, d1, wb, n2, d2);
    }

    // ---- y face between j and j+1 ----
    if (kin && iin && j <= ny - 2) {
        T ub, wb, neg_div = T(0);
        bool done = false;
        if (j == 0 || j == ny - 2) {
            long long a = (j == 0) ? q + Y : q;
            ub = RealConst<T>::half * (Uo[a - X] + Uo[a]);
            wb = RealConst<T>::half * (Wo[a - Z] + Wo[a]);
        } else if (i == 1 && !vv_fix) {
            Vn[q] = (pass & 1) ? T(0) : Vadv[q];
            done = true;
        } else {
            ub = RealConst<T>::quat * (((Uo[q - X + Y] + Uo[q + Y]) + Uo[q]) + Uo[q - X]);
            wb = RealConst<T>::quat * (((Wo[q + Y - Z] + Wo[q + Y]) + Wo[q]) + Wo[q - Z]);
            if (use_div) {
                T ul2u = (i >= 2) ? Uo[q - 2 * X + Y] : T(0);
                T ul2 = (i >= 2) ? Uo[q - 2 * X] : T(0);
                T s = Vo[q + Y] - Vo[q - Y];
                s = s + Wo[q + Y - Z];
                s = s - Wo[q + Y];
                s = s - Wo[q];
                s = s + Wo[q - Z];
                s = s + Uo[q - X + Y];
                s = s - ul2u;
                s = s - ul2;
                s = s + Uo[q - X];
                neg_div = -((RealConst<T>::quat * Vo[q]) * s);
            } else {
                neg_div = -T(0);
            }
        }
        if (!done) {
            T n1, d1, n2, d2;
            grad_pair(c[q + X + Y], c[q + X], c[q - X], c[q - X + Y], n1, d1);
            grad_pair(c[q + Y + Z], c[q + Z], c[q - Z], c[q + Y - Z], n2, d2);
            Vn[q] = face_pattern(neg_div, Vo[q], c[q], c[q + Y], ub, n1, d1, wb, n2, d2);
        }
    }

    // ---- z face between k and k+1 ----
    if (jin && iin && k <= ns - 2) {
        T ub, vb, neg_div = T(0);
        if (k == 0 || k == ns - 2) {
            long long a = (k == 0) ? q + Z : q;
            ub = RealConst<T>::half * (Uo[a - X] + Uo[a]);
            vb = RealConst<T>::half * (Vo[a - Y] + Vo[a]);
        } else {
            ub = RealConst<T>::quat * (((Uo[q] + Uo[q + Z]) + Uo[q - X + Z]) + Uo[q - X]);
            vb = RealConst<T>::quat * (((Vo[q - Y + Z] + Vo[q + Z]) + Vo[q]) + Vo[q - Y]);
            if (use_div) {
                T s = Wo[q + Z] - Wo[q - Z];
                s = s + Uo[q - X + Z];
                s = s - Uo[q + Z];
                s = s - Uo[q];
                s = s + Uo[q - X];
                s = s + Vo[q - Y + Z];
                s = s - Vo[q + Z];
                s = s - Vo[q];
                s = s + Vo[q - Y];
                neg_div = -((RealConst<T>::quat * Wo[q]) * s);
            } else {
                neg_div = -T(0);
            }
        }
        T n1, d1, n2, d2;
        grad_pair(c[q + X + Z], c[q + X], c[q - X], c[q - X + Z], n1, d1);
        grad_pair(c[q + Y + Z], c[q + Y], c[q - Y], c[q - Y + Z], n2, d2);
        Wn[q] = face_pattern<T, false, true>(neg_div, Wo[q], c[q], c[q + Z], ub, n1, d1, vb, n2,
                                             d2);
    }
}

// Limiter ratios of every interior cell (no reference counterpart;
// Smolarkiewicz & Grabowski 1990): bounds from c (this pass's input) and
// cn (the step's input) over the cell and its face neighbours (z neighbours
// only when ns > 3), in/out sums of the donor fluxes through the six faces.
// A = accumulation type (double for the FP32-storage form).
template <typename T, typename A>
__global__ void k_fct_beta(Dims d, const T* __restrict__ c, const T* __restrict__ cn,
                           const T* __restrict__ U, const T* __restrict__ V,
                           const T* __restrict__ W, T* __restrict__ bup, T* __restrict__ bdn)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    int k = blockIdx.z;
    if (i < 1 || j < 1 || k < 1 || i > d.nx - 2 || j > d.ny - 2 || k > d.ns - 2) return;
    const long long X = 1, Y = d.px, Z = d.pp;
    const long long q = cell(d, i, j, k);
    T psi = c[q];
    T mx = psi, mn = psi, t;
#define MPD_BOUND(v) do { t = (v); mx = vmax(t, mx); mn = vmin(t, mn); } while (0)
    MPD_BOUND(cn[q]);
    MPD_BOUND(c[q - X]); MPD_BOUND(cn[q - X]);
    MPD_BOUND(c[q + X]); MPD_BOUND(cn[q + X]);
    MPD_BOUND(c[q - Y]); MPD_BOUND(cn[q - Y]);
    MPD_BOUND(c[q + Y]); MPD_BOUND(cn[q + Y]);
    if (d.ns > 3) {
        MPD_BOUND(c[q - Z]); MPD_BOUND(cn[q - Z]);
        MPD_BOUND(c[q + Z]); MPD_BOUND(cn[q + Z]);
    }
#undef MPD_BOUND
    A fin = A(0), fout = A(0);
    lim_acc(lim_flux<T, A>(U[q - X], c[q - X], psi), false, fin, fout);
    lim_acc(lim_flux<T, A>(U[q], psi, c[q + X]), true, fin, fout);
    lim_acc(lim_flux<T, A>(V[q - Y], c[q - Y], psi), false, fin, fout);
    lim_acc(lim_flux<T, A>(V[q], psi, c[q + Y]), true, fin, fout);
    lim_acc(lim_flux<T, A>(W[q - Z], c[q - Z], psi), false, fin, fout);
    lim_acc(lim_flux<T, A>(W[q], psi, c[q + Z]), true, fin, fout);
    bup[q] = T((A(mx) - A(psi)) / (fin + lim_tiny<A>()));
    bdn[q] = T((A(psi) - A(mn)) / (fout + lim_tiny<A>()));
}

// Apply the limiter to every used face (raw faces Ui/Vi/Wi -> limited
// U/V/W; in place when they alias); shell cells count as beta = 1.
template <typename T>
__global__ void k_fct_apply(Dims d, const T* __restrict__ bup, const T* __restrict__ bdn,
                            const T* Ui, const T* Vi, const T* Wi, T* U, T* V, T* W)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    int k = blockIdx.z;
    if (i >= d.nx || j >= d.ny) return;
    const long long X = 1, Y = d.px, Z = d.pp;
    const long long q = cell(d, i, j, k);
    const int nx = d.nx, ny = d.ny, ns = d.ns;
    auto in = [&](int a, int b, int c_) {
        return a >= 1 && a <= nx - 2 && b >= 1 && b <= ny - 2 && c_ >= 1 && c_ <= ns - 2;
    };
    auto up = [&](long long p, bool interior) { return interior ? bup[p] : T(1); };
    auto dn = [&](long long p, bool interior) { return interior ? bdn[p] : T(1); };
    const bool kin = k >= 1 && k <= ns - 2, jin = j >= 1 && j <= ny - 2, iin = i >= 1 && i <= nx - 2;
    if (kin && jin && i <= nx - 2) {
        bool lo = in(i, j, k), hi = in(i + 1, j, k);
        U[q] = limit_face(Ui[q], up(q, lo), dn(q, lo), up(q + X, hi), dn(q + X, hi));
    }
    if (kin && iin && j <= ny - 2) {
        bool lo = in(i, j, k), hi = in(i, j + 1, k);
        V[q] = limit_face(Vi[q], up(q, lo), dn(q, lo), up(q + Y, hi), dn(q + Y, hi));
    }
    if (jin && iin && k <= ns - 2) {
        bool lo = in(i, j, k), hi = in(i, j, k + 1);
        W[q] = limit_face(Wi[q], up(q, lo), dn(q, lo), up(q + Z, hi), dn(q + Z, hi));
    }
}

// Donor-cell pass (smolar_pass.c:30-57) over the interior; with copy_shell
// the fixed boundary shell is copied from c0 as bndcpy does (smolar.c:5-31).
template <typename T>
__global__ void k_donor(Dims d, const T* __restrict__ c0, const T* __restrict__ U,
                        const T* __restrict__ V, const T* __restrict__ W, T* __restrict__ c1,
                        int copy_shell)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    int k = blockIdx.z;
    if (i >= d.nx || j >= d.ny) return;
    const long long X = 1, Y = d.px, Z = d.pp;
    const long long q = cell(d, i, j, k);
    if (i >= 1 && j >= 1 && k >= 1 && i <= d.nx - 2 && j <= d.ny - 2 && k <= d.ns - 2) {
        c1[q] = donor_update(c0[q], c0[q - X], c0[q + X], c0[q - Y], c0[q + Y], c0[q - Z],
                             c0[q + Z], U[q], U[q - X], V[q], V[q - Y], W[q], W[q - Z]);
    } else if (copy_shell) {
        c1[q] = c0[q];
    }
}

// 16 bytes of consecutive elements (4 floats / 2 doubles), moved as one vector.
template <typename T> struct Vec16 {
    static constexpr int N = 16 / (int)sizeof(T);
    T v[N];
};
template <typename T> __device__ __forceinline__ Vec16<T> ld16(const T* p)
{
    Vec16<T> r;
    *reinterpret_cast<uint4*>(r.v) = __ldg(reinterpret_cast<const uint4*>(p));
    return r;
}
template <typename T> __device__ __forceinline__ void st16(T* p, const Vec16<T>& r)
{
    *reinterpret_cast<uint4*>(p) = *reinterpret_cast<const uint4*>(r.v);
}

// The same donor-cell pass, z-marching: each thread owns 16 bytes of a row
// (4 FP32 / 2 FP64 cells) and steps them through a chunk of `depth` planes,
// keeping the own column's c and z faces of neighbouring planes in
// registers; rows and faces move as 16-byte vectors (row pitch and pitch
// offsets are multiples of 16 bytes).  Shell cells of a vector keep their c0
// value (bndcpy's copy, smolar.c:5-31, is the same value in every level);
// shell rows and planes are not touched.  Same donor_update expression as
// k_donor, so both give the same bits.
template <typename T>
__global__ void __launch_bounds__(256) k_donor_v(Dims d, const T* __restrict__ c0,
                                                 const T* __restrict__ U, const T* __restrict__ V,
                                                 const T* __restrict__ W, T* __restrict__ c1,
                                                 int depth, int zb, int ze)
{
    constexpr int N = Vec16<T>::N;
    const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * N;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i0 >= d.px || j > d.ny - 2) return;
    const int k0 = zb + (int)blockIdx.z * depth, k1 = min(ze, k0 + depth);
    const long long Y = d.px, Z = d.pp;
    long long q = cell(d, i0, j, k0);
    Vec16<T> cm = ld16(c0 + q - Z), cc = ld16(c0 + q), wm = ld16(W + q - Z);
    for (int k = k0; k < k1; k++, q += Z) {
        const Vec16<T> cp = ld16(c0 + q + Z), cd = ld16(c0 + q - Y), cu = ld16(c0 + q + Y);
        const Vec16<T> u = ld16(U + q), v = ld16(V + q), vd = ld16(V + q - Y), w = ld16(W + q);
        // x neighbours across the vector's edges (the previous / next row element
        // at the row ends: in bounds, only used by shell cells, whose result is dropped)
        const T cl = __ldg(c0 + q - 1), cr = __ldg(c0 + q + N), ul = __ldg(U + q - 1);
        Vec16<T> out;
#pragma unroll
        for (int e = 0; e < N; e++) {
            const int i = i0 + e;
            const T left = e == 0 ? cl : cc.v[e > 0 ? e - 1 : 0];
            const T right = e == N - 1 ? cr : cc.v[e < N - 1 ? e + 1 : 0];
            const T uleft = e == 0 ? ul : u.v[e > 0 ? e - 1 : 0];
            out.v[e] = (i >= 1 && i <= d.nx - 2)
                           ? donor_update(cc.v[e], left, right, cd.v[e], cu.v[e], cm.v[e], cp.v[e],
                                          u.v[e], uleft, v.v[e], vd.v[e], w.v[e], wm.v[e])
                           : cc.v[e];
        }
        st16(c1 + q, out);
        cm = cc;
        cc = cp;
        wm = w;
    }
}

// Pass 0 fused with the advective faces (R5 + R4, the per-call work of
// smolar(): uu.c:126-138, vv.c:137-149, ww.c:143-155 then
// smolar_pass.c:30-57).  The k_donor_v march, but the faces each cell needs
// are formed from the cell velocities in registers and also stored for the
// corrective passes.  Each face value is rounded on its own (explicit
// multiply, nothing contracts it into the donor update), so faces and field
// are the same bits as k_courant followed by k_donor_v.  Stores: U for
// i <= nx-2, V and W for interior i (0 in the other lanes of a vector, as
// k_courant writes), on interior rows of planes [zb, ze); the boundary faces
// V(j = 0) by the j = 1 threads and W(k = 0) by a chunk starting at plane 1.
// Face entries no pass reads (shell rows and planes) are left untouched.
// ONE_LEVEL: u1, v1, w1 are u0, v0, w0 (drivers pass one array for both time
// levels, reference tests/ring2d/test.c:89-91); each is loaded once and the
// sums take the same operands in the same order, so the bits are the same.
// Both float marches are held to 80 registers, three CTAs per SM.  The
// two-level one spills 48 bytes there and still runs 7 % faster than at 128
// registers and two CTAs (B200, 512 x 512 x 256: 0.483 vs 0.519 ms).
template <typename T> __device__ __forceinline__ T mul_rn(T a, T b);
template <> __device__ __forceinline__ float mul_rn<float>(float a, float b) { return __fmul_rn(a, b); }
template <> __device__ __forceinline__ double mul_rn<double>(double a, double b) { return __dmul_rn(a, b); }

// The advective faces alone (R5: uu.c:126-138, vv.c:137-149, ww.c:143-155)
// of planes [k0, k1), every entry of those planes written as k_courant
// writes it (0 where a face does not exist; columns i >= nx untouched), as a
// z march over 16-byte vectors: QUAT dt / dx[i] and QUAT dt / dy[j] are formed
// once per thread, QUAT dt / ds[k] once per plane, and the upper z plane of
// w is carried to the next plane, so each velocity element is read once
// (ONE_LEVEL: u1, v1, w1 are u0, v0, w0, loaded once).  The operands and
// their order are k_courant's: the same bits.
template <typename T, bool ONE_LEVEL>
__global__ void __launch_bounds__(256) k_courant_v(
    Dims d, const T* __restrict__ dx, const T* __restrict__ dy, const T* __restrict__ ds, T dt,
    const T* __restrict__ u0, const T* __restrict__ u1, const T* __restrict__ v0,
    const T* __restrict__ v1, const T* __restrict__ w0, const T* __restrict__ w1,
    T* __restrict__ U, T* __restrict__ V, T* __restrict__ W, int depth, int k0, int k1)
{
    constexpr int N = Vec16<T>::N;
    const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * N;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i0 >= d.nx || j >= d.ny) return;
    const int kb = k0 + (int)blockIdx.z * depth, ke = min(k1, kb + depth);
    const int nx = d.nx, ny = d.ny, ns = d.ns;
    const long long Y = d.px, Z = d.pp;
    const T qdt = RealConst<T>::quat * dt;
    const bool jin = j >= 1 && j <= ny - 2, jv = j <= ny - 2;
    T rx[N];
#pragma unroll
    for (int e = 0; e < N; e++) rx[e] = (i0 + e <= nx - 2) ? ratio<false>(qdt, dx[i0 + e]) : T(0);
    const T ry = jv ? ratio<false>(qdt, dy[j]) : T(0);
    // the last lane's x face reads the first velocity of the next vector
    const bool need_r = i0 + N - 1 <= nx - 2;
    const bool full = i0 + N <= nx;  // every lane is a cell of the row
    auto iin = [&](int e) { return i0 + e >= 1 && i0 + e <= nx - 2; };
    long long q = cell(d, i0, j, kb);
    Vec16<T> wc0{}, wc1{};  // w of plane k (both time levels), carried
    if (jin && kb < ke && kb <= ns - 2) {
        wc0 = ld16(w0 + q);
        wc1 = ONE_LEVEL ? wc0 : ld16(w1 + q);
    }
    for (int k = kb; k < ke; k++, q += Z) {
        const bool kin = k >= 1 && k <= ns - 2;
        Vec16<T> uf, vf, wf;
#pragma unroll
        for (int e = 0; e < N; e++) uf.v[e] = vf.v[e] = wf.v[e] = T(0);
        if (kin && jin) {
            const Vec16<T> a0 = ld16(u0 + q), a1 = ONE_LEVEL ? a0 : ld16(u1 + q);
            T a0r = T(0), a1r = T(0);
            if (need_r) {
                a0r = __ldg(u0 + q + N);
                a1r = ONE_LEVEL ? a0r : __ldg(u1 + q + N);
            }
#pragma unroll
            for (int e = 0; e < N; e++) {
                const T r0 = e < N - 1 ? a0.v[e < N - 1 ? e + 1 : 0] : a0r;
                const T r1 = e < N - 1 ? a1.v[e < N - 1 ? e + 1 : 0] : a1r;
                if (i0 + e <= nx - 2) uf.v[e] = mul_rn(rx[e], ((a0.v[e] + r0) + a1.v[e]) + r1);
            }
        }
        if (kin && jv) {
            const Vec16<T> b0 = ld16(v0 + q), b0u = ld16(v0 + q + Y);
            const Vec16<T> b1 = ONE_LEVEL ? b0 : ld16(v1 + q), b1u = ONE_LEVEL ? b0u : ld16(v1 + q + Y);
#pragma unroll
            for (int e = 0; e < N; e++)
                if (iin(e)) vf.v[e] = mul_rn(ry, ((b0.v[e] + b0u.v[e]) + b1.v[e]) + b1u.v[e]);
        }
        if (jin && k <= ns - 2) {
            const Vec16<T> wp0 = ld16(w0 + q + Z), wp1 = ONE_LEVEL ? wp0 : ld16(w1 + q + Z);
            const T rz = ratio<false>(qdt, ds[k]);
#pragma unroll
            for (int e = 0; e < N; e++)
                if (iin(e)) wf.v[e] = mul_rn(rz, ((wc0.v[e] + wp0.v[e]) + wc1.v[e]) + wp1.v[e]);
            wc0 = wp0;
            wc1 = wp1;
        }
        if (full) {
            st16(U + q, uf);
            st16(V + q, vf);
            st16(W + q, wf);
        } else {
#pragma unroll
            for (int e = 0; e < N; e++)
                if (i0 + e < nx) {
                    U[q + e] = uf.v[e];
                    V[q + e] = vf.v[e];
                    W[q + e] = wf.v[e];
                }
        }
    }
}

template <typename T, bool ONE_LEVEL>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 3 : 1) k_courant_donor_v(
    Dims d, const T* __restrict__ dx, const T* __restrict__ dy, const T* __restrict__ ds, T dt,
    const T* __restrict__ u0, const T* __restrict__ u1, const T* __restrict__ v0,
    const T* __restrict__ v1, const T* __restrict__ w0, const T* __restrict__ w1,
    const T* __restrict__ c0, T* __restrict__ U, T* __restrict__ V, T* __restrict__ W,
    T* __restrict__ c1, int depth, int zb, int ze)
{
    constexpr int N = Vec16<T>::N;
    const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * N;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i0 >= d.px || j > d.ny - 2) return;
    const int k0 = zb + (int)blockIdx.z * depth, k1 = min(ze, k0 + depth);
    const long long Y = d.px, Z = d.pp;
    const int nx = d.nx;
    const T qdt = RealConst<T>::quat * dt;
    // per-column and per-row Courant factors (QUAT dt / dx[i], uu.c:132)
    T rx[N], rxl = T(0);
#pragma unroll
    for (int e = 0; e < N; e++) rx[e] = (i0 + e <= nx - 2) ? ratio<false>(qdt, dx[i0 + e]) : T(0);
    const bool has_l = i0 >= 1 && i0 - 1 <= nx - 2;  // the face below the vector exists
    if (has_l) rxl = ratio<false>(qdt, dx[i0 - 1]);
    const T ry = ratio<false>(qdt, dy[j]), ryl = ratio<false>(qdt, dy[j - 1]);
    auto in_x = [&](int e) { return i0 + e >= 1 && i0 + e <= nx - 2; };

    long long q = cell(d, i0, j, k0);
    Vec16<T> cm = ld16(c0 + q - Z), cc = ld16(c0 + q);
    // z faces: W(k-1) from planes k-1, k; the planes k+1 are loaded per step
    Vec16<T> wa = ld16(w0 + q - Z), wc = ld16(w0 + q);
    Vec16<T> wb = ONE_LEVEL ? wa : ld16(w1 + q - Z), wd = ONE_LEVEL ? wc : ld16(w1 + q);
    Vec16<T> wlo;
    {
        const T rz = ratio<false>(qdt, ds[k0 - 1]);
#pragma unroll
        for (int e = 0; e < N; e++)
            wlo.v[e] = in_x(e) ? mul_rn(rz, ((wa.v[e] + wc.v[e]) + wb.v[e]) + wd.v[e]) : T(0);
        if (k0 == 1) st16(W + q - Z, wlo);  // face plane 0
    }
    for (int k = k0; k < k1; k++, q += Z) {
        const Vec16<T> cp = ld16(c0 + q + Z), cd = ld16(c0 + q - Y), cu = ld16(c0 + q + Y);
        const T cl = __ldg(c0 + q - 1), cr = __ldg(c0 + q + N);
        // x faces of the vector's cells and the one below its first cell
        const Vec16<T> a0 = ld16(u0 + q), a1 = ONE_LEVEL ? a0 : ld16(u1 + q);
        const T a0r = __ldg(u0 + q + N), a1r = ONE_LEVEL ? a0r : __ldg(u1 + q + N);
        Vec16<T> uf;
#pragma unroll
        for (int e = 0; e < N; e++) {
            const T r0 = e < N - 1 ? a0.v[e < N - 1 ? e + 1 : 0] : a0r;
            const T r1 = e < N - 1 ? a1.v[e < N - 1 ? e + 1 : 0] : a1r;
            uf.v[e] = (i0 + e <= nx - 2) ? mul_rn(rx[e], ((a0.v[e] + r0) + a1.v[e]) + r1) : T(0);
        }
        T ufl = T(0);
        if (has_l)
            {
            const T l0 = __ldg(u0 + q - 1), l1 = ONE_LEVEL ? l0 : __ldg(u1 + q - 1);
            ufl = mul_rn(rxl, ((l0 + a0.v[0]) + l1) + a1.v[0]);
        }
        // y faces j+1/2 and j-1/2
        const Vec16<T> b0 = ld16(v0 + q), b0u = ld16(v0 + q + Y), b0d = ld16(v0 + q - Y);
        const Vec16<T> b1 = ONE_LEVEL ? b0 : ld16(v1 + q), b1u = ONE_LEVEL ? b0u : ld16(v1 + q + Y),
                       b1d = ONE_LEVEL ? b0d : ld16(v1 + q - Y);
        Vec16<T> vf, vfl;
#pragma unroll
        for (int e = 0; e < N; e++) {
            vf.v[e] = in_x(e) ? mul_rn(ry, ((b0.v[e] + b0u.v[e]) + b1.v[e]) + b1u.v[e]) : T(0);
            vfl.v[e] = in_x(e) ? mul_rn(ryl, ((b0d.v[e] + b0.v[e]) + b1d.v[e]) + b1.v[e]) : T(0);
        }
        // z face k+1/2
        const Vec16<T> wp0 = ld16(w0 + q + Z), wp1 = ONE_LEVEL ? wp0 : ld16(w1 + q + Z);
        const T rz = ratio<false>(qdt, ds[k]);
        Vec16<T> wf;
#pragma unroll
        for (int e = 0; e < N; e++)
            wf.v[e] = in_x(e) ? mul_rn(rz, ((wc.v[e] + wp0.v[e]) + wd.v[e]) + wp1.v[e]) : T(0);
        st16(U + q, uf);
        st16(V + q, vf);
        if (j == 1) st16(V + q - Y, vfl);
        st16(W + q, wf);
        Vec16<T> out;
#pragma unroll
        for (int e = 0; e < N; e++) {
            const int i = i0 + e;
            const T left = e == 0 ? cl : cc.v[e > 0 ? e - 1 : 0];
            const T right = e == N - 1 ? cr : cc.v[e < N - 1 ? e + 1 : 0];
            const T uleft = e == 0 ? ufl : uf.v[e > 0 ? e - 1 : 0];
            out.v[e] = (i >= 1 && i <= nx - 2)
                           ? donor_update(cc.v[e], left, right, cd.v[e], cu.v[e], cm.v[e], cp.v[e],
                                          uf.v[e], uleft, vf.v[e], vfl.v[e], wf.v[e], wlo.v[e])
                           : cc.v[e];
        }
        st16(c1 + q, out);
        cm = cc;
        cc = cp;
        wlo = wf;
        wc = wp0;
        wd = wp1;
    }
}
