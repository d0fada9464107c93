"""Seeded synthetic inputs for the benchmark and test configurations.

No datasets are involved: every field is generated here from a fixed seed
with the shapes, flows and value distributions the configurations state.
Faces are returned in the solver's face layout (full-grid arrays; the entry
at (k, j, i) is the face on the high side of cell (i, j, k) along the axis)
and are face Courant numbers (dx = dy = ds = dt = 1).

Configurations:
  ring2d   128x128 (reference form 128x128x3), solid-body rotation with max
           Courant 0.5, Gaussian blob sigma 8 peak 1 at 32 cells right of
           centre, zero background, IORD 2, no limiter, zero-flux boundaries.
  ring3d   128^3, rotation about z (max Courant 0.4) + uniform w Courant 0.1,
           Gaussian sphere sigma 6 peak 1, 30 cells off axis, background 1e-6,
           IORD 2 with limiter.
  roofline 512x512x256, streamfunction flow (8 random Fourier modes,
           wavenumbers 1-8) + z-shear w = 0.05 sin(2 pi x / Lx), max Courant
           0.4, lognormal(0, 1) field smoothed by a 5-point box filter, IORD 3
           with limiter.
"""
from __future__ import annotations

import numpy as np

SEED = 20261203


def zero_flux_velocity(u: np.ndarray, v: np.ndarray, w: np.ndarray) -> None:
    """Make every boundary face Courant number exactly zero through the
    reference's cell-velocity API: each ghost cell gets minus its inner
    neighbour, so the face average (uu.c:132-134) vanishes.  In place."""
    u[:, :, 0] = -u[:, :, 1]
    u[:, :, -1] = -u[:, :, -2]
    v[:, 0, :] = -v[:, 1, :]
    v[:, -1, :] = -v[:, -2, :]
    w[0, :, :] = -w[1, :, :]
    w[-1, :, :] = -w[-2, :, :]


def faces_from_cells(u, v, w, dt=1.0):
    """Advective faces of cell velocities with dx = dy = ds = 1 and u0 = u1
    (the reference's uu.c:132-134 formula, in float64)."""
    ns, ny, nx = u.shape
    U = np.zeros_like(u); V = np.zeros_like(u); W = np.zeros_like(u)
    q = 0.25 * dt
    U[1:-1, 1:-1, :-1] = q * (2 * u[1:-1, 1:-1, :-1] + 2 * u[1:-1, 1:-1, 1:])
    V[1:-1, :-1, 1:-1] = q * (2 * v[1:-1, :-1, 1:-1] + 2 * v[1:-1, 1:, 1:-1])
    W[:-1, 1:-1, 1:-1] = q * (2 * w[:-1, 1:-1, 1:-1] + 2 * w[1:, 1:-1, 1:-1])
    return U, V, W


def cell_velocities(U, V, W):
    """Cell velocities for the cell-velocity smolar() API whose face averages
    (uu.c:132-134 with u0 = u1, dx = dt = 1) approximate the given faces:
    interior cells take the mean of their two faces, ghost cells the face
    next to them."""
    u = np.zeros_like(U); v = np.zeros_like(V); w = np.zeros_like(W)
    u[:, :, 1:-1] = 0.5 * (U[:, :, :-2] + U[:, :, 1:-1])
    u[:, :, 0] = U[:, :, 0]; u[:, :, -1] = U[:, :, -2]
    v[:, 1:-1, :] = 0.5 * (V[:, :-2, :] + V[:, 1:-1, :])
    v[:, 0, :] = V[:, 0, :]; v[:, -1, :] = V[:, -2, :]
    w[1:-1] = 0.5 * (W[:-2] + W[1:-1])
    w[0] = W[0]; w[-1] = W[-2]
    return u, v, w


def max_courant(U, V, W) -> float:
    return float(max(np.abs(U).max(), np.abs(V).max(), np.abs(W).max()))


def ring2d(n: int = 128, courant: float = 0.5, sigma: float = 8.0, offset: float = 32.0,
           zero_flux: bool = True):
    """Reference-form 2D ring case (n x n x 3): returns dict with cell
    velocities u, v, w, the initial field c0 (all float64) and dt."""
    ns = 3
    yc = xc = (n - 1) / 2.0
    y, x = np.mgrid[0:n, 0:n].astype(np.float64)
    # faces of interior rows/columns take the cell value (u independent of x)
    rmax = max(np.abs(np.arange(1, n - 1) - yc).max(), 1e-30)
    omega = courant / rmax
    u2 = -omega * (y - yc)
    v2 = omega * (x - xc)
    u = np.repeat(u2[None], ns, 0)
    v = np.repeat(v2[None], ns, 0)
    w = np.zeros((ns, n, n))
    if zero_flux:
        zero_flux_velocity(u, v, w)
        w[:] = 0.0
    g = np.exp(-0.5 * ((x - (xc + offset)) ** 2 + (y - yc) ** 2) / sigma ** 2)
    c0 = np.repeat(g[None], ns, 0)
    return dict(u=u, v=v, w=w, c0=c0, dt=1.0, order=2, limiter=False)


def ring3d(n: int = 128, ns: int | None = None, courant: float = 0.4, wcourant: float = 0.1,
           sigma: float = 6.0, offset: float = 30.0, background: float = 1e-6,
           zero_flux: bool = True):
    """3D ring case: rotation about z plus a uniform w."""
    ns = n if ns is None else ns
    yc = xc = (n - 1) / 2.0
    zc = (ns - 1) / 2.0
    k, y, x = np.mgrid[0:ns, 0:n, 0:n].astype(np.float64)
    rmax = max(np.abs(np.arange(1, n - 1) - yc).max(), 1e-30)
    omega = courant / rmax
    u = -omega * (y - yc)
    v = omega * (x - xc)
    w = np.full_like(u, wcourant)
    if zero_flux:
        zero_flux_velocity(u, v, w)
    c0 = background + np.exp(-0.5 * ((x - (xc + offset)) ** 2 + (y - yc) ** 2 + (k - zc) ** 2)
                             / sigma ** 2)
    return dict(u=u, v=v, w=w, c0=c0, dt=1.0, order=2, limiter=True)


def roofline(nx: int = 512, ny: int = 512, ns: int = 256, courant: float = 0.4,
             modes: int = 8, seed: int = SEED):
    """Streamfunction flow and lognormal field; returns faces U, V, W and c0
    (float64).  The x-y faces are differences of a corner streamfunction, so
    the x-y flow is exactly discretely divergence-free; W = 0.05 sin(2 pi x/Lx)
    has no z derivative."""
    rng = np.random.default_rng(seed)
    Lx, Ly = float(nx), float(ny)
    kx = rng.integers(1, 9, modes)
    ly = rng.integers(1, 9, modes)
    ph = rng.uniform(0, 2 * np.pi, modes)
    amp = rng.uniform(0.5, 1.0, modes)
    # psi at cell corners (x = i + 1/2, y = j + 1/2), for i in -1..nx-1, j in -1..ny-1
    xs = np.arange(-1, nx) + 0.5
    ys = np.arange(-1, ny) + 0.5
    psi = np.zeros((ny + 1, nx + 1))
    for m in range(modes):
        psi += amp[m] * np.sin(2 * np.pi * (kx[m] * xs[None, :] / Lx + ly[m] * ys[:, None] / Ly)
                               + ph[m])
    # U at face (i+1/2, j) = psi(i+1/2, j+1/2) - psi(i+1/2, j-1/2)
    U2 = psi[1:, 1:] - psi[:-1, 1:]           # shape (ny, nx): [j, i]
    # V at face (i, j+1/2) = -(psi(i+1/2, j+1/2) - psi(i-1/2, j+1/2))
    V2 = -(psi[1:, 1:] - psi[1:, :-1])
    W2 = 0.05 * np.sin(2 * np.pi * (np.arange(nx) + 0.0) / Lx)[None, :].repeat(ny, 0)
    U = np.zeros((ns, ny, nx)); V = np.zeros((ns, ny, nx)); W = np.zeros((ns, ny, nx))
    U[1:-1, 1:-1, :-1] = U2[None, 1:-1, :-1]
    V[1:-1, :-1, 1:-1] = V2[None, :-1, 1:-1]
    W[:-1, 1:-1, 1:-1] = W2[None, 1:-1, 1:-1]
    s = courant / max_courant(U, V, W)
    U *= s; V *= s; W *= s
    c = rng.lognormal(0.0, 1.0, (ns, ny, nx))
    cs = c.copy()
    cs[:, 1:-1, 1:-1] = (c[:, 1:-1, 1:-1] + c[:, :-2, 1:-1] + c[:, 2:, 1:-1] + c[:, 1:-1, :-2]
                         + c[:, 1:-1, 2:]) / 5.0
    return dict(U=U, V=V, W=W, c0=cs, order=3, limiter=True)


def random_case(nx, ny, ns, seed=0, courant=0.3, positive=True):
    """Random cell velocities (two time levels), non-uniform grid steps and a
    positive field: exercises every formula, the x=1 column included."""
    rng = np.random.default_rng(seed)
    sh = (ns, ny, nx)
    u0 = rng.uniform(-courant, courant, sh); u1 = u0 + rng.uniform(-0.05, 0.05, sh)
    v0 = rng.uniform(-courant, courant, sh); v1 = v0 + rng.uniform(-0.05, 0.05, sh)
    w0 = rng.uniform(-courant, courant, sh); w1 = w0 + rng.uniform(-0.05, 0.05, sh)
    c = rng.uniform(0.0, 1.0, sh) if positive else rng.uniform(-1.0, 1.0, sh)
    dx = rng.uniform(0.8, 1.2, nx); dy = rng.uniform(0.8, 1.2, ny); ds = rng.uniform(0.8, 1.2, ns)
    return dict(u0=u0, u1=u1, v0=v0, v1=v1, w0=w0, w1=w1, c0=c, dx=dx, dy=dy, ds=ds, dt=0.9)


def integer_case(nx, ny, ns, seed=0, cmax=40, moving=0.15):
    """Inputs for the reference's INTEGER build (real = long): int64 arrays.
    Grid steps 1 or 2 and dt 1 or 2 (so some faces truncate to 0: QUAT dt /
    dx is an integer division), sparse cell velocities in {-1, 0, 1} (a
    fraction `moving` of the cells, two time levels), a field of small
    non-negative integers.  Values stay small over a few steps, but the
    integer scheme is not positivity-preserving: a later step may divide by
    zero (c_hi + c_lo + MINVAL = 0), which callers detect."""
    rng = np.random.default_rng(seed)
    sh = (ns, ny, nx)

    def vel():
        return np.where(rng.random(sh) < moving, rng.integers(-1, 2, sh), 0).astype(np.int64)

    u0, v0, w0 = vel(), vel(), vel()
    u1 = np.where(rng.random(sh) < 0.5, u0, vel()).astype(np.int64)
    v1 = np.where(rng.random(sh) < 0.5, v0, vel()).astype(np.int64)
    w1 = np.where(rng.random(sh) < 0.5, w0, vel()).astype(np.int64)
    c = rng.integers(0, cmax + 1, sh).astype(np.int64)
    dx = rng.integers(1, 3, nx).astype(np.int64)
    dy = rng.integers(1, 3, ny).astype(np.int64)
    ds = rng.integers(1, 3, ns).astype(np.int64)
    return dict(u0=u0, u1=u1, v0=v0, v1=v1, w0=w0, w1=w1, c0=c, dx=dx, dy=dy, ds=ds,
                dt=int(rng.integers(1, 3)))


def ensemble(n: int = 256, lo: int = 64, hi: int = 512, seed: int = SEED + 4):
    """Batched-ensemble configuration: n independent 2D instances, NX, NY
    uniform in [lo, hi], solid-body rotation with max Courant uniform in
    [0.2, 0.5], Gaussian blob (sigma 4-16 cells, centre at least 3 sigma from
    the edges), IORD 2 with the limiter.  Returns a list of dicts with 2D
    faces U, V (float64) and field c0, shape (ny, nx)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx = int(rng.integers(lo, hi + 1)); ny = int(rng.integers(lo, hi + 1))
        cour = rng.uniform(0.2, 0.5)
        sig = rng.uniform(4.0, 16.0)
        sig = min(sig, (min(nx, ny) - 3) / 6.0 - 1e-3)
        cx = rng.uniform(3 * sig, nx - 1 - 3 * sig)
        cy = rng.uniform(3 * sig, ny - 1 - 3 * sig)
        yc, xc = (ny - 1) / 2.0, (nx - 1) / 2.0
        y, x = np.mgrid[0:ny, 0:nx].astype(np.float64)
        U = np.zeros((ny, nx)); V = np.zeros((ny, nx))
        # faces of interior rows/columns; boundary faces zero (closed box)
        U[1:-1, 1:-1] = -(y[1:-1, 1:-1] - yc)
        V[1:-1, 1:-1] = (x[1:-1, 1:-1] - xc)
        U[:, 0] = 0.0; U[:, -1] = 0.0; U[:, -2] = 0.0
        V[0, :] = 0.0; V[-1, :] = 0.0; V[-2, :] = 0.0
        s = cour / max(np.abs(U).max(), np.abs(V).max())
        c0 = np.exp(-0.5 * ((x - cx) ** 2 + (y - cy) ** 2) / sig ** 2)
        out.append(dict(nx=nx, ny=ny, U=U * s, V=V * s, c0=c0))
    return out
