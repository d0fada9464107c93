"""GPU tests of the hand-written adjoint (mpdata_adjoint_*).

Checks (tolerances stated here):
  * FP64 adjoint vs central finite differences of the FP64 forward window
    along random directions: relative error <= 1e-6;
  * the dot-product identity <M v, w> = <v, M^T w> of the linear (order 1)
    step: relative 1e-12 (FP64);
  * FP32 adjoint vs the FP64 adjoint: relative L2 <= 1e-4;
  * the checkpoint interval does not change the gradient (FP64, 1e-10);
  * the torch.autograd.Function harness: a receptor loss differentiated with
    respect to the initial field and a source amplitude agrees with central
    differences to <= 1e-4 (FP32 adjoint, FP64 differences).
"""
import numpy as np
import pytest

from mpdata_b200 import workloads

pytestmark = pytest.mark.gpu


def _setup(n=20, ns=12, seed=0):
    """Smooth positive field, rotation about z plus a uniform w (boundary faces
    active: the shell takes part).  The field varies everywhere: on an exactly
    uniform background the limiter ratio is 0/(0 + tiny), a point where the
    limited flux is not differentiable (any perturbation moves the ratio by
    O(1)), so finite differences and the frozen-branch adjoint legitimately
    differ there."""
    r = workloads.ring3d(n=n, ns=ns, courant=0.35, wcourant=0.08, sigma=3.0, offset=3.0,
                         background=0.1, zero_flux=False)
    rng = np.random.default_rng(seed)
    k, j, i = np.mgrid[0:ns, 0:n, 0:n].astype(np.float64)
    c0 = r["c0"] + 0.04 * (1.0 + np.sin(0.7 * i + 0.3) * np.cos(0.45 * j - 0.2) *
                           np.cos(0.6 * k + 0.1))
    U, V, W = workloads.faces_from_cells(r["u"], r["v"], r["w"])
    return (U, V, W), c0, rng


def _fwd(faces, c0, nsteps, order, dtype=np.float64, **opts):
    import mpdata_b200.adjoint as ma
    with ma.Adjoint(c0.shape[2], c0.shape[1], c0.shape[0], order=order, dtype=dtype,
                    checkpoint_every=4, **opts) as a:
        a.set_faces(*(np.ascontiguousarray(f, dtype) for f in faces))
        return a.forward(np.ascontiguousarray(c0, dtype), nsteps).astype(np.float64)


def _grad(faces, c0, w, nsteps, order, dtype=np.float64, every=2, **opts):
    import mpdata_b200.adjoint as ma
    with ma.Adjoint(c0.shape[2], c0.shape[1], c0.shape[0], order=order, dtype=dtype,
                    checkpoint_every=every, **opts) as a:
        a.set_faces(*(np.ascontiguousarray(f, dtype) for f in faces))
        a.forward(np.ascontiguousarray(c0, dtype), nsteps)
        return a.backward(np.ascontiguousarray(w, dtype)).astype(np.float64)


@pytest.mark.parametrize("order,limiter", [(1, 0), (2, 0), (2, 1), (3, 0), (3, 1)])
def test_adjoint_matches_finite_differences_fp64(order, limiter):
    faces, c0, rng = _setup(seed=order + 10 * limiter)
    nsteps = 5
    w = rng.standard_normal(c0.shape)  # loss = <w, c^N>
    g = _grad(faces, c0, w, nsteps, order, limiter=bool(limiter))
    for _ in range(6):
        v = rng.standard_normal(c0.shape) * 0.05
        eps = 1e-6
        fp = float(np.sum(w * _fwd(faces, c0 + eps * v, nsteps, order, limiter=bool(limiter))))
        fm = float(np.sum(w * _fwd(faces, c0 - eps * v, nsteps, order, limiter=bool(limiter))))
        fd = (fp - fm) / (2 * eps)
        ad = float(np.sum(g * v))
        assert abs(fd - ad) <= 1e-6 * max(abs(fd), 1e-3), (fd, ad)


@pytest.mark.parametrize("nsteps", [1, 4])
def test_dot_product_identity_of_the_linear_step_fp64(nsteps):
    """Order 1 (the donor-cell pass alone) is linear in c, c^N = M c^0, so the
    adjoint must be its exact transpose: <M v, w> = <v, M^T w> to FP64
    rounding (relative 1e-12), for dense random v and w of both signs."""
    faces, c0, rng = _setup(seed=31 + nsteps)
    v = rng.standard_normal(c0.shape)
    w = rng.standard_normal(c0.shape)
    mv = _fwd(faces, v, nsteps, 1)
    mtw = _grad(faces, v, w, nsteps, 1)  # the transpose does not depend on the state
    lhs, rhs = float(np.sum(mv * w)), float(np.sum(v * mtw))
    scale = float(np.sum(np.abs(mv * w)))
    assert abs(lhs - rhs) <= 1e-12 * scale, (lhs, rhs)


@pytest.mark.parametrize("limiter", [0, 1])
def test_fp32_adjoint_close_to_fp64(limiter):
    faces, c0, rng = _setup(seed=3)
    w = rng.standard_normal(c0.shape)
    g64 = _grad(faces, c0, w, 6, 2, np.float64, limiter=bool(limiter))
    g32 = _grad(faces, c0, w, 6, 2, np.float32, limiter=bool(limiter))
    assert np.linalg.norm(g32 - g64) / np.linalg.norm(g64) <= 1e-4


def test_checkpoint_interval_does_not_change_gradient():
    faces, c0, rng = _setup(seed=4)
    w = rng.standard_normal(c0.shape)
    gs = [_grad(faces, c0, w, 7, 2, np.float64, every=e, limiter=True) for e in (1, 3, 10)]
    for g in gs[1:]:
        assert np.linalg.norm(g - gs[0]) / np.linalg.norm(gs[0]) <= 1e-10


def test_torch_harness_receptor_inversion():
    import torch

    import mpdata_b200.adjoint as ma
    nx = ny = 40
    ns = 20
    r = workloads.ring3d(n=nx, ns=ns, courant=0.4, wcourant=0.1, sigma=4.0, offset=8.0,
                         background=1e-6)
    faces = workloads.faces_from_cells(r["u"], r["v"], r["w"])
    k, j, i = np.mgrid[0:ns, 0:ny, 0:nx].astype(np.float64)
    # blob + a smoothly varying background (no exactly uniform region, see _setup)
    blob = (r["c0"] - 1e-6) + 1e-3 * (1.5 + np.sin(0.5 * i) * np.cos(0.4 * j + 0.3 * k))
    rng = np.random.default_rng(11)
    rec = rng.integers(0, nx * ny * ns, 16)
    tr = workloads.ring3d(n=nx, ns=ns, courant=0.4, wcourant=0.1, sigma=5.0, offset=-6.0,
                          background=1e-6)["c0"].reshape(-1)[rec]
    nsteps, every = 30, 10
    dev = torch.device("cuda", 0)
    Window = ma.window_function()

    def loss_fn(c0_t, adj):
        cN = Window.apply(c0_t, adj, nsteps)
        return ((cN.reshape(-1)[torch.as_tensor(rec, device=dev)]
                 - torch.as_tensor(tr, device=dev, dtype=cN.dtype)) ** 2).sum()

    with ma.Adjoint(nx, ny, ns, order=2, dtype=np.float32, checkpoint_every=every,
                    limiter=True) as adj32:
        adj32.set_faces(*(np.ascontiguousarray(f, np.float32) for f in faces))
        amp = torch.tensor(1.3, device=dev, dtype=torch.float32, requires_grad=True)
        base = torch.as_tensor(blob, device=dev, dtype=torch.float32)
        c0 = (1e-6 + amp * base).contiguous()
        c0.retain_grad()
        L = loss_fn(c0, adj32)
        L.backward()
        g_amp = float(amp.grad)
        g_c0 = c0.grad.double().cpu().numpy()

    def loss64(a_val, dc=None):
        c = 1e-6 + a_val * blob
        if dc is not None:
            c = c + dc
        cN = _fwd(faces, c, nsteps, 2, np.float64, limiter=True).reshape(-1)
        return float(np.sum((cN[rec] - tr) ** 2))

    h = 1e-4
    fd_amp = (loss64(1.3 + h) - loss64(1.3 - h)) / (2 * h)
    assert abs(g_amp - fd_amp) <= 1e-4 * abs(fd_amp) + 1e-7
    for _ in range(4):
        v = rng.standard_normal(blob.shape) * blob * 0.1  # relative: keeps the field positive
        e = 1e-4
        fd = (loss64(1.3, e * v) - loss64(1.3, -e * v)) / (2 * e)
        ad = float(np.sum(g_c0 * v))
        assert abs(fd - ad) <= 1e-4 * max(abs(fd), 1e-6) + 1e-7


def _c5_problem():
    """The adjoint configuration: 128x128x64, ring3d-type flow (rotation about
    z, max Courant 0.4, uniform w 0.1), Gaussian blob on a smoothly varying
    background, 64 seeded receptors against a target from another blob."""
    n, ns = 128, 64
    r = workloads.ring3d(n=n, ns=ns, courant=0.4, wcourant=0.1, sigma=6.0, offset=30.0,
                         background=1e-6)
    tr = workloads.ring3d(n=n, ns=ns, courant=0.4, wcourant=0.1, sigma=8.0, offset=-25.0,
                          background=1e-6)["c0"]
    faces = workloads.faces_from_cells(r["u"], r["v"], r["w"])
    k, j, i = np.mgrid[0:ns, 0:n, 0:n].astype(np.float64)
    c0 = r["c0"] + 1e-4 * (1.5 + np.sin(0.3 * i) * np.cos(0.25 * j + 0.2 * k))
    rng = np.random.default_rng(workloads.SEED + 5)
    rec = rng.integers(0, c0.size, 64)
    return faces, c0, rec, tr.reshape(-1)[rec], rng


def test_c5_window_adjoint():
    """The adjoint configuration at its size and length (200 steps,
    checkpoint every 20, IORD 2 + limiter with frozen branches):

    * FP64 adjoint against FP64 central differences along 8 random
      directions: median relative error <= 1e-5;
    * FP32 adjoint against the FP64 adjoint: relative L2 <= 0.1 and no more
      than 4x the FP64 adjoint's own change when c0 moves by 2^-20 per cell
      (relative), the size by which the FP32 forward leaves the FP64 one over
      the window (the limiter's frozen selections move with the trajectory);
    * two FP32 reverse sweeps of the same window agree to relative L2 1e-5
      (the scatter-adds are atomic, so their summation order varies)."""
    import mpdata_b200.adjoint as ma
    faces, c0, rec, t_rec, rng = _c5_problem()
    nsteps, every = 200, 20
    shape = c0.shape

    def lam_of(cN):
        lam = np.zeros(c0.size)
        np.add.at(lam, rec, 2.0 * (cN.reshape(-1)[rec] - t_rec))
        return lam.reshape(shape)

    def loss_of(cN):
        return float(np.sum((cN.reshape(-1)[rec] - t_rec) ** 2))

    def grad(a, c, dtype):
        cN = a.forward(np.ascontiguousarray(c, dtype), nsteps).astype(np.float64)
        return a.backward(np.ascontiguousarray(lam_of(cN), dtype)).astype(np.float64)

    with ma.Adjoint(shape[2], shape[1], shape[0], order=2, dtype=np.float64,
                    checkpoint_every=every, limiter=True) as a64:
        a64.set_faces(*(np.ascontiguousarray(f, np.float64) for f in faces))
        g64 = grad(a64, c0, np.float64)
        cp = c0 * (1.0 + np.random.default_rng(11).uniform(-2.0 ** -20, 2.0 ** -20, shape))
        sens = np.linalg.norm(grad(a64, cp, np.float64) - g64) / np.linalg.norm(g64)
        c64 = a64.forward(np.ascontiguousarray(c0), nsteps)
        errs = []
        for _ in range(8):
            v = rng.standard_normal(shape) * c0 * 1e-3
            e = 1e-5
            lp = loss_of(a64.forward(np.ascontiguousarray(c0 + e * v), nsteps))
            lm = loss_of(a64.forward(np.ascontiguousarray(c0 - e * v), nsteps))
            fd = (lp - lm) / (2 * e)
            errs.append(abs(fd - float(np.sum(g64 * v))) / max(abs(fd), 1e-30))
    assert float(np.median(errs)) <= 1e-5, errs
    with ma.Adjoint(shape[2], shape[1], shape[0], order=2, dtype=np.float32,
                    checkpoint_every=every, limiter=True) as a32:
        a32.set_faces(*(np.ascontiguousarray(f, np.float32) for f in faces))
        g32 = grad(a32, c0, np.float32)
        cN = a32.forward(np.ascontiguousarray(c0, np.float32), nsteps).astype(np.float64)
        # the FP32 window leaves the FP64 one by about the perturbation above
        assert np.linalg.norm(cN - c64) / np.linalg.norm(c64) <= 4e-6
        lam = np.ascontiguousarray(lam_of(cN), np.float32)
        g32b = a32.backward(lam).astype(np.float64)
        g32c = a32.backward(lam).astype(np.float64)
    rel32 = np.linalg.norm(g32 - g64) / np.linalg.norm(g64)
    assert rel32 <= 0.1 and rel32 <= 4.0 * sens + 1e-6, (rel32, sens)
    assert np.linalg.norm(g32b - g32c) / np.linalg.norm(g32b) <= 1e-5
