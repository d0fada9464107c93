"""Ring-case drivers: the reference's own ring2d/ring3d programs (tests/ring2d/test.c,
tests/ring3d/test.c with tests/init.c), linked once against the reference core and
once against libmpdata_b200.so, and the package's C driver mpdata_b200/drivers/ring.

CPU tests check the C driver's set-up (no steps, so no GPU call) against the
reference's test_init() byte for byte.  GPU tests run the same binaries for a few
steps and compare their output files.
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BIN = os.path.join(ROOT, "oracle", "_ref")
RING = os.path.join(ROOT, "mpdata_b200", "drivers", "ring")


def _bin(name):
    path = os.path.join(REF_BIN, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not built (reference sources absent when building)")
    return path


def _ring():
    if not os.path.exists(RING):
        pytest.skip("mpdata_b200/drivers/ring not built")
    return RING


def run(cmd, cwd, env_opts=None):
    env = dict(os.environ)
    env.pop("MPDATA_B200_OPTIONS", None)
    if env_opts is not None:
        env["MPDATA_B200_OPTIONS"] = env_opts
    p = subprocess.run(cmd, cwd=cwd, env=env, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, f"{cmd} failed: {p.stdout}\n{p.stderr}"
    return p.stdout


def frames(path, n):
    """ring2d.bin: per step the u, v and c planes of level 1 (tests/ring2d/test.c:39-53)."""
    a = np.fromfile(path, dtype=np.float32)
    return a.reshape(-1, 3, n, n)


def test_ring_setup_matches_reference_2d(tmp_path):
    ref, own = tmp_path / "ref", tmp_path / "own"
    ref.mkdir(), own.mkdir()
    run([_bin("ring2d_ref"), "64", "0"], ref)
    run([_ring(), "64", "3", "0", "--frames", "ring2d.bin"], own)
    assert (ref / "ring2d.bin").read_bytes() == (own / "ring2d.bin").read_bytes()


def test_ring_setup_matches_reference_3d(tmp_path):
    ref, own = tmp_path / "ref", tmp_path / "own"
    ref.mkdir(), own.mkdir()
    run([_bin("ring3d_ref"), "24", "0"], ref)
    run([_ring(), "24", "24", "0", "--final", "c.bin"], own)
    # the reference's raw VAPOR scratch file ends up holding the last field it wrote: c
    assert (ref / "data.bin").read_bytes() == (own / "c.bin").read_bytes()


def test_ring_usage_errors(tmp_path):
    p = subprocess.run([_ring(), "2", "3", "1"], cwd=tmp_path, capture_output=True)
    assert p.returncode == 2
    p = subprocess.run([_ring(), "16", "3", "1", "--bogus"], cwd=tmp_path, capture_output=True)
    assert p.returncode == 2


@pytest.mark.gpu
@pytest.mark.parametrize("n,nt", [(64, 25), (101, 12)])
def test_reference_ring2d_driver_on_gpu_strict(tmp_path, n, nt):
    """The reference's unmodified ring2d driver, linked against the GPU library with
    strict arithmetic, writes the same bytes as when linked against the reference core."""
    ref, gpu = tmp_path / "ref", tmp_path / "gpu"
    ref.mkdir(), gpu.mkdir()
    out_ref = run([_bin("ring2d_ref"), str(n), str(nt)], ref)
    out_gpu = run([_bin("ring2d_b200"), str(n), str(nt)], gpu, env_opts="strict")
    assert out_ref == out_gpu
    assert (ref / "ring2d.bin").read_bytes() == (gpu / "ring2d.bin").read_bytes()
    assert (ref / "ring2d.ctl").read_bytes() == (gpu / "ring2d.ctl").read_bytes()


@pytest.mark.gpu
def test_reference_ring2d_driver_on_gpu_default(tmp_path):
    """Default (FMA-contracted) arithmetic: within FP32 rounding of the reference."""
    n, nt = 64, 25
    ref, gpu = tmp_path / "ref", tmp_path / "gpu"
    ref.mkdir(), gpu.mkdir()
    run([_bin("ring2d_ref"), str(n), str(nt)], ref)
    run([_bin("ring2d_b200"), str(n), str(nt)], gpu)
    a = frames(ref / "ring2d.bin", n)
    b = frames(gpu / "ring2d.bin", n)
    np.testing.assert_array_equal(a[:, :2], b[:, :2])
    assert float(np.abs(a[:, 2] - b[:, 2]).max()) <= 2e-6


@pytest.mark.gpu
def test_reference_ring3d_driver_on_gpu_strict(tmp_path):
    n, nt = 32, 6
    ref, gpu = tmp_path / "ref", tmp_path / "gpu"
    ref.mkdir(), gpu.mkdir()
    out_ref = run([_bin("ring3d_ref"), str(n), str(nt)], ref)
    out_gpu = run([_bin("ring3d_b200"), str(n), str(nt)], gpu, env_opts="strict")
    assert out_ref == out_gpu
    assert (ref / "data.bin").read_bytes() == (gpu / "data.bin").read_bytes()


@pytest.mark.gpu
@pytest.mark.parametrize("device", [False, True])
def test_own_ring_driver_matches_reference(tmp_path, device):
    n, nt = 64, 25
    ref, own = tmp_path / "ref", tmp_path / "own"
    ref.mkdir(), own.mkdir()
    out_ref = run([_bin("ring2d_ref"), str(n), str(nt)], ref)
    cmd = [_ring(), str(n), "3", str(nt), "--strict", "--frames", "ring2d.bin"]
    out_own = run(cmd + (["--device"] if device else []), own)
    assert out_ref == out_own
    assert (ref / "ring2d.bin").read_bytes() == (own / "ring2d.bin").read_bytes()


@pytest.mark.gpu
def test_own_ring_driver_3d_matches_reference(tmp_path):
    n, nt = 32, 6
    ref, own = tmp_path / "ref", tmp_path / "own"
    ref.mkdir(), own.mkdir()
    run([_bin("ring3d_ref"), str(n), str(nt)], ref)
    run([_ring(), str(n), str(n), str(nt), "--strict", "--device", "--final", "c.bin"], own)
    assert (ref / "data.bin").read_bytes() == (own / "c.bin").read_bytes()


@pytest.mark.gpu
def test_own_ring_driver_limiter(tmp_path, oracle_mod):
    """Nonoscillatory switch: positive, mass-conserving, and equal to the oracle."""
    n, nt = 48, 10
    run([_ring(), str(n), "3", str(nt), "--limiter", "--strict", "--device",
         "--frames", "f.bin", "--final", "c.bin"], tmp_path)
    f = frames(tmp_path / "f.bin", n)
    assert float(f[:, 2].min()) >= 0.0
    last = np.fromfile(tmp_path / "c.bin", dtype=np.float32).reshape(3, n, n)
    # the oracle replays the same set-up from the reference's test_init
    cfg = oracle_mod.ref_test_init(n, 3, "f32")
    c = cfg["c0"].astype(np.float32)
    U, V, W = oracle_mod.courant(cfg["dx"], cfg["dy"], cfg["ds"], cfg["dt"], cfg["u"], cfg["u"],
                                 cfg["v"], cfg["v"], cfg["w"], cfg["w"], dtype=np.float32)
    for _ in range(nt):
        c = oracle_mod.step_faces(U, V, W, c, 3, limiter=1)
    np.testing.assert_array_equal(last, c)
