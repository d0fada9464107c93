#!/usr/bin/env python
"""Throughput of the MPDATA step on B200: Gcell-steps/s and HBM roofline.

Workload (the single-grid roofline configuration): 512 x 512 x 256 FP32,
IORD 3 with the nonoscillatory limiter, steady streamfunction flow (8 seeded
Fourier modes + z-shear, max Courant 0.4), lognormal field smoothed by a
5-point box filter.  Synthetic, seeded (mpdata_b200/workloads.py).  Every
field is 268 MB, larger than the 126 MB L2, so no L2 flush is needed between
steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

One JSON line on rank 0.  value: interior cell-steps per second over all
ranks (each rank steps its own grid: replicas, weak scaling), timed with
CUDA events on the solver's stream, max over ranks.  e2e: the same metric
through the reference-compatible smolar() C-ABI call with pinned host
buffers (velocity and field uploads, newest and previous field downloads
inside the timed region).  roofline: the fused corrective-pass kernel's
algorithmic bytes per launch over its CUDA-event launch time.  cpu_baseline:
the reference's own smolar() (compiled from its sources with its CMake
flags, oracle/_ref) on the host cores.

--impl reference runs only that CPU reference path (rank 0) and prints its
line with "impl": "reference".
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gcell-steps/s & % HBM roofline on 1 B200, plain vs chosen at stated FP64 error"
UNIT = "Gcell-steps/s"
NX, NY, NS, ORDER = 512, 512, 256, 3


def _set_size(nx, ny, ns):
    global NX, NY, NS, CELLS, FIELD_BYTES
    NX, NY, NS = nx, ny, ns
    CELLS = (NX - 2) * (NY - 2) * (NS - 2)
    FIELD_BYTES = NX * NY * NS * 4


_set_size(NX, NY, NS)
# Algorithmic bytes per interior cell (FP32, d = 3, IORD 3, limiter on):
#   donor pass        reads c^n + 3 faces, writes c^(1)                      5
#   corrective pass 1 reads c^(1), c^n, 3 faces; writes c^(2) + 3 faces      9
#   corrective pass 2 reads c^(2), c^n, 3 faces; writes c^(3)                6
B_DONOR, B_CORR_FACES, B_CORR_LAST = 5 * 4, 9 * 4, 6 * 4
B_STEP = B_DONOR + B_CORR_FACES + B_CORR_LAST  # 80 B per cell-step
# Ensemble (2D, IORD 2, limiter), counted as separate passes: donor reads c and
# 2 faces, writes c (4 elements); the corrective pass reads c^(1), c^n, 2 faces
# and writes c^(2) (5 elements).  The fused form keeps c^(1) on chip (4 elements
# move: c^n, 2 faces in, c^(2) out).
B_ENSEMBLE = 9 * 4
B_ENSEMBLE_FUSED = 4 * 4
FALLBACK_HBM_GBS = 6650.0
# Arithmetic forms timed, all on the two-cell pass: "plain" = IEEE FP32
# throughout (round-to-nearest division); "precision_form" =
# FP32 storage and faces (hardware-reciprocal face ratios) with the limiter's
# sums and ratios in FP64; "approx_div" = FP32 with hardware-reciprocal ratios
# everywhere.  The headline value is the fastest form within the FP64 error
# bound (see the selection below).
FORMS = [("plain", {}), ("precision_form", {"precision_form": True, "approx_div": True}),
         ("approx_div", {"approx_div": True})]
FP64_REL_L2_BOUND = 1e-5
# Options of the throughput workload beside the form: the y faces of the x = 1
# column are computed (vv_fix).  The reference leaves them unwritten
# (vv.c:81-82): its first corrective pass reads an uninitialised buffer there
# and, with IORD 3, its second one applies the advective velocity as an
# antidiffusive one in that column.  The accuracy check reports that rule too.
WORKLOAD_OPTS = {"vv_fix": True}
ACC_STEPS = 100  # horizon of the FP64 accuracy check: the configuration's length
# The corrective-pass kernel each form runs (the solver's default kernel choice).
KERNEL_OF_FORM = {
    "plain": "k_pass_pair<limiter, IEEE division> (fused corrective pass, two cells per thread)",
    "precision_form": "k_pass_pair<limiter, approx, FP64 limiter ratios> (fused corrective pass, "
                      "two cells per thread)",
    "approx_div": "k_pass_pair<limiter, approx> (fused corrective pass, two cells per thread)",
}


# Solver kernel choices (mpdata_options.kernel) that --kernel can force on the
# timed forms, for profiling captures of the other kernels; forms a kernel
# cannot run (approx_div needs the fused kernels) are dropped.
KERNEL_CHOICES = {
    1: "k_antidiff + k_fct_beta + k_fct_apply + k_donor (one kernel per reference routine)",
    2: "k_pass_tma<limiter> (fused corrective pass, one cell per thread)",
    3: None,  # the two-cell pass: the default labels above
}


def _set_kernel(kernel):
    global FORMS, KERNEL_OF_FORM
    forms = [(n, o) for n, o in FORMS if not (kernel == 1 and o.get("approx_div"))]
    FORMS = [(n, dict(o, kernel=kernel)) for n, o in forms]
    if KERNEL_CHOICES[kernel] is not None:
        KERNEL_OF_FORM = {n: KERNEL_CHOICES[kernel] for n, _ in FORMS}


def _add_form_options(**kw):
    """Options added to every timed form (profiling captures)."""
    global FORMS
    FORMS = [(n, dict(o, **kw)) for n, o in FORMS]


def config_text():
    return (f"roofline: {NX}x{NY}x{NS} FP32, IORD {ORDER} + nonoscillatory limiter, "
            "streamfunction flow, y faces of the x = 1 column computed (vv_fix)")


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def traffic_from_profile():
    """DRAM bytes per corrective-pass launch from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "roofline_traffic.txt")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


# ---------------------------------------------------------------------------
# clocks

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        """Start sampling and return once the sampler has written its first
        row (nvidia-smi needs ~0.1-0.5 s to start), so the timed region that
        follows is covered from its beginning; rows written before that are
        dropped by stop()."""
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.skip = 0
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "10"],  # several per 0.1 s
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        t_end = time.time() + 5.0
        while time.time() < t_end and self.proc.poll() is None:
            with open(self.path) as f:
                n = sum(1 for line in f if line.endswith("\n"))
            if n:
                self.skip = n
                break
            time.sleep(0.01)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        lines = open(self.path).readlines()
        # rows written before the timed region; keep them only if nothing came after
        if len(lines) > self.skip:
            lines = lines[self.skip:]
        for line in lines:
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                rows.append((float(p[1]), float(p[2]), p[5:]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        sm = sorted(r[0] for r in rows)
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[2]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": max(r[1] for r in rows),
                "reasons": sorted(reasons), "samples": len(rows)}


# ---------------------------------------------------------------------------
# CPU reference path (the reference's own smolar, compiled from its sources)

def cpu_reference(steps: int, warmup: int, threads: int | None = None):
    """Reference smolar() (FP32, -ffast-math -O3 build) on the host cores:
    `threads` independent z-slab instances of the roofline grid, 32 interior
    planes each (the sample), one smolar call per instance per step."""
    import ctypes as C

    import oracle
    if not oracle.ref_available("f32_fast"):
        return None
    lib = oracle.ref_lib("f32_fast")
    T = threads or min(os.cpu_count() or 1, 64)
    planes = 32
    wl = _workload()
    u, v, w = _workloads_module().cell_velocities(wl["U"], wl["V"], wl["W"])
    insts = []
    for t in range(T):
        z0 = (t * planes) % (NS - planes - 2)
        sl = slice(z0, z0 + planes + 2)
        arrs = {k: np.ascontiguousarray(a[sl], np.float32) for k, a in
                (("u", u), ("v", v), ("w", w), ("c0", wl["c0"]))}
        arrs["c1"] = np.zeros_like(arrs["c0"])
        insts.append(arrs)
    dx = np.ones(NX, np.float32); dy = np.ones(NY, np.float32); ds = np.ones(planes + 2, np.float32)
    P = C.POINTER(C.c_float)

    def run(inst, nsteps):
        p0 = C.cast(inst["c0"].ctypes.data, P)
        p1 = C.cast(inst["c1"].ctypes.data, P)
        vel = [inst[k].ctypes.data_as(P) for k in ("u", "u", "v", "v", "w", "w")]
        for _ in range(nsteps):
            lib.smolar(NX, NY, planes + 2, dx.ctypes.data_as(P), dy.ctypes.data_as(P),
                       ds.ctypes.data_as(P), C.c_float(1.0), *vel, C.byref(p0), C.byref(p1), 1,
                       ORDER)
            p0, p1 = p1, p0

    def run_all(nsteps):
        th = [threading.Thread(target=run, args=(i, nsteps)) for i in insts]
        t0 = time.perf_counter()
        for x in th:
            x.start()
        for x in th:
            x.join()
        return time.perf_counter() - t0

    if warmup:
        run_all(warmup)
    dt = run_all(steps)
    cells = T * (NX - 2) * (NY - 2) * planes
    rate = cells * steps / dt / 1e9
    return {"value": rate, "unit": UNIT, "cores": T, "kind": "reference",
            "sample": f"{T} thread(s) x independent {NX}x{NY}x{planes + 2} z-slab of the "
                      f"roofline grid, IORD {ORDER}, reference smolar() built with its CMake "
                      f"flags (-ffast-math -O3; the reference has no limiter), {steps} step(s)",
            "seconds": dt, "instances": T, "slab": [NX, NY, planes + 2]}


# ---------------------------------------------------------------------------
# GPU

_WL = None


def _workloads_module():
    """mpdata_b200/workloads.py loaded on its own (it needs only numpy).  The
    reference arm uses this: importing the package would map
    libmpdata_b200.so into a process that must run the reference alone."""
    import importlib.util
    path = os.path.join(ROOT, "mpdata_b200", "workloads.py")
    spec = importlib.util.spec_from_file_location("mpdata_b200_workloads", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _workload():
    global _WL
    if _WL is None:
        wl = _workloads_module().roofline(NX, NY, NS)
        _WL = {k: (v.astype(np.float32) if isinstance(v, np.ndarray) else v)
               for k, v in wl.items()}
    return _WL


def half_ulp_perturbed(c, seed=11):
    """c (FP64) times 1 + u, u uniform in [-2^-24, 2^-24] per cell (seeded):
    a perturbation of the size of one rounding of the field to FP32."""
    rng = np.random.default_rng(seed)
    return c.astype(np.float64) * (1.0 + rng.uniform(-2.0 ** -24, 2.0 ** -24, c.shape))


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_gpu(args):
    import datetime

    import torch
    import mpdata_b200 as m

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    wl = _workload()
    stream = torch.cuda.current_stream()

    def timed_form(opts):
        """W untimed steps, then EXACTLY K timed steps of one arithmetic form."""
        s = m.Solver(NX, NY, NS, order=ORDER, limiter=True, **WORKLOAD_OPTS, **opts)
        s.set_stream(stream.cuda_stream)
        s.set_faces(wl["U"], wl["V"], wl["W"])
        s.set_field(wl["c0"])
        s.step(args.warmup)
        torch.cuda.synchronize()
        s.enable_pass_timing(True)
        s.pass_times(reset=True)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        clocks = ClockSampler(local)
        clocks.start()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            s.step(1)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        clk = clocks.stop()
        t_ms = e0.elapsed_time(e1)
        if dist:
            t = torch.tensor([t_ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            t_ms = float(t.item())
            dist.barrier()
        ms, n = s.pass_times()
        s.enable_pass_timing(False)
        mn, nneg = s.min()
        r = dict(t_ms=t_ms, ms=ms, n=n, min=mn, nneg=nneg, clk=clk,
                 launches=s.launches_per_step() * args.steps, final=s.get_field())
        s.close()
        return r

    results = {name: timed_form(o) for name, o in FORMS}

    def fp64_run(nsteps, c0=None, **wopts):
        s64 = m.Solver(NX, NY, NS, order=ORDER, dtype=np.float64, limiter=True, **wopts)
        s64.set_stream(stream.cuda_stream)
        s64.set_faces(*(wl[k].astype(np.float64) for k in ("U", "V", "W")))
        s64.set_field(wl["c0"].astype(np.float64) if c0 is None else c0)
        s64.step(nsteps)
        out = s64.get_field()
        s64.close()
        return out

    def rel(a, ref, nref):
        diff = a.astype(np.float64) - ref
        return float(np.linalg.norm(diff)) / nref, float(np.abs(diff).max())

    # Accuracy of each FP32 form against an FP64 run of the plain method over
    # the configuration's own length (ACC_STEPS from c0, independent of K),
    # and at the end of the timed run (W + K steps).  Beside them, the FP64
    # scheme's own sensitivity: the same FP64 run started from c0 perturbed
    # by half an FP32 ulp (relative) per cell -- the error any FP32-storage
    # form incurs by rounding the field once.
    def form_run(o, nsteps, **wopts):
        s = m.Solver(NX, NY, NS, order=ORDER, limiter=True, **wopts, **o)
        s.set_stream(stream.cuda_stream)
        s.set_faces(wl["U"], wl["V"], wl["W"])
        s.set_field(wl["c0"])
        s.step(nsteps)
        out = s.get_field()
        s.close()
        return out

    ref64 = fp64_run(ACC_STEPS, **WORKLOAD_OPTS)
    nref = float(np.linalg.norm(ref64))
    acc = {name: rel(form_run(o, ACC_STEPS, **WORKLOAD_OPTS), ref64, nref) for name, o in FORMS}
    floor = rel(fp64_run(ACC_STEPS, half_ulp_perturbed(wl["c0"]), **WORKLOAD_OPTS), ref64, nref)
    # the reference's column rule (y faces of x = 1 unwritten), same horizon
    ref64 = fp64_run(ACC_STEPS)
    nref = float(np.linalg.norm(ref64))
    ref_rule = {}
    for name, o in FORMS:
        b, _ = error_breakdown(form_run(o, ACC_STEPS), ref64, nref)
        ref_rule[name] = {k: b[k] for k in ("rel_l2", "max_abs", "share_column_x1",
                                            "rel_l2_without_x_le_2")}
    ref64 = fp64_run(args.warmup + args.steps, **WORKLOAD_OPTS)
    nref = float(np.linalg.norm(ref64))
    forms = {}
    for name, r in results.items():
        r["rel_l2_vs_fp64"], r["max_abs_vs_fp64"] = acc[name]
        r["rel_l2_vs_fp64_end"], r["max_abs_vs_fp64_end"] = rel(r.pop("final"), ref64, nref)
        r["value"] = world * CELLS * args.steps / (r["t_ms"] * 1e-3) / 1e9
        forms[name] = r
    del ref64
    # The headline form: the fastest one within the bound after ACC_STEPS with
    # no negative cell.  If no FP32 form meets the bound, the fastest one no
    # less accurate than the plain FP32 method (the reference precision) at
    # that horizon, with the bound reported as not met.
    ok_forms = [k for k, r in forms.items()
                if r["rel_l2_vs_fp64"] <= FP64_REL_L2_BOUND and r["nneg"] == 0]
    bound_met = bool(ok_forms)
    if not ok_forms:
        cap = forms["plain"]["rel_l2_vs_fp64"]
        ok_forms = [k for k, r in forms.items() if r["rel_l2_vs_fp64"] <= cap and r["nneg"] == 0]
    chosen = max(ok_forms, key=lambda k: forms[k]["value"]) if ok_forms else "plain"
    sel = forms[chosen]
    t_ms, ms, n, clk = sel["t_ms"], sel["ms"], sel["n"], sel["clk"]
    mn, nneg, launches, value = sel["min"], sel["nneg"], sel["launches"], sel["value"]

    # e2e through the reference-facing smolar() with pinned host buffers
    e2e = None
    if rank == 0 and not args.no_e2e:
        e2e = run_e2e(m, args, dict(FORMS)[chosen])
    tdep = None
    if rank == 0 and not args.no_time_dependent:
        tdep = run_time_dependent(m, torch, dict(FORMS)[chosen])
    ens = None
    if rank == 0 and not args.no_ensemble:
        ens = run_ensemble(m, torch, args.ensemble_steps, 10)
    adj = None
    if rank == 0 and not args.no_adjoint:
        adj = run_adjoint(m, torch)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return None

    peak, peak_kind = hbm_peak()
    corr_bytes = (n[1] * B_CORR_FACES + n[2] * B_CORR_LAST) * CELLS
    corr_ms = ms[1] + ms[2]
    achieved = corr_bytes / (corr_ms * 1e-3) / 1e9 if corr_ms > 0 else None
    traffic = traffic_from_profile()
    step_gbs = B_STEP * CELLS * args.steps / (t_ms * 1e-3) / 1e9 / 1  # per GPU
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": config_text(), "nx": NX, "ny": NY, "ns": NS, "order": ORDER,
                   "limiter": True, "interior_cells": CELLS,
                   "l2": "inputs larger than L2 (268 MB per field); no flush",
                   "parallelism": f"replicas x{world} (one grid per GPU)" if world > 1 else "single GPU"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     "traffic": traffic, "peak_source": f"{peak_kind} hbm_gbs",
                     "kernel": KERNEL_OF_FORM[chosen],
                     "bytes_per_launch": {"writes_faces": B_CORR_FACES * CELLS,
                                          "last_pass": B_CORR_LAST * CELLS},
                     "launch_ms": {"donor": ms[0] / max(n[0], 1),
                                   "corrective_writes_faces": ms[1] / max(n[1], 1),
                                   "corrective_last": ms[2] / max(n[2], 1)},
                     "step": {"bytes_per_cell_step": B_STEP, "achieved": step_gbs,
                              "frac": step_gbs / peak}},
        "gpu_launches": launches,
        "positivity": {"min": mn, "negative_cells": nneg},
        "form": chosen,
        "forms": {k: {"value": r["value"], "ms_per_step": r["t_ms"] / args.steps,
                      "rel_l2_vs_fp64": r["rel_l2_vs_fp64"], "max_abs_vs_fp64": r["max_abs_vs_fp64"],
                      "rel_l2_vs_fp64_end": r["rel_l2_vs_fp64_end"],
                      "max_abs_vs_fp64_end": r["max_abs_vs_fp64_end"],
                      "negative_cells": r["nneg"], "options": dict(FORMS)[k]}
                  for k, r in forms.items()},
    }
    line["config"]["form"] = chosen
    line["config"]["fp64_error_bound"] = (
        f"relative L2 <= {FP64_REL_L2_BOUND} against an FP64 run of the plain method after "
        f"{ACC_STEPS} steps from c0 (rel_l2_vs_fp64) and no negative cell; when no FP32 form "
        "meets it, the fastest form no less accurate than the plain FP32 method")
    line["fp64_bound_met"] = bound_met
    line["reference_column_rule_accuracy"] = {
        "steps": ACC_STEPS, "forms": ref_rule,
        "how": "the same forms and FP64 run with the reference's rule for the y faces of the "
               "x = 1 column (unwritten by vv.c:81-82: 0 on odd passes, the advective face on "
               "even ones); share_column_x1 = share of the squared error in that column"}
    line["fp64_sensitivity_floor"] = {
        "rel_l2": floor[0], "max_abs": floor[1], "steps": ACC_STEPS,
        "how": "FP64 run from c0 perturbed by a seeded relative +-2^-24 (half an FP32 ulp) "
               "per cell, against the unperturbed FP64 run"}
    if clk:
        line["clocks"] = clk
    if e2e:
        line["e2e"] = e2e
    if ens:
        line["ensemble"] = ens
    if tdep is not None:
        line["time_dependent"] = tdep
    if adj:
        line["adjoint"] = adj
    if world == 1 and not args.no_cpu:
        cb = cpu_reference(steps=2, warmup=1)
        if cb:
            line["cpu_baseline"] = cb
    return line


def run_ensemble(m, torch, steps: int, base_steps: int):
    """Batched-ensemble configuration: 256 independent 2D instances (NX, NY in
    [64, 512]), IORD 2 + limiter, FP32 with hardware-reciprocal ratios (the
    headline form), one persistent launch per step (pass 0 formed inside the
    corrective pass) replayed as a CUDA graph with the autotuned tile shape,
    clocks sampled over the timed region; against the same instances
    stepped one after another through per-instance solvers (nx x ny x 3 form,
    256 sequential solver steps per ensemble step).  Both timed with CUDA
    events on one stream."""
    from mpdata_b200 import workloads
    cfg = workloads.ensemble()
    nx = [d["nx"] for d in cfg]
    ny = [d["ny"] for d in cfg]
    cells = sum((a - 2) * (b - 2) for a, b in zip(nx, ny))
    stream = torch.cuda.Stream()  # graph capture needs a non-default stream
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    e = m.Ensemble(nx, ny, order=2, limiter=True, approx_div=True)
    e.set_stream(stream.cuda_stream)
    for q, d in enumerate(cfg):
        e.set_faces(q, f32(d["U"]), f32(d["V"]))
        e.set_field(q, f32(d["c0"]))
    tile, tune_ms = e.autotune(trial_steps=5)
    for q, d in enumerate(cfg):
        e.set_field(q, f32(d["c0"]))
    e.step(steps)  # captures the graph (and warms up)
    for q, d in enumerate(cfg):
        e.set_field(q, f32(d["c0"]))
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    e0.record(stream)
    e.step(steps)
    e1.record(stream)
    e1.synchronize()
    clk = clocks.stop()
    t_ens = e0.elapsed_time(e1)
    mins = [float(e.get_field(q)[1:-1, 1:-1].min()) for q in range(len(cfg))]
    e.close()
    # per-instance baseline
    solvers = []
    for d in cfg:
        s = m.Solver(d["nx"], d["ny"], 3, order=2, limiter=True, approx_div=True)
        s.set_stream(stream.cuda_stream)
        U = np.zeros((3, d["ny"], d["nx"]), np.float32); V = np.zeros_like(U)
        U[1] = d["U"]; V[1] = d["V"]
        s.set_faces(U, V, np.zeros_like(U))
        s.set_field(np.repeat(f32(d["c0"])[None], 3, 0))
        solvers.append(s)
    for s in solvers:
        s.step(1)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(base_steps):
        for s in solvers:
            s.step(1)
    e1.record(stream)
    e1.synchronize()
    t_seq = e0.elapsed_time(e1)
    for s in solvers:
        s.close()
    ens_rate = cells * steps / (t_ens * 1e-3) / 1e9
    seq_rate = cells * base_steps / (t_seq * 1e-3) / 1e9
    peak, peak_kind = hbm_peak()
    ens_gbs = ens_rate * B_ENSEMBLE  # Gcell-steps/s x bytes per cell-step = GB/s
    return {"value": ens_rate, "unit": UNIT, "instances": len(cfg), "steps": steps,
            "interior_cells_per_step": cells, "ms_per_step": t_ens / steps,
            "tile": list(m.Ensemble.TILES[tile]),
            "kernel": "y-march (warp per 32-column strip)" if tile == m.Ensemble.MARCH
                      else "tile kernel", "autotune_ms_per_step": tune_ms,
            "sequential": {"value": seq_rate, "steps": base_steps,
                           "ms_per_step": t_seq / base_steps,
                           "how": "256 per-instance solvers (nx x ny x 3), stepped one after another"},
            "speedup_vs_sequential": ens_rate / seq_rate,
            "clocks": clk,
            "roofline": {"bound": "hbm", "bytes_per_cell_step": B_ENSEMBLE,
                         "achieved": ens_gbs, "peak": peak, "unit": "GB/s",
                         "frac": ens_gbs / peak, "peak_source": f"{peak_kind} hbm_gbs",
                         "fused_bytes_per_cell_step": B_ENSEMBLE_FUSED,
                         "frac_of_fused_bytes": ens_rate * B_ENSEMBLE_FUSED / peak,
                         "note": "whole step; bytes_per_cell_step counts the donor and "
                                 "corrective passes separately, fused_bytes_per_cell_step the "
                                 "one fused launch (c^(1) stays on chip); the arena partly "
                                 "fits in the 126 MB L2"},
            "min_interior_value": min(mins)}


def run_adjoint(m, torch, nsteps: int = 200, every: int = 20, ndir: int = 32):
    """Adjoint source-inversion configuration: 128x128x64, ring3d-type flow,
    IORD 2 + limiter (branches frozen), FP32 forward and adjoint, window of
    200 steps with a checkpoint every 20, loss = sum of squared differences at
    64 seeded receptors against a target from a different blob.  Reports the
    reverse sweep's cost per step against a forward step (the fused
    production step and the recording forward the adjoint replays), and the
    agreement of the FP32 and FP64 adjoints with FP64 central differences
    along 32 random directions, and of the FP32 adjoint with the FP64 one."""
    import mpdata_b200.adjoint as ma
    from mpdata_b200 import workloads
    n, ns = 128, 64
    r = workloads.ring3d(n=n, ns=ns, courant=0.4, wcourant=0.1, sigma=6.0, offset=30.0,
                         background=1e-6)
    tr = workloads.ring3d(n=n, ns=ns, courant=0.4, wcourant=0.1, sigma=8.0, offset=-25.0,
                          background=1e-6)["c0"]
    faces = workloads.faces_from_cells(r["u"], r["v"], r["w"])
    k, j, i = np.mgrid[0:ns, 0:n, 0:n].astype(np.float64)
    # smoothly varying background: no exactly uniform region (where the
    # limiter ratio is 0/0 and the frozen-branch derivative is not defined)
    c0 = r["c0"] + 1e-4 * (1.5 + np.sin(0.3 * i) * np.cos(0.25 * j + 0.2 * k))
    rng = np.random.default_rng(workloads.SEED + 5)
    rec = rng.integers(0, c0.size, 64)
    t_rec = tr.reshape(-1)[rec]

    def lam_of(cN):
        lam = np.zeros(c0.size)
        np.add.at(lam, rec, 2.0 * (cN.reshape(-1)[rec] - t_rec))
        return lam.reshape(c0.shape)

    def loss_of(cN):
        return float(np.sum((cN.reshape(-1)[rec] - t_rec) ** 2))

    out = {"grid": [n, n, ns], "steps": nsteps, "checkpoint_every": every, "receptors": 64}
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.current_stream()
    grads, fwd = {}, {}
    for dt in (np.float32, np.float64):
        a = ma.Adjoint(n, n, ns, order=2, dtype=dt, checkpoint_every=every, limiter=True)
        a.set_stream(stream.cuda_stream)
        a.set_faces(*(np.ascontiguousarray(f, dt) for f in faces))
        cd = np.ascontiguousarray(c0, dt)
        a.forward(cd, nsteps)  # warm-up
        ev0.record(stream)
        cN = a.forward(cd, nsteps)
        ev1.record(stream)
        ev1.synchronize()
        t_f = ev0.elapsed_time(ev1)
        fwd[np.dtype(dt).name] = cN.astype(np.float64)
        lam = np.ascontiguousarray(lam_of(cN.astype(np.float64)), dt)
        ev0.record(stream)
        g = a.backward(lam)
        ev1.record(stream)
        ev1.synchronize()
        t_b = ev0.elapsed_time(ev1)
        grads[np.dtype(dt).name] = g.astype(np.float64)
        if dt is np.float32:
            out["t_fwd_recording_ms_per_step"] = t_f / nsteps
            out["t_adj_first_call_ms_per_step"] = t_b / nsteps
            # A second sweep of the same window: its segment graphs exist now
            # (the first call captures and instantiates them), so this is the
            # per-step cost of every later sweep.  The reverse scatter-adds are
            # atomic: it sums in another order.
            ev0.record(stream)
            g2 = a.backward(lam)
            ev1.record(stream)
            ev1.synchronize()
            out["t_adj_ms_per_step"] = ev0.elapsed_time(ev1) / nsteps
            g2 = g2.astype(np.float64)
            out["fp32_adjoint_run_to_run_rel_l2"] = float(
                np.linalg.norm(g2 - grads["float32"]) / np.linalg.norm(grads["float32"]))
        else:
            # the FP64 adjoint's own sensitivity: the same window (same seed
            # lambda) from c0 perturbed per cell by half an FP32 ulp (one
            # rounding) and by 2^-20 (the FP32 forward's distance from the FP64
            # one after the 200 steps)
            lam64 = np.ascontiguousarray(lam_of(cN.astype(np.float64)))
            for key, amp in (("half_ulp", 2.0 ** -24), ("2^-20", 2.0 ** -20)):
                rng_p = np.random.default_rng(11)
                cp = c0 * (1.0 + rng_p.uniform(-amp, amp, c0.shape))
                a.forward(np.ascontiguousarray(cp), nsteps)
                gp = a.backward(lam64).astype(np.float64)
                out[f"fp64_adjoint_sensitivity_{key}_rel_l2"] = float(
                    np.linalg.norm(gp - grads["float64"]) / np.linalg.norm(grads["float64"]))
        a.close()
    # production forward step (fused kernels) on the same problem
    s = m.Solver(n, n, ns, order=2, limiter=True)
    s.set_stream(stream.cuda_stream)
    s.set_faces(*(np.ascontiguousarray(f, np.float32) for f in faces))
    s.set_field(np.ascontiguousarray(c0, np.float32))
    s.step(5)
    ev0.record(stream)
    s.step(nsteps)
    ev1.record(stream)
    ev1.synchronize()
    out["t_fwd_fused_ms_per_step"] = ev0.elapsed_time(ev1) / nsteps
    s.close()
    out["t_adj_over_t_fwd_fused"] = out["t_adj_ms_per_step"] / out["t_fwd_fused_ms_per_step"]
    out["t_adj_over_t_fwd_recording"] = out["t_adj_ms_per_step"] / out["t_fwd_recording_ms_per_step"]
    g32, g64 = grads["float32"], grads["float64"]
    out["fp32_vs_fp64_adjoint_rel_l2"] = float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64))
    out["fp32_vs_fp64_forward_rel_l2"] = float(
        np.linalg.norm(fwd["float32"] - fwd["float64"]) / np.linalg.norm(fwd["float64"]))
    # central differences of the FP64 window along random directions
    a64 = ma.Adjoint(n, n, ns, order=2, dtype=np.float64, checkpoint_every=every, limiter=True)
    a64.set_faces(*(np.ascontiguousarray(f, np.float64) for f in faces))
    errs, errs64 = [], []
    # The step is piecewise smooth (the limiter's min / max selections): the
    # difference step must be small enough that few selections switch inside
    # it (relative perturbation 1e-8 of c0; FP64 rounding stays near 1e-8).
    for _ in range(ndir):
        v = rng.standard_normal(c0.shape) * c0 * 1e-3
        e = 1e-5
        lp = loss_of(a64.forward(np.ascontiguousarray(c0 + e * v), nsteps))
        lm = loss_of(a64.forward(np.ascontiguousarray(c0 - e * v), nsteps))
        fd = (lp - lm) / (2 * e)
        errs.append(abs(fd - float(np.sum(g32 * v))) / max(abs(fd), 1e-30))
        errs64.append(abs(fd - float(np.sum(g64 * v))) / max(abs(fd), 1e-30))
    a64.close()
    out["fd_directions"] = ndir
    out["fd_max_rel_err_fp64_adjoint"] = max(errs64)
    out["fd_median_rel_err_fp64_adjoint"] = float(np.median(errs64))
    out["fd_max_rel_err_fp32_adjoint"] = max(errs)
    out["fd_median_rel_err_fp32_adjoint"] = float(np.median(errs))
    return out


def run_time_dependent(m, torch, form_opts, steps: int = 20):
    """The throughput workload with a velocity update before every step
    (mpdata_set_velocity lending device arrays, then one step): the update's
    face Courant numbers are formed by that step's donor pass in one march,
    which reads the velocities in place.
    Velocities alternate between two seeded fields so each step really gets
    new faces.  Reported beside the steady-flow step of the same solver."""
    wl = _workload()
    u, v, w = _workloads_module().cell_velocities(wl["U"], wl["V"], wl["W"])
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    vel = [[dev(u), dev(v), dev(w)], [dev(0.9 * u), dev(0.9 * v), dev(0.9 * w)]]
    dxyz = [dev(np.ones(n, np.float32)) for n in (NX, NY, NS)]
    stream = torch.cuda.current_stream()
    s = m.Solver(NX, NY, NS, order=ORDER, limiter=True, **WORKLOAD_OPTS, **form_opts)
    try:
        s.set_stream(stream.cuda_stream)
        s.set_field(wl["c0"])

        def update(q):
            a = vel[q & 1]
            s.set_velocity(*dxyz, 1.0, a[0], a[0], a[1], a[1], a[2], a[2], borrow=True)

        for q in range(3):
            update(q)
            s.step(1)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for q in range(steps):
            update(q)
            s.step(1)
        e1.record(stream)
        e1.synchronize()
        t_upd = e0.elapsed_time(e1) / steps
        e0.record(stream)
        s.step(steps)
        e1.record(stream)
        e1.synchronize()
        t_steady = e0.elapsed_time(e1) / steps
    finally:
        s.close()
    return {"value": CELLS / (t_upd * 1e-3) / 1e9, "unit": UNIT, "steps": steps,
            "ms_per_step": t_upd, "steady_ms_per_step": t_steady,
            "how": "set_velocity (3 distinct device arrays lent, read in place) + step(1) "
                   "per step; faces formed in the step's donor pass"}


def run_e2e(m, args, form_opts):
    """Same workload through smolar() (the drop-in entry point) with pinned
    host arrays; per step: upload of the 3 distinct velocity arrays + field,
    download of the newest field and the previous level."""
    import ctypes as C

    wl = _workload()
    u, v, w = _workloads_module().cell_velocities(wl["U"], wl["V"], wl["W"])

    def pinned(a):
        p = m.library().mpdata_host_alloc(a.nbytes)
        if not p:
            raise MemoryError("pinned allocation failed")
        buf = np.ctypeslib.as_array((C.c_float * a.size).from_address(p)).reshape(a.shape)
        buf[...] = a
        return buf, p

    bufs = [pinned(x) for x in (u, v, w, wl["c0"], np.zeros_like(wl["c0"]))]
    hu, hv, hw, c0, c1 = (b for b, _ in bufs)
    dx = np.ones(NX, np.float32); dy = np.ones(NY, np.float32); ds = np.ones(NS, np.float32)
    m.set_default_options(m.SolverOptions(limiter=True, **WORKLOAD_OPTS, **form_opts))
    steps = max(1, min(args.steps, args.e2e_steps))
    try:
        for it in range(2 + steps):
            if it == 2:
                t0 = time.perf_counter()
            a, b = m.smolar(NX, NY, NS, dx, dy, ds, 1.0, hu, hu, hv, hv, hw, hw, c0, c1,
                            order=ORDER)
            c0, c1 = b, a  # driver exchange (reference tests/ring2d/test.c:104-105)
        dt = time.perf_counter() - t0
    finally:
        m.set_default_options(None)
        for _, p in bufs:
            m.library().mpdata_host_free(C.c_void_p(p))
    h2d = 4 * FIELD_BYTES + (NX + NY + NS) * 4
    d2h = 2 * FIELD_BYTES
    floor_ms = copy_floor_ms(h2d, d2h)
    value = CELLS * steps / dt / 1e9
    bound = CELLS / (floor_ms * 1e-3) / 1e9
    return {"value": value, "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "steps": steps,
            "api": "smolar() C ABI, pinned host buffers, wall clock",
            "copy_floor_ms": floor_ms, "copy_bound": bound, "frac_of_copy_bound": value / bound,
            "copy_floor_how": "the step's host->device and device->host bytes as two plain "
                              "pinned-memory copies on two streams at once (best of 3)"}


def copy_floor_ms(h2d_bytes, d2h_bytes, reps=3):
    """Wall time of the step's transfers alone: one pinned host->device copy of
    h2d_bytes and one device->host copy of d2h_bytes, concurrent (full-duplex
    PCIe), best of `reps` -- the lower bound of a host-array step."""
    import torch
    n_up, n_down = h2d_bytes // 4, d2h_bytes // 4
    hu = torch.empty(n_up, dtype=torch.float32, pin_memory=True)
    hd = torch.empty(n_down, dtype=torch.float32, pin_memory=True)
    du = torch.empty(n_up, dtype=torch.float32, device="cuda")
    dd = torch.zeros(n_down, dtype=torch.float32, device="cuda")
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    best = float("inf")
    for _ in range(reps):
        torch.cuda.synchronize()
        t = time.perf_counter()
        with torch.cuda.stream(s1):
            du.copy_(hu, non_blocking=True)
        with torch.cuda.stream(s2):
            hd.copy_(dd, non_blocking=True)
        torch.cuda.synchronize()
        best = min(best, time.perf_counter() - t)
    del hu, hd, du, dd
    return best * 1e3


ACC_MARKS = (10, 25, 50, 100)


def error_breakdown(a, ref, nref, ref_interior=None):
    """Relative L2 / max-abs of a against ref, and where the error sits:
    the share of the squared error carried by the largest 0.01 %, 0.1 % and
    1 % of the per-cell errors."""
    e3 = np.abs(a.astype(np.float64) - ref)
    e = e3.ravel()
    tot = float(np.dot(e, e))
    x1 = float(np.sum(e3[:, :, 1] ** 2))
    inner = e3[:, :, 3:]
    out = {"rel_l2": float(np.sqrt(tot)) / nref, "max_abs": float(e.max()),
           "negative_cells": int(np.count_nonzero(a < 0)),
           "share_column_x1": x1 / tot if tot > 0 else 0.0,
           "rel_l2_without_x_le_2": float(np.sqrt(np.sum(inner ** 2))) / nref}
    for frac in (1e-4, 1e-3, 1e-2):
        k = max(1, int(e.size * frac))
        top = np.partition(e, e.size - k)[e.size - k:]
        out[f"share_top_{frac:g}"] = float(np.dot(top, top)) / tot if tot > 0 else 0.0
    return out, e


def local_extremum(c, flat_idx):
    """Whether each cell (flat indices into the full grid) is >= or <= all six
    face neighbours; shell cells count as not."""
    ns, ny, nx = c.shape
    k, j, i = np.unravel_index(flat_idx, c.shape)
    inner = (i > 0) & (i < nx - 1) & (j > 0) & (j < ny - 1) & (k > 0) & (k < ns - 1)
    k, j, i = k[inner], j[inner], i[inner]
    v = c[k, j, i]
    nb = np.stack([c[k, j, i - 1], c[k, j, i + 1], c[k, j - 1, i], c[k, j + 1, i],
                   c[k - 1, j, i], c[k + 1, j, i]])
    ext = np.zeros(flat_idx.shape, bool)
    ext[inner] = (v >= nb.max(0)) | (v <= nb.min(0))
    return ext


def run_accuracy(args):
    """--accuracy: the FP32 forms' error against an FP64 run of the plain
    method over the configuration's 100 steps (at steps 10, 25, 50, 100), next
    to the FP64 scheme's own sensitivity (FP64 from a half-ulp-perturbed c0;
    FP64 with the field rounded to FP32 after every step; FP64 without the
    limiter from the perturbed c0), with the error's concentration in few
    cells and whether those cells are local extrema of the FP64 field."""
    import torch
    import mpdata_b200 as m
    torch.cuda.set_device(0)
    wl = _workload()
    stream = torch.cuda.current_stream()

    def run(dtype, c0, limiter=True, round_each=False, vv_fix=False, **opts):
        s = m.Solver(NX, NY, NS, order=ORDER, dtype=dtype, limiter=limiter, vv_fix=vv_fix,
                     **opts)
        s.set_stream(stream.cuda_stream)
        s.set_faces(*(np.ascontiguousarray(wl[k], dtype) for k in ("U", "V", "W")))
        s.set_field(np.ascontiguousarray(c0, dtype))
        done = 0
        try:
            for mk in ACC_MARKS:
                if round_each:
                    for _ in range(mk - done):
                        s.step(1)
                        s.set_field(s.get_field().astype(np.float32).astype(np.float64))
                else:
                    s.step(mk - done)
                done = mk
                yield mk, s.get_field()
        finally:
            s.close()

    c0 = wl["c0"].astype(np.float64)
    # references by (limiter, column rule): vv_fix computes the y faces of the
    # x = 1 column (vv.c:81-82 leaves them unwritten)
    refs = {(True, False): {mk: f for mk, f in run(np.float64, c0)},
            (False, False): {mk: f for mk, f in run(np.float64, c0, limiter=False)},
            (True, True): {mk: f for mk, f in run(np.float64, c0, vv_fix=True)}}
    norms = {key: {mk: float(np.linalg.norm(f)) for mk, f in r.items()} for key, r in refs.items()}
    pert = half_ulp_perturbed(wl["c0"])
    cases = [("fp64_half_ulp_perturbed_c0", dict(dtype=np.float64, c0=pert)),
             ("fp64_rounded_to_fp32_each_step", dict(dtype=np.float64, c0=c0, round_each=True)),
             ("fp64_no_limiter_half_ulp_perturbed_c0",
              dict(dtype=np.float64, c0=pert, limiter=False)),
             ("fp64_vv_fix_half_ulp_perturbed_c0", dict(dtype=np.float64, c0=pert, vv_fix=True))]
    cases += [(f"fp32_{name}", dict(dtype=np.float32, c0=wl["c0"], **o)) for name, o in FORMS]
    cases += [(f"fp32_vv_fix_{name}", dict(dtype=np.float32, c0=wl["c0"], vv_fix=True, **o))
              for name, o in FORMS]
    rng = np.random.default_rng(3)
    sample = rng.integers(0, c0.size, 1_000_000)
    out = {"workload": config_text(), "steps": list(ACC_MARKS),
           "reference": "FP64 run of the plain method (IEEE division), same limiter setting",
           "local_extremum_fraction_all_cells": float(
               local_extremum(refs[(True, False)][ACC_MARKS[-1]], sample).mean()),
           "cases": {}}
    for name, kw in cases:
        key = (kw.get("limiter", True), kw.get("vv_fix", False))
        res = {}
        for mk, f in run(**kw):
            b, e = error_breakdown(f, refs[key][mk], norms[key][mk])
            if mk == ACC_MARKS[-1]:
                k = max(1, int(e.size * 1e-4))
                hot = np.argpartition(e, e.size - k)[e.size - k:]
                b["top_0.0001_local_extremum_fraction"] = float(
                    local_extremum(refs[key][mk], hot).mean())
            res[mk] = b
        out["cases"][name] = res
        print(json.dumps({name: res}), file=sys.stderr, flush=True)
    return out


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return None
    cb = cpu_reference(steps=args.steps, warmup=args.warmup)
    if cb is None:
        return {"impl": "reference",
                "unavailable": "reference build oracle/_ref/libref_f32_fast.so missing"}
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": cb["seconds"] / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": (f"{cb['instances']} x independent "
                                    f"{'x'.join(str(v) for v in cb['slab'])} z-slabs of the "
                                    f"{NX}x{NY}x{NS} roofline grid, IORD {ORDER}, no limiter "
                                    "(the reference has none), one host thread per slab"),
                       "nx": cb["slab"][0], "ny": cb["slab"][1], "ns": cb["slab"][2],
                       "instances": cb["instances"], "order": ORDER, "limiter": False,
                       "metric_cells": "interior cells of the slabs"},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "gpu_launches": 0}
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-time-dependent", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--ensemble-steps", type=int, default=500)
    ap.add_argument("--acc-steps", type=int, default=None,
                    help="horizon of the FP64 accuracy check (default: the configuration's "
                         "100 steps; shorter only for profiling captures)")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="run only the adjoint configuration")
    ap.add_argument("--adjoint-directions", type=int, default=32,
                    help="finite-difference directions of the adjoint check")
    ap.add_argument("--ensemble-only", action="store_true",
                    help="run only the batched-ensemble configuration")
    ap.add_argument("--accuracy", action="store_true",
                    help="print the FP64 error breakdown of the FP32 forms (no timing)")
    ap.add_argument("--size", default=None,
                    help="nx,ny,ns override (profiling captures of a smaller grid only)")
    ap.add_argument("--kernel", type=int, default=None, choices=sorted(KERNEL_CHOICES),
                    help="force the solver's corrective-pass kernel on the timed forms "
                         "(profiling captures of the other kernels; default: the solver's choice)")
    ap.add_argument("--check-courant", action="store_true",
                    help="the timed forms run with the Courant check (profiling captures of "
                         "its kernels)")
    args = ap.parse_args()
    if args.check_courant:
        _add_form_options(check_courant=True)
    if args.size:
        _set_size(*(int(v) for v in args.size.split(",")))
    if args.kernel is not None:
        _set_kernel(args.kernel)
    if args.acc_steps:
        global ACC_STEPS
        ACC_STEPS = args.acc_steps
    if args.warmup < 3 and args.impl == "b200":
        args.warmup = 3
    if args.accuracy:
        print(json.dumps(run_accuracy(args)), flush=True)
        return
    if args.adjoint_only:  # the adjoint configuration alone (profiling captures)
        import torch
        import mpdata_b200 as m
        torch.cuda.set_device(0)
        print(json.dumps(run_adjoint(m, torch, ndir=args.adjoint_directions)), flush=True)
        return
    if args.ensemble_only:  # the batched-ensemble configuration alone (profiling captures)
        import torch
        import mpdata_b200 as m
        torch.cuda.set_device(0)
        print(json.dumps(run_ensemble(m, torch, args.ensemble_steps, 2)), flush=True)
        return
    line = run_reference(args) if args.impl == "reference" else run_gpu(args)
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
