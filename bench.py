#!/usr/bin/env python
"""Benchmark: D32 oscillating-sphere steps/s on B200 (and the CPU reference arm).

Workload: the D = 32 oscillating sphere -- three nested levels (half widths
2D, 4D, 8D: a 16D cube of 5,767,168 cells, 17,548,032 edges), A = 0.2 D,
Re0 = 0.2, omega = 3.6, 200 steps per period, 3217 Fibonacci markers, closed
no-slip cavity, float64.  A step is one ``Driver.step`` (4 Picard passes, each
with a PCG solve to the reference's mixed 1e-10/1e-9 criterion checked every
20 iterations).  Data are synthetic (the analytic sphere and its prescribed
motion); nothing is read from disk.

``value``    steps/s from CUDA events on the library stream over K steps,
             fields resident in HBM (the prescribed marker positions of each
             step, 154 KB, are its only host input).
``e2e``      the same K steps through the public driver API (``SphereRun.advance``)
             with the marker positions uploaded and the body load read back
             every step, host wall clock.
``roofline`` the PCG iteration: 80 algorithmic bytes per edge per iteration
             (10 float64 edge streams) over its CUDA-event time, against the
             measured HBM copy bandwidth.
``cpu_baseline`` / ``--impl reference``: the NumPy restatement of the
             reference's CPU path (oracle/) timed on the host on a bounded
             sample (see ``reference_sample``).

Multi-GPU: a single case does not shard (every CG iteration has global
reductions); ``--gpus N`` under torchrun runs N independent replicas with no
collective on the data path and reports the sum of their throughputs.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

ALGO_BYTES_PER_EDGE_ITER = 80.0     # 10 float64 edge streams per PCG iteration
ALGO_BYTES_PER_EDGE_MATVEC = 16.0   # read p, write w


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def matvec_plan(sv):
    """The autotuner's matvec plan: per precision, whether it ran, the cell- and
    node-tile z depths, and whether curl+interp and viscous run as one kernel."""
    out = (C.c_int32 * 8)()
    sv.h.call("pyib_matvec_plan", out)
    plan = {}
    for q, name in enumerate(("float64", "float32")):
        t, kz, kzr, av = (int(x) for x in out[4 * q:4 * q + 4])
        if t:
            plan[name] = {"cell_tile": [32, 8, kz], "node_tile": [32, 8, kzr], "curl_interp_viscous_fused": bool(av)}
    return plan


def matvec_kernel_ms(mv, fused_av):
    """Per-kernel times of pyib_bench_matvec (slots 1..6) under the kernels' names."""
    if fused_av:
        names = ["curl_interp_viscous", "curl_interp_patch", None, "viscous_patch", "integr_rot_dot",
                 "integr_rot_patch_reduce"]
    else:
        names = ["curl_interp", "curl_interp_patch", "viscous", "viscous_patch", "integr_rot_dot",
                 "integr_rot_patch_reduce"]
    return {n: float(x) for n, x in zip(names, list(mv)[1:7]) if n is not None}


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def maybe_init_dist(world, local, backend="nccl"):
    if world <= 1:
        return None
    import datetime

    import torch
    import torch.distributed as dist
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
    return dist


def _reduce_device(dist):
    """NCCL reduces CUDA tensors, gloo host tensors."""
    import torch
    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def reduce_max(dist, value):
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=_reduce_device(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(dist, value):
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=_reduce_device(dist))
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


# ---------------------------------------------------------------------------
# CPU reference arm: the oracle (NumPy restatement of the reference CPU path)
# ---------------------------------------------------------------------------
def cpu_info():
    """Host threads this process may use and the CPU model name (/proc/cpuinfo)."""
    model = "unknown"
    try:
        for ln in Path("/proc/cpuinfo").read_text().splitlines():
            if ln.startswith("model name"):
                model = ln.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return cores_used(), model


def committed_iterations_per_step(case):
    """CG iterations per step of ``case`` from the committed bench record, if any."""
    f = ROOT / "profiles" / f"bench_{case.name.split('_')[0]}_float64.json"
    try:
        return float(json.loads(f.read_text().splitlines()[0])["config"]["cg_iterations_per_step"]), f.name
    except (OSError, ValueError, KeyError, IndexError):
        return D32_ITERS_PER_STEP, "bench.D32_ITERS_PER_STEP"


class ReferenceSample:
    """The oracle -- the reference's CPU algorithm restated in NumPy -- on the FULL layout.

    Setup builds the workload's own mesh description (the layout's export in the
    reference's conventions) and the oracle driver on it: the unstructured
    incidence operators with ``bincount`` reductions of ``ib_core_np.py``.  Then:

    * ``time_ops`` times one ``calc_vel``, one ``conv_diff`` and one
      ``rot(integr_c2f(.))`` and weights them by their calls per step in
      ``Driver.step`` (6, 5 and 4, ``ib_driver_np.py:412-532``);
    * ``time_iterations`` runs real PCG iterations of ``helm_solve``'s recurrence
      (``ib_driver_np.py:386-403``: w = A p masked, alpha = eta / p.w, x and r
      updates, z = prec r, beta = eta' / eta) on a residual of the step's form,
      once with the default BLAS threads and once limited to one thread.

    A full step needs its CG iteration count of such iterations (about 19,400 at
    D = 32: 37 CPU hours), so steps/s is the measured per-operation times times
    that count: an extrapolation of measured full-size work, labelled as such.
    """

    def __init__(self, case):
        sys.path.insert(0, str(ROOT / "oracle"))
        import pyib_oracle as O
        t0 = time.perf_counter()
        lay = case.layout().build()
        desc, _ = lay.export_mesh()
        self.m = O.MeshDesc(**desc)
        self.drv = O.OracleDriver(self.m, case.viscosity, case.density, cavity=case.cavity)
        self.setup_s = time.perf_counter() - t0
        self.dt = case.time_step
        self.ne = self.m.E2N.shape[0]
        self.nc = self.m.ncell
        rng = np.random.default_rng(0)
        self.s = rng.standard_normal(self.ne) * 1e-3
        drv = self.drv
        _, _, vc = drv.calc_vel(self.s)
        res = drv.g.rot(drv.g.integr_c2f(vc[:self.nc] * 0.01))
        self.r = np.where(drv.dir_mask, 0.0, res)
        self.x = self.s.copy()
        self.p = self.r * drv.prec
        self.eta = float(self.p.dot(self.r))

    def time_ops(self):
        drv = self.drv
        t0 = time.perf_counter()
        _, U, vc = drv.calc_vel(self.s)
        t1 = time.perf_counter()
        drv.conv_diff(U, vc)
        t2 = time.perf_counter()
        drv.g.rot(drv.g.integr_c2f(vc[:self.nc]))
        t3 = time.perf_counter()
        self.ops = {"calc_vel": t1 - t0, "conv_diff": t2 - t1, "rot_integr": t3 - t2}
        return 6 * (t1 - t0) + 5 * (t2 - t1) + 4 * (t3 - t2)

    def iteration(self):
        drv = self.drv
        w = drv.apply(self.p, self.dt)
        w[drv.dir_mask] = 0.0
        den = self.p.dot(w)
        alf = self.eta / (den if den != 0.0 else np.inf)
        self.x += alf * self.p
        self.r -= alf * w
        z = self.r * drv.prec
        eta_new = float(z.dot(self.r))
        beta = eta_new / (self.eta if self.eta != 0.0 else np.inf)
        self.p = z + beta * self.p
        self.eta = eta_new

    def time_iterations(self, n, single_thread=False):
        from contextlib import nullcontext
        ctx = nullcontext()
        if single_thread:
            from threadpoolctl import threadpool_limits
            ctx = threadpool_limits(limits=1)
        with ctx:
            t0 = time.perf_counter()
            for _ in range(n):
                self.iteration()
            return (time.perf_counter() - t0) / n


def reference_sample(case, iters_per_step, iters_source, sample=None, n_iter=1):
    """One bounded sample of the reference's step at full size; returns (steps/s, details)."""
    rs = sample if sample is not None else ReferenceSample(case)
    t_ops = rs.time_ops()
    t_it = rs.time_iterations(n_iter)
    t_it1 = rs.time_iterations(n_iter, single_thread=True)
    cores, model = cpu_info()
    det = {
        "t_ops_per_step_s": t_ops, "ops_s": rs.ops, "t_iteration_s": t_it,
        "t_iteration_single_thread_s": t_it1, "cg_iterations_per_step": iters_per_step,
        "cg_iterations_source": iters_source, "setup_s": rs.setup_s, "cores": cores, "cpu_model": model,
        "value_single_thread": 1.0 / (t_ops + iters_per_step * t_it1), "extrapolated": True,
        "sample": (f"oracle on the full layout ({rs.nc} cells, {rs.ne} edges): one calc_vel, conv_diff and "
                   f"rot(integr_c2f) weighted 6/5/4 per step = {t_ops:.2f} s, {n_iter} PCG iteration(s) of the "
                   f"reference recurrence at {t_it:.2f} s each ({t_it1:.2f} s with one BLAS thread), times "
                   f"{iters_per_step:.0f} CG iterations per step ({iters_source})"),
    }
    return 1.0 / (t_ops + iters_per_step * t_it), det


def full_edge_count(case):
    """Existing edges of a concentric nested layout (closed form, no tables).

    A level box of n^3 cells has 3 n (n+1)^2 edges; the edges of the closed
    hole box (m = n_inner / 2 cells a side) are absent (inside the hole) or
    belong to the finer level (on the hole surface).
    """
    n = [int(round(2 * w * case.cells_per_diameter / 2 ** L)) for L, w in enumerate(case.half_widths_d)]
    tot = 0
    for L, nL in enumerate(n):
        tot += 3 * nL * (nL + 1) ** 2
        if L > 0:
            m = n[L - 1] // 2
            tot -= 3 * m * (m + 1) ** 2
    return tot


def cores_used():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# D32 float64 CG iterations per step (all four Picard passes) after the three
# warm-up steps, measured by the b200 arm (19,450 on steps 4-5); the oracle
# follows the same iterates (the parity tests match iteration counts).
D32_ITERS_PER_STEP = 19450.0


def full_cell_count(case):
    """Existing cells of a concentric nested layout: n^3 per level minus its hole."""
    n = [int(round(2 * w * case.cells_per_diameter / 2 ** L)) for L, w in enumerate(case.half_widths_d)]
    return sum(nL ** 3 - ((n[L - 1] // 2) ** 3 if L > 0 else 0) for L, nL in enumerate(n))


def run_reference(args, world, rank):
    """The reference arm: the reference's CPU algorithm (the oracle port) on this host.

    Rank 0 alone works.  Setup builds the oracle on the full workload layout; each
    warm-up and timed step is one bounded sample (``reference_sample``): the step's
    operators and one real PCG iteration at full size, scaled to the step's CG
    iteration count, which is labelled ``extrapolated`` in the line.
    """
    import _pyib_b200_import
    _pyib_b200_import.load()
    from pyib_b200.cases import CASES
    case = CASES[args.workload]
    if rank != 0:
        return 0
    t_run = time.perf_counter()
    iters, source = committed_iterations_per_step(case)
    rs = ReferenceSample(case)
    vals, vals1, det = [], [], {}
    for k in range(args.warmup + args.steps):
        v, det = reference_sample(case, iters, source, sample=rs)
        if k >= args.warmup:
            vals.append(v)
            vals1.append(det["value_single_thread"])
    value = float(np.mean(vals))
    cores, model = cpu_info()
    markers = int(case.markers()[0].shape[0])
    det["value_single_thread"] = float(np.mean(vals1))
    det["timed_seconds"] = time.perf_counter() - t_run
    line = {
        "impl": "reference", "metric": "D32 sphere steps/s", "value": value, "unit": "steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 / value, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": case.name, "cells": full_cell_count(case), "edges": full_edge_count(case),
                   "levels": len(case.half_widths_d), "markers": markers, "precision": "float64",
                   "parallelism": "replicas1", "l2": "inputs larger than L2 (working set > 2 GB)",
                   "cg_iterations_per_step": iters},
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": cores, "kind": "port",
                         "sample": det["sample"], "cpu_model": model,
                         "value_one_blas_thread": det["value_single_thread"]},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "extrapolated": True, "reference_detail": det,
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def run_b200(args, world, rank, local):
    import _pyib_b200_import
    _pyib_b200_import.load()
    from pyib_b200 import _lib, build
    from pyib_b200.cases import CASES
    from pyib_b200.runner import SphereRun

    from pyib_b200.device import LayoutTables

    build.build_library()
    dist = maybe_init_dist(world, local)
    case = CASES[args.workload]
    t_setup = time.perf_counter()
    tables = LayoutTables(case.layout().build(), case.cavity)
    run = SphereRun(case, device=local if world > 1 else 0, precision=args.precision,
                    mixed_tol=args.mixed_tol, tables=tables)
    drv = run.drv
    sv = drv.solver
    setup_s = time.perf_counter() - t_setup
    for _ in range(args.warmup):
        run.advance()
    # the state entering the timed steps, so that the end-to-end leg repeats the same steps
    snap = dict(s=np.asarray(run.s).copy(), s_old=np.asarray(run.s_old).copy(), state=drv.ib_state_dict(),
                step=run.step_index, time=drv.time, loads=np.asarray(run.loads.current).copy())
    barrier(dist)
    sampler = ClockSampler(local if world > 1 else int(os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0] or 0))
    sampler.start()
    timing = (C.c_double * 5)()
    sv.h.call("pyib_cg_timing", timing, 1)
    iters = []
    ev_ms = C.c_double(0.0)
    sv.h.call("pyib_event", 0, None)
    for _ in range(args.steps):
        k = run.step_index + 1
        drv.time = (k - 1) * run.dt
        run.s, run.vc, run.s_old = drv.step(run.s, run.s_old, run.dt, run.dt, inner=4)
        drv.time = k * run.dt
        run.step_index = k
        iters.append(drv.helmholtz_total_iterations_last_step)
    sv.h.call("pyib_event", 1, C.byref(ev_ms))
    sv.h.call("pyib_cg_timing", timing, 1)
    cg_s, cg_it, launches = float(timing[0]), float(timing[1]), int(timing[2])
    tiles = matvec_plan(sv).get("float64", {})
    av = bool(tiles.get("curl_interp_viscous_fused", False))
    t_dev = ev_ms.value / 1000.0
    barrier(dist)
    # e2e: the same steps again from the same state, through the public API, with the
    # marker positions uploaded and the step's body load read back every step
    dev_state = dict(s=np.asarray(run.s).copy(), fE=np.asarray(drv.ib_force_E).copy())
    run.s, run.s_old = snap["s"].copy(), snap["s_old"].copy()
    drv.load_ib_state_dict(snap["state"])
    drv.ib_force_update_count = snap["state"]["force_update_count"]
    run.step_index, drv.time = snap["step"], snap["time"]
    run.loads.current = snap["loads"].copy()
    if run.motion is not None:
        mk, vel = run.motion(drv.time)
        drv.set_ib(drv.ib, mk, drv.ib_ds, vel)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        load = run.advance()
        _ = float(load["body_force"][0])
    t_e2e = time.perf_counter() - t0
    clocks = sampler.stop()
    # the repeated steps must reproduce the device-timed ones bit for bit
    e2e_same = bool(np.array_equal(np.asarray(run.s), dev_state["s"]) and
                    np.array_equal(np.asarray(drv.ib_force_E), dev_state["fE"]))
    # standalone matvec timing
    mv = (C.c_double * 7)()
    sv.set("WORK_E", np.random.default_rng(0).standard_normal(sv.lay.NE) * sv.lay.edge_exists)
    sv.h.call("pyib_bench_matvec", 50, C.c_double(run.dt), mv)
    mv_ms = C.c_double(mv[0])
    mv_kernels = matvec_kernel_ms(mv, av)
    mvf = (C.c_double * 6)()
    sv.h.call("pyib_bench_matvec_fused", 50, C.c_double(run.dt), mvf)
    mvf_kernels = dict(zip(["exact_vc_rows_and_list", "exact_vq_rows", "k_mvF", "exact_w_rows_dot"],
                           [float(x) for x in mvf[1:5]]))
    fused = os.environ.get("PYIB_FUSED_MATVEC", "0") == "1"
    ne = int(sv.lay.edge_exists.sum())
    t_dev_max = reduce_max(dist, t_dev)
    t_e2e_max = reduce_max(dist, t_e2e)
    total_steps = args.steps * world
    value = total_steps / t_dev_max
    e2e = total_steps / t_e2e_max
    peak, peak_kind = peaks()
    t_iter = cg_s / max(cg_it, 1.0)
    achieved = ALGO_BYTES_PER_EDGE_ITER * ne / t_iter / 1e9
    traffic = None
    tf = ROOT / "profiles" / "cg_iteration_d32_traffic.json"
    if tf.exists():
        d = json.loads(tf.read_text())
        traffic = d.get("bytes_per_edge_iteration", 0.0) * ne
    mv_achieved = ALGO_BYTES_PER_EDGE_MATVEC * ne / (mv_ms.value / 1e3) / 1e9
    mvf_achieved = ALGO_BYTES_PER_EDGE_MATVEC * ne / (float(mvf[0]) / 1e3) / 1e9
    M = drv.ib_markers.shape[0]
    mixed = None
    if world == 1 and args.precision == "float64" and not args.no_mixed:
        final = dict(U=sv.get("U"), vc=np.asarray(run.vc).copy(), fL=np.asarray(drv.ib_force_L).copy(),
                     force=np.asarray(run.loads.latest["body_force"]).copy())
        steps_done = run.step_index
        sv.h.close()
        mixed = mixed_leg(case, tables, args, steps_done, final)
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            v, det = reference_sample(case, float(np.mean(iters)),
                                      "this run's CG iterations per step on the GPU")
            cpu = {"value": v, "unit": "steps/s", "cores": det["cores"], "kind": "port",
                   "sample": det["sample"], "cpu_model": det["cpu_model"],
                   "value_one_blas_thread": det["value_single_thread"], "extrapolated": True}
        line = {
            "metric": "D32 sphere steps/s", "value": value, "unit": "steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * t_dev_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "cell_updates_per_s": value * int(sv.lay.cell_active.sum()),
            "config": {"workload": case.name, "cells": int(sv.lay.cell_active.sum()), "edges": ne,
                       "levels": sv.lay.N, "markers": M, "precision": args.precision,
                       "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (working set > 2 GB)",
                       "cg_iterations_per_step": float(np.mean(iters)), "setup_seconds": setup_s},
            "e2e": {"value": e2e, "unit": "steps/s", "h2d_bytes_per_step": 2 * 3 * M * 8,
                    "d2h_bytes_per_step": 13 * 8, "same_steps_as_value": e2e_same},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": ("PCG iteration (fused matvec k_mvF with its exact rows + update + direction)"
                                    if fused else
                                    "PCG iteration (matvec AV/RI + update + direction)" if av else
                                    "PCG iteration (matvec A/V/RI + update + direction)"),
                         "algorithmic_bytes_per_launch": ALGO_BYTES_PER_EDGE_ITER * ne,
                         "peak_kind": peak_kind},
            "matvec": {"fused": {"ms": float(mvf[0]), "achieved_gbs": mvf_achieved, "frac": mvf_achieved / peak,
                                 "kernel_ms": mvf_kernels, "node_planes_per_block": int(mvf[5])},
                       "tuned": {"ms": mv_ms.value, "achieved_gbs": mv_achieved, "frac": mv_achieved / peak,
                                 "form": "AV, RI" if av else "A, V, RI", "kernel_ms": mv_kernels},
                       "algorithmic_bytes": ALGO_BYTES_PER_EDGE_MATVEC * ne,
                       "used_by_cg": "fused" if fused else "tuned"},
            "cg": {"seconds": cg_s, "iterations": cg_it, "ms_per_iteration": 1e3 * t_iter,
                   "gbs": achieved},
            "gpu_launches": launches,
            "autotuned_tiles": tiles,
            "clocks": clocks,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        if mixed is not None:
            mixed["speedup_vs_float64"] = mixed["value"] / value
            line["mixed"] = mixed
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def run_matvec(args):
    """Standalone float64 matvec timings on a workload's layout (no time stepping).

    Prints one JSON line with the autotuned matvec (``pyib_bench_matvec``: curl+interp
    and viscous apart or fused, then integr+rot, whichever the tuner picked; pin one
    with PYIB_MATVEC_AV=0/1) and the single-pass fused matvec
    (``pyib_bench_matvec_fused``), each averaged over 50 calls with CUDA events, and
    their algorithmic HBM rates (16 B per edge).
    """
    import _pyib_b200_import
    _pyib_b200_import.load()
    from pyib_b200 import build
    from pyib_b200.cases import CASES
    from pyib_b200.device import DeviceSolver
    build.build_library()
    case = CASES[args.workload]
    lay = case.layout().build()
    sv = DeviceSolver(lay, rou=case.density, visc=case.viscosity, cavity=case.cavity)
    sv.set("WORK_E", np.random.default_rng(0).standard_normal(lay.NE) * lay.edge_exists)
    three = (C.c_double * 7)()
    sv.h.call("pyib_bench_matvec", 50, C.c_double(case.time_step), three)
    av = bool(matvec_plan(sv).get("float64", {}).get("curl_interp_viscous_fused", False))
    fused = (C.c_double * 6)()
    sv.h.call("pyib_bench_matvec_fused", 50, C.c_double(case.time_step), fused)
    ne = int(lay.edge_exists.sum())
    peak, peak_kind = peaks()
    gbs = lambda ms: ALGO_BYTES_PER_EDGE_MATVEC * ne / (ms / 1e3) / 1e9
    line = {"workload": case.name, "edges": ne, "cells": int(lay.cell_active.sum()),
            "tuned": {"ms": three[0], "gbs": gbs(three[0]), "form": "AV, RI" if av else "A, V, RI",
                      "kernel_ms": matvec_kernel_ms(three, av)},
            "fused": {"ms": fused[0], "gbs": gbs(fused[0]), "kz": int(fused[5]), "kernel_ms": dict(zip(
                ["exact_vc_rows_and_list", "exact_vq_rows", "k_mvF", "exact_w_rows_dot"], list(fused)[1:5]))},
            "peak_gbs": peak, "peak_kind": peak_kind}
    print(json.dumps(line), flush=True)
    sv.h.close()
    return 0


def run_adjoint(args):
    """Gradient of the first-harmonic axial force amplitude over the last period of
    the adjoint configuration (D = 16, 2 levels, A = 0.2 D, Re0 = 1, 200 steps per
    period, 804 markers; ``--adjoint-steps`` steps, default 400) with respect to A,
    T and the marker positions, by the discrete adjoint with at most 20 stored
    states, and central differences (step 1e-6 relative; 1e-6 h along seeded unit
    marker directions) of the same float64 model for the quantities in
    ``--adjoint-fd``.  The reference markers carry the seeded perturbation
    0.01 h N(0, 1) of the configuration.  One JSON line; wall-clock seconds."""
    import _pyib_b200_import
    _pyib_b200_import.load()
    import torch
    from pyib_b200 import adjoint as AD
    from pyib_b200 import build
    from pyib_b200.cases import CASES
    build.build_library()
    case = CASES["d16_adjoint_sphere" if args.workload == "d32_oscillating_sphere" else args.workload]
    steps = args.adjoint_steps
    window = args.adjoint_window or case.steps_per_period
    model = AD.CavityModel(case, tol=args.adjoint_tol)
    rng = np.random.default_rng(0)
    ref = model.ref0 + torch.from_numpy(0.01 * model.h0 * rng.standard_normal(tuple(model.ref0.shape))).to(model.dev)
    A, T = case.amplitude, case.period
    t0 = time.perf_counter()
    report = lambda text: print("#", text, file=sys.stderr, flush=True)
    J, gA, gT, gref, info = AD.force_amplitude_and_gradient(model, A, T, ref, steps, window,
                                                            snapshots=args.adjoint_snapshots, progress=report)
    t_grad = time.perf_counter() - t0
    print("# gradient", json.dumps({"J": J, "dJ_dA": gA, "dJ_dT": gT, "seconds": t_grad}), file=sys.stderr, flush=True)
    fd = {}
    t0 = time.perf_counter()
    eps = 1e-6
    f = lambda a, tt, r: AD.force_amplitude(model, a, tt, r, steps, window)
    for item in [x for x in args.adjoint_fd.split(",") if x]:
        if item == "A":
            fd["A"] = ((f(A * (1 + eps), T, ref) - f(A * (1 - eps), T, ref)) / (2 * eps * A), gA)
        elif item == "T":
            fd["T"] = ((f(A, T * (1 + eps), ref) - f(A, T * (1 - eps), ref)) / (2 * eps * T), gT)
        elif item.startswith("dir"):
            q = int(item[3:])
            d = np.random.default_rng(100 + q).standard_normal(tuple(ref.shape))
            d /= np.linalg.norm(d)
            dt_ = torch.from_numpy(d).to(model.dev)
            h = eps * model.h0
            fd[item] = ((f(A, T, ref + h * dt_) - f(A, T, ref - h * dt_)) / (2 * h), float(np.sum(gref * d)))
        print("# finite difference", item, fd[item], time.perf_counter() - t0, file=sys.stderr, flush=True)
    t_fd = time.perf_counter() - t0
    rel = {k: abs(v[1] - v[0]) / max(abs(v[0]), 1e-300) for k, v in fd.items()}
    line = {"workload": case.name, "metric": "adjoint gradient of the force amplitude", "steps": steps,
            "window_steps": window, "cells": int(model.lay.cell_active.sum()),
            "markers": int(model.ref0.shape[0]), "J": J, "dJ_dA": gA, "dJ_dT": gT,
            "dJ_dmarkers_norm": float(np.linalg.norm(gref)), "finite_differences": fd,
            "relative_differences": rel, "max_stored_states": info["max_stored_states"],
            "recomputed_steps": info["recomputed_steps"], "forward_cg_iterations": info["forward_cg_iterations"],
            "total_cg_iterations": info["total_cg_iterations"], "cell_cg_iterations": info["cell_cg_iterations"],
            "gradient_seconds": t_grad, "finite_difference_seconds": t_fd, "tolerance": args.adjoint_tol,
            "snapshots": args.adjoint_snapshots,
            "seconds": {k: info[k] for k in ("forward_seconds", "solve_seconds", "cell_solve_seconds")}}
    print(json.dumps(line), flush=True)
    return 0


def mixed_leg(case, tables, args, steps_done, final):
    """The mixed form on the same case and start: steps/s over ``args.steps`` steps
    (CUDA events, after ``args.warmup`` steps) and, after the same total number of
    steps as the float64 run, the relative errors of U, vc, fL and the body force."""
    from pyib_b200.runner import SphereRun
    run = SphereRun(case, device=0, precision="mixed", mixed_tol=args.mixed_tol, tables=tables)
    sv = run.drv.solver
    for _ in range(args.warmup):
        run.advance()
    ev = C.c_double(0.0)
    its = 0
    sv.h.call("pyib_event", 0, None)
    for _ in range(args.steps):
        run.advance()
        its += run.drv.helmholtz_total_iterations_last_step
    sv.h.call("pyib_event", 1, C.byref(ev))
    while run.step_index < steps_done:
        run.advance()
    sv.h.call("pyib_calc_vel")
    got = dict(U=sv.get("U"), vc=np.asarray(run.vc), fL=np.asarray(run.drv.ib_force_L),
               force=np.asarray(run.loads.latest["body_force"]))
    err = {k: float(np.linalg.norm(got[k] - final[k]) / max(np.linalg.norm(final[k]), 1e-300)) for k in got}
    mv = (C.c_double * 7)()
    sv.set("WORK_E", np.random.default_rng(0).standard_normal(sv.lay.NE) * sv.lay.edge_exists)
    sv.h.call("pyib_bench_matvec", 50, C.c_double(run.dt), mv)
    plan32 = matvec_plan(sv).get("float32", {})
    kernels = {"matvec": float(mv[0]), **matvec_kernel_ms(mv, plan32.get("curl_interp_viscous_fused", False))}
    sv.h.close()
    t = ev.value / 1000.0
    return {"value": args.steps / t, "unit": "steps/s", "ms_per_step": 1000.0 * t / args.steps,
            "inner_iterations_per_step": its / args.steps, "mixed_tolerance": args.mixed_tol,
            "errors_vs_float64_after_steps": steps_done, "errors_vs_float64": err,
            "float32_matvec_kernel_ms": kernels, "float32_matvec_plan": plan32}


# ---------------------------------------------------------------------------
# Mixed precision against float64 on the same case
# ---------------------------------------------------------------------------
def run_precision_compare(args, world, rank, local):
    """Steps/s of the float64 and mixed forms and the mixed form's errors against float64.

    Both forms start from the same state and advance warmup + steps steps; the
    timings are CUDA events over the last ``steps`` steps, the errors are
    relative l2 norms of the final fields (stream function s, face flux U = curl s,
    cell velocity vc, marker forces fL, Eulerian force fE) and of the body-force
    history over all steps.
    """
    import _pyib_b200_import
    _pyib_b200_import.load()
    from pyib_b200 import build
    from pyib_b200.cases import CASES
    from pyib_b200.device import LayoutTables
    from pyib_b200.runner import SphereRun

    build.build_library()
    if world > 1:
        raise SystemExit("the precision comparison runs on one GPU")
    case = CASES[args.workload]
    tables = LayoutTables(case.layout().build(), case.cavity)
    out = {}
    for prec in ("float64", "mixed"):
        run = SphereRun(case, device=0, tables=tables, precision=prec, mixed_tol=args.mixed_tol)
        sv = run.drv.solver
        forces = []
        for _ in range(args.warmup):
            forces.append(run.advance()["body_force"].copy())
        ev = C.c_double(0.0)
        sv.h.call("pyib_event", 0, None)
        its = 0
        for _ in range(args.steps):
            forces.append(run.advance()["body_force"].copy())
            its += run.drv.helmholtz_total_iterations_last_step
        sv.h.call("pyib_event", 1, C.byref(ev))
        sv.h.call("pyib_calc_vel")
        out[prec] = dict(seconds=ev.value / 1000.0, iterations=its, s=np.asarray(run.s).copy(),
                         U=sv.get("U"), vc=np.asarray(run.vc).copy(), fL=np.asarray(run.drv.ib_force_L).copy(),
                         fE=np.asarray(run.drv.ib_force_E).copy(), force=np.array(forces))
        sv.h.close()

    def rel(a, b):
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

    f64, mix = out["float64"], out["mixed"]
    line = {
        "metric": "mixed vs float64 steps/s and errors", "workload": case.name,
        "steps": args.steps, "warmup": args.warmup, "mixed_tolerance": args.mixed_tol,
        "float64": {"steps_per_s": args.steps / f64["seconds"], "cg_iterations": f64["iterations"]},
        "mixed": {"steps_per_s": args.steps / mix["seconds"], "inner_iterations": mix["iterations"]},
        "errors_vs_float64": {k: rel(mix[k], f64[k]) for k in ("s", "U", "vc", "fL", "fE", "force")},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# Force harmonic error of the full oscillation run, float64 and mixed
# ---------------------------------------------------------------------------
def run_harmonic(args, world, rank, local):
    """Six periods of the workload in float64 and in mixed precision; the axial body
    force of each is fitted over 4T < t <= 6T against the analytic unsteady-Stokes
    force (``pyib_b200.harmonic``), and the two harmonic errors are compared."""
    import _pyib_b200_import
    _pyib_b200_import.load()
    from pyib_b200 import build
    from pyib_b200.cases import CASES, R
    from pyib_b200.device import LayoutTables
    from pyib_b200.harmonic import harmonic_error
    from pyib_b200.runner import SphereRun

    build.build_library()
    if world > 1:
        raise SystemExit("the harmonic run uses one GPU")
    case = CASES[args.workload]
    if case.amplitude == 0.0:
        raise SystemExit("the harmonic check needs an oscillating case")
    tables = LayoutTables(case.layout().build(), case.cavity)
    steps = args.periods * case.steps_per_period
    axis = np.asarray(case.axis, dtype=np.float64) / np.linalg.norm(case.axis)
    mu = case.viscosity
    out = {}
    for prec in ("float64", "mixed"):
        run = SphereRun(case, device=0, tables=tables, precision=prec, mixed_tol=args.mixed_tol)
        sv = run.drv.solver
        times, fax, its = [], [], 0
        ev = C.c_double(0.0)
        sv.h.call("pyib_event", 0, None)
        for _ in range(steps):
            load = run.advance()
            times.append(run.step_index * run.dt)
            fax.append(float(np.asarray(load["body_force"]) @ axis))
            its += run.drv.helmholtz_total_iterations_last_step
        sv.h.call("pyib_event", 1, C.byref(ev))
        sv.h.close()
        err = harmonic_error(times, fax, mu=mu, radius=R, amplitude=case.amplitude, omega=case.omega,
                             phase=case.phase, nu=mu / case.density)
        out[prec] = {"steps_per_s": steps / (ev.value / 1000.0), "cg_iterations": its, **err}
    diff_pp = 100.0 * abs(out["mixed"]["harmonic_vector_error"] - out["float64"]["harmonic_vector_error"])
    line = {"metric": "force harmonic error, float64 and mixed", "workload": case.name, "steps": steps,
            "periods": args.periods, "mixed_tolerance": args.mixed_tol, "float64": out["float64"],
            "mixed": out["mixed"], "difference_percentage_points": diff_pp}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# Batched sweep: independent cases of uneven size, concurrent vs one at a time
# ---------------------------------------------------------------------------
def aggregate_batch(dist, seconds_concurrent, seconds_sequential, cells, launches, cg_iterations,
                    max_case_iterations):
    """Whole-job figures of a sharded sweep: the slowest rank's times, the sums of
    the per-rank work (every rank calls the same reductions in the same order)."""
    return {
        "seconds_concurrent": reduce_max(dist, float(seconds_concurrent)),
        "seconds_sequential": reduce_max(dist, float(seconds_sequential)),
        "cells": reduce_sum(dist, float(cells)),
        "launches": reduce_sum(dist, float(launches)),
        "cg_iterations": reduce_sum(dist, float(cg_iterations)),
        "max_case_iterations": reduce_max(dist, float(max_case_iterations)),
    }


def run_batch(args, world, rank, local):
    """Aggregate cell-updates/s of the seeded sweep: batched (``value``: one
    ``pyib_batch``, the CG iterations of all cases as one launch per kernel stage,
    graph-captured), concurrently (one host thread and stream per case) and one
    case at a time.

    Each timing advances every case by the same ``--steps`` steps from the same
    state (every case is snapshotted after the warm-up and restored before each
    phase), so the three phases do the same work, and the line says whether they
    ended in the same bits; host wall clock around each phase, every case's last
    call having waited for its own stream.
    The batched phase also reports the CUDA-event time of its batched CG chunks
    and their algorithmic HBM rate (80 B per edge and CG iteration, summed over
    the cases) against the measured peak.  Under
    torchrun the cases are split across the ranks by cost (cells x steps,
    longest first, ``batch.partition``): each rank runs its own share with no
    collective on the data path, and the line reports the summed work over the
    slowest rank's time.
    """
    from collections import Counter

    import _pyib_b200_import
    _pyib_b200_import.load()
    from pyib_b200 import build
    from pyib_b200.batch import BatchRun, partition, sweep_cases

    build.build_library()
    dist = maybe_init_dist(world, local)
    cases = sweep_cases(args.batch_cases, seed=0)
    parts, loads = partition(cases, world, steps=args.steps)
    mine = [cases[q] for q in parts[rank]]
    t_setup = time.perf_counter()
    batch = BatchRun(mine, device=local if world > 1 else 0, precision=args.precision, mixed_tol=args.mixed_tol)
    batch.tune()
    setup_s = time.perf_counter() - t_setup
    cells = batch.cells
    for _ in range(args.warmup):
        batch.advance(1, concurrent=True)
    barrier(dist)
    sampler = ClockSampler(local if world > 1 else 0) if rank == 0 else None
    if sampler:
        sampler.start()
    empty = {"cg_iterations": 0, "max_case_iterations": 0, "per_case_iterations": []}
    snap = batch.snapshot()
    batch.batch_timing(reset=True)
    t_bat, st_bat = batch.advance(args.steps, batched=True) if mine else (0.0, empty)
    fp_bat = batch.fingerprint() if mine else []
    bt = batch.batch_timing(reset=True)
    edges = [int(r.drv.layout.edge_exists.sum()) for r in batch.runs]
    per_edge = ALGO_BYTES_PER_EDGE_ITER if args.precision == "float64" else ALGO_BYTES_PER_EDGE_ITER / 2
    cg_bytes = float(sum(per_edge * e * it for e, it in zip(edges, st_bat["per_case_iterations"])))
    barrier(dist)
    batch.restore(snap)
    t_con, st_con = batch.advance(args.steps, concurrent=True) if mine else (0.0, empty)
    fp_con = batch.fingerprint() if mine else []
    batch.restore(snap)
    barrier(dist)
    t_seq, st_seq = batch.advance(args.steps, concurrent=False) if mine else (0.0, empty)
    fp_seq = batch.fingerprint() if mine else []
    same = all(all(np.array_equal(x, y) for x, y in zip(a, b)) and all(np.array_equal(x, y) for x, y in zip(a, c))
               for a, b, c in zip(fp_bat, fp_con, fp_seq))
    same = -reduce_max(dist, -1.0 if same else 0.0) > 0.5   # every rank agrees
    del snap, fp_bat, fp_con, fp_seq
    clocks = sampler.stop() if sampler else None
    launches = 0
    timing = (C.c_double * 5)()
    for r in batch.runs:
        r.drv.solver.h.call("pyib_cg_timing", timing, 0)
        launches += int(timing[2])
    con = aggregate_batch(dist, t_con, t_seq, sum(cells), launches, st_con["cg_iterations"],
                          st_con["max_case_iterations"])
    bat = aggregate_batch(dist, t_bat, bt["chunk_seconds"], sum(cells), bt["batched_launches"],
                          st_bat["cg_iterations"], st_bat["max_case_iterations"])
    bat_bytes = reduce_sum(dist, cg_bytes)
    seq = aggregate_batch(dist, t_con, t_seq, sum(cells), 0, st_seq["cg_iterations"],
                          st_seq["max_case_iterations"])
    batch.close()
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    upd = con["cells"] * args.steps
    peak, peak_kind = peaks()
    # bat: seconds_concurrent = the batched phase's wall clock, seconds_sequential = its
    # CUDA-event chunk time (max over ranks)
    chunk_s = bat["seconds_sequential"]
    line = {
        "metric": "batched sweep cell-updates/s", "value": upd / bat["seconds_concurrent"],
        "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * bat["seconds_concurrent"] / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f64" if args.precision == "float64" else "f32+f64", "data": "synthetic",
        "config": {"workload": "batched_sweep", "cases": len(cases), "seed": 0,
                   "cells_per_diameter_histogram": dict(sorted(Counter(c.cells_per_diameter
                                                                       for c in cases).items())),
                   "total_cells": int(con["cells"]), "levels": 2, "precision": args.precision,
                   "setup_seconds": setup_s, "l2": "inputs larger than L2",
                   "parallelism": f"cases split over {world} GPU(s) by cells x steps",
                   "cells_per_rank": [int(x // args.steps) for x in loads]},
        "batched": {"seconds": bat["seconds_concurrent"], "cg_iterations": int(bat["cg_iterations"]),
                    "max_case_iterations": int(bat["max_case_iterations"]),
                    "cg_chunk_seconds": chunk_s, "batched_kernel_launches": int(bat["launches"]),
                    "graph_captures": int(bt["graph_captures"]),
                    "roofline": {"bound": "hbm", "achieved": bat_bytes / max(chunk_s, 1e-12) / 1e9, "peak": peak,
                                 "unit": "GB/s", "frac": bat_bytes / max(chunk_s, 1e-12) / 1e9 / peak,
                                 "peak_kind": peak_kind,
                                 "algorithmic_bytes": bat_bytes,
                                 "kernel": "batched CG iteration chunks (80 B per edge and iteration in "
                                           "float64, 40 B in the float32 iterations of the mixed form; all cases)"}},
        "concurrent": {"value": upd / con["seconds_concurrent"], "seconds": con["seconds_concurrent"],
                       "cg_iterations": int(con["cg_iterations"]),
                       "max_case_iterations": int(con["max_case_iterations"])},
        "same_steps_bit_identical": same,
        "one_at_a_time": {"value": upd / seq["seconds_sequential"], "seconds": seq["seconds_sequential"],
                          "cg_iterations": int(seq["cg_iterations"]),
                          "max_case_iterations": int(seq["max_case_iterations"])},
        "gpu_launches_since_setup": int(con["launches"]),
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    return 0


PRESSURE_AXIS = 128          # cells per axis of the pressure-recovery lattice (2,097,152 cells)
PRESSURE_CPU_AXIS = 64       # the CPU sample: the same lattice at 64^3 (262,144 cells)


def pressure_inputs(axis):
    """Uniform lattice graph of the offline pressure recovery (the reference's test
    construction) with a quadratic gradient plus seeded noise."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pressure_oracle as PO
    pos, faces, area = PO.uniform_graph(axis, 1.0 / axis)
    rng = np.random.default_rng(17)
    grad = PO.quadratic_gradient(pos) + 0.1 * rng.standard_normal(pos.shape)
    return pos, faces, area, grad


def pressure_cpu_sample():
    """scipy CG of the reference's recover_pressure (the oracle restatement) on the
    64^3 sample; returns (row-iterations/s, seconds, sample text)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pressure_oracle as PO
    pos, faces, area, grad = pressure_inputs(PRESSURE_CPU_AXIS)
    t0 = time.perf_counter()
    _, diag = PO.recover_pressure(pos, faces, area, grad)
    sec = time.perf_counter() - t0
    rows = PRESSURE_CPU_AXIS ** 3 - 1
    return rows * diag["iterations"] / sec, sec, (f"oracle (scipy cg, the reference's algorithm) recover_pressure on "
                                                  f"{PRESSURE_CPU_AXIS}^3 cells, {diag['iterations']} iterations, "
                                                  f"{sec:.2f} s including assembly")


def run_pressure(args, world, rank, local):
    """Offline pressure recovery: graph-CG row-iterations/s on a 128^3 lattice graph.

    ``value``: rows x iterations / device time of the CG (events around the
    iterations; the matrix already resident).  ``e2e``: the same work over the
    wall time of ``recover_pressure`` (shape checks, copies of the inputs, device
    assembly and checks, CG, gauge, copy of the pressure).  Replicas
    for N > 1 (each rank recovers its own snapshot).
    """
    import _pyib_b200_import
    _pyib_b200_import.load()
    if args.impl == "reference":
        if rank != 0:
            return 0
        vals, sample = [], ""
        for k in range(args.warmup + args.steps):
            v, _, sample = pressure_cpu_sample()
            if k >= args.warmup:
                vals.append(v)
        value = float(np.mean(vals))
        print(json.dumps({
            "impl": "reference", "metric": "pressure-recovery CG row-iterations/s", "value": value,
            "unit": "row-iterations/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": "pressure_recovery_128", "cpu_sample_axis": PRESSURE_CPU_AXIS},
            "cpu_baseline": {"value": value, "unit": "row-iterations/s", "cores": 1, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "row-iterations/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }), flush=True)
        return 0
    from pyib_b200 import build
    from pyib_b200 import postprocess as PP
    build.build_library()
    import torch
    torch.cuda.set_device(local)
    dist = maybe_init_dist(world, local)
    pos, faces, area, grad = pressure_inputs(PRESSURE_AXIS)
    h = PP.bare_handle(local)
    timing = (C.c_double * 5)()
    for _ in range(args.warmup):
        PP.recover_pressure(pos, faces, area, grad, handle=h)
    barrier(dist)
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    h.call("pyib_cg_timing", timing, 1)
    solve_ms, dev_ms, e2e_s, iters, nnz, sweeps = [], [], [], [], 0, 0
    for _ in range(args.steps):
        t = {}
        t0 = time.perf_counter()
        _, diag = PP.recover_pressure(pos, faces, area, grad, handle=h, timing=t)
        e2e_s.append(time.perf_counter() - t0)
        solve_ms.append(t["solve_ms"])
        dev_ms.append(t["device_ms"])
        iters.append(diag["iterations"])
        nnz, sweeps = t["nnz"], t["sweeps"]
    clocks = sampler.stop() if sampler else None
    h.call("pyib_cg_timing", timing, 0)
    launches = int(timing[2])
    rows = PRESSURE_AXIS ** 3 - 1
    dev_s = reduce_max(dist, sum(solve_ms) / 1000.0)
    wall = reduce_max(dist, sum(e2e_s))
    work = float(rows) * sum(iters) * world
    # algorithmic bytes of one CG iteration: the matvec + p.q kernel reads ptr and p once
    # per row and col + val per nonzero and writes q (24 B per row + 12 B per nonzero);
    # the update reads p, q, dinv, x, r and writes x, r, z (64 B); the direction reads
    # z, p and writes p (24 B)
    bytes_iter = 112.0 * (rows + 1) + 12.0 * nnz
    hbm, peak_kind = peaks()
    achieved = bytes_iter * sum(iters) / (sum(solve_ms) / 1000.0) / 1e9
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, sec, sample = pressure_cpu_sample()
        cpu = {"value": v, "unit": "row-iterations/s", "cores": 1, "kind": "port", "sample": sample}
    h.close()
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": "pressure-recovery CG row-iterations/s", "value": work / dev_s, "unit": "row-iterations/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * dev_s / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "pressure_recovery_128", "cells": rows + 1, "faces": int(len(faces)),
                   "csr_nonzeros": nnz, "cg_iterations": iters, "tolerance": 1e-10,
                   "device_ms_per_recovery": sum(dev_ms) / len(dev_ms), "connectivity_sweeps": sweeps,
                   "l2": "inputs larger than L2 (the CG streams 0.42 GB per iteration)"},
        "e2e": {"value": work / wall, "unit": "row-iterations/s", "seconds_per_recovery": wall / args.steps,
                "h2d_bytes_per_step": int(48 * (rows + 1) + 24 * len(faces)),
                "d2h_bytes_per_step": int(8 * (rows + 1))},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": None, "peak_source": peak_kind,
                     "bytes_per_iteration": bytes_iter},
        "cpu_baseline": cpu, "gpu_launches": launches, "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="d32_oscillating_sphere")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the mixed-precision leg of the default float64 run")
    ap.add_argument("--precision", default="float64", choices=["float64", "mixed"])
    ap.add_argument("--mixed-tol", type=float, default=0.1)
    ap.add_argument("--batch-cases", type=int, default=64)
    ap.add_argument("--harmonic", action="store_true",
                    help="run --periods oscillation periods in float64 and mixed and fit the force")
    ap.add_argument("--periods", type=int, default=6)
    ap.add_argument("--adjoint", action="store_true",
                    help="gradient of the force amplitude by the discrete adjoint (workload d16_adjoint_sphere)")
    ap.add_argument("--adjoint-steps", type=int, default=400)
    ap.add_argument("--adjoint-fd", default="A,T,dir0",
                    help="comma list of central-difference checks: A, T, dir0, dir1, ...")
    ap.add_argument("--adjoint-tol", type=float, default=1e-13)
    ap.add_argument("--adjoint-window", type=int, default=0,
                    help="steps fitted at the end (default: one period of the configuration)")
    ap.add_argument("--adjoint-snapshots", type=int, default=20)
    ap.add_argument("--matvec-only", action="store_true",
                    help="time the standalone float64 matvecs (three-kernel and fused) on the workload's layout")
    ap.add_argument("--compare-precision", action="store_true",
                    help="run the workload in float64 and mixed precision and report the errors")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    world, rank, local = dist_env()
    if args.workload == "batched_sweep":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the batched sweep has no reference "
                              "counterpart (the reference runs one case per process)"}), flush=True)
            return 0
        return run_batch(args, world, rank, local)
    if args.workload == "pressure_recovery_128":
        return run_pressure(args, world, rank, local)
    if args.matvec_only:
        return run_matvec(args)
    if args.adjoint:
        return run_adjoint(args)
    if args.compare_precision:
        return run_precision_compare(args, world, rank, local)
    if args.harmonic:
        return run_harmonic(args, world, rank, local)
    if args.impl == "reference":
        return run_reference(args, world, rank)
    return run_b200(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
