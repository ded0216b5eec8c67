"""Batched sweep: many independent oscillating-sphere cases of uneven size on one GPU.

Each case is a full ``SphereRun`` (its own library context, CUDA stream, CG
graphs and autotuned tiles).  ``BatchRun.advance`` steps the cases in one of
three ways:

* batched: one ``pyib_batch`` over all contexts; each step runs every case's
  step parts on its own stream, and the CG iterations of all cases' Helmholtz
  solves run together, one launch per kernel stage over the tiles of every case
  still iterating, ``check`` iterations to one CUDA graph;
* concurrent: every case from its own host thread (one context per host thread),
  so the cases' graph replays and kernels overlap on their streams; the library
  calls release the Python interpreter lock (ctypes);
* one case after the other.

All three give every case the same bits.

Cases with the same resolution share one ``LayoutTables`` (operators, masks,
patch rows), built once on the host.

The sweep draw follows the batched configuration: seeded
``numpy.random.default_rng(seed)``; per case, in this order, ``D`` cells per
diameter from {12, 16, 20, 24, 32}, amplitude ``A/D`` uniform in [0.05, 0.3],
``Re0`` log-uniform in [0.1, 10]; two nested levels (half widths 2D and 4D),
closed no-slip walls, omega = 3.6, 200 steps per period.
"""
from __future__ import annotations

import threading
import time
from collections import Counter

import numpy as np

from .cases import SphereCase
from . import _lib
from .device import LayoutTables
from .runner import SphereRun, advance_batch

SWEEP_CELLS_PER_DIAMETER = (12, 16, 20, 24, 32)


def sweep_cases(count=64, seed=0, cg_max_iterations=20000):
    """The seeded sweep: ``count`` cases drawn as described in the module docstring."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(int(count)):
        d = int(rng.choice(SWEEP_CELLS_PER_DIAMETER))
        a = float(rng.uniform(0.05, 0.3))
        re0 = float(10.0 ** rng.uniform(-1.0, 1.0))
        out.append(SphereCase(name=f"sweep_{i:02d}_d{d}", cells_per_diameter=d, half_widths_d=(2.0, 4.0),
                              reynolds=re0, amplitude_d=a, cg_max_iterations=cg_max_iterations))
    return out


def case_cost(case, steps=1):
    """Work of one case: existing cells x steps (every case advances the same
    number of steps, each step touching every cell).  Level L of the concentric
    layout is a box of ``2 hw_L n / 2^L`` cells per axis (``n`` cells per
    diameter), less the finer box it contains."""
    n = int(case.cells_per_diameter)
    cells, finer = 0, 0
    for L, hw in enumerate(case.half_widths_d):
        side = int(round(2.0 * float(hw) * n / 2 ** L))
        cells += side ** 3 - (finer // 2) ** 3
        finer = side
    return cells * int(steps)


def partition(cases, world, steps=1):
    """Cases split across ``world`` GPUs by cost: longest first, each to the rank with
    the least work so far (lowest rank on ties).  Deterministic; every case appears
    once; each rank's list keeps the sweep order."""
    world = int(world)
    if world < 1:
        raise ValueError("world must be at least 1")
    costs = [case_cost(c, steps) for c in cases]
    load = [0] * world
    owner = [0] * len(cases)
    for q in sorted(range(len(cases)), key=lambda i: (-costs[i], i)):
        r = min(range(world), key=lambda k: (load[k], k))
        owner[q] = r
        load[r] += costs[q]
    return [[q for q in range(len(cases)) if owner[q] == r] for r in range(world)], load


class BatchRun:
    """Independent sphere cases on one GPU, stepped concurrently or one at a time."""

    def __init__(self, cases, device=0, precision="float64", mixed_tol=0.1):
        self.cases = list(cases)
        self.tables = {}
        self.runs = []
        self._batch = None
        for c in self.cases:
            key = (c.cells_per_diameter, tuple(c.half_widths_d), bool(c.cavity))
            if key not in self.tables:
                self.tables[key] = LayoutTables(c.layout().build(), c.cavity)
            self.runs.append(SphereRun(c, device=device, tables=self.tables[key], precision=precision,
                                       mixed_tol=mixed_tol))

    @property
    def cells(self):
        """Existing cells of every case (the unit of cell-updates/s)."""
        return [int(r.drv.layout.cell_active.sum()) for r in self.runs]

    def histogram(self):
        return dict(sorted(Counter(c.cells_per_diameter for c in self.cases).items()))

    def tune(self):
        """Run each context's matvec autotuner alone, before any concurrent work."""
        import ctypes as C
        ms = (C.c_double * 7)()
        for r in self.runs:
            sv = r.drv.solver
            sv.set("WORK_E", np.zeros(sv.lay.NE))
            sv.h.call("pyib_bench_matvec", 1, C.c_double(r.dt), ms)

    def _stats(self, per_run_iters):
        return {"cg_iterations": int(sum(sum(x) for x in per_run_iters)),
                "max_case_iterations": int(max(sum(x) for x in per_run_iters)),
                "per_case_iterations": [int(sum(x)) for x in per_run_iters]}

    def advance(self, steps=1, concurrent=True, batched=False):
        """Advance every case by ``steps`` steps; returns (seconds, stats).

        ``batched``: every step of all cases goes through one ``pyib_batch`` (the CG
        iterations of all cases as one launch per kernel stage); otherwise each case
        steps on its own context, from its own host thread (``concurrent``) or one
        case after the other."""
        iters = [[] for _ in self.runs]
        errors = []
        if batched:
            if self._batch is None:
                self._batch = _lib.Batch([r.drv.solver.h for r in self.runs])
            t0 = time.perf_counter()
            for _ in range(steps):
                advance_batch(self._batch, self.runs)
                for q, r in enumerate(self.runs):
                    iters[q].append(r.drv.helmholtz_total_iterations_last_step)
            return time.perf_counter() - t0, self._stats(iters)

        def work(q):
            r = self.runs[q]
            try:
                for _ in range(steps):
                    r.advance()
                    iters[q].append(r.drv.helmholtz_total_iterations_last_step)
            except BaseException as exc:       # re-raised on the calling thread
                errors.append((q, exc))

        t0 = time.perf_counter()
        if concurrent:
            threads = [threading.Thread(target=work, args=(q,), daemon=True) for q in range(len(self.runs))]
            for t in threads:
                t.start()
            for t in threads:
                t.join()
        else:
            for q in range(len(self.runs)):
                work(q)
                if errors:
                    break
        seconds = time.perf_counter() - t0
        if errors:
            q, exc = errors[0]
            raise RuntimeError(f"case {self.cases[q].name} failed: {exc}") from exc
        return seconds, self._stats(iters)

    def snapshot(self):
        """Every case's state (``SphereRun.snapshot``)."""
        return [r.snapshot() for r in self.runs]

    def restore(self, snaps):
        """Every case back to ``snapshot``'s state."""
        for r, snap in zip(self.runs, snaps):
            r.restore(snap)

    def fingerprint(self):
        """Every case's stream function, Lagrangian force and body force (host copies),
        to compare two ways of taking the same steps."""
        return [(np.asarray(r.s).copy(), np.asarray(r.drv.ib_force_L).copy(),
                 np.asarray(r.loads.latest["body_force"]).copy()) for r in self.runs]

    def batch_timing(self, reset=True):
        """CUDA-event seconds of the batched CG chunks, batched kernels launched and
        graph captures since the last reset (pyib_batch_timing)."""
        import ctypes as C
        out = (C.c_double * 3)()
        if self._batch is not None:
            self._batch.call("pyib_batch_timing", out, int(reset))
        return {"chunk_seconds": out[0], "batched_launches": int(out[1]), "graph_captures": int(out[2])}

    def close(self):
        """Release the batch and every case's device context."""
        if self._batch is not None:
            self._batch.close()
            self._batch = None
        for r in self.runs:
            if r.drv._solver is not None:
                r.drv._solver.h.close()
        self.runs = []
