"""Assemble a B200 sphere run (driver + loads) and advance it, as ``ib_case.run_case`` does.

``SphereRun`` mirrors the step loop of ``ib_case.run_case`` (lines 1518-1530):
the clock is anchored to the integer step, ``Driver.step`` advances the fluid,
then the closed-sphere load correction (``ib_interior.py:268-308``) turns
the Eulerian IB force and the interior momentum into the body load.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .cases import R, SphereCase
from .driver import B200Driver, step_batch


class SphereLoads:
    """Closed-sphere load correction on the device (ClosedSphereLoadCorrection)."""

    def __init__(self, drv: B200Driver, centre0, max_translation, radius, width, density,
                 support_width):
        lay = drv.layout
        act = np.nonzero(lay.cell_active)[0]
        pos = lay.cpos[act]
        c0 = np.asarray(centre0, dtype=np.float64)
        mt = np.abs(np.asarray(max_translation, dtype=np.float64))
        hw = radius + 0.5 * width + mt
        cand = act[np.all((pos >= c0 - hw) & (pos <= c0 + hw), axis=1)]
        fw = radius + support_width + mt
        fw = fw + 8.0 * np.finfo(np.float64).eps * np.maximum(1.0, np.abs(c0) + fw)
        fidx = act[np.all((pos >= c0 - fw) & (pos <= c0 + fw), axis=1)]
        if cand.size == 0:
            raise ValueError("the closed-sphere indicator contains no Eulerian cells")
        self.drv = drv
        drv.solver.set_load_lists(cand, fidx)
        self.c0 = c0
        self.fixed = bool(np.all(mt == 0.0))
        self.radius, self.width, self.density = float(radius), float(width), float(density)
        self.current = None
        self.latest = None

    def evaluate(self, centre):
        out = (C.c_double * 13)()
        c = np.ascontiguousarray(centre, dtype=np.float64)
        self.drv.solver.h.call("pyib_loads", c.ctypes.data_as(C.POINTER(C.c_double)),
                               C.c_double(self.radius), C.c_double(self.width), C.c_double(self.density),
                               int(self.fixed), self.c0.ctypes.data_as(C.POINTER(C.c_double)), out)
        return np.array(out[:])

    def initialize(self, centre):
        self.current = self.evaluate(centre)
        self.latest = None
        return self.current

    def advance(self, centre, dt):
        prev = self.current
        cur = self.evaluate(centre)
        lrate = (cur[6:9] - prev[6:9]) / dt
        arate = (cur[9:12] - prev[9:12]) / dt
        ff, mf = cur[0:3], cur[3:6]
        self.current = cur
        self.latest = dict(force_fluid=ff, moment_fluid=mf, body_force=-ff + lrate,
                           body_moment=-mf + arate, linear_momentum=cur[6:9],
                           angular_momentum=cur[9:12], indicator_volume=cur[12],
                           linear_rate=lrate, angular_rate=arate)
        return self.latest


class SphereRun:
    """One sphere case on one GPU: driver, markers, loads and the current state."""

    def __init__(self, case: SphereCase, device=0, layout=None, check_interval=20,
                 precision="float64", mixed_tol=0.1, tables=None):
        self.case = case
        if tables is not None:
            lay = tables.lay
        else:
            lay = layout if layout is not None else case.layout()
        drv = B200Driver(lay, case.viscosity, case.density,
                         cg_max_iterations=case.cg_max_iterations, device=device,
                         precision=precision, mixed_tol=mixed_tol, tables=tables)
        drv.cg_check_interval = int(check_interval)
        if case.cavity:
            drv.set_cavity(0.0, False)
        ref, ds = case.markers()
        self.motion = case.motion()
        if self.motion is not None:
            mk0, vel0 = self.motion(0.0)
            drv.set_ib(None, mk0, ds, vel0)
            drv.set_motion(self.motion, 0.0)
            max_tr = np.abs(np.asarray(case.axis, float) / np.linalg.norm(case.axis)) * case.amplitude
        else:
            drv.set_ib(None, ref, ds, np.zeros_like(ref))
            max_tr = np.zeros(3)
        self.drv = drv
        self.dt = case.time_step
        self.loads = SphereLoads(drv, np.zeros(3), max_tr, R, case.h, case.density, 1.5 * case.h)
        s = drv.initial_stream_function(case.inflow)
        self.s, _, self.vc = drv.calc_vel(s)
        self.s_old = np.asarray(self.s).copy()
        self.loads.initialize(self.centre(0.0))
        self.step_index = 0

    def centre(self, t):
        if self.motion is None:
            return np.zeros(3)
        return self.motion.centre(t)

    def snapshot(self):
        """The state that the next steps start from (host copies)."""
        return dict(s=np.asarray(self.s).copy(), s_old=np.asarray(self.s_old).copy(),
                    state=self.drv.ib_state_dict(), step=self.step_index, time=self.drv.time,
                    loads=np.asarray(self.loads.current).copy())

    def restore(self, snap):
        """Return to a snapshot: the following steps repeat the ones taken after it
        bit for bit."""
        drv = self.drv
        self.s, self.s_old = snap["s"].copy(), snap["s_old"].copy()
        if snap["state"] is not None:
            drv.load_ib_state_dict(snap["state"])
            drv.ib_force_update_count = snap["state"]["force_update_count"]
        self.step_index, drv.time = snap["step"], snap["time"]
        self.loads.current = snap["loads"].copy()
        if self.motion is not None:
            mk, vel = self.motion(drv.time)
            drv.set_ib(drv.ib, mk, drv.ib_ds, vel)

    def advance(self, inner=4):
        k = self.step_index + 1
        self.drv.time = (k - 1) * self.dt
        self.s, self.vc, self.s_old = self.drv.step(self.s, self.s_old, self.dt, self.dt, inner=inner)
        self.drv.time = k * self.dt
        load = self.loads.advance(self.centre(self.drv.time), self.dt)
        self.step_index = k
        return load


def advance_batch(batch, runs, inner=4):
    """``SphereRun.advance`` of several runs at once: one step of every run through the
    ``pyib_batch`` ``batch`` (built over the runs' contexts, in this order), the
    Helmholtz solves batched; returns each run's load.  Each run ends in the state
    its own ``advance`` would give."""
    for r in runs:
        r.drv.time = r.step_index * r.dt
    out = step_batch(batch, [r.drv for r in runs], [(r.s, r.s_old) for r in runs], [r.dt for r in runs],
                     [r.dt for r in runs], inner=inner)
    loads = []
    for r, (s, vc, s_old) in zip(runs, out):
        k = r.step_index + 1
        r.s, r.vc, r.s_old = s, vc, s_old
        r.drv.time = k * r.dt
        loads.append(r.loads.advance(r.centre(r.drv.time), r.dt))
        r.step_index = k
    return loads
