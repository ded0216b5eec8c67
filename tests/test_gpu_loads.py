"""Closed-sphere loads along a trajectory against the reference's own load history."""
import numpy as np
import pytest

import pyib_oracle as O
import parity_util as PU
from pyib_b200.driver import B200Driver
from pyib_b200.runner import SphereLoads

pytestmark = pytest.mark.gpu


def test_body_force_history_matches_reference():
    """``ClosedSphereLoadCorrection.advance`` (ib_interior.py:268-308) per step.

    The reference fixture records, per step, the body force, the fluid force and
    the body moment (``tr_hist`` columns 2-10) of the 3-level oscillating sphere
    in the closed cavity.  The B200 run goes through the device load sums and
    ``SphereLoads``; the fields agree with the reference's to about 1e-10, so the
    loads do too.
    """
    name = "n3_osc"
    g = PU.golden(name)
    par = g["params"]
    lay = PU.layout_for(name)
    drv = B200Driver(lay, float(g["visc"]), float(g["rou"]))
    drv.set_cavity(0.0, False)
    ref, ds = g["ref_markers"], g["ib_ds"]
    motion = O.Oscillation(ref, par["axis"], par["amplitude"], par["frequency"], par["phase"])
    mk0, vel0 = motion(0.0)
    drv.set_ib(None, mk0, ds, vel0)
    drv.set_motion(motion, 0.0)
    h = float(par["h"])
    radius = float(par.get("radius", 0.25))
    axis = np.asarray(par["axis"], dtype=float) / np.linalg.norm(par["axis"])
    loads = SphereLoads(drv, np.zeros(3), np.abs(axis) * par["amplitude"], radius, h, float(g["rou"]), 1.5 * h)

    def centre(t):
        ang = 2.0 * np.pi * par["frequency"] * t + par["phase"]
        return par["amplitude"] * np.sin(ang) * axis

    dt = float(g["dt"])
    s = drv.initial_stream_function(0.0)
    s, _, vc = drv.calc_vel(s)
    s_old = np.asarray(s).copy()
    loads.initialize(centre(0.0))
    rows = []
    for k in range(1, int(g["tr_steps"]) + 1):
        drv.time = (k - 1) * dt
        s, vc, s_old = drv.step(s, s_old, dt, dt, inner=4)
        drv.time = k * dt
        ld = loads.advance(centre(drv.time), dt)
        rows.append(np.concatenate([ld["body_force"], ld["force_fluid"], ld["body_moment"]]))
    got = np.array(rows)
    hist = g["tr_hist"]
    for lo, what in ((2, "body_force"), (5, "force_fluid")):
        want = hist[:, lo:lo + 3]
        err = np.linalg.norm(got[:, lo - 2:lo + 1] - want) / np.linalg.norm(want)
        assert err < 1e-8, (what, err)
    # the moment of a sphere oscillating along its axis vanishes up to rounding
    scale = np.max(np.abs(hist[:, 2:5]))
    assert np.max(np.abs(got[:, 6:9])) <= 1e-8 * scale + np.max(np.abs(hist[:, 8:11])) + 1e-14
