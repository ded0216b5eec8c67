"""GPU parity of whole steps: ``Driver.step`` trajectories against the reference goldens."""
import numpy as np
import pytest

import pyib_oracle as O
import parity_util as PU
from pyib_b200.driver import B200Driver

pytestmark = pytest.mark.gpu


def run_b200(name, steps=None):
    g = PU.golden(name)
    par = g["params"]
    lay = PU.layout_for(name)
    drv = B200Driver(lay, float(g["visc"]), float(g["rou"]))
    if bool(g["cavity"]):
        drv.set_cavity(0.0, False)
    ref = g["ref_markers"]
    ds = g["ib_ds"]
    amp = float(par.get("amplitude", 0.0))
    if amp != 0.0:
        motion = O.Oscillation(ref, par["axis"], amp, par["frequency"], par["phase"])
        mk0, vel0 = motion(0.0)
        drv.set_ib(None, mk0, ds, vel0)
        drv.set_motion(motion, 0.0)
    else:
        drv.set_ib(None, ref, ds, np.zeros_like(ref))
    dt = float(g["dt"])
    s = drv.initial_stream_function(float(par.get("inflow", 1.0)))
    s, _, vc = drv.calc_vel(s)
    s_old = np.asarray(s).copy()
    iters = []
    n = int(g["tr_steps"]) if steps is None else steps
    for k in range(1, n + 1):
        drv.time = (k - 1) * dt
        s, vc, s_old = drv.step(s, s_old, dt, dt, inner=4)
        drv.time = k * dt
        iters.append(drv.helmholtz_iterations_last_step)
    return drv, np.asarray(s), np.asarray(s_old), np.asarray(vc), iters


@pytest.mark.parametrize("name", PU.CASES)
def test_trajectory_matches_reference(name):
    g = PU.golden(name)
    drv, s, s_old, vc, iters = run_b200(name)
    assert iters == [int(v) for v in g["tr_hist"][:, 1]]
    tol = 1e-10
    assert PU.rel(PU.edge_from_dense(name, s), g["tr_s"]) < tol
    assert PU.rel(PU.edge_from_dense(name, s_old), g["tr_s_old"]) < tol
    nc = drv.layout.NC
    assert PU.rel(PU.cell3_from_dense(name, vc[:, :nc]), g["tr_vc"]) < tol
    fE = np.asarray(drv.ib_force_E)
    assert PU.rel(PU.cell3_from_dense(name, fE), g["tr_fE"]) < tol
    assert PU.rel(drv.ib_force_L, g["tr_fL"]) < tol
