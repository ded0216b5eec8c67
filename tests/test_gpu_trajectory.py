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


def l2rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("name", PU.CASES)
def test_trajectory_matches_reference(name):
    """Whole steps against the reference's own float64 run.

    Two float64 runs of the reference algorithm that differ only in rounding
    order (its CSR matvec versus its matrix-free flow_mat) differ after the
    trajectory by the ``envelope_*`` values stored with the oracle fixture
    (up to 2.3e-10 for fL on n2, 1.1e-9 for the gauge part of s on n3).  The
    B200 path must stay within 5x that envelope, and never looser than needed
    below 1e-10, from the reference's trajectory and from the oracle's.  (The
    1e-10 bar against the reference's matrix-free path is
    ``test_gpu_trajectory_mf.py``.)

    CG iteration counts must be identical for the inflow cases.  In the closed
    cavity every boundary edge is Dirichlet and the operator keeps a large gauge
    null space, so the preconditioned residual carries a rounding floor; there
    the reference's own ratio eta/threshold at a check can sit within a few per
    cent of 1 (1.0226 at iteration 340 of step 8 of n3_osc), and a different
    rounding order may stop one or two checks earlier or later.  For the cavity
    case each step's count may differ by at most two check intervals.
    """
    g = PU.golden(name)
    env = dict(np.load(PU.GOLDEN / f"oracle_traj_{name}.npz"))
    drv, s, s_old, vc, iters = run_b200(name)
    ref_iters = [int(v) for v in g["tr_hist"][:, 1]]
    if bool(g["cavity"]):
        assert all(abs(a - b) <= 40 for a, b in zip(iters, ref_iters)), (iters, ref_iters)
    else:
        assert iters == ref_iters
    nc = drv.layout.NC
    got = {
        "s": PU.edge_from_dense(name, s),
        "vc": PU.cell3_from_dense(name, vc[:, :nc]),
        "fE": PU.cell3_from_dense(name, np.asarray(drv.ib_force_E)),
        "fL": drv.ib_force_L,
    }
    ref = {"s": g["tr_s"], "vc": g["tr_vc"], "fE": g["tr_fE"], "fL": g["tr_fL"]}
    report = {}
    for k in got:
        e_ref = l2rel(got[k], ref[k])
        e_orc = l2rel(got[k], env[k])
        report[k] = (e_ref, e_orc, float(env["envelope_" + k]))
        assert e_ref <= max(1e-10, 5.0 * float(env["envelope_" + k])), (k, report[k])
        # and the same bar against the oracle's own trajectory of the reference algorithm
        assert e_orc <= max(1e-10, 5.0 * float(env["envelope_" + k])), (k, report[k])
    print(name, "iters", iters, "ref", ref_iters, report)
