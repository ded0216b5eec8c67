"""Golden trajectories of the reference's ``direct`` IB force mode, explicit and implicit.

Run where the reference tree is present, named by ``PYIB_REFERENCE_ROOT``:

    python tests/golden/make_golden_direct.py

The 2-level fixed sphere of ``n2_fixed`` (h = 0.125, half widths 0.75 and 1.5,
uniform inflow, Re = 100) runs 5 steps of ``Driver.step`` with
``force_mode = "direct"`` (the driver's ``"replacement"``) and ``ib_alpha = 0.5``, once with the explicit force
(``ImmersedBoundary.direct_force``) and once with the implicit one
(``ImmersedBoundary.implicit_force``: the marker coupling matrix M = D S solved
at every inner iteration).  Each ``n2_direct_<kind>.npz`` holds the final fields,
the marker forces and the per-step history.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import refharness as R  # noqa: E402

H, HWS = 0.125, [0.75, 1.5]
KW = dict(inflow=1.0, Re=100.0, dt=0.0625, force_mode="replacement")
STEPS, ALPHA = 5, 0.5


def generate(kind):
    R.import_reference()
    case = R.RefCase(H, HWS, **KW)
    drv = case.driver
    drv.ib_implicit = kind == "implicit"
    drv.ib_alpha = ALPHA
    hist = []

    def cb(step, s, s_old, vc, load):
        hist.append([step, drv.helmholtz_iterations_last_step, drv.ib_force_updates_last_step])

    s, s_old, vc = case.run(STEPS, cb)
    nc = case.core.ncell
    out = dict(tr_s=s, tr_s_old=s_old, tr_vc=vc[:nc], tr_fE=np.asarray(drv.ib_force_E),
               tr_fL=np.asarray(drv.ib_force_L), tr_hist=np.asarray(hist), tr_steps=np.int64(STEPS),
               alpha=np.float64(ALPHA), implicit=np.bool_(kind == "implicit"),
               params_json=np.bytes_(json.dumps(dict(h=H, half_widths=HWS, steps=STEPS, alpha=ALPHA,
                                                     kind=kind, **KW))))
    np.savez_compressed(HERE / f"n2_direct_{kind}.npz", **out)
    print(kind, "iters", [int(r[1]) for r in hist], "updates", [int(r[2]) for r in hist])


if __name__ == "__main__":
    for k in sys.argv[1:] or ["explicit", "implicit"]:
        generate(k)
