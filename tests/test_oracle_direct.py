"""The oracle's ``direct`` IB force mode (explicit and implicit) against the reference."""
import json

import numpy as np
import pytest

import pyib_oracle as O
import parity_util as PU


def run_oracle_direct(kind):
    g = PU.golden("n2_fixed")
    d = dict(np.load(PU.GOLDEN / f"n2_direct_{kind}.npz"))
    m = O.MeshDesc.from_npz(g)
    drv = O.OracleDriver(m, float(g["visc"]), float(g["rou"]), cavity=False)
    ib = O.IBStencil(m)
    ref = g["ref_markers"]
    drv.set_ib(ib, ref, g["ib_ds"], np.zeros_like(ref), force_mode="replacement",
               implicit=bool(d["implicit"]), alpha=float(d["alpha"]))
    geo = drv.g
    s = geo.epos[:, 1] * geo.te[:, 2]
    s, _, vc = drv.calc_vel(s)
    so = s.copy()
    dt = float(g["dt"])
    its = []
    for k in range(1, int(d["tr_steps"]) + 1):
        drv.time = (k - 1) * dt
        s, vc, so = drv.step(s, so, dt, dt, 4)
        drv.time = k * dt
        its.append(max(st.iterations for st in drv.last_stats))
    return d, drv, s, vc, its


@pytest.mark.parametrize("kind", ["explicit", "implicit"])
def test_oracle_direct_mode_matches_reference(kind):
    d, drv, s, vc, its = run_oracle_direct(kind)
    assert its == [int(v) for v in d["tr_hist"][:, 1]]
    nc = drv.g.ncell
    for got, key in ((s, "tr_s"), (vc[:nc], "tr_vc"), (drv.fE, "tr_fE"), (drv.fL, "tr_fL")):
        want = d[key]
        assert np.linalg.norm(got - want) <= 1e-9 * np.linalg.norm(want), key
