"""Trajectory fixtures from the oracle (the reference algorithm run matrix-free).

    python tests/golden/make_oracle_traj.py [case ...]

The reference's goldens (make_golden.py) were produced with its CSR matvec
(``solver.sparse = true``); the oracle applies the same operator matrix-free
(``IBCore.flow_mat``, the reference's ``sparse = false`` path).  The two float64
runs of the same algorithm differ only by rounding order; their difference
after the trajectory is the reference's own reproducibility envelope, stored
here as ``envelope_*`` next to the oracle's fields.
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
import pyib_oracle as O  # noqa: E402


def l2rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def run(name):
    d = dict(np.load(HERE / f"{name}.npz"))
    import json
    par = json.loads(bytes(d["params_json"]).decode())
    m = O.MeshDesc.from_npz(d)
    drv = O.OracleDriver(m, float(d["visc"]), float(d["rou"]), cavity=bool(d["cavity"]))
    ib = O.IBStencil(m)
    ref, ds = d["ref_markers"], d["ib_ds"]
    amp = float(par.get("amplitude", 0.0))
    if amp:
        mo = O.Oscillation(ref, par["axis"], amp, par["frequency"], par["phase"])
        mk0, v0 = mo(0.0)
        drv.set_ib(ib, mk0, ds, v0)
        drv.set_motion(mo, 0.0)
    else:
        drv.set_ib(ib, ref, ds, np.zeros_like(ref))
    geo = drv.g
    s = float(par.get("inflow", 1.0)) * geo.epos[:, 1] * geo.te[:, 2]
    s, _, vc = drv.calc_vel(s)
    so = s.copy()
    dt = float(d["dt"])
    its = []
    for k in range(1, int(d["tr_steps"]) + 1):
        drv.time = (k - 1) * dt
        s, vc, so = drv.step(s, so, dt, dt, 4)
        drv.time = k * dt
        its.append(max(st.iterations for st in drv.last_stats))
    nc = m.ncell
    U = geo.curl(s)
    out = dict(s=s, s_old=so, vc=vc[:nc], U=U, fE=drv.fE, fL=drv.fL, iters=np.array(its))
    env = {}
    for k, ref_key in (("s", "tr_s"), ("vc", "tr_vc"), ("fE", "tr_fE"), ("fL", "tr_fL")):
        env["envelope_" + k] = np.float64(l2rel(out[k], d[ref_key]))
    env["envelope_U"] = np.float64(l2rel(U, geo.curl(d["tr_s"])))
    np.savez_compressed(HERE / f"oracle_traj_{name}.npz", **out, **env)
    print(name, {k: float(v) for k, v in env.items()}, "iters equal",
          its == [int(v) for v in d["tr_hist"][:, 1]])


if __name__ == "__main__":
    for n in sys.argv[1:] or ["u1_fixed", "n2_fixed", "n3_osc"]:
        run(n)
