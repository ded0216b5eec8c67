"""Record the reference's own run-to-run spread in a matrix-free trajectory golden.

    python tests/golden/add_self_spread.py CASE OTHER_RUN.npz [OTHER_RUN.npz ...] [--stride=K]

Each ``OTHER_RUN.npz`` is the same case produced by ``make_golden_mf.py`` with
another BLAS thread count (``OPENBLAS_NUM_THREADS=1``, 2, 3, ...); the golden
itself was produced with the default thread count.  NumPy's ``dot`` (the CG
inner products of ``ib_driver_np.py:389,396``) sums in a different order with a
different thread count, so runs of the unmodified reference differ by rounding
alone.  For each of s, vc, fE and fL after the last step, the largest relative
L2 difference between the golden and any other run is stored as ``spread_*``:
the float64 reproducibility of the reference itself, which the GPU test uses
as the bar for the sensitive force fields.  ``spread_runs`` counts the other
runs.

With ``--stride=K`` (K > 1) the golden then keeps every K-th entry of s and of
vc (``s_stride``, ``vc_stride``; the spreads are those of the whole fields), so
that a case of a few hundred thousand cells stays a fixture of a few MB.  On
a thinned golden the spreads of s and vc are taken over the kept entries.
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def l2rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


if __name__ == "__main__":
    opts = [a for a in sys.argv[1:] if a.startswith("--")]
    pos = [a for a in sys.argv[1:] if not a.startswith("--")]
    name, others = pos[0], pos[1:]
    stride = 1
    for a in opts:
        if a.startswith("--stride="):
            stride = int(a.split("=", 1)[1])
        else:
            raise SystemExit(f"unknown option {a}")
    if not others:
        raise SystemExit("give at least one other run")
    g = dict(np.load(HERE / f"{name}.npz"))
    # a golden already thinned keeps its stride; the other runs are compared on it
    ss, vs = int(g.get("s_stride", 1)), int(g.get("vc_stride", 1))
    if (ss > 1 or vs > 1) and stride > 1:
        raise SystemExit("this golden is thinned already")
    spread = {"spread_s": 0.0, "spread_vc": 0.0, "spread_fE": 0.0, "spread_fL": 0.0}
    iters_equal, maxdiff = True, 0
    for other in others:
        o = np.load(other)
        if not np.array_equal(g["fE_idx"], o["fE_idx"]):
            raise SystemExit(f"{other}: different force support")
        one = {"spread_s": l2rel(o["s"][::ss], g["s"]), "spread_vc": l2rel(o["vc"][:, ::vs], g["vc"]),
               "spread_fE": l2rel(o["fE_val"], g["fE_val"]), "spread_fL": l2rel(o["fL"], g["fL"])}
        print(other, one)
        spread = {k: max(spread[k], one[k]) for k in spread}
        iters_equal &= bool(np.array_equal(g["solve_iters"], o["solve_iters"]))
        # largest difference of one step's total CG iterations between two reference runs
        maxdiff = max(maxdiff, int(np.max(np.abs(g["solve_iters"].sum(1) - o["solve_iters"].sum(1)))))
    g.update({k: np.float64(v) for k, v in spread.items()})
    g["spread_runs"] = np.int64(len(others))
    g["spread_iters_equal"] = np.bool_(iters_equal)
    g["spread_iters_maxdiff"] = np.int64(maxdiff)
    if stride > 1:
        g["s"], g["vc"] = g["s"][::stride].copy(), g["vc"][:, ::stride].copy()
        g["s_stride"], g["vc_stride"] = np.int64(stride), np.int64(stride)
    np.savez_compressed(HERE / f"{name}.npz", **g)
    print(name, spread, "iterations equal:", iters_equal)
