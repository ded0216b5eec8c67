"""Record the reference's own run-to-run spread in a matrix-free trajectory golden.

    python tests/golden/add_self_spread.py CASE OTHER_RUN.npz [STRIDE]

``OTHER_RUN.npz`` is the same case produced by ``make_golden_mf.py`` with one
BLAS thread (``OPENBLAS_NUM_THREADS=1``); the golden itself was produced with
the default thread count.  NumPy's ``dot`` (the CG inner products of
``ib_driver_np.py:389,396``) sums in a different order with a different thread
count, so the two runs of the unmodified reference differ by rounding alone.
Their relative L2 differences of s, vc, fE and fL after the last step are
stored as ``spread_*``: the float64 reproducibility of the reference itself,
which the GPU test uses as the bar for the sensitive force fields.

With ``STRIDE`` > 1 the golden then keeps every STRIDE-th entry of s and of vc
(``s_stride``, ``vc_stride``; the spreads are those of the whole fields), so
that a case of a few hundred thousand cells stays a fixture of a few MB.
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def l2rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


if __name__ == "__main__":
    name, other = sys.argv[1], sys.argv[2]
    stride = int(sys.argv[3]) if len(sys.argv) > 3 else 1
    g = dict(np.load(HERE / f"{name}.npz"))
    o = np.load(other)
    if "s_stride" in g:
        raise SystemExit("this golden keeps thinned fields; regenerate it first")
    if not np.array_equal(g["fE_idx"], o["fE_idx"]):
        raise SystemExit("the two runs have different force supports")
    spread = {"spread_s": l2rel(o["s"], g["s"]), "spread_vc": l2rel(o["vc"], g["vc"]),
              "spread_fE": l2rel(o["fE_val"], g["fE_val"]), "spread_fL": l2rel(o["fL"], g["fL"])}
    g.update({k: np.float64(v) for k, v in spread.items()})
    g["spread_iters_equal"] = np.bool_(np.array_equal(g["solve_iters"], o["solve_iters"]))
    # largest difference of one step's total CG iterations between the two reference runs
    g["spread_iters_maxdiff"] = np.int64(np.max(np.abs(g["solve_iters"].sum(1) - o["solve_iters"].sum(1))))
    if stride > 1:
        g["s"], g["vc"] = g["s"][::stride].copy(), g["vc"][:, ::stride].copy()
        g["s_stride"], g["vc_stride"] = np.int64(stride), np.int64(stride)
    np.savez_compressed(HERE / f"{name}.npz", **g)
    print(name, spread, "iterations equal:", bool(g["spread_iters_equal"]))
