"""Golden outputs of the reference's pressure band repair.

Run where the reference tree is present, named by ``PYIB_REFERENCE_ROOT``:

    python tests/golden/make_band_golden.py

Runs the reference's ``repair_pressure_band`` (``ib_postprocess.py:213-250``) on
lattices built by ``pressure_oracle.band_case`` (inputs only):

* ``q17``: the reference's own case (``tests/test_ib_postprocess.py:86-95``):
  17^3 cells of 0.25, sphere of radius 0.6, quadratic truth with a defect on
  the band, exact gradient, width 1.5 h;
* ``n40``: 40^3 cells of 1/16, the same sphere, the gradient with seeded noise
  (0.05, seed 7) so that the band's equations are inconsistent, 2 % of the raw
  values NaN (seed 7), widths 1.5 h and 2.5 h;
* the two rejections: a width that swallows every valid cell (no anchor) and a
  sphere that leaves no cell in the band.

and writes ``band_golden.npz``: for each case the target mask, the repaired
values on it, the lsqr iteration count, and the error messages.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parent.parent))
import refharness as R  # noqa: E402
from oracle import pressure_oracle as PO  # noqa: E402  (input builders only)

CASES = {
    "q17": dict(count=17, spacing=0.25, width=1.5),
    "n40w15": dict(count=40, spacing=1.0 / 16, width=1.5, noise=0.05, seed=7, holes=0.02),
    "n40w25": dict(count=40, spacing=1.0 / 16, width=2.5, noise=0.05, seed=7, holes=0.02),
}


def lattice(P, count, spacing):
    ids = np.arange(count ** 3).reshape((count,) * 3)
    return P.UniformLattice(ids, np.full(3, -0.5 * (count - 1) * spacing), spacing)


def main():
    R.import_reference()
    import ib_postprocess as P
    out = {}
    for name, c in CASES.items():
        kw = {k: c[k] for k in ("noise", "seed", "holes") if k in c}
        _, dist, _, raw, grad = PO.band_case(c["count"], c["spacing"], **kw)
        rep, target, it = P.repair_pressure_band(lattice(P, c["count"], c["spacing"]), raw, grad, dist,
                                                 width=c["width"])
        out[f"{name}_target"] = target
        out[f"{name}_values"] = rep[target]
        out[f"{name}_iterations"] = np.int64(it)
        print(name, int(target.sum()), "cells,", it, "lsqr iterations")
    _, dist, _, raw, grad = PO.band_case(17, 0.25)
    for key, (d, width) in {"unanchored": (dist, 100.0), "empty": (dist + 10.0, 1.5)}.items():
        try:
            P.repair_pressure_band(lattice(P, 17, 0.25), raw, grad, d, width=width)
            raise SystemExit(f"{key}: the reference accepted it")
        except ValueError as e:
            out[f"{key}_message"] = str(e)
            print(key, e)
    np.savez_compressed(HERE / "band_golden.npz", **out)


if __name__ == "__main__":
    main()
