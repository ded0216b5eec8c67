"""Golden outputs of the reference's offline pressure recovery.

Run where the reference tree is present, named by ``PYIB_REFERENCE_ROOT``:

    python tests/golden/make_pressure_golden.py

Runs the reference's ``recover_pressure`` (``ib_postprocess.py:49-107``) on

* ``n2``: the cell graph of the 2-level fixed-sphere mesh of ``n2_fixed.npz``
  (cell centres ``geo_cpos``, face pairs ``mesh_F2C``, areas ``geo_Af``: 3240
  cells, 10476 faces, 864 of them on the boundary), with a smooth gradient plus
  seeded noise, so that the projection is not exact;
* ``q9``: the reference's own 9^3 quadratic case (``tests/test_ib_postprocess.py:76-84``).

and writes ``pressure_golden.npz`` with the inputs it needs beyond ``n2_fixed.npz``
and each case's pressure and diagnostics.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parent.parent))
import refharness as R  # noqa: E402
from oracle import pressure_oracle as PO  # noqa: E402  (input builders only)


def n2_inputs():
    g = np.load(HERE / "n2_fixed.npz")
    n = int(g["mesh_ncell"])
    pos = g["geo_cpos"][:n]
    rng = np.random.default_rng(2024)
    grad = PO.quadratic_gradient(pos) + 0.05 * rng.standard_normal((n, 3))
    return pos, g["mesh_F2C"], g["geo_Af"], grad


def main():
    R.import_reference()
    import ib_postprocess as P
    out = {}
    pos, faces, area, grad = n2_inputs()
    p, diag = P.recover_pressure(pos, faces, area, grad)
    out["n2_gradient"] = grad
    out["n2_pressure"] = p
    out["n2_diag"] = json.dumps(diag)
    pos, faces, area = PO.uniform_graph(9, 0.25)
    p, diag = P.recover_pressure(pos, faces, area, PO.quadratic_gradient(pos))
    out["q9_pressure"] = p
    out["q9_diag"] = json.dumps(diag)
    np.savez_compressed(HERE / "pressure_golden.npz", **out)
    print({k: v.shape for k, v in out.items() if hasattr(v, "shape")})


if __name__ == "__main__":
    main()
