"""Oracle trajectories of the ``direct`` IB force mode and their envelope against the reference.

    python tests/golden/make_oracle_direct.py

Runs the oracle on the 2-level fixed sphere of ``n2_direct_<kind>.npz`` (made by
``make_golden_direct.py`` from the reference) and stores its final fields next to
``envelope_*``: the oracle's relative difference from the reference's own run,
i.e. the reproducibility envelope of the same algorithm under a different
rounding order (the reference assembles CSR operators and inverts the marker
coupling matrix densely; the oracle applies the operators matrix-free).
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
for p in (ROOT, ROOT / "oracle", ROOT / "tests"):
    sys.path.insert(0, str(p))
import _pyib_b200_import  # noqa: E402

_pyib_b200_import.load()
from test_oracle_direct import run_oracle_direct  # noqa: E402


def main(kinds):
    for kind in kinds:
        d, drv, s, vc, its = run_oracle_direct(kind)
        nc = drv.g.ncell
        fields = {"s": (s, "tr_s"), "vc": (vc[:nc], "tr_vc"), "fE": (drv.fE, "tr_fE"), "fL": (drv.fL, "tr_fL")}
        env = {"envelope_" + k: np.float64(np.linalg.norm(v - d[key]) / np.linalg.norm(d[key]))
               for k, (v, key) in fields.items()}
        np.savez_compressed(HERE / f"oracle_direct_{kind}.npz", **{k: v for k, (v, _) in fields.items()}, **env)
        print(kind, {k: float(v) for k, v in env.items()})


if __name__ == "__main__":
    main(sys.argv[1:] or ["explicit", "implicit"])
