"""B200 run directories of the two reference run cases, for the validator check.

Run on a machine with a B200 (the case runner has no CPU path):

    python tests/golden/make_b200_runs.py OUTDIR

Runs ``pyib_b200.case.run_case`` on the configurations of
``run_artifacts.json`` (``osc_box``, ``fixed_concentric``) with
``runtime.device = "b200"`` and writes each run directory (metadata, history,
checkpoint, final field, snapshots) under ``OUTDIR``.  Copied into
``tests/golden/b200_runs/``, they are checked on the CPU by the reference's own
result validator (``tests/test_validate_b200_runs.py``).
"""
from __future__ import annotations

import json
import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
import _pyib_b200_import  # noqa: E402

_pyib_b200_import.load()
from pyib_b200 import case as CASE  # noqa: E402


def main(out: Path):
    gold = json.loads((HERE / "run_artifacts.json").read_text())
    out.mkdir(parents=True, exist_ok=True)
    for name in sorted(gold):
        cfg = json.loads(json.dumps(gold[name]["config"]))
        cfg["runtime"]["device"] = "b200"
        run = out / name
        if run.exists():
            shutil.rmtree(run)
        CASE.run_case(cfg, run, quiet=True)
        print(name, sorted(p.name for p in run.rglob("*") if p.is_file()))


if __name__ == "__main__":
    main(Path(sys.argv[1]))
