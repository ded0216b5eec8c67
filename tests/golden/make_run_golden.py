"""Reference run artefacts: history, metadata, checkpoint and field snapshots of small cases.

    PYIB_REFERENCE_ROOT=<reference tree> python tests/golden/make_run_golden.py

Runs the unmodified reference CLI (``solver/cfdagent_ib.py``, CPU backend,
float64) in a fresh process per case, exactly as ``pyib-run CASE.json --outdir
RUN`` does, and records what ``ib_case.run_case`` (``ib_case.py:1413-1648``)
wrote: every ``history.csv`` row (41 columns, ``ib_case.py:112-154``), the
metadata keys (``ib_case.py:1331-1366``), the schema-3 checkpoint payload keys
and scalar values (``ib_case.py:823-870``) and the field-snapshot keys
(``ib_case.py:879-911``).  The case runner of the B200 path is checked against
these values on the GPU (``tests/test_gpu_run_artifacts.py``).

Cases (JSON in ``run_cases.json``):

* ``osc_box`` -- the reference's ``examples/cpu_oscillating_sphere_smoke.json``
  (uniform 8^3 box, oscillating sphere, 4 steps), with field snapshots every
  2 steps;
* ``fixed_concentric`` -- the reference's nested 5-level preset
  (``sphere_concentric``, 8 cells per diameter, 18,432 cells), fixed sphere in
  uniform inflow, 3 steps, matrix-free operator.
"""
from __future__ import annotations

import csv
import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import refharness  # noqa: E402

CASES = {
    "osc_box": {
        "schema_version": 1, "name": "osc_box", "case": {"kind": "oscillating_sphere"},
        "runtime": {"device": "cpu", "precision": "float64"},
        "mesh": {"kind": "uniform_box", "dx": 0.25, "bounds": [[-1.0, 1.0], [-1.0, 1.0], [-1.0, 1.0]],
                 "verbose": False},
        "physics": {"reynolds": 100.0, "density": 1.0, "inflow_speed": 1.0},
        "time": {"dt": 0.01, "steps": 4, "inner_iterations": 4},
        "ib": {"radius": 0.25, "center": [0.0, 0.0, 0.0], "marker_spacing": 0.25,
               "force_mode": "accumulated_explicit", "implicit": False, "alpha": 1.0,
               "motion": {"kind": "oscillation", "axis": [0.0, 1.0, 0.0], "amplitude": 0.05,
                          "frequency": 0.5, "phase": 0.0}},
        "solver": {"sparse": True},
        "output": {"sample_every": 1, "checkpoint_every": 2, "field_every": 2, "save_field": True},
    },
    "fixed_concentric": {
        "schema_version": 1, "name": "fixed_concentric", "case": {"kind": "fixed_sphere"},
        "runtime": {"device": "cpu", "precision": "float64"},
        "mesh": {"kind": "sphere_concentric", "cells_per_diameter": 8, "verbose": False},
        "physics": {"reynolds": 100.0, "density": 1.0, "inflow_speed": 1.0},
        "time": {"dt": 0.025, "steps": 3, "inner_iterations": 4},
        "ib": {"radius": 0.25, "center": [0.0, 0.0, 0.0], "marker_spacing": 0.0625,
               "force_mode": "accumulated_explicit", "implicit": False, "alpha": 1.0,
               "motion": {"kind": "none", "axis": [0.0, 1.0, 0.0], "amplitude": 0.0,
                          "frequency": 1.0, "phase": 0.0}},
        "solver": {"sparse": False},
        "output": {"sample_every": 1, "checkpoint_every": 1000, "save_field": True},
    },
}


def _describe_npz(path):
    out = {}
    with np.load(path, allow_pickle=False) as d:
        for k in sorted(d.files):
            a = d[k]
            entry = {"dtype": a.dtype.kind, "shape": list(a.shape)}
            if a.ndim == 0:
                entry["value"] = a.item() if a.dtype.kind in "iufb" else str(a)
            out[k] = entry
    return out


def run(name, cfg, workdir):
    root = refharness.reference_root()
    case = Path(workdir) / f"{name}.json"
    case.write_text(json.dumps(cfg))
    outdir = Path(workdir) / name
    stubs = Path(workdir) / "stubs"
    stubs.mkdir(exist_ok=True)
    (stubs / "h5py.py").write_text("")
    (stubs / "meshio.py").write_text("")
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join([str(stubs), str(root / "src" / "pyib"),
                                         str(root / "src" / "pyib" / "solver"), str(root / "src")])
    code = ("import sys; sys.argv.append('--nometis'); import cfdagent_ib; "
            f"raise SystemExit(cfdagent_ib.main([{str(case)!r}, '--outdir', {str(outdir)!r}, '--quiet']))")
    subprocess.run([sys.executable, "-c", code], check=True, env=env)
    with (outdir / "history.csv").open() as fh:
        rows = list(csv.reader(fh))
    header, body = rows[0], np.asarray([[float(v) for v in r] for r in rows[1:]])
    meta = json.loads((outdir / "metadata.json").read_text())
    snaps = sorted(p.name for p in (outdir / "snapshots").glob("field_*.npz")) \
        if (outdir / "snapshots").exists() else []
    rec = {
        "config": cfg,
        "history_header": header,
        "history": body.tolist(),
        "metadata_keys": sorted(meta),
        "metadata_backend": meta["backend"],
        "metadata_mesh": meta["mesh"],
        "checkpoint": _describe_npz(outdir / "checkpoint.npz"),
        "final_field": _describe_npz(outdir / "final_field.npz") if (outdir / "final_field.npz").exists() else None,
        "snapshots": snaps,
        "snapshot": _describe_npz(outdir / "snapshots" / snaps[0]) if snaps else None,
    }
    return rec


if __name__ == "__main__":
    out = {}
    with tempfile.TemporaryDirectory(prefix="pyib_run_golden_") as wd:
        for name, cfg in CASES.items():
            out[name] = run(name, cfg, wd)
            print(name, "rows", len(out[name]["history"]), "checkpoint keys", len(out[name]["checkpoint"]))
    (HERE / "run_artifacts.json").write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")
