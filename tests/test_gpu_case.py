"""The JSON case runner on the GPU: history, checkpoint and an exact resume."""
import json

import numpy as np
import pytest

from pyib_b200 import case as CS

pytestmark = pytest.mark.gpu

OSC = {
    "schema_version": 1, "name": "osc", "case": {"kind": "oscillating_sphere"},
    "runtime": {"device": "b200", "precision": "float64"},
    "mesh": {"kind": "nested_boxes", "cells_per_diameter": 8, "half_widths_d": [1.5, 3.0]},
    "physics": {"reynolds": 0.2, "density": 1.0, "inflow_speed": 0.0},
    "time": {"dt": 0.00872664626, "steps": 6, "inner_iterations": 4},
    "ib": {"radius": 0.25, "center": [0, 0, 0], "marker_spacing": 0.0625,
           "motion": {"kind": "oscillation", "axis": [1, 0, 0], "amplitude": 0.1,
                      "frequency": 0.5729577951, "phase": -1.5707963268}},
    "solver": {"cg_max_iterations": 5000},
    "output": {"sample_every": 1, "checkpoint_every": 3},
}


def test_run_and_resume_reproduce_the_straight_run(tmp_path):
    straight = CS.run_case(OSC, tmp_path / "a", quiet=True)
    rows = list(__import__("csv").DictReader(open(tmp_path / "a" / "history.csv")))
    assert [int(r["step"]) for r in rows] == [1, 2, 3, 4, 5, 6]
    assert all(float(r["force_balance_relerr"]) < 1e-9 for r in rows)
    # stop after 3 steps, then resume to 6
    first = json.loads(json.dumps(OSC))
    first["time"]["steps"] = 3
    CS.run_case(first, tmp_path / "b", quiet=True)
    resumed = CS.run_case(OSC, tmp_path / "b", resume=True, quiet=True)
    assert resumed["completed_step"] == 6
    a = np.load(tmp_path / "a" / "checkpoint.npz")
    b = np.load(tmp_path / "b" / "checkpoint.npz")
    for k in ("s", "s_old", "ib_force_E", "ib_force_L", "force_fluid", "interior_momentum",
              "interior_angular_momentum", "body_force"):
        assert np.array_equal(a[k], b[k]), k                 # deterministic kernels: bit-identical
    assert np.array_equal(straight["body_force"], resumed["body_force"])


def test_resume_rejects_other_configuration(tmp_path):
    cfg = json.loads(json.dumps(OSC))
    cfg["time"]["steps"] = 3
    CS.run_case(cfg, tmp_path, quiet=True)
    other = json.loads(json.dumps(OSC))
    other["physics"]["reynolds"] = 0.5
    with pytest.raises(CS.CaseConfigError, match="different configuration"):
        CS.run_case(other, tmp_path, resume=True, quiet=True)
