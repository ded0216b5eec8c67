"""Case configuration: the reference's schema v1 with the b200 device (no GPU needed)."""
import json

import numpy as np
import pytest

from pyib_b200 import case as CS

SMOKE = {
    "schema_version": 1, "name": "smoke", "case": {"kind": "fixed_sphere"},
    "runtime": {"device": "b200", "precision": "float64"},
    "mesh": {"kind": "uniform_box", "dx": 0.25, "bounds": [[-1, 1], [-1, 1], [-1, 1]]},
    "physics": {"reynolds": 100.0, "density": 1.0, "inflow_speed": 1.0},
    "time": {"dt": 0.01, "steps": 5, "inner_iterations": 4},
    "ib": {"radius": 0.25, "center": [0, 0, 0], "marker_spacing": 0.25},
    "output": {"sample_every": 1, "checkpoint_every": 2},
}


def test_defaults_and_normalisation():
    cfg = CS.validate_config(SMOKE)
    assert cfg["solver"]["cg_check_interval"] == 20
    assert cfg["ib"]["motion"]["axis"] == [0.0, 1.0, 0.0]
    assert "mixed_tolerance" not in cfg["runtime"]          # float64: the reference's runtime keys
    mixed = json.loads(json.dumps(SMOKE))
    mixed["runtime"]["precision"] = "mixed"
    assert CS.validate_config(mixed)["runtime"]["mixed_tolerance"] == pytest.approx(0.1)


@pytest.mark.parametrize("patch, msg", [
    ({"runtime": {"device": "cuda"}}, "b200"),
    ({"runtime": {"precision": "float32"}}, "precision"),
    ({"mesh": {"kind": "uniform_box", "dx": 0.3, "bounds": [[-1, 1], [-1, 1], [-1, 1]]}}, "multiples"),
    ({"time": {"inner_iterations": 1}}, "two fluid inner"),
    ({"ib": {"force_mode": "replacement"}}, "force_mode must be"),
    ({"ib": {"implicit": True}}, "explicit IB method"),
    ({"ib": {"alpha": 0.5}}, "alpha=1.0"),
    ({"ib": {"force_mode": "direct", "implicit": True, "alpha": 0.9}}, "alpha <= 0.7"),
    ({"case": {"kind": "oscillating_sphere"}}, "requires ib.motion.kind"),
    ({"bogus": 1}, "unknown key"),
    ({"mesh": {"kind": "nested_boxes", "cells_per_diameter": 8}}, "half_widths_d"),
])
def test_rejections(patch, msg):
    raw = json.loads(json.dumps(SMOKE))
    for k, v in patch.items():
        if isinstance(v, dict) and isinstance(raw.get(k), dict):
            raw[k].update(v)
        else:
            raw[k] = v
    with pytest.raises(CS.CaseConfigError, match=msg):
        CS.validate_config(raw)


def test_direct_force_mode_is_accepted():
    raw = json.loads(json.dumps(SMOKE))
    raw["ib"].update({"force_mode": "direct", "implicit": True, "alpha": 0.5})
    raw["time"]["inner_iterations"] = 1
    cfg = CS.validate_config(raw)
    assert cfg["ib"]["force_mode"] == "direct" and cfg["ib"]["implicit"] and cfg["ib"]["alpha"] == 0.5


def test_fingerprint_ignores_output_and_steps():
    a = CS.validate_config(SMOKE)
    b = json.loads(json.dumps(SMOKE))
    b["time"]["steps"] = 50
    b["output"]["sample_every"] = 7
    b["name"] = "other"
    assert CS.config_fingerprint(a) == CS.config_fingerprint(CS.validate_config(b))
    c = json.loads(json.dumps(SMOKE))
    c["physics"]["reynolds"] = 50.0
    assert CS.config_fingerprint(a) != CS.config_fingerprint(CS.validate_config(c))


def test_layouts_of_mesh_kinds():
    wake = dict(SMOKE, mesh={"kind": "sphere_wake", "cells_per_diameter": 8})
    lay, h, fine = CS.build_layout(CS.validate_config(wake))
    assert lay.N == 4 and h == pytest.approx(0.0625)
    assert np.allclose(fine[0], [-0.5, 1.5])
    conc = dict(SMOKE, mesh={"kind": "sphere_concentric", "cells_per_diameter": 8})
    lay, h, _ = CS.build_layout(CS.validate_config(conc))
    assert lay.N == 5 and [int(v) for v in lay.levels[0].n] == [16, 16, 16]
    nb = dict(SMOKE, mesh={"kind": "nested_boxes", "cells_per_diameter": 32, "half_widths_d": [2, 4, 8]})
    lay, h, _ = CS.build_layout(CS.validate_config(nb))
    assert [int(lv.n[0]) for lv in lay.levels] == [128, 128, 128]
