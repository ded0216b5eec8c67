"""The case runner's artefacts against the reference's own run of the same JSON cases.

``tests/golden/run_artifacts.json`` holds what the unmodified reference CLI
wrote for two small cases (``tests/golden/make_run_golden.py``): every history
row, the metadata keys, the schema-3 checkpoint payload and the field
snapshots.  The B200 runner gets the same configurations with
``runtime.device = "b200"``; its history must carry the same 41 columns and
values, its checkpoint and snapshots the same keys, shapes and scalar values.
"""
import csv
import json

import numpy as np
import pytest

import parity_util as PU
from pyib_b200 import case as CASE

pytestmark = pytest.mark.gpu

GOLD = json.loads((PU.GOLDEN / "run_artifacts.json").read_text())

# history columns compared with a relative tolerance against the column's scale;
# the rest: exact (counts) or skipped (wall-clock timing)
EXACT = {"step", "ib_force_updates", "helmholtz_iterations"}
SKIP = {"milliseconds_per_step"}
LOOSE = {"helmholtz_relative_residual": 1e-3, "helmholtz_tolerance_ratio": 1e-3}
ROUNDING = {"mass_residual_inf": 1e-12, "force_balance_relerr": 1e-12}   # rounding-level values


def _config(name):
    cfg = json.loads(json.dumps(GOLD[name]["config"]))
    cfg["runtime"]["device"] = "b200"
    return cfg


def _history(path):
    with open(path, newline="") as fh:
        rows = list(csv.reader(fh))
    return rows[0], np.asarray([[float(v) for v in r] for r in rows[1:]])


def _npz_desc(path):
    with np.load(path, allow_pickle=False) as d:
        return {k: (d[k].dtype.kind, list(d[k].shape), d[k].item() if d[k].ndim == 0 else None)
                for k in d.files}


@pytest.mark.parametrize("name", sorted(GOLD))
def test_history_and_artifacts_match_reference(name, tmp_path):
    g = GOLD[name]
    out = tmp_path / name
    CASE.run_case(_config(name), out, quiet=True)
    header, got = _history(out / "history.csv")
    assert header == g["history_header"] == CASE.HISTORY_COLUMNS
    ref = np.asarray(g["history"])
    assert got.shape == ref.shape
    for c, col in enumerate(header):
        if col in SKIP:
            continue
        a, b = got[:, c], ref[:, c]
        if col in EXACT:
            assert np.array_equal(a, b), (col, a, b)
        elif col in ROUNDING:
            assert np.all(np.abs(a) <= ROUNDING[col]) and np.all(np.abs(b) <= ROUNDING[col]), (col, a, b)
        else:
            tol = LOOSE.get(col, 1e-8)
            scale = max(float(np.max(np.abs(b))), 1e-300)
            assert np.max(np.abs(a - b)) <= tol * scale, (col, a, b)
    meta = json.loads((out / "metadata.json").read_text())
    assert set(meta) == set(g["metadata_keys"])
    assert meta["backend"] == "b200/cuda" and meta["complete"] is True
    assert meta["mesh"]["edges"] == g["metadata_mesh"]["edges"]
    assert meta["mesh"]["faces"] == g["metadata_mesh"]["faces"]
    # checkpoint: the reference's payload keys, kinds and shapes; its scalars
    ck = _npz_desc(out / "checkpoint.npz")
    assert set(ck) == set(g["checkpoint"])
    for k, ent in g["checkpoint"].items():
        kind, shape, val = ck[k]
        assert shape == ent["shape"], (k, shape, ent["shape"])
        assert (kind in "iu") == (ent["dtype"] in "iu") and (kind == "f") == (ent["dtype"] == "f"), k
        if k in ("checkpoint_schema", "update_phase", "step", "dt", "previous_dt", "precision",
                 "ib_force_mode", "ib_force_update_count"):
            assert val == ent["value"], (k, val, ent["value"])
        if k == "physical_time":
            assert abs(val - ent["value"]) <= 1e-15
        if k == "interior_indicator_volume":
            assert abs(val - ent["value"]) <= 1e-12 * abs(ent["value"])
    assert ck["device"][2] == "b200"
    # field snapshots
    snaps = sorted(p.name for p in (out / "snapshots").glob("field_*.npz")) \
        if (out / "snapshots").exists() else []
    assert snaps == g["snapshots"]
    ff = _npz_desc(out / "final_field.npz")
    assert set(ff) == set(g["final_field"])
    for k, ent in g["final_field"].items():
        assert ff[k][1] == ent["shape"], (k, ff[k][1], ent["shape"])
    if g["snapshot"] is not None:
        sn = _npz_desc(out / "snapshots" / snaps[0])
        assert set(sn) == set(g["snapshot"])


def test_resume_continues_bit_identically(tmp_path):
    """Two steps, stop, resume to four: the same state as four steps in one run."""
    name = "osc_box"
    cfg4 = _config(name)
    straight = tmp_path / "straight"
    CASE.run_case(cfg4, straight, quiet=True)
    cfg2 = _config(name)
    cfg2["time"]["steps"] = 2
    split = tmp_path / "split"
    CASE.run_case(cfg2, split, quiet=True)
    CASE.run_case(cfg4, split, resume=True, quiet=True)
    with np.load(straight / "checkpoint.npz") as a, np.load(split / "checkpoint.npz") as b:
        for k in ("s", "s_old", "ib_force_E", "ib_force_L", "body_force", "interior_momentum_rate"):
            assert np.array_equal(a[k], b[k]), k
    h1 = _history(straight / "history.csv")[1]
    h2 = _history(split / "history.csv")[1]
    keep = [i for i, c in enumerate(CASE.HISTORY_COLUMNS) if c != "milliseconds_per_step"]
    assert np.array_equal(h1[:, keep], h2[:, keep])
    meta = json.loads((split / "metadata.json").read_text())
    assert meta["resume_count"] == 1 and meta["start_step"] == 2


def test_resume_rejects_other_configuration(tmp_path):
    name = "osc_box"
    cfg2 = _config(name)
    cfg2["time"]["steps"] = 2
    out = tmp_path / "run"
    CASE.run_case(cfg2, out, quiet=True)
    other = _config(name)
    other["physics"]["reynolds"] = 50.0
    with pytest.raises(CASE.CaseConfigError):
        CASE.run_case(other, out, resume=True, quiet=True)
