"""B200 run directories accepted by the reference's own result validator.

``tests/golden/b200_runs/`` holds the run directories that the B200 case runner
wrote on a B200 for the two reference run cases (``tests/golden/make_b200_runs.py``).
This test loads the reference's ``validate_ib_result.py`` from the tree named by
``PYIB_REFERENCE_ROOT`` (skipped without it), applies in memory the change a
maintainer makes to accept the new device -- the one given in
``INTEGRATION.md``:

* ``config.runtime.device`` may be ``"b200"`` (``validate_ib_result.py:416``);
* its metadata backend is ``"b200/cuda"`` (``validate_ib_result.py:1350``);
* its numerical-source hashes are those of the B200 package's own sources
  (``pyib_b200.case.source_hashes``), checked in place of the reference
  solver files (``validate_ib_result.py:1398-1403``), and the checkpoint's and
  final field's copies of them are checked against the metadata's keys rather
  than the reference's file list (``validate_ib_result.py:821-837``);

and runs ``validate_result`` on each directory: every other check (schema,
fingerprints, history columns and CG evidence, checkpoint and final-field
payloads, load algebra, the Eulerian force and interior momenta recomputed
from the saved fields, the prescribed marker state) is the reference's own.
For cpu and cuda runs the patched validator behaves as the original.
"""
import os
import sys
import types
from pathlib import Path

import pytest

import parity_util as PU

RUNS = PU.GOLDEN / "b200_runs"
ROOT = os.environ.get("PYIB_REFERENCE_ROOT")

pytestmark = pytest.mark.skipif(not ROOT or not (RUNS / "osc_box" / "metadata.json").exists(),
                                reason="needs PYIB_REFERENCE_ROOT and the B200 run fixtures")

# (original, replacement) pairs, each found exactly once in the reference file
PATCH = [
    ('_require(device in {"cpu", "cuda"}, "config.runtime.device must be cpu or cuda")',
     '_require(device in {"cpu", "cuda", "b200"}, "config.runtime.device must be cpu, cuda or b200")'),
    ('expected_backend = "cuda/cupy" if config["runtime"]["device"] == "cuda" else "cpu/numpy"',
     'expected_backend = {"cuda": "cuda/cupy", "b200": "b200/cuda"}.get(config["runtime"]["device"], "cpu/numpy")'),
    ('    _exact_keys(source_hashes, set(SOURCE_FILES), "metadata.source_sha256")\n'
     '    solver_directory = Path(__file__).resolve().parent\n'
     '    for key, filename in SOURCE_FILES.items():\n',
     '    if config["runtime"]["device"] == "b200":\n'
     '        from pyib_b200.case import source_hashes as _b200_sources\n'
     '        _current = _b200_sources()\n'
     '        _exact_keys(source_hashes, set(_current), "metadata.source_sha256")\n'
     '        for key, value in _current.items():\n'
     '            _require(source_hashes[key] == value, f"numerical source hash mismatch for {key}")\n'
     '    else:\n'
     '        _exact_keys(source_hashes, set(SOURCE_FILES), "metadata.source_sha256")\n'
     '    solver_directory = Path(__file__).resolve().parent\n'
     '    for key, filename in (() if config["runtime"]["device"] == "b200" else SOURCE_FILES.items()):\n'),
    ('    _exact_keys(parsed, NUMERICAL_SOURCE_KEYS, label)\n'
     '    validated: dict[str, str] = {}\n'
     '    for key in sorted(NUMERICAL_SOURCE_KEYS):\n',
     '    _exact_keys(parsed, set(metadata_hashes), label)\n'
     '    validated: dict[str, str] = {}\n'
     '    for key in sorted(metadata_hashes):\n'),
    ('            f"{label} disagrees with metadata for {SOURCE_FILES[key]}",\n',
     '            f"{label} disagrees with metadata for {SOURCE_FILES.get(key, key)}",\n'),
]


def _validator(patched):
    path = Path(ROOT) / "src" / "pyib" / "solver" / "validate_ib_result.py"
    src = path.read_text()
    if patched:
        for old, new in PATCH:
            assert src.count(old) == 1, old
            src = src.replace(old, new)
    mod = types.ModuleType("validate_ib_result_under_test")
    mod.__file__ = str(path)
    sys.modules[mod.__name__] = mod
    exec(compile(src, str(path), "exec"), mod.__dict__)
    return mod


@pytest.mark.parametrize("name", ["osc_box", "fixed_concentric"])
def test_reference_validator_accepts_b200_run(name):
    v = _validator(patched=True)
    summary = v.validate_result(RUNS / name)
    assert summary["backend"] == "b200/cuda"
    assert summary["coverage"] == "full_field"
    assert summary["force_balance_max"] <= summary["force_balance_atol"]


def test_patched_validator_still_rejects_a_wrong_backend(tmp_path):
    import json
    import shutil
    v = _validator(patched=True)
    run = tmp_path / "osc_box"
    shutil.copytree(RUNS / "osc_box", run)
    meta = json.loads((run / "metadata.json").read_text())
    meta["backend"] = "cuda/cupy"
    (run / "metadata.json").write_text(json.dumps(meta))
    with pytest.raises(v.ValidationError, match="backend"):
        v.validate_result(run)
