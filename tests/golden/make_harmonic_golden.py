"""Golden values for the force harmonic fit, from the reference's own check tool.

Run where the reference tree is present, named by ``PYIB_REFERENCE_ROOT``:

    python tests/golden/make_harmonic_golden.py

Imports ``fit`` from ``tools/check_pressure_validation.py`` (it imports no PyIB
code) and evaluates it on a seeded synthetic axial force history; the inputs
and the reference's coefficients and residual go to ``harmonic_fit.json``.
"""
import importlib.util
import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import refharness  # noqa: E402

REF = refharness.reference_root()

spec = importlib.util.spec_from_file_location("check_pressure_validation",
                                              REF / "tools" / "check_pressure_validation.py")
tool = importlib.util.module_from_spec(spec)
spec.loader.exec_module(tool)

rng = np.random.default_rng(11)
omega, phase = 3.6, -np.pi / 2
period = 2 * np.pi / omega
times = np.arange(1, 1201) * period / 200
values = 0.7 * np.cos(omega * times + phase) - 0.3 * np.sin(omega * times + phase) + 0.05 \
    + 0.01 * rng.standard_normal(times.size)
use = (times > 4 * period + 1e-10 * period) & (times <= 6 * period + 1e-10 * period)
coeff, residual = tool.fit(times[use], values[use], omega, phase)
out = {"omega": omega, "phase": phase, "times": times.tolist(), "values": values.tolist(),
       "window_samples": int(use.sum()), "coeff": [float(c) for c in coeff], "residual": float(residual)}
(HERE / "harmonic_fit.json").write_text(json.dumps(out))
print("coeff", coeff, "residual", residual, "samples", int(use.sum()))
