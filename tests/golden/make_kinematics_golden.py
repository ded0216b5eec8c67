"""Golden values of the reference's marker placement and prescribed motion.

    PYIB_REFERENCE_ROOT=<reference tree> python tests/golden/make_kinematics_golden.py

Evaluates the reference's ``fibonacci_sphere`` (``ib_case.py:554-563``) for the
marker counts the sphere cases use and ``Oscillation`` (``ib_kinematics.py:31-40``)
at a few times, axes and phases; ``tests/test_kinematics.py`` checks the
product's ``cases.fibonacci_sphere`` and ``cases.Oscillation`` against them bit
for bit.
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import refharness  # noqa: E402

COUNTS = (4, 13, 50, 201, 804, 3217, 5027)
CENTRES = ((0.0, 0.0, 0.0), (0.125, -0.3, 0.7))
MOTIONS = (  # axis, amplitude, frequency, phase
    ((1.0, 0.0, 0.0), 0.1, 3.6 / (2 * np.pi), -np.pi / 2),
    ((0.0, 1.0, 0.0), 0.05, 0.5, 0.0),
    ((1.0, 2.0, -0.5), 0.0375, 1.7, 0.3),
)
TIMES = (0.0, 0.00872664626, 0.1, 0.37, 1.0, 2.5, 10.471975511965978)

if __name__ == "__main__":
    ic = refharness.import_reference()
    from ib_kinematics import Oscillation
    out = {}
    for n in COUNTS:
        for c, centre in enumerate(CENTRES):
            out[f"fib_{n}_{c}"] = ic.fibonacci_sphere(n, 0.25, np.asarray(centre))
    ref = ic.fibonacci_sphere(201, 0.25, np.zeros(3))
    out["osc_ref"] = ref
    for q, (axis, A, f, ph) in enumerate(MOTIONS):
        mo = Oscillation(ref, axis=axis, A=A, freq=f, phase=ph)
        for t_i, t in enumerate(TIMES):
            mk, vel = mo(t)
            out[f"osc_{q}_{t_i}_mk"] = mk
            out[f"osc_{q}_{t_i}_vel"] = vel
    np.savez_compressed(HERE / "kinematics.npz", **out)
    print(len(out), "arrays")
