"""Marker placement and prescribed motion against the reference's own values (CPU).

The fixture ``golden/kinematics.npz`` comes from the reference's
``fibonacci_sphere`` (``ib_case.py:554-563``) and ``Oscillation``
(``ib_kinematics.py:31-40``); see ``golden/make_kinematics_golden.py``.  The
product's host-side versions must reproduce them bit for bit: the marker
positions feed the ``rint`` stencil base, whose cells must be identical.
"""
import numpy as np
import pytest

import parity_util as PU
from pyib_b200 import cases as CS

G = np.load(PU.GOLDEN / "kinematics.npz")
COUNTS = (4, 13, 50, 201, 804, 3217, 5027)
CENTRES = ((0.0, 0.0, 0.0), (0.125, -0.3, 0.7))
MOTIONS = (
    ((1.0, 0.0, 0.0), 0.1, 3.6 / (2 * np.pi), -np.pi / 2),
    ((0.0, 1.0, 0.0), 0.05, 0.5, 0.0),
    ((1.0, 2.0, -0.5), 0.0375, 1.7, 0.3),
)
TIMES = (0.0, 0.00872664626, 0.1, 0.37, 1.0, 2.5, 10.471975511965978)


@pytest.mark.parametrize("n", COUNTS)
def test_fibonacci_sphere_bit_exact(n):
    for c, centre in enumerate(CENTRES):
        assert np.array_equal(CS.fibonacci_sphere(n, 0.25, np.asarray(centre)), G[f"fib_{n}_{c}"])


def test_fibonacci_sphere_rejects_fewer_than_four():
    with pytest.raises(ValueError):
        CS.fibonacci_sphere(3, 0.25, np.zeros(3))


@pytest.mark.parametrize("q", range(len(MOTIONS)))
def test_oscillation_bit_exact(q):
    axis, A, f, ph = MOTIONS[q]
    mo = CS.Oscillation(G["osc_ref"], axis, A, f, ph)
    for t_i, t in enumerate(TIMES):
        mk, vel = mo(t)
        assert np.array_equal(mk, G[f"osc_{q}_{t_i}_mk"]), (q, t)
        assert np.array_equal(vel, G[f"osc_{q}_{t_i}_vel"]), (q, t)
