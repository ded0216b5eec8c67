"""Force harmonic error (restatement of the reference's runtime-load check)."""
import json

import numpy as np
import pytest

import parity_util as PU
from pyib_b200 import harmonic as H


def test_fit_matches_reference_tool():
    d = json.loads((PU.GOLDEN / "harmonic_fit.json").read_text())
    t, v = np.array(d["times"]), np.array(d["values"])
    period = 2 * np.pi / d["omega"]
    use = (t > 4 * period + 1e-10 * period) & (t <= 6 * period + 1e-10 * period)
    assert int(use.sum()) == d["window_samples"]
    coeff, residual = H.fit(t[use], v[use], d["omega"], d["phase"])
    np.testing.assert_allclose(coeff, d["coeff"], rtol=1e-12, atol=1e-14)
    assert residual == pytest.approx(d["residual"], rel=1e-12)


def test_analytic_force_limits_and_error_measures():
    mu, radius, omega, nu, amp = 0.9, 0.25, 3.6, 0.9, 0.1
    speed = amp * omega
    # the Stokes drag is the low-frequency limit
    f0 = H.analytic_force(mu, radius, speed, 1e-12, nu)
    assert f0.real == pytest.approx(-6 * np.pi * mu * radius * speed, rel=1e-5)
    f = H.analytic_force(mu, radius, speed, omega, nu)
    period = 2 * np.pi / omega
    t = np.arange(1, 1201) * period / 200
    th = omega * t - np.pi / 2
    exact = f.real * np.cos(th) - f.imag * np.sin(th)
    kw = dict(mu=mu, radius=radius, amplitude=amp, omega=omega, phase=-np.pi / 2, nu=nu)
    e = H.harmonic_error(t, exact + 0.2, **kw)
    assert e["harmonic_vector_error"] < 1e-12 and abs(e["phase_error_degrees"]) < 1e-9
    assert e["mean"] == pytest.approx(0.2)
    e = H.harmonic_error(t, 1.05 * exact, **kw)
    assert e["amplitude_error_relative"] == pytest.approx(0.05, rel=1e-9)
    assert e["harmonic_vector_error"] == pytest.approx(0.05, rel=1e-9)
    # a force lagging by 10 degrees rotates its (cosine, sine) pair by +10 degrees,
    # the reference's sign convention
    lag = np.radians(10.0)
    shifted = f.real * np.cos(th - lag) - f.imag * np.sin(th - lag)
    e = H.harmonic_error(t, shifted, **kw)
    assert e["phase_error_degrees"] == pytest.approx(10.0, abs=1e-9)
