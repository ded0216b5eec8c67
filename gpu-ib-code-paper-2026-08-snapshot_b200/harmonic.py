"""Force harmonic error of the oscillating sphere against the analytic unsteady-Stokes force.

Restates the runtime-load check of ``tools/check_pressure_validation.py``:

* the analytic force on a sphere oscillating with velocity ``U0 cos(omega t + phase)``
  in an unbounded viscous fluid, ``F = -6 pi mu R U0 (1 + lam + lam^2 / 9)`` with
  ``lam = (1 + i) R / delta`` and the Stokes layer ``delta = sqrt(2 nu / omega)``
  (lines 76-80); its cosine / sine coefficients are ``(Re F, -Im F)``;
* a least-squares fit of the axial body force to ``[cos(omega t + phase),
  sin(omega t + phase), 1]`` (lines 31-37) over ``4T < t <= 6T`` (lines 90-93);
* the harmonic-vector error: the distance between fitted and analytic
  coefficient pairs over the analytic amplitude (lines 94-97), with the
  amplitude and phase errors beside it.
"""
from __future__ import annotations

import numpy as np


def analytic_force(mu, radius, speed, omega, nu):
    """Complex amplitude of the unsteady-Stokes force (cosine part real)."""
    k = radius / np.sqrt(2.0 * nu / omega)
    lam = (1.0 + 1.0j) * k
    return -6.0 * np.pi * mu * radius * speed * (1.0 + lam + lam ** 2 / 9.0)


def fit(times, values, omega, phase):
    """Cosine, sine and mean coefficients of ``values`` and the rms fit residual."""
    angle = omega * np.asarray(times, dtype=np.float64) + phase
    design = np.column_stack([np.cos(angle), np.sin(angle), np.ones_like(angle)])
    coeff, _, rank, _ = np.linalg.lstsq(design, np.asarray(values, dtype=np.float64), rcond=None)
    if rank != 3:
        raise ValueError("harmonic fit does not have full rank")
    return coeff, float(np.sqrt(np.mean((values - design @ coeff) ** 2)))


def harmonic_error(times, axial_force, *, mu, radius, amplitude, omega, phase, nu, periods=(4, 6)):
    """Errors of the fitted axial body force against the analytic force.

    ``times`` and ``axial_force`` are the step times and the body force along the
    oscillation axis; the fit window is ``periods[0] T < t <= periods[1] T``.
    """
    times = np.asarray(times, dtype=np.float64)
    axial_force = np.asarray(axial_force, dtype=np.float64)
    period = 2.0 * np.pi / omega
    speed = amplitude * omega
    f_hat = analytic_force(mu, radius, speed, omega, nu)
    ref = np.array([f_hat.real, -f_hat.imag])
    amp = abs(f_hat)
    eps = 1e-10 * period
    use = (times > periods[0] * period + eps) & (times <= periods[1] * period + eps)
    if use.sum() < 3:
        raise ValueError("the fit window holds fewer than three samples")
    coeff, residual = fit(times[use], axial_force[use], omega, phase)
    phase_err = (np.degrees(np.arctan2(coeff[1], coeff[0]) - np.arctan2(ref[1], ref[0])) + 180.0) % 360.0 - 180.0
    return {
        "cosine": float(coeff[0]), "sine": float(coeff[1]), "mean": float(coeff[2]),
        "amplitude": float(np.linalg.norm(coeff[:2])),
        "analytic_amplitude": float(amp),
        "amplitude_error_relative": float(np.linalg.norm(coeff[:2]) / amp - 1.0),
        "phase_error_degrees": float(phase_err),
        "harmonic_vector_error": float(np.linalg.norm(coeff[:2] - ref) / amp),
        "fit_residual_rms_over_amplitude": residual / amp,
        "samples": int(use.sum()),
    }
