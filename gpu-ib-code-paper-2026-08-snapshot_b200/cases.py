"""Named workloads: the nested sphere cases the benchmarks and tests run.

Each case follows the reference's runtime assembly (``ib_case.py:633-809``):
sphere of diameter ``D = 0.5`` at the origin, Fibonacci markers with
``round(4 pi R^2 / h^2)`` points and volume width ``(4 pi R^2 h / M)^(1/3)``
(``ib_case.py:723-727``), viscosity from the Reynolds number on the diameter
and the inflow speed or the oscillation speed ``2 pi f A`` (``ib_case.py:697-708``),
closed no-slip cavity for the concentric oscillating cases
(``ib_case.py:717-718``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .layout import concentric_layout

D = 0.5
R = 0.25


def fibonacci_sphere(count, radius, centre):
    """Fibonacci-lattice surface points (the layout of ``ib_case.py:554-563``)."""
    if count < 4:
        raise ValueError("a sphere surface requires at least four markers")
    k = np.arange(count, dtype=np.float64)
    polar = np.arccos(1.0 - 2.0 * (k + 0.5) / count)
    azim = np.pi * (1.0 + np.sqrt(5.0)) * k
    u = np.stack([np.sin(polar) * np.cos(azim), np.sin(polar) * np.sin(azim), np.cos(polar)], axis=1)
    return np.asarray(centre, dtype=np.float64) + radius * u


class Oscillation:
    """x(t) = ref + A sin(2 pi f t + phase) axis and its analytic velocity (ib_kinematics.py:31-40)."""

    def __init__(self, ref, axis, A, freq, phase=0.0):
        ax = np.asarray(axis, dtype=np.float64)
        self.axis = ax / np.linalg.norm(ax)
        self.ref = np.asarray(ref, dtype=np.float64)
        self.A, self.freq, self.phase = float(A), float(freq), float(phase)

    def __call__(self, t):
        w = 2.0 * np.pi * self.freq
        mk = self.ref + np.asarray(self.A * np.sin(w * t + self.phase) * self.axis, dtype=float)
        vel = np.tile(np.asarray(self.A * w * np.cos(w * t + self.phase) * self.axis, dtype=float),
                      (self.ref.shape[0], 1))
        return mk, vel

    def centre(self, t):
        w = 2.0 * np.pi * self.freq
        return self.A * np.sin(w * t + self.phase) * self.axis


@dataclass
class SphereCase:
    name: str
    cells_per_diameter: int
    half_widths_d: tuple          # level half widths in diameters, innermost first
    reynolds: float
    inflow: float = 0.0
    amplitude_d: float = 0.0      # oscillation amplitude in diameters
    omega: float = 3.6
    phase: float = -math.pi / 2
    axis: tuple = (1.0, 0.0, 0.0)
    steps_per_period: int = 200
    dt: float | None = None
    cavity: bool = True
    density: float = 1.0
    cg_max_iterations: int = 5000
    extra: dict = field(default_factory=dict)

    @property
    def h(self):
        return D / self.cells_per_diameter

    def layout(self):
        return concentric_layout(self.h, [w * D for w in self.half_widths_d])

    @property
    def amplitude(self):
        return self.amplitude_d * D

    @property
    def frequency(self):
        return self.omega / (2.0 * math.pi)

    @property
    def period(self):
        return 2.0 * math.pi / self.omega

    @property
    def time_step(self):
        if self.dt is not None:
            return self.dt
        return self.period / self.steps_per_period

    @property
    def reference_speed(self):
        if self.inflow != 0.0:
            return abs(self.inflow)
        return 2.0 * math.pi * self.frequency * self.amplitude

    @property
    def viscosity(self):
        """Dynamic viscosity rho * U * D / Re."""
        return self.density * self.reference_speed * D / self.reynolds

    def markers(self):
        h = self.h
        count = max(12, int(round(4.0 * np.pi * R ** 2 / h ** 2)))
        ref = fibonacci_sphere(count, R, np.zeros(3))
        width = (4.0 * np.pi * R ** 2 * h / count) ** (1.0 / 3.0)
        return ref, np.full(count, width)

    def motion(self):
        ref, _ = self.markers()
        if self.amplitude == 0.0:
            return None
        return Oscillation(ref, self.axis, self.amplitude, self.frequency, self.phase)


# The benchmark's workload: D = 32 cells, three nested levels (half widths 2D, 4D, 8D:
# the 16D cube), A = 0.2 D, Re0 = 0.2, omega = 3.6, 200 steps per period, about 3200 markers.
D32_OSCILLATING = SphereCase(name="d32_oscillating_sphere", cells_per_diameter=32,
                             half_widths_d=(2.0, 4.0, 8.0), reynolds=0.2, amplitude_d=0.2)
# Same geometry at D = 40 cells (about 5000 markers).
D40_OSCILLATING = SphereCase(name="d40_oscillating_sphere", cells_per_diameter=40,
                             half_widths_d=(2.0, 4.0, 8.0), reynolds=0.2, amplitude_d=0.2)
# The same workload at D = 16 cells (720,896 cells): profiling-sized.
D16_OSCILLATING = SphereCase(name="d16_oscillating_sphere", cells_per_diameter=16,
                             half_widths_d=(2.0, 4.0, 8.0), reynolds=0.2, amplitude_d=0.2)
# D = 24 cells (2.4 M cells, 64 MB per edge vector: larger than L2): profiling-sized.
D24_OSCILLATING = SphereCase(name="d24_oscillating_sphere", cells_per_diameter=24,
                             half_widths_d=(2.0, 4.0, 8.0), reynolds=0.2, amplitude_d=0.2)
# The same workload at D = 8 cells (90,112 cells, 201 markers): six periods (1200 steps)
# are cheap, so the force harmonic error of the analytic check can be run to the end.
D8_OSCILLATING = SphereCase(name="d8_oscillating_sphere", cells_per_diameter=8,
                            half_widths_d=(2.0, 4.0, 8.0), reynolds=0.2, amplitude_d=0.2)
# Fixed sphere, D = 8 cells, 2 levels (finest box [-2D,2D], outer 16D cube), U = 1, Re = 100, CFL 0.5.
D8_FIXED = SphereCase(name="d8_fixed_sphere", cells_per_diameter=8, half_widths_d=(2.0, 8.0),
                      reynolds=100.0, inflow=1.0, amplitude_d=0.0, cavity=False,
                      dt=0.5 * (D / 8) / 1.0, cg_max_iterations=1000)

# The adjoint configuration: D = 16 cells, two levels (half widths 2D, 4D), A = 0.2 D,
# Re0 = 1, 200 steps per period (804 markers); its gradient runs over 400 steps.
D16_ADJOINT = SphereCase(name="d16_adjoint_sphere", cells_per_diameter=16, half_widths_d=(2.0, 4.0),
                         reynolds=1.0, amplitude_d=0.2)

CASES = {c.name: c for c in (D32_OSCILLATING, D40_OSCILLATING, D24_OSCILLATING, D16_OSCILLATING, D8_OSCILLATING,
                               D8_FIXED, D16_ADJOINT)}
