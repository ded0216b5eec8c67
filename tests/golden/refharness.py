"""Drive the unmodified PyIB reference (CPU NumPy/SciPy path) to produce golden data.

This script runs only where the reference source tree is present; its location
comes from the environment variable ``PYIB_REFERENCE_ROOT``.  It is never
imported by the product, by ``bench.py`` or by the GPU tests.  It builds cases the way ``solver/ib_case.py:build_runtime``
(lines 633-809) does, but with nested box lists chosen here, because the
reference's presets do not cover the workloads used by the tests.

Two stub modules stand in for ``h5py`` and ``meshio``: the reference imports
them at ``make_euler_mesh.py:126-127`` but only its file writers use them.
"""
from __future__ import annotations

import os
import sys
import tempfile
from pathlib import Path

import numpy as np

def reference_root() -> Path:
    """The reference source tree, named by the environment variable PYIB_REFERENCE_ROOT."""
    root = os.environ.get("PYIB_REFERENCE_ROOT")
    if not root:
        raise RuntimeError("set PYIB_REFERENCE_ROOT to the PyIB reference source tree "
                           "(the directory that holds src/pyib)")
    path = Path(root)
    if not (path / "src" / "pyib" / "solver").is_dir():
        raise RuntimeError(f"PYIB_REFERENCE_ROOT={root} does not hold src/pyib/solver")
    return path


def import_reference():
    """Put the reference's modules on sys.path (CPU backend, float64)."""
    if "ib_case" in sys.modules:
        return sys.modules["ib_case"]
    REFERENCE_ROOT = reference_root()
    stubs = Path(tempfile.mkdtemp(prefix="pyib_stubs_"))
    (stubs / "h5py.py").write_text("")
    (stubs / "meshio.py").write_text("")
    os.environ["IB_GPU"] = "0"
    os.environ["IB_FP32"] = "0"
    if "--nometis" not in sys.argv:
        sys.argv.append("--nometis")
    src = REFERENCE_ROOT / "src"
    for p in (stubs, src / "pyib", src / "pyib" / "solver", src):
        sys.path.insert(0, str(p))
    import ib_case  # noqa: F401  (imports backend, core, driver, immersed, ...)
    return ib_case


def make_mesh(h, half_widths=None, bounds=None):
    """Nested concentric cubes (half widths innermost first) or explicit bounds."""
    import make_euler_mesh as M
    boxes = []
    if bounds is not None:
        for b in bounds:
            boxes.append(M._build_box(("bounds", tuple(float(v) for v in b))))
    else:
        for hw in half_widths:
            boxes.append(M._build_box(("bounds", (-hw, hw, -hw, hw, -hw, hw))))
    return M.make_nested_mesh(float(h), boxes, refinement_ratio=2)


class RefCase:
    """A reference runtime assembled from its public classes.

    Parameters follow ``ib_case.build_runtime``: density ``rho``, Reynolds
    number ``Re`` on diameter ``2R``; with ``inflow != 0`` the viscosity uses
    the inflow speed, otherwise the oscillation speed ``2 pi f A``.
    """

    def __init__(self, h, half_widths, *, radius=0.25, inflow=1.0, Re=100.0, rho=1.0,
                 dt=0.01, inner=4, cavity=False, amplitude=0.0, frequency=1.0,
                 phase=0.0, axis=(1.0, 0.0, 0.0), marker_spacing=None,
                 sparse=True, cg_check_interval=20, cg_max_iterations=1000,
                 force_mode="accumulated_explicit"):
        ic = import_reference()
        from ib_core_np import IBCore
        from ib_driver_np import Driver
        from ib_immersed import ImmersedBoundary
        from ib_interior import ClosedSphereLoadCorrection
        from ib_kinematics import Oscillation

        self.mesh = mesh = make_mesh(h, half_widths)
        self.core = core = IBCore(mesh)
        self.h = float(h)
        D = 2.0 * radius
        if inflow != 0.0:
            ref_speed = abs(inflow)
        else:
            ref_speed = 2.0 * np.pi * frequency * amplitude
        nu = ref_speed * D / Re
        self.visc = rho * nu
        self.driver = drv = Driver(core, mesh, visc=rho * nu, rou=rho)
        drv.cg_check_interval = int(cg_check_interval)
        drv.cg_max_iterations = int(cg_max_iterations)
        drv.fail_on_cg_nonconvergence = False
        if cavity:
            drv.set_cavity(U_lid=0.0, spanwise_zerograd=False)
        self.dt = float(dt)
        self.inner = int(inner)
        if sparse:
            drv.enable_sparse(self.dt)
        spacing = h if marker_spacing is None else marker_spacing
        count = max(12, int(round(4.0 * np.pi * radius ** 2 / spacing ** 2)))
        centre = np.zeros(3)
        markers = ic.fibonacci_sphere(count, radius, centre)
        width = (4.0 * np.pi * radius ** 2 * h / count) ** (1.0 / 3.0)
        self.marker_widths = np.full(count, width)
        self.reference_markers = markers
        self.ib = ib = ImmersedBoundary(mesh)
        vel = np.zeros((count, 3))
        self.motion = None
        if amplitude != 0.0:
            self.motion = Oscillation(markers, axis=axis, A=amplitude, freq=frequency, phase=phase)
            mk0, vel = self.motion(0.0)
            drv.set_ib(ib, mk0, self.marker_widths, vel, force_mode=force_mode)
            drv.set_motion(self.motion, t0=0.0)
        else:
            drv.set_ib(ib, markers, self.marker_widths, vel, force_mode=force_mode)
        ax = np.asarray(axis, float) / np.linalg.norm(axis)
        self.axis = ax
        self.amplitude = amplitude
        self.frequency = frequency
        self.phase = phase
        max_tr = np.abs(ax) * amplitude if amplitude != 0.0 else np.zeros(3)
        self.load = ClosedSphereLoadCorrection(
            core.cpos[: core.ncell], 1.0 / core.vol_ci, reference_center=centre,
            maximum_translation=max_tr, radius=radius, smoothing_width=h,
            density=rho, force_support_width=1.5 * ib.hh)
        self.inflow = inflow

    def centre(self, t):
        if self.amplitude == 0.0:
            return np.zeros(3)
        ang = 2.0 * np.pi * self.frequency * t + self.phase
        return self.amplitude * np.sin(ang) * self.axis

    def initial_state(self):
        """``ib_case._initial_state`` (lines 812-820)."""
        core = self.core
        s = self.inflow * core.epos[:, 1] * core.te[:, 2]
        s, _, vc = self.driver.calc_vel(s)
        self.load.initialize(vc[: core.ncell], self.centre(self.driver.time))
        return s, s.copy(), vc

    def run(self, steps, callback=None):
        """The step loop of ``ib_case.run_case`` (lines 1518-1530)."""
        s, s_old, vc = self.initial_state()
        drv = self.driver
        for step in range(1, steps + 1):
            drv.time = (step - 1) * self.dt
            s, vc, s_old = drv.step(s, s_old, self.dt, dt_old=self.dt, inner=self.inner)
            drv.time = step * self.dt
            load = self.load.advance(vc[: self.core.ncell], self.centre(drv.time), self.dt,
                                     drv.ib_force_E)
            if callback is not None:
                callback(step, s, s_old, vc, load)
        return s, s_old, vc
