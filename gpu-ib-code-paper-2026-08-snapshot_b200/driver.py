"""Driver-compatible Python object over the B200 library.

``B200Driver`` keeps the method names, arguments and return shapes of the
reference ``Driver`` (``src/pyib/solver/ib_driver_np.py:94-532``) that
``ib_case.run_case`` and ``ib_case.diagnostics`` call, so a case runner can
swap it in for ``--device b200``.  Differences, all deliberate:

* fields live on the GPU in the dense nested-level layout; ``step`` and
  ``calc_vel`` return :class:`DeviceField` handles that download on
  ``np.asarray``;  ``to_reference_*`` convert to the reference numbering and
  orientation when an exact reference-layout array is needed;
* only the accumulated explicit force mode exists (the configs use it; the
  reference rejects implicit forcing with it, ``ib_case.py:361-363``);
* cavity mode supports the closed no-slip box the concentric sphere cases use
  (``set_cavity(U_lid=0.0, spanwise_zerograd=False)``, ``ib_case.py:717-718``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .device import DeviceSolver
from .layout import NestedLayout


class DeviceField:
    """A field resident on the GPU; ``np.asarray(field)`` downloads it."""

    def __init__(self, solver, name, shape=None, version=None):
        self.solver, self.name, self.shape = solver, name, shape
        self.version = version

    def __array__(self, dtype=None, copy=None):
        a = self.solver.get(self.name)
        if self.shape is not None:
            a = a.reshape(self.shape)
        return a if dtype is None else a.astype(dtype)

    def numpy(self):
        return np.asarray(self)


class B200Driver:
    cg_max_iterations = 1000
    fail_on_cg_nonconvergence = False

    def __init__(self, layout: NestedLayout, visc, rou=1.0, ac=0.5, ad=0.5, *,
                 cg_max_iterations=1000, fail_on_cg_nonconvergence=False, device=0,
                 precision="float64", mixed_tol=0.1, tables=None):
        if precision not in ("float64", "mixed"):
            raise ValueError("precision must be 'float64' or 'mixed'")
        self.precision = precision
        self.mixed_tol = float(mixed_tol)
        if isinstance(cg_max_iterations, bool) or int(cg_max_iterations) <= 0:
            raise ValueError("cg_max_iterations must be a positive integer")
        if not isinstance(fail_on_cg_nonconvergence, (bool, np.bool_)):
            raise ValueError("fail_on_cg_nonconvergence must be a boolean")
        self.layout = layout if getattr(layout, "_built", False) else layout.build()
        self.visc, self.rou, self.ac, self.ad = float(visc), float(rou), float(ac), float(ad)
        self.cg_max_iterations = int(cg_max_iterations)
        self.fail_on_cg_nonconvergence = bool(fail_on_cg_nonconvergence)
        self.cg_check_interval = 20
        self.device = int(device)
        self.cavity = False
        self.ib = None
        self.motion = None
        self.time = 0.0
        self._step_count = 0
        self._solver = None
        self.helmholtz_iterations_last_step = 0
        self.helmholtz_relative_residual_last_step = 0.0
        self.helmholtz_tolerance_ratio_last_step = 0.0
        self.helmholtz_converged_last_step = True
        self.helmholtz_total_iterations_last_step = 0
        self.ib_force_updates_last_step = 0
        self.ib_force_update_count = 0
        self.ib_implicit = False       # force_mode "replacement": solve M f = rhs (implicit_force)
        self.ib_alpha = 1.0            # force_mode "replacement": relaxation of the replaced force
        self.ib_force_mode = "accumulated_explicit"
        self.last_step_dt = None
        self.last_helm_m = 0
        self._tables = tables          # shared LayoutTables of this layout (optional)

    # ---- configuration ------------------------------------------------------
    def set_cavity(self, U_lid=0.0, spanwise_zerograd=False):
        """Closed no-slip box (ib_driver_np.py:155-177 with U_lid=0, six walls)."""
        if float(U_lid) != 0.0 or spanwise_zerograd:
            raise NotImplementedError("only the six-wall, zero-lid cavity of the sphere cases exists on b200")
        self.cavity = True
        self._solver = None
        return self

    def set_ib(self, ib, markers, ds, vel_desired, force_mode="accumulated_explicit"):
        """Attach the body (ib_driver_np.py:179-201).

        ``accumulated_explicit`` (alias ``fortran_accumulated``): one explicit force
        increment per step, held and carried with the body.  ``replacement`` (the
        public ``direct``): the force of every inner iteration replaces the last,
        scaled by ``ib_alpha``, explicit or, with ``ib_implicit``, solved with the
        marker coupling matrix.
        """
        if force_mode not in ("accumulated_explicit", "fortran_accumulated", "replacement"):
            raise ValueError(f"unsupported IB force_mode: {force_mode!r}")
        self.ib = ib if ib is not None else True
        self.ib_force_mode = "replacement" if force_mode == "replacement" else "accumulated_explicit"
        self._markers = np.asarray(markers, dtype=np.float64).reshape(-1, 3)
        self._vel = np.asarray(vel_desired, dtype=np.float64).reshape(-1, 3)
        self._ds = np.asarray(ds, dtype=np.float64).reshape(-1)
        self._ib_dirty = True
        return self

    def set_motion(self, motion, t0=0.0):
        self.motion = motion
        self.time = float(t0)
        return self

    def enable_sparse(self, dt):
        """The B200 matvec is matrix-free; kept for API compatibility."""
        return self

    @property
    def solver(self) -> DeviceSolver:
        if self._solver is None:
            self._solver = DeviceSolver(self.layout, rou=self.rou, visc=self.visc, cavity=self.cavity,
                                        cg_check_interval=self.cg_check_interval,
                                        cg_max_iterations=self.cg_max_iterations,
                                        strict=self.fail_on_cg_nonconvergence, ac=self.ac, ad=self.ad,
                                        device=self.device, precision=self.precision,
                                        mixed_tol=self.mixed_tol,
                                        tables=self._tables if self._tables is not None
                                        and self._tables.cavity == self.cavity else None)
            self._ib_dirty = True
        sv = self._solver
        mode = 0 if self.ib_force_mode == "accumulated_explicit" else (2 if self.ib_implicit else 1)
        want = dict(check=int(self.cg_check_interval), cg_max=int(self.cg_max_iterations),
                    strict=int(bool(self.fail_on_cg_nonconvergence)), ib_mode=mode,
                    ib_alpha=float(self.ib_alpha))
        if any(sv.params[k] != v for k, v in want.items()):
            sv.params.update(want)
            sv._push_params()
        if self.ib is not None and self._ib_dirty:
            sv.set_markers(self._markers, self._vel, self._ds)
            self._ib_dirty = False
        return sv

    # ---- state ----------------------------------------------------------------
    def _put_edges(self, name, s):
        if isinstance(s, DeviceField) and s.solver is self._solver and s.name == name:
            return
        self.solver.set(name, np.asarray(s, dtype=np.float64))

    def initial_stream_function(self, inflow_speed):
        """s = U * epos_y * te_z (ib_case.py:815) in the +a orientation."""
        lay = self.layout
        hz = np.where(lay.edge_axis == 2, lay.edge_h, 0.0)
        s = inflow_speed * (lay.epos[:, 1] * hz)
        s[~lay.edge_exists] = 0.0
        return s

    def calc_vel(self, s):
        """ib_driver_np.py:267-291 -> (s_bc, U, vc) as device fields."""
        sv = self.solver
        self._put_edges("S", s)
        sv.h.call("pyib_calc_vel")
        return (DeviceField(sv, "S"), DeviceField(sv, "U"),
                DeviceField(sv, "VC", (3, sv.lay.NC + sv.bfaces.size)))

    def step(self, s, s_old, dt, dt_old, inner=4):
        """One fluid step, ib_driver_np.py:412-532."""
        mk, vel = self._step_inputs(s, s_old, dt)
        st = _lib.StepStats()
        try:
            self.solver.h.call("pyib_step", C.c_double(dt), C.c_double(dt_old), int(inner), mk, vel, C.byref(st))
        finally:
            self._step_stats(st)
        return self._step_outputs(dt)

    # the parts of step around the library call (shared with step_batch)
    def _step_inputs(self, s, s_old, dt):
        self._put_edges("S", s)
        self._put_edges("S_OLD", s_old)
        self._step_count += 1
        self.time += dt
        mk = vel = None
        if self.ib is not None and self.motion is not None:
            m, v = self.motion(self.time)
            self._markers = np.ascontiguousarray(m, dtype=np.float64)
            self._vel = np.ascontiguousarray(v, dtype=np.float64)
            mk = self._markers.ctypes.data_as(C.c_void_p)
            vel = self._vel.ctypes.data_as(C.c_void_p)
        return mk, vel

    def _step_stats(self, st):
        self.helmholtz_iterations_last_step = int(st.max_iterations)
        self.helmholtz_total_iterations_last_step = int(st.total_iterations)
        self.helmholtz_relative_residual_last_step = float(st.max_rel_residual)
        self.helmholtz_tolerance_ratio_last_step = float(st.max_tol_ratio)
        self.helmholtz_converged_last_step = bool(st.all_converged)
        self.ib_force_updates_last_step = int(st.ib_updates)
        self.ib_force_update_count += int(st.ib_updates)

    def _step_outputs(self, dt):
        sv = self.solver
        self.last_step_dt = float(dt)
        self.last_helm_m = self.helmholtz_iterations_last_step
        return (DeviceField(sv, "S"), DeviceField(sv, "VC", (3, sv.lay.NC + sv.bfaces.size)),
                DeviceField(sv, "S_OLD"))

    def helm_solve(self, res_e, s, dt):
        """ib_driver_np.py:311-410 on host arrays (dense layout); returns (x, iterations)."""
        sv = self.solver
        sv.set("RES_E", np.asarray(res_e, dtype=np.float64))
        sv.set("S", np.asarray(s, dtype=np.float64))
        st = _lib.SolveStats()
        sv.h.call("pyib_helm_solve", C.c_double(dt), C.byref(st))
        self.last_helm_m = int(st.iterations)
        self.last_helm_rel_residual = float(st.rel_residual)
        self.last_helm_tolerance_ratio = float(st.tol_ratio)
        self.last_helm_converged = bool(st.converged)
        return sv.get("S"), int(st.iterations)

    # ---- IB state (ib_driver_np.py:203-239) -----------------------------------
    @property
    def ib_force_E(self):
        return DeviceField(self.solver, "FE", (3, self.layout.NC))

    @property
    def ib_force_L(self):
        return self.solver.get("FL").reshape(-1, 3)

    @property
    def ib_markers(self):
        return self._markers

    @property
    def ib_vel(self):
        return self._vel

    @property
    def ib_ds(self):
        return self._ds

    @property
    def last_momentum_residual(self):
        return DeviceField(self.solver, "RES_C", (3, self.layout.NC))

    @property
    def last_face_flux(self):
        return DeviceField(self.solver, "U")

    def ib_state_dict(self):
        if self.ib is None:
            return None
        return {"force_mode": self.ib_force_mode, "force_E": np.asarray(self.ib_force_E).copy(),
                "force_L": self.ib_force_L.copy(), "force_update_count": int(self.ib_force_update_count)}

    def load_ib_state_dict(self, state):
        if self.ib is None:
            raise RuntimeError("set_ib must be called before loading IB state")
        if str(state["force_mode"]) != self.ib_force_mode:
            raise ValueError(f"IB force-mode mismatch: checkpoint={state['force_mode']!r}, "
                             f"run={self.ib_force_mode!r}")
        fE = np.asarray(state["force_E"], dtype=np.float64)
        fL = np.asarray(state["force_L"], dtype=np.float64)
        if fE.shape != (3, self.layout.NC):
            raise ValueError(f"Eulerian IB-force shape mismatch: {fE.shape} != {(3, self.layout.NC)}")
        if fL.shape != self._markers.shape:
            raise ValueError(f"Lagrangian IB-force shape mismatch: {fL.shape} != {self._markers.shape}")
        sv = self.solver
        sv.set("FE", fE)
        sv.set("FL", fL)
        self.ib_force_update_count = int(state.get("force_update_count", 0))
        self.ib_force_updates_last_step = 0
        return self

    # ---- reference numbering ----------------------------------------------------
    def reference_maps(self):
        if not hasattr(self, "_maps"):
            self._desc, self._maps = self.layout.export_mesh()
        return self._desc, self._maps


def step_batch(batch, drivers, states, dts, dt_olds, inner=4):
    """``Driver.step`` of several drivers at once through one ``pyib_batch`` (built
    over the drivers' contexts, in this order): ``states`` holds each driver's
    ``(s, s_old)``; returns each driver's ``(s, vc, s_old)`` as ``step`` does.  The
    Helmholtz solves of all drivers run as batched CG iterations; every driver ends
    in the state its own ``step`` would give."""
    n = len(drivers)
    mks = (C.c_void_p * n)()
    vels = (C.c_void_p * n)()
    use_markers = False
    for q, (drv, (s, s_old), dt) in enumerate(zip(drivers, states, dts)):
        mk, vel = drv._step_inputs(s, s_old, dt)
        if mk is not None:
            use_markers = True
            mks[q], vels[q] = mk.value, vel.value
    stats = (_lib.StepStats * n)()
    dt_a = (C.c_double * n)(*[float(x) for x in dts])
    dto_a = (C.c_double * n)(*[float(x) for x in dt_olds])
    try:
        batch.call("pyib_batch_step", dt_a, dto_a, int(inner), mks if use_markers else None,
                   vels if use_markers else None, stats)
    finally:
        for drv, st in zip(drivers, stats):
            drv._step_stats(st)
    return [drv._step_outputs(dt) for drv, dt in zip(drivers, dts)]
