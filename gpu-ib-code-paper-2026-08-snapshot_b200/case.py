"""JSON case runner for the B200 path: config, runtime assembly, step loop, history, checkpoints.

The configuration is the reference's schema v1 (``ib_case.py:56-110``) with one
added device value, ``runtime.device = "b200"``, and the precisions
``"float64"`` (the reference's arithmetic) and ``"mixed"`` (float32 PCG inside
float64 refinement).  Mesh kinds follow the reference (``uniform_box``,
``sphere_concentric``, ``sphere_wake``) plus ``nested_boxes`` (concentric cubes
with explicit half widths in diameters), which the benchmark configurations
use.  The loop mirrors ``ib_case.run_case`` (``ib_case.py:1413-1648``): the
clock is anchored to the integer step, sampled steps write a ``history.csv``
row, checkpoints are atomic NPZ files written after the history is durable,
SIGTERM/SIGINT/SIGUSR1 stop after the current step with a checkpoint, and a
resume validates the configuration fingerprint before restoring the state.
"""
from __future__ import annotations

import copy
import csv
import hashlib
import json
import math
import os
import signal
import time
import uuid
from dataclasses import dataclass
from pathlib import Path
from typing import Any

import numpy as np

from .cases import Oscillation, fibonacci_sphere
from .driver import B200Driver
from .layout import NestedLayout
from .runner import SphereLoads

SCHEMA_VERSION = 1
CHECKPOINT_SCHEMA_VERSION = 3    # the reference's payload (ib_case.py:823-870)
RESULT_SCHEMA_VERSION = 5        # metadata and field snapshots (ib_case.py:53)

DEFAULT_CONFIG: dict[str, Any] = {
    "schema_version": SCHEMA_VERSION,
    "name": "fixed_sphere",
    "case": {"kind": "fixed_sphere"},
    "runtime": {"device": "b200", "precision": "float64"},
    "mesh": {"kind": "uniform_box", "dx": 0.25, "bounds": [[-1.0, 1.0], [-1.0, 1.0], [-1.0, 1.0]],
             "verbose": False},
    "physics": {"reynolds": 100.0, "density": 1.0, "inflow_speed": 1.0},
    "time": {"dt": 0.01, "steps": 5, "inner_iterations": 4},
    "ib": {"radius": 0.25, "center": [0.0, 0.0, 0.0], "marker_spacing": 0.25,
           "force_mode": "accumulated_explicit", "implicit": False, "alpha": 1.0,
           "motion": {"kind": "none", "axis": [0.0, 1.0, 0.0], "amplitude": 0.0, "frequency": 1.0,
                      "phase": 0.0}},
    "solver": {"sparse": True, "cg_check_interval": 20, "cg_max_iterations": 1000,
               "fail_on_cg_nonconvergence": False},
    "output": {"sample_every": 10, "checkpoint_every": 1000, "field_every": 0, "field_start_step": 0,
               "save_field": True},
}

_ALLOWED = {
    "root": {"schema_version", "name", "case", "runtime", "mesh", "physics", "time", "ib", "solver", "output"},
    "case": {"kind"},
    "runtime": {"device", "precision", "mixed_tolerance"},
    "mesh": {"kind", "dx", "bounds", "cells_per_diameter", "half_widths_d", "verbose"},
    "physics": {"reynolds", "density", "inflow_speed"},
    "time": {"dt", "steps", "inner_iterations"},
    "ib": {"radius", "center", "marker_spacing", "force_mode", "implicit", "alpha", "motion"},
    "motion": {"kind", "axis", "amplitude", "frequency", "phase", "spin_ratio"},
    "solver": {"sparse", "cg_check_interval", "cg_max_iterations", "fail_on_cg_nonconvergence"},
    "output": {"sample_every", "checkpoint_every", "field_every", "field_start_step", "save_field"},
}

# Reference presets (solver/sphere_quiescent_mesh.py:41, solver/sphere_wake_mesh.py:46-51)
CONCENTRIC_HALF_WIDTHS_D = (1.0, 2.0, 4.0, 8.0, 16.0)
WAKE_BOUNDS_D = ((-1.0, 3.0, -1.0, 1.0, -1.0, 1.0), (-2.0, 6.0, -2.0, 2.0, -2.0, 2.0),
                 (-4.0, 12.0, -4.0, 4.0, -4.0, 4.0), (-8.0, 16.0, -8.0, 8.0, -8.0, 8.0))

HISTORY_COLUMNS = [
    "step", "time", "Cd", "Cy", "Cz", "body_force_x", "body_force_y", "body_force_z",
    "force_fluid_x", "force_fluid_y", "force_fluid_z", "body_moment_x", "body_moment_y",
    "body_moment_z", "moment_fluid_x", "moment_fluid_y", "moment_fluid_z",
    "interior_momentum_x", "interior_momentum_y", "interior_momentum_z",
    "interior_angular_momentum_x", "interior_angular_momentum_y", "interior_angular_momentum_z",
    "interior_momentum_rate_x", "interior_momentum_rate_y", "interior_momentum_rate_z",
    "interior_angular_momentum_rate_x", "interior_angular_momentum_rate_y",
    "interior_angular_momentum_rate_z",
    "interior_indicator_volume", "slip_max", "slip_rms", "speed_max", "cfl", "mass_residual_inf",
    "force_balance_relerr", "ib_force_updates", "helmholtz_iterations",
    "helmholtz_relative_residual", "helmholtz_tolerance_ratio", "milliseconds_per_step",
]


class CaseConfigError(ValueError):
    """Invalid case configuration (the reference's ``CaseConfigError``)."""


def _merge(base, over):
    out = copy.deepcopy(base)
    for k, v in over.items():
        if isinstance(v, dict) and isinstance(out.get(k), dict):
            out[k] = _merge(out[k], v)
        else:
            out[k] = copy.deepcopy(v)
    return out


def _reject_unknown(section, d):
    extra = set(d) - _ALLOWED[section]
    if extra:
        raise CaseConfigError(f"unknown key(s) in {section}: {sorted(extra)}")


def _positive(name, v):
    try:
        x = float(v)
    except (TypeError, ValueError):
        raise CaseConfigError(f"{name} must be a number") from None
    if isinstance(v, bool) or not math.isfinite(x) or x <= 0.0:
        raise CaseConfigError(f"{name} must be finite and positive")
    return x


def _positive_int(name, v):
    if isinstance(v, bool) or not isinstance(v, (int, np.integer)) or int(v) <= 0:
        raise CaseConfigError(f"{name} must be a positive integer")
    return int(v)


def validate_config(raw: dict) -> dict:
    """Merge defaults, reject typos and return a normalized configuration (ib_case.py:262-441)."""
    if not isinstance(raw, dict):
        raise CaseConfigError("the case file must contain a JSON object")
    _reject_unknown("root", raw)
    for sec in ("case", "runtime", "mesh", "physics", "time", "ib", "solver", "output"):
        if sec in raw:
            if not isinstance(raw[sec], dict):
                raise CaseConfigError(f"{sec} must be a JSON object")
            _reject_unknown(sec, raw[sec])
    if isinstance(raw.get("ib"), dict) and isinstance(raw["ib"].get("motion"), dict):
        _reject_unknown("motion", raw["ib"]["motion"])
    cfg = _merge(DEFAULT_CONFIG, raw)
    if cfg["schema_version"] != SCHEMA_VERSION or isinstance(cfg["schema_version"], bool):
        raise CaseConfigError(f"unsupported schema_version={cfg['schema_version']}; expected {SCHEMA_VERSION}")
    if not isinstance(cfg["name"], str) or not cfg["name"].strip():
        raise CaseConfigError("name must be a non-empty string")
    kind = str(cfg["case"]["kind"])
    if kind not in {"fixed_sphere", "oscillating_sphere", "rotating_sphere"}:
        raise CaseConfigError(f"unsupported case.kind={kind!r}")
    rt = cfg["runtime"]
    if rt["device"] != "b200":
        raise CaseConfigError("runtime.device must be 'b200' here ('cpu'/'cuda' are the reference's backends)")
    if rt["precision"] not in {"float64", "mixed"}:
        raise CaseConfigError("runtime.precision must be 'float64' or 'mixed'")
    # the mixed form's update tolerance; absent from a float64 configuration, whose
    # runtime block keeps the reference's keys
    if rt["precision"] == "mixed":
        rt["mixed_tolerance"] = _positive("runtime.mixed_tolerance", rt.get("mixed_tolerance", 0.1))
    else:
        rt.pop("mixed_tolerance", None)
    mesh = cfg["mesh"]
    mk = str(mesh["kind"])
    if mk not in {"uniform_box", "sphere_concentric", "sphere_wake", "nested_boxes"}:
        raise CaseConfigError(f"unsupported mesh.kind={mk!r}")
    if mk == "uniform_box":
        mesh["dx"] = _positive("mesh.dx", mesh["dx"])
        b = np.asarray(mesh["bounds"], dtype=float)
        if b.shape != (3, 2) or not np.all(np.isfinite(b)) or np.any(b[:, 1] <= b[:, 0]):
            raise CaseConfigError("mesh.bounds must be three finite [lower, upper] pairs")
        cells = (b[:, 1] - b[:, 0]) / mesh["dx"]
        if not np.allclose(cells, np.rint(cells), rtol=0.0, atol=1e-10):
            raise CaseConfigError("uniform-box side lengths must be integer multiples of mesh.dx")
        mesh["bounds"] = b.tolist()
    else:
        mesh["cells_per_diameter"] = _positive_int("mesh.cells_per_diameter", mesh.get("cells_per_diameter", 16))
        if mk != "nested_boxes" and mesh["cells_per_diameter"] % 8:
            raise CaseConfigError("nested-sphere cells_per_diameter must be a multiple of 8")
        if mk == "nested_boxes":
            hw = mesh.get("half_widths_d")
            if not isinstance(hw, list) or not hw or any(_positive("mesh.half_widths_d", x) <= 0 for x in hw):
                raise CaseConfigError("nested_boxes needs mesh.half_widths_d (innermost first)")
            mesh["half_widths_d"] = [float(x) for x in hw]
        mesh.pop("dx", None)
        mesh.pop("bounds", None)
    ph = cfg["physics"]
    ph["reynolds"] = _positive("physics.reynolds", ph["reynolds"])
    ph["density"] = _positive("physics.density", ph["density"])
    ph["inflow_speed"] = float(ph["inflow_speed"])
    tm = cfg["time"]
    tm["dt"] = _positive("time.dt", tm["dt"])
    tm["steps"] = _positive_int("time.steps", tm["steps"])
    tm["inner_iterations"] = _positive_int("time.inner_iterations", tm["inner_iterations"])
    ib = cfg["ib"]
    ib["radius"] = _positive("ib.radius", ib["radius"])
    ib["marker_spacing"] = _positive("ib.marker_spacing", ib["marker_spacing"])
    # IB force mode, as ib_case.py:354-371 validates it
    if ib["force_mode"] not in ("direct", "accumulated_explicit"):
        raise CaseConfigError("ib.force_mode must be 'accumulated_explicit' or 'direct'")
    if not isinstance(ib["implicit"], (bool, np.bool_)):
        raise CaseConfigError("ib.implicit must be a boolean")
    ib["alpha"] = _positive("ib.alpha", ib["alpha"])
    if ib["force_mode"] == "accumulated_explicit":
        if ib["implicit"]:
            raise CaseConfigError("accumulated_explicit is an explicit IB method")
        if ib["alpha"] != 1.0:
            raise CaseConfigError("accumulated_explicit requires ib.alpha=1.0")
        if tm["inner_iterations"] < 2:
            raise CaseConfigError("accumulated_explicit requires at least two fluid inner iterations")
    elif ib["implicit"] and ib["alpha"] > 0.7:
        raise CaseConfigError("implicit IB currently requires ib.alpha <= 0.7")
    mo = ib["motion"]
    expected = {"fixed_sphere": "none", "oscillating_sphere": "oscillation", "rotating_sphere": "rotation"}[kind]
    if mo["kind"] != expected:
        raise CaseConfigError(f"case.kind={kind!r} requires ib.motion.kind={expected!r}")
    ax = np.asarray(mo["axis"], dtype=float)
    if ax.shape != (3,) or not np.all(np.isfinite(ax)) or np.linalg.norm(ax) == 0.0:
        raise CaseConfigError("ib.motion.axis must be a finite non-zero vector")
    mo["axis"] = (ax / np.linalg.norm(ax)).tolist()
    mo["amplitude"] = float(mo["amplitude"])
    mo["frequency"] = _positive("ib.motion.frequency", mo["frequency"])
    mo["phase"] = float(mo["phase"])
    if kind == "oscillating_sphere" and mo["amplitude"] <= 0.0:
        raise CaseConfigError("oscillating_sphere requires a positive motion amplitude")
    if kind != "oscillating_sphere" and mo["amplitude"] != 0.0:
        raise CaseConfigError(f"{kind} requires zero translational amplitude")
    if kind == "rotating_sphere":
        if "spin_ratio" not in mo:
            raise CaseConfigError("rotating_sphere requires ib.motion.spin_ratio")
        mo["spin_ratio"] = float(mo["spin_ratio"])
    if kind in {"fixed_sphere", "rotating_sphere"} and ph["inflow_speed"] == 0.0:
        raise CaseConfigError(f"{kind} requires non-zero physics.inflow_speed")
    so = cfg["solver"]
    so["cg_check_interval"] = _positive_int("solver.cg_check_interval", so["cg_check_interval"])
    so["cg_max_iterations"] = _positive_int("solver.cg_max_iterations", so["cg_max_iterations"])
    if not isinstance(so["fail_on_cg_nonconvergence"], bool):
        raise CaseConfigError("solver.fail_on_cg_nonconvergence must be true or false")
    out = cfg["output"]
    out["sample_every"] = _positive_int("output.sample_every", out["sample_every"])
    out["checkpoint_every"] = int(out["checkpoint_every"])
    if mk in {"sphere_wake", "sphere_concentric", "nested_boxes"}:
        if not np.allclose(ib["center"], 0.0) or not np.isclose(ib["radius"], 0.25):
            raise CaseConfigError("nested sphere meshes require ib.center=[0,0,0] and ib.radius=0.25")
    return cfg


def config_fingerprint(cfg: dict) -> str:
    stable = copy.deepcopy(cfg)
    for k in ("name", "output"):
        stable.pop(k, None)
    stable["time"].pop("steps", None)
    return hashlib.sha256(json.dumps(stable, sort_keys=True, separators=(",", ":")).encode()).hexdigest()


def build_layout(cfg):
    """The nested box list of the configured mesh (make_nested_mesh inputs)."""
    mesh = cfg["mesh"]
    D = 2.0 * float(cfg["ib"]["radius"])
    if mesh["kind"] == "uniform_box":
        b = np.asarray(mesh["bounds"], float)
        return NestedLayout(mesh["dx"], [(b[:, 0], b[:, 1])]), float(mesh["dx"]), b
    h = D / mesh["cells_per_diameter"]
    if mesh["kind"] == "sphere_wake":
        boxes = [((bd[0] * D, bd[2] * D, bd[4] * D), (bd[1] * D, bd[3] * D, bd[5] * D)) for bd in WAKE_BOUNDS_D]
    else:
        hws = CONCENTRIC_HALF_WIDTHS_D if mesh["kind"] == "sphere_concentric" else mesh["half_widths_d"]
        boxes = [((-w * D,) * 3, (w * D,) * 3) for w in hws]
    lo, hi = np.asarray(boxes[0][0]), np.asarray(boxes[0][1])
    return NestedLayout(h, boxes), h, np.stack([lo, hi], axis=1)


@dataclass
class CaseRuntime:
    config: dict
    layout: NestedLayout
    driver: B200Driver
    loads: SphereLoads
    motion: Any
    dx: float
    dt: float
    steps: int
    inner: int
    reference_force: float
    reference_speed: float
    fingerprint: str
    reference_markers: Any = None
    compact: Any = None
    layout_fingerprint: str = ""
    source_hashes: Any = None


def build_runtime(cfg) -> CaseRuntime:
    """Assemble the B200 runtime as ib_case.build_runtime does (ib_case.py:633-809)."""
    cfg = validate_config(cfg)
    lay, dx, fine_bounds = build_layout(cfg)
    ib = cfg["ib"]
    radius = float(ib["radius"])
    centre = np.asarray(ib["center"], float)
    mo = ib["motion"]
    exc = np.abs(np.asarray(mo["axis"])) * mo["amplitude"] if mo["kind"] == "oscillation" else np.zeros(3)
    if np.any(centre - exc - radius - 2.5 * dx < fine_bounds[:, 0] - 1e-12) or \
            np.any(centre + exc + radius + 2.5 * dx > fine_bounds[:, 1] + 1e-12):
        raise CaseConfigError("the sphere or its IB support leaves the finest uniform mesh region")
    ph = cfg["physics"]
    rho = ph["density"]
    Dref = 2.0 * radius
    if ph["inflow_speed"] != 0.0:
        uref = abs(ph["inflow_speed"])
    else:
        uref = 2.0 * np.pi * mo["frequency"] * mo["amplitude"]
    nu = uref * Dref / ph["reynolds"]
    so = cfg["solver"]
    drv = B200Driver(lay, visc=rho * nu, rou=rho, cg_max_iterations=so["cg_max_iterations"],
                     fail_on_cg_nonconvergence=so["fail_on_cg_nonconvergence"],
                     precision=cfg["runtime"]["precision"], mixed_tol=cfg["runtime"].get("mixed_tolerance", 0.1))
    drv.cg_check_interval = so["cg_check_interval"]
    if cfg["mesh"]["kind"] in {"sphere_concentric", "nested_boxes"}:
        drv.set_cavity(U_lid=0.0, spanwise_zerograd=False)
    fm = "replacement" if ib["force_mode"] == "direct" else "accumulated_explicit"
    drv.ib_implicit = bool(ib["implicit"])
    drv.ib_alpha = float(ib["alpha"])
    count = max(12, int(round(4.0 * np.pi * radius ** 2 / ib["marker_spacing"] ** 2)))
    markers = fibonacci_sphere(count, radius, centre)
    width = (4.0 * np.pi * radius ** 2 * dx / count) ** (1.0 / 3.0)
    ds = np.full(count, width)
    motion = None
    if mo["kind"] == "oscillation":
        motion = Oscillation(markers, mo["axis"], mo["amplitude"], mo["frequency"], mo["phase"])
        mk0, v0 = motion(0.0)
        drv.set_ib(None, mk0, ds, v0, force_mode=fm)
        drv.set_motion(motion, 0.0)
    elif mo["kind"] == "rotation":
        omega = np.asarray(mo["axis"]) * mo["spin_ratio"] * uref / radius
        drv.set_ib(None, markers, ds, np.cross(omega, markers - centre), force_mode=fm)
    else:
        drv.set_ib(None, markers, ds, np.zeros_like(markers), force_mode=fm)
    loads = SphereLoads(drv, centre, exc, radius, dx, rho, 1.5 * dx)
    rt = CaseRuntime(config=cfg, layout=lay, driver=drv, loads=loads, motion=motion, dx=dx,
                     dt=cfg["time"]["dt"], steps=cfg["time"]["steps"],
                     inner=cfg["time"]["inner_iterations"],
                     reference_force=0.5 * rho * uref ** 2 * np.pi * radius ** 2, reference_speed=uref,
                     fingerprint=config_fingerprint(cfg), reference_markers=markers,
                     compact=CompactIds(drv.layout), source_hashes=source_hashes())
    rt.layout_fingerprint = layout_fingerprint(rt)
    return rt


def sphere_center(rt: CaseRuntime, t):
    c = np.asarray(rt.config["ib"]["center"], float)
    if rt.motion is None:
        return c
    return c + rt.motion.centre(t)


def diagnostics(rt: CaseRuntime, step, ms_per_step):
    """A history row with the reference's 41 columns (ib_case.py:1129-1224)."""
    drv, load = rt.driver, rt.loads.latest
    if load is None:
        raise RuntimeError("closed-body load correction was not advanced for this step")
    import ctypes as C
    out = (C.c_double * 4)()
    drv.solver.h.call("pyib_diagnostics", out)
    d = np.asarray(out[:])
    fL = drv.ib_force_L
    lag = (fL * (drv.ib_ds ** 3)[:, None]).sum(axis=0)
    ff = load["force_fluid"]
    den = max(float(np.linalg.norm(lag)), float(np.linalg.norm(ff)), 1e-300)
    balance = float(np.linalg.norm(ff - lag)) / den
    coef = load["body_force"] / rt.reference_force
    row = {"step": int(step), "time": float(drv.time), "Cd": float(coef[0]), "Cy": float(coef[1]),
           "Cz": float(coef[2]),
           "interior_indicator_volume": float(load["indicator_volume"]), "slip_max": d[2], "slip_rms": d[3],
           "speed_max": d[0], "cfl": d[0] * rt.dt / rt.dx, "mass_residual_inf": d[1],
           "force_balance_relerr": balance, "ib_force_updates": int(drv.ib_force_updates_last_step),
           "helmholtz_iterations": int(drv.helmholtz_iterations_last_step),
           "helmholtz_relative_residual": float(drv.helmholtz_relative_residual_last_step),
           "helmholtz_tolerance_ratio": float(drv.helmholtz_tolerance_ratio_last_step),
           "milliseconds_per_step": float(ms_per_step)}
    for name, key in (("body_force", "body_force"), ("force_fluid", "force_fluid"),
                      ("body_moment", "body_moment"), ("moment_fluid", "moment_fluid"),
                      ("interior_momentum", "linear_momentum"),
                      ("interior_angular_momentum", "angular_momentum"),
                      ("interior_momentum_rate", "linear_rate"),
                      ("interior_angular_momentum_rate", "angular_rate")):
        for a, ax in enumerate("xyz"):
            row[f"{name}_{ax}"] = float(load[key][a])
    vals = np.asarray([float(row[c]) for c in HISTORY_COLUMNS])
    if not np.all(np.isfinite(vals)):
        raise FloatingPointError(f"non-finite diagnostic at step {step}: {row}")
    if balance > 1e-9 and rt.config["runtime"]["precision"] == "float64":
        raise RuntimeError(f"IB force-spread balance failed at step {step}: {balance:.3e}")
    expected = 1 if rt.config["ib"]["force_mode"] == "accumulated_explicit" else rt.inner
    if row["ib_force_updates"] != expected:
        raise RuntimeError(f"IB update-count invariant failed at step {step}: "
                           f"{row['ib_force_updates']} != {expected}")
    return row


# ---------------------------------------------------------------------------
# run artefacts in the reference's schema
# ---------------------------------------------------------------------------
class CompactIds:
    """Dense layout ids <-> the compact numbering of the exported mesh.

    Checkpoints and field snapshots hold one entry per existing edge / cell /
    face (the reference's array sizes), in ascending dense id, edge and face
    values oriented along +axis.
    """

    def __init__(self, lay):
        self.lay = lay
        self.cells = np.nonzero(lay.cell_active)[0]
        self.faces = np.nonzero(lay.face_exists)[0]
        self.edges = np.nonzero(lay.edge_exists)[0]

    def edge(self, v):
        return np.asarray(v, dtype=np.float64)[self.edges]

    def edge_dense(self, v):
        out = np.zeros(self.lay.NE)
        out[self.edges] = v
        return out

    def cell3(self, v3):
        return np.ascontiguousarray(np.asarray(v3, dtype=np.float64)[:, self.cells].T)

    def cell3_dense(self, v):
        out = np.zeros((3, self.lay.NC))
        out[:, self.cells] = np.asarray(v, dtype=np.float64).T
        return out


_SOURCE_FILES = ("case.py", "driver.py", "device.py", "layout.py", "operators.py", "templates.py",
                 "runner.py", "cases.py", "_lib.py", "csrc/pyib_b200.cu")


def source_hashes() -> dict:
    """sha256 of the numerical sources of this path (ib_case.py:474-487 does the same for its own)."""
    here = Path(__file__).resolve().parent
    return {name: hashlib.sha256((here / name).read_bytes()).hexdigest() for name in _SOURCE_FILES}


def layout_fingerprint(rt: CaseRuntime) -> str:
    """sha256 of the exported mesh description and the Lagrangian quadrature (ib_case.py:490-510)."""
    desc, _ = rt.driver.reference_maps()
    dg = hashlib.sha256()
    for name in ("nodes", "F2C", "F2E", "E2N", "link_fe_insert", "bc_edge", "bc_face", "index_cell",
                 "pos_ref"):
        a = np.ascontiguousarray(np.asarray(desc[name]))
        dg.update(name.encode() + b"\0" + a.dtype.str.encode() + b"\0" + json.dumps(a.shape).encode() + b"\0")
        dg.update(a.tobytes())
    dg.update(np.float64(desc["dx"]).tobytes())
    for name, value in (("markers", rt.reference_markers), ("marker_widths", rt.driver.ib_ds)):
        a = np.ascontiguousarray(np.asarray(value, dtype=np.float64))
        dg.update(name.encode() + b"\0" + json.dumps(a.shape).encode() + b"\0")
        dg.update(a.tobytes())
    return dg.hexdigest()


def mesh_summary(rt: CaseRuntime) -> dict:
    """The metadata ``mesh`` block (ib_case.py:640-688): kind, counts, level geometry."""
    cfg, lay = rt.config, rt.layout
    desc, _ = rt.driver.reference_maps()
    mesh = cfg["mesh"]
    out = {"kind": mesh["kind"], "faces": int(lay.face_exists.sum()), "edges": int(lay.edge_exists.sum()),
           "markers": int(rt.reference_markers.shape[0])}
    if mesh["kind"] == "uniform_box":
        out.update(cells=int(lay.cell_active.sum()), dx=float(mesh["dx"]),
                   bounds=[list(map(float, b)) for b in mesh["bounds"]])
    else:
        D = 2.0 * float(cfg["ib"]["radius"])
        per = [int(np.count_nonzero(lay.cell_active & (lay.cell_level == L))) for L in range(lay.N)]
        # the analytic counts: each level's box minus the box of the finer level inside it
        expected = [int(np.prod(lv.n)) - (int(np.prod(lay.levels[L - 1].n)) // 8 if L > 0 else 0)
                    for L, lv in enumerate(lay.levels)]
        top = lay.levels[-1]
        out.update(D_over_dx=int(mesh["cells_per_diameter"]), diameter=D, dx_fine=float(rt.dx),
                   outer_domain_D={ax: [float(top.lo[a] / D), float((top.lo[a] + top.n[a] * top.h) / D)]
                                   for a, ax in enumerate("xyz")},
                   layer_cells=per, expected_layer_cells=expected,
                   total_cells=int(sum(per)), expected_total_cells=int(sum(expected)),
                   nodes=int(desc["nodes"].shape[0]),
                   layer_spacing_D=[float(lv.h / D) for lv in lay.levels],
                   layer_bounds_D=[[float((lv.lo[a] + s * lv.n[a] * lv.h) / D)
                                    for a in range(3) for s in (0, 1)] for lv in lay.levels])
    return out


def _checkpoint_payload(rt: CaseRuntime, run_id, step, s, s_old) -> dict:
    """The schema-3 checkpoint payload (ib_case.py:823-870); arrays in compact order."""
    drv = rt.driver
    st = drv.ib_state_dict()
    if st is None:
        raise RuntimeError("cannot checkpoint an IB case before Driver.set_ib")
    load = rt.loads.latest
    if load is None or rt.loads.current is None:
        raise RuntimeError("cannot checkpoint before closed-body load bookkeeping")
    cid = rt.compact
    return {
        "checkpoint_schema": np.int64(CHECKPOINT_SCHEMA_VERSION),
        "update_phase": np.str_("post_step"),
        "run_id": np.str_(run_id),
        "config_fingerprint": np.str_(rt.fingerprint),
        "layout_fingerprint": np.str_(rt.layout_fingerprint),
        "step": np.int64(step),
        "physical_time": np.float64(drv.time),
        "dt": np.float64(rt.dt),
        "previous_dt": np.float64(rt.dt),
        "precision": np.str_(rt.config["runtime"]["precision"]),
        "device": np.str_("b200"),
        "source_hashes_json": np.str_(json.dumps(rt.source_hashes, sort_keys=True, separators=(",", ":"))),
        "s": cid.edge(s),
        "s_old": cid.edge(s_old),
        "markers": np.asarray(drv.ib_markers, dtype=np.float64),
        "marker_velocity": np.asarray(drv.ib_vel, dtype=np.float64),
        "ib_force_mode": np.str_(rt.config["ib"]["force_mode"]),
        "ib_force_E": cid.cell3(st["force_E"]),
        "ib_force_L": np.asarray(st["force_L"], dtype=np.float64),
        "ib_force_update_count": np.int64(st["force_update_count"]),
        "force_fluid": np.asarray(load["force_fluid"], dtype=np.float64),
        "moment_fluid": np.asarray(load["moment_fluid"], dtype=np.float64),
        "body_force": np.asarray(load["body_force"], dtype=np.float64),
        "body_moment": np.asarray(load["body_moment"], dtype=np.float64),
        "interior_momentum": np.asarray(load["linear_momentum"], dtype=np.float64),
        "interior_angular_momentum": np.asarray(load["angular_momentum"], dtype=np.float64),
        "interior_indicator_volume": np.float64(load["indicator_volume"]),
        "interior_momentum_rate": np.asarray(load["linear_rate"], dtype=np.float64),
        "interior_angular_momentum_rate": np.asarray(load["angular_rate"], dtype=np.float64),
    }


def save_checkpoint(path: Path, rt: CaseRuntime, run_id, step, s, s_old):
    _atomic_npz(path, **_checkpoint_payload(rt, run_id, step, s, s_old))


def save_field_snapshot(path: Path, rt: CaseRuntime, run_id, step, s, s_old, vc):
    """One self-contained field for the offline pressure recovery (ib_case.py:873-911)."""
    drv, lay, cid = rt.driver, rt.layout, rt.compact
    if drv.last_step_dt != rt.dt:
        raise RuntimeError("no current-step momentum residual for pressure recovery")
    desc, _ = drv.reference_maps()
    payload = _checkpoint_payload(rt, run_id, step, s, s_old)
    for name in ("checkpoint_schema", "update_phase", "physical_time", "previous_dt"):
        payload.pop(name)
    payload.update(
        result_schema=np.int64(RESULT_SCHEMA_VERSION),
        time=np.float64(drv.time),
        vc=cid.cell3(np.asarray(vc)[:, :lay.NC]),
        cpos=np.ascontiguousarray(lay.cpos[cid.cells]),
        cell_volume=np.ascontiguousarray(lay.cell_vol[cid.cells]),
        marker_volume_weight=np.asarray(drv.ib_ds, dtype=np.float64) ** 3,
        momentum_residual=cid.cell3(drv.last_momentum_residual),
        helmholtz_relative_residual=np.float64(drv.helmholtz_relative_residual_last_step),
        helmholtz_tolerance_ratio=np.float64(drv.helmholtz_tolerance_ratio_last_step),
        face_cells=np.asarray(desc["F2C"], dtype=np.int64),
        face_area=np.ascontiguousarray(lay.face_Af[cid.faces]),
        index_cell=np.asarray(desc["index_cell"], dtype=np.int64),
        lattice_origin=np.asarray(desc["pos_ref"], dtype=np.float64),
        lattice_spacing=np.float64(rt.dx),
        sphere_center=np.asarray(sphere_center(rt, drv.time), dtype=np.float64),
        sphere_radius=np.float64(rt.config["ib"]["radius"]),
        density=np.float64(drv.rou),
        kinematic_viscosity=np.float64(drv.visc / drv.rou),
    )
    _atomic_npz(path, **payload)


def _sync_directory(directory: Path) -> None:
    """Flush a directory entry (a rename) to disk; best effort, as on filesystems without dir fsync."""
    try:
        fd = os.open(directory, os.O_RDONLY)
    except OSError:
        return
    try:
        os.fsync(fd)
    except OSError:
        pass
    finally:
        os.close(fd)


def _atomic_npz(path: Path, **arrays):
    """Write, fsync, rename over ``path``, then fsync the directory so the rename survives a crash."""
    tmp = path.with_name(f".{path.stem}.{uuid.uuid4().hex}.tmp.npz")
    try:
        np.savez(tmp, **arrays)
        with tmp.open("r+b") as fh:
            fh.flush()
            os.fsync(fh.fileno())
        os.replace(tmp, path)
        _sync_directory(path.parent)
    finally:
        if tmp.exists():
            tmp.unlink()


def _str(d, k):
    return str(d[k].item() if hasattr(d[k], "item") else d[k])


def load_checkpoint(path: Path, rt: CaseRuntime):
    """Validate and restore a schema-3 checkpoint (ib_case.py:914-1121, the checks this path has)."""
    try:
        d = np.load(path, allow_pickle=False)
    except (OSError, ValueError) as exc:
        raise CaseConfigError(f"cannot read checkpoint {path}: {exc}") from exc
    with d:
        if "checkpoint_schema" not in d.files or int(d["checkpoint_schema"]) != CHECKPOINT_SCHEMA_VERSION:
            raise CaseConfigError("unsupported checkpoint schema")
        if _str(d, "update_phase") != "post_step":
            raise CaseConfigError("checkpoint is not a post-step state")
        if _str(d, "config_fingerprint") != rt.fingerprint:
            raise CaseConfigError("checkpoint was written for a different configuration")
        if _str(d, "layout_fingerprint") != rt.layout_fingerprint:
            raise CaseConfigError("checkpoint layout fingerprint does not match the configured mesh")
        if _str(d, "device") != "b200" or _str(d, "precision") != rt.config["runtime"]["precision"]:
            raise CaseConfigError("checkpoint device/precision differ from the configuration")
        if float(d["dt"]) != rt.dt or float(d["previous_dt"]) != rt.dt:
            raise CaseConfigError("checkpoint dt differs from the configuration")
        if json.loads(_str(d, "source_hashes_json")) != rt.source_hashes:
            raise CaseConfigError("checkpoint was written by different numerical source files")
        cid = rt.compact
        s, s_old = np.asarray(d["s"]), np.asarray(d["s_old"])
        if s.shape != (cid.edges.size,) or s_old.shape != (cid.edges.size,):
            raise CaseConfigError("checkpoint layout does not match the configuration")
        arrays = {k: np.asarray(d[k]) for k in d.files if d[k].dtype.kind == "f"}
        for k, arr in arrays.items():
            if not np.all(np.isfinite(arr)):
                raise CaseConfigError(f"checkpoint field {k} holds non-finite values")
        step = int(d["step"])
        drv = rt.driver
        if abs(float(d["physical_time"]) - step * rt.dt) > 1e-12 * max(1.0, step * rt.dt):
            raise CaseConfigError("checkpoint time is not anchored to its step")
        drv.time = step * rt.dt
        if rt.motion is not None:
            mk, v = rt.motion(drv.time)
            drv.set_ib(drv.ib, mk, drv.ib_ds, v, force_mode=drv.ib_force_mode)
        if not np.array_equal(np.asarray(d["markers"]), np.asarray(drv.ib_markers)):
            raise CaseConfigError("checkpoint markers disagree with the prescribed motion")
        fE = cid.cell3_dense(d["ib_force_E"])
        mode = "replacement" if _str(d, "ib_force_mode") == "direct" else "accumulated_explicit"
        drv.load_ib_state_dict({"force_mode": mode, "force_E": fE, "force_L": np.asarray(d["ib_force_L"]),
                                "force_update_count": int(d["ib_force_update_count"])})
        cur = np.concatenate([d["force_fluid"], d["moment_fluid"], d["interior_momentum"],
                              d["interior_angular_momentum"], [float(d["interior_indicator_volume"])]])
        rt.loads.current = cur
        run_id = _str(d, "run_id")
        return step, cid.edge_dense(s), cid.edge_dense(s_old), run_id


def _atomic_json(path: Path, payload: dict):
    tmp = path.with_name(f".{path.name}.{uuid.uuid4().hex}.tmp")
    try:
        with tmp.open("x", encoding="utf-8") as fh:
            fh.write(json.dumps(payload, indent=2, allow_nan=False) + "\n")
            fh.flush()
            os.fsync(fh.fileno())
        os.replace(tmp, path)
        _sync_directory(path.parent)
    finally:
        if tmp.exists():
            tmp.unlink()


def _metadata(rt: CaseRuntime, run_id, outdir: Path, start_step, resumed_from):
    """metadata.json with the reference's keys (ib_case.py:1331-1366); backend ``b200/cuda``."""
    import platform
    from datetime import datetime, timezone
    from . import _lib
    return {
        "result_schema": RESULT_SCHEMA_VERSION,
        "run_id": run_id,
        "created_utc": datetime.now(timezone.utc).isoformat(),
        "case_name": rt.config["name"],
        "case_kind": rt.config["case"]["kind"],
        "backend": "b200/cuda",
        "precision": rt.config["runtime"]["precision"],
        "python": platform.python_version(),
        "array_backend_version": _lib.version(),
        "config_fingerprint": rt.fingerprint,
        "layout_fingerprint": rt.layout_fingerprint,
        "config": rt.config,
        "mesh": mesh_summary(rt),
        "dt": rt.dt,
        "target_steps": rt.steps,
        "start_step": start_step,
        "resumed_from": str(Path(resumed_from).resolve()) if resumed_from else None,
        "output_directory": str(outdir.resolve()),
        "source_sha256": rt.source_hashes,
        "closed_body_load": {
            "method": "Uhlmann interior-fluid momentum correction",
            "force": "-force_fluid + backward_difference(interior_momentum)",
            "moment": "-moment_fluid + backward_difference(interior_angular_momentum)",
            "indicator": "analytic sphere with one-cell linear smoothing",
            "moment_origin": [0.0, 0.0, 0.0],
        },
    }


def _archive(outdir: Path, paths):
    """Move earlier artefacts aside instead of deleting them (ib_case.py:_archive_known_outputs)."""
    present = [p for p in paths if p.exists()]
    if not present:
        return None
    dest = outdir / "archive" / f"{time.strftime('%Y%m%dT%H%M%S')}-{uuid.uuid4().hex[:8]}"
    dest.mkdir(parents=True)
    for p in present:
        os.replace(p, dest / p.name)
    _sync_directory(outdir)
    return dest


def _history_prefix(path: Path, start_step: int):
    """Rows up to the checkpoint step, checked for the reference's columns (ib_case.py:1227-1291)."""
    if not path.exists():
        raise CaseConfigError("resume needs the run's history.csv")
    with path.open(newline="") as fh:
        reader = csv.DictReader(fh)
        if reader.fieldnames != HISTORY_COLUMNS:
            raise CaseConfigError("history.csv does not have the expected columns")
        rows = [r for r in reader if int(float(r["step"])) <= start_step]
    if not rows or int(float(rows[-1]["step"])) != start_step:
        raise CaseConfigError("history.csv has no row for the checkpoint step")
    return rows


def run_case(config, outdir, *, resume=False, overwrite=False, quiet=False):
    """Run one case and write the reference's artefacts (ib_case.py:1413-1648).

    Artefacts: ``history.csv`` (41 columns), ``metadata.json``, ``checkpoint.npz``
    (schema 3), ``snapshots/field_*.npz`` every ``output.field_every`` steps and
    ``final_field.npz``.  ``resume=True`` continues from ``checkpoint.npz``.
    """
    setup0 = time.perf_counter()
    rt = build_runtime(config)
    out = Path(outdir)
    out.mkdir(parents=True, exist_ok=True)
    hist_path, ckpt, meta_path = out / "history.csv", out / "checkpoint.npz", out / "metadata.json"
    final_path, snap_dir = out / "final_field.npz", out / "snapshots"
    known = (hist_path, ckpt, meta_path, final_path, snap_dir)
    if not resume and not overwrite and any(p.exists() for p in known):
        raise FileExistsError(f"{out} already contains run artifacts; pass overwrite=True or resume=True")
    drv = rt.driver
    previous = None
    if resume:
        start, s, s_old, run_id = load_checkpoint(ckpt, rt)
        if start >= rt.steps:
            raise CaseConfigError(f"target steps ({rt.steps}) must exceed checkpoint step ({start})")
        rows = _history_prefix(hist_path, start)
        if meta_path.exists():
            previous = json.loads(meta_path.read_text())
            if previous.get("run_id") != run_id:
                raise CaseConfigError("metadata.json belongs to a different run")
        _archive(out, (final_path,))
        stale = [p for p in snap_dir.glob("field_*.npz") if p.stem[6:].isdigit() and int(p.stem[6:]) > start]
        _archive(out, stale)
        s, _, _ = drv.calc_vel(s)
    else:
        start = 0
        s = drv.initial_stream_function(rt.config["physics"]["inflow_speed"])
        s, _, _ = drv.calc_vel(s)
        s_old = np.asarray(s).copy()
        rt.loads.initialize(sphere_center(rt, 0.0))
        run_id = str(uuid.uuid4())
        rows = []
        if overwrite:
            _archive(out, known)
    meta = _metadata(rt, run_id, out, start, ckpt if resume else None)
    if previous is not None:
        from datetime import datetime, timezone
        meta["created_utc"] = previous["created_utc"]
        meta["resume_count"] = int(previous.get("resume_count", 0)) + 1
        meta["last_resume_utc"] = datetime.now(timezone.utc).isoformat()
    else:
        meta["resume_count"] = 0
    meta["setup_seconds"] = time.perf_counter() - setup0
    _atomic_json(meta_path, meta)
    fh = hist_path.open("w", newline="")
    writer = csv.DictWriter(fh, fieldnames=HISTORY_COLUMNS)
    writer.writeheader()
    for r in rows:
        writer.writerow(r)
    fh.flush()
    os.fsync(fh.fileno())
    stop = {"flag": False}
    old = {}
    for nm in ("SIGTERM", "SIGINT", "SIGUSR1"):
        if hasattr(signal, nm):
            sig = getattr(signal, nm)
            try:
                old[sig] = signal.getsignal(sig)
                signal.signal(sig, lambda *_: stop.__setitem__("flag", True))
            except (OSError, ValueError):
                pass
    o = rt.config["output"]
    done = start
    t0, s0 = time.perf_counter(), start
    vc = None

    def sample_row(step):
        nonlocal t0, s0
        now = time.perf_counter()
        row = diagnostics(rt, step, (now - t0) * 1000.0 / max(step - s0, 1))
        t0, s0 = now, step
        writer.writerow(row)
        fh.flush()
        if not quiet:
            print(f"step={step:6d} t={row['time']:9.5f} Cd={row['Cd']:10.5f} slip={row['slip_max']:.4e} "
                  f"mass={row['mass_residual_inf']:.2e} CG={row['helmholtz_iterations']:5d} "
                  f"{row['milliseconds_per_step']:8.1f} ms/step", flush=True)

    try:
        for step in range(start + 1, rt.steps + 1):
            drv.time = (step - 1) * rt.dt
            s, vc, s_old = drv.step(s, s_old, rt.dt, rt.dt, inner=rt.inner)
            drv.time = step * rt.dt
            rt.loads.advance(sphere_center(rt, drv.time), rt.dt)
            done = step
            ce = int(o["checkpoint_every"])
            due = bool((ce and step % ce == 0) or step == rt.steps or stop["flag"])
            sample = step <= 3 or step % o["sample_every"] == 0 or step == rt.steps or due
            if sample:
                sample_row(step)
            if due:
                # the history row must be durable before the checkpoint that names it
                fh.flush()
                os.fsync(fh.fileno())
                save_checkpoint(ckpt, rt, run_id, step, s, s_old)
            fe = int(o["field_every"])
            if fe and step >= int(o["field_start_step"]) and step % fe == 0 and \
                    not (step == rt.steps and o["save_field"]):
                snap_dir.mkdir(exist_ok=True)
                save_field_snapshot(snap_dir / f"field_{step:09d}.npz", rt, run_id, step, s, s_old, vc)
            if stop["flag"] and not due:
                if not sample:
                    sample_row(step)
                fh.flush()
                os.fsync(fh.fileno())
                save_checkpoint(ckpt, rt, run_id, step, s, s_old)
            if stop["flag"]:
                break
    finally:
        fh.close()
        for sig, h in old.items():
            try:
                signal.signal(sig, h)
            except (OSError, ValueError):
                pass
    if done == rt.steps and o["save_field"] and vc is not None:
        save_field_snapshot(final_path, rt, run_id, done, s, s_old, vc)
    from datetime import datetime, timezone
    meta.update(completed_utc=datetime.now(timezone.utc).isoformat(), completed_step=done,
                complete=done == rt.steps)
    _atomic_json(meta_path, meta)
    return {"completed_step": done, "stopped": done != rt.steps, "run_id": run_id,
            "body_force": rt.loads.latest["body_force"] if rt.loads.latest is not None else None}


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description="Run a PyIB case on the B200 path")
    ap.add_argument("config")
    ap.add_argument("--outdir", required=True)
    ap.add_argument("--resume", action="store_true")
    ap.add_argument("--overwrite", action="store_true")
    ap.add_argument("--steps", type=int)
    ap.add_argument("--precision", choices=["float64", "mixed"])
    a = ap.parse_args(argv)
    try:
        cfg = json.loads(Path(a.config).read_text())
        cfg.setdefault("runtime", {})["device"] = "b200"
        if a.precision:
            cfg["runtime"]["precision"] = a.precision
        if a.steps:
            cfg.setdefault("time", {})["steps"] = a.steps
        run_case(cfg, a.outdir, resume=a.resume, overwrite=a.overwrite)
    except (CaseConfigError, RuntimeError, FloatingPointError, FileExistsError) as exc:
        print(f"error: {exc}")
        return 2
    return 0
