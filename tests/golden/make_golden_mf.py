"""Trajectory goldens from the reference's matrix-free path (``solver.sparse = false``).

    PYIB_REFERENCE_ROOT=<reference tree> python tests/golden/make_golden_mf.py [case ...] [--out=PATH]

    # the reference's own spread: the same case with one BLAS thread, then
    OPENBLAS_NUM_THREADS=1 ... make_golden_mf.py CASE --out=/tmp/CASE_blas1.npz
    python tests/golden/add_self_spread.py CASE /tmp/CASE_blas1.npz

The reference's ``sparse = false`` path applies the Helmholtz operator with
``IBCore.flow_mat`` (``ib_core_np.py:168-175``) instead of its assembled CSR
matrix (``ib_sparse.py:69-96``).  It is the same algorithm as the structured
matvec of the B200 path, so the trajectories of the two differ only by the
rounding of each product.

Cases:

* ``c1_fixed`` -- the smoke configuration: sphere of D = 8 finest cells
  (h = D/8 = 0.0625), finest box [-2D, 2D]^3, the 16D cube [-8D, 8D]^3 at 2h
  (2 levels, 290,816 cells, 901,872 edges), uniform inflow U = 1, Re = 100,
  201 Fibonacci markers, dt = CFL 0.5 * h / U = 0.03125, 4 inner iterations,
  CG tolerances 1e-10 / 1e-9, check interval 20, at most 1000 CG iterations
  (the reference defaults, ``ib_case.py:56-97``), 20 steps from the
  uniform-flow stream function.  Several CPU hours.
* ``n2_fixed_mf`` / ``n3_osc_mf`` -- the small fixtures of ``make_golden.py``
  rerun through the matrix-free path (minutes).

Fields are stored in the B200 layout's dense order (existing entities in
ascending dense id, edge values signed to the +axis orientation), so the test
needs neither the reference mesh nor its numbering.  The map from reference ids
to dense ids is built here from entity positions; ``geo_sha256`` records the
reference geometry in that order, and a CPU test rebuilds the layout and checks
that its own geometry hashes to the same value.
"""
from __future__ import annotations

import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(ROOT))
import refharness as R  # noqa: E402

CASES = {
    "c1_fixed": (0.0625, [1.0, 4.0], dict(inflow=1.0, Re=100.0, dt=0.03125, cg_max_iterations=1000), 20),
    "n2_fixed_mf": (0.125, [0.75, 1.5], dict(inflow=1.0, Re=100.0, dt=0.0625), 20),
    "n3_osc_mf": (0.125, [0.75, 1.5, 3.0],
                  dict(inflow=0.0, Re=0.2, dt=2 * np.pi / 3.6 / 200.0, cavity=True,
                       amplitude=0.1, frequency=3.6 / (2 * np.pi), phase=-np.pi / 2,
                       axis=(1.0, 0.0, 0.0)), 10),
}


def _keys(pos, axis, h):
    k = np.rint(pos / (h / 2)).astype(np.int64)
    return ((k[:, 0] * 4_000_003 + k[:, 1]) * 4_000_037 + k[:, 2]) * 3 + axis


def _perm(pm, am, pr, ar, h):
    """p[i] = index into the product's list of the reference entity i."""
    km, kr = _keys(pm, am, h), _keys(pr, ar, h)
    om, orr = np.argsort(km), np.argsort(kr)
    if not np.array_equal(km[om], kr[orr]):
        raise AssertionError("entity sets differ")
    p = np.empty(kr.size, dtype=np.int64)
    p[orr] = om
    return p


def geometry_hash(epos, fpos, cpos):
    """sha256 over edge, face and cell positions (dense-existing order)."""
    h = hashlib.sha256()
    for a in (epos, fpos, cpos):
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def dense_maps(case, h, half_widths):
    """Reference id -> position in the dense-existing lists, and edge signs."""
    import _pyib_b200_import
    _pyib_b200_import.load()
    from pyib_b200 import layout as LY
    lay = LY.concentric_layout(h, half_widths).build()
    core = case.core
    e = np.nonzero(lay.edge_exists)[0]
    f = np.nonzero(lay.face_exists)[0]
    c = np.nonzero(lay.cell_active)[0]
    te, nf = np.asarray(core.te), np.asarray(core.nf)
    ea = np.argmax(np.abs(te), axis=1)
    fa = np.argmax(np.abs(nf), axis=1)
    pe = _perm(lay.epos[e], lay.edge_axis[e], np.asarray(core.epos), ea, h)
    pf = _perm(lay.fpos[f], lay.face_axis[f], np.asarray(core.fpos), fa, h)
    pc = _perm(lay.cpos[c], np.zeros(c.size, int), np.asarray(core.cpos)[: core.ncell],
               np.zeros(core.ncell, int), h)
    se = np.sign(te[np.arange(te.shape[0]), ea])
    # reference geometry in dense-existing order
    epos_d = np.empty_like(np.asarray(core.epos)); epos_d[pe] = core.epos
    fpos_d = np.empty_like(np.asarray(core.fpos)); fpos_d[pf] = core.fpos
    cpos_d = np.empty((core.ncell, 3)); cpos_d[pc] = np.asarray(core.cpos)[: core.ncell]
    ghash = geometry_hash(epos_d, fpos_d, cpos_d)
    own = geometry_hash(lay.epos[e], lay.fpos[f], lay.cpos[c])
    for nm, a, b in (("epos", epos_d, lay.epos[e]), ("fpos", fpos_d, lay.fpos[f]), ("cpos", cpos_d, lay.cpos[c])):
        if not np.array_equal(a, b):
            print("geometry differs:", nm, float(np.max(np.abs(a - b))), flush=True)
    return pe, pf, pc, se, ghash, own


def to_dense_edge(v, pe, se):
    out = np.empty(v.shape[0]); out[pe] = v * se
    return out


def to_dense_cell3(v, pc):
    out = np.empty((3, pc.size)); out[:, pc] = np.asarray(v)[: pc.size].T
    return out


def generate(name, h, hws, kw, steps, progress_dir=None, out_path=None):
    R.import_reference()
    case = R.RefCase(h, hws, sparse=False, **kw)
    core, drv = case.core, case.driver
    pe, pf, pc, se, ghash, own = dense_maps(case, h, hws)
    print(name, "cells", core.ncell, "edges", core.nedge, "markers", case.reference_markers.shape[0],
          "geometry hash equal:", ghash == own, flush=True)
    solves = []
    orig = drv.helm_solve

    def counted(*a, **k):
        out = orig(*a, **k)
        solves[-1].append((int(drv.last_helm_m), float(drv.last_helm_rel_residual),
                           float(drv.last_helm_tolerance_ratio)))
        return out

    drv.helm_solve = counted
    hist = []
    stencil = {}
    t0 = time.time()

    def cb(step, s, s_old, vc, load):
        d = case.driver
        hist.append([step, d.helmholtz_iterations_last_step, *load.body_force, *load.force_fluid,
                     *load.body_moment, d.helmholtz_relative_residual_last_step])
        if step == 1:
            cell, w = case.ib._build_cells_weights(np.asarray(d.ib_markers))
            stencil["cell"], stencil["w"] = np.asarray(cell), np.asarray(w)
        print(f"{name} step {step} solves {[x[0] for x in solves[-1]]} "
              f"elapsed {time.time() - t0:.0f}s", flush=True)
        if progress_dir is not None:
            np.savez(Path(progress_dir) / f"{name}_step{step:03d}.npz", s=s, vc=vc[: core.ncell],
                     fE=np.asarray(d.ib_force_E), fL=np.asarray(d.ib_force_L))

    s, s_old, vc = _run(case, steps, cb, solves)
    fE = to_dense_cell3(np.asarray(drv.ib_force_E), pc)
    nz = np.nonzero(np.any(fE != 0.0, axis=0))[0]
    inv_c = np.empty(core.ncell, dtype=np.int64); inv_c[:] = pc        # reference cell -> dense-existing
    cell = stencil["cell"]
    out = dict(
        s=to_dense_edge(np.asarray(s), pe, se),
        vc=to_dense_cell3(vc, pc),
        fE_idx=nz.astype(np.int32), fE_val=fE[:, nz],
        fL=np.asarray(drv.ib_force_L),
        markers=np.asarray(drv.ib_markers), ref_markers=case.reference_markers,
        ib_ds=case.marker_widths,
        stencil_cell=np.where(cell >= 0, inv_c[np.maximum(cell, 0)], -1).astype(np.int32),
        stencil_w=stencil["w"],
        solve_iters=np.array([[x[0] for x in st] for st in solves], dtype=np.int64),
        solve_rel=np.array([[x[1] for x in st] for st in solves]),
        solve_ratio=np.array([[x[2] for x in st] for st in solves]),
        hist=np.asarray(hist), visc=np.float64(drv.visc), rou=np.float64(drv.rou),
        dt=np.float64(case.dt), cavity=np.bool_(drv.cavity), steps=np.int64(steps),
        ncell=np.int64(core.ncell), nedge=np.int64(core.nedge),
        geo_sha256=np.bytes_(ghash),
        seconds=np.float64(time.time() - t0),
    )
    params = dict(h=h, half_widths=list(hws), steps=steps, sparse=False,
                  **{k: (list(v) if isinstance(v, tuple) else v) for k, v in kw.items()})
    out["params_json"] = np.bytes_(json.dumps(params))
    np.savez_compressed(Path(out_path) if out_path else HERE / f"{name}.npz", **out)
    print(name, "done", "iters per step", [int(r[1]) for r in hist], f"{time.time() - t0:.0f}s", flush=True)


def _run(case, steps, cb, solves):
    """The step loop of ``ib_case.run_case`` (lines 1518-1530), opening a solve log per step."""
    s, s_old, vc = case.initial_state()
    drv = case.driver
    for step in range(1, steps + 1):
        solves.append([])
        drv.time = (step - 1) * case.dt
        s, vc, s_old = drv.step(s, s_old, case.dt, dt_old=case.dt, inner=case.inner)
        drv.time = step * case.dt
        load = case.load.advance(vc[: case.core.ncell], case.centre(drv.time), case.dt, drv.ib_force_E)
        cb(step, s, s_old, vc, load)
    return s, s_old, vc


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    prog = out = None
    for a in sys.argv[1:]:
        if a.startswith("--progress="):
            prog = a.split("=", 1)[1]
        if a.startswith("--out="):
            out = a.split("=", 1)[1]
    for n in args or list(CASES):
        generate(n, *CASES[n], progress_dir=prog, out_path=out)
