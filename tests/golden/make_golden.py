"""Generate the golden fixtures in this folder by running the unmodified reference.

Run where the reference tree is present, named by ``PYIB_REFERENCE_ROOT``:

    python tests/golden/make_golden.py

Each ``<case>.npz`` holds the reference mesh description (``mesh_*``), its
geometry, operator outputs on seeded random inputs, immersed-boundary
stencils and force updates, one PCG solve, and a short trajectory of
``Driver.step`` with the closed-sphere loads.  The tests compare the oracle
against these values and then the product against the oracle.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import refharness as R  # noqa: E402

# name -> (h, half widths innermost first, case kwargs, trajectory steps)
CASES = {
    # uniform box like examples/cpu_fixed_sphere_smoke.json
    "u1_fixed": (0.25, [1.0], dict(inflow=1.0, Re=100.0, dt=0.01), 5),
    # two nested levels, fixed sphere in uniform inflow (the smoke-case layout at small size)
    "n2_fixed": (0.125, [0.75, 1.5], dict(inflow=1.0, Re=100.0, dt=0.0625), 20),
    # three nested levels, closed cavity, oscillating sphere (the D32 layout at small size)
    "n3_osc": (0.125, [0.75, 1.5, 3.0],
               dict(inflow=0.0, Re=0.2, dt=2 * np.pi / 3.6 / 200.0, cavity=True,
                    amplitude=0.1, frequency=3.6 / (2 * np.pi), phase=-np.pi / 2,
                    axis=(1.0, 0.0, 0.0)), 10),
}


def mesh_arrays(case):
    m = case.mesh
    return {
        "mesh_nodes": m.nodes, "mesh_F2C": m.faces_to_cells, "mesh_F2E": m.faces_to_edges,
        "mesh_E2N": m.edges_to_nodes, "mesh_link_fe_insert": m.link_fe_insert.reshape(-1, 2),
        "mesh_bc_edge": m.bc_edge, "mesh_bc_face": m.bc_face,
        "mesh_ncell": np.int64(m.cells.shape[0]), "mesh_index_cell": m.index_cell,
        "mesh_pos_ref": np.asarray(m.pos_ref), "mesh_dx": np.float64(np.asarray(m.dx_uniform)[0]),
    }


def generate(name, h, hws, kw, steps):
    R.import_reference()
    from ib_sparse import build_A
    from ib_driver_np import diag_preconditioner

    case = R.RefCase(h, hws, **kw)
    core, drv = case.core, case.driver
    out = mesh_arrays(case)
    for k in ("epos", "te", "fpos", "cpos", "nf", "Af", "vol_ci", "AoL", "fe_sign_link", "rf1", "rf2"):
        out["geo_" + k] = np.asarray(getattr(core, k))
    out["prec"] = np.asarray(drv.prec)
    out["dir_mask"] = np.asarray(drv.dir_mask)
    out["inlet"] = np.asarray(drv.inlet_edges)
    out["visc"] = np.float64(drv.visc)
    out["rou"] = np.float64(drv.rou)
    out["dt"] = np.float64(case.dt)
    out["cavity"] = np.bool_(drv.cavity)
    out["prec_dirall"] = np.asarray(diag_preconditioner(core, drv.bc_edge > 0))

    rng = np.random.default_rng(1234)
    ne, nf, nc = core.nedge, core.nface, core.ncell
    p = rng.standard_normal(ne)
    fvals = rng.standard_normal(nf)
    cvec = rng.standard_normal((nc, 3))
    cs = rng.standard_normal(nc)
    out.update(in_edge=p, in_face=fvals, in_cellvec=cvec, in_cell=cs)
    out["op_curl"] = core.curl(p)
    out["op_rot"] = core.rot(fvals)
    out["op_cdiv"] = core.cdiv(fvals)
    out["op_interp"] = core.interp_f2c(fvals)
    out["op_integr"] = core.integr_c2f(cvec)
    out["op_cgrad0"] = core.cgrad_cellscalar(cs)
    out["op_flow0"] = core.flow_mat(p)
    out["op_flowv"] = core.flow_mat(p, alpd=0.5, visc=drv.visc, rou=drv.rou, dt=case.dt)
    A = build_A(core, alpd=0.5, visc=drv.visc, rou=drv.rou, dt=case.dt)
    out["op_Ap"] = A @ p

    # velocity reconstruction + convection/diffusion on a smooth-ish random stream function
    s_in = 0.1 * rng.standard_normal(ne) + np.asarray(core.epos[:, 1] * core.te[:, 2])
    out["cv_s_in"] = s_in
    s_bc, U, vc = drv.calc_vel(s_in)
    out.update(cv_s=s_bc, cv_U=U, cv_vc=vc)
    conv, diff = drv.conv_diff(U, vc)
    out.update(cd_conv=conv, cd_diff=diff)

    # IB stencils and force update
    ib = case.ib
    mk = case.reference_markers + 0.3 * h * rng.standard_normal(case.reference_markers.shape)
    out["ib_markers"] = mk
    cell, w = ib._build_cells_weights(mk)
    out.update(ib_cell=cell, ib_w=w)
    out["ib_base"] = np.rint((mk - ib.pos_ref) / ib.dx).astype(np.int64)
    vcell = vc[:nc]
    out["ib_interp"] = ib.interp(vcell, mk)
    fl = rng.standard_normal(mk.shape)
    out["ib_fl"] = fl
    out["ib_spread"] = ib.spread(fl, mk, case.marker_widths)
    vel = rng.standard_normal(mk.shape) * 0.1
    out["ib_vel"] = vel
    fE, fL = ib.direct_force(vcell, mk, vel, case.dt, case.marker_widths)
    out.update(ib_dfE=fE, ib_dfL=fL, ib_ds=case.marker_widths)

    # one PCG solve from a warm start
    s0 = s_bc.copy()
    res_e = core.rot(core.integr_c2f(cvec * 0.01))
    out.update(hs_res=res_e, hs_s=s0)
    x, m = drv.helm_solve(res_e, s0, case.dt)
    out.update(hs_x=x, hs_iters=np.int64(m), hs_rel=np.float64(drv.last_helm_rel_residual),
               hs_ratio=np.float64(drv.last_helm_tolerance_ratio))

    # trajectory
    case2 = R.RefCase(h, hws, **kw)
    hist = []

    def cb(step, s, s_old, vc, load):
        d = case2.driver
        hist.append([step, d.helmholtz_iterations_last_step, *load.body_force, *load.force_fluid,
                     *load.body_moment, d.helmholtz_relative_residual_last_step])

    s, s_old, vc = case2.run(steps, cb)
    d2 = case2.driver
    out.update(tr_s=s, tr_s_old=s_old, tr_vc=vc[:nc], tr_fE=d2.ib_force_E, tr_fL=d2.ib_force_L,
               tr_markers=np.asarray(d2.ib_markers), tr_hist=np.asarray(hist),
               tr_steps=np.int64(steps), ref_markers=case.reference_markers,
               tr_res=np.asarray(d2.last_momentum_residual), tr_U=np.asarray(d2.last_face_flux))
    case_params = dict(h=h, half_widths=list(hws), steps=steps, **{k: (list(v) if isinstance(v, tuple) else v)
                                                                  for k, v in kw.items()})
    out["params_json"] = np.bytes_(__import__("json").dumps(case_params))
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print(name, "cells", nc, "faces", nf, "edges", ne, "links", core.lf_face.size,
          "iters", [int(r[1]) for r in hist])


if __name__ == "__main__":
    names = sys.argv[1:] or list(CASES)
    for n in names:
        generate(n, *CASES[n])
