"""GPU parity: the CUDA path through the C ABI against the oracle and the reference goldens."""
import ctypes as C

import numpy as np
import pytest

import pyib_oracle as O
import parity_util as PU
from pyib_b200 import _lib
from pyib_b200.device import DeviceSolver
from pyib_b200.driver import B200Driver

pytestmark = pytest.mark.gpu


def _solver(name, **kw):
    g = PU.golden(name)
    lay = PU.layout_for(name)
    return DeviceSolver(lay, rou=float(g["rou"]), visc=float(g["visc"]), cavity=bool(g["cavity"]), **kw)


@pytest.mark.parametrize("name", PU.CASES)
def test_matvec_matches_reference(name):
    g = PU.golden(name)
    sv = _solver(name)
    p = PU.edge_to_dense(name, g["in_edge"])
    sv.set("WORK_E", p)
    dt = float(g["dt"])
    sv.h.call("pyib_matvec", _lib.F["WORK_E"], _lib.F["WORK_E2"], C.c_double(dt), 1)
    w = sv.get("WORK_E2")
    ref = g["op_flowv"].copy()
    ref[g["dir_mask"]] = 0.0
    assert PU.rel(PU.edge_from_dense(name, w), ref) < 1e-13
    # the numpy mirror of the same kernels agrees too
    mirror = sv.plan.apply(p, float(g["rou"]), float(g["visc"]), dt)
    assert PU.rel(w, mirror) < 1e-13
    # alpd = 0 (no viscous block)
    sv.h.call("pyib_matvec", _lib.F["WORK_E"], _lib.F["WORK_E2"], C.c_double(dt), 0)
    ref0 = g["op_flow0"].copy()
    ref0[g["dir_mask"]] = 0.0
    assert PU.rel(PU.edge_from_dense(name, sv.get("WORK_E2")), ref0) < 1e-13


@pytest.mark.parametrize("name", PU.CASES)
def test_step_operators(name):
    g = PU.golden(name)
    sv = _solver(name)
    lay = sv.lay
    sv.set("WORK_E", PU.edge_to_dense(name, g["in_edge"]))
    sv.h.call("pyib_operator", 0)
    assert PU.rel(PU.face_from_dense(name, sv.get("WORK_F")), g["op_curl"]) < 1e-14
    sv.set("WORK_F", PU.face_to_dense(name, g["in_face"]))
    sv.h.call("pyib_operator", 1)
    assert PU.rel(PU.edge_from_dense(name, sv.get("WORK_E")), g["op_rot"]) < 1e-14
    sv.h.call("pyib_operator", 2)
    v = sv.get("WORK_C3").reshape(3, -1)
    assert PU.rel(PU.cell3_from_dense(name, v), g["op_interp"]) < 1e-14
    sv.set("WORK_C3", PU.cell3_to_dense(name, g["in_cellvec"]))
    sv.h.call("pyib_operator", 3)
    assert PU.rel(PU.face_from_dense(name, sv.get("WORK_F")), g["op_integr"]) < 1e-14


@pytest.mark.parametrize("name", PU.CASES)
def test_calc_vel_and_conv_diff(name):
    g = PU.golden(name)
    sv = _solver(name)
    sv.set("S", PU.edge_to_dense(name, g["cv_s_in"]))
    sv.h.call("pyib_calc_vel")
    assert PU.rel(PU.edge_from_dense(name, sv.get("S")), g["cv_s"]) < 1e-15
    assert PU.rel(PU.face_from_dense(name, sv.get("U")), g["cv_U"]) < 1e-14
    nc_ref = int(g["mesh_ncell"])
    vc = sv.vc_cells()
    assert PU.rel(PU.cell3_from_dense(name, vc), g["cv_vc"][:nc_ref]) < 1e-14
    sv.h.call("pyib_conv_diff")
    conv = sv.get("WORK_C3").reshape(3, -1)
    diff = sv.get("RES_C").reshape(3, -1)
    assert PU.rel(PU.cell3_from_dense(name, conv), g["cd_conv"]) < 1e-13
    assert PU.rel(PU.cell3_from_dense(name, diff), g["cd_diff"]) < 1e-13


@pytest.mark.parametrize("name", PU.CASES)
def test_ib_stencil_bit_exact_and_transfer(name):
    g = PU.golden(name)
    sv = _solver(name)
    mk = g["ib_markers"]
    sv.set_markers(mk, g["ib_vel"], g["ib_ds"])
    sv.h.call("pyib_ib_stencil")
    base = sv.get("IB_BASE").reshape(-1, 3)
    assert np.array_equal(base, g["ib_base"])
    cell = sv.get("IB_CELL").reshape(-1, 125)
    w = sv.get("IB_W").reshape(-1, 125)
    lay, pe, pf, pc, se, sf = PU.ref_maps(name)
    assert np.array_equal(cell, pc[g["ib_cell"]])          # same cells, bit-exact
    assert np.array_equal(w, g["ib_w"])                    # same weights, bit-exact
    sv.set("VC", np.concatenate([PU.cell3_to_dense(name, g["cv_vc"][:int(g["mesh_ncell"])]),
                                 np.zeros((3, sv.bfaces.size))], axis=1))
    sv.h.call("pyib_ib_interp")
    assert PU.rel(sv.get("LAG_TMP").reshape(-1, 3), g["ib_interp"]) < 1e-14
    sv.set("FL", g["ib_fl"])
    sv.h.call("pyib_ib_spread")
    fE = sv.get("FE").reshape(3, -1)
    # spreading sums in np.bincount order: bit-exact
    assert np.array_equal(PU.cell3_from_dense(name, fE), g["ib_spread"])


@pytest.mark.parametrize("name", PU.CASES)
def test_helm_solve(name):
    g = PU.golden(name)
    lay = PU.layout_for(name)
    drv = B200Driver(lay, float(g["visc"]), float(g["rou"]))
    if bool(g["cavity"]):
        drv.set_cavity(0.0, False)
    x, m = drv.helm_solve(PU.edge_to_dense(name, g["hs_res"]), PU.edge_to_dense(name, g["hs_s"]),
                          float(g["dt"]))
    assert m == int(g["hs_iters"])
    assert PU.rel(PU.edge_from_dense(name, x), g["hs_x"]) < 1e-10
