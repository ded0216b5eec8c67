"""Pin the oracle against the unmodified reference (golden fixtures in tests/golden)."""
import numpy as np
import pytest

import pyib_oracle as O
import parity_util as PU


@pytest.mark.parametrize("name", PU.CASES)
def test_geometry_and_operators(name):
    g = PU.golden(name)
    m = PU.ref_mesh(name)
    geo = O.Geometry(m)
    for k in ("epos", "te", "fpos", "cpos", "nf", "Af", "vol_ci", "AoL", "fe_sign_link", "rf1", "rf2"):
        assert np.array_equal(getattr(geo, k), g["geo_" + k]), k
    assert np.array_equal(geo.curl(g["in_edge"]), g["op_curl"])
    assert np.array_equal(geo.rot(g["in_face"]), g["op_rot"])
    assert np.array_equal(geo.cdiv(g["in_face"]), g["op_cdiv"])
    assert np.array_equal(geo.interp_f2c(g["in_face"]), g["op_interp"])
    assert PU.rel(geo.integr_c2f(g["in_cellvec"]), g["op_integr"]) < 1e-15
    assert np.array_equal(geo.cgrad0(g["in_cell"]), g["op_cgrad0"])
    assert PU.rel(geo.flow_mat(g["in_edge"]), g["op_flow0"]) < 1e-15
    v = float(g["visc"]); dt = float(g["dt"]); rou = float(g["rou"])
    assert PU.rel(geo.flow_mat(g["in_edge"], 0.5, v, rou, dt), g["op_flowv"]) < 1e-15
    # the assembled CSR (ib_sparse.build_A) applies the same operator
    assert PU.rel(g["op_Ap"], g["op_flowv"]) < 1e-14


@pytest.mark.parametrize("name", PU.CASES)
def test_driver_pieces(name):
    g = PU.golden(name)
    m = PU.ref_mesh(name)
    drv = O.OracleDriver(m, float(g["visc"]), float(g["rou"]), cavity=bool(g["cavity"]))
    assert np.array_equal(drv.prec, g["prec"])
    assert np.array_equal(drv.dir_mask, g["dir_mask"])
    s, U, vc = drv.calc_vel(g["cv_s_in"])
    assert np.array_equal(s, g["cv_s"]) and np.array_equal(U, g["cv_U"]) and np.array_equal(vc, g["cv_vc"])
    conv, diff = drv.conv_diff(U, vc)
    assert np.array_equal(conv, g["cd_conv"]) and np.array_equal(diff, g["cd_diff"])
    x, st = drv.helm_solve(g["hs_res"], g["hs_s"], float(g["dt"]))
    # the reference solves with its CSR matrix, the oracle matrix-free: same iterations,
    # iterates equal to rounding amplified by CG
    assert st.iterations == int(g["hs_iters"])
    assert PU.rel(x, g["hs_x"]) < 1e-10


@pytest.mark.parametrize("name", PU.CASES)
def test_immersed_boundary(name):
    g = PU.golden(name)
    m = PU.ref_mesh(name)
    ib = O.IBStencil(m)
    st = ib.build(g["ib_markers"])
    assert np.array_equal(ib.base_index(g["ib_markers"]), g["ib_base"])
    assert np.array_equal(st[0], g["ib_cell"]) and np.array_equal(st[1], g["ib_w"])
    nc = int(g["mesh_ncell"])
    assert np.array_equal(ib.interp(g["cv_vc"][:nc], st), g["ib_interp"])
    assert np.array_equal(ib.spread(g["ib_fl"], st, g["ib_ds"]), g["ib_spread"])
    fE, fL = ib.direct_force(g["cv_vc"][:nc], g["ib_markers"], g["ib_vel"], float(g["dt"]), g["ib_ds"])
    assert np.array_equal(fE, g["ib_dfE"]) and np.array_equal(fL, g["ib_dfL"])


def test_partition_of_unity_and_conservation():
    """ib_immersed.py:192-209 self-tests, restated on the oracle."""
    name = "n2_fixed"
    m = PU.ref_mesh(name)
    g = PU.golden(name)
    ib = O.IBStencil(m)
    rng = np.random.default_rng(0)
    mk = rng.uniform(-0.4, 0.4, size=(200, 3))
    st = ib.build(mk)
    one = np.ones((m.ncell, 1))
    assert np.max(np.abs(ib.interp(one, st)[:, 0] - 1.0)) < 1e-13
    x = g["geo_cpos"][:, 0:1]
    assert np.max(np.abs(ib.interp(x, st)[:, 0] - mk[:, 0])) < 1e-13
    ds = np.full(200, 0.125)
    f = rng.standard_normal((200, 3))
    FE = ib.spread(f, st, ds)
    assert np.max(np.abs(FE.sum(axis=0) * ib.hh ** 3 - (f * ds[:, None] ** 3).sum(axis=0))) < 1e-14


def test_oracle_trajectory_short():
    """Five steps of the oracle against the reference trajectory's first steps (u1_fixed)."""
    name = "u1_fixed"
    g = PU.golden(name)
    par = g["params"]
    m = PU.ref_mesh(name)
    drv = O.OracleDriver(m, float(g["visc"]), float(g["rou"]))
    ib = O.IBStencil(m)
    ref = g["ref_markers"]
    drv.set_ib(ib, ref, g["ib_ds"], np.zeros_like(ref))
    geo = drv.g
    s = 1.0 * geo.epos[:, 1] * geo.te[:, 2]
    s, _, vc = drv.calc_vel(s)
    s_old = s.copy()
    dt = float(g["dt"])
    its = []
    for k in range(int(g["tr_steps"])):
        s, vc, s_old = drv.step(s, s_old, dt, dt, 4)
        its.append(max(st.iterations for st in drv.last_stats))
    assert its == [int(v) for v in g["tr_hist"][:, 1]]
    assert PU.rel(s, g["tr_s"]) < 1e-10
    assert PU.rel(drv.fL, g["tr_fL"]) < 1e-10
