"""The nested layout reproduces the reference mesh; templates + patches reproduce the operators."""
import numpy as np
import pytest

import pyib_oracle as O
import parity_util as PU
from pyib_b200 import layout as LY
from pyib_b200.operators import Operators
from pyib_b200.templates import MatvecPlan


@pytest.mark.parametrize("name", PU.CASES)
def test_export_equals_reference_mesh(name):
    g = PU.golden(name)
    lay = PU.layout_for(name)
    desc, maps = lay.export_mesh()
    m = O.MeshDesc(**desc)
    gm = O.Geometry(m)
    mr = PU.ref_mesh(name)
    assert (m.ncell, m.F2C.shape[0], m.E2N.shape[0]) == (mr.ncell, mr.F2C.shape[0], mr.E2N.shape[0])
    assert m.link_fe_insert.shape == mr.link_fe_insert.shape
    lay_, pe, pf, pc, se, sf = PU.ref_maps(name)
    e_of, f_of, c_of = maps["e_of"], maps["f_of"], maps["c_of"]
    # same geometry, orientation and boundary families per entity
    assert np.array_equal(gm.te[e_of[pe]], g["geo_te"])
    assert np.array_equal(gm.nf[f_of[pf]], g["geo_nf"])
    assert np.array_equal(gm.cpos[c_of[pc]], g["geo_cpos"])
    assert np.array_equal(gm.AoL[f_of[pf]], g["geo_AoL"])
    assert np.array_equal(gm.vol_ci[c_of[pc]], g["geo_vol_ci"])
    assert np.array_equal(m.bc_edge[e_of[pe]], g["mesh_bc_edge"])
    assert np.array_equal(m.bc_face[f_of[pf]], g["mesh_bc_face"])
    assert np.array_equal(c_of[pc][g["mesh_index_cell"]], m.index_cell)
    # the product's true geometry equals the corrected reference geometry
    assert np.array_equal(lay.cpos[pc], g["geo_cpos"])
    assert np.array_equal(lay.fpos[pf], g["geo_fpos"])


@pytest.mark.parametrize("name", PU.CASES)
def test_operators_match_oracle(name):
    g = PU.golden(name)
    lay = PU.layout_for(name)
    ops = Operators(lay)
    cav = bool(g["cavity"])
    p = PU.edge_to_dense(name, g["in_edge"])
    w = ops.flow_mat(p, 0.5, float(g["visc"]), float(g["rou"]), float(g["dt"]))
    assert PU.rel(PU.edge_from_dense(name, w), g["op_flowv"]) < 1e-14
    prec = ops.prec(ops.dir_mask(cav))
    assert np.array_equal(PU.edge_from_dense(name, prec) * PU.ref_maps(name)[4], g["prec"])
    dm = ops.dir_mask(cav)
    assert np.array_equal(dm[PU.ref_maps(name)[1]], g["dir_mask"])


@pytest.mark.parametrize("name", PU.CASES)
def test_templates_plus_patches_equal_exact(name):
    g = PU.golden(name)
    lay = PU.layout_for(name)
    ops = Operators(lay)
    dm = ops.dir_mask(bool(g["cavity"]))
    plan = MatvecPlan(ops, dm)
    rng = np.random.default_rng(11)
    for _ in range(3):
        p = rng.standard_normal(lay.NE)
        p[~lay.edge_exists] = rng.standard_normal(int((~lay.edge_exists).sum())) * 1e3  # garbage
        exact = ops.flow_mat(np.where(lay.edge_exists, p, 0.0), 0.5, 0.7, 1.3, 0.05)
        exact[~plan.mask] = 0.0
        assert PU.rel(plan.apply(p, 1.3, 0.7, 0.05), exact) < 1e-13


def test_layout_rejects_bad_boxes():
    with pytest.raises(LY.LayoutError):
        LY.NestedLayout(0.1, [((-0.25, -0.25, -0.25), (0.2, 0.25, 0.25))])        # not a multiple
    with pytest.raises(LY.LayoutError):
        LY.concentric_layout(0.125, [1.0, 1.0])                                     # not strictly inside
    with pytest.raises(LY.LayoutError):
        LY.NestedLayout(0.125, [((-0.375,) * 3, (0.375,) * 3), ((-1.0,) * 3, (1.0,) * 3)])  # odd inner count


def test_config1_layout_counts():
    """The D8 smoke layout has the reference's C1 entity counts."""
    lay = LY.concentric_layout(0.0625, [1.0, 4.0]).build()
    assert int(lay.cell_active.sum()) == 290_816
    assert int(lay.face_exists.sum()) == 887_040
    assert int(lay.edge_exists.sum()) == 901_872
    assert int(lay.link_extra.sum()) == 3_264
