"""Offline pressure recovery: the oracle pinned to the reference's outputs, and the
product's host-side assembly and validation (no GPU)."""
import json

import numpy as np
import pytest
from scipy.sparse import coo_matrix, diags

import pressure_oracle as PO
import parity_util as PU
from pyib_b200 import postprocess as PP

GOLD = np.load(PU.GOLDEN / "pressure_golden.npz")


def n2_inputs():
    g = PU.golden("n2_fixed")
    n = int(g["mesh_ncell"])
    return g["geo_cpos"][:n], g["mesh_F2C"], g["geo_Af"], GOLD["n2_gradient"]


def test_oracle_matches_reference_on_nested_mesh_graph():
    p, diag = PO.recover_pressure(*n2_inputs())
    want = GOLD["n2_pressure"]
    ref = json.loads(str(GOLD["n2_diag"]))
    assert np.max(np.abs(p - want)) <= 1e-13 * np.max(np.abs(want))
    assert diag["gauge"] == ref["gauge"]
    assert diag["gradient_projection_weighted_rms"] == pytest.approx(ref["gradient_projection_weighted_rms"],
                                                                     rel=1e-10)


def test_oracle_quadratic_known_answer():
    """The reference's 9^3 manufactured quadratic (tests/test_ib_postprocess.py:76-84)."""
    pos, faces, area = PO.uniform_graph(9, 0.25)
    p, diag = PO.recover_pressure(pos, faces, area, PO.quadratic_gradient(pos))
    expected = PO.quadratic(pos)
    boundary = np.unique(faces[faces[:, 1] < 0, 0])
    expected -= expected[boundary].mean()
    np.testing.assert_allclose(p, expected, atol=3e-9, rtol=1e-8)
    assert abs(p[boundary].mean()) < 1e-14
    assert diag["gradient_projection_weighted_rms"] < 1e-9
    np.testing.assert_allclose(p, GOLD["q9_pressure"], rtol=0, atol=1e-13)


def test_assembly_matches_the_incidence_form():
    """The product's sorted-key Laplacian and right-hand side equal B^T W B and B^T W j."""
    pos, faces, area, grad = n2_inputs()
    ptr, col, val, rhs, fc = PP.assemble(pos, faces, area, grad)
    n = len(pos)
    inner = faces[:, 1] >= 0
    a, b = faces[inner, 0], faces[inner, 1]
    d = pos[b] - pos[a]
    w = area[inner] / np.linalg.norm(d, axis=1)
    m = len(a)
    inc = coo_matrix((np.r_[-np.ones(m), np.ones(m)], (np.r_[np.arange(m), np.arange(m)], np.r_[a, b])),
                     shape=(m, n)).tocsr()
    lap = (inc.T @ diags(w) @ inc).tocsr()[1:, 1:].toarray()
    mine = np.zeros((n - 1, n - 1))
    rows = np.repeat(np.arange(n - 1), np.diff(ptr))
    np.add.at(mine, (rows, col), val)
    assert np.max(np.abs(mine - lap)) <= 1e-15 * np.max(np.abs(lap))
    assert np.all(np.diff(col)[np.diff(rows) == 0] > 0)        # ascending columns, no duplicates
    jump = 0.5 * np.sum((grad[a] + grad[b]) * d, axis=1)
    want = np.asarray(inc.T @ (w * jump))[1:]
    assert np.max(np.abs(rhs - want)) <= 1e-14 * np.max(np.abs(want))
    assert col.dtype == np.int32 and ptr.dtype == np.int64 and ptr[-1] == len(col)


@pytest.mark.parametrize("case, message", [
    (dict(pos=np.zeros((1, 3))), "at least two"),
    (dict(pos=np.full((1, 3), np.nan)), "cell_positions contains non-finite"),
    (dict(faces=np.array([[0.0, 1.0]])), "integer"),
    (dict(faces=np.array([[0.0, 1.0]]), grad=np.full((2, 3), np.inf)), "gradient contains non-finite"),
    (dict(grad=np.zeros((3, 3))), "gradient must have shape"),
    (dict(area=np.ones(2)), "face_area must have shape"),
    (dict(area=np.ones(2), faces=np.array([[0, 7]])), "invalid cell ids"),
])
def test_shape_errors_as_the_reference(case, message):
    """Shape and type errors are found on the host, in the reference's order."""
    kw = dict(pos=np.array([[0.0, 0, 0], [1.0, 0, 0]]), faces=np.array([[0, 1]]), area=np.ones(1),
              grad=np.zeros((2, 3)))
    kw.update(case)
    with pytest.raises(ValueError, match=message):
        PP.recover_pressure(kw["pos"], kw["faces"], kw["area"], kw["grad"])


def test_oracle_rejects_disconnected_graph():
    """The reference's own case (tests/test_ib_postprocess.py:112-116)."""
    args = (np.array([[0., 0., 0.], [1., 0., 0.], [3., 0., 0.]]), np.array([[0, 1], [2, -1]]), np.ones(2),
            np.zeros((3, 3)))
    with pytest.raises(ValueError, match="disconnected"):
        PO.recover_pressure(*args)


# ---- band repair (ib_postprocess.py:200-250) ---------------------------------
BAND = np.load(PU.GOLDEN / "band_golden.npz")
BAND_CASES = {
    "q17": dict(count=17, spacing=0.25, width=1.5),
    "n40w15": dict(count=40, spacing=1.0 / 16, width=1.5, noise=0.05, seed=7, holes=0.02),
    "n40w25": dict(count=40, spacing=1.0 / 16, width=2.5, noise=0.05, seed=7, holes=0.02),
}


def band_inputs(name):
    c = BAND_CASES[name]
    kw = {k: c[k] for k in ("noise", "seed", "holes") if k in c}
    _, dist, truth, raw, grad = PO.band_case(c["count"], c["spacing"], **kw)
    return c, dist, truth, raw, grad


@pytest.mark.parametrize("name", sorted(BAND_CASES))
def test_band_oracle_matches_reference(name):
    """The restated lsqr repair reproduces the reference's output and iteration count."""
    c, dist, _, raw, grad = band_inputs(name)
    rep, target, it = PO.repair_pressure_band(dist.shape, c["spacing"], raw, grad, dist, c["width"])
    np.testing.assert_array_equal(target, BAND[f"{name}_target"])
    assert np.max(np.abs(rep[target] - BAND[f"{name}_values"])) <= 1e-13 * np.max(np.abs(BAND[f"{name}_values"]))
    assert it == int(BAND[f"{name}_iterations"])
    np.testing.assert_array_equal(np.isnan(rep[~target]), np.isnan(raw[~target]))
    keep = ~target & np.isfinite(raw)
    np.testing.assert_array_equal(rep[keep], raw[keep])


def test_band_oracle_known_answer():
    """The reference's own bound (tests/test_ib_postprocess.py:86-95)."""
    c, dist, truth, raw, grad = band_inputs("q17")
    rep, target, _ = PO.repair_pressure_band(dist.shape, c["spacing"], raw, grad, dist)
    np.testing.assert_allclose(rep[target], truth[target], atol=1e-9, rtol=1e-9)
    np.testing.assert_array_equal(rep[~target], raw[~target])


@pytest.mark.parametrize("name", sorted(BAND_CASES))
def test_band_normal_equations_give_the_reference_solution(name):
    """The product's host system (``band_system``): the same band, a symmetric
    matrix, and -- solved exactly here -- the reference's least-squares answer to
    within lsqr's own stopping error (1e-9 of the pressure range)."""
    from scipy.sparse import csr_matrix
    from scipy.sparse.linalg import spsolve
    c, dist, _, raw, grad = band_inputs(name)
    target, ids, ptr, col, val, rhs = PP.band_system(dist.shape, c["spacing"], raw, grad, dist, c["width"])
    np.testing.assert_array_equal(target, BAND[f"{name}_target"])
    np.testing.assert_array_equal(ids, np.flatnonzero(target.ravel()))
    A = csr_matrix((val, col, ptr), shape=(len(ids), len(ids)))
    assert abs(A - A.T).max() == 0.0
    assert np.all(np.diff(col[ptr[0]:ptr[1]]) > 0)
    x = spsolve(A.tocsc(), rhs)
    want = BAND[f"{name}_values"]
    assert np.max(np.abs(x - want)) <= 1e-9 * np.max(np.abs(want))


def test_band_lattice_edges_follow_the_reference_order():
    c, dist, _, raw, _ = band_inputs("n40w15")
    valid = (dist >= 0) & np.isfinite(raw)
    for a, b in zip(PP.lattice_edges(dist.shape, valid), PO.lattice_edges(dist.shape, valid)):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("key,shift,width", [("unanchored", 0.0, 100.0), ("empty", 10.0, 1.5)])
def test_band_rejections_as_the_reference(key, shift, width):
    c, dist, _, raw, grad = band_inputs("q17")
    msg = str(BAND[f"{key}_message"])
    with pytest.raises(ValueError, match=msg.split(";")[0]):
        PO.repair_pressure_band(dist.shape, 0.25, raw, grad, dist + shift, width)
    with pytest.raises(ValueError, match=msg.split(";")[0]):
        PP.band_system(dist.shape, 0.25, raw, grad, dist + shift, width)


def test_uniform_lattice_checks_and_field():
    with pytest.raises(ValueError, match="3D integer"):
        PP.UniformLattice(np.zeros((3, 3)), np.zeros(3), 0.1)
    with pytest.raises(ValueError, match="at least two cells"):
        PP.UniformLattice(np.zeros((1, 3, 3), dtype=int), np.zeros(3), 0.1)
    ids = np.arange(27).reshape(3, 3, 3)
    ids[0, 0, 0] = -1
    lat = PP.UniformLattice(ids, np.array([1.0, 2.0, 3.0]), 0.5)
    np.testing.assert_array_equal(lat.coordinates()[2, 1, 0], [2.0, 2.5, 3.0])
    f = lat.field(np.arange(27.0))
    assert np.isnan(f[0, 0, 0]) and f[2, 2, 2] == 26.0
