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
