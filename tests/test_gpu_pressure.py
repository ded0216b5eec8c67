"""Offline pressure recovery with the graph CG on the device, against the oracle
and the reference's outputs (tests/golden/pressure_golden.npz)."""
import ctypes as C
import json

import numpy as np
import pytest

import pressure_oracle as PO
import parity_util as PU
from pyib_b200 import _lib
from pyib_b200 import postprocess as PP

pytestmark = pytest.mark.gpu

GOLD = np.load(PU.GOLDEN / "pressure_golden.npz")


def n2_inputs():
    g = PU.golden("n2_fixed")
    n = int(g["mesh_ncell"])
    return g["geo_cpos"][:n], g["mesh_F2C"], g["geo_Af"], GOLD["n2_gradient"]


def test_nested_mesh_graph_matches_reference():
    """Same stop test as scipy's cg: the pressure agrees to rounding of the
    iterates (1e-9 of its range; the CG stops at |r| < 1e-10 |b|)."""
    args = n2_inputs()
    p, diag = PP.recover_pressure(*args)
    want = GOLD["n2_pressure"]
    ref = json.loads(str(GOLD["n2_diag"]))
    assert np.max(np.abs(p - want)) <= 1e-9 * np.max(np.abs(want))
    assert diag["gauge"] == ref["gauge"]
    assert diag["gradient_projection_weighted_rms"] == pytest.approx(ref["gradient_projection_weighted_rms"],
                                                                     rel=1e-8)
    _, odiag = PO.recover_pressure(*args)
    assert abs(diag["iterations"] - odiag["iterations"]) <= 2
    # deterministic: a second call gives the same bits
    p2, _ = PP.recover_pressure(*args)
    np.testing.assert_array_equal(p, p2)


def test_quadratic_known_answer_9():
    """The reference's 9^3 case and bounds (tests/test_ib_postprocess.py:76-84)."""
    pos, faces, area = PO.uniform_graph(9, 0.25)
    p, diag = PP.recover_pressure(pos, faces, area, PO.quadratic_gradient(pos))
    expected = PO.quadratic(pos)
    boundary = np.unique(faces[faces[:, 1] < 0, 0])
    expected -= expected[boundary].mean()
    np.testing.assert_allclose(p, expected, atol=3e-9, rtol=1e-8)
    assert abs(p[boundary].mean()) < 1e-14
    assert diag["gradient_projection_weighted_rms"] < 1e-9
    np.testing.assert_allclose(p, GOLD["q9_pressure"], rtol=0, atol=1e-12)


def test_noisy_48_matches_oracle():
    pos, faces, area = PO.uniform_graph(48, 1.0 / 48)
    rng = np.random.default_rng(3)
    grad = PO.quadratic_gradient(pos) + 0.1 * rng.standard_normal(pos.shape)
    p, diag = PP.recover_pressure(pos, faces, area, grad)
    q, odiag = PO.recover_pressure(pos, faces, area, grad)
    assert np.max(np.abs(p - q)) <= 1e-9 * np.max(np.abs(q))
    assert abs(diag["iterations"] - odiag["iterations"]) <= 2
    assert diag["gradient_projection_weighted_rms"] == pytest.approx(odiag["gradient_projection_weighted_rms"],
                                                                     rel=1e-8)


def test_quadratic_known_answer_128_cubed():
    """2.1 M cells: the projection of an exact quadratic gradient is the quadratic
    (second-order jumps are exact on a uniform lattice), to the CG tolerance."""
    c = 128
    pos, faces, area = PO.uniform_graph(c, 1.0 / c)
    p, diag = PP.recover_pressure(pos, faces, area, PO.quadratic_gradient(pos))
    expected = PO.quadratic(pos)
    boundary = np.unique(faces[faces[:, 1] < 0, 0])
    expected -= expected[boundary].mean()
    assert np.max(np.abs(p - expected)) <= 1e-9
    assert diag["gradient_projection_weighted_rms"] < 1e-9
    assert 0 < diag["iterations"] < 10 * c ** 3


def test_default_context_is_kept_and_can_be_released():
    args = n2_inputs()
    PP.recover_pressure(*args)
    h = PP.default_handle(0)
    PP.recover_pressure(*args)
    assert PP.default_handle(0) is h            # the same context, its workspace kept
    PP.close_default_handles()
    assert not h.ptr
    p, _ = PP.recover_pressure(*args)           # a new one is made on demand
    assert PP.default_handle(0) is not h
    assert np.max(np.abs(p - GOLD["n2_pressure"])) <= 1e-9 * np.max(np.abs(GOLD["n2_pressure"]))


def test_solver_handle_is_reused_and_errors_are_reported():
    args = n2_inputs()
    h = PP.bare_handle(0)
    try:
        p, _ = PP.recover_pressure(*args, handle=h)
        np.testing.assert_array_equal(p, PP.recover_pressure(*args)[0])
        ptr, col, val, rhs, _ = PP.assemble(*args)
        with pytest.raises(_lib.B200Error) as exc:
            PP.graph_pcg(h, ptr, col, val, rhs, 1e-10, 3)
        assert exc.value.code == _lib.E_NOCONV
        bad = col.copy()
        bad[5] = len(rhs)                   # rejected on the host before any launch
        with pytest.raises(_lib.B200Error) as exc:
            PP.graph_pcg(h, ptr, bad, val, rhs, 1e-10, 100)
        assert exc.value.code == _lib.E_ARG
        # the context stays usable after both errors
        x, it = PP.graph_pcg(h, ptr, col, val, rhs, 1e-10, 5000)
        assert it > 0 and np.all(np.isfinite(x))
    finally:
        h.close()


@pytest.mark.parametrize("case, message", [
    (dict(faces=np.array([[0, 5]])), "face_cells contains invalid cell ids"),
    (dict(faces=np.array([[0, 1], [1, -2]]), area=np.ones(2)), "face_cells contains invalid cell ids"),
    (dict(area=np.array([-1.0])), "face areas must be positive"),
    (dict(area=np.array([np.nan])), "face_area contains non-finite values"),
    (dict(grad=np.full((2, 3), np.nan)), "gradient contains non-finite values"),
    (dict(pos=np.array([[0.0, 0, 0], [np.inf, 0, 0]]), area=np.array([-1.0])),
     "cell_positions contains non-finite values"),
    (dict(faces=np.array([[0, -1]])), "pressure graph has no valid internal faces"),
    (dict(pos=np.zeros((2, 3))), "pressure graph has no valid internal faces"),
])
def test_value_errors_found_on_the_device(case, message):
    """Value checks run on the device and report the reference's first failing check."""
    kw = dict(pos=np.array([[0.0, 0, 0], [1.0, 0, 0]]), faces=np.array([[0, 1]]), area=np.ones(1),
              grad=np.zeros((2, 3)))
    kw.update(case)
    with pytest.raises(ValueError, match=message):
        PP.recover_pressure(kw["pos"], kw["faces"], kw["area"], kw["grad"])
    with pytest.raises(ValueError, match=message):
        PO.recover_pressure_checked(kw["pos"], kw["faces"], kw["area"], kw["grad"])


def test_disconnected_graph_is_rejected():
    """The reference's own case (tests/test_ib_postprocess.py:112-116), and a
    two-block lattice with no face between the blocks."""
    with pytest.raises(ValueError, match="disconnected"):
        PP.recover_pressure(np.array([[0., 0., 0.], [1., 0., 0.], [3., 0., 0.]]), np.array([[0, 1], [2, -1]]),
                            np.ones(2), np.zeros((3, 3)))
    pos, faces, area = PO.uniform_graph(8, 0.25)
    keep = ~((faces[:, 1] >= 0) & ((pos[faces[:, 0], 0] < 0) != (pos[np.maximum(faces[:, 1], 0), 0] < 0)))
    with pytest.raises(ValueError, match="disconnected"):
        PP.recover_pressure(pos, faces[keep], area[keep], np.zeros_like(pos))


def test_device_assembly_matches_host_assembly():
    """The device's CSR (sorted rows, diagonal first) and the host's sorted-key CSR
    solve the same system: the pressures agree to the CG tolerance."""
    args = n2_inputs()
    p, diag = PP.recover_pressure(*args)
    h = PP.bare_handle(0)
    try:
        ptr, col, val, rhs, _ = PP.assemble(*args)
        x, it = PP.graph_pcg(h, ptr, col, val, rhs, 1e-10, 32400)
    finally:
        h.close()
    q = np.r_[0.0, x]
    boundary = np.unique(args[1][args[1][:, 1] < 0, 0])
    q -= q[boundary].mean()
    assert np.max(np.abs(p - q)) <= 1e-9 * np.max(np.abs(q))
    assert abs(it - diag["iterations"]) <= 2


def test_edge_cases_match_oracle():
    """The smallest graph, duplicate faces between one pair of cells (summed in the
    reference's Laplacian, kept as separate entries here), and unsigned face ids
    with no boundary face (gauge: the mean over all cells)."""
    rng = np.random.default_rng(21)
    # two cells, one internal face, two boundary faces
    pos = np.array([[0.0, 0.0, 0.0], [0.5, 0.0, 0.0]])
    faces = np.array([[0, 1], [0, -1], [1, -1]])
    grad = rng.standard_normal((2, 3))
    p, d = PP.recover_pressure(pos, faces, np.ones(3), grad)
    q, e = PO.recover_pressure(pos, faces, np.ones(3), grad)
    np.testing.assert_allclose(p, q, rtol=0, atol=1e-14)
    assert d["gauge"] == e["gauge"] == "mean boundary-adjacent cells = 0"
    # duplicate faces on a 6^3 lattice: every x face listed twice with split areas
    pos, faces, area = PO.uniform_graph(6, 0.25)
    xf = (faces[:, 1] >= 0) & (pos[np.maximum(faces[:, 1], 0), 0] != pos[faces[:, 0], 0])
    faces2 = np.concatenate([faces, faces[xf]])
    area2 = np.concatenate([np.where(xf, 0.25 * area, area), 0.75 * area[xf]])
    grad = PO.quadratic_gradient(pos) + 0.05 * rng.standard_normal(pos.shape)
    p, d = PP.recover_pressure(pos, faces2, area2, grad)
    q, e = PO.recover_pressure(pos, faces2, area2, grad)
    assert np.max(np.abs(p - q)) <= 1e-9 * np.max(np.abs(q))
    assert abs(d["gradient_projection_weighted_rms"] - e["gradient_projection_weighted_rms"]) <= \
        1e-8 * e["gradient_projection_weighted_rms"]
    # unsigned ids, internal faces only
    inner = faces[faces[:, 1] >= 0].astype(np.uint32)
    p, d = PP.recover_pressure(pos, inner, np.ones(len(inner)), grad)
    q, e = PO.recover_pressure(pos, inner, np.ones(len(inner)), grad)
    assert d["gauge"] == e["gauge"] == "mean cells = 0"
    assert abs(p.mean()) < 1e-14
    assert np.max(np.abs(p - q)) <= 1e-9 * np.max(np.abs(q))


# ---- band repair on the device (ib_postprocess.py:213-250) -------------------
BAND = np.load(PU.GOLDEN / "band_golden.npz")
BAND_CASES = {
    "q17": dict(count=17, spacing=0.25, width=1.5),
    "n40w15": dict(count=40, spacing=1.0 / 16, width=1.5, noise=0.05, seed=7, holes=0.02),
    "n40w25": dict(count=40, spacing=1.0 / 16, width=2.5, noise=0.05, seed=7, holes=0.02),
}


def _band(name):
    c = BAND_CASES[name]
    kw = {k: c[k] for k in ("noise", "seed", "holes") if k in c}
    _, dist, truth, raw, grad = PO.band_case(c["count"], c["spacing"], **kw)
    ids = np.arange(c["count"] ** 3).reshape((c["count"],) * 3)
    lat = PP.UniformLattice(ids, np.full(3, -0.5 * (c["count"] - 1) * c["spacing"]), c["spacing"])
    return c, lat, dist, truth, raw, grad


@pytest.mark.parametrize("name", sorted(BAND_CASES))
def test_band_repair_matches_reference(name):
    """The device CG on the normal equations reaches the reference's lsqr answer
    to lsqr's own stopping error (1e-9 of the pressure range); cells outside the
    band are returned bit for bit."""
    c, lat, dist, _, raw, grad = _band(name)
    rep, target, it = PP.repair_pressure_band(lat, raw, grad, dist, width=c["width"])
    np.testing.assert_array_equal(target, BAND[f"{name}_target"])
    want = BAND[f"{name}_values"]
    assert np.max(np.abs(rep[target] - want)) <= 1e-9 * np.max(np.abs(want))
    keep = ~target & np.isfinite(raw)
    np.testing.assert_array_equal(rep[keep], raw[keep])
    np.testing.assert_array_equal(np.isnan(rep), np.isnan(raw) & ~target)
    assert 0 < it <= max(500, 20 * int(target.sum()))
    rep2, _, it2 = PP.repair_pressure_band(lat, raw, grad, dist, width=c["width"])
    np.testing.assert_array_equal(rep, rep2)
    assert it2 == it


def test_band_repair_known_answer():
    """The reference's own case and bound (tests/test_ib_postprocess.py:86-95)."""
    c, lat, dist, truth, raw, grad = _band("q17")
    rep, target, _ = PP.repair_pressure_band(lat, raw, grad, dist)
    np.testing.assert_allclose(rep[target], truth[target], atol=1e-9, rtol=1e-9)
    np.testing.assert_array_equal(rep[~target], raw[~target])


@pytest.mark.parametrize("key,shift,width", [("unanchored", 0.0, 100.0), ("empty", 10.0, 1.5)])
def test_band_repair_rejections(key, shift, width):
    c, lat, dist, _, raw, grad = _band("q17")
    with pytest.raises(ValueError) as e:
        PP.repair_pressure_band(lat, raw, grad, dist + shift, width=width)
    assert str(e.value) == str(BAND[f"{key}_message"])
