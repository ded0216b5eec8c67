"""The dense order of the matrix-free trajectory goldens is pinned to the reference geometry.

``golden/make_golden_mf.py`` stores fields per existing edge / face / cell in
ascending dense id of the layout, mapping the reference's numbering by entity
position, and records the sha256 of the reference's edge, face and cell
positions in that order.  The layout rebuilt here must hash to the same value,
so the GPU test compares like with like.
"""
import hashlib
import json

import numpy as np
import pytest

import parity_util as PU
from pyib_b200 import layout as LY

CASES = [n for n in ("n2_fixed_mf", "n3_osc_mf", "c1_fixed") if (PU.GOLDEN / f"{n}.npz").exists()]


@pytest.mark.parametrize("name", CASES)
def test_layout_order_matches_reference_geometry(name):
    d = np.load(PU.GOLDEN / f"{name}.npz")
    par = json.loads(bytes(d["params_json"]).decode())
    lay = LY.concentric_layout(par["h"], par["half_widths"]).build()
    e = np.nonzero(lay.edge_exists)[0]
    f = np.nonzero(lay.face_exists)[0]
    c = np.nonzero(lay.cell_active)[0]
    h = hashlib.sha256()
    for a in (lay.epos[e], lay.fpos[f], lay.cpos[c]):
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    assert h.hexdigest() == bytes(d["geo_sha256"]).decode()
    ss = int(d["s_stride"]) if "s_stride" in d.files else 1
    vs = int(d["vc_stride"]) if "vc_stride" in d.files else 1
    assert d["s"].shape == (e[::ss].size,) and d["vc"].shape == (3, c[::vs].size)
    assert int(d["nedge"]) == e.size and int(d["ncell"]) == c.size
