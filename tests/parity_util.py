"""Shared helpers: golden fixtures, layouts and reference<->dense id maps."""
from __future__ import annotations

import json
from functools import lru_cache
from pathlib import Path

import numpy as np

import pyib_oracle as O
from pyib_b200 import layout as LY

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = ("u1_fixed", "n2_fixed", "n3_osc")


@lru_cache(maxsize=None)
def golden(name):
    d = np.load(GOLDEN / f"{name}.npz")
    out = {k: d[k] for k in d.files}
    out["params"] = json.loads(bytes(out["params_json"]).decode())
    return out


def layout_for(name):
    par = golden(name)["params"]
    return LY.concentric_layout(par["h"], par["half_widths"]).build()


def _keys(pos, axis, h):
    k = np.rint(pos / (h / 2)).astype(np.int64)
    return ((k[:, 0] * 4_000_003 + k[:, 1]) * 4_000_037 + k[:, 2]) * 3 + axis


def _perm(pm, am, pr, ar, h):
    km, kr = _keys(pm, am, h), _keys(pr, ar, h)
    om, orr = np.argsort(km), np.argsort(kr)
    if not np.array_equal(km[om], kr[orr]):
        raise AssertionError("entity sets differ")
    p = np.empty(kr.size, dtype=np.int64)
    p[orr] = om
    return p


@lru_cache(maxsize=None)
def ref_maps(name):
    """Dense ids of the reference's edges/faces/cells and the +a orientation signs."""
    g = golden(name)
    lay = layout_for(name)
    h = g["params"]["h"]
    e = np.nonzero(lay.edge_exists)[0]
    f = np.nonzero(lay.face_exists)[0]
    c = np.nonzero(lay.cell_active)[0]
    te, nf = g["geo_te"], g["geo_nf"]
    ea = np.argmax(np.abs(te), axis=1)
    fa = np.argmax(np.abs(nf), axis=1)
    pe = e[_perm(lay.epos[e], lay.edge_axis[e], g["geo_epos"], ea, h)]
    pf = f[_perm(lay.fpos[f], lay.face_axis[f], g["geo_fpos"], fa, h)]
    pc = c[_perm(lay.cpos[c], np.zeros(c.size, int), g["geo_cpos"], np.zeros(g["geo_cpos"].shape[0], int), h)]
    se = np.sign(te[np.arange(te.shape[0]), ea])
    sf = np.sign(nf[np.arange(nf.shape[0]), fa])
    return lay, pe, pf, pc, se, sf


def edge_to_dense(name, v_ref):
    lay, pe, pf, pc, se, sf = ref_maps(name)
    out = np.zeros(lay.NE)
    out[pe] = v_ref * se
    return out


def edge_from_dense(name, v):
    lay, pe, pf, pc, se, sf = ref_maps(name)
    return v[pe] * se


def face_from_dense(name, v):
    lay, pe, pf, pc, se, sf = ref_maps(name)
    return v[pf] * sf


def face_to_dense(name, v_ref):
    lay, pe, pf, pc, se, sf = ref_maps(name)
    out = np.zeros(lay.NF)
    out[pf] = v_ref * sf
    return out


def cell3_from_dense(name, v3):
    """(3, NC) dense -> (ncell_ref, 3)."""
    lay, pe, pf, pc, se, sf = ref_maps(name)
    return np.asarray(v3)[:, pc].T


def cell3_to_dense(name, v_ref):
    lay, pe, pf, pc, se, sf = ref_maps(name)
    out = np.zeros((3, lay.NC))
    out[:, pc] = np.asarray(v_ref).T
    return out


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def ref_mesh(name):
    return O.MeshDesc.from_npz(golden(name))
