"""The single-pass fused float64 matvec (k_mvF) against the three-kernel matvec.

The fused kernel evaluates the same template rows term for term and keeps the
exact CSR rows at level interfaces, so its product must equal the three-kernel
product bit for bit (``pyib_matvec`` with alpd 3 against alpd 1), on the small
reference fixtures and on the D16 and D32 oscillating-sphere layouts (several
tiles per level, holes, level interfaces, closed cavity).  The CG that uses it
must give the same iteration count as the CG on the three-kernel matvec and an
iterate within the solve's tolerance of it: only the summation order of p.w
differs (measured 7e-12 relative on the cavity fixture).
"""
import ctypes as C
import os

import numpy as np
import pytest

import parity_util as PU
from pyib_b200 import _lib
from pyib_b200.cases import CASES
from pyib_b200.device import DeviceSolver

pytestmark = pytest.mark.gpu


def _mv(sv, x, dt, alpd):
    sv.set("WORK_E", x)
    sv.h.call("pyib_matvec", _lib.F["WORK_E"], _lib.F["WORK_E2"], C.c_double(dt), alpd)
    return sv.get("WORK_E2")


@pytest.mark.parametrize("name", PU.CASES)
def test_fused_matvec_bit_identical_on_fixtures(name):
    g = PU.golden(name)
    lay = PU.layout_for(name)
    sv = DeviceSolver(lay, rou=float(g["rou"]), visc=float(g["visc"]), cavity=bool(g["cavity"]))
    rng = np.random.default_rng(7)
    for _ in range(2):
        x = rng.standard_normal(lay.NE) * lay.edge_exists
        a = _mv(sv, x, float(g["dt"]), 1)
        b = _mv(sv, x, float(g["dt"]), 3)
        assert np.array_equal(a, b), float(np.max(np.abs(a - b)))
    sv.h.close()


@pytest.mark.parametrize("case", ["d16_oscillating_sphere", "d32_oscillating_sphere"])
def test_fused_matvec_bit_identical_full_size(case):
    cs = CASES[case]
    lay = cs.layout().build()
    sv = DeviceSolver(lay, rou=cs.density, visc=cs.viscosity, cavity=cs.cavity)
    rng = np.random.default_rng(16)
    x = rng.standard_normal(lay.NE) * lay.edge_exists
    a = _mv(sv, x, cs.time_step, 1)
    b = _mv(sv, x, cs.time_step, 3)
    assert np.array_equal(a, b), float(np.max(np.abs(a - b)))
    ms = (C.c_double * 6)()
    sv.set("WORK_E", x)
    sv.h.call("pyib_bench_matvec_fused", 5, C.c_double(cs.time_step), ms)
    print(case, "fused matvec ms", list(ms))
    sv.h.close()


def test_fused_cg_matches_three_kernel_cg():
    """Same solve with PYIB_FUSED_MATVEC=1 and =0: same iterations, iterates within 1e-10."""
    name = "n3_osc"
    g = PU.golden(name)
    lay = PU.layout_for(name)
    out = {}
    for mode in ("1", "0"):
        old = os.environ.get("PYIB_FUSED_MATVEC")
        os.environ["PYIB_FUSED_MATVEC"] = mode
        try:
            sv = DeviceSolver(lay, rou=float(g["rou"]), visc=float(g["visc"]), cavity=True)
        finally:
            if old is None:
                os.environ.pop("PYIB_FUSED_MATVEC")
            else:
                os.environ["PYIB_FUSED_MATVEC"] = old
        sv.set("RES_E", PU.edge_to_dense(name, g["hs_res"]))
        sv.set("S", PU.edge_to_dense(name, g["hs_s"]))
        st = _lib.SolveStats()
        sv.h.call("pyib_helm_solve", C.c_double(float(g["dt"])), C.byref(st))
        out[mode] = (int(st.iterations), sv.get("S"))
        sv.h.close()
    assert out["1"][0] == out["0"][0] == int(g["hs_iters"])
    a, b = out["1"][1], out["0"][1]
    assert np.linalg.norm(a - b) <= 1e-10 * np.linalg.norm(b)
