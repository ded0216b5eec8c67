"""The fused curl+interp / viscous kernel (k_mvAV) against the two-kernel form.

k_mvAV evaluates the template rows of kernels A and V term for term and keeps
the exact CSR rows at level interfaces, so ``pyib_matvec`` with alpd 5 (fused)
must equal alpd 9 (two kernels) bit for bit on the reference fixtures and on the
D16 and D32 oscillating-sphere layouts (several tiles per level, holes, level
interfaces, closed cavity).  The rest of the CG is untouched, so a solve with
the fused form pinned (PYIB_MATVEC_AV=1) must reproduce the solve with the two
kernels pinned (PYIB_MATVEC_AV=0) bit for bit, in float64 and in the mixed
solver's float32 iterations alike.
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
def test_av_matvec_bit_identical_on_fixtures(name):
    g = PU.golden(name)
    lay = PU.layout_for(name)
    sv = DeviceSolver(lay, rou=float(g["rou"]), visc=float(g["visc"]), cavity=bool(g["cavity"]))
    rng = np.random.default_rng(11)
    for _ in range(2):
        x = rng.standard_normal(lay.NE) * lay.edge_exists
        a = _mv(sv, x, float(g["dt"]), 9)
        b = _mv(sv, x, float(g["dt"]), 5)
        c = _mv(sv, x, float(g["dt"]), 1)
        assert np.array_equal(a, b), float(np.max(np.abs(a - b)))
        assert np.array_equal(a, c)
    sv.h.close()


@pytest.mark.parametrize("case", ["d16_oscillating_sphere", "d32_oscillating_sphere"])
def test_av_matvec_bit_identical_full_size(case):
    cs = CASES[case]
    lay = cs.layout().build()
    sv = DeviceSolver(lay, rou=cs.density, visc=cs.viscosity, cavity=cs.cavity)
    rng = np.random.default_rng(17)
    x = rng.standard_normal(lay.NE) * lay.edge_exists
    a = _mv(sv, x, cs.time_step, 9)
    b = _mv(sv, x, cs.time_step, 5)
    assert np.array_equal(a, b), float(np.max(np.abs(a - b)))
    # twice in a row: the fused kernel keeps no state between calls
    b2 = _mv(sv, x, cs.time_step, 5)
    assert np.array_equal(a, b2)
    sv.h.close()


def _solve(name, pin, precision):
    g = PU.golden(name)
    lay = PU.layout_for(name)
    old = os.environ.get("PYIB_MATVEC_AV")
    os.environ["PYIB_MATVEC_AV"] = pin
    try:
        sv = DeviceSolver(lay, rou=float(g["rou"]), visc=float(g["visc"]), cavity=True, precision=precision)
    finally:
        if old is None:
            os.environ.pop("PYIB_MATVEC_AV")
        else:
            os.environ["PYIB_MATVEC_AV"] = old
    sv.set("RES_E", PU.edge_to_dense(name, g["hs_res"]))
    sv.set("S", PU.edge_to_dense(name, g["hs_s"]))
    st = _lib.SolveStats()
    sv.h.call("pyib_helm_solve", C.c_double(float(g["dt"])), C.byref(st))
    plan = (C.c_int32 * 8)()
    sv.h.call("pyib_matvec_plan", plan)
    out = (int(st.iterations), sv.get("S"), list(plan))
    sv.h.close()
    return out


@pytest.mark.parametrize("precision", ["float64", "mixed"])
def test_av_cg_bit_identical_to_two_kernel_cg(precision):
    name = "n3_osc"
    fused = _solve(name, "1", precision)
    apart = _solve(name, "0", precision)
    q = 0 if precision == "float64" else 4
    assert fused[2][q] == 1 and fused[2][q + 3] == 1
    assert apart[2][q] == 1 and apart[2][q + 3] == 0
    assert fused[0] == apart[0]
    if precision == "float64":
        assert fused[0] == int(PU.golden(name)["hs_iters"])
    assert np.array_equal(fused[1], apart[1])
