"""pyib_spread_noalloc: deterministic spreading for callers that cannot allocate.

Some callers cannot call cudaMalloc -- a code that runs inside a device-memory
budget fixed at start-up, or one whose framework allocator owns all device
memory.  The entry point keeps its scratch in a fixed device array inside the
library, so the caller only provides inputs and the output.  This test calls it
twice in a row through the C ABI and checks each result against the existing
entry point pyib_ib_spread on the same stencil and forces.  It lives in its own
file so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import parity_util as PU
from pyib_b200 import _lib
from pyib_b200.device import DeviceSolver

pytestmark = pytest.mark.gpu


def test_spread_noalloc_matches_spread_twice():
    torch = pytest.importorskip("torch")
    name = "n3_osc"
    g = PU.golden(name)
    lay = PU.layout_for(name)
    sv = DeviceSolver(lay, rou=float(g["rou"]), visc=float(g["visc"]), cavity=True)
    sv.set_markers(g["ib_markers"], g["ib_vel"], g["ib_ds"])
    sv.h.call("pyib_ib_stencil")
    cell = sv.get("IB_CELL")
    w = sv.get("IB_W")
    ds3 = sv.get("DS")
    M = g["ib_markers"].shape[0]
    dev = torch.device("cuda", 0)
    t_cell = torch.from_numpy(cell).to(dev)
    t_w = torch.from_numpy(w).to(dev)
    t_ds3 = torch.from_numpy(ds3).to(dev)
    t_out = torch.full((3 * lay.NC,), float("nan"), dtype=torch.float64, device=dev)
    lib = _lib.load()
    for scale in (1.0, -2.5):
        f = g["ib_fl"] * scale
        sv.set("FL", f)
        sv.h.call("pyib_ib_spread")
        expected = sv.get("FE")
        t_f = torch.from_numpy(np.ascontiguousarray(f).reshape(-1)).to(dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = lib.pyib_spread_noalloc(C.c_void_p(t_cell.data_ptr()), C.c_void_p(t_w.data_ptr()),
                                     C.c_void_p(t_ds3.data_ptr()), C.c_void_p(t_f.data_ptr()),
                                     int(M), int(lay.NC), C.c_void_p(t_out.data_ptr()),
                                     C.c_void_p(stream))
        torch.cuda.synchronize(dev)
        assert rc == _lib.OK
        got = t_out.cpu().numpy()
        # same sort, same summation order: identical to the existing entry point
        assert np.array_equal(got, expected)


def test_spread_noalloc_rejects_too_many_markers():
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    x = torch.zeros(16, dtype=torch.float64, device=dev)
    p = C.c_void_p(x.data_ptr())
    assert lib.pyib_spread_noalloc(p, p, p, p, 8193, 10, p, None) == _lib.E_ARG


def test_spread_noalloc_rejects_bad_cell_ids():
    """Ids outside [0, ncell) are skipped and reported; nothing lands outside out."""
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(5)
    M, ncell, guard = 4, 300, 64
    cell = rng.integers(0, ncell, size=M * 125).astype(np.int32)
    cell[7] = ncell            # one past the end
    cell[130] = ncell + 1000   # far past the end
    cell[260] = -3             # negative
    w = rng.random(M * 125)
    ds3 = rng.random(M) + 0.5
    f = rng.standard_normal(3 * M)
    ok = (cell >= 0) & (cell < ncell)
    m = np.arange(M * 125) // 125
    expected = np.zeros(3 * ncell)
    for d in range(3):
        contrib = f[3 * m + d] * (w * ds3[m])
        expected[d * ncell:(d + 1) * ncell] = np.bincount(cell[ok], weights=contrib[ok], minlength=ncell)
    buf = torch.full((3 * ncell + guard,), float("nan"), dtype=torch.float64, device=dev)
    t_cell = torch.from_numpy(cell).to(dev)
    t_w = torch.from_numpy(w).to(dev)
    t_ds3 = torch.from_numpy(ds3).to(dev)
    t_f = torch.from_numpy(f).to(dev)
    for _ in range(2):
        rc = lib.pyib_spread_noalloc(C.c_void_p(t_cell.data_ptr()), C.c_void_p(t_w.data_ptr()),
                                     C.c_void_p(t_ds3.data_ptr()), C.c_void_p(t_f.data_ptr()),
                                     int(M), int(ncell), C.c_void_p(buf.data_ptr()), None)
        torch.cuda.synchronize(dev)
        assert rc == _lib.E_DEVICE
        got = buf.cpu().numpy()
        assert np.all(np.isnan(got[3 * ncell:]))          # guard after out untouched
        np.testing.assert_allclose(got[:3 * ncell], expected, rtol=1e-13, atol=1e-15)
    # a clean call afterwards succeeds: the reject counter starts at zero every call
    t_cell.clamp_(0, ncell - 1)
    rc = lib.pyib_spread_noalloc(C.c_void_p(t_cell.data_ptr()), C.c_void_p(t_w.data_ptr()),
                                 C.c_void_p(t_ds3.data_ptr()), C.c_void_p(t_f.data_ptr()),
                                 int(M), int(ncell), C.c_void_p(buf.data_ptr()), None)
    torch.cuda.synchronize(dev)
    assert rc == _lib.OK
