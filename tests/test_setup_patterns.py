"""The table setup builds its cell-face operators from shared entry orders; they
must equal scipy's canonical COO -> CSR conversion bit for bit (no GPU)."""
import numpy as np
import scipy.sparse as sp

import parity_util as PU
from pyib_b200.operators import Operators


def test_pattern_csr_equals_scipy_conversion():
    rng = np.random.default_rng(3)
    nrows, ncols, n = 500, 700, 20000
    key = rng.choice(nrows * ncols, size=n, replace=False)       # unique (row, col) pairs
    rows, cols = key // ncols, key % ncols
    cache = {}
    pat = Operators._pattern(rows, cols, nrows)
    for _ in range(3):                                            # several matrices on one pattern
        vals = rng.standard_normal(n)
        vals[rng.random(n) < 0.1] = 0.0                           # explicit zeros are kept
        mine = Operators._csr(pat, vals, (nrows, ncols), cache)
        ref = sp.csr_matrix((vals, (rows, cols)), shape=(nrows, ncols))
        assert mine.indptr.dtype == ref.indptr.dtype and mine.indices.dtype == ref.indices.dtype
        np.testing.assert_array_equal(mine.indptr, ref.indptr)
        np.testing.assert_array_equal(mine.indices, ref.indices)
        np.testing.assert_array_equal(mine.data, ref.data)


def test_fixture_operators_equal_coo_assembly():
    """On the 3-level fixture: P, I, D and G0 equal their COO assemblies."""
    lay = PU.layout_for("n3_osc")
    ops = Operators(lay)
    fc = ops.faces
    f, lo, hi, mlo, mhi, dlo, dhi = (fc[k] for k in ("f", "lo", "hi", "mlo", "mhi", "dlo", "dhi"))
    rows, cols = fc["rows"], fc["cols"]
    NC, NF = lay.NC, lay.NF
    for d in range(3):
        vals = np.concatenate([ops.vol_ci[lo[mlo]] * dlo[:, d], -ops.vol_ci[hi[mhi]] * dhi[:, d]])
        for mine, ref in ((ops.P[d], sp.csr_matrix((vals, (rows, cols)), shape=(NC, NF))),
                          (ops.I[d], sp.csr_matrix((np.concatenate([dlo[:, d], -dhi[:, d]]), (cols, rows)),
                                                   shape=(NF, NC)))):
            np.testing.assert_array_equal(mine.indptr, ref.indptr)
            np.testing.assert_array_equal(mine.indices, ref.indices)
            np.testing.assert_array_equal(mine.data, ref.data)
    ones = np.concatenate([np.ones(mlo.sum()), -np.ones(mhi.sum())])
    for mine, ref in ((ops.D, sp.csr_matrix((ones, (rows, cols)), shape=(NC, NF))),
                      (ops.G0, sp.csr_matrix((-ones, (cols, rows)), shape=(NF, NC)))):
        np.testing.assert_array_equal(mine.indptr, ref.indptr)
        np.testing.assert_array_equal(mine.indices, ref.indices)
        np.testing.assert_array_equal(mine.data, ref.data)
