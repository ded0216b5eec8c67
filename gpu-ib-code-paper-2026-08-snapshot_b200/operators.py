"""Exact incidence operators of the nested layout as sparse matrices (host, built once).

All matrices use the dense ids of :mod:`layout` and the +a orientation of
faces and edges.  They restate, row for row, the reference's operators
(``ib_core_np.py:129-183``) in that orientation:

* ``C``    curl, edges -> faces          (``IBCore.curl``, ib_core_np.py:133)
* ``R``    rot = C^T, faces -> edges     (``IBCore.rot``, ib_core_np.py:129)
* ``P[d]`` interp_f2c component d        (ib_core_np.py:150-157)
* ``I[d]`` integr_c2f component d        (ib_core_np.py:144-148)
* ``D``    cdiv, faces -> cells          (ib_core_np.py:136-139)
* ``G0``   cgrad with zero ghost         (ib_core_np.py:177-183)
* ``Vd``   vol * D * diag(AoL) * G0, the viscous block of ``flow_mat``
  (ib_core_np.py:168-175) without the ``-0.5*dt*visc`` factor

These are the ground truth the GPU templates are checked against; rows the
structured templates cannot reproduce become explicit patch rows.
"""
from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor

import numpy as np
import scipy.sparse as sp


class Operators:
    def __init__(self, lay):
        if not getattr(lay, "_built", False):
            lay.build()
        self.lay = lay
        NC, NF, NE = lay.NC, lay.NF, lay.NE

        def curl():
            C = sp.csr_matrix((lay.link_sign, (lay.link_face, lay.link_edge)), shape=(NF, NE))
            C.sum_duplicates()
            return C, C.T.tocsr()

        # the curl pair and the face geometry are independent of the cell-face
        # matrices below: they are built on host threads meanwhile (the array and
        # sparse kernels release the interpreter lock; the values do not change)
        with ThreadPoolExecutor(max_workers=2) as pool:
            f_curl = pool.submit(curl)
            f_aol = pool.submit(lay.face_AoL)
            self._cell_face(lay, NC, NF)
            self.C, self.R = f_curl.result()
            self.AoL = f_aol.result()
        # vol * D * diag(AoL) is a row and column scaling of D's entries, in the order
        # the two diagonal products take (the same bits); then one sparse product
        D = self.D
        drow = np.repeat(np.arange(D.shape[0]), np.diff(D.indptr))
        Dw = sp.csr_matrix(((self.vol_ci[drow] * D.data) * self.AoL[D.indices], D.indices, D.indptr),
                           shape=D.shape)
        self.Vd = (Dw @ self.G0).tocsr()

    def _cell_face(self, lay, NC, NF):
        """P, I, D, G0 and the face data and entry orders they share."""
        f = np.nonzero(lay.face_exists)[0]
        lo, hi = lay.face_lo[f], lay.face_hi[f]
        mlo, mhi = lo >= 0, hi >= 0
        vol_ci = np.zeros(NC)
        vol_ci[lay.cell_active] = 1.0 / lay.cell_vol[lay.cell_active]
        self.vol_ci = vol_ci
        dlo = lay.fpos[f[mlo]] - lay.cpos[lo[mlo]]
        dhi = lay.fpos[f[mhi]] - lay.cpos[hi[mhi]]
        # cell-face incidence entries (the -a side cells first), and the two orders
        # that list them as rows of cells x faces and of faces x cells
        rows = np.concatenate([lo[mlo], hi[mhi]])
        cols = np.concatenate([f[mlo], f[mhi]])
        with ThreadPoolExecutor(max_workers=2) as pool:      # two independent sorts
            f_cf = pool.submit(self._pattern, rows, cols, NC)
            f_fc = pool.submit(self._pattern, cols, rows, NF)
            self.cf, self.fc = f_cf.result(), f_fc.result()
        self.faces = dict(f=f, lo=lo, hi=hi, mlo=mlo, mhi=mhi, dlo=dlo, dhi=dhi, rows=rows, cols=cols)
        self.P, self.I = [], []
        ccf, cfc = {}, {}
        for d in range(3):
            vals = np.concatenate([vol_ci[lo[mlo]] * dlo[:, d], -vol_ci[hi[mhi]] * dhi[:, d]])
            self.P.append(self._csr(self.cf, vals, (NC, NF), ccf))
            self.I.append(self._csr(self.fc, np.concatenate([dlo[:, d], -dhi[:, d]]), (NF, NC), cfc))
        self.D = self._csr(self.cf, np.concatenate([np.ones(mlo.sum()), -np.ones(mhi.sum())]), (NC, NF), ccf)
        self.G0 = self._csr(self.fc, np.concatenate([-np.ones(mlo.sum()), np.ones(mhi.sum())]), (NF, NC), cfc)

    @staticmethod
    def _pattern(rows, cols, nrows):
        """(order, indptr, indices) listing the entries (rows, cols) by row and then
        column: the canonical CSR of scipy's COO conversion, for entries without
        duplicate (row, column) pairs, computed once per pattern."""
        key = (rows.astype(np.int64) << 32) | cols.astype(np.int64)
        order = np.argsort(key, kind="stable")
        indptr = np.zeros(nrows + 1, dtype=np.int64)
        np.cumsum(np.bincount(rows, minlength=nrows), out=indptr[1:])
        return order, indptr, cols[order]

    @staticmethod
    def _csr(pattern, vals, shape, cache):
        """CSR of ``vals`` on a pattern.  The index arrays, in the index type scipy
        picks for the size, are converted once (``cache``, one per pattern) and
        shared by the pattern's matrices."""
        order, indptr, indices = pattern
        idx_t = np.int32 if max(shape) < 2**31 and indices.size < 2**31 else np.int64
        if idx_t not in cache:
            cache[idx_t] = (indices.astype(idx_t), indptr.astype(idx_t))
        ind, ptr = cache[idx_t]
        return sp.csr_matrix((vals[order], ind, ptr), shape=shape)

    # ---- boundary conditions (ib_driver_np.py:120-121, 155-166) -----------
    def dir_mask(self, cavity):
        lay = self.lay
        if cavity:
            m = lay.edge_bc > 0
        else:
            m = np.isin(lay.edge_bc, (3, 4, 5, 6))
        return m

    def inlet_mask(self, cavity):
        if cavity:
            return np.zeros(self.lay.NE, dtype=bool)
        return self.lay.edge_bc == 1

    def prec(self, dir_mask):
        """Geometric diagonal preconditioner, ib_driver_np.py:78-88 (0 on Dirichlet/absent edges)."""
        lay = self.lay
        rf = lay.face_rf()
        ax = lay.face_axis.astype(np.int64)
        q = np.zeros(lay.NF)
        ok = lay.face_exists
        q[ok] = rf[ok, ax[ok]] / lay.face_Af[ok]            # (rf.nf)/Af^2 with nf = Af e_a
        d = np.bincount(lay.link_edge, weights=q[lay.link_face], minlength=lay.NE)
        d[dir_mask | ~lay.edge_exists] = 0.0
        out = np.zeros(lay.NE)
        nz = d != 0.0
        out[nz] = 1.0 / d[nz]
        return out

    # ---- composite operators ---------------------------------------------
    def V(self, rou, visc, dt):
        return (rou * sp.identity(self.lay.NC, format="csr") - (0.5 * dt * visc) * self.Vd).tocsr()

    def flow_mat(self, p, alpd=0.0, visc=0.0, rou=1.0, dt=0.0):
        U = self.C @ p
        v = [self.P[d] @ U for d in range(3)]
        if alpd != 0.0:
            v = [rou * vd - (0.5 * dt * visc) * (self.Vd @ vd) for vd in v]
        return self.R @ sum(self.I[d] @ v[d] for d in range(3))
