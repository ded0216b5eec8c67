"""Host-side assembly of the GPU tables and a thin object over one library context.

``DeviceSolver`` builds, once per layout, everything the kernels read:

* the structured-matvec patch rows (``templates.MatvecPlan``),
* CSR gathers for the step operators (curl, rot, interp_f2c, integr_c2f),
* per-cell signed face lists, face-cell links with ghost slots, AoL, 1/volume,
* boundary (ghost) face records, inlet edges, the preconditioner,
* the closed-sphere load-correction cell lists,

then uploads them through ``pyib_upload`` and keeps the state on the device.
Fields cross the C ABI in the dense layout; ``B200Driver`` converts to the
reference numbering where a caller needs it.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import scipy.sparse as sp

from . import _lib
from .layout import NestedLayout
from .operators import Operators
from .templates import MatvecPlan


def _csr_arrays(M):
    M = M.tocsr()
    M.sort_indices()
    return (M.indptr.astype(np.int64), M.indices.astype(np.int32), M.data.astype(np.float64))


def _bits(mask):
    n = mask.size
    words = np.zeros((n + 31) // 32, dtype=np.uint32)
    idx = np.nonzero(mask)[0]
    np.bitwise_or.at(words, idx >> 5, (np.uint32(1) << (idx & 31).astype(np.uint32)))
    return words


def _rowmap(n, rows):
    m = np.full(n, -1, dtype=np.int32)
    m[rows] = np.arange(rows.size, dtype=np.int32)
    return m


def _triplets_sorted(pattern, vals3):
    """CSR arrays of (row, col, 3 values) entries in row-then-column order, from an
    entry pattern of ``Operators._pattern``."""
    order, indptr, indices = pattern
    return indptr.copy(), indices.astype(np.int32), np.ascontiguousarray(vals3[order], dtype=np.float64)


class LayoutTables:
    """Host-side tables of one layout and boundary kind, built once and shared.

    Everything a context uploads that depends only on the geometry (operators,
    boundary masks, preconditioner, structured-matvec patches): several contexts
    on the same nested layout -- the cases of a batched sweep with equal
    resolution -- reuse one instance instead of rebuilding it per case.
    """

    def __init__(self, lay: NestedLayout, cavity):
        if not getattr(lay, "_built", False):
            lay.build()
        self.lay = lay
        self.cavity = bool(cavity)
        self.ops = ops = Operators(lay)
        self.dir_mask = ops.dir_mask(self.cavity)
        self.inlet = ops.inlet_mask(self.cavity) & lay.edge_exists
        self.prec = ops.prec(self.dir_mask)
        self.plan = MatvecPlan(ops, self.dir_mask)
        self.bfaces = lay.boundary_faces()
        self.arrays = {}
        self._build()

    def _build(self):
        lay, ops, A = self.lay, self.ops, self.arrays
        NC, NF, NE = lay.NC, lay.NF, lay.NE
        A["PREC"] = self.prec
        # per level, the value of the regular edges; edges that differ are flagged
        reg = np.zeros(lay.N)
        irregular = np.zeros(NE, dtype=bool)
        for lv in lay.levels:
            lo_e = lay.edge_base[lv.L][0]
            hi_e = lay.edge_base[lv.L][2] + int(np.prod(lv.edge_dims(2)))
            vals, counts = np.unique(self.prec[lo_e:hi_e], return_counts=True)
            nz = vals != 0.0
            reg[lv.L] = vals[nz][np.argmax(counts[nz])] if nz.any() else 0.0
            irregular[lo_e:hi_e] = self.prec[lo_e:hi_e] != reg[lv.L]
        A["PREC_BITS"] = _bits(irregular)
        A["PREC_REG"] = reg
        self.prec_regular = reg
        ie = np.nonzero(self.inlet)[0]
        hz = np.where(lay.edge_axis[ie] == 2, lay.edge_h[ie], 0.0)
        A["INLET_IDX"] = ie.astype(np.int32)
        A["INLET_VAL"] = lay.epos[ie, 1] * hz
        for name, M in (("CURL", ops.C), ("ROT", ops.R)):
            A[name + "_PTR"], A[name + "_COL"], A[name + "_VAL"] = _csr_arrays(M)
        fc = ops.faces
        f, lo, hi, mlo, mhi, dlo, dhi = (fc[k] for k in ("f", "lo", "hi", "mlo", "mhi", "dlo", "dhi"))
        vol_ci = ops.vol_ci
        # interp_f2c: rows cells, cols faces, 3 values (the operators' cell x face order)
        v3 = np.concatenate([vol_ci[lo[mlo], None] * dlo, -vol_ci[hi[mhi], None] * dhi])
        A["P_PTR"], A["P_COL"], A["P_VAL3"] = _triplets_sorted(ops.cf, v3)
        # integr_c2f: rows faces, cols cells
        A["I_PTR"], A["I_COL"], A["I_VAL3"] = _triplets_sorted(ops.fc, np.concatenate([dlo, -dhi]))
        # cell -> signed faces (bit 0 set: the face's +a side is this cell), by cell and
        # then face: the cell x face order, since 2 face + side grows with the face
        code = np.concatenate([(f[mlo] << 1), (f[mhi] << 1) | 1]).astype(np.int64)
        order, indptr, _ = ops.cf
        A["CF_PTR"] = indptr.copy()
        A["CF_FACE"] = code[order].astype(np.int32)
        # face cells with ghost slots
        bf = self.bfaces
        gslot = np.full(NF, -1, dtype=np.int64)
        gslot[bf] = NC + np.arange(bf.size)
        flo = np.where(lay.face_lo >= 0, lay.face_lo, np.where(gslot >= 0, gslot, 0))
        fhi = np.where(lay.face_hi >= 0, lay.face_hi, np.where(gslot >= 0, gslot, 0))
        A["F_LO"] = flo.astype(np.int32)
        A["F_HI"] = fhi.astype(np.int32)
        A["F_AOL"] = ops.AoL
        A["VOLCI"] = vol_ci
        inner = np.where(lay.face_lo[bf] >= 0, lay.face_lo[bf], lay.face_hi[bf])
        info = lay.face_axis[bf].astype(np.int32)
        if self.cavity:
            info |= 8
        else:
            info |= np.where(lay.face_bc[bf] == 1, 4, 0).astype(np.int32)
        A["BF_FACE"] = bf.astype(np.int32)
        A["BF_CELL"] = inner.astype(np.int32)
        A["BF_INFO"] = info
        A["BF_AF"] = lay.face_Af[bf]
        # structured-matvec patches
        plan = self.plan
        for tag, (rows_p, M), n in (("PA", plan.patchA, NC), ("PV", plan.patchV, NC),
                                    ("PR", plan.patchRI, NE)):
            mask = np.zeros(n, dtype=bool)
            mask[rows_p] = True
            A[tag + "_BITS"] = _bits(mask)
            A[tag + "_IDS"] = np.asarray(rows_p, dtype=np.int32)
            A[tag + "_ROW"] = _rowmap(n, rows_p)
            A[tag + "_PTR"], A[tag + "_COL"], A[tag + "_VAL"] = _csr_arrays(M)
        self.patch_counts = (plan.patchA[0].size, plan.patchV[0].size, plan.patchRI[0].size,
                             int(plan.upper_exact))


class DeviceSolver:
    """One GPU context holding a nested layout, its operators and the solver state."""

    def __init__(self, lay: NestedLayout, *, rou, visc, cavity, cg_check_interval=20,
                 cg_max_iterations=1000, strict=False, ac=0.5, ad=0.5, tol1=1e-10, tol2=1e-9,
                 device=0, precision="float64", mixed_tol=0.1, mixed_max_sweeps=200, tables=None,
                 ib_mode=0, ib_alpha=1.0):
        if tables is None:
            tables = LayoutTables(lay, cavity)
        elif tables.lay is not lay or tables.cavity != bool(cavity):
            raise ValueError("tables were built for another layout or boundary kind")
        lay = tables.lay
        self.lay = lay
        self.tables = tables
        self.ops = ops = tables.ops
        self.cavity = tables.cavity
        self.dir_mask = tables.dir_mask
        self.inlet = tables.inlet
        self.prec = tables.prec
        self.plan = tables.plan
        self.bfaces = tables.bfaces
        self.prec_regular = tables.prec_regular
        NC, NF, NE = lay.NC, lay.NF, lay.NE
        L = _lib.Layout()
        L.nlevels = lay.N
        for lv in lay.levels:
            for a in range(3):
                L.n[lv.L][a] = int(lv.n[a])
                L.lo[lv.L][a] = float(lv.lo[a])
                if lv.hole_lo is not None:
                    L.hole_lo[lv.L][a] = int(lv.hole_lo[a])
                    L.hole_n[lv.L][a] = int(lv.hole_n[a])
            L.h[lv.L] = lv.h
        L.ncell, L.nface, L.nedge = NC, NF, NE
        L.nbface = int(self.bfaces.size)
        L.device = int(device)
        self.h = _lib.Handle(L)
        self._upload_tables()
        self.params = dict(rou=float(rou), visc=float(visc), ac=ac, ad=ad, tol1=tol1, tol2=tol2,
                           cavity=int(self.cavity), check=int(cg_check_interval),
                           cg_max=int(cg_max_iterations), strict=int(bool(strict)),
                           precision={"float64": 0, "mixed": 1}[precision],
                           nmarkers=0, hh=lay.h0, hh3=lay.h0 ** 3, mixed_tol=float(mixed_tol),
                           mixed_max_sweeps=int(mixed_max_sweeps), ib_mode=int(ib_mode),
                           ib_alpha=float(ib_alpha))
        self._push_params()
        pos_ref = (lay.levels[0].lo + 0.5 * lay.h0).astype(np.float64)
        self.pos_ref = pos_ref
        self.h.call("pyib_set_ib_geometry", pos_ref.ctypes.data_as(C.POINTER(C.c_double)),
                    C.c_double(lay.h0))
        self.M = 0

    # ---- tables --------------------------------------------------------------
    def _upload_tables(self):
        h = self.h
        for name, arr in self.tables.arrays.items():
            h.upload(name, arr)
        counts = (C.c_int64 * 4)(*self.tables.patch_counts)
        h.call("pyib_finalize", counts, 4)
        h.upload("LC_CPOS", np.ascontiguousarray(self.lay.cpos))

    def _push_params(self):
        P = _lib.Params(**self.params)
        self.h.call("pyib_set_params", C.byref(P))

    # ---- immersed boundary ----------------------------------------------------
    def set_markers(self, markers, vel, ds):
        markers = np.asarray(markers, dtype=np.float64).reshape(-1, 3)
        M = markers.shape[0]
        if M != self.M:
            self.params["nmarkers"] = M
            self._push_params()
            self.M = M
        self.h.set_field("MARKERS", markers)
        self.h.set_field("MVEL", np.asarray(vel, dtype=np.float64).reshape(-1, 3))
        ds = np.asarray(ds, dtype=np.float64).reshape(-1)
        self.h.set_field("DS", ds ** 3)

    def set_load_lists(self, cand, fidx):
        self.h.upload("LC_CAND", np.asarray(cand, dtype=np.int32))
        self.h.upload("LC_FIDX", np.asarray(fidx, dtype=np.int32))

    # ---- field access (dense layout) -------------------------------------------
    def get(self, name):
        lay = self.lay
        n = {"S": lay.NE, "S_OLD": lay.NE, "RES_E": lay.NE, "WORK_E": lay.NE, "WORK_E2": lay.NE,
             "U": lay.NF, "WORK_F": lay.NF, "RES_C": 3 * lay.NC, "FE": 3 * lay.NC,
             "WORK_C3": 3 * lay.NC, "VC": 3 * (lay.NC + self.bfaces.size),
             "FL": 3 * self.M, "MARKERS": 3 * self.M, "MVEL": 3 * self.M, "DS": self.M,
             "LAG_TMP": 3 * self.M}
        if name in ("IB_CELL",):
            return self.h.get_field(name, 125 * self.M, np.int32)
        if name == "IB_W":
            return self.h.get_field(name, 125 * self.M)
        if name == "IB_BASE":
            return self.h.get_field(name, 3 * self.M, np.int32)
        return self.h.get_field(name, n[name])

    def set(self, name, arr):
        self.h.set_field(name, arr)

    def get_dinv(self):
        """The mixed solver's float32 Jacobi preconditioner 1/diag(A) (0 on masked edges)."""
        return self.h.get_field("DINV", self.lay.NE, np.float32).astype(np.float64)

    def vc_cells(self):
        """Cell velocity (3, NC) without ghosts."""
        v = self.get("VC").reshape(3, -1)
        return v[:, :self.lay.NC]
