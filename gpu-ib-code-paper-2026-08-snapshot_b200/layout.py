"""Structured nested-level layout for the B200 path (host-side, built once).

The reference keeps every nested level in ONE unstructured incidence graph
(``make_euler_mesh.py:330-463`` builds it, ``make_euler_mesh.py:787-950``
stitches the 2:1 interfaces).  On the B200 every level ``L`` (spacing
``h*2^L``) is instead a dense box of cells, and faces/edges of each axis are
dense boxes too, stored x-fastest in HBM::

    cells   (nx,   ny,   nz)            per level
    faces a (n + e_a)                   per level and normal axis a
    edges a (n + 1 - e_a)               per level and tangent axis a

Slots that the reference mesh does not contain (cells in the hole of an
outer level, the aliased coarse faces and collapsed coarse edges on a hole
surface) stay in the arrays and hold zero.  Every face is oriented along
+a and every edge along +a, so structured kernels need no per-entity signs.

Interface rules, restated from the reference's finalisation
(``make_euler_mesh.py:761-950``):

* a coarse face on a hole surface is removed; the 4 fine faces behind it get
  the coarse cell as their second cell;
* a coarse edge lying in a hole surface is removed; a remaining coarse face
  that used it gets its two fine sub-edges instead (the second one is an
  "extra link", ``link_fe_insert``).

Geometry is the true geometry of the boxes: the reference's hanging-node
corrections (``ib_core_np.py:74-102``) move the shifted face and cell centres
back to the geometric centres for a 2:1 ratio, which the oracle tests check.

The module also exports the layout as an unstructured mesh description in the
reference's conventions (cell order of faces, edge orientation by node rank),
so the oracle can run on exactly the same mesh.
"""
from __future__ import annotations

from dataclasses import dataclass

from concurrent.futures import ThreadPoolExecutor

import numpy as np

OUT, ACTIVE, HOLE = 0, 1, 2
_E = np.eye(3, dtype=np.int64)


class LayoutError(ValueError):
    """Invalid nested box list (mirrors the reference's builder rejections)."""


@dataclass
class Level:
    L: int
    h: float
    lo: np.ndarray          # (3,) float, box lower corner
    n: np.ndarray           # (3,) int, cells per axis
    hole_lo: np.ndarray     # (3,) int, first hole cell (level L>0), else None
    hole_n: np.ndarray      # (3,) int, hole cells per axis

    def face_dims(self, a):
        return self.n + _E[a]

    def edge_dims(self, a):
        return self.n + 1 - _E[a]


def _flat(dims, ijk):
    return (ijk[..., 2] * dims[1] + ijk[..., 1]) * dims[0] + ijk[..., 0]


def _unflat(dims, flat):
    i = flat % dims[0]
    j = (flat // dims[0]) % dims[1]
    k = flat // (dims[0] * dims[1])
    return np.stack([i, j, k], axis=-1)


def _grid(dims):
    """All integer index triples of a box, x fastest, as an (N,3) int64 array."""
    k, j, i = np.meshgrid(np.arange(dims[2]), np.arange(dims[1]), np.arange(dims[0]), indexing="ij")
    return np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.int64)


class NestedLayout:
    """Nested 2:1 Cartesian boxes, innermost first.

    ``boxes`` is a list of ``(lo, hi)`` corner pairs; level ``L`` has spacing
    ``h * 2**L``.  Rules (as ``make_euler_mesh.py:236-290``): every box side
    is a multiple of its spacing, every inner box corner lies on the next
    outer grid.  This build also requires an even cell count per axis for
    inner boxes and at least one outer cell around every hole.
    """

    def __init__(self, h, boxes):
        h = float(h)
        if not (h > 0 and np.isfinite(h)):
            raise LayoutError("spacing must be positive")
        if len(boxes) < 1:
            raise LayoutError("at least one box is required")
        self.h0 = h
        self.levels: list[Level] = []
        for L, (lo, hi) in enumerate(boxes):
            lo = np.asarray(lo, dtype=np.float64)
            hi = np.asarray(hi, dtype=np.float64)
            hL = h * 2 ** L
            size = (hi - lo) / hL
            n = np.rint(size).astype(np.int64)
            if np.any(hi <= lo) or not np.allclose(size, n, rtol=0, atol=1e-8) or np.any(n < 1):
                raise LayoutError(f"level {L}: box size is not a positive multiple of {hL}")
            self.levels.append(Level(L, hL, lo, n, None, None))
        for L in range(1, len(self.levels)):
            inner, outer = self.levels[L - 1], self.levels[L]
            off = (inner.lo - outer.lo) / outer.h
            offi = np.rint(off).astype(np.int64)
            if not np.allclose(off, offi, rtol=0, atol=1e-8):
                raise LayoutError(f"level {L-1} corner is not on the level {L} grid")
            if np.any(inner.n % 2):
                raise LayoutError(f"level {L-1} needs an even cell count per axis")
            hn = inner.n // 2
            if np.any(offi < 1) or np.any(offi + hn > outer.n - 1):
                raise LayoutError(f"level {L-1} must lie strictly inside level {L}")
            outer.hole_lo, outer.hole_n = offi, hn
        self.N = len(self.levels)
        self._bases()

    # ---- dense numbering ---------------------------------------------------
    def _bases(self):
        cb, fb, eb = [], [], []
        nc = nf = ne = 0
        for lv in self.levels:
            cb.append(nc)
            nc += int(np.prod(lv.n))
            fb.append([])
            for a in range(3):
                fb[-1].append(nf)
                nf += int(np.prod(lv.face_dims(a)))
        for lv in self.levels:
            eb.append([])
            for a in range(3):
                eb[-1].append(ne)
                ne += int(np.prod(lv.edge_dims(a)))
        self.cell_base, self.face_base, self.edge_base = cb, fb, eb
        self.NC, self.NF, self.NE = nc, nf, ne

    def cell_id(self, L, ijk):
        return self.cell_base[L] + _flat(self.levels[L].n, ijk)

    def face_id(self, L, a, ijk):
        return self.face_base[L][a] + _flat(self.levels[L].face_dims(a), ijk)

    def edge_id(self, L, a, ijk):
        return self.edge_base[L][a] + _flat(self.levels[L].edge_dims(a), ijk)

    def cell_state(self, L, ijk):
        """OUT / ACTIVE / HOLE for level-L cell index triples (any shape (...,3))."""
        lv = self.levels[L]
        inb = np.all((ijk >= 0) & (ijk < lv.n), axis=-1)
        st = np.where(inb, ACTIVE, OUT)
        if lv.hole_lo is not None:
            inh = np.all((ijk >= lv.hole_lo) & (ijk < lv.hole_lo + lv.hole_n), axis=-1)
            st = np.where(inh, HOLE, st)
        return st

    # ---- per-entity tables (lazy) -----------------------------------------
    def _state3(self, L, dims, off):
        """cell_state of the level-L cells (i, j, k) - off for every index triple of a
        box of ``dims``, as a (dims[2], dims[1], dims[0]) array (x fastest when
        flattened): in-box and in-hole tests factor per axis."""
        lv = self.levels[L]
        idx = [np.arange(dims[t]) - off[t] for t in range(3)]
        inb = [(idx[t] >= 0) & (idx[t] < lv.n[t]) for t in range(3)]
        st = np.where(inb[2][:, None, None] & inb[1][None, :, None] & inb[0][None, None, :], ACTIVE, OUT)
        if lv.hole_lo is not None:
            inh = [(idx[t] >= lv.hole_lo[t]) & (idx[t] < lv.hole_lo[t] + lv.hole_n[t]) for t in range(3)]
            st = np.where(inh[2][:, None, None] & inh[1][None, :, None] & inh[0][None, None, :], HOLE, st)
        return st

    @staticmethod
    def _flat3(dims, base, off, step):
        """base + flat(step, (i, j, k) - off) for every index triple of a box of ``dims``
        (``step`` the dims of the numbered grid), as a 3D array like ``_state3``."""
        i = np.arange(dims[0], dtype=np.int64) - off[0]
        j = np.arange(dims[1], dtype=np.int64) - off[1]
        k = np.arange(dims[2], dtype=np.int64) - off[2]
        return base + (k[:, None, None] * step[1] + j[None, :, None]) * step[0] + i[None, None, :]

    @staticmethod
    def _coords3(dims, lo, h, shift, out):
        """out[...] = lo + h (ijk + shift) for every index triple of a box (out: (N, 3))."""
        o = out.reshape(dims[2], dims[1], dims[0], 3)
        o[..., 0] = (lo[0] + h * (np.arange(dims[0]) + shift[0]))[None, None, :]
        o[..., 1] = (lo[1] + h * (np.arange(dims[1]) + shift[1]))[None, :, None]
        o[..., 2] = (lo[2] + h * (np.arange(dims[2]) + shift[2]))[:, None, None]

    def _build_level(self, lv):
        """Cells, faces and edges of one level (disjoint slices of every table)."""
        zero = np.zeros(3, dtype=np.int64)
        L, hL = lv.L, lv.h
        cb = self.cell_base[L]
        ncl = int(np.prod(lv.n))
        cs = slice(cb, cb + ncl)
        self.cell_active[cs] = (self._state3(L, lv.n, zero) == ACTIVE).ravel()
        self.cell_h[cs] = hL
        self.cell_level[cs] = L
        self._coords3(lv.n, lv.lo, hL, (0.5, 0.5, 0.5), self.cpos[cs])
        for a in range(3):
            # faces of axis a
            fd = lv.face_dims(a)
            fb = self.face_base[L][a]
            fs = slice(fb, fb + int(np.prod(fd)))
            slo = self._state3(L, fd, _E[a])
            shi = self._state3(L, fd, zero)
            ex = ((slo == ACTIVE) & (shi == ACTIVE)) | ((slo == ACTIVE) & (shi == OUT)) \
                | ((slo == OUT) & (shi == ACTIVE))
            self.face_exists[fs] = ex.ravel()
            self.face_axis[fs] = a
            self.face_h[fs] = hL
            self.face_level[fs] = L
            self._coords3(fd, lv.lo, hL, 0.5 * (1 - _E[a]), self.fpos[fs])
            lo_c = np.where(slo == ACTIVE, self._flat3(fd, cb, _E[a], lv.n), -1)
            hi_c = np.where(shi == ACTIVE, self._flat3(fd, cb, zero, lv.n), -1)
            if L + 1 < self.N:                        # interface faces: coarse neighbour
                up = self.levels[L + 1]
                for m, c3, sub in ((ex & (slo == OUT), lo_c, _E[a]), (ex & (shi == OUT), hi_c, zero)):
                    kk, jj, ii = np.nonzero(m)
                    fg = np.stack([ii, jj, kk], axis=1).astype(np.int64)
                    cc = up.hole_lo + np.floor_divide(fg - sub, 2)
                    c3[m] = self.cell_id(L + 1, cc)
            else:                                     # domain boundary families 1..6
                ia = np.arange(fd[a])
                fam1 = np.zeros(fd[a], dtype=np.int8)
                fam_lo, fam_hi = {0: (1, 2), 1: (6, 5), 2: (4, 3)}[a]
                fam1[ia == 0] = fam_lo
                fam1[ia == lv.n[a]] = fam_hi
                shape = [1, 1, 1]
                shape[2 - a] = fd[a]
                self.face_bc[fs] = np.broadcast_to(fam1.reshape(shape), (fd[2], fd[1], fd[0])).ravel()
            self.face_lo[fs] = np.where(ex, lo_c, -1).ravel()
            self.face_hi[fs] = np.where(ex, hi_c, -1).ravel()
            # edges of axis a
            ed = lv.edge_dims(a)
            eb = self.edge_base[L][a]
            es = slice(eb, eb + int(np.prod(ed)))
            b, c = (a + 1) % 3, (a + 2) % 3
            any_act = np.zeros((ed[2], ed[1], ed[0]), dtype=bool)
            any_hole = np.zeros_like(any_act)
            for db in (0, 1):
                for dc in (0, 1):
                    st = self._state3(L, ed, db * _E[b] + dc * _E[c])
                    any_act |= st == ACTIVE
                    any_hole |= st == HOLE
            self.edge_exists[es] = (any_act & ~any_hole).ravel()
            self.edge_axis[es] = a
            self.edge_h[es] = hL
            self.edge_level[es] = L
            self._coords3(ed, lv.lo, hL, 0.5 * _E[a], self.epos[es])

    def _level_links(self, lv):
        """Face-edge links of one level's faces, in face order (needs the edges of
        this level and of the finer one)."""
        L = lv.L
        zero = np.zeros(3, dtype=np.int64)
        lk_f, lk_e, lk_s, lk_x = [], [], [], []
        for a in range(3):
            fd = lv.face_dims(a)
            fb = self.face_base[L][a]
            keep = self.face_exists[fb:fb + int(np.prod(fd))]
            kept = np.flatnonzero(keep)
            fid = fb + kept
            b, c = (a + 1) % 3, (a + 2) % 3
            for ax, off, sgn in ((b, zero, 1.0), (c, _E[b], 1.0), (b, _E[c], -1.0), (c, zero, -1.0)):
                eid = self._flat3(fd, self.edge_base[L][ax], -off, lv.edge_dims(ax)).ravel()[kept]
                ok = self.edge_exists[eid]
                lk_f.append(fid[ok]); lk_e.append(eid[ok])
                lk_s.append(np.full(int(ok.sum()), sgn)); lk_x.append(np.zeros(int(ok.sum()), bool))
                if not np.all(ok):                    # collapsed coarse edge -> 2 fine sub-edges
                    if L == 0:
                        raise AssertionError("missing edge on the finest level")
                    lvf = self.levels[L - 1]
                    eg = _unflat(fd, kept[~ok]) + off
                    fine0 = 2 * (eg - lv.hole_lo)
                    for j, add in enumerate((0, _E[ax])):
                        sub = self.edge_id(L - 1, ax, fine0 + add)
                        if not np.all(self.edge_exists[sub]) or np.any(fine0 + add < 0) \
                                or np.any(fine0 + add >= lvf.edge_dims(ax)):
                            raise AssertionError("collapsed edge without fine sub-edges")
                        lk_f.append(fid[~ok]); lk_e.append(sub)
                        lk_s.append(np.full(sub.size, sgn)); lk_x.append(np.full(sub.size, j == 1))
        return lk_f, lk_e, lk_s, lk_x

    def build(self):
        """Existence masks, face cells, face-edge links and geometry (dense ids).

        Every entity of one level and axis has a contiguous range of dense ids in
        x-fastest order, so each table is filled by slices of 3D arrays built from
        per-axis 1D tests.
        """
        NC, NF, NE = self.NC, self.NF, self.NE
        self._rf = None
        self.cell_active = np.zeros(NC, dtype=bool)
        self.cell_h = np.zeros(NC)
        self.cpos = np.zeros((NC, 3))
        self.face_exists = np.zeros(NF, dtype=bool)
        self.face_axis = np.zeros(NF, dtype=np.int8)
        self.face_h = np.zeros(NF)
        self.face_lo = np.full(NF, -1, dtype=np.int64)     # -a side cell (dense) or -1
        self.face_hi = np.full(NF, -1, dtype=np.int64)     # +a side cell (dense) or -1
        self.face_bc = np.zeros(NF, dtype=np.int8)
        self.fpos = np.zeros((NF, 3))
        self.edge_exists = np.zeros(NE, dtype=bool)
        self.edge_axis = np.zeros(NE, dtype=np.int8)
        self.edge_h = np.zeros(NE)
        self.epos = np.zeros((NE, 3))
        self.edge_level = np.zeros(NE, dtype=np.int8)
        self.face_level = np.zeros(NF, dtype=np.int8)
        self.cell_level = np.zeros(NC, dtype=np.int8)
        # levels fill disjoint slices, so they are built on host threads (the array
        # kernels release the interpreter lock); the links of each level, which
        # read the finer level's edges, follow, concatenated in level order
        with ThreadPoolExecutor(max_workers=max(1, min(4, self.N))) as pool:
            list(pool.map(self._build_level, self.levels))
            parts = list(pool.map(self._level_links, self.levels))
        lk_f = [x for pt in parts for x in pt[0]]
        lk_e = [x for pt in parts for x in pt[1]]
        lk_s = [x for pt in parts for x in pt[2]]
        lk_x = [x for pt in parts for x in pt[3]]
        self.link_face = np.concatenate(lk_f)
        self.link_edge = np.concatenate(lk_e)
        self.link_sign = np.concatenate(lk_s)
        self.link_extra = np.concatenate(lk_x)
        self.face_Af = self.face_h ** 2
        self.cell_vol = self.cell_h ** 3
        # edge boundary family = max over boundary faces containing it (make_euler_mesh.py:594-601)
        self.edge_bc = np.zeros(NE, dtype=np.int8)
        bfl = self.face_bc[self.link_face] > 0
        np.maximum.at(self.edge_bc, self.link_edge[bfl], self.face_bc[self.link_face[bfl]])
        self._built = True
        return self

    # ---- geometry needed by the operators ---------------------------------
    def face_rf(self):
        """rf = (cpos_hi or fpos) - (cpos_lo or fpos), the +a oriented centre-to-centre vector
        (computed once per built layout; callers must not modify it)."""
        if getattr(self, "_rf", None) is not None:
            return self._rf
        self._rf = self._face_rf()
        return self._rf

    def _face_rf(self):
        lo, hi = self.face_lo, self.face_hi
        a = np.where(lo >= 0, 0, 1)
        plo = np.where((lo >= 0)[:, None], self.cpos[np.maximum(lo, 0)], self.fpos)
        phi = np.where((hi >= 0)[:, None], self.cpos[np.maximum(hi, 0)], self.fpos)
        del a
        return phi - plo

    def face_AoL(self):
        rf = self.face_rf()
        ax = self.face_axis.astype(np.int64)
        rfa = rf[np.arange(rf.shape[0]), ax]
        den = np.einsum("ij,ij->i", rf, rf)
        out = np.zeros(self.NF)
        ok = self.face_exists & (den > 0)
        out[ok] = rfa[ok] * self.face_Af[ok] / den[ok]
        return out

    def boundary_faces(self):
        return np.nonzero(self.face_exists & (self.face_bc > 0))[0]

    # ---- reference-convention export --------------------------------------
    def node_first_level(self, L, ijk):
        """Coarsest level owning a level-L grid node (L, or L+1 on the box surface at even index)."""
        lv = self.levels[L]
        if L + 1 >= self.N:
            return np.full(ijk.shape[0], L)
        surf = np.any((ijk == 0) | (ijk == lv.n), axis=1)
        even = np.all(ijk % 2 == 0, axis=1)
        return np.where(surf & even, L + 1, L)

    def edge_sigma(self):
        """+1 where the reference edge tangent points +a, -1 where it points -a.

        The reference orders an edge's two nodes by node id
        (``make_euler_mesh.py:574-583``); node ids are assigned outermost level
        first (``make_euler_mesh.py:355-394``), so a tangent points away from a
        node first created on a coarser level.
        """
        sig = np.ones(self.NE)
        for lv in self.levels:
            for a in range(3):
                eg = _grid(lv.edge_dims(a))
                eid = self.edge_id(lv.L, a, eg)
                fa = self.node_first_level(lv.L, eg)
                fb = self.node_first_level(lv.L, eg + _E[a])
                sig[eid] = np.where(fb > fa, -1.0, 1.0)
        return sig

    def face_sigma(self):
        """+1 where the reference face normal points +a.

        The reference orients a face from its first cell to its second
        (``ib_core_np.py:64-67``); the first cell is the lower cell id, i.e.
        the fine cell at an interface and the only cell at the domain boundary.
        """
        lo, hi = self.face_lo, self.face_hi
        sig = np.ones(self.NF)
        lvl = self.cell_level
        lo_ok, hi_ok = lo >= 0, hi >= 0
        # boundary: only a +a side cell -> normal points -a
        sig[~lo_ok & hi_ok] = -1.0
        both = lo_ok & hi_ok
        coarse_lo = np.zeros(self.NF, dtype=bool)
        coarse_lo[both] = lvl[lo[both]] > lvl[hi[both]]
        sig[coarse_lo] = -1.0
        return sig

    def export_mesh(self):
        """Compact unstructured description in the reference's conventions.

        Returns ``(desc, maps)`` where ``desc`` has the fields of the oracle's
        ``MeshDesc`` and ``maps`` holds the dense<->compact id maps.
        """
        cells = np.nonzero(self.cell_active)[0]
        faces = np.nonzero(self.face_exists)[0]
        edges = np.nonzero(self.edge_exists)[0]
        c_of = np.full(self.NC, -1, dtype=np.int64); c_of[cells] = np.arange(cells.size)
        f_of = np.full(self.NF, -1, dtype=np.int64); f_of[faces] = np.arange(faces.size)
        e_of = np.full(self.NE, -1, dtype=np.int64); e_of[edges] = np.arange(edges.size)
        fsig = self.face_sigma()
        lo, hi = self.face_lo[faces], self.face_hi[faces]
        first = np.where(fsig[faces] > 0, lo, hi)
        second = np.where(fsig[faces] > 0, hi, lo)
        F2C = np.stack([c_of[first], np.where(second >= 0, c_of[np.maximum(second, 0)], -1)], axis=1)
        base = ~self.link_extra
        order = np.argsort(self.link_face[base], kind="stable")
        lf, le = self.link_face[base][order], self.link_edge[base][order]
        if not np.array_equal(np.bincount(f_of[lf], minlength=faces.size), np.full(faces.size, 4)):
            raise AssertionError("every face must have 4 base links")
        F2E = e_of[le].reshape(-1, 4)
        # faces are in dense order, links sorted by face -> rows align with compact face order
        extra = np.stack([f_of[self.link_face[self.link_extra]], e_of[self.link_edge[self.link_extra]]], axis=1)
        # nodes + edge orientation
        esig = self.edge_sigma()[edges]
        origin = self.levels[-1].lo
        p0 = self.epos[edges] - 0.5 * self.edge_h[edges, None] * _E[self.edge_axis[edges]]
        p1 = p0 + self.edge_h[edges, None] * _E[self.edge_axis[edges]]
        k0 = np.rint((p0 - origin) / self.h0).astype(np.int64)
        k1 = np.rint((p1 - origin) / self.h0).astype(np.int64)
        allk = np.concatenate([k0, k1])
        uniq, inv = np.unique(allk, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        nodes = origin + uniq * self.h0
        n0, n1 = inv[:edges.size], inv[edges.size:]
        E2N = np.where((esig > 0)[:, None], np.stack([n0, n1], 1), np.stack([n1, n0], 1))
        lv0 = self.levels[0]
        ic = c_of[self.cell_id(0, _grid(lv0.n))].reshape(lv0.n[2], lv0.n[1], lv0.n[0]).transpose(2, 1, 0)
        desc = dict(nodes=nodes, F2C=F2C, F2E=F2E, E2N=E2N, link_fe_insert=extra,
                    bc_edge=self.edge_bc[edges].astype(np.int64),
                    bc_face=self.face_bc[faces].astype(np.int64), ncell=int(cells.size),
                    index_cell=np.ascontiguousarray(ic), pos_ref=lv0.lo + 0.5 * self.h0, dx=self.h0)
        maps = dict(cells=cells, faces=faces, edges=edges, c_of=c_of, f_of=f_of, e_of=e_of,
                    face_sigma=fsig[faces], edge_sigma=esig)
        return desc, maps


def concentric_layout(h, half_widths):
    """Concentric cubes ``[-w, w]^3`` (innermost first), as the sphere cases use."""
    return NestedLayout(h, [((-w, -w, -w), (w, w, w)) for w in half_widths])
