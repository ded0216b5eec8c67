"""Structured stencil templates of the CG matvec and their patch rows (host side).

The matvec ``w = R I V P C p`` (``ib_core_np.py:168-175``) runs on the GPU as
three structured kernels per level, each evaluating one constant-coefficient
template for every slot of the level box:

* ``A``  (curl + interp_f2c):  vc_d[c] = (U_d[c-] + U_d[c+]) / (2 h^2), with
  U_a on an a-face the signed sum of its 4 edges;
* ``V``  (viscous block):      vq[c] = rou v[c] - k (sum_nb (v[nb]-v[c])),
  k = dt visc / (2 h^2), a neighbour outside the box counting as a zero ghost
  across a face with AoL = 2h (the domain boundary);
* ``RI`` (integr_c2f + rot):   F_a = (h/2)(vq_a[lo] + vq_a[hi]) on a-faces,
  w_t[e] = F_{t+2}[e] - F_{t+2}[e-e_{t+1}] + F_{t+1}[e-e_{t+2}] - F_{t+1}[e].

Rows where a template differs from the exact operator (interfaces between
levels, hole surfaces, collapsed edges) are found by evaluating both on
random inputs that also fill every absent slot with random values, so a
template row that reads an absent slot is caught too.  Those rows are
replaced on the GPU by explicit CSR rows ("patches") of the exact composite.

The functions here are the NumPy mirror of the CUDA kernels; the GPU tests
compare the kernels with them and with the exact operators.
"""
from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor

import numpy as np
import scipy.sparse as sp

from .layout import _grid


def edge_views(lay, vec):
    """Per level, the three edge arrays of a dense edge vector as (z,y,x) views."""
    out = []
    for lv in lay.levels:
        vs = []
        for a in range(3):
            dims = lv.edge_dims(a)
            b = lay.edge_base[lv.L][a]
            vs.append(vec[b:b + int(np.prod(dims))].reshape(dims[2], dims[1], dims[0]))
        out.append(vs)
    return out


def cell_view(lay, vec, L):
    lv = lay.levels[L]
    b = lay.cell_base[L]
    return vec[b:b + int(np.prod(lv.n))].reshape(lv.n[2], lv.n[1], lv.n[0])


def face_views(lay, vec):
    out = []
    for lv in lay.levels:
        vs = []
        for a in range(3):
            dims = lv.face_dims(a)
            b = lay.face_base[lv.L][a]
            vs.append(vec[b:b + int(np.prod(dims))].reshape(dims[2], dims[1], dims[0]))
        out.append(vs)
    return out


def curl_faces(ex, ey, ez):
    """Face circulations of one level (numpy (z,y,x) axis order)."""
    Ux = ey[:-1, :, :] + ez[:, 1:, :] - ey[1:, :, :] - ez[:, :-1, :]
    Uy = ez[:, :, :-1] + ex[1:, :, :] - ez[:, :, 1:] - ex[:-1, :, :]
    Uz = ex[:, :-1, :] + ey[:, :, 1:] - ex[:, 1:, :] - ey[:, :, :-1]
    return Ux, Uy, Uz


def t_A(lay, p):
    """Template A: p (NE) -> vc (3, NC)."""
    vc = np.zeros((3, lay.NC))
    for lv, (ex, ey, ez) in zip(lay.levels, edge_views(lay, p)):
        Ux, Uy, Uz = curl_faces(ex, ey, ez)
        s = 1.0 / (2.0 * lv.h * lv.h)
        cell_view(lay, vc[0], lv.L)[...] = (Ux[:, :, :-1] + Ux[:, :, 1:]) * s
        cell_view(lay, vc[1], lv.L)[...] = (Uy[:, :-1, :] + Uy[:, 1:, :]) * s
        cell_view(lay, vc[2], lv.L)[...] = (Uz[:-1] + Uz[1:]) * s
    return vc


def t_V(lay, v, rou, visc, dt):
    """Template V for one component: v (NC) -> vq (NC)."""
    out = np.zeros(lay.NC)
    for lv in lay.levels:
        c = cell_view(lay, v, lv.L)
        k = 0.5 * dt * visc / (lv.h * lv.h)
        s = np.zeros_like(c)
        for ax in range(3):
            up = np.roll(c, -1, axis=2 - ax)
            dn = np.roll(c, 1, axis=2 - ax)
            sl_hi = [slice(None)] * 3
            sl_lo = [slice(None)] * 3
            sl_hi[2 - ax] = -1
            sl_lo[2 - ax] = 0
            tu = up - c
            td = dn - c
            tu[tuple(sl_hi)] = -2.0 * c[tuple(sl_hi)]
            td[tuple(sl_lo)] = -2.0 * c[tuple(sl_lo)]
            s = s + tu + td
        cell_view(lay, out, lv.L)[...] = rou * c - k * s
    return out


def t_RI(lay, vq):
    """Template RI: vq (3, NC) -> w (NE), unmasked."""
    w = np.zeros(lay.NE)
    wv = edge_views(lay, w)
    for lv in lay.levels:
        h2 = 0.5 * lv.h
        cv = [cell_view(lay, vq[d], lv.L) for d in range(3)]
        nz, ny, nx = cv[0].shape
        F = []
        for a in range(3):
            c = cv[a]
            shp = list(c.shape)
            shp[2 - a] += 1
            lo = np.zeros(shp)
            hi = np.zeros(shp)
            sl = [slice(None)] * 3
            sl[2 - a] = slice(0, -1)
            hi[tuple(sl)] = c                         # face idx has hi cell idx
            sl[2 - a] = slice(1, None)
            lo[tuple(sl)] = c                         # face idx has lo cell idx-1
            F.append(h2 * (lo + hi))
        for t in range(3):
            f2 = F[(t + 2) % 3]
            f1 = F[(t + 1) % 3]
            dims = lv.edge_dims(t)
            out = np.zeros((dims[2], dims[1], dims[0]))
            out += _shift_read(f2, dims, 0, None)
            out -= _shift_read(f2, dims, (t + 1) % 3, -1)
            out += _shift_read(f1, dims, (t + 2) % 3, -1)
            out -= _shift_read(f1, dims, 0, None)
            wv[lv.L][t][...] = out
    return w


def _shift_read(F, dims, axis, off):
    """out[idx] = F[idx + off*e_axis] (zero outside F) over an edge box of ``dims``."""
    out = np.zeros((dims[2], dims[1], dims[0]))
    fz, fy, fx = F.shape
    shape_f = (fx, fy, fz)
    src = [slice(None)] * 3
    dst = [slice(None)] * 3
    for ax in range(3):
        n_out = dims[ax]
        o = off if (off is not None and ax == axis) else 0
        lo = max(0, -o)
        hi = min(n_out, shape_f[ax] - o)
        dst[2 - ax] = slice(lo, hi)
        src[2 - ax] = slice(lo + o, hi + o)
    out[tuple(dst)] = F[tuple(src)]
    return out


class MatvecPlan:
    """Templates + patch rows for ``w = mask * (R I V P C) p`` on one layout.

    The classification does not depend on density, viscosity or dt: the V
    patch stores rows of ``Vd`` and the kernel forms ``rou v - kfac (Vd v)``
    with ``kfac = dt visc / 2``.
    """

    def __init__(self, ops, dir_mask, seed=7, probes=2):
        lay = ops.lay
        self.ops, self.lay = ops, lay
        self.mask = lay.edge_exists & ~dir_mask
        rng = np.random.default_rng(seed)
        act = lay.cell_active
        # the probe vectors, drawn in a fixed order; the comparisons of the three
        # stages run on host threads (the array and sparse kernels release the
        # interpreter lock) and their flags are or-ed, so the result is the same
        draws = []
        for _ in range(probes):
            p = rng.standard_normal(lay.NE)
            v = rng.standard_normal(lay.NC)
            vq = rng.standard_normal((3, lay.NC))
            draws.append((p, v, vq))

        def stage_a(p):
            U = ops.C @ p
            ex = np.stack([ops.P[d] @ U for d in range(3)])
            return np.any(_differs(t_A(lay, p), ex), axis=0) & act

        def stage_v(v):
            # rou=0, visc=2, dt=1 -> template computes -(Vd v)
            return _differs(t_V(lay, v, 0.0, 2.0, 1.0), -(ops.Vd @ v)) & act

        def stage_ri(vq):
            exw = ops.R @ sum(ops.I[d] @ vq[d] for d in range(3))
            return _differs(t_RI(lay, vq), exw) & self.mask

        with ThreadPoolExecutor(max_workers=min(6, 3 * probes)) as pool:
            fa = [pool.submit(stage_a, p) for p, _, _ in draws]
            fv = [pool.submit(stage_v, v) for _, v, _ in draws]
            fr = [pool.submit(stage_ri, vq) for _, _, vq in draws]
            upper = pool.submit(upper_face_edges, lay)
            irrA = np.logical_or.reduce([x.result() for x in fa])
            irrV = np.logical_or.reduce([x.result() for x in fv])
            irrRI = np.logical_or.reduce([x.result() for x in fr])
            upper = upper.result()
        # the edges of the nodes on a level's upper faces (i = nx, j = ny or k = nz) are
        # interface or boundary edges; when every one of them is already an exact row or
        # masked (closed cavities), the RI kernel covers only nodes i < nx, j < ny, k < nz
        self.upper_exact = not np.any(upper & self.mask & ~irrRI)
        self.irrA, self.irrV, self.irrRI = irrA, irrV, irrRI
        ra = np.nonzero(irrA)[0]
        # exact composite rows: component-major blocks of the same cell list
        self.patchA = (ra, sp.vstack([(ops.P[d][ra] @ ops.C) for d in range(3)]).tocsr())
        rv = np.nonzero(irrV)[0]
        self.patchV = (rv, ops.Vd[rv].tocsr())
        re = np.nonzero(irrRI)[0]
        RI = sp.hstack([(ops.R[re] @ ops.I[d]).tocsr() for d in range(3)]).tocsr()
        self.patchRI = (re, RI)        # columns: d*NC + cell

    def apply(self, p, rou=1.0, visc=0.0, dt=0.0, alpd=True):
        """NumPy mirror of the three GPU kernels with patches (for tests)."""
        lay = self.lay
        vc = t_A(lay, p)
        rows, M = self.patchA
        n = rows.size
        pa = M @ p
        for d in range(3):
            vc[d, rows] = pa[d * n:(d + 1) * n]
        if alpd:
            vq = np.stack([t_V(lay, vc[d], rou, visc, dt) for d in range(3)])
            rows, M = self.patchV
            for d in range(3):
                vq[d, rows] = rou * vc[d, rows] - (0.5 * dt * visc) * (M @ vc[d])
        else:
            vq = vc
        w = t_RI(lay, vq)
        rows, M = self.patchRI
        w[rows] = M @ vq.reshape(-1)
        w[~self.mask] = 0.0
        return w

    def summary(self):
        return dict(patchA=int(self.patchA[0].size), patchV=int(self.patchV[0].size),
                    patchRI=int(self.patchRI[0].size), nnzA=int(self.patchA[1].nnz),
                    nnzV=int(self.patchV[1].nnz), nnzRI=int(self.patchRI[1].nnz))


def upper_face_edges(lay):
    """Edges whose lower node lies on an upper face of its level box (a coordinate == n)."""
    out = np.zeros(lay.NE, dtype=bool)
    for lv in lay.levels:
        for a in range(3):
            ed = lv.edge_dims(a)
            i, j, k = (np.arange(ed[t]) == lv.n[t] for t in range(3))
            up = k[:, None, None] | j[None, :, None] | i[None, None, :]
            eb = lay.edge_base[lv.L][a]
            out[eb:eb + up.size] = up.ravel()
    return out


def _differs(a, b, rtol=1e-12):
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return np.abs(a - b) > rtol * scale
