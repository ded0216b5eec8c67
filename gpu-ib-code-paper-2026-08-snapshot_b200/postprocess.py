"""Offline pressure recovery with the graph solve on the device.

``recover_pressure`` has the signature, validation, gauge and diagnostics of
the reference's ``recover_pressure`` (``ib_postprocess.py:49-107``):

* internal faces (second cell >= 0) give the jump ``p2 - p1 = (g1 + g2)/2 . (x2 - x1)``
  weighted by ``A / |x2 - x1|``;
* the weighted graph Laplacian ``B^T W B`` with the first cell pinned is solved
  from zero by Jacobi-preconditioned CG with the stop ``|r| < tolerance |b|``
  (scipy's ``cg`` with ``atol = 0``) and at most ``max(2000, 10 n)`` iterations;
* the mean over the boundary-adjacent cells (every cell if none) is removed.

Everything after the shape checks runs on the device in one call
(``pyib_recover_pressure``): the value checks, the face weights and jumps, the
Laplacian in CSR (rows sorted by neighbour and face), the connectivity check,
the CG and the gauge, all with sums in fixed orders.  ``assemble`` builds the
same reduced system on the host for callers of the generic CSR solver
``graph_pcg`` (``pyib_graph_pcg``).  There is no CPU solve: the calls fail if
the library is missing.

``repair_pressure_band`` is the reference's band repair
(``ib_postprocess.py:200-250``) on a ``UniformLattice`` (``ib_postprocess.py:108-140``):
the least-squares fit of the band cells' pressure to the lattice-edge jumps,
the cells outside the band held.  The reference solves it with ``lsqr``; here
its normal equations (a graph Laplacian plus one diagonal term per edge to a
held cell, positive definite once every band component is anchored) are
solved by ``graph_pcg`` on the device to a tighter tolerance than lsqr's
``atol = btol = 1e-11``, so both reach the same least-squares solution.
"""
from __future__ import annotations

import ctypes as C
import threading
from dataclasses import dataclass

import numpy as np
from scipy.sparse import csr_matrix
from scipy.sparse.csgraph import connected_components

from . import _lib


def _finite(name, values, shape=None):
    values = np.asarray(values, dtype=np.float64)
    if shape is not None and values.shape != shape:
        raise ValueError(f"{name} must have shape {shape}, got {values.shape}")
    if not np.isfinite(values).all():
        raise ValueError(f"{name} contains non-finite values")
    return values


def bare_handle(device=0):
    """A context with a one-cell layout: a device, a stream, an error slot and a
    grow-only workspace for the calls that take all their data from the caller
    (``pyib_recover_pressure``, ``pyib_graph_pcg``)."""
    lay = _lib.Layout()
    lay.nlevels = 1
    lay.n[0][0] = lay.n[0][1] = lay.n[0][2] = 1
    lay.h[0] = 1.0
    lay.ncell, lay.nface, lay.nedge = 1, 6, 12
    lay.device = int(device)
    return _lib.Handle(lay)


_local = threading.local()


def default_handle(device=0):
    """This host thread's context on ``device`` for calls made without a handle:
    made on first use and kept, so its workspace is reused by later calls (one
    context per host thread, as the library requires)."""
    handles = getattr(_local, "handles", None)
    if handles is None:
        handles = _local.handles = {}
    h = handles.get(int(device))
    if h is None or not h.ptr:
        h = handles[int(device)] = bare_handle(device)
    return h


def close_default_handles():
    """Release this host thread's default contexts and their workspaces."""
    handles = getattr(_local, "handles", None) or {}
    for h in handles.values():
        h.close()
    handles.clear()


def laplacian_csr(count, first, second, weights):
    """CSR of ``B^T diag(w) B`` (B: the signed face-cell incidence), duplicates summed,
    columns ascending within each row."""
    rows = np.concatenate([first, second, first, second])
    cols = np.concatenate([second, first, first, second])
    vals = np.concatenate([-weights, -weights, weights, weights])
    key = rows.astype(np.int64) * count + cols
    order = np.argsort(key, kind="stable")
    key, vals = key[order], vals[order]
    start = np.flatnonzero(np.r_[True, key[1:] != key[:-1]])
    summed = np.add.reduceat(vals, start)
    ukey = key[start]
    r, c = ukey // count, ukey % count
    ptr = np.zeros(count + 1, dtype=np.int64)
    np.cumsum(np.bincount(r, minlength=count), out=ptr[1:])
    return ptr, c.astype(np.int32), summed


def graph_pcg(handle, ptr, col, val, rhs, tolerance, max_iterations, timing=None):
    """Solve the CSR system on the device; returns (x, iterations).  ``timing``
    (a dict) receives ``solve_ms``, the device time of the iterations."""
    n = len(rhs)
    ptr = np.ascontiguousarray(ptr, dtype=np.int64)
    col = np.ascontiguousarray(col, dtype=np.int32)
    val = np.ascontiguousarray(val, dtype=np.float64)
    rhs = np.ascontiguousarray(rhs, dtype=np.float64)
    x = np.empty(n)
    it = C.c_int32(0)
    ms = C.c_double(0.0)
    handle.call("pyib_graph_pcg", C.c_int64(n), ptr.ctypes.data_as(C.c_void_p),
                col.ctypes.data_as(C.c_void_p), val.ctypes.data_as(C.c_void_p),
                rhs.ctypes.data_as(C.c_void_p), x.ctypes.data_as(C.c_void_p),
                C.c_double(tolerance), C.c_int32(int(max_iterations)), C.byref(it), C.byref(ms))
    if timing is not None:
        timing["solve_ms"] = ms.value
    return x, int(it.value)


def assemble(cell_positions, face_cells, face_area, gradient):
    """The reduced system on the host, for ``graph_pcg`` (``ib_postprocess.py:58-89``).

    Returns ``(ptr, col, val, rhs, graph)``: the CSR of the Laplacian with cell 0
    pinned (rows and columns 1..n-1), its right-hand side, and a dict with the
    face data the gauge and diagnostics need.  Raises ValueError as the reference does.
    """
    positions = _finite("cell_positions", cell_positions)
    count = len(positions)
    if positions.shape != (count, 3) or count < 2:
        raise ValueError("pressure recovery needs at least two 3D cells")
    gradient = _finite("gradient", gradient, positions.shape)
    pairs = np.asarray(face_cells)
    if pairs.ndim != 2 or pairs.shape[1] != 2 or pairs.dtype.kind not in "iu":
        raise ValueError("face_cells must be an integer (number_of_faces, 2) array")
    if np.any(pairs[:, 0] < 0) or np.any(pairs >= count) or np.any(pairs[:, 1] < -1):
        raise ValueError("face_cells contains invalid cell ids")
    areas = _finite("face_area", face_area, (len(pairs),))
    if np.any(areas <= 0):
        raise ValueError("face areas must be positive")
    internal = pairs[:, 1] >= 0
    first, second = (pairs[internal].T).astype(np.int64)
    displacement = positions[second] - positions[first]
    distance = np.linalg.norm(displacement, axis=1)
    if not len(distance) or np.any(distance <= 0):
        raise ValueError("pressure graph has no valid internal faces")
    weights = areas[internal] / distance
    ptr, col, val = laplacian_csr(count, first, second, weights)
    graph = csr_matrix((np.ones(len(col)), col, ptr), shape=(count, count))
    if connected_components(graph, directed=False, return_labels=False) != 1:
        raise ValueError("pressure graph is disconnected; a unique gauge is unavailable")
    jumps = 0.5 * np.sum((gradient[first] + gradient[second]) * displacement, axis=1)
    wj = weights * jumps
    rhs = np.bincount(second, wj, minlength=count) - np.bincount(first, wj, minlength=count)
    # the reduced system: drop row and column 0 (the pinned cell)
    seg_col, seg_val = col[ptr[1]:], val[ptr[1]:]
    seg_row = np.repeat(np.arange(count - 1), np.diff(ptr)[1:])
    keep = seg_col != 0
    rptr = np.zeros(count, dtype=np.int64)
    np.cumsum(np.bincount(seg_row[keep], minlength=count - 1), out=rptr[1:])
    faces = {"count": count, "pairs": pairs, "internal": internal, "first": first, "second": second,
             "weights": weights, "jumps": jumps}
    return rptr, seg_col[keep] - 1, seg_val[keep], rhs[1:], faces


def _validate_host(cell_positions, face_cells, face_area, gradient):
    """The reference's checks in its order, on the host: run only when an input's
    shape or type already fails, so that the first failing check is the one reported."""
    positions = _finite("cell_positions", cell_positions)
    count = len(positions)
    if positions.shape != (count, 3) or count < 2:
        raise ValueError("pressure recovery needs at least two 3D cells")
    _finite("gradient", gradient, positions.shape)
    pairs = np.asarray(face_cells)
    if pairs.ndim != 2 or pairs.shape[1] != 2 or pairs.dtype.kind not in "iu":
        raise ValueError("face_cells must be an integer (number_of_faces, 2) array")
    if np.any(pairs[:, 0] < 0) or np.any(pairs >= count) or np.any(pairs[:, 1] < -1):
        raise ValueError("face_cells contains invalid cell ids")
    _finite("face_area", face_area, (len(pairs),))


def recover_pressure(cell_positions, face_cells, face_area, gradient, *, tolerance=1e-10,
                     handle=None, device=0, timing=None):
    """Cell pressure whose face jumps best match the cell pressure gradients.

    Same arguments, result and errors as the reference (ValueError for invalid or
    disconnected input, RuntimeError when the solve does not converge).  Shapes and
    types are checked here; the value checks, the assembly, the connectivity check,
    the CG, the gauge and the residual run on the device (``pyib_recover_pressure``).
    ``handle`` reuses an existing context (a solver's ``h``); otherwise this host
    thread's context on ``device`` is used (``default_handle``).  The diagnostics
    add ``iterations``; ``timing`` (a dict) receives
    ``solve_ms`` (the CG), ``device_ms`` (the whole call on the device, copies
    included), ``sweeps`` (connectivity) and ``nnz``.
    """
    pos = np.asarray(cell_positions, dtype=np.float64)
    grad = np.asarray(gradient, dtype=np.float64)
    pairs = np.asarray(face_cells)
    area = np.asarray(face_area, dtype=np.float64)
    if not (pos.ndim == 2 and pos.shape[1] == 3 and len(pos) >= 2 and grad.shape == pos.shape
            and pairs.ndim == 2 and pairs.shape[1] == 2 and pairs.dtype.kind in "iu"
            and area.shape == (len(pairs),)):
        _validate_host(pos, pairs, area, grad)
        raise ValueError("invalid pressure-recovery inputs")
    pos = np.ascontiguousarray(pos)
    grad = np.ascontiguousarray(grad)
    area = np.ascontiguousarray(area)
    pairs64 = np.ascontiguousarray(pairs, dtype=np.int64)
    if pairs.dtype.kind == "u" and len(pairs) and pairs.max() >= len(pos):
        _validate_host(pos, pairs, area, grad)     # ids that do not fit int64
    count = len(pos)
    max_it = max(2000, 10 * count)
    out = np.empty(count)
    info = np.zeros(7)
    h = default_handle(device) if handle is None else handle
    rc = h.lib.pyib_recover_pressure(
        h.ptr, C.c_int64(count), pos.ctypes.data_as(C.c_void_p), C.c_int64(len(pairs64)),
        pairs64.ctypes.data_as(C.c_void_p), area.ctypes.data_as(C.c_void_p), grad.ctypes.data_as(C.c_void_p),
        C.c_double(tolerance), C.c_int32(int(max_it)), out.ctypes.data_as(C.c_void_p),
        info.ctypes.data_as(C.c_void_p))
    if rc == _lib.E_ARG:
        raise ValueError(h.error())
    if rc == _lib.E_NOCONV:
        raise RuntimeError(h.error())
    if rc != _lib.OK:
        raise _lib.B200Error(rc, f"pyib_recover_pressure: {h.error()}")
    if timing is not None:
        timing.update(solve_ms=float(info[3]), device_ms=float(info[4]), sweeps=int(info[5]), nnz=int(info[6]))
    diagnostics = {
        "gauge": "mean boundary-adjacent cells = 0" if info[2] else "mean cells = 0",
        "gradient_projection_weighted_rms": float(info[0]),
        "iterations": int(info[1]),
    }
    return out, diagnostics


@dataclass
class UniformLattice:
    """The finest uniform block of a saved snapshot (``ib_postprocess.py:108-140``):
    global cell ids (-1 where the block has no cell), origin and spacing."""

    cell_ids: np.ndarray
    origin: np.ndarray
    spacing: float

    def __post_init__(self):
        self.cell_ids = np.asarray(self.cell_ids)
        self.origin = _finite("lattice_origin", self.origin, (3,))
        self.spacing = float(self.spacing)
        if self.cell_ids.ndim != 3 or self.cell_ids.dtype.kind not in "iu":
            raise ValueError("index_cell must be a 3D integer array")
        if min(self.cell_ids.shape) < 2 or not np.isfinite(self.spacing) or self.spacing <= 0:
            raise ValueError("the lattice needs at least two cells per axis and positive spacing")

    @property
    def shape(self):
        return self.cell_ids.shape

    def coordinates(self):
        return self.origin + self.spacing * np.indices(self.shape).transpose(1, 2, 3, 0)

    def field(self, cell_field):
        """A per-cell field gathered onto the lattice (NaN where there is no cell)."""
        cell_field = np.asarray(cell_field)
        valid = self.cell_ids >= 0
        out = np.full(self.shape + cell_field.shape[1:], np.nan)
        out[valid] = cell_field[self.cell_ids[valid]]
        return out


def lattice_edges(shape, valid):
    """Axis-neighbour pairs of a lattice with both cells valid, x edges first, then
    y, then z, each in C order of the lower cell (``ib_postprocess.py:200-210``):
    (first, second, axis)."""
    ids = np.arange(int(np.prod(shape)), dtype=np.int64).reshape(shape)
    vflat = np.asarray(valid).ravel()
    parts = []
    for axis in range(3):
        lo, hi = [slice(None)] * 3, [slice(None)] * 3
        lo[axis], hi[axis] = slice(None, -1), slice(1, None)
        a, b = ids[tuple(lo)].ravel(), ids[tuple(hi)].ravel()
        keep = vflat[a] & vflat[b]
        parts.append((a[keep], b[keep], np.full(int(keep.sum()), axis, dtype=np.int64)))
    return tuple(np.concatenate([p[k] for p in parts]) for k in range(3))


def band_system(shape, spacing, raw_pressure, regular_gradient, signed_distance, width=1.5):
    """The band repair's least-squares problem and its normal equations, on the host.

    Band (target) cells: valid (signed distance >= 0, finite raw pressure) within
    ``width * spacing`` of the surface.  Every valid edge touching the band asks
    ``p[second] - p[first] = spacing (g[first] + g[second])_axis / 2``; a cell outside
    the band keeps its raw value, moved to the right-hand side.  Returns
    ``(target, ids, ptr, col, val, rhs)``: the mask, the band's flat lattice ids,
    and the CSR and right-hand side of ``B^T B x = B^T r``.  Raises the reference's
    ValueErrors for an empty or an unanchored band.
    """
    raw = np.asarray(raw_pressure, dtype=np.float64)
    dist = np.asarray(signed_distance, dtype=np.float64)
    grad = np.asarray(regular_gradient, dtype=np.float64)
    if raw.shape != tuple(shape) or dist.shape != tuple(shape) or grad.shape != tuple(shape) + (3,):
        raise ValueError("band repair fields must match the lattice shape")
    with np.errstate(invalid="ignore"):
        valid = (dist >= 0) & np.isfinite(raw)
        target = valid & (dist <= width * spacing)
    first, second, axes = lattice_edges(shape, valid)
    tflat = target.ravel()
    sel = tflat[first] | tflat[second]
    first, second, axes = first[sel], second[sel], axes[sel]
    ids = np.flatnonzero(tflat)
    n = len(ids)
    if not n:
        raise ValueError("pressure repair band contains no cells; refine the grid")
    local = np.full(tflat.size, -1, dtype=np.int64)
    local[ids] = np.arange(n)
    g = grad.reshape(-1, 3)
    r = 0.5 * spacing * (g[first, axes] + g[second, axes])
    rflat = raw.ravel()
    la, lb = local[first], local[second]
    both = (la >= 0) & (lb >= 0)
    only_a = (la >= 0) & (lb < 0)        # second cell held: p[a] = raw[b] - r
    only_b = (la < 0) & (lb >= 0)        # first cell held: p[b] = raw[a] + r
    # anchored components: every connected piece of the band needs a held neighbour
    count, labels = connected_components(
        csr_matrix((np.ones(int(both.sum())), (la[both], lb[both])), shape=(n, n)), directed=False)
    anchored = np.zeros(count, dtype=bool)
    anchored[labels[la[only_a]]] = True
    anchored[labels[lb[only_b]]] = True
    if not anchored.all():
        raise ValueError("pressure repair has an unanchored band; enlarge the finest region")
    # normal equations: B^T B (Laplacian of band-band edges, +1 on the diagonal per
    # held neighbour) and B^T r (r with the held values moved over)
    rows = np.concatenate([la[both], lb[both], la[both], lb[both], la[only_a], lb[only_b]])
    cols = np.concatenate([lb[both], la[both], la[both], lb[both], la[only_a], lb[only_b]])
    m = int(both.sum())
    vals = np.concatenate([-np.ones(2 * m), np.ones(2 * m), np.ones(int(only_a.sum()) + int(only_b.sum()))])
    key = rows * n + cols
    order = np.argsort(key, kind="stable")
    key, vals = key[order], vals[order]
    start = np.flatnonzero(np.r_[True, key[1:] != key[:-1]])
    val = np.add.reduceat(vals, start)
    ukey = key[start]
    ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(ukey // n, minlength=n), out=ptr[1:])
    col = (ukey % n).astype(np.int32)
    rhs = (np.bincount(lb[both], r[both], minlength=n) - np.bincount(la[both], r[both], minlength=n)
           + np.bincount(la[only_a], rflat[second[only_a]] - r[only_a], minlength=n)
           + np.bincount(lb[only_b], rflat[first[only_b]] + r[only_b], minlength=n))
    return target, ids, ptr, col, val, rhs


def repair_pressure_band(lattice, raw_pressure, regular_gradient, signed_distance, *, width=1.5,
                         tolerance=1e-13, handle=None, device=0, timing=None):
    """The reference's band repair (``ib_postprocess.py:213-250``): the band cells'
    pressure refitted in the least-squares sense to the gradient jumps, every other
    cell returned unchanged.

    Same arguments, result ``(repaired, target, iterations)`` and errors as the
    reference (ValueError for an empty or unanchored band, RuntimeError when the
    solve fails).  ``iterations`` counts the device CG's iterations on the normal
    equations (the reference reports lsqr's).  ``lattice`` needs ``shape`` and
    ``spacing`` (a ``UniformLattice``).  The solve stops at
    ``|r| < tolerance |b|``, with at most ``max(500, 20 n)`` iterations as the
    reference's lsqr.
    """
    shape = tuple(lattice.shape)
    target, ids, ptr, col, val, rhs = band_system(shape, float(lattice.spacing), raw_pressure,
                                                  regular_gradient, signed_distance, width)
    h = default_handle(device) if handle is None else handle
    try:
        x, iterations = graph_pcg(h, ptr, col, val, rhs, tolerance, max(500, 20 * len(ids)), timing)
    except _lib.B200Error as e:
        raise RuntimeError(f"pressure band solve failed ({e})") from e
    if not np.isfinite(x).all():
        raise RuntimeError("pressure band solve failed (non-finite result)")
    repaired = np.asarray(raw_pressure, dtype=np.float64).ravel().copy()
    repaired[ids] = x
    return repaired.reshape(shape), target, iterations
