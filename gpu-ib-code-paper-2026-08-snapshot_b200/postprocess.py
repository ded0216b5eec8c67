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
the library is missing.  The reference's band repair
(``ib_postprocess.py:213-250``, an lsqr on the few cells next to the body) is
not part of this module.
"""
from __future__ import annotations

import ctypes as C
import threading

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
