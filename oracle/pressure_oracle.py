"""CPU oracle of the offline pressure recovery (test infrastructure only).

THIS MODULE IS THE CHECKER, NOT THE PRODUCT.  Only ``tests/`` and the CPU
leg of ``bench.py`` may import it.

Restates ``recover_pressure`` of the reference (``src/pyib/solver/ib_postprocess.py:49-107``)
with SciPy, as the reference itself computes it: the signed face-cell incidence B
over internal faces, weights ``A / |x2 - x1|``, jumps ``(g1 + g2)/2 . (x2 - x1)``,
the Laplacian ``B^T W B`` reduced by pinning cell 0 (rows and columns 1..n-1),
``scipy.sparse.linalg.cg`` with the Jacobi preconditioner, ``rtol = tolerance``,
``atol = 0``, ``maxiter = max(2000, 10 n)``, then the boundary-adjacent mean
removed (``ib_postprocess.py:99-102``).

Also restates the band repair ``repair_pressure_band``
(``ib_postprocess.py:200-250``): the lattice edges between valid cells, the
edges touching the band, their jumps, the incidence with the values of the
cells outside the band moved to the right-hand side, the anchor check, and
``scipy.sparse.linalg.lsqr`` with ``atol = btol = 1e-11``.

Parity pin: ``tests/test_pressure_oracle.py`` checks these restatements against
``tests/golden/pressure_golden.npz`` and ``tests/golden/band_golden.npz``, made by
running the reference's own functions (``tests/golden/make_pressure_golden.py``,
``tests/golden/make_band_golden.py``), and against the reference's known-answer
cases (``tests/test_ib_postprocess.py:76-84, 86-95``).
"""
from __future__ import annotations

import numpy as np
from scipy.sparse import coo_matrix, diags
from scipy.sparse.csgraph import connected_components
from scipy.sparse.linalg import cg, lsqr


def recover_pressure_checked(cell_positions, face_cells, face_area, gradient, *, tolerance=1e-10):
    """The reference's input checks in its order (``ib_postprocess.py:58-79``), then the solve."""
    def finite(name, values, shape=None):
        values = np.asarray(values, dtype=np.float64)
        if shape is not None and values.shape != shape:
            raise ValueError(f"{name} must have shape {shape}, got {values.shape}")
        if not np.isfinite(values).all():
            raise ValueError(f"{name} contains non-finite values")
        return values

    pos = finite("cell_positions", cell_positions)
    n = len(pos)
    if pos.shape != (n, 3) or n < 2:
        raise ValueError("pressure recovery needs at least two 3D cells")
    grad = finite("gradient", gradient, pos.shape)
    pairs = np.asarray(face_cells)
    if pairs.ndim != 2 or pairs.shape[1] != 2 or pairs.dtype.kind not in "iu":
        raise ValueError("face_cells must be an integer (number_of_faces, 2) array")
    if np.any(pairs[:, 0] < 0) or np.any(pairs >= n) or np.any(pairs[:, 1] < -1):
        raise ValueError("face_cells contains invalid cell ids")
    area = finite("face_area", face_area, (len(pairs),))
    if np.any(area <= 0):
        raise ValueError("face areas must be positive")
    inner = pairs[:, 1] >= 0
    dist = np.linalg.norm(pos[pairs[inner, 1]] - pos[pairs[inner, 0]], axis=1)
    if not len(dist) or np.any(dist <= 0):
        raise ValueError("pressure graph has no valid internal faces")
    return recover_pressure(pos, pairs, area, grad, tolerance=tolerance)


def recover_pressure(cell_positions, face_cells, face_area, gradient, *, tolerance=1e-10):
    """Returns (pressure, diagnostics) with the reference's keys plus ``iterations``."""
    pos = np.asarray(cell_positions, dtype=np.float64)
    grad = np.asarray(gradient, dtype=np.float64)
    pairs = np.asarray(face_cells)
    area = np.asarray(face_area, dtype=np.float64)
    n = len(pos)
    inner = pairs[:, 1] >= 0
    a, b = pairs[inner, 0], pairs[inner, 1]
    d = pos[b] - pos[a]
    w = area[inner] / np.linalg.norm(d, axis=1)
    m = len(a)
    inc = coo_matrix((np.r_[-np.ones(m), np.ones(m)], (np.r_[np.arange(m), np.arange(m)], np.r_[a, b])),
                     shape=(m, n)).tocsr()
    lap = (inc.T @ diags(w) @ inc).tocsr()
    if connected_components(lap, directed=False, return_labels=False) != 1:
        raise ValueError("pressure graph is disconnected; a unique gauge is unavailable")
    jump = 0.5 * np.sum((grad[a] + grad[b]) * d, axis=1)
    rhs = np.asarray(inc.T @ (w * jump))
    red = lap[1:, 1:]
    count = [0]

    def tick(_):
        count[0] += 1

    p = np.zeros(n)
    p[1:], status = cg(red, rhs[1:], M=diags(1.0 / red.diagonal()), rtol=tolerance, atol=0.0,
                       maxiter=max(2000, 10 * n), callback=tick)
    if status != 0:
        raise RuntimeError(f"pressure graph solve failed to converge (status {status})")
    edge = np.unique(pairs[~inner, 0])
    if not len(edge):
        edge = np.arange(n)
    p -= p[edge].mean()
    mis = inc @ p - jump
    return p, {
        "gauge": "mean boundary-adjacent cells = 0" if np.any(~inner) else "mean cells = 0",
        "gradient_projection_weighted_rms": float(np.sqrt(np.sum(w * mis**2) / w.sum())),
        "iterations": count[0],
    }


def uniform_graph(count, spacing):
    """Cell centres, face pairs (boundary faces with -1) and areas of a count^3 block,
    built as in the reference's test helper (``tests/test_ib_postprocess.py:18-33``)."""
    ids = np.arange(count**3).reshape((count,) * 3)
    axes = (np.arange(count) - 0.5 * (count - 1)) * spacing
    pos = np.stack(np.meshgrid(axes, axes, axes, indexing="ij"), axis=-1).reshape(-1, 3)
    faces = []
    for axis in range(3):
        lo, hi = [slice(None)] * 3, [slice(None)] * 3
        lo[axis], hi[axis] = slice(None, -1), slice(1, None)
        faces.append(np.column_stack((ids[tuple(lo)].ravel(), ids[tuple(hi)].ravel())))
        for side in (0, -1):
            sel = [slice(None)] * 3
            sel[axis] = side
            cells = ids[tuple(sel)].ravel()
            faces.append(np.column_stack((cells, np.full(len(cells), -1))))
    faces = np.concatenate(faces)
    return pos, faces, np.full(len(faces), spacing**2)


def quadratic(points):
    """The manufactured pressure of the reference's test (``tests/test_ib_postprocess.py:44-46``)."""
    x, y, z = np.asarray(points).T
    return 1.3 + 0.2 * x - 0.5 * y + 0.7 * z + 0.4 * x * x - 0.2 * y * y + 0.3 * z * z + 0.1 * x * y


def quadratic_gradient(points):
    """Its gradient (``tests/test_ib_postprocess.py:49-51``)."""
    x, y, z = np.asarray(points).T
    return np.column_stack((0.2 + 0.8 * x + 0.1 * y, -0.5 - 0.4 * y + 0.1 * x, 0.7 + 0.6 * z))


def lattice_edges(shape, valid):
    """Edges between axis neighbours that are both valid, axis by axis
    (``ib_postprocess.py:200-210``): first cell, second cell, axis."""
    ids = np.arange(int(np.prod(shape))).reshape(shape)
    out = [[], [], []]
    for axis in range(3):
        lo, hi = [slice(None)] * 3, [slice(None)] * 3
        lo[axis], hi[axis] = slice(None, -1), slice(1, None)
        a, b = ids[tuple(lo)].ravel(), ids[tuple(hi)].ravel()
        keep = valid.ravel()[a] & valid.ravel()[b]
        out[0].append(a[keep])
        out[1].append(b[keep])
        out[2].append(np.full(int(keep.sum()), axis))
    return tuple(np.concatenate(v) for v in out)


def repair_pressure_band(shape, spacing, raw_pressure, regular_gradient, signed_distance, width=1.5):
    """The reference's band repair (``ib_postprocess.py:213-250``); returns
    (repaired, target, lsqr iterations)."""
    target = (signed_distance >= 0) & (signed_distance <= width * spacing) & np.isfinite(raw_pressure)
    valid = (signed_distance >= 0) & np.isfinite(raw_pressure)
    first, second, axes = lattice_edges(shape, valid)
    sel = target.ravel()[first] | target.ravel()[second]
    first, second, axes = first[sel], second[sel], axes[sel]
    ids = np.flatnonzero(target.ravel())
    if not len(ids):
        raise ValueError("pressure repair band contains no cells; refine the grid")
    local = np.full(target.size, -1)
    local[ids] = np.arange(len(ids))
    g = regular_gradient.reshape(-1, 3)
    rhs = 0.5 * spacing * (g[first, axes] + g[second, axes])
    raw = raw_pressure.ravel()
    rows, cols, vals = [], [], []
    for sign, cells in ((-1.0, first), (1.0, second)):
        inside = local[cells] >= 0
        rows.append(np.flatnonzero(inside))
        cols.append(local[cells[inside]])
        vals.append(np.full(int(inside.sum()), sign))
        rhs[~inside] -= sign * raw[cells[~inside]]
    B = coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                   shape=(len(first), len(ids))).tocsr()
    count, labels = connected_components((B.T @ B).tocsr(), directed=False)
    anchors = np.zeros(len(ids), dtype=bool)
    for a, b in ((first, second), (second, first)):
        hit = (local[a] >= 0) & (local[b] < 0)
        anchors[local[a[hit]]] = True
    if len(np.unique(labels[anchors])) != count:
        raise ValueError("pressure repair has an unanchored band; enlarge the finest region")
    sol = lsqr(B, rhs, atol=1e-11, btol=1e-11, iter_lim=max(500, 20 * len(ids)))
    if sol[1] not in (0, 1, 2, 4, 5) or not np.isfinite(sol[0]).all():
        raise RuntimeError(f"pressure band solve failed (status {sol[1]})")
    out = raw.copy()
    out[ids] = sol[0]
    return out.reshape(shape), target, int(sol[2])


def band_case(count=17, spacing=0.25, radius=0.6, noise=0.0, seed=0, holes=0.0):
    """Lattice inputs of the reference's band test (``tests/test_ib_postprocess.py:86-95``):
    a count^3 block centred on the origin, the signed distance to a sphere of
    ``radius``, the quadratic truth, a raw pressure with the defect
    ``0.8 cos(x)`` on the band, and the quadratic's gradient; ``noise`` adds a
    seeded normal perturbation to the gradient so that the band's equations are
    inconsistent, and ``holes`` sets that fraction of the raw values (seeded)
    to NaN, cells the repair must leave out.  Returns (positions, distance,
    truth, raw, gradient), the
    lattice arrays shaped (count, count, count[, 3])."""
    shape = (count,) * 3
    axes = (np.arange(count) - 0.5 * (count - 1)) * spacing
    pos = np.stack(np.meshgrid(axes, axes, axes, indexing="ij"), axis=-1)
    flat = pos.reshape(-1, 3)
    distance = (np.linalg.norm(flat, axis=1) - radius).reshape(shape)
    truth = quadratic(flat).reshape(shape)
    band = (distance >= 0) & (distance <= 1.5 * spacing)
    raw = truth.copy()
    raw[band] += 0.8 * np.cos(pos[band, 0])
    grad = quadratic_gradient(flat)
    rng = np.random.default_rng(seed)
    if noise:
        grad = grad + noise * rng.standard_normal(grad.shape)
    if holes:
        raw[rng.random(shape) < holes] = np.nan
    return pos, distance, truth, raw, grad.reshape(shape + (3,))
