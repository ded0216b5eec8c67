"""CPU oracle: a NumPy restatement of PyIB's per-step hot path (test infrastructure only).

THIS MODULE IS THE CHECKER, NOT THE PRODUCT.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
it.  The B200 path never calls it and must fail loudly when its CUDA library is
missing.

It restates, in float64, the algorithms of the reference (paths relative to
``src/pyib/solver`` of XuZhaoyue1995/gpu-ib-code-paper-2026-08-snapshot):

* geometry and incidence operators  -- ``ib_core_np.py:24-183``
* diagonal preconditioner           -- ``ib_driver_np.py:78-88``
* ghost-cell velocity, convection/diffusion, PCG with the mixed stopping test
  and the Crank-Nicolson/Picard step with accumulated explicit IB forcing
                                     -- ``ib_driver_np.py:260-532``
* Roma-Peskin 3-point delta, 5^3 stencil, interpolation, spreading, direct
  forcing                           -- ``ib_immersed.py:12-120``
* prescribed oscillation            -- ``ib_kinematics.py:17-40``
* closed-sphere load correction     -- ``ib_interior.py:57-70, 116-308``

The mesh is passed as a plain description (see :class:`MeshDesc`): nodes,
face->cell, face->edge (4 per face) plus extra face/edge links, edge->node,
boundary families, and the finest-level structured cell index.  The same
description can come from the reference's own mesh builder (golden fixtures)
or from the product's layout export, which is how the two are compared.

Parity pin: ``tests/test_oracle_golden.py`` checks every function here
against fixtures produced by running the unmodified reference
(``tests/golden/make_golden.py``).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


# ---------------------------------------------------------------------------
# mesh description
# ---------------------------------------------------------------------------
@dataclass
class MeshDesc:
    nodes: np.ndarray            # (nn,3) float64
    F2C: np.ndarray              # (nf,2) int64, second column -1 on boundary faces
    F2E: np.ndarray              # (nf,4) int64
    E2N: np.ndarray              # (ne,2) int64
    link_fe_insert: np.ndarray   # (K,2) int64 extra (face, edge) links
    bc_edge: np.ndarray          # (ne,) boundary family 0..6
    bc_face: np.ndarray          # (nf,) boundary family 0..6
    ncell: int
    index_cell: np.ndarray       # (nx,ny,nz) finest-level cell ids
    pos_ref: np.ndarray          # (3,) centre of finest cell (0,0,0)
    dx: float                    # finest spacing

    @staticmethod
    def from_npz(d, prefix="mesh_"):
        g = lambda k: np.asarray(d[prefix + k])
        return MeshDesc(nodes=g("nodes").astype(np.float64), F2C=g("F2C").astype(np.int64),
                        F2E=g("F2E").astype(np.int64), E2N=g("E2N").astype(np.int64),
                        link_fe_insert=g("link_fe_insert").astype(np.int64).reshape(-1, 2),
                        bc_edge=g("bc_edge").astype(np.int64), bc_face=g("bc_face").astype(np.int64),
                        ncell=int(g("ncell")), index_cell=g("index_cell").astype(np.int64),
                        pos_ref=g("pos_ref").astype(np.float64), dx=float(g("dx")))


def _scatter(index, values, n):
    """Sum ``values`` into ``n`` bins by ``index`` (works for 1-D and 2-D values)."""
    values = np.asarray(values, dtype=np.float64)
    if values.ndim == 1:
        return np.bincount(index, weights=values, minlength=n)
    out = np.zeros((n,) + values.shape[1:])
    np.add.at(out, index, values)
    return out


# ---------------------------------------------------------------------------
# geometry + incidence operators  (ib_core_np.py:24-183)
# ---------------------------------------------------------------------------
class Geometry:
    """Face/edge/cell geometry with the 2:1 hanging-node corrections.

    Follows ib_core_np.py:36-121: link list = 4 base links per face plus the
    extra links (39-41); edge centres/tangents (44-45); face and cell centres
    as means of their edges/faces (46-53); link signs from (epos-fpos) x te
    against rf (64-67); area vectors (68-72); then the interface centre
    corrections at |r|^2 = 0.36 Af and 4/9 Af (74-102), vol_ci (104-108) and
    AoL (110-111).
    """

    def __init__(self, m: MeshDesc):
        self.m = m
        F2C, F2E, E2N = m.F2C, m.F2E, m.E2N
        nf, ne, nc = F2C.shape[0], E2N.shape[0], m.ncell
        self.nface, self.nedge, self.ncell = nf, ne, nc
        internal = F2C[:, 1] >= 0
        self.m1 = internal
        extra = m.link_fe_insert.reshape(-1, 2)
        self.lf_face = np.concatenate([np.repeat(np.arange(nf), 4), extra[:, 0]])
        self.lf_edge = np.concatenate([F2E.reshape(-1), extra[:, 1]])
        lf, le = self.lf_face, self.lf_edge

        x = m.nodes
        self.epos = epos = 0.5 * (x[E2N[:, 0]] + x[E2N[:, 1]])
        self.te = te = x[E2N[:, 1]] - x[E2N[:, 0]]
        nlinks = np.bincount(lf, minlength=nf).astype(np.float64)
        fpos = _scatter(lf, epos[le], nf) / nlinks[:, None]

        c1 = F2C[:, 0]
        c2 = F2C[internal, 1]

        def cell_centres(fp):
            num = _scatter(c1, fp, nc) + _scatter(c2, fp[internal], nc)
            cnt = np.bincount(c1, minlength=nc) + np.bincount(c2, minlength=nc)
            return num / cnt[:, None].astype(np.float64)

        cpos = cell_centres(fpos)
        rf = np.empty((nf, 3))
        rf[internal] = cpos[F2C[internal, 1]] - cpos[F2C[internal, 0]]
        rf[~internal] = fpos[~internal] - cpos[F2C[~internal, 0]]
        arm = np.cross(epos[le] - fpos[lf], te[le])
        sgn = np.sign(np.einsum("ij,ij->i", arm, rf[lf]))
        sgn[sgn == 0] = 1.0
        self.fe_sign_link = sgn
        nvec = _scatter(lf, arm * sgn[:, None], nf) * 0.5      # 1/(ND-1), ND=3
        self.nf = nvec
        self.Af = Af = np.sqrt(np.einsum("ij,ij->i", nvec, nvec))

        # interface corrections (Modify_geom)
        tol = 1e-6 * Af
        arm_r = epos[le] - fpos[lf]
        hit = np.abs(np.einsum("ij,ij->i", arm_r, arm_r) - 0.36 * Af[lf]) < tol[lf]
        fpos = fpos.copy()
        np.add.at(fpos, lf[hit], arm_r[hit] / 6.0)
        cpos = cell_centres(fpos)
        r1 = fpos - cpos[c1]
        r2 = np.zeros((nf, 3))
        r2[internal] = fpos[internal] - cpos[F2C[internal, 1]]
        a49 = Af * (4.0 / 9.0)
        hit1 = np.abs(np.einsum("ij,ij->i", r1, r1) - a49) < tol
        np.add.at(cpos, c1[hit1], r1[hit1] * 0.25)
        hit2 = (~hit1) & internal & (np.abs(np.einsum("ij,ij->i", r2, r2) - a49) < tol)
        np.add.at(cpos, F2C[hit2, 1], r2[hit2] * 0.25)
        self.fpos, self.cpos = fpos, cpos
        self.rf1 = fpos - cpos[c1]
        self.rf2 = np.zeros((nf, 3))
        self.rf2[internal] = fpos[internal] - cpos[F2C[internal, 1]]
        self.rf = self.rf1 - self.rf2

        vraw = _scatter(c1, np.einsum("ij,ij->i", nvec, self.rf1), nc) \
            - _scatter(c2, np.einsum("ij,ij->i", nvec[internal], self.rf2[internal]), nc)
        self.vol_ci = np.where(np.abs(vraw) > 1e-14, 3.0 / np.where(vraw == 0, 1.0, vraw), 0.0)
        self.AoL = np.einsum("ij,ij->i", self.rf, nvec) / np.einsum("ij,ij->i", self.rf, self.rf)
        self.F2C = F2C

    # ---- operators -----------------------------------------------------
    def rot(self, face):                       # ib_core_np.py:129-131
        return _scatter(self.lf_edge, self.fe_sign_link * face[self.lf_face], self.nedge)

    def curl(self, edge):                      # ib_core_np.py:133-134
        return _scatter(self.lf_face, self.fe_sign_link * edge[self.lf_edge], self.nface)

    def cdiv(self, face):                      # ib_core_np.py:136-139
        m1 = self.m1
        return _scatter(self.F2C[:, 0], face, self.ncell) - _scatter(self.F2C[m1, 1], face[m1], self.ncell)

    def integr_c2f(self, cv):                  # ib_core_np.py:144-148
        out = np.einsum("ij,ij->i", cv[self.F2C[:, 0]], self.rf1)
        m1 = self.m1
        out[m1] -= np.einsum("ij,ij->i", cv[self.F2C[m1, 1]], self.rf2[m1])
        return out

    def interp_f2c(self, face):                # ib_core_np.py:150-157
        m1 = self.m1
        out = _scatter(self.F2C[:, 0], face[:, None] * self.rf1, self.ncell) \
            - _scatter(self.F2C[m1, 1], face[m1][:, None] * self.rf2[m1], self.ncell)
        return out * self.vol_ci[:, None]

    def cgrad0(self, cell):                    # ib_core_np.py:177-183
        m1 = self.m1
        out = -cell[self.F2C[:, 0]]
        out[m1] += cell[self.F2C[m1, 1]]
        return out

    def flow_mat(self, p, alpd=0.0, visc=0.0, rou=1.0, dt=0.0):   # ib_core_np.py:168-175
        v = self.interp_f2c(self.curl(p))
        if alpd != 0.0:
            for k in range(3):
                q = self.AoL * visc * self.cgrad0(v[:, k])
                v[:, k] = rou * v[:, k] - 0.5 * dt * self.vol_ci * self.cdiv(q)
        return self.rot(self.integr_c2f(v))


def diag_preconditioner(g: Geometry, dir_mask):
    """ib_driver_np.py:78-88: 1 / sum over a edge's faces of (rf.nf)/Af^2."""
    q = np.einsum("ij,ij->i", g.rf, g.nf) / (g.Af * g.Af)
    d = _scatter(g.lf_edge, np.abs(g.fe_sign_link) * q[g.lf_face], g.nedge)
    d[dir_mask] = 0.0
    out = np.zeros(g.nedge)
    nz = d != 0.0
    out[nz] = 1.0 / d[nz]
    return out


# ---------------------------------------------------------------------------
# immersed boundary  (ib_immersed.py:12-120)
# ---------------------------------------------------------------------------
def delta_h3(r, h):
    """Roma-Peskin three-point kernel, ib_immersed.py:12-19."""
    a = np.abs(r / h)
    inner = (1.0 + np.sqrt(np.clip(1.0 - 3.0 * a * a, 0.0, None))) / (3.0 * h)
    outer = (5.0 - 3.0 * a - np.sqrt(np.clip(1.0 - 3.0 * (1.0 - a) ** 2, 0.0, None))) / (6.0 * h)
    return np.where(a <= 0.5, inner, np.where(a <= 1.5, outer, 0.0))


class IBStencil:
    """5^3 support cells and weights, ib_immersed.py:63-81 (no cache)."""

    def __init__(self, m: MeshDesc, hh=None):
        self.index_cell = m.index_cell
        self.n = np.asarray(m.index_cell.shape)
        self.pos_ref = np.asarray(m.pos_ref, dtype=np.float64)
        self.dx = float(m.dx)
        self.hh = float(self.dx if hh is None else hh)
        self.ncell = m.ncell
        o = np.arange(-2, 3)
        oi, oj, ok = np.meshgrid(o, o, o, indexing="ij")
        self.off = np.stack([oi.ravel(), oj.ravel(), ok.ravel()], axis=1)   # (125,3)

    def base_index(self, markers):
        return np.rint((markers - self.pos_ref) / self.dx).astype(np.int64)

    def build(self, markers):
        base = self.base_index(markers)
        ijk = base[:, None, :] + self.off[None, :, :]                     # (M,125,3)
        n = self.n
        inside = np.all((ijk >= 0) & (ijk < n), axis=2)
        cl = np.clip(ijk, 0, n - 1)
        cell = self.index_cell[cl[..., 0], cl[..., 1], cl[..., 2]]
        ok = inside & (cell >= 0)
        w = np.ones(ok.shape)
        for d in range(3):
            gd = self.pos_ref[d] + ijk[..., d] * self.dx - markers[:, d:d + 1]
            w = w * delta_h3(gd, self.hh) if d else delta_h3(gd, self.hh)
        w = np.where(ok, w, 0.0)
        cell = np.where(ok, cell, 0)
        return cell, w

    def interp(self, vc, stencil):             # ib_immersed.py:87-93
        cell, w = stencil
        ww = w * self.hh ** 3
        return np.stack([(vc[cell, c] * ww).sum(axis=1) for c in range(vc.shape[1])], axis=1)

    def spread(self, f, stencil, ds):          # ib_immersed.py:103-111
        cell, w = stencil
        ww = w * (np.asarray(ds) ** 3)[:, None]
        flat = cell.ravel()
        return np.stack([np.bincount(flat, weights=(f[:, c:c + 1] * ww).ravel(), minlength=self.ncell)
                         for c in range(f.shape[1])], axis=1)

    def direct_force(self, vc, markers, vel, dt, ds):     # ib_immersed.py:113-120
        st = self.build(markers)
        fl = (vel - self.interp(vc, st)) / dt
        return self.spread(fl, st, ds), fl

    def coupling_matrix(self, stencil, ds, reg=1e-8):
        """M = D S + reg tr(M)/nmk I, ib_immersed.py:122-146.

        D[i, c] = sum_k w_ik hh^3 [cell_ik = c] (interpolation), S[c, j] = sum_k
        w_jk ds_j^3 [cell_jk = c] (spreading); dense nmk x nmk.
        """
        import scipy.sparse as sp
        cell, w = stencil
        nmk = cell.shape[0]
        rows = np.repeat(np.arange(nmk), cell.shape[1])
        cols = cell.ravel()
        D = sp.csr_matrix(((w * self.hh ** 3).ravel(), (rows, cols)), shape=(nmk, self.ncell))
        S = sp.csr_matrix(((w * (np.asarray(ds) ** 3)[:, None]).ravel(), (cols, rows)), shape=(self.ncell, nmk))
        M = np.asarray((D @ S).todense())
        M += reg * np.trace(M) / nmk * np.eye(nmk)
        return M

    def implicit_force(self, vc, markers, vel, dt, ds):   # ib_immersed.py:154-174
        """Solve M f = (vel - interp(vc))/dt with the coupling matrix; F_E = spread(f)."""
        st = self.build(markers)
        rhs = (vel - self.interp(vc, st)) / dt
        f = np.linalg.inv(self.coupling_matrix(st, ds)) @ rhs
        return self.spread(f, st, ds), f


# ---------------------------------------------------------------------------
# kinematics and closed-sphere loads
# ---------------------------------------------------------------------------
def fibonacci_sphere(count, radius, centre):
    """Fibonacci-lattice markers, ib_case.py:554-563."""
    k = np.arange(count, dtype=np.float64)
    polar = np.arccos(1.0 - 2.0 * (k + 0.5) / count)
    azim = np.pi * (1.0 + np.sqrt(5.0)) * k
    u = np.stack([np.sin(polar) * np.cos(azim), np.sin(polar) * np.sin(azim), np.cos(polar)], axis=1)
    return np.asarray(centre, dtype=np.float64) + radius * u


class Oscillation:
    """x(t) = ref + A sin(2 pi f t + phase) axis, ib_kinematics.py:17-40."""

    def __init__(self, ref, axis, A, freq, phase=0.0):
        ax = np.asarray(axis, dtype=np.float64)
        self.axis = ax / np.linalg.norm(ax)
        self.ref = np.asarray(ref, dtype=np.float64)
        self.A, self.freq, self.phase = float(A), float(freq), float(phase)

    def __call__(self, t):
        om = 2.0 * np.pi * self.freq
        disp = self.A * np.sin(om * t + self.phase) * self.axis
        vel = self.A * om * np.cos(om * t + self.phase) * self.axis
        return self.ref + disp, np.tile(vel, (self.ref.shape[0], 1))


class SphereLoads:
    """ClosedSphereLoadCorrection restated (ib_interior.py:57-70, 116-308)."""

    def __init__(self, cpos, vol, centre0, max_translation, radius, width, density, support):
        self.pos, self.vol = cpos, vol
        hw = radius + 0.5 * width + np.abs(max_translation)
        sel = np.all((cpos >= centre0 - hw) & (cpos <= centre0 + hw), axis=1)
        self.cand = np.nonzero(sel)[0]
        fw = radius + support + np.abs(max_translation)
        fw = fw + 8.0 * np.finfo(np.float64).eps * np.maximum(1.0, np.abs(centre0) + fw)
        fsel = np.all((cpos >= centre0 - fw) & (cpos <= centre0 + fw), axis=1)
        self.fidx = np.nonzero(fsel)[0]
        self.radius, self.width, self.rho = radius, width, density
        self.fixed = bool(np.all(np.asarray(max_translation) == 0.0))
        self.centre0 = np.asarray(centre0, dtype=np.float64)
        self.current = None

    def _weights(self, centre):
        p = self.pos[self.cand]
        d = np.linalg.norm(p - (self.centre0 if self.fixed else centre), axis=1)
        ind = np.clip((self.radius + 0.5 * self.width - d) / self.width, 0.0, 1.0)
        return ind * self.vol[self.cand]

    def evaluate(self, vc, centre):
        w = self._weights(centre)
        v = vc[self.cand]
        p = self.pos[self.cand]
        lin = self.rho * (v * w[:, None]).sum(axis=0)
        ang = self.rho * (np.cross(p, v) * w[:, None]).sum(axis=0)
        return lin, ang, w.sum()

    def initialize(self, vc, centre):
        self.current = self.evaluate(vc, centre)

    def advance(self, vc, centre, dt, fE):
        prev = self.current
        cur = self.evaluate(vc, centre)
        lrate = (cur[0] - prev[0]) / dt
        arate = (cur[1] - prev[1]) / dt
        f = fE[self.fidx]
        p = self.pos[self.fidx]
        v = self.vol[self.fidx]
        ff = (f * v[:, None]).sum(axis=0)
        mf = (np.cross(p, f) * v[:, None]).sum(axis=0)
        self.current = cur
        return dict(force_fluid=ff, moment_fluid=mf, body_force=-ff + lrate,
                    body_moment=-mf + arate, linear_momentum=cur[0],
                    angular_momentum=cur[1], indicator_volume=cur[2],
                    linear_rate=lrate, angular_rate=arate)


# ---------------------------------------------------------------------------
# driver  (ib_driver_np.py:104-532)
# ---------------------------------------------------------------------------
@dataclass
class SolveStats:
    iterations: int = 0
    rel_residual: float = 0.0
    tol_ratio: float = 0.0
    converged: bool = True


class OracleDriver:
    """Crank-Nicolson stream-function stepper with IB forcing (float64)."""

    def __init__(self, m: MeshDesc, visc, rou=1.0, ac=0.5, ad=0.5, cavity=False,
                 cg_check_interval=20, cg_max_iterations=1000, geometry=None):
        self.m = m
        self.g = g = geometry if geometry is not None else Geometry(m)
        self.visc, self.rou, self.ac, self.ad = float(visc), float(rou), ac, ad
        self.bf = np.nonzero(~g.m1)[0]
        self.nghost = self.bf.size
        self.ghost_of = np.full(g.nface, -1, dtype=np.int64)
        self.ghost_of[self.bf] = g.ncell + np.arange(self.nghost)
        self.F2C_ext = g.F2C.copy()
        self.F2C_ext[self.bf, 1] = self.ghost_of[self.bf]
        self.bf_fam = m.bc_face[self.bf]
        self.cavity = bool(cavity)
        if cavity:                                       # ib_driver_np.py:155-177 (U_lid=0, 6 walls)
            self.inlet = np.zeros(g.nedge, dtype=bool)
            self.dir_mask = m.bc_edge > 0
        else:                                            # ib_driver_np.py:120-121
            self.inlet = m.bc_edge == 1
            self.dir_mask = np.isin(m.bc_edge, [3, 4, 5, 6])
        self.prec = diag_preconditioner(g, self.dir_mask)
        self.check = int(cg_check_interval)
        self.cg_max = int(cg_max_iterations)
        self.ib = None
        self.motion = None
        self.time = 0.0
        self.last_stats = []

    # -- IB wiring (ib_driver_np.py:179-201, 241-249)
    def set_ib(self, stencil: IBStencil, markers, ds, vel, force_mode="accumulated_explicit", implicit=False,
               alpha=1.0):
        """force_mode: "accumulated_explicit" (ib_driver_np.py:447-451, 511-525) or
        "replacement" (the public "direct": the force of every inner iteration replaces
        the last one, scaled by alpha, explicit or implicit, ib_driver_np.py:466-486)."""
        if force_mode not in ("accumulated_explicit", "replacement"):
            raise ValueError(force_mode)
        self.force_mode, self.implicit, self.alpha = force_mode, bool(implicit), float(alpha)
        self.ib = stencil
        self.markers = np.asarray(markers, dtype=np.float64)
        self.ds = np.asarray(ds, dtype=np.float64)
        self.vel = np.asarray(vel, dtype=np.float64)
        self.fE = np.zeros((self.g.ncell, 3))
        self.fL = np.zeros_like(self.vel)

    def set_motion(self, motion, t0=0.0):
        self.motion = motion
        self.time = float(t0)

    # -- velocity with ghosts (ib_driver_np.py:267-291)
    def calc_vel(self, s):
        g = self.g
        s = s.copy()
        s[self.inlet] = g.epos[self.inlet, 1] * g.te[self.inlet, 2]
        U = g.curl(s)
        vc = np.zeros((g.ncell + self.nghost, 3))
        vc[:g.ncell] = g.interp_f2c(U)
        bf = self.bf
        inner = vc[g.F2C[bf, 0]]
        gh = self.ghost_of[bf]
        if self.cavity:
            vc[gh] = -inner
            return s, U, vc
        n = g.nf[bf]
        a2 = (g.Af[bf] ** 2)[:, None]
        ub = U[bf][:, None]
        inl = self.bf_fam == 1
        vals = inner + (ub - np.sum(inner * n, axis=1, keepdims=True)) * n / a2
        vals[inl] = (ub * n / a2)[inl]
        vc[gh] = vals
        return s, U, vc

    # -- central convection + diffusion (ib_driver_np.py:293-303)
    def conv_diff(self, U, vc):
        g = self.g
        a, b = self.F2C_ext[:, 0], self.F2C_ext[:, 1]
        conv = np.empty((g.ncell, 3))
        diff = np.empty((g.ncell, 3))
        for j in range(3):
            col = vc[:, j]
            grad = col[b] - col[a]
            diff[:, j] = g.vol_ci * g.cdiv(g.AoL * self.visc * grad)
            avg = col[a] * (0.5 * U) + col[b] * (0.5 * U)
            conv[:, j] = g.vol_ci * g.cdiv(avg)
        return conv, diff

    def apply(self, p, dt):
        return self.g.flow_mat(p, alpd=self.ad, visc=self.visc, rou=self.rou, dt=dt)

    # -- PCG with the mixed criterion (ib_driver_np.py:311-410)
    def helm_solve(self, res_e, s, dt, tol1=1e-10, tol2=1e-9, cg_max=None):
        cg_max = self.cg_max if cg_max is None else int(cg_max)
        dm = self.dir_mask
        r = res_e.copy()
        r[dm] = 0.0
        l2_0 = r.dot(r)
        x = s.copy()
        p = r * self.prec
        eta = p.dot(r)
        eta0 = eta
        thresh = (x.dot(x) + 1e-16) * tol1 ** 2 + tol2 ** 2 * eta0
        m_done = 0
        if not eta < thresh:
            for m in range(1, cg_max + 1):
                w = self.apply(p, dt)
                w[dm] = 0.0
                den = p.dot(w)
                alpha = eta / (den if den != 0.0 else np.inf)
                x += alpha * p
                r -= alpha * w
                z = r * self.prec
                eta_new = z.dot(r)
                m_done = m
                if m % self.check == 0:
                    if not np.isfinite(eta_new) or eta_new < thresh:
                        break
                beta = eta_new / (eta if eta != 0.0 else np.inf)
                p = z + beta * p
                eta = eta_new
            true_r = res_e - self.apply(x - s, dt)
            true_r[dm] = 0.0
        else:
            true_r = r
        eta_f = (true_r * self.prec).dot(true_r)
        l2_f = true_r.dot(true_r)
        st = SolveStats(iterations=m_done)
        st.rel_residual = float(np.sqrt(l2_f / l2_0)) if l2_0 > 0 else (0.0 if l2_f == 0 else np.inf)
        st.tol_ratio = float(np.sqrt(eta_f / thresh)) if thresh > 0 else (0.0 if eta_f == 0 else np.inf)
        st.converged = bool(np.isfinite(eta_f) and eta_f <= thresh)
        return x, st

    # -- one time step, accumulated explicit forcing (ib_driver_np.py:412-532)
    def step(self, s, s_old, dt, dt_old, inner=4):
        g = self.g
        nc = g.ncell
        rou, ac, ad = self.rou, self.ac, self.ad
        self.time += dt
        stats = []
        accumulated = self.ib is None or self.force_mode == "accumulated_explicit"
        if self.ib is not None and self.motion is not None:
            self.markers, self.vel = self.motion(self.time)
            if accumulated:
                st = self.ib.build(self.markers)
                self.fE = self.ib.spread(self.fL, st, self.ds)
        _, U, vc = self.calc_vel(s)
        conv0, diff0 = self.conv_diff(U, vc)
        res0 = rou * vc[:nc] - (1 - ac) * dt * rou * conv0 + (1 - ad) * dt * diff0
        prev = s.copy()
        s = s + (s - s_old) * dt / dt_old
        s, U, vc = self.calc_vel(s)
        s_old = prev
        self.last_res = None
        for it in range(1, inner + 1):
            conv, diff = self.conv_diff(U, vc)
            res = res0 - rou * vc[:nc] - ac * dt * rou * conv + ad * dt * diff
            if self.ib is not None:
                if not accumulated:
                    # the force of this inner iteration replaces the last (ib_driver_np.py:466-486)
                    force = self.ib.implicit_force if self.implicit else self.ib.direct_force
                    fE, fL = force(vc[:nc], self.markers, self.vel, dt, self.ds)
                    self.fE = (rou * self.alpha) * fE
                    self.fL = (rou * self.alpha) * fL
                res = res + dt * self.fE
            if it == inner:
                self.last_res = res
            res_e = g.rot(g.integr_c2f(res))
            s, st = self.helm_solve(res_e, s, dt)
            stats.append(st)
            s, U, vc = self.calc_vel(s)
            if self.ib is not None and accumulated and it == 1:
                dE, dL = self.ib.direct_force(vc[:nc], self.markers, self.vel, dt, self.ds)
                self.fE = self.fE + rou * dE
                self.fL = self.fL + rou * dL
        self.last_U = U
        self.last_stats = stats
        return s, vc, s_old
