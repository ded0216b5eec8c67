"""Discrete adjoint of the time step and the gradient of the sphere's force amplitude.

The forward model is the step of ``Driver.step`` (``ib_driver_np.py:412-532``) for
the closed-cavity oscillating sphere with accumulated explicit forcing, restated
on the GPU as a composition of differentiable pieces, each a
``torch.autograd.Function`` with a hand-written backward:

* ``SparseOp``: a constant linear operator of the step -- curl, interp_f2c,
  integr_c2f, rot (``ib_core_np.py:129-157``) -- applied as a CSR product; its
  backward applies the transposed operator, assembled once on the host;
* ``ConvDiff``: the central convection and the diffusion of ``Driver.conv_diff``
  (``ib_driver_np.py:293-303``) with the cavity's no-slip ghost cells
  (``ib_driver_np.py:276-284``); its backward is the transposed linearisation
  about the forward state (the convective flux is bilinear in U and vc);
* ``HelmSolve``: ``helm_solve`` (``ib_driver_np.py:311-410``) on the device PCG;
  A is symmetric, so its backward is a solve with the same operator (after a
  projection that makes the singular system consistent, see ``CavityModel.pinv``);
* ``MarkerInterp`` / ``MarkerSpread``: interpolation and spreading
  (``ib_immersed.py:87-111``) with the weights as an input, so that gradients
  reach the marker positions through the Roma-Peskin kernel; spreading and the
  interpolation's transpose run the library's deterministic sort-and-sum
  spreading (``pyib_spread_noalloc``), so repeated runs give the same bits.

The closed-sphere loads (``ib_interior.py:57-70, 268-308``) and the objective --
the first-harmonic amplitude of the axial body force over the last period,
fitted as ``tools/check_pressure_validation.py:31-37`` does -- are plain torch
expressions.  ``force_amplitude_and_gradient`` runs the steps forward, then
reverses them with binomial checkpointing (at most ``snapshots`` stored
states, recomputing forward segments from them), and returns the gradient
with respect to the oscillation amplitude A, the period T and the reference
marker positions.  The physical viscosity, density and time step are held at
their nominal values: A and T enter through the prescribed motion, its
velocity, the interior-momentum indicator's centre and the harmonic fit.

Every solve, product and spreading runs on the device through the library;
without it ``CavityModel`` fails on construction.  (The CPU tests check the
same model with a NumPy mirror of the device PCG and of the spreading, a
subclass that lives with the tests.)
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np
import scipy.sparse as sp
import torch

from . import _lib
from .cases import R as SPHERE_RADIUS
from .device import DeviceSolver


def _csr_tensor(M, device):
    M = M.tocsr()
    M.sum_duplicates()
    return torch.sparse_csr_tensor(torch.from_numpy(M.indptr.astype(np.int64)),
                                   torch.from_numpy(M.indices.astype(np.int64)),
                                   torch.from_numpy(M.data.astype(np.float64)),
                                   size=M.shape, dtype=torch.float64, device=device)


class _Pair:
    """A sparse operator and its transpose on the device."""

    def __init__(self, M, device):
        self.M = _csr_tensor(M, device)
        self.MT = _csr_tensor(M.T, device)


class SparseOp(torch.autograd.Function):
    """y = M x (x a vector or a matrix of columns); backward: M^T g."""

    @staticmethod
    def forward(ctx, x, op):
        ctx.op = op
        return op.M @ x

    @staticmethod
    def backward(ctx, g):
        return ctx.op.MT @ g.contiguous(), None


class ConvDiff(torch.autograd.Function):
    """conv, diff (both (NC, 3)) of the face flux U and the cell velocity vc (NC, 3).

    With the cavity's ghost values folded in (ghost = -interior, so a wall face
    carries no convective flux and twice the interior value in the gradient):
        conv_d = vol * K (U/2 * (LH vc_d)),   diff_d = vol * K (aolv * (HL vc_d))
    K is the signed cell-face incidence (cdiv), LH sums the two cells of a face,
    HL differences them, aolv = AoL * visc.
    """

    @staticmethod
    def forward(ctx, U, vc, ops):
        ctx.ops = ops
        hU = 0.5 * U
        avg = ops.LH.M @ vc                        # (NF, 3)
        jump = ops.HL.M @ vc
        conv = ops.vol[:, None] * (ops.K.M @ (hU[:, None] * avg))
        diff = ops.vol[:, None] * (ops.K.M @ (ops.aolv[:, None] * jump))
        ctx.save_for_backward(hU, avg)
        return conv, diff

    @staticmethod
    def backward(ctx, g_conv, g_diff):
        ops = ctx.ops
        hU, avg = ctx.saved_tensors
        hc = ops.K.MT @ (ops.vol[:, None] * g_conv).contiguous()     # (NF, 3)
        hd = ops.K.MT @ (ops.vol[:, None] * g_diff).contiguous()
        g_U = 0.5 * (avg * hc).sum(dim=1)
        g_vc = ops.LH.MT @ (hU[:, None] * hc).contiguous() + ops.HL.MT @ (ops.aolv[:, None] * hd).contiguous()
        return g_U, g_vc, None


class HelmSolve(torch.autograd.Function):
    """x = s + A+ res on the free edges (x = s elsewhere), by the device PCG.

    In the closed cavity A is singular: its null space holds the gradients of
    node fields and, at level interfaces, face-flux patterns that interpolate to
    zero cell velocity.  PCG from a zero correction with the diagonal
    preconditioner M returns the M-weighted pseudo-inverse
    A+ = M^1/2 (M^1/2 A M^1/2)^+ M^1/2, a symmetric map, so the backward applies
    the same A+ to the incoming gradient.  That gradient need not lie in the range
    of A, and PCG on an inconsistent system diverges; ``CavityModel.pinv`` first
    projects it with a cell-space solve and then solves a consistent system.
    """

    @staticmethod
    def forward(ctx, res_e, s, model):
        ctx.model = model
        return model.solve(res_e, s)

    @staticmethod
    def backward(ctx, g):
        m = ctx.model
        return m.pinv(g * m.free), g, None


def _spread(model, cells32, w, ds3, f):
    """out (NC, 3) = sum over contributions of f[m] * w * ds3[m] (``model.spread``)."""
    return model.spread(cells32, w, ds3, f)


def _spread_device(model, cells32, w, ds3, f):
    """The library's deterministic sort-and-sum spreading (``pyib_spread_noalloc``)."""
    M = f.shape[0]
    out = torch.empty(3 * model.NC, dtype=torch.float64, device=f.device)
    fm = f.contiguous().reshape(-1)
    wm = w.contiguous().reshape(-1)
    d3 = ds3.contiguous()
    torch.cuda.synchronize(f.device)
    rc = model.lib.pyib_spread_noalloc(C.c_void_p(cells32.data_ptr()), C.c_void_p(wm.data_ptr()),
                                       C.c_void_p(d3.data_ptr()), C.c_void_p(fm.data_ptr()), int(M),
                                       int(model.NC), C.c_void_p(out.data_ptr()), None)
    if rc != _lib.OK:
        raise _lib.B200Error(rc, "pyib_spread_noalloc failed")
    return out.reshape(3, model.NC).t()


class MarkerSpread(torch.autograd.Function):
    """fE (NC, 3) = sum w ds^3 f over each marker's 125 cells; gradients for f and w."""

    @staticmethod
    def forward(ctx, f, w, cells, model):
        ctx.model = model
        ctx.save_for_backward(f, w, cells)
        return _spread(model, model.cells32(cells), w, model.ds3, f)

    @staticmethod
    def backward(ctx, g):
        f, w, cells = ctx.saved_tensors
        m = ctx.model
        gc = g[cells]                                           # (M, 125, 3)
        g_f = m.ds3[:, None] * (w[:, :, None] * gc).sum(dim=1)
        g_w = m.ds3[:, None] * (gc * f[:, None, :]).sum(dim=2)
        return g_f, g_w, None, None


class MarkerInterp(torch.autograd.Function):
    """u (M, 3) = sum w hh^3 vc[cell]; gradients for vc and w."""

    @staticmethod
    def forward(ctx, vc, w, cells, model):
        ctx.model = model
        ctx.save_for_backward(vc, w, cells)
        return model.hh3 * (w[:, :, None] * vc[cells]).sum(dim=1)

    @staticmethod
    def backward(ctx, g):
        vc, w, cells = ctx.saved_tensors
        m = ctx.model
        hh3 = torch.full((w.shape[0],), m.hh3, dtype=torch.float64, device=g.device)
        g_vc = _spread(m, m.cells32(cells), w, hh3, g)
        g_w = m.hh3 * (vc[cells] * g[:, None, :]).sum(dim=2)
        return g_vc, g_w, None, None


def delta_h3(r, h):
    """Roma-Peskin 3-point kernel (``ib_immersed.py:12-19``), differentiable in r.

    The square roots take their arguments only where their branch is selected,
    so no infinite derivative of a clipped root reaches the gradient.
    """
    a = torch.abs(r / h)
    m1 = a <= 0.5
    m2 = (a > 0.5) & (a <= 1.5)
    q1 = torch.where(m1, 1.0 - 3.0 * a * a, torch.ones_like(a))
    q2 = torch.where(m2, 1.0 - 3.0 * (1.0 - a) ** 2, torch.ones_like(a))
    inner = (1.0 + torch.sqrt(torch.clamp(q1, min=0.0))) / (3.0 * h)
    outer = (5.0 - 3.0 * a - torch.sqrt(torch.clamp(q2, min=0.0))) / (6.0 * h)
    return torch.where(m1, inner, torch.where(m2, outer, torch.zeros_like(a)))


def step_operators(lay, ops, visc, device, into=None):
    """The step's constant sparse operators on ``device`` (attributes of ``into``).

    Cop (curl), Rop (rot), Pop (interp_f2c, component-major rows), Iop
    (integr_c2f, component-major columns), K (cdiv), LH / HL (face sum and face
    jump of the two cells, with the closed cavity's ghost = -interior folded in),
    vol (vol_ci) and aolv (AoL * visc).
    """
    from types import SimpleNamespace
    o = into if into is not None else SimpleNamespace()
    NC, NF = lay.NC, lay.NF
    o.Cop = _Pair(ops.C, device)
    o.Rop = _Pair(ops.R, device)
    o.Pop = _Pair(sp.vstack([ops.P[0], ops.P[1], ops.P[2]]), device)
    o.Iop = _Pair(sp.hstack([ops.I[0], ops.I[1], ops.I[2]]), device)
    o.K = _Pair(ops.D, device)
    f = np.nonzero(lay.face_exists)[0]
    lo, hi = lay.face_lo[f], lay.face_hi[f]
    both, glo, ghi = (lo >= 0) & (hi >= 0), lo < 0, hi < 0
    rows = np.concatenate([f[both], f[both]])
    cols = np.concatenate([lo[both], hi[both]])
    o.LH = _Pair(sp.csr_matrix((np.ones(rows.size), (rows, cols)), shape=(NF, NC)), device)
    rows = np.concatenate([f[both], f[both], f[glo], f[ghi]])
    cols = np.concatenate([lo[both], hi[both], hi[glo], lo[ghi]])
    vals = np.concatenate([-np.ones(both.sum()), np.ones(both.sum()), 2.0 * np.ones(glo.sum()),
                           -2.0 * np.ones(ghi.sum())])
    o.HL = _Pair(sp.csr_matrix((vals, (rows, cols)), shape=(NF, NC)), device)
    o.vol = torch.from_numpy(ops.vol_ci).to(device)
    o.aolv = torch.from_numpy(ops.AoL * visc).to(device)
    o.NC, o.NF, o.NE = lay.NC, lay.NF, lay.NE
    return o


class CavityModel:
    """The differentiable step of one closed-cavity oscillating-sphere case.

    ``case`` is a :class:`pyib_b200.cases.SphereCase` (closed cavity, prescribed
    oscillation); ``tol`` is the PCG's mixed stopping tolerance (tol1, and tol2
    unless given), tighter than the reference's 1e-10 / 1e-9 so that finite
    differences of the objective resolve the gradient.  ``device`` is a CUDA
    ordinal.
    """

    def __init__(self, case, *, device=0, tol=1e-13, tol2=None, cg_max_iterations=200000):
        if not case.cavity or case.amplitude == 0.0:
            raise ValueError("the adjoint covers the closed-cavity oscillating sphere")
        self.case = case
        lay = case.layout().build()
        self.lay = lay
        self.NC, self.NF, self.NE = lay.NC, lay.NF, lay.NE
        self.rou, self.visc = float(case.density), float(case.viscosity)
        self.dt = float(case.time_step)
        self.ac = self.ad = 0.5
        self.tol1, self.tol2 = float(tol), float(tol if tol2 is None else tol2)
        self.cg_max = int(cg_max_iterations)
        ops, prec = self._setup_solver(device)
        d = self.dev
        step_operators(lay, ops, self.visc, d, into=self)
        # Jacobi preconditioner of K = T M T^T (cells): diag K = (T o T) diag M
        Tm = (sp.hstack([ops.I[0], ops.I[1], ops.I[2]]).T @ ops.C).tocsr()
        dK = Tm.multiply(Tm) @ np.asarray(prec, dtype=np.float64)
        self.kdiag_inv = torch.from_numpy(np.where(dK > 0.0, 1.0 / np.where(dK > 0.0, dK, 1.0), 0.0)).to(d)
        self._k_prev = None
        self.seconds = {"solve": 0.0, "cells": 0.0}
        self.free = torch.from_numpy((prec != 0.0).astype(np.float64)).to(d)
        self.prec_t = torch.from_numpy(np.asarray(prec, dtype=np.float64)).to(d)
        # immersed boundary: finest-level lattice (ib_immersed.py:29-40)
        lv0 = lay.levels[0]
        self.h0 = float(lay.h0)
        self.hh3 = self.h0 ** 3
        self.pos_ref = torch.tensor(np.asarray(lv0.lo, dtype=np.float64) + 0.5 * self.h0, device=d)
        self.n0 = [int(v) for v in lv0.n]
        o = torch.arange(-2, 3, device=d)
        gi, gj, gk = torch.meshgrid(o, o, o, indexing="ij")
        self.off = torch.stack([gi.reshape(-1), gj.reshape(-1), gk.reshape(-1)], dim=1)   # (125, 3)
        ref, ds = case.markers()
        self.ref0 = torch.from_numpy(ref).to(d)
        self.ds3 = torch.from_numpy(ds ** 3).to(d)
        self.axis = torch.tensor(np.asarray(case.axis, float) / np.linalg.norm(case.axis), device=d)
        self.phase = float(case.phase)
        # closed-sphere loads: candidate and force-support cells (runner.SphereLoads)
        act = np.nonzero(lay.cell_active)[0]
        pos = lay.cpos[act]
        width = self.h0
        mt = np.abs(np.asarray(case.axis, float) / np.linalg.norm(case.axis)) * case.amplitude
        hw = SPHERE_RADIUS + 0.5 * width + mt
        cand = act[np.all(np.abs(pos) <= hw, axis=1)]
        fw = SPHERE_RADIUS + 1.5 * self.h0 + mt
        fw = fw + 8.0 * np.finfo(np.float64).eps * np.maximum(1.0, fw)
        fidx = act[np.all(np.abs(pos) <= fw, axis=1)]
        self.cand = torch.from_numpy(cand).to(d)
        self.cand_pos = torch.from_numpy(lay.cpos[cand]).to(d)
        self.cand_vol = torch.from_numpy(lay.cell_vol[cand]).to(d)
        self.fidx = torch.from_numpy(fidx).to(d)
        self.fidx_vol = torch.from_numpy(lay.cell_vol[fidx]).to(d)
        self.width = width
        self.solve_iterations = 0
        self.cell_iterations = 0

    # ---- solves ---------------------------------------------------------------------
    def _setup_solver(self, device):
        """The device context of the case's layout; returns (operators, preconditioner)."""
        self.dev = torch.device("cuda", device)
        self.solver = DeviceSolver(self.lay, rou=self.rou, visc=self.visc, cavity=True, tol1=self.tol1,
                                   tol2=self.tol2, cg_max_iterations=self.cg_max, device=device)
        self.lib = _lib.load()
        return self.solver.ops, self.solver.prec

    def cells32(self, cells):
        return cells.to(torch.int32).contiguous().reshape(-1)

    def spread(self, cells32, w, ds3, f):
        return _spread_device(self, cells32, w, ds3, f)

    def solve(self, res_e, s):
        """helm_solve: s + A+ res on the free edges (the device PCG)."""
        t0 = time.perf_counter()
        try:
            return self._solve_device(res_e, s)
        finally:
            self.seconds["solve"] += time.perf_counter() - t0

    def _solve_device(self, res_e, s):
        sv = self.solver
        sv.set("RES_E", res_e.detach().cpu().numpy())
        sv.set("S", s.detach().cpu().numpy())
        st = _lib.SolveStats()
        sv.h.call("pyib_helm_solve", C.c_double(self.dt), C.byref(st))
        self.solve_iterations += int(st.iterations)
        return torch.from_numpy(sv.get("S")).to(self.dev)

    def matvec(self, x):
        """A x with the masked rows zeroed (the CG's operator)."""
        sv = self.solver
        sv.set("WORK_E", x.detach().cpu().numpy())
        sv.h.call("pyib_matvec", _lib.F["WORK_E"], _lib.F["WORK_E2"], C.c_double(self.dt), 1)
        return torch.from_numpy(sv.get("WORK_E2")).to(self.dev)

    def _T(self, x):
        """T x = integr_c2f^T curl x: edges -> component-major cell vectors (3 NC)."""
        return self.Iop.MT @ (self.Cop.M @ x)

    def _Tt(self, k):
        """T^T k = rot integr_c2f k: the residual map of the step."""
        return self.Rop.M @ (self.Iop.M @ k)

    def _cg(self, op, b, tol, x0=None, dinv=None, check=10):
        """CG for a consistent symmetric positive semi-definite system, from ``x0``
        (zero if None), preconditioned by the diagonal ``dinv`` (none if None);
        stops when |r| <= tol |b| (tested every ``check`` iterations).  A start that
        does not reduce the residual below |b| is replaced by zero, and b = 0
        returns zero."""
        bb = b @ b
        if not bool(bb > 0.0):
            return torch.zeros_like(b)
        stop = (tol * tol) * bb
        x, r = torch.zeros_like(b), b.clone()
        if x0 is not None:
            r0 = b - op(x0)
            if bool((r0 @ r0) < bb):
                x, r = x0.clone(), r0
        z = r if dinv is None else dinv * r
        p = z.clone()
        rz = r @ z
        for it in range(self.cg_max):
            if it % check == 0 and not bool((r @ r) > stop):
                break
            Ap = op(p)
            pAp = p @ Ap
            if it % check == 0 and not bool(pAp > 0.0):
                break                      # the residual left is in the null space
            a = rz / pAp
            x += a * p
            r -= a * Ap
            z = r if dinv is None else dinv * r
            rz_new = r @ z
            p = z + (rz_new / rz) * p
            rz = rz_new
            self.cell_iterations += 1
        return x

    def pinv(self, g):
        """z with T z = T A+ g for any g on the free edges (see HelmSolve).

        A = T^T W T with T = integr_c2f^T curl (W the viscous block with the cell
        volumes), so the null space of A is the null space of T, and downstream the
        solve's gradient is only used through T.  A+ acts on the projection of
        M^1/2 g onto the range of M^1/2 T^T, which is M^1/2 T^T K+ T M g with
        K = T M T^T: one CG solve with K on cell vectors (Jacobi-preconditioned,
        started from the previous call's k, which the reverse sweep's consecutive
        solves keep close), after which A+ (T^T k) is a consistent solve by the
        device PCG.
        """
        t0 = time.perf_counter()
        k = self._cg(lambda v: self._T(self.prec_t * self._Tt(v)), self._T(self.prec_t * g), self.tol2,
                     x0=self._k_prev, dinv=self.kdiag_inv)
        self._k_prev = k
        u = self._Tt(k) * self.free
        self.seconds["cells"] += time.perf_counter() - t0
        return self.solve(u, torch.zeros_like(g)) * self.free

    # ---- the step's pieces ------------------------------------------------------------
    def calc_vel(self, s):
        """U = curl s, vc = interp_f2c U (closed cavity: no inlet edges; ghosts in LH/HL)."""
        U = SparseOp.apply(s, self.Cop)
        vc = SparseOp.apply(U, self.Pop).reshape(3, self.NC).t()
        return U, vc

    def stencil(self, markers):
        """Cells (M, 125) and Roma-Peskin weights of the markers (ib_immersed.py:63-81)."""
        base = torch.round((markers.detach() - self.pos_ref) / self.h0).to(torch.int64)   # rint
        ijk = base[:, None, :] + self.off[None, :, :]                                     # (M, 125, 3)
        n = self.n0
        inb = ((ijk >= 0) & (ijk < torch.tensor(n, device=self.dev))).all(dim=2)
        cells = torch.where(inb, (ijk[..., 2] * n[1] + ijk[..., 1]) * n[0] + ijk[..., 0], 0)
        g = (self.pos_ref + ijk.to(torch.float64) * self.h0) - markers[:, None, :]
        w = delta_h3(g[..., 0], self.h0) * delta_h3(g[..., 1], self.h0) * delta_h3(g[..., 2], self.h0)
        return cells, torch.where(inb, w, torch.zeros_like(w))

    def motion(self, t, A, omega, ref):
        """Markers, their velocity and the centre at time t (ib_kinematics.py:31-40)."""
        ang = omega * t + self.phase
        mk = ref + (A * torch.sin(ang)) * self.axis
        vel = ((A * omega) * torch.cos(ang)) * self.axis
        return mk, vel.expand_as(mk), (A * torch.sin(ang)) * self.axis

    def interior_momentum(self, vc, centre):
        """rho * sum chi * vol * vc over the candidate cells (ib_interior.py:57-70)."""
        dist = torch.linalg.norm(self.cand_pos - centre, dim=1)
        chi = torch.clamp((SPHERE_RADIUS + 0.5 * self.width - dist) / self.width, 0.0, 1.0)
        return self.rou * ((chi * self.cand_vol)[:, None] * vc[self.cand]).sum(dim=0)

    def initial_state(self, A, omega, ref):
        """Zero stream function (no inflow), zero held force, the interior momentum at t = 0."""
        s = torch.zeros(self.NE, dtype=torch.float64, device=self.dev)
        _, vc = self.calc_vel(s)
        _, _, c0 = self.motion(0.0, A, omega, ref)
        return (s, s.clone(), torch.zeros_like(ref), self.interior_momentum(vc, c0))

    def step(self, state, n, A, omega, ref):
        """State after step n (time n dt) from the state after step n - 1, and the
        axial body force of step n (ib_driver_np.py:412-532, ib_interior.py:268-308)."""
        s, s_old, fL, Pm = state
        dt, rou, ac, ad = self.dt, self.rou, self.ac, self.ad
        mk, vel, centre = self.motion(n * dt, A, omega, ref)
        cells, w = self.stencil(mk)
        fE = MarkerSpread.apply(fL, w, cells, self)               # the held force follows the body
        U, vc = self.calc_vel(s)
        conv0, diff0 = ConvDiff.apply(U, vc, self)
        res_c0 = rou * vc - (1 - ac) * dt * rou * conv0 + (1 - ad) * dt * diff0
        s_cur = s + (s - s_old) * dt / dt                          # Guess_s
        s_old_new = s
        U, vc = self.calc_vel(s_cur)
        for i in range(1, 5):
            conv, diff = ConvDiff.apply(U, vc, self)
            res_c = res_c0 - rou * vc - ac * dt * rou * conv + ad * dt * diff + dt * fE
            res_f = SparseOp.apply(res_c.t().reshape(-1), self.Iop)
            res_e = SparseOp.apply(res_f, self.Rop)
            s_cur = HelmSolve.apply(res_e, s_cur, self)
            U, vc = self.calc_vel(s_cur)
            if i == 1:
                uL = MarkerInterp.apply(vc, w, cells, self)
                dL = (vel - uL) / dt
                fE = fE + rou * MarkerSpread.apply(dL, w, cells, self)
                fL = fL + rou * dL
        F_fluid = (fE[self.fidx] * self.fidx_vol[:, None]).sum(dim=0)
        P = self.interior_momentum(vc, centre)
        body = -F_fluid + (P - Pm) / dt
        return (s_cur, s_old_new, fL, P), body[0]


def harmonic_amplitude(force, times, omega, phase):
    """First-harmonic amplitude of a force history: least squares on
    [cos(omega t + phase), sin(omega t + phase), 1] (check_pressure_validation.py:31-37)."""
    ang = omega * times + phase
    X = torch.stack([torch.cos(ang), torch.sin(ang), torch.ones_like(ang)], dim=1)
    coeff = torch.linalg.solve(X.t() @ X, X.t() @ force)
    return torch.sqrt(coeff[0] ** 2 + coeff[1] ** 2)


def _beta(s, t):
    """Steps reversible with s snapshots and t forward repetitions: C(s + t, t)."""
    return math.comb(s + t, t)


class Reverser:
    """Reverse sweep of the steps with at most ``snapshots`` stored states.

    Binomial checkpointing (Griewank's rule): to reverse steps i0+1 .. i1 from the
    stored state at i0 with s further snapshots, let t be the least repetition
    count with beta(s, t) >= n (n = i1 - i0), advance to
    m = i0 + max(min(beta(s, t - 1), n - 1), n - beta(s - 1, t), 1), store the
    state at m, reverse m .. i1 with s - 1 snapshots, then i0 .. m with s; the
    split keeps the right part within beta(s - 1, t) steps and the left part
    within beta(s, t - 1).  With no snapshot left, each step is reached by
    advancing again from i0.  One step is reversed by recomputing it from its
    stored input state with the autograd tape on and pulling the adjoint back.
    """

    def __init__(self, model, params, gF, snapshots):
        self.m = model
        self.A, self.omega, self.ref = params
        self.gF = gF                       # dJ / dF_n, n = 1 .. N (zero outside the window)
        self.snapshots = int(snapshots)
        self.lam = None                    # adjoint of the state after the current step
        self.grad = [torch.zeros_like(p) for p in params]
        self.recomputed = 0
        self.max_live = 1                  # the initial state is stored throughout
        self._live = 0
        self.progress = None
        self._reversed = 0
        self._t0 = time.perf_counter()

    def advance(self, state, i0, i1):
        with torch.no_grad():
            for n in range(i0 + 1, i1 + 1):
                state, _ = self.m.step(state, n, self.A, self.omega, self.ref)
                self.recomputed += 1
        return state

    def reverse_step(self, state, n):
        """lam <- (d state_n / d state_{n-1})^T lam + (d F_n / d state_{n-1})^T gF_n."""
        inp = [x.detach().requires_grad_(True) for x in state]
        params = [p.detach().requires_grad_(True) for p in (self.A, self.omega, self.ref)]
        with torch.enable_grad():
            out, F = self.m.step(tuple(inp), n, *params)
            outs = [o for o in out] + [F]
            gouts = [l for l in self.lam] + [self.gF[n - 1]]
            grads = torch.autograd.grad(outs, inp + params, grad_outputs=gouts, allow_unused=True)
        k = len(inp)
        self.lam = [g if g is not None else torch.zeros_like(x) for g, x in zip(grads[:k], inp)]
        self._reversed += 1
        if self.progress is not None and self._reversed % 20 == 0:
            self.progress(f"reversed {self._reversed} steps (at step {n}), {self.recomputed} recomputed, "
                          f"{time.perf_counter() - self._t0:.1f} s, {self.m.solve_iterations} PCG and "
                          f"{self.m.cell_iterations} cell CG iterations")
        for j, g in enumerate(grads[k:]):
            if g is not None:
                self.grad[j] = self.grad[j] + g.detach()

    def reverse(self, state, i0, i1, s):
        n = i1 - i0
        if n == 1:
            self.reverse_step(state, i1)
        elif s <= 0:
            for j in range(i1, i0, -1):
                self.reverse_step(self.advance(state, i0, j - 1), j)
        else:
            t = 1
            while _beta(s, t) < n:
                t += 1
            # the left part has t - 1 repetitions left, the right part s - 1 snapshots
            m = i0 + max(min(_beta(s, t - 1), n - 1), n - _beta(s - 1, t), 1)
            mid = self.advance(state, i0, m)
            self._live += 1                      # stored states besides the initial one
            self.max_live = max(self.max_live, 1 + self._live)
            self.reverse(mid, m, i1, s - 1)
            del mid
            self._live -= 1
            self.reverse(state, i0, m, s)


def _params(model, A, T, ref):
    dev = model.dev
    return (torch.tensor(float(A), dtype=torch.float64, device=dev),
            torch.tensor(2.0 * math.pi / float(T), dtype=torch.float64, device=dev),
            torch.as_tensor(ref, dtype=torch.float64, device=dev))


def _history(model, A_t, om_t, ref_t, steps):
    with torch.no_grad():
        state0 = model.initial_state(A_t, om_t, ref_t)
        state = state0
        F = []
        for n in range(1, steps + 1):
            state, Fn = model.step(state, n, A_t, om_t, ref_t)
            F.append(Fn)
    return state0, state, torch.stack(F)


def force_amplitude(model, A, T, ref, steps, window):
    """The objective alone (one forward run), for finite differences."""
    A_t, om_t, ref_t = _params(model, A, T, ref)
    _, _, F = _history(model, A_t, om_t, ref_t, steps)
    times = torch.arange(1, steps + 1, dtype=torch.float64, device=model.dev) * model.dt
    return float(harmonic_amplitude(F[steps - window:], times[steps - window:], om_t, model.phase))


def force_amplitude_and_gradient(model, A, T, ref, steps, window, snapshots=20, progress=None):
    """J = harmonic amplitude of the axial body force over the last ``window`` steps,
    and dJ/dA, dJ/dT, dJ/dref by the discrete adjoint with binomial checkpointing.

    ``A`` and ``T`` are floats, ``ref`` the (M, 3) reference marker positions.
    ``progress`` (optional) is called with a short text after the forward run and
    every 20 reverse steps.  Returns (J, dJ/dA, dJ/dT, dJ/dref (M, 3), info).
    """
    A_t, om_t, ref_t = _params(model, A, T, ref)
    model.solve_iterations = model.cell_iterations = 0
    model.seconds = {"solve": 0.0, "cells": 0.0}
    model._k_prev = None
    t0 = time.perf_counter()
    state0, state, F = _history(model, A_t, om_t, ref_t, steps)
    fwd_iters = model.solve_iterations
    t_fwd = time.perf_counter() - t0
    if progress is not None:
        progress(f"forward {steps} steps {t_fwd:.1f} s, {fwd_iters} CG iterations")
    times = torch.arange(1, steps + 1, dtype=torch.float64, device=model.dev) * model.dt
    Fw = F.detach().clone().requires_grad_(True)
    om_f = om_t.detach().clone().requires_grad_(True)
    with torch.enable_grad():
        J = harmonic_amplitude(Fw[steps - window:], times[steps - window:], om_f, model.phase)
        gF, g_om_fit = torch.autograd.grad(J, [Fw, om_f])
    # reverse sweep; J depends on the forces, so the final state's adjoint is zero
    rv = Reverser(model, (A_t, om_t, ref_t), gF, snapshots)
    rv.progress = progress
    rv.lam = [torch.zeros_like(x) for x in state]
    rv.reverse(state0, 0, steps, snapshots - 1)
    # the initial state depends on the parameters only through its interior momentum
    inp = [p.detach().requires_grad_(True) for p in (A_t, om_t, ref_t)]
    with torch.enable_grad():
        st0 = model.initial_state(*inp)
        pairs = [(o, l) for o, l in zip(st0, rv.lam) if o.requires_grad]
        g0 = (torch.autograd.grad([o for o, _ in pairs], inp, grad_outputs=[l for _, l in pairs],
                                  allow_unused=True) if pairs else (None, None, None))
    add = lambda a, b: a + b if b is not None else a
    gA = add(rv.grad[0], g0[0])
    gom = add(rv.grad[1], g0[1]) + g_om_fit
    gref = add(rv.grad[2], g0[2])
    dJdT = gom * (-2.0 * math.pi / float(T) ** 2)
    info = {"forward_cg_iterations": fwd_iters, "total_cg_iterations": model.solve_iterations,
            "cell_cg_iterations": model.cell_iterations, "recomputed_steps": rv.recomputed,
            "forward_seconds": t_fwd, "solve_seconds": model.seconds["solve"],
            "cell_solve_seconds": model.seconds["cells"],
            "max_stored_states": rv.max_live, "force": F.cpu().numpy()}
    return float(J), float(gA), float(dJdT), gref.cpu().numpy(), info


class ForceAmplitude(torch.autograd.Function):
    """J(A, T, ref) = the first-harmonic axial force amplitude; backward by the adjoint."""

    @staticmethod
    def forward(ctx, A, T, ref, model, steps, window, snapshots):
        J, gA, gT, gref, info = force_amplitude_and_gradient(
            model, float(A), float(T), ref.detach(), steps, window, snapshots)
        ctx.save_for_backward(torch.tensor(gA, dtype=torch.float64), torch.tensor(gT, dtype=torch.float64),
                              torch.from_numpy(gref))
        ctx.info = info
        return torch.tensor(J, dtype=torch.float64, device=ref.device)

    @staticmethod
    def backward(ctx, g):
        gA, gT, gref = ctx.saved_tensors
        gs = g.detach().cpu()
        return ((gs * gA).to(g.device), (gs * gT).to(g.device), (gs * gref).to(g.device),
                None, None, None, None)
