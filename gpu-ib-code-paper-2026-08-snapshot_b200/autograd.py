"""``torch.autograd.Function`` wrappers of the step's linear pieces and their adjoints.

These are building blocks of a discrete adjoint of the step, run by the same
hand-written kernels as the forward path:

* ``HelmholtzSolve``: the stream-function solve of ``Driver.helm_solve``
  (``ib_driver_np.py:311-410``), ``x = s + A_ff^-1 res_f`` on the free edges
  (``x = s`` on masked edges).  A is symmetric, so the adjoint is the same PCG
  on the masked incoming gradient from a zero start; the gradient with respect
  to ``s`` is the identity.
* ``MarkerInterp``: ``u_L = sum_k w_k vc[cell_k] hh^3`` (``ib_immersed.py:87-93``).
  Its transpose is spreading with ``hh^3`` in place of the marker volumes.
* ``MarkerSpread``: ``f_E = sum w f_L ds^3`` (``ib_immersed.py:103-111``).  Its
  transpose is interpolation scaled by ``ds^3 / hh^3`` per marker.
* ``MarkerInterpAt``: the interpolation at given marker positions, with the
  gradient with respect to those positions through the delta-kernel weights
  (``pyib_ib_interp_dx``, the per-marker 3x3 Jacobian).
* ``MarkerSpreadAt``: spreading at given marker positions; its position gradient
  is the interpolation Jacobian of the incoming gradient field, scaled by
  ``ds^3 / hh^3`` and contracted with the marker forces.
* ``CalcVel``: the cell velocity of ``Driver.calc_vel`` (``ib_driver_np.py:267-291``),
  ``vc = P C s`` with the inlet edges of s replaced by their prescribed values.
  Its transpose is ``R I (vol * g)`` (``R = C^T``; the interpolation ``P`` is the
  integration ``I`` weighted by the cell volume factor), zero on inlet edges.

``MarkerInterp`` and ``MarkerSpread`` use the stencil of the markers last set
on the solver.  Tensors are float64 in the solver's dense
layout (edges: ``NE``; cell vectors: ``(3, NC)``; markers: ``(M, 3)``) on any
device: they cross the C ABI as host arrays.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib


def _np(t):
    return t.detach().to("cpu", torch.float64).contiguous().numpy()


def _like(a, ref):
    return torch.from_numpy(np.ascontiguousarray(a)).to(ref.device)


def solve(solver, res_e, s, dt):
    """One Helmholtz solve on the device: returns x (float64, dense edges)."""
    solver.set("RES_E", res_e)
    solver.set("S", s)
    st = _lib.SolveStats()
    solver.h.call("pyib_helm_solve", C.c_double(dt), C.byref(st))
    return solver.get("S")


class HelmholtzSolve(torch.autograd.Function):
    """x = helm_solve(res_e, s); backward solves A y = mask * grad_x."""

    @staticmethod
    def forward(ctx, res_e, s, solver, dt):
        ctx.solver, ctx.dt = solver, float(dt)
        return _like(solve(solver, _np(res_e), _np(s), ctx.dt), res_e)

    @staticmethod
    def backward(ctx, grad_x):
        sv = ctx.solver
        free = sv.prec != 0.0
        g = _np(grad_x) * free
        y = solve(sv, g, np.zeros_like(g), ctx.dt) * free
        return _like(y, grad_x), grad_x, None, None


def _stencil(solver):
    solver.h.call("pyib_ib_stencil")


def interp(solver, vc3):
    """u_L (M, 3) from a cell vector field (3, NC)."""
    lay = solver.lay
    full = np.zeros((3, lay.NC + solver.bfaces.size))
    full[:, :lay.NC] = vc3
    solver.set("VC", full)
    _stencil(solver)
    solver.h.call("pyib_ib_interp")
    return solver.get("LAG_TMP").reshape(-1, 3)


def spread(solver, f_l, ds):
    """f_E (3, NC) = sum w f_L ds^3, with the given per-marker widths ``ds``."""
    solver.set("DS", np.asarray(ds, dtype=np.float64) ** 3)
    solver.set("FL", f_l)
    _stencil(solver)
    solver.h.call("pyib_ib_spread")
    return solver.get("FE").reshape(3, -1)


class MarkerInterp(torch.autograd.Function):
    """u_L = interp(vc); backward spreads grad_u with hh^3 weights."""

    @staticmethod
    def forward(ctx, vc3, solver, ds):
        ctx.solver, ctx.ds = solver, np.asarray(ds, dtype=np.float64)
        return _like(interp(solver, _np(vc3)), vc3)

    @staticmethod
    def backward(ctx, grad_u):
        sv = ctx.solver
        hh = np.full(ctx.ds.shape, sv.lay.h0)
        g = spread(sv, _np(grad_u), hh)
        sv.set("DS", ctx.ds ** 3)                # restore the marker volumes
        return _like(g, grad_u), None, None


class MarkerSpread(torch.autograd.Function):
    """f_E = spread(f_L); backward interpolates grad_fE and scales by ds^3 / hh^3."""

    @staticmethod
    def forward(ctx, f_l, solver, ds):
        ctx.solver, ctx.ds = solver, np.asarray(ds, dtype=np.float64)
        return _like(spread(solver, _np(f_l), ctx.ds), f_l)

    @staticmethod
    def backward(ctx, grad_fe):
        sv = ctx.solver
        u = interp(sv, _np(grad_fe))
        scale = (ctx.ds ** 3 / sv.lay.h0 ** 3)[:, None]
        return _like(u * scale, grad_fe), None, None


def interp_dx(solver, vc3):
    """Per-marker Jacobian d u_L[m, c] / d x_m[d], shape (M, 3, 3), at the current markers."""
    lay = solver.lay
    full = np.zeros((3, lay.NC + solver.bfaces.size))
    full[:, :lay.NC] = vc3
    solver.set("VC", full)
    _stencil(solver)
    jac = np.empty(9 * solver.M)
    solver.h.call("pyib_ib_interp_dx", jac.ctypes.data_as(C.POINTER(C.c_double)))
    return jac.reshape(-1, 3, 3)


class MarkerInterpAt(torch.autograd.Function):
    """u_L = interp(vc) at ``markers`` (M, 3); gradients for vc and for the markers."""

    @staticmethod
    def forward(ctx, vc3, markers, solver, ds):
        ds = np.asarray(ds, dtype=np.float64)
        mk = _np(markers)
        solver.set_markers(mk, np.zeros_like(mk), ds)
        v = _np(vc3)
        ctx.solver, ctx.ds, ctx.v, ctx.mk = solver, ds, v, mk
        return _like(interp(solver, v), vc3)

    @staticmethod
    def backward(ctx, grad_u):
        sv = ctx.solver
        sv.set_markers(ctx.mk, np.zeros_like(ctx.mk), ctx.ds)   # the forward's positions
        g = _np(grad_u)
        jac = interp_dx(sv, ctx.v)
        grad_mk = np.einsum("mc,mcd->md", g, jac)
        hh = np.full(ctx.ds.shape, sv.lay.h0)
        grad_vc = spread(sv, g, hh)
        sv.set("DS", ctx.ds ** 3)
        return _like(grad_vc, grad_u), _like(grad_mk, grad_u), None, None


class MarkerSpreadAt(torch.autograd.Function):
    """f_E = spread(f_L) at ``markers``; gradients for f_L and for the markers."""

    @staticmethod
    def forward(ctx, f_l, markers, solver, ds):
        ds = np.asarray(ds, dtype=np.float64)
        mk = _np(markers)
        solver.set_markers(mk, np.zeros_like(mk), ds)
        f = _np(f_l)
        ctx.solver, ctx.ds, ctx.mk, ctx.f = solver, ds, mk, f
        return _like(spread(solver, f, ds), f_l)

    @staticmethod
    def backward(ctx, grad_fe):
        sv = ctx.solver
        sv.set_markers(ctx.mk, np.zeros_like(ctx.mk), ctx.ds)   # the forward's positions
        g = _np(grad_fe)
        scale = (ctx.ds ** 3 / sv.lay.h0 ** 3)[:, None]
        grad_f = interp(sv, g) * scale
        jac = interp_dx(sv, g)
        grad_mk = np.einsum("mc,mcd->md", ctx.f, jac) * scale
        return _like(grad_f, grad_fe), _like(grad_mk, grad_fe), None, None


def calc_vel(solver, s):
    """Cell velocity (3, NC) of ``s`` (the inlet edges take their prescribed values)."""
    solver.set("S", s)
    solver.h.call("pyib_calc_vel")
    return solver.vc_cells()


def calc_vel_transpose(solver, g):
    """s-gradient (NE) of sum(g * calc_vel(s)): R I (vol * g), zero on inlet edges."""
    solver.set("WORK_C3", np.asarray(g, dtype=np.float64) * solver.ops.vol_ci[None, :])
    solver.h.call("pyib_operator", 3)        # integr_c2f: WORK_C3 -> WORK_F
    solver.h.call("pyib_operator", 1)        # rot: WORK_F -> WORK_E
    out = solver.get("WORK_E")
    out[solver.inlet] = 0.0
    return out


class CalcVel(torch.autograd.Function):
    """vc = calc_vel(s) on the active cells; backward applies its transpose."""

    @staticmethod
    def forward(ctx, s, solver):
        ctx.solver = solver
        return _like(calc_vel(solver, _np(s)), s)

    @staticmethod
    def backward(ctx, grad_vc):
        return _like(calc_vel_transpose(ctx.solver, _np(grad_vc)), grad_vc), None

