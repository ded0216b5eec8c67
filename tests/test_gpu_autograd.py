"""Adjoint building blocks behind torch.autograd: transpose identities on the GPU kernels."""
import ctypes as C

import numpy as np
import pytest
import torch

import parity_util as PU
from pyib_b200 import _lib
from pyib_b200 import autograd as AG
from pyib_b200.device import DeviceSolver

pytestmark = pytest.mark.gpu


def _solver(name="n3_osc", tol=None):
    g = PU.golden(name)
    lay = PU.layout_for(name)
    kw = {} if tol is None else {"tol1": tol, "tol2": tol}
    sv = DeviceSolver(lay, rou=float(g["rou"]), visc=float(g["visc"]), cavity=bool(g["cavity"]),
                      cg_max_iterations=20000, **kw)
    sv.set_markers(g["ib_markers"], g["ib_vel"], g["ib_ds"])
    return g, sv


def _matvec(sv, z, dt):
    sv.set("WORK_E", z)
    sv.h.call("pyib_matvec", _lib.F["WORK_E"], _lib.F["WORK_E2"], C.c_double(dt), 1)
    return sv.get("WORK_E2")


def test_helmholtz_solve_adjoint_is_the_same_solve():
    """<c, A^-1 d> through autograd equals <A^-1 c, d> and the exact <A y, z>.

    d = A z and c = A y lie in the range of A (the closed cavity leaves a gauge
    null space), so both solves have solutions, and A being symmetric, <c, x> is
    the same for every solution x.  The CG runs to a mixed tolerance of 1e-13, so
    both sides agree with the exact value to 1e-9.
    """
    g, sv = _solver(tol=1e-13)
    dt = float(g["dt"])
    free = sv.prec != 0.0
    rng = np.random.default_rng(5)
    z = rng.standard_normal(sv.lay.NE) * free
    y = rng.standard_normal(sv.lay.NE) * free
    d, c = _matvec(sv, z, dt), _matvec(sv, y, dt)
    exact = float(np.dot(c, z))
    d_t = torch.tensor(d, dtype=torch.float64, requires_grad=True)
    s_t = torch.zeros(sv.lay.NE, dtype=torch.float64, requires_grad=True)
    x = AG.HelmholtzSolve.apply(d_t, s_t, sv, dt)
    loss = (torch.tensor(c) * x).sum()
    loss.backward()
    adjoint = float(torch.dot(d_t.grad, torch.tensor(d)))
    print("solve adjoint: relative differences", abs(loss.item() - exact) / abs(exact),
          abs(adjoint - exact) / abs(exact))
    assert abs(loss.item() - exact) <= 1e-9 * abs(exact)
    assert abs(adjoint - exact) <= 1e-9 * abs(exact)
    np.testing.assert_array_equal(s_t.grad.numpy(), c)       # d x / d s = identity
    assert np.all(d_t.grad.numpy()[~free] == 0.0)


def test_marker_interp_and_spread_are_transposes():
    g, sv = _solver()
    lay = sv.lay
    rng = np.random.default_rng(7)
    act = lay.cell_active
    M = g["ib_markers"].shape[0]
    ds = g["ib_ds"]
    # interpolation: <interp(v), u> = <v, interp^T u>
    v = torch.tensor(rng.standard_normal((3, lay.NC)) * act, dtype=torch.float64, requires_grad=True)
    u = torch.tensor(rng.standard_normal((M, 3)), dtype=torch.float64)
    out = AG.MarkerInterp.apply(v, sv, ds)
    lhs = (out * u).sum()
    lhs.backward()
    rhs = (v.grad * v.detach()).sum()
    assert abs(lhs.item() - rhs.item()) <= 1e-12 * abs(lhs.item())
    # the forward matches the reference's interpolation of its golden field
    vc = PU.cell3_to_dense("n3_osc", g["cv_vc"][:int(g["mesh_ncell"])])
    assert PU.rel(AG.interp(sv, vc), g["ib_interp"]) < 1e-14
    # spreading: <spread(f), h> = <f, spread^T h>
    f = torch.tensor(rng.standard_normal((M, 3)), dtype=torch.float64, requires_grad=True)
    h = torch.tensor(rng.standard_normal((3, lay.NC)) * act, dtype=torch.float64)
    fe = AG.MarkerSpread.apply(f, sv, ds)
    lhs = (fe * h).sum()
    lhs.backward()
    rhs = (f.grad * f.detach()).sum()
    assert abs(lhs.item() - rhs.item()) <= 1e-12 * abs(lhs.item())
    # the marker volumes are restored after an interpolation backward
    np.testing.assert_array_equal(sv.get("DS"), ds ** 3)


def test_marker_position_gradient_matches_finite_differences():
    """d/dx of sum(w * interp(vc) at markers x) against a central difference.

    The Roma-Peskin kernel is continuously differentiable, so the difference
    along a random unit direction converges to the kernel's Jacobian (step 1e-6 h,
    tolerance 1e-6 relative).
    """
    g, sv = _solver()
    rng = np.random.default_rng(9)
    vc = PU.cell3_to_dense("n3_osc", g["cv_vc"][:int(g["mesh_ncell"])])
    mk0, ds = np.asarray(g["ib_markers"]), g["ib_ds"]
    w = rng.standard_normal(mk0.shape)
    vc_t = torch.tensor(vc, dtype=torch.float64)
    mk_t = torch.tensor(mk0, dtype=torch.float64, requires_grad=True)
    u = AG.MarkerInterpAt.apply(vc_t, mk_t, sv, ds)
    (u * torch.tensor(w)).sum().backward()
    ad_grad = mk_t.grad.numpy().copy()

    def f(mk):
        return float((AG.MarkerInterpAt.apply(vc_t, torch.tensor(mk), sv, ds).numpy() * w).sum())

    direction = rng.standard_normal(mk0.shape)
    direction /= np.linalg.norm(direction)
    eps = 1e-6 * sv.lay.h0
    fd = (f(mk0 + eps * direction) - f(mk0 - eps * direction)) / (2.0 * eps)
    ad = float(np.sum(ad_grad * direction))
    print("interp position gradient: relative difference", abs(fd - ad) / abs(ad))
    assert abs(fd - ad) <= 1e-6 * abs(ad), (fd, ad)
    # per marker: the Jacobian of one marker's velocity along x
    m, c = 3, 0
    e = np.zeros_like(mk0)
    e[m, 0] = 1.0
    fp = AG.MarkerInterpAt.apply(vc_t, torch.tensor(mk0 + eps * e), sv, ds).numpy()[m, c]
    fm = AG.MarkerInterpAt.apply(vc_t, torch.tensor(mk0 - eps * e), sv, ds).numpy()[m, c]
    sv.set_markers(mk0, np.zeros_like(mk0), ds)
    jac = AG.interp_dx(sv, vc)
    print("interp Jacobian entry: relative difference",
          abs((fp - fm) / (2.0 * eps) - jac[m, c, 0]) / np.max(np.abs(jac[m])))
    assert abs((fp - fm) / (2.0 * eps) - jac[m, c, 0]) <= 1e-6 * np.max(np.abs(jac[m])) + 1e-12



@pytest.mark.parametrize("name", ["n3_osc", "n2_fixed"])
def test_calc_vel_transpose(name):
    """<calc_vel(s) - calc_vel(0), g> = <s, calc_vel^T g>; the inflow case is affine
    (its inlet edges take prescribed values), the cavity case linear."""
    g, sv = _solver(name)
    lay = sv.lay
    rng = np.random.default_rng(11)
    s = rng.standard_normal(lay.NE) * lay.edge_exists
    gv = rng.standard_normal((3, lay.NC)) * lay.cell_active
    s_t = torch.tensor(s, dtype=torch.float64, requires_grad=True)
    vc = AG.CalcVel.apply(s_t, sv)
    base = AG.calc_vel(sv, np.zeros(lay.NE))
    lhs = float(((vc.detach().numpy() - base) * gv).sum())
    (vc * torch.tensor(gv)).sum().backward()
    rhs = float((s_t.grad.numpy() * s).sum())
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs), (lhs, rhs)
    assert np.all(s_t.grad.numpy()[sv.inlet] == 0.0)


def test_marker_spread_position_gradient_matches_finite_differences():
    g, sv = _solver()
    lay = sv.lay
    rng = np.random.default_rng(13)
    mk0, ds = np.asarray(g["ib_markers"]), g["ib_ds"]
    f = rng.standard_normal(mk0.shape)
    # a smooth weight field: the reference's own cell velocity
    h = PU.cell3_to_dense("n3_osc", g["cv_vc"][:int(g["mesh_ncell"])])
    f_t = torch.tensor(f, dtype=torch.float64, requires_grad=True)
    mk_t = torch.tensor(mk0, dtype=torch.float64, requires_grad=True)
    fe = AG.MarkerSpreadAt.apply(f_t, mk_t, sv, ds)
    (fe * torch.tensor(h)).sum().backward()
    ad_mk, ad_f = mk_t.grad.numpy().copy(), f_t.grad.numpy().copy()

    def loss(mk, ff):
        return float((AG.MarkerSpreadAt.apply(torch.tensor(ff), torch.tensor(mk), sv, ds).numpy() * h).sum())

    direction = rng.standard_normal(mk0.shape)
    direction /= np.linalg.norm(direction)
    eps = 1e-6 * lay.h0
    fd = (loss(mk0 + eps * direction, f) - loss(mk0 - eps * direction, f)) / (2.0 * eps)
    ad = float(np.sum(ad_mk * direction))
    print("spread position gradient: relative difference", abs(fd - ad) / abs(ad))
    assert abs(fd - ad) <= 1e-6 * abs(ad), (fd, ad)
    # linear in the forces: the gradient is exact
    assert abs(loss(mk0, f) - float(np.sum(ad_f * f))) <= 1e-12 * abs(loss(mk0, f))
