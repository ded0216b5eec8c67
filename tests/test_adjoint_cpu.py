"""Pieces of the discrete adjoint that run on the CPU.

* the differentiable convection/diffusion restatement equals the reference's
  ``Driver.conv_diff`` on the closed-cavity fixture (its no-slip ghosts folded
  into the face operators);
* its hand-written backward is the transpose of its linearisation, and the
  sparse operators' backwards are their transposes;
* the differentiable Roma-Peskin kernel equals the reference's formula to one
  rounding and its derivative matches central differences;
* the harmonic amplitude equals the restated fit of the reference's check tool;
* the binomial checkpointing reverse sweep gives the gradient of the full tape
  while storing at most the allowed number of states;
* with a NumPy mirror of the device PCG (``adjoint_cpu_model``), the projected
  pseudo-inverse of the singular cavity operator agrees with the solve on
  consistent vectors, and one whole step's adjoint (its solves see inconsistent
  gradients) matches central differences for the amplitude and the marker
  positions.
"""
import math

import numpy as np
import pytest
import torch

import parity_util as PU
from adjoint_cpu_model import CpuCavityModel
from pyib_b200 import adjoint as AD
from pyib_b200 import harmonic as H
from pyib_b200.cases import SphereCase
from pyib_b200.operators import Operators

pytestmark = pytest.mark.filterwarnings("ignore::UserWarning")

# closed cavity, 2 levels at h = D/4 (3240 cells, 50 markers), Re0 = 1, 10 steps per period
TINY = SphereCase(name="adjoint_tiny", cells_per_diameter=4, half_widths_d=(1.5, 3.0), reynolds=1.0,
                  amplitude_d=0.2, steps_per_period=10)


@pytest.fixture(scope="module")
def cavity():
    name = "n3_osc"
    g = PU.golden(name)
    lay = PU.layout_for(name)
    ops = Operators(lay)
    o = AD.step_operators(lay, ops, float(g["visc"]), torch.device("cpu"))
    return name, g, lay, o


@pytest.fixture(scope="module")
def tiny():
    torch.set_num_threads(min(4, torch.get_num_threads()))
    return CpuCavityModel(TINY, tol=1e-13)


def test_conv_diff_equals_reference(cavity):
    name, g, lay, o = cavity
    U = torch.from_numpy(PU.face_to_dense(name, g["cv_U"]))
    nc_ref = g["cd_conv"].shape[0]
    vc = torch.from_numpy(PU.cell3_to_dense(name, g["cv_vc"][:nc_ref]).T.copy())
    conv, diff = AD.ConvDiff.apply(U, vc, o)
    got_c = PU.cell3_from_dense(name, conv.numpy().T)
    got_d = PU.cell3_from_dense(name, diff.numpy().T)
    assert PU.rel(got_c, g["cd_conv"]) < 1e-13
    assert PU.rel(got_d, g["cd_diff"]) < 1e-13


def test_conv_diff_backward_is_the_transposed_linearisation(cavity):
    name, g, lay, o = cavity
    torch.manual_seed(0)
    U = torch.randn(lay.NF, dtype=torch.float64, requires_grad=True)
    vc = torch.randn(lay.NC, 3, dtype=torch.float64, requires_grad=True)
    conv, diff = AD.ConvDiff.apply(U, vc, o)
    gc, gd = torch.randn_like(conv), torch.randn_like(diff)
    gU, gvc = torch.autograd.grad([conv, diff], [U, vc], [gc, gd])
    dU, dvc = torch.randn_like(U) * 1e-6, torch.randn_like(vc) * 1e-6
    with torch.no_grad():
        c2, d2 = AD.ConvDiff.apply(U + dU, vc + dvc, o)
        c1, d1 = AD.ConvDiff.apply(U - dU, vc - dvc, o)
    lhs = float(((c2 - c1) * gc).sum() + ((d2 - d1) * gd).sum()) / 2.0     # exact for a bilinear map
    rhs = float((gU * dU).sum() + (gvc * dvc).sum())
    assert abs(lhs - rhs) <= 1e-8 * abs(rhs)


def test_sparse_operator_backwards_are_transposes(cavity):
    name, g, lay, o = cavity
    torch.manual_seed(1)
    for op, n_in in ((o.Cop, lay.NE), (o.Rop, lay.NF), (o.Pop, lay.NF), (o.Iop, 3 * lay.NC)):
        x = torch.randn(n_in, dtype=torch.float64, requires_grad=True)
        y = AD.SparseOp.apply(x, op)
        gy = torch.randn_like(y)
        (gx,) = torch.autograd.grad(y, x, gy)
        scale = float(torch.linalg.norm(y) * torch.linalg.norm(gy))
        assert abs(float((y * gy).sum() - (x * gx).sum())) <= 1e-12 * scale


def test_delta_kernel_values_and_derivative():
    h = 0.0625
    r = torch.linspace(-1.7 * h, 1.7 * h, 1001, dtype=torch.float64)
    a = np.abs(r.numpy() / h)
    ref = np.zeros_like(a)
    m1 = a <= 0.5
    ref = np.where(m1, (1.0 + np.sqrt(np.clip(1.0 - 3.0 * a * a, 0.0, None))) / (3.0 * h), ref)
    m2 = (a > 0.5) & (a <= 1.5)
    ref = np.where(m2, (5.0 - 3.0 * a - np.sqrt(np.clip(1.0 - 3.0 * (1.0 - a) ** 2, 0.0, None))) / (6.0 * h), ref)
    # same formula; torch's vector kernels may round a product differently (1 ulp)
    assert np.max(np.abs(AD.delta_h3(r, h).numpy() - ref)) <= 1e-15 * np.max(ref)
    x = (r + 1e-4 * h).clone().requires_grad_(True)      # away from the exact break points
    (g,) = torch.autograd.grad(AD.delta_h3(x, h).sum(), x)
    e = 1e-7 * h
    fd = (AD.delta_h3(x.detach() + e, h) - AD.delta_h3(x.detach() - e, h)) / (2 * e)
    assert torch.max(torch.abs(g - fd)) <= 1e-5 * float(torch.max(torch.abs(fd)))


def test_harmonic_amplitude_equals_fit():
    rng = np.random.default_rng(3)
    om, ph = 3.6, -math.pi / 2
    t = np.arange(1, 41) * (2 * math.pi / om / 40)
    f = 0.7 * np.cos(om * t + ph) - 0.2 * np.sin(om * t + ph) + 0.1 + 1e-3 * rng.standard_normal(t.size)
    coeff, _ = H.fit(t, f, om, ph)
    amp = AD.harmonic_amplitude(torch.from_numpy(f), torch.from_numpy(t), torch.tensor(om, dtype=torch.float64), ph)
    assert abs(float(amp) - float(np.hypot(coeff[0], coeff[1]))) <= 1e-13


class _Toy:
    """A small nonlinear step with the model's signature, for the reverse sweep."""

    def __init__(self):
        g = torch.Generator().manual_seed(5)
        self.W = torch.randn(6, 6, generator=g, dtype=torch.float64) * 0.3

    def step(self, state, n, A, omega, ref):
        x, y = state
        x2 = torch.tanh(self.W @ x + A * torch.sin(omega * n * 0.1) + ref.sum(dim=1)[:6] * 0.01) + 0.1 * y
        y2 = y * 0.9 + 0.05 * x * x
        return (x2, y2), (x2 * x2).sum() * torch.cos(omega * n * 0.05)


@pytest.mark.parametrize("steps,snapshots", [(1, 3), (7, 2), (24, 4), (40, 20), (400, 20)])
def test_reverse_sweep_equals_full_tape(steps, snapshots):
    toy = _Toy()
    A = torch.tensor(0.3, dtype=torch.float64, requires_grad=True)
    om = torch.tensor(1.7, dtype=torch.float64, requires_grad=True)
    ref = torch.randn(8, 3, dtype=torch.float64, generator=torch.Generator().manual_seed(2), requires_grad=True)
    x0 = (torch.full((6,), 0.1, dtype=torch.float64), torch.zeros(6, dtype=torch.float64))
    gF = torch.linspace(0.5, 1.5, steps, dtype=torch.float64)
    st, J = x0, 0.0
    for n in range(1, steps + 1):
        st, F = toy.step(st, n, A, om, ref)
        J = J + gF[n - 1] * F
    full = torch.autograd.grad(J, [A, om, ref])
    rv = AD.Reverser(toy, (A.detach(), om.detach(), ref.detach()), gF, snapshots)
    with torch.no_grad():
        st = x0
        for n in range(1, steps + 1):
            st, _ = toy.step(st, n, A, om, ref)
    rv.lam = [torch.zeros_like(v) for v in st]
    rv.reverse(x0, 0, steps, snapshots - 1)
    for a, b in zip(rv.grad, full):
        assert torch.allclose(a, b, rtol=1e-12, atol=1e-14)
    assert rv.max_live <= snapshots
    if steps == 400:
        assert rv.recomputed <= 3 * steps         # binomial schedule: 969 advances for 400 steps


def test_pseudo_inverse_agrees_with_the_solve_on_consistent_vectors(tiny):
    """For g = A v the projected pseudo-inverse and the forward solve agree on T."""
    m = tiny
    rng = np.random.default_rng(0)
    v = torch.from_numpy(rng.standard_normal(m.NE)) * m.free
    Av = m.matvec(v)
    x = m.solve(Av, torch.zeros(m.NE, dtype=torch.float64)) * m.free
    z = m.pinv(Av)
    Tx, Tz = m._T(x), m._T(z)
    assert float(torch.linalg.norm(Tz - Tx)) <= 1e-9 * float(torch.linalg.norm(Tx))


def test_one_step_adjoint_matches_finite_differences(tiny):
    m = tiny
    A = torch.tensor(TINY.amplitude, dtype=torch.float64)
    om = torch.tensor(TINY.omega, dtype=torch.float64)
    ref = m.ref0.clone()
    with torch.no_grad():
        st = m.initial_state(A, om, ref)
        for n in range(1, 3):
            st, _ = m.step(st, n, A, om, ref)
    rng = np.random.default_rng(0)
    W = [torch.from_numpy(rng.standard_normal(x.shape)) for x in st]

    def obj(state, A_, om_, ref_):
        out, F = m.step(state, 3, A_, om_, ref_)
        return sum((o * w).sum() for o, w in zip(out, W)) + 0.7 * F

    inp = [x.clone().requires_grad_(True) for x in st]
    pa = [A.clone().requires_grad_(True), om.clone().requires_grad_(True), ref.clone().requires_grad_(True)]
    g = torch.autograd.grad(obj(inp, *pa), inp + pa)
    for i, name in ((4, "A"), (6, "ref")):
        base = (inp + pa)[i].detach()
        d = torch.from_numpy(rng.standard_normal(base.shape)) if base.dim() > 0 else torch.tensor(1.0, dtype=torch.float64)
        if name == "s":
            d = d * m.free
        e = 1e-6 * (float(base.abs().max()) if base.dim() > 0 else abs(float(base)))
        if name == "ref":
            # a unit direction and a step of 1e-6 h: the Roma-Peskin kernel's second
            # derivative jumps at |r| = h/2 and 3h/2, so a longer step across a jump
            # would carry a difference error proportional to the step
            d = d / torch.linalg.norm(d)
            e = 1e-6 * m.h0
        vals = []
        for sgn in (1.0, -1.0):
            args = [x.detach() for x in inp] + [p.detach() for p in pa]
            args[i] = base + sgn * e * d
            with torch.no_grad():
                vals.append(float(obj(args[:4], *args[4:])))
        fd = (vals[0] - vals[1]) / (2 * e)
        an = float((g[i] * d).sum())
        assert abs(an - fd) <= 1e-6 * abs(fd), (name, an, fd)
