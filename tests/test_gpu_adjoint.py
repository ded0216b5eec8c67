"""The discrete adjoint of the oscillating-sphere step on the GPU.

* The differentiable restatement of the step (``adjoint.CavityModel``) follows
  the product's device step: the same stream function, Lagrangian force and
  body force history, with the reference's CG tolerances.
* The gradient of the first-harmonic axial force amplitude with respect to the
  oscillation amplitude A, the period T and the reference marker positions,
  from the hand-written adjoint with binomial checkpointing (5 stored states for
  24 steps), agrees with central finite differences of the same model (step
  1e-6 relative for A and T, 1e-6 h along unit marker directions) to 1e-6
  relative.  The forward solves run to a 1e-13 mixed tolerance so that the
  differences resolve the gradient.
"""
import numpy as np
import pytest
import torch

from pyib_b200 import adjoint as AD
from pyib_b200.cases import SphereCase
from pyib_b200.runner import SphereRun

pytestmark = [pytest.mark.gpu, pytest.mark.filterwarnings("ignore::UserWarning")]

# D = 8 cells, 2 levels (half widths 2D, 4D), closed cavity, A = 0.2 D, Re0 = 1,
# 20 steps per period: 61,440 cells, 201 markers
CASE = SphereCase(name="adjoint_small", cells_per_diameter=8, half_widths_d=(2.0, 4.0), reynolds=1.0,
                  amplitude_d=0.2, steps_per_period=20)


def test_restated_step_follows_the_device_step():
    model = AD.CavityModel(CASE, tol=1e-10, tol2=1e-9)
    run = SphereRun(CASE)
    dev = model.dev
    A = torch.tensor(CASE.amplitude, dtype=torch.float64, device=dev)
    om = torch.tensor(CASE.omega, dtype=torch.float64, device=dev)
    ref = model.ref0.clone()
    with torch.no_grad():
        st = model.initial_state(A, om, ref)
        for n in range(1, 7):
            st, F = model.step(st, n, A, om, ref)
            load = run.advance()
            s_dev = np.asarray(run.s)
            s_m = st[0].cpu().numpy()
            assert np.linalg.norm(s_m - s_dev) <= 1e-10 * np.linalg.norm(s_dev), n
            fl = np.asarray(run.drv.ib_force_L)
            assert np.linalg.norm(st[2].cpu().numpy() - fl) <= 1e-10 * np.linalg.norm(fl), n
            assert abs(float(F) - float(load["body_force"][0])) <= 1e-9 * abs(float(load["body_force"][0])), n


def _rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def test_force_amplitude_gradient_matches_finite_differences():
    model = AD.CavityModel(CASE, tol=1e-13)
    steps, window = 24, 20
    A, T = CASE.amplitude, CASE.period
    ref = model.ref0.clone()
    J, gA, gT, gref, info = AD.force_amplitude_and_gradient(model, A, T, ref, steps, window, snapshots=5)
    assert info["max_stored_states"] <= 5
    eps = 1e-6
    fd = lambda a, t, r: AD.force_amplitude(model, a, t, r, steps, window)
    dA = eps * A
    fdA = (fd(A + dA, T, ref) - fd(A - dA, T, ref)) / (2 * dA)
    dT = eps * T
    fdT = (fd(A, T + dT, ref) - fd(A, T - dT, ref)) / (2 * dT)
    report = {"J": J, "dA": (gA, fdA), "dT": (gT, fdT)}
    rng = np.random.default_rng(0)
    step = eps * model.h0
    for q in range(2):
        d = rng.standard_normal(ref.shape)
        d /= np.linalg.norm(d)
        dt_ = torch.from_numpy(d).to(ref.device)
        fdm = (fd(A, T, ref + step * dt_) - fd(A, T, ref - step * dt_)) / (2 * step)
        report[f"dir{q}"] = (float(np.sum(gref * d)), fdm)
    print("adjoint", report, {k: v for k, v in info.items() if k != "force"})
    assert _rel(gA, fdA) <= 1e-6
    assert _rel(gT, fdT) <= 1e-6
    for q in range(2):
        g, f = report[f"dir{q}"]
        assert _rel(g, f) <= 1e-6
