"""A CPU mirror of ``adjoint.CavityModel`` for the tests that run without a GPU.

Test infrastructure only.  The same differentiable model, with the two calls
that need the library replaced by NumPy: the PCG runs the device's recurrence
and mixed stopping test (``ib_driver_np.py:331-403``, tested every iteration)
on the assembled operator, and spreading sums with ``bincount`` in (marker,
offset) order.
"""
import numpy as np
import torch

from pyib_b200 import adjoint as AD
from pyib_b200.operators import Operators


class CpuCavityModel(AD.CavityModel):
    def __init__(self, case, **kw):
        kw.pop("device", None)
        super().__init__(case, device="cpu", **kw)

    def _setup_solver(self, device):
        self.dev = torch.device("cpu")
        self.solver = None
        ops = Operators(self.lay)
        prec = ops.prec(ops.dir_mask(True))
        A = ops.R @ sum(ops.I[q] @ ops.V(self.rou, self.visc, self.dt) @ ops.P[q] for q in range(3)) @ ops.C
        self._free_idx = np.nonzero(prec != 0.0)[0]
        self._Aff = A.tocsr()[self._free_idx][:, self._free_idx]
        self._prec_f = prec[self._free_idx]
        return ops, prec

    def spread(self, cells32, w, ds3, f):
        c = cells32.cpu().numpy()
        ww = (w * ds3[:, None]).cpu().numpy().reshape(-1)
        fm = f.detach().cpu().numpy()
        out = np.stack([np.bincount(c, weights=np.repeat(fm[:, q], 125) * ww, minlength=self.NC)
                        for q in range(3)], axis=1)
        return torch.from_numpy(out)

    def solve(self, res_e, s):
        x = s.detach().cpu().numpy().copy()
        xf = x[self._free_idx]
        r = res_e.detach().cpu().numpy()[self._free_idx].copy()
        mdiag = self._prec_f
        y = np.zeros_like(r)
        z = r * mdiag
        p = z.copy()
        eta = z @ r
        thresh = (xf @ xf + 1e-16) * self.tol1 ** 2 + self.tol2 ** 2 * eta
        for _ in range(self.cg_max):
            if not eta >= thresh:
                break
            w = self._Aff @ p
            alf = eta / (p @ w)
            y += alf * p
            r -= alf * w
            z = r * mdiag
            eta_new = z @ r
            p = z + (eta_new / eta) * p
            eta = eta_new
            self.solve_iterations += 1
        x[self._free_idx] = xf + y
        return torch.from_numpy(x)

    def matvec(self, x):
        out = torch.zeros_like(x)
        out[self._free_idx] = torch.from_numpy(self._Aff @ x.detach().cpu().numpy()[self._free_idx])
        return out
