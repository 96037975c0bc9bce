"""torch.autograd wrapper of the adjoint gradient, and a VQE driver.

`CircuitEnergy.apply(params, problem)` returns E(params) = Re <psi|H|psi> as a
float64 torch scalar whose backward pass is the engine's adjoint sweep
(kt_adjoint_forward / kt_adjoint_backward).  `vqe()` runs a parameter
optimisation on top of it: the cost function the reference's VQE example
evaluates (example/algorithms/vqe_basic.cpp:61-96: set parameters, simulate,
expectation value), here with an analytic gradient.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from . import capi


@dataclass
class Problem:
    """A parameterised circuit and a Hamiltonian on n qubits, bound to one device state."""

    n_qubits: int
    gates: np.ndarray
    strings: np.ndarray
    coeffs: np.ndarray
    dtype: int = capi.KT_C128
    checkpoint_every: int = 0
    _sv: capi.Statevector | None = field(default=None, repr=False)
    _adj: capi.Adjoint | None = field(default=None, repr=False)

    def handles(self):
        if self._sv is None:
            self._sv = capi.Statevector(self.n_qubits, self.dtype)
            self._adj = capi.Adjoint(self._sv, self.checkpoint_every)
        return self._sv, self._adj

    def energy_and_grad(self, params: np.ndarray):
        sv, adj = self.handles()
        sv.set_basis(0)
        e = adj.forward(self.gates, params, self.strings, self.coeffs)
        g = adj.backward()
        return e, g

    def energy(self, params: np.ndarray) -> float:
        sv, _ = self.handles()
        sv.set_basis(0)
        sv.apply(self.gates, params)
        _, total = sv.expect(self.strings, self.coeffs)
        return total.real

    def close(self):
        if self._adj is not None:
            self._adj.close()
        if self._sv is not None:
            self._sv.close()
        self._adj = self._sv = None


class CircuitEnergy(torch.autograd.Function):
    """E(params) with the adjoint gradient as its backward."""

    @staticmethod
    def forward(ctx, params: torch.Tensor, problem: Problem):
        p = params.detach().to("cpu", torch.float64).numpy()
        e, g = problem.energy_and_grad(p)
        ctx.save_for_backward(torch.from_numpy(g).to(params.device, params.dtype))
        return torch.tensor(e, dtype=torch.float64, device=params.device)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out * g, None


def vqe(problem: Problem, params0: np.ndarray, iterations: int = 50, method: str = "L-BFGS-B"):
    """Minimise E(params) for `iterations` optimiser iterations with scipy.

    The reference drives nlopt's derivative-free LN_COBYLA (vqe_basic.cpp:88);
    nlopt is not available here, so the loop uses scipy.optimize with the
    adjoint gradient ("COBYLA" is accepted too, without gradient).  Returns
    (best energy, best params, energies per evaluation)."""
    from scipy.optimize import minimize

    history = []

    def fun(x):
        if method.upper() == "COBYLA":
            e = problem.energy(x)
            history.append(e)
            return e
        e, g = problem.energy_and_grad(x)
        history.append(e)
        return e, g

    opts = {"maxiter": iterations}
    res = minimize(fun, np.asarray(params0, dtype=np.float64), jac=(method.upper() != "COBYLA"), method=method,
                   options=opts)
    return float(res.fun), np.asarray(res.x), history
