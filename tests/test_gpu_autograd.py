"""torch.autograd wrapper and VQE driver over the adjoint C-ABI."""
import numpy as np
import pytest
import torch

from kettle_b200 import workloads as W
from kettle_b200.autograd import CircuitEnergy, Problem, vqe

pytestmark = pytest.mark.gpu


def test_autograd_matches_finite_differences(engine):
    n = 8
    gates, params = W.hea(n, 2, seed=4)
    strings, coeffs = W.xxz_chain(n, seed=4)
    prob = Problem(n, gates, strings, coeffs)
    x = torch.tensor(params, dtype=torch.float64, requires_grad=True)
    e = CircuitEnergy.apply(x, prob)
    e.backward()
    h = 1e-5
    fd = np.array([(prob.energy(params + h * np.eye(params.size)[k]) - prob.energy(params - h * np.eye(params.size)[k]))
                   / (2 * h) for k in range(params.size)])
    assert abs(e.item() - prob.energy(params)) < 1e-12
    assert np.abs(x.grad.numpy() - fd).max() < 1e-8
    prob.close()


def test_vqe_lowers_the_energy(engine):
    n = 6
    gates, params = W.hea(n, 2, seed=5)
    strings, coeffs = W.xxz_chain(n, seed=5)
    prob = Problem(n, gates, strings, coeffs)
    e0 = prob.energy(params)
    best, x, hist = vqe(prob, params, iterations=30)
    assert best < e0 - 0.5
    assert abs(prob.energy(x) - best) < 1e-10
    prob.close()
