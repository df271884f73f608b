"""The CPU restatement of the threshold predictor's network (oracle/mlp_ref.py) against central finite
differences of its own loss: the checker the GPU gradients are compared with is itself right."""
import numpy as np
import pytest

from oracle import mlp_ref


@pytest.mark.parametrize("tau", [0.0, 0.05], ids=["mse", "pinball"])
def test_mlp_ref_gradient_matches_finite_differences(tau):
    rng = np.random.default_rng(5)
    din, h, B = 7, 5, 9
    n = din * h + h + h * h + h + h + 1
    p = rng.standard_normal(n) * 0.5
    X = rng.standard_normal((B, din))
    t = rng.standard_normal(B)
    _, g = mlp_ref.loss_and_grad(p, X, t, din, h, tau)
    eps = 1e-6
    num = np.zeros(n)
    for i in range(n):
        e = np.zeros(n)
        e[i] = eps
        num[i] = (mlp_ref.loss_and_grad(p + e, X, t, din, h, tau)[0] -
                  mlp_ref.loss_and_grad(p - e, X, t, din, h, tau)[0]) / (2 * eps)
    assert np.allclose(g, num, rtol=1e-6, atol=1e-8)
