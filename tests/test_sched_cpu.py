"""The MLP CPU reference itself: analytic gradient vs finite differences."""
import numpy as np

import _mlp_ref as ref


def test_reference_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.3, ref.NPARAMS)
    X = rng.normal(0, 1, (40, ref.NIN))
    T = rng.normal(0, 1, (40, ref.NOUT))
    T[rng.random(T.shape) < 0.2] = np.nan
    g = ref.grad(p, X, T)
    idx = rng.choice(ref.NPARAMS, 60, replace=False)
    assert np.allclose(g[idx], ref.fd_grad(p, X, T, idx), rtol=1e-5, atol=1e-8)
