"""CPU: the float64 restatement of the picker network's gradients (the
oracle the GPU kernels are checked against) agrees with central finite
differences."""
import numpy as np

from oracle import mlp_ref


def test_reference_gradients_match_finite_differences():
    nin, h, nout, B = 5, 7, 4, 6
    rng = np.random.default_rng(0)
    n = nin * h + h + h * h + h + h * nout + nout
    p = rng.standard_normal(n) * 0.5
    x = rng.standard_normal((B, nin))
    t = rng.standard_normal((B, nout))
    loss, g = mlp_ref.loss_and_grads(p, x, t, nin, h, nout)
    eps = 1e-6
    for i in rng.choice(n, 40, replace=False):
        q = p.copy()
        q[i] += eps
        lp, _ = mlp_ref.loss_and_grads(q, x, t, nin, h, nout)
        q[i] -= 2 * eps
        lm, _ = mlp_ref.loss_and_grads(q, x, t, nin, h, nout)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])
