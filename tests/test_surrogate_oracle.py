"""Pin of the surrogate's CPU oracle: its hand-derived backward pass must
match finite differences of its forward pass (float64, no BF16 rounding)."""
import numpy as np

import __graft_entry__
from oracle import surrogate_oracle as so

pkg = __graft_entry__.load_package()


def test_oracle_backward_matches_finite_differences():
    H, W, B = 5, 4, 2
    rng = np.random.default_rng(1)
    params = pkg.surrogate.init_params(seed=3)
    x = rng.standard_normal((B, H * W, so.N_IN))
    target = rng.standard_normal((B, H * W, so.N_OUT))
    ora = so.Oracle(H, W, bf16=False)
    out, saved = ora.forward(params, x)
    grads = ora.backward(params, saved, out, target)
    direction = {k: rng.standard_normal(v.shape) for k, v in params.items()}
    eps = 1e-6
    plus = {k: v + eps * direction[k] for k, v in params.items()}
    minus = {k: v - eps * direction[k] for k, v in params.items()}
    fd = (ora.loss(ora.forward(plus, x)[0], target) -
          ora.loss(ora.forward(minus, x)[0], target)) / (2 * eps)
    an = sum(float((grads[k] * direction[k]).sum()) for k in params)
    assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (fd, an)
    # and per parameter block, so a wrong block cannot hide behind the others
    for name in ("W_in", "b_in", "W0", "R1", "b3", "W_p1", "b_p2"):
        d = {k: (direction[k] if k == name else np.zeros_like(v)) for k, v in params.items()}
        p1 = {k: v + eps * d[k] for k, v in params.items()}
        m1 = {k: v - eps * d[k] for k, v in params.items()}
        fd1 = (ora.loss(ora.forward(p1, x)[0], target) -
               ora.loss(ora.forward(m1, x)[0], target)) / (2 * eps)
        an1 = float((grads[name] * direction[name]).sum())
        assert abs(fd1 - an1) <= 1e-6 * max(1.0, abs(an1)), (name, fd1, an1)


def test_bases_are_separable_fourier_products():
    F, G = so.bases(6, 5)
    Fp, Gp = pkg.surrogate.bases(6, 5)
    np.testing.assert_allclose(F, Fp, rtol=0, atol=1e-15)
    np.testing.assert_allclose(G, Gp, rtol=0, atol=1e-15)
    assert F.shape == (256, 30) and G.shape == (30, 256)
    # the constant mode averages
    np.testing.assert_allclose(F[0], np.full(30, 1 / 30))
