"""The surrogate network on the GPU (tcgen05 BF16 GEMMs, FP32 element-wise
kernels) against its CPU oracle with the same BF16 operand rounding:
forward output, loss and every parameter gradient; and Adam training that
lowers the loss."""
import numpy as np
import pytest

import __graft_entry__
from oracle import surrogate_oracle as so

pytestmark = pytest.mark.gpu
pkg = __graft_entry__.load_package()


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def setup(H=12, W=9, B=2, seed=0):
    import torch
    rng = np.random.default_rng(seed)
    params = pkg.surrogate.init_params(seed=seed + 1)
    x = rng.standard_normal((B, H * W, so.N_IN))
    target = rng.standard_normal((B, H * W, so.N_OUT))
    net = pkg.surrogate.SpectralOperator(H, W, B, params=params)
    net.load_inputs(x)
    tgt = torch.from_numpy(target.reshape(-1, so.N_OUT).astype(np.float32)).cuda()
    return params, x, target, net, tgt


def test_forward_and_gradients_match_oracle():
    params, x, target, net, tgt = setup()
    out = net.forward()
    net.loss_and_grad(tgt)
    net.backward()
    net.wait()
    ora = so.Oracle(12, 9, bf16=True)
    # the oracle sees the parameters as the GPU holds them (FP32)
    p32 = {k: v.astype(np.float32).astype(np.float64) for k, v in params.items()}
    x32 = x.astype(np.float32).astype(np.float64)
    t32 = target.astype(np.float32).astype(np.float64)
    o_out, saved = ora.forward(p32, x32)
    got = out.cpu().numpy().reshape(o_out.shape)
    assert rel(got, o_out) < 1e-2
    assert abs(float(net.loss.cpu()[0]) - ora.loss(got, t32)) <= 1e-6 * ora.loss(got, t32)
    o_g = ora.backward(p32, saved, o_out, t32)
    g = net.grads()
    for k in o_g:
        assert rel(g[k], o_g[k]) < 3e-2, (k, rel(g[k], o_g[k]))


def test_adam_training_lowers_the_loss():
    params, x, target, net, tgt = setup(H=10, W=8, B=2, seed=4)
    losses = []
    for _ in range(60):
        net.forward()
        net.loss_and_grad(tgt)
        net.backward()
        net.adam_step(lr=2e-3)
        losses.append(float(net.loss.cpu()[0]))
    net.wait()
    assert losses[-1] < 0.5 * losses[0], losses[::10]


def test_trained_warm_start_beats_cold_start():
    """What the trained network gains: on held-out parameter draws the plain
    time march converges (L-inf residual <= 1e-8) in fewer steps from the
    surrogate's prediction than from the workload's initial condition, and
    to the same steady state."""
    res = pkg.warmstart.run_pipeline(n_train=160, n_eval=12, grid=(40, 16), epochs=40,
                                     plain_sample=2, log=lambda s: None)
    assert res["both_converged"] >= 6, res["both_converged"]
    assert res["warm_converged"] >= res["cold_converged"]
    assert res["warm_steps_both"] < 0.7 * res["cold_steps_both"], \
        (res["warm_steps_both"], res["cold_steps_both"])
    # both runs stop at residual 1e-8, which leaves each about 1e-5 from the
    # exact fixed point of the scheme; they agree to that level
    assert max(res["warm_vs_cold_state_rel_linf_max"]) < 1e-4


def test_untrained_surrogate_falls_back_to_cold_start():
    """A deliberately poor surrogate (an untrained network): the plain march
    stays the judge.  Its predictions get a small step budget; every solve
    that does not reach the residual within it is solved again from the
    workload's initial condition and then ends exactly as the cold solve
    (same bits, same convergence), with both attempts' steps counted."""
    WS, S = pkg.warmstart, pkg.surrogate
    grid = (40, 16)
    params = WS.draws(range(1_000_000, 1_000_006), grid)
    cold = WS.solve_all(params, max_steps=200_000, tol=1e-8)
    assert cold.converged.all()
    Y = np.stack([f.reshape(-1, S.N_OUT) for f in cold.fields])
    net = S.SpectralOperator(grid[0], grid[1] + 1, 16, seed=3)   # never trained
    floor = np.array([0.05 * Y[..., 0].min(), 0.05 * Y[..., 4].min()])
    tr = WS.Trained(net, S.Normalizer.fit(Y), [], 0.0, floor)
    ics, _ = WS.predicted_ics(tr, params, grid, floor)
    budget = int(0.1 * np.median(cold.steps))
    warm, fell = WS.solve_warm(params, ics, max_steps=200_000, tol=1e-8, budget=budget)
    assert fell.sum() >= len(params) // 2, fell
    for i in np.flatnonzero(fell):
        assert warm.converged[i] and warm.steps[i] >= cold.steps[i]
        np.testing.assert_array_equal(warm.fields[i], cold.fields[i])
    for i in np.flatnonzero(~fell):
        assert warm.converged[i] and warm.steps[i] <= budget


def test_each_draw_is_predicted_by_the_nearest_surrogate():
    """Two surrogates on different grids (untrained: only the routing is
    checked): each draw's prediction comes from the one trained nearest its
    grid and is interpolated onto the draw's own grid, so it equals that
    surrogate's prediction alone, in the draw's shape."""
    WS, S = pkg.warmstart, pkg.surrogate
    rng = np.random.default_rng(0)
    Y = rng.standard_normal((4, 1, S.N_OUT)) * 0.1 + 1.0
    trs = []
    for H, W in ((24, 11), (96, 41)):
        net = S.SpectralOperator(H, W, 16, seed=H)
        trs.append(WS.Trained(net, S.Normalizer.fit(Y), [], 0.0, np.array([1e-3, 1e-3])))
    params = [WS.SweepParams(L, M, 1.0, 0.2, 0.1, 0.05)
              for L, M in ((24, 10), (48, 20), (96, 40), (192, 80))]
    ics, _, pick = WS.predicted_ics_nearest(trs, params)
    assert pick == [0, 1, 1, 1]
    for p, ic, k in zip(params, ics, pick):
        alone, _ = WS.predicted_ics(trs[k], [p], None, trs[k].floor)
        if alone[0] is None:
            assert ic is None
            continue
        assert ic.shape == alone[0].shape
        np.testing.assert_array_equal(ic, alone[0])
