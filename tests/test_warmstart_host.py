"""Host-side pieces of the learned warm start (no GPU): the coarse-to-fine
bilinear interpolation of predicted fields and the widened sweep draws."""
import numpy as np

from tests import cases

WS = cases.pkg.warmstart


def test_upsample_reproduces_bilinear_fields():
    """A field linear in (z, y) is interpolated exactly from a 100 x 40 grid
    onto 400 x 160 (rows past the coarse grid's last keep its values)."""
    Hc, Wc = 100, 41
    z = np.arange(Hc) / Hc
    y = np.arange(Wc) / (Wc - 1)
    f = np.stack([(k + 1) * z[:, None] - 0.5 * k * y[None, :] for k in range(8)], -1)
    g = WS.upsample_fields(f, 400, 160)
    assert g.shape == (400, 161, 8)
    zf = np.minimum(np.arange(400) / 400, (Hc - 1) / Hc)
    yf = np.arange(161) / 160
    for k in range(8):
        want = (k + 1) * zf[:, None] - 0.5 * k * yf[None, :]
        np.testing.assert_allclose(g[..., k], want, rtol=0, atol=1e-13)


def test_upsample_same_grid_is_identity():
    rng = np.random.default_rng(1)
    f = rng.standard_normal((40, 17, 8))
    np.testing.assert_allclose(WS.upsample_fields(f, 40, 16), f, rtol=0, atol=1e-14)


def test_widened_draws_keep_the_sweep_box_stream():
    """a_max only rescales the wall amplitude: every other parameter of a
    draw is the sweep box's, and a stays within [0, a_max)."""
    for seed in range(20):
        p = WS.draws([seed], (100, 40))[0]
        q = WS.draws([seed], (100, 40), a_max=0.35)[0]
        assert (p.amp, p.beta, p.vz) == (q.amp, q.beta, q.vz)
        assert q.a == p.a * 0.35 / 0.2 or abs(q.a - p.a * 1.75) < 1e-15
        assert 0.0 <= q.a < 0.35


def test_interpolation_onto_a_coarser_grid_is_exact_for_linear_fields():
    """A 400 x 160 prediction sampled onto a 200 x 80 draw (the sweep's finer
    surrogate used for a coarser grid) keeps a field linear in (z, y)."""
    Hc, Wc = 400, 161
    z = np.arange(Hc) / Hc
    y = np.arange(Wc) / (Wc - 1)
    f = np.stack([(k + 1) * z[:, None] + 0.25 * k * y[None, :] for k in range(8)], -1)
    g = WS.upsample_fields(f, 200, 80)
    assert g.shape == (200, 81, 8)
    zf, yf = np.arange(200) / 200, np.arange(81) / 80
    for k in range(8):
        np.testing.assert_allclose(g[..., k], (k + 1) * zf[:, None] + 0.25 * k * yf[None, :],
                                   rtol=0, atol=1e-13)


def test_each_draw_takes_the_surrogate_trained_nearest_its_grid():
    class Net:
        def __init__(self, H):
            self.H, self.W = H, H // 4 + 1

    class Tr:
        def __init__(self, H):
            self.net = Net(H)

    trs = [Tr(100), Tr(400)]
    assert [WS.nearest_surrogate(trs, L) for L in (100, 200, 400, 800)] == [0, 1, 1, 1]
    assert WS.nearest_surrogate([Tr(100)], 800) == 0
    assert [WS.nearest_surrogate([Tr(400), Tr(100)], L) for L in (100, 200)] == [1, 0]


def test_plain_sample_has_the_sweeps_grid_mix():
    params = [WS.sweep_params(i) for i in range(256)]
    idx = WS.stratified_sample(params, 32)
    assert len(idx) == 32 and len(set(idx)) == 32 and idx == sorted(idx)
    from collections import Counter
    full = Counter((p.L, p.M) for p in params)
    got = Counter((params[i].L, params[i].M) for i in idx)
    for g, c in full.items():
        assert abs(got[g] - 32 * c / 256) < 1.0
    # each grid's first draws
    for g in full:
        mine = [i for i in idx if (params[i].L, params[i].M) == g]
        first = [i for i, p in enumerate(params) if (p.L, p.M) == g][:len(mine)]
        assert mine == first
