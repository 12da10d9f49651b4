"""The FP64 guide oracle's analytic gradients against central finite
differences of its own loss (the guide has no counterpart in the reference,
so the oracle is pinned by calculus)."""
import numpy as np

import guide_oracle as G


def _setup(seed=0, n=6):
    rng = np.random.default_rng(seed)
    grid = rng.uniform(-0.5, 0.5, (G.LEVELS, G.T, G.FEAT))
    W = rng.uniform(-0.3, 0.3, (G.LAYERS, 64, 64))
    W[0][:, 43:] = 0
    b = rng.uniform(-0.1, 0.1, (G.LAYERS, 64))
    bmin, binv = np.zeros(3), np.ones(3) / 5.0
    recs = []
    for _ in range(n):
        x = rng.uniform(0.5, 4.5, 3)
        wo = rng.normal(size=3); wo /= np.linalg.norm(wo)
        nn = rng.normal(size=3); nn /= np.linalg.norm(nn)
        w = rng.normal(size=3); w /= np.linalg.norm(w)
        recs.append(np.concatenate([x, wo, nn, w, [rng.uniform(0.1, 2.0)]]))
    return grid, W, b, bmin, binv, recs


def test_weight_and_bias_gradients_match_finite_differences():
    grid, W, b, bmin, binv, recs = _setup()
    gW, gb, _ = G.gradients(grid, W, b, bmin, binv, recs)
    rng = np.random.default_rng(1)
    h = 1e-6
    for _ in range(12):
        l, o, i = rng.integers(0, G.LAYERS), rng.integers(0, 40 if rng.random() < 0.5 else 64), rng.integers(0, 43)
        Wp, Wm = W.copy(), W.copy()
        Wp[l, o, i] += h
        Wm[l, o, i] -= h
        fd = (G.loss(grid, Wp, b, bmin, binv, recs) - G.loss(grid, Wm, b, bmin, binv, recs)) / (2 * h)
        assert abs(fd - gW[l, o, i]) <= 1e-6 + 1e-4 * abs(fd), (l, o, i, fd, gW[l, o, i])
    for _ in range(6):
        l, o = rng.integers(0, G.LAYERS), rng.integers(0, 64)
        bp, bm = b.copy(), b.copy()
        bp[l, o] += h
        bm[l, o] -= h
        fd = (G.loss(grid, W, bp, bmin, binv, recs) - G.loss(grid, W, bm, bmin, binv, recs)) / (2 * h)
        assert abs(fd - gb[l, o]) <= 1e-6 + 1e-4 * abs(fd)


def test_grid_gradients_match_finite_differences():
    grid, W, b, bmin, binv, recs = _setup(seed=2, n=3)
    _, _, gg = G.gradients(grid, W, b, bmin, binv, recs)
    nz = np.argwhere(np.abs(gg) > 1e-6)
    rng = np.random.default_rng(3)
    h = 1e-6
    for j in rng.choice(len(nz), 8, replace=False):
        l, e, f = nz[j]
        gp, gm = grid.copy(), grid.copy()
        gp[l, e, f] += h
        gm[l, e, f] -= h
        fd = (G.loss(gp, W, b, bmin, binv, recs) - G.loss(gm, W, b, bmin, binv, recs)) / (2 * h)
        assert abs(fd - gg[l, e, f]) <= 1e-7 + 1e-4 * abs(fd)


def test_mixture_is_a_density():
    rng = np.random.default_rng(4)
    o = rng.normal(size=64)
    # Monte Carlo integral of q over the sphere ~ 1
    v = rng.normal(size=(200000, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    mus, kaps, pis = G.lobes(o)
    q = sum(pis[k] * kaps[k] / (2 * np.pi * (-np.expm1(-2 * kaps[k]))) * np.exp(kaps[k] * (v @ mus[k] - 1))
            for k in range(G.LOBES))
    assert abs(q.mean() * 4 * np.pi - 1) < 0.02


def test_bf16_rounding_is_nearest_even():
    import guide_oracle as G
    x = np.array([1.0, 1 + 2 ** -8, 1 + 3 * 2 ** -8, -(1 + 2 ** -7), 3.0e38, 1e-40])
    got = G.bf16(x)
    np.testing.assert_array_equal(got[:4], [1.0, 1.0, 1 + 2 ** -6, -(1 + 2 ** -7)])
    assert np.isfinite(got[4]) and abs(got[4] / 3.0e38 - 1) < 2 ** -8
    # BF16 keeps FP32's exponent range: tiny values are not flushed
    assert got[5] > 0


def test_selection_gradients_match_finite_differences():
    """Learned selection: the loss of the one-sample MIS density
    s q + (1 - s) p_bsdf; output 40 (the selection logit) and the lobes both
    get gradients."""
    grid, W, b, bmin, binv, recs = _setup(seed=4, n=5)
    rng = np.random.default_rng(5)
    recs = [np.concatenate([r, [rng.uniform(0.0, 2.0)]]) for r in recs]
    recs[0][13] = 0.0  # a direction the BSDF cannot sample
    b[4][40] = 0.3
    gW, gb, gg = G.gradients(grid, W, b, bmin, binv, recs, learn_select=True)
    h = 1e-6
    L = lambda W_, b_: G.loss(grid, W_, b_, bmin, binv, recs, learn_select=True)
    for o in (40, 3, 7, 12):
        bp, bm = b.copy(), b.copy()
        bp[4, o] += h
        bm[4, o] -= h
        fd = (L(W, bp) - L(W, bm)) / (2 * h)
        assert abs(fd - gb[4, o]) <= 1e-7 + 1e-4 * abs(fd), (o, fd, gb[4, o])
    for _ in range(8):
        l, o, i = rng.integers(0, G.LAYERS), rng.integers(0, 41), rng.integers(0, 43)
        Wp, Wm = W.copy(), W.copy()
        Wp[l, o, i] += h
        Wm[l, o, i] -= h
        fd = (L(Wp, b) - L(Wm, b)) / (2 * h)
        assert abs(fd - gW[l, o, i]) <= 1e-6 + 1e-4 * abs(fd), (l, o, i, fd, gW[l, o, i])
    assert abs(gb[4, 40]) > 1e-6


def test_gradients_where_every_lobe_density_underflows():
    """Sharp lobes (kappa up to 5000) far from the recorded direction: every
    vMF density underflows, but the log-space responsibilities keep the
    gradient finite and equal to finite differences of the log-space loss."""
    grid, W, b, bmin, binv, recs = _setup(seed=6, n=4)
    b[4][3:40:5] = 2000.0  # every lobe's kappa near 2000 (below the clamp)
    logq = [G.log_terms(G.forward(W, b, G.encode(grid, bmin, binv, r[0:3], r[3:6], r[6:9])[0])[0], r[9:12])[1]
            for r in recs]
    assert min(logq) < -745  # q itself underflows to 0 in FP64 for some record
    g = G.gradients(grid, W, b, bmin, binv, recs)
    assert all(np.isfinite(a).all() for a in g)
    h = 1e-6
    for o in (0, 1, 2, 3, 4, 8, 9):
        bp, bm = b.copy(), b.copy()
        bp[4, o] += h
        bm[4, o] -= h
        fd = (G.loss(grid, W, bp, bmin, binv, recs) - G.loss(grid, W, bm, bmin, binv, recs)) / (2 * h)
        assert abs(fd - g[1][4, o]) <= 1e-6 + 1e-4 * abs(fd), (o, fd, g[1][4, o])
