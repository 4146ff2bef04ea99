"""The CPU oracle of the learned proposal, pinned on its own terms.

There is no reference implementation of the proposal (the reference only has
the full sweep), so the float64 oracle is checked for internal consistency:
analytic gradients against central finite differences, the convolution
against a direct loop, the search-set rule on hand-made cases.
"""
import numpy as np

import proposal_oracle as po


def tiny_case(seed=0, Hd=5, Wd=14, D=63, nlab=6):
    rng = np.random.default_rng(seed)
    xL = po.bf16_round(rng.normal(0, 1, (Hd, Wd, po.CH)))
    xR = po.bf16_round(rng.normal(0, 1, (Hd, Wd, po.CH)))
    cx = rng.integers(4, Wd, nlab)
    cy = rng.integers(0, Hd, nlab)
    lab = np.stack([cx, cy, rng.integers(0, 8, nlab)], axis=1)
    theta = po.init_params(seed).astype(np.float64)
    return xL, xR, lab, theta, D


def test_param_count():
    assert po.NPARAMS == 36992
    assert po.unpack(po.init_params())[0][0].shape == (9, 32, 32)


def test_conv_matches_direct_loop():
    rng = np.random.default_rng(1)
    x = rng.normal(0, 1, (4, 5, po.CH))
    W = rng.normal(0, 1, (9, po.CH, po.CH))
    b = rng.normal(0, 1, po.CH)
    y = po.conv_fwd(x, W, b, relu=False)
    ref = np.zeros_like(y)
    for i in range(4):
        for j in range(5):
            acc = b.copy()
            for t, (dy, dx) in enumerate(po.TAP_OFFSETS):
                ii, jj = i + dy, j + dx
                if 0 <= ii < 4 and 0 <= jj < 5:
                    acc += x[ii, jj] @ W[t]
            ref[i, j] = acc
    np.testing.assert_allclose(y, ref, rtol=1e-12, atol=1e-12)


def test_gradient_matches_finite_differences():
    xL, xR, lab, theta, D = tiny_case()
    loss, g, _ = po.loss_and_grad(xL, xR, lab, theta, D)
    assert np.isfinite(loss) and loss > 0
    rng = np.random.default_rng(2)
    idx = np.concatenate([rng.choice(po.NPARAMS, 24, replace=False),
                          [po.LAYER_PARAMS - 1, 2 * po.LAYER_PARAMS - 5, po.NPARAMS - 1]])
    eps = 1e-6
    for i in idx:
        tp = theta.copy()
        tm = theta.copy()
        tp[i] += eps
        tm[i] -= eps
        num = (po.loss_and_grad(xL, xR, lab, tp, D)[0] - po.loss_and_grad(xL, xR, lab, tm, D)[0]) / (2 * eps)
        assert abs(num - g[i]) <= 1e-6 + 1e-4 * abs(num), (i, num, g[i])


def test_bins_and_search_set():
    assert po.bin_width(255) == 4 and po.bin_width(511) == 8 and po.bin_width(63) == 1
    assert list(po.bin_shifts(255)[:4]) == [0, 1, 2, 3]
    assert list(po.bin_shifts(511)[:3]) == [1, 3, 5]
    s = np.zeros(64)
    s[[5, 7, 9, 11, 40]] = [3.0, 5.0, 5.0, 1.0, 4.0]
    valid = np.ones(64, bool)
    valid[40] = False
    assert po.topk_bins(s, valid) == [7, 9, 5, 11]
    # bins 7 and 9 at width 4: [26, 33] and [34, 41] merge; clipped at dmax 36
    assert po.search_set([7, 9], 255, 0, 36) == list(range(26, 37))


def test_bf16_round_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 1.0 + 2 ** -9])
    r = po.bf16_round(x)
    assert list(r) == [1.0, 1.0, 1.0 + 2 ** -6, -2.5, 1.0]


def test_features_exact_values():
    desc = np.full((8, 8, 16), 128, np.uint8)
    desc[:4, :4, 0] = 192
    desc[:4, :4, 1] = 0
    f = po.features(desc)
    assert f.shape == (2, 2, 32)
    assert f[0, 0, 0] == 1.0 and f[0, 0, 1] == -2.0 and f[0, 0, 16] == 1.0 and f[0, 0, 17] == 2.0
    assert f[1, 1, 0] == 0.0 and f[1, 1, 16] == 0.0
