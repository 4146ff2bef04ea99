"""The learned support-point proposal on the GPU against its CPU oracle.

* the training kernels (fp32 forward, backward, correlation loss): loss and
  every gradient against the float64 oracle;
* the tcgen05 inference path: against the oracle's bf16 forward pass;
* the pooled features: bit-exact;
* the learned support sweep: given the GPU's bins, the candidate lattice is
  bit-exact with the oracle's restatement, and the settled / fallback
  counts agree;
* what the trained network gains over the plain sweep and over untrained
  weights on held-out pairs.
"""
import os

import numpy as np
import pytest

import elas_b200 as eb
import oracle
import proposal_oracle as po

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t

    return t


def test_training_gradients_match_oracle(torch):
    import proposal

    rng = np.random.default_rng(5)
    hd, wd, D = 6, 24, 63
    xL = po.bf16_round(rng.normal(0, 1, (hd, wd, po.CH)))
    xR = po.bf16_round(rng.normal(0, 1, (hd, wd, po.CH)))
    lab = np.stack([rng.integers(4, wd, 12), rng.integers(0, hd, 12), rng.integers(0, 16, 12)], axis=1)
    theta = po.init_params(7).astype(np.float64)
    theta[po.TAPS * po.CH * po.CH:po.LAYER_PARAMS] = rng.normal(0, 0.1, po.CH)   # non-zero biases
    ref_loss, ref_g, ref_hits = po.loss_and_grad(xL, xR, lab, theta, D)

    net = proposal.Net(torch, hd, wd, 1)
    x = torch.from_numpy(np.stack([xL, xR]).astype(np.float32)).cuda()
    th = torch.from_numpy(theta.astype(np.float32)).cuda()
    g = torch.zeros_like(th)
    labels = torch.from_numpy(np.concatenate([np.zeros((12, 1), np.int64), lab], 1).astype(np.int32)).cuda()
    loss_sum, hits = net.forward_backward(th, g, x, labels, 1, D)
    assert abs(loss_sum / 12 - ref_loss) <= 1e-4 * abs(ref_loss)
    assert hits == ref_hits
    gg = g.cpu().numpy().astype(np.float64)
    scale = np.abs(ref_g).max()
    assert np.abs(gg - ref_g).max() <= 1e-4 * scale, np.abs(gg - ref_g).max() / scale
    for l in range(po.LAYERS):   # every layer's block, relative to its own size
        sl = slice(l * po.LAYER_PARAMS, (l + 1) * po.LAYER_PARAMS)
        assert np.abs(gg[sl] - ref_g[sl]).max() <= 1e-3 * np.abs(ref_g[sl]).max() + 1e-9


@pytest.mark.parametrize("hd,wd", [(5, 300), (3, 64), (4, 128), (2, 257)])
def test_tensor_core_inference_matches_oracle(torch, hd, wd):
    rng = np.random.default_rng(hd * 1000 + wd)
    theta = po.init_params(11).astype(np.float64)
    for l in range(po.LAYERS):
        o = l * po.LAYER_PARAMS + po.TAPS * po.CH * po.CH
        theta[o:o + po.CH] = rng.normal(0, 0.1, po.CH)
    x = po.bf16_round(rng.normal(0, 1, (2, hd, wd, po.CH)))
    ref = po.net_fwd(x, po.unpack(theta), round_bf16=True)[-1]
    e = eb.Elas(eb.params_config(255))
    e.set_proposal(theta.astype(np.float32))
    xin = torch.from_numpy(x.astype(np.float32)).to(torch.bfloat16).cuda()
    out = torch.empty_like(xin)
    e.pn_infer(xin.data_ptr(), out.data_ptr(), hd, wd)
    got = out.float().cpu().numpy().astype(np.float64)
    e.close()
    err = np.abs(got - ref)
    assert err.max() <= 2e-2 * np.abs(ref).max(), err.max() / np.abs(ref).max()
    assert err.mean() <= 2e-3 * np.abs(ref).mean()


def test_features_bit_exact():
    L, R, _, _ = eb.synth_pair(0, 21)
    e = eb.Elas(eb.params_config(63))
    e.set_proposal(po.init_params(1))
    e.process(L, R)
    H, W = L.shape
    hd, wd = H // 4, W // 4
    dl = e.stage("desc_left").reshape(H, W, 16)
    dr = e.stage("desc_right").reshape(H, W, 16)
    f = eb.bf16_to_f32(e.stage("pn_features")).reshape(2, hd, wd, 32)
    e.close()
    assert np.array_equal(f[0], po.features(dl).astype(np.float32))
    assert np.array_equal(f[1], po.features(dr).astype(np.float32))


def _weights_or_random():
    if os.path.exists(eb.PN_WEIGHTS):
        return eb.load_proposal()
    return po.init_params(2)


@pytest.mark.parametrize("preset,seed", [(0, 31), (1, 32)])
def test_learned_support_matches_oracle(preset, seed):
    L, R, _, _ = eb.synth_pair(preset, seed)
    W, H, D = eb.synth_dims(preset)
    p = eb.params_config(D)
    e = eb.Elas(p)
    e.set_proposal(_weights_or_random())
    e.process(L, R)
    step = p.candidate_stepsize
    ch, cw = H // step, W // step
    can_lr = e.stage("can_lr").view(np.int32).reshape(ch, cw)
    bins = e.stage("pn_bins").view(np.uint32).reshape(ch, cw)
    dl = e.stage("desc_left").reshape(H, W, 16)
    dr = e.stage("desc_right").reshape(H, W, 16)
    settled, fell = e.proposal_stats()
    e.close()
    _, _, o = oracle.process(L, R, p, dumps=True)
    exp, s_ref, f_ref = po.learned_can_lr(dl, dr, bins, o["can_lr"], p)
    assert (settled, fell) == (s_ref, f_ref)
    assert np.array_equal(can_lr, exp), np.count_nonzero(can_lr != exp)


def _quality(D1, gt):
    valid = np.isfinite(gt) & (gt > 0)
    bad = (np.abs(D1 - gt) > 2) | (D1 < 0)
    return float(bad[valid].mean())


def test_trained_proposal_gain():
    """Held-out pairs: the trained network settles most candidates (untrained
    weights settle far fewer) at nearly the plain method's bad-2px."""
    if not os.path.exists(eb.PN_WEIGHTS):
        pytest.skip("no trained proposal weights in the package")
    seeds = [300000 + k for k in range(6)]
    p = eb.params_config(255)
    plain = eb.Elas(p)
    learned = eb.Elas(p)
    learned.set_proposal(eb.load_proposal())
    untrained = eb.Elas(p)
    untrained.set_proposal(po.init_params(0))
    fb_t, fb_u, bad_p, bad_l = [], [], [], []
    for s in seeds:
        L, R, gt, _ = eb.synth_pair(1, s)
        d_plain, _ = plain.process(L, R)
        d_learn, _ = learned.process(L, R)
        st, fl = learned.proposal_stats()
        fb_t.append(fl / max(st + fl, 1))
        untrained.process(L, R)
        st, fl = untrained.proposal_stats()
        fb_u.append(fl / max(st + fl, 1))
        bad_p.append(_quality(d_plain, gt))
        bad_l.append(_quality(d_learn, gt))
    for e in (plain, learned, untrained):
        e.close()
    print(f"fallback trained {np.mean(fb_t):.3f} untrained {np.mean(fb_u):.3f}; "
          f"bad-2px plain {np.mean(bad_p):.4f} learned {np.mean(bad_l):.4f}")
    assert np.mean(fb_t) < 0.5
    assert np.mean(fb_u) > np.mean(fb_t) + 0.1
    assert np.mean(bad_l) - np.mean(bad_p) < 0.01


@pytest.mark.parametrize("preset,seed", [(1, 33), (2, 34)])
def test_topk_bins_match_float64_scores(preset, seed):
    """The packed top-4 bins of every candidate, from the GPU's own network
    output: valid, distinct, as many as there are valid bins (up to four),
    and the four best of the float64 scores.  Where two scores lie within
    float rounding of each other either order is accepted, so the check
    compares the scores of the chosen bins, not the bin numbers."""
    L, R, _, _ = eb.synth_pair(preset, seed)
    W, H, D = eb.synth_dims(preset)
    p = eb.params_config(D)
    e = eb.Elas(p)
    e.set_proposal(_weights_or_random())
    e.process(L, R)
    step = p.candidate_stepsize
    ch, cw = H // step, W // step
    hd, wd = H // 4, W // 4
    F = eb.bf16_to_f32(e.stage("pn_output")).reshape(2, hd, wd, 32).astype(np.float64)
    bins = e.stage("pn_bins").view(np.uint32).reshape(ch, cw)
    e.close()
    sh = po.bin_shifts(D)
    cys = np.minimum(np.arange(ch) * step // 4, hd - 1)
    cxs = np.minimum(np.arange(cw) * step // 4, wd - 1)
    worst = 0.0
    for vc in range(ch):
        cy = cys[vc]
        xr = cxs[:, None] - sh[None, :]                       # (cw, 64)
        valid = xr >= 0
        s = po.SCALE * np.einsum("ck,cbk->cb", F[0, cy, cxs], F[1, cy, np.maximum(xr, 0)])
        s = np.where(valid, s, -np.inf)
        exp_sorted = -np.sort(-s, axis=1)[:, :po.TOPK]
        for ci in range(cw):
            got = po.unpack_bins(bins[vc, ci])
            nvalid = int(valid[ci].sum())
            assert len(got) == min(po.TOPK, nvalid)
            assert len(set(got)) == len(got)
            assert all(valid[ci, b] for b in got)
            gs = s[ci, got]
            es = exp_sorted[ci, :len(got)]
            tol = 1e-5 * (1.0 + np.abs(es))
            assert np.all(np.diff(gs) <= tol[1:]), (vc, ci, got, gs)
            if len(got):
                worst = max(worst, float(np.max(np.abs(gs - es) / tol)))
    assert worst <= 1.0, worst
