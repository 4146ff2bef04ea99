"""CPU float64 restatement of the learned support-point proposal.

TEST INFRASTRUCTURE ONLY: imported by tests/ (and the bench's CPU leg), never
by the library.  The library computes all of this on the GPU
(csrc/k_proposal.cu); this module is the checker it is compared with.

The reference has no learned component (its support matching is the full
disparity sweep, src/Kernels/KerSupportMatches.cu:12-193); the proposal is
this project's addition and its definition lives here and in
csrc/k_proposal.cu, restated identically:

* Input, per view: the 16-byte descriptors pooled over 4x4 pixel blocks into
  Hd x Wd = (H//4) x (W//4) cells of 32 channels -- channel c < 16 is
  (mean_c - 128) / 64, channel 16 + c is mean|byte_c - 128| / 64 -- rounded
  to bf16 (round to nearest even).
* Network (shared by both views): four 3x3 convolutions, 32 -> 32 channels,
  zero padding, bias, ReLU after the first three.  Parameters, per layer:
  W[tap][ci][co] (tap = 3*(dy+1) + (dx+1)) then b[co]; 4 * 9248 = 36992.
* Scores of cell (x, y) of the left view: 64 disparity bins of width
  w = ceil((D+1)/64) pixels; bin b compares with the right-view cell
  x - s_b, s_b = (b*w + w//2) // 4 (the bin centre in cells):
  score_b = 0.125 * <F_L(x, y), F_R(x - s_b, y)>, bins with x - s_b < 0
  are invalid.
* Training loss: softmax cross-entropy of the scores at the cell of every
  support point (u, v, d) that plain ELAS accepted, target bin min(d // w, 63).
* Proposal: the 4 best valid bins (ties to the lower bin); the search set of
  a candidate is the union of [b*w - 2, b*w + w - 1 + 2] over them, clipped
  to the candidate's disparity range.
"""
import numpy as np

NBINS = 64
CH = 32
LAYERS = 4
TAPS = 9
SCALE = 0.125
TOPK = 4
MARGIN = 2
LAYER_PARAMS = TAPS * CH * CH + CH
NPARAMS = LAYERS * LAYER_PARAMS


def bf16_round(x):
    """Round to bf16 (nearest even) and return as float64."""
    f = np.asarray(x, np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def unpack(theta):
    """Flat parameter vector -> [(W (9, 32, 32), b (32,))] per layer."""
    theta = np.asarray(theta, np.float64)
    assert theta.size == NPARAMS
    out = []
    for l in range(LAYERS):
        p = theta[l * LAYER_PARAMS:(l + 1) * LAYER_PARAMS]
        out.append((p[:TAPS * CH * CH].reshape(TAPS, CH, CH), p[TAPS * CH * CH:]))
    return out


def pack(layers):
    return np.concatenate([np.concatenate([W.reshape(-1), b.reshape(-1)]) for W, b in layers])


def init_params(seed=0):
    """He-style initialisation (what the training starts from)."""
    rng = np.random.default_rng(seed)
    layers = []
    for _ in range(LAYERS):
        W = rng.normal(0.0, np.sqrt(2.0 / (TAPS * CH)), (TAPS, CH, CH))
        layers.append((W, np.zeros(CH)))
    return pack(layers).astype(np.float32)


def features(desc):
    """desc (H, W, 16) uint8 -> (H//4, W//4, 32) bf16-rounded features (float64)."""
    H, W = desc.shape[:2]
    Hd, Wd = H // 4, W // 4
    blk = desc[:Hd * 4, :Wd * 4].astype(np.int64).reshape(Hd, 4, Wd, 4, 16)
    s = blk.sum(axis=(1, 3))
    a = np.abs(blk - 128).sum(axis=(1, 3))
    m = s.astype(np.float64) / 16.0
    f = np.concatenate([(m - 128.0) / 64.0, a.astype(np.float64) / 1024.0], axis=-1)
    return bf16_round(f)


def _shift(x, dy, dx):
    """y[..., i, j, :] = x[..., i+dy, j+dx, :] with zeros outside."""
    out = np.zeros_like(x)
    H, W = x.shape[-3], x.shape[-2]
    ys, yd = (slice(dy, H), slice(0, H - dy)) if dy >= 0 else (slice(0, H + dy), slice(-dy, H))
    xs, xd = (slice(dx, W), slice(0, W - dx)) if dx >= 0 else (slice(0, W + dx), slice(-dx, W))
    out[..., yd, xd, :] = x[..., ys, xs, :]
    return out


TAP_OFFSETS = [(dy, dx) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]


def conv_fwd(x, W, b, relu):
    """x (..., H, W, 32) -> y = act(sum_taps shift(x) @ W[tap] + b)."""
    y = np.zeros(x.shape[:-1] + (CH,))
    for t, (dy, dx) in enumerate(TAP_OFFSETS):
        y += _shift(x, dy, dx) @ W[t]
    y += b
    return np.maximum(y, 0.0) if relu else y


def conv_bwd(x, y, W, dy_out, relu):
    """Gradients of conv_fwd: returns dx, dW, db (dy_out is dL/dy after the activation)."""
    g = dy_out * (y > 0) if relu else dy_out
    dW = np.zeros_like(W)
    dx = np.zeros_like(x)
    flat_g = g.reshape(-1, CH)
    for t, (dy, dx_) in enumerate(TAP_OFFSETS):
        xs = _shift(x, dy, dx_)
        dW[t] = xs.reshape(-1, CH).T @ flat_g
        # y[i] += x[i + off] W  =>  dx[j] += g[j - off] W^T
        dx += _shift(g @ W[t].T, -dy, -dx_)
    db = flat_g.sum(axis=0)
    return dx, dW, db


def net_fwd(x, layers, round_bf16=False):
    """Activations [x, a1, a2, a3, F]; round_bf16 mimics the inference path
    (bf16 weights and activations, fp32 biases)."""
    acts = [x]
    for l, (W, b) in enumerate(layers):
        Wl = bf16_round(W) if round_bf16 else W
        y = conv_fwd(acts[-1], Wl, b, relu=l < LAYERS - 1)
        acts.append(bf16_round(y) if round_bf16 else y)
    return acts


def bin_width(D):
    return (D + 1 + NBINS - 1) // NBINS


def bin_shifts(D):
    w = bin_width(D)
    return np.array([(b * w + w // 2) // 4 for b in range(NBINS)], np.int64)


def scores_at(FL, FR, cx, cy, D):
    """Scores (64,) and validity of left cell (cx, cy); FL/FR (Hd, Wd, 32)."""
    sh = bin_shifts(D)
    xr = cx - sh
    valid = xr >= 0
    s = np.zeros(NBINS)
    s[valid] = SCALE * (FR[cy, xr[valid]] @ FL[cy, cx])
    return s, valid


def label_cells(uvd, D, Hd, Wd):
    """Support points (u, v, d) -> (cx, cy, bin) training targets inside the cell grid."""
    w = bin_width(D)
    cx, cy = uvd[:, 0] // 4, uvd[:, 1] // 4
    keep = (cx < Wd) & (cy < Hd)
    return np.stack([cx[keep], cy[keep], np.minimum(uvd[keep, 2] // w, NBINS - 1)], axis=1)


def loss_and_grad(xL, xR, labels, theta, D):
    """Mean cross-entropy over labels and its gradient w.r.t. theta (float64).

    xL, xR: (Hd, Wd, 32) inputs; labels: (n, 3) (cx, cy, bin)."""
    layers = unpack(theta)
    aL = net_fwd(xL, layers)
    aR = net_fwd(xR, layers)
    FL, FR = aL[-1], aR[-1]
    sh = bin_shifts(D)
    dFL = np.zeros_like(FL)
    dFR = np.zeros_like(FR)
    n = len(labels)
    loss = 0.0
    correct = 0
    for cx, cy, tb in labels:
        s, valid = scores_at(FL, FR, cx, cy, D)
        if not valid[tb]:
            continue
        z = np.where(valid, s, -np.inf)
        zmax = z.max()
        e = np.where(valid, np.exp(z - zmax), 0.0)
        p = e / e.sum()
        loss -= np.log(p[tb])
        correct += int(np.argmax(np.where(valid, s, -np.inf)) == tb)
        g = p.copy()
        g[tb] -= 1.0
        g /= n
        for b in np.nonzero(valid)[0]:
            dFL[cy, cx] += SCALE * g[b] * FR[cy, cx - sh[b]]
            dFR[cy, cx - sh[b]] += SCALE * g[b] * FL[cy, cx]
    grads = []
    gL, gR = dFL, dFR
    for l in range(LAYERS - 1, -1, -1):
        W, b = layers[l]
        relu = l < LAYERS - 1
        dxL, dWL, dbL = conv_bwd(aL[l], aL[l + 1], W, gL, relu)
        dxR, dWR, dbR = conv_bwd(aR[l], aR[l + 1], W, gR, relu)
        grads.append((dWL + dWR, dbL + dbR))
        gL, gR = dxL, dxR
    return loss / max(n, 1), pack(grads[::-1]), correct


def topk_bins(s, valid, k=TOPK):
    """The k best valid bins, best first; ties go to the lower bin."""
    order = sorted([b for b in range(NBINS) if valid[b]], key=lambda b: (-s[b], b))
    return order[:k]


def search_set(bins, D, dmin, dmax):
    w = bin_width(D)
    out = set()
    for b in bins:
        for d in range(b * w - MARGIN, b * w + w + MARGIN):
            if dmin <= d <= dmax:
                out.add(d)
    return sorted(out)


# ---- the learned support sweep (restated from k_support_sweep<*, true>) ----

INF_E = 0x7FFFFFFF


def unpack_bins(word):
    """Packed bin set (one byte per bin, best first, 0xff = none) -> list."""
    out = []
    for r in range(TOPK):
        b = (int(word) >> (8 * r)) & 0xFF
        if b != 0xFF:
            out.append(b)
    return out


def _energy(selfd, othd, u, v, d, direction):
    uw = u + direction * d
    pairs = ((selfd[v - 2, u - 2], othd[v - 2, uw - 2]), (selfd[v - 2, u + 2], othd[v - 2, uw + 2]),
             (selfd[v + 2, u - 2], othd[v + 2, uw - 2]), (selfd[v + 2, u + 2], othd[v + 2, uw + 2]))
    return int(sum(np.abs(a.astype(np.int32) - b.astype(np.int32)).sum() for a, b in pairs))


def restricted_match(selfd, othd, u, v, dmin, dmax, direction, thr, bins, D):
    """Best disparity of the search set if it is attained once and
    (float)E1 < thr * (float)E2 (E2 over the other disparities), else -1."""
    S = search_set(bins, D, dmin, dmax)
    if not S:
        return -1
    E = [_energy(selfd, othd, u, v, d, direction) for d in S]
    e1 = min(E)
    if E.count(e1) != 1:
        return -1
    d1 = S[E.index(e1)]
    rest = [e for e, d in zip(E, S) if d != d1]
    e2 = min(rest) if rest else INF_E
    return d1 if np.float32(e1) < np.float32(thr) * np.float32(e2) else -1


def texture(desc_px):
    return int(np.abs(desc_px.astype(np.int32) - 128).sum())


def learned_can_lr(descL, descR, bins, plain_can_lr, p):
    """Candidate lattice after both sweeps with the proposal: a candidate the
    search set settles (uniqueness and L/R tests passed on it) takes that
    disparity, every other candidate past the texture / range gate keeps the
    full sweep's result.  Returns (can_lr, settled, fell_back)."""
    H, W = descL.shape[:2]
    step = p.candidate_stepsize
    ch, cw = H // step, W // step
    D, dmin = p.disp_max, max(p.disp_min, 0)
    out = np.array(plain_can_lr, np.int32).reshape(ch, cw).copy()
    settled = fell = 0
    for vc in range(ch):
        v = vc * step
        if v < 5 or v > H - 6:
            continue
        for ci in range(cw):
            u = ci * step
            if u < 5 or u > W - 6 or texture(descL[v, u]) < p.support_texture:
                continue
            dmax = min(D, u - 5)
            if dmax - dmin < 10:
                continue
            b = unpack_bins(bins[vc, ci])
            ok = False
            rl = restricted_match(descL, descR, u, v, dmin, dmax, -1, p.support_threshold, b, D) if b else -1
            if rl >= 0:
                ur = u - rl
                dmaxr = min(D, W - ur - 5)
                if texture(descR[v, ur]) >= p.support_texture and dmaxr - dmin >= 10:
                    rr = restricted_match(descR, descL, ur, v, dmin, dmaxr, +1, p.support_threshold, b, D)
                    ok = rr >= 0 and abs(rl - rr) <= p.lr_threshold
            if ok:
                out[vc, ci] = rl
                settled += 1
            else:
                fell += 1
    return out, settled, fell
