"""CPU oracle of the learned motion-vector proposals (test infrastructure only).

The reference has no learned component: this restates, in numpy, what the device computes for
the proposal network (libvc1_b200/csrc/vc1cu_lp.cu) so that the tests can check its features,
translation hint, candidates, loss and every gradient:

- quarter-resolution pictures (rounded 4x4 means, clamped at the picture edge);
- the translation hint, coarse to fine: the least 1/16-resolution SAD over [-R16, R16]^2, then
  the 7x7 quarter-resolution displacements about 4x that, then the 5x5 full-resolution vectors
  (SAD at stride 2) about 4x that, ties by (cost, |dx|+|dy|, dy, dx), clamped to the search range;
- the 16 input channels (bf16): cur, ref, ref shifted by the hint, their differences, cur's
  gradients, the hint / 64, zeros;
- four 3x3 convolutions (zero padding) with bias and ReLU, activations rounded to bf16 where the
  device stores them, weights rounded to bf16;
- per macroblock the mean of its 16 samples, the fp32 projection to (logit0, logit1, offsets),
  the candidates, the loss (two logistic terms and smooth-L1 offsets) and the backward pass,
  with the device's bf16 rounding of the stored gradients.

Parity with the device is within the tolerances the tests state (sums are accumulated in a
different order on the tensor cores); the integer parts (pictures, hint, features) are exact.
"""
from __future__ import annotations

import numpy as np

C = 32
CIN0 = 16
LAYERS = 4
HEAD = 8
K = 4
OFF_SCALE = 4
OFF_CLIP = 4


def cin(l: int) -> int:
    return CIN0 if l == 0 else C


def wcount(l: int) -> int:
    return C * 9 * cin(l)


def param_count() -> int:
    return sum(wcount(l) + C for l in range(LAYERS)) + HEAD * C + HEAD


def split_params(p: np.ndarray):
    """(W[l] (C, 9, cin), b[l] (C,)) for each layer, then Wh (8, 32), bh (8,)."""
    out, o = [], 0
    for l in range(LAYERS):
        w = p[o:o + wcount(l)].reshape(C, 9, cin(l))
        o += wcount(l)
        b = p[o:o + C]
        o += C
        out.append((w, b))
    wh = p[o:o + HEAD * C].reshape(HEAD, C)
    o += HEAD * C
    bh = p[o:o + HEAD]
    return out, wh, bh


def join_grads(layers, dwh, dbh) -> np.ndarray:
    parts = []
    for dw, db in layers:
        parts += [dw.reshape(-1), db.reshape(-1)]
    parts += [dwh.reshape(-1), dbh.reshape(-1)]
    return np.concatenate(parts)


def bf16(x) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(a.shape)


def bf16_bits_to_f32(bits: np.ndarray) -> np.ndarray:
    return (np.asarray(bits, np.uint32) << 16).view(np.float32)


# ---- pictures, hint, features ----------------------------------------------------------------

def geometry(w: int, h: int):
    mbw, mbh = (w + 15) // 16, (h + 15) // 16
    return 4 * mbw, 4 * mbh, mbw, mbh


def downsample(y: np.ndarray, w4: int, h4: int, dx: int = 0, dy: int = 0) -> np.ndarray:
    """(sum of the 4x4 block at (4x+dx, 4y+dy), clamped sampling, + 8) >> 4."""
    h, w = y.shape
    ys = np.clip(4 * np.arange(h4)[:, None] + np.arange(4)[None, :] + dy, 0, h - 1)  # (h4, 4)
    xs = np.clip(4 * np.arange(w4)[:, None] + np.arange(4)[None, :] + dx, 0, w - 1)  # (w4, 4)
    blk = y.astype(np.int64)[ys[:, :, None, None], xs[None, None, :, :]]  # (h4, 4, w4, 4)
    return ((blk.sum(axis=(1, 3)) + 8) >> 4).astype(np.int64)


def _shift_clamped(a: np.ndarray, dx: int, dy: int) -> np.ndarray:
    h, w = a.shape
    ys = np.clip(np.arange(h) + dy, 0, h - 1)
    xs = np.clip(np.arange(w) + dx, 0, w - 1)
    return a[ys[:, None], xs[None, :]]


def _hint_less(a, b):
    ca, ax, ay = a
    cb, bx, by = b
    return (ca, abs(ax) + abs(ay), ay, ax) < (cb, abs(bx) + abs(by), by, bx)


def hint_search(cur_y: np.ndarray, ref_y: np.ndarray, search_range: int):
    """Coarse to fine: 1/16 resolution over [-R16, R16]^2 (R16 = min(16, ceil(range/16))), 1/4
    resolution over the 7x7 about 4x that (within +-ceil(range/4)), full resolution at stride 2
    over the 5x5 about 4x that (within +-range)."""
    h, w = cur_y.shape
    w4, h4, mbw, mbh = geometry(w, h)
    c4, r4 = downsample(cur_y, w4, h4), downsample(ref_y, w4, h4)
    c16 = (c4.reshape(mbh, 4, mbw, 4).sum(axis=(1, 3)) + 8) >> 4
    r16 = (r4.reshape(mbh, 4, mbw, 4).sum(axis=(1, 3)) + 8) >> 4

    def least(cands, cost):
        best = None
        for dx, dy in cands:
            c = cost(dx, dy)
            if best is None or _hint_less((c, dx, dy), best):
                best = (c, dx, dy)
        return best[1], best[2]

    R = min(16, (search_range + 15) // 16)
    ax, ay = least([(dx, dy) for dy in range(-R, R + 1) for dx in range(-R, R + 1)],
                   lambda dx, dy: int(np.abs(c16 - _shift_clamped(r16, dx, dy)).sum()))
    r4r = (search_range + 3) // 4
    bx, by = least([(min(max(4 * ax + k % 7 - 3, -r4r), r4r), min(max(4 * ay + k // 7 - 3, -r4r), r4r))
                    for k in range(49)],
                   lambda dx, dy: int(np.abs(c4 - _shift_clamped(r4, dx, dy)).sum()))
    cur2 = cur_y[::2, ::2].astype(np.int64)

    def full(dx, dy):
        ys = np.clip(np.arange(0, h, 2) + dy, 0, h - 1)
        xs = np.clip(np.arange(0, w, 2) + dx, 0, w - 1)
        return int(np.abs(cur2 - ref_y.astype(np.int64)[ys[:, None], xs[None, :]]).sum())

    return least([(min(max(4 * bx + k % 5 - 2, -search_range), search_range),
                   min(max(4 * by + k // 5 - 2, -search_range), search_range)) for k in range(25)], full)


def features(cur_y: np.ndarray, ref_y: np.ndarray, hint) -> np.ndarray:
    """(H4, W4, 16) float32 holding bf16 values."""
    h, w = cur_y.shape
    w4, h4, _, _ = geometry(w, h)
    gx, gy = hint
    c4, r4 = downsample(cur_y, w4, h4), downsample(ref_y, w4, h4)
    rg = downsample(ref_y, w4, h4, gx, gy)
    hx = c4[:, np.minimum(np.arange(w4) + 1, w4 - 1)] - c4[:, np.maximum(np.arange(w4) - 1, 0)]
    vy = c4[np.minimum(np.arange(h4) + 1, h4 - 1), :] - c4[np.maximum(np.arange(h4) - 1, 0), :]
    k = np.float32(1.0 / 64.0)
    f = np.zeros((h4, w4, CIN0), np.float32)
    f[..., 0] = (c4 - 128).astype(np.float32) * k
    f[..., 1] = (r4 - 128).astype(np.float32) * k
    f[..., 2] = (rg - 128).astype(np.float32) * k
    f[..., 3] = (c4 - r4).astype(np.float32) * k
    f[..., 4] = (c4 - rg).astype(np.float32) * k
    f[..., 5] = hx.astype(np.float32) * k
    f[..., 6] = vy.astype(np.float32) * k
    f[..., 7] = np.float32(gx) * k
    f[..., 8] = np.float32(gy) * k
    return bf16(f)


# ---- the network -----------------------------------------------------------------------------

OFFS = [(tap % 3 - 1, tap // 3 - 1) for tap in range(9)]  # (dx, dy) of tap = ty * 3 + tx


def _shift_zero(x: np.ndarray, dx: int, dy: int) -> np.ndarray:
    """out[.., y, x, :] = x[.., y + dy, x + dx, :] (zero outside)."""
    out = np.zeros_like(x)
    H, W = x.shape[-3], x.shape[-2]
    ys0, ys1 = max(0, -dy), min(H, H - dy)
    xs0, xs1 = max(0, -dx), min(W, W - dx)
    if ys0 < ys1 and xs0 < xs1:
        out[..., ys0:ys1, xs0:xs1, :] = x[..., ys0 + dy:ys1 + dy, xs0 + dx:xs1 + dx, :]
    return out


def conv_fwd(x: np.ndarray, w: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Pre-activation Z[f, y, x, co] = sum_tap sum_ci x[f, y+dy, x+dx, ci] w[co, tap, ci] + b[co]."""
    x64 = x.astype(np.float64)
    z = np.zeros(x.shape[:-1] + (w.shape[0],), np.float64)
    for tap, (dx, dy) in enumerate(OFFS):
        z += _shift_zero(x64, dx, dy) @ w[:, tap, :].astype(np.float64).T
    return z + b.astype(np.float64)


def conv_dgrad(dz: np.ndarray, w: np.ndarray) -> np.ndarray:
    """dX[q] = sum_tap dZ[q - off(tap)] w[:, tap, :]."""
    dz64 = dz.astype(np.float64)
    dx_ = np.zeros(dz.shape[:-1] + (w.shape[2],), np.float64)
    for tap, (dx, dy) in enumerate(OFFS):
        dx_ += _shift_zero(dz64, -dx, -dy) @ w[:, tap, :].astype(np.float64)
    return dx_


def conv_wgrad(x: np.ndarray, dz: np.ndarray) -> np.ndarray:
    """dW[co, tap, ci] = sum_p x[p + off(tap)][ci] dZ[p][co]."""
    x64, dz64 = x.astype(np.float64), dz.astype(np.float64)
    co = dz.shape[-1]
    out = np.zeros((co, 9, x.shape[-1]), np.float64)
    d2 = dz64.reshape(-1, co)
    for tap, (dx, dy) in enumerate(OFFS):
        out[:, tap, :] = d2.T @ _shift_zero(x64, dx, dy).reshape(-1, x.shape[-1])
    return out


def _identity(x):
    return np.asarray(x, np.float64)


def forward(params: np.ndarray, x0: np.ndarray, rounding: bool = True):
    """x0: (F, H4, W4, 16) bf16 values. Returns the stored (bf16) outputs of every layer
    (rounding=False: exact float64 arithmetic throughout, for finite-difference checks)."""
    r = bf16 if rounding else _identity
    layers, _, _ = split_params(params)
    acts, x = [], x0
    for w, b in layers:
        z = conv_fwd(x, r(w), b)
        x = r(np.maximum(z, 0.0).astype(np.float32 if rounding else np.float64))
        acts.append(x)
    return acts


def head(params: np.ndarray, y4: np.ndarray, mbw: int, mbh: int):
    """Per picture and MB: (pooled (32,), out (8,))."""
    _, wh, bh = split_params(params)
    F = y4.shape[0]
    pooled = y4.astype(np.float64).reshape(F, mbh, 4, mbw, 4, C).mean(axis=(2, 4)).reshape(F, mbh * mbw, C)
    out = pooled @ wh.astype(np.float64).T + bh.astype(np.float64)
    return pooled, out


def candidates(out: np.ndarray, hints, search_range: int) -> np.ndarray:
    """(F, mbs, 4, 2) int: both hypotheses' refined vectors, then the raw hints, ordered by logit."""
    F, mbs, _ = out.shape
    res = np.zeros((F, mbs, K, 2), np.int64)
    for f in range(F):
        h = np.array([[0, 0], list(hints[f])], np.int64)
        o = out[f]
        ref = []
        for k in range(2):
            off = np.clip(o[:, 2 + 2 * k:4 + 2 * k].astype(np.float32), -OFF_CLIP, OFF_CLIP) * np.float32(OFF_SCALE)
            ref.append(np.clip(h[k] + np.rint(off).astype(np.int64), -search_range, search_range))
        first = (o[:, 1].astype(np.float32) > o[:, 0].astype(np.float32)).astype(np.int64)
        for i in range(mbs):
            a = first[i]
            res[f, i] = [ref[a][i], ref[1 - a][i], h[a], h[1 - a]]
    return res


def loss_and_grads(params: np.ndarray, x0: np.ndarray, hints, labels: np.ndarray, mbw: int, mbh: int,
                   rounding: bool = True):
    """Mean loss over the batch's macroblocks and the gradient of every parameter (the device's
    rounding points: bf16 activations and stored gradients, fp32 projection; rounding=False:
    exact float64 arithmetic)."""
    r = bf16 if rounding else _identity
    ft = np.float32 if rounding else np.float64
    layers, wh, bh = split_params(params)
    F = x0.shape[0]
    acts = forward(params, x0, rounding)
    y4 = acts[-1]
    pooled, out = head(params, y4, mbw, mbh)
    n = F * mbw * mbh
    dout = np.zeros_like(out)
    loss = 0.0
    for f in range(F):
        h = np.array([[0, 0], list(hints[f])], np.int64)
        L = labels[f].astype(np.int64)  # (mbs, 2)
        d0 = np.abs(L - h[0]).sum(1)
        d1 = np.abs(L - h[1]).sum(1)
        hs = np.where(d0 <= d1, 0, 1)
        for k in range(2):
            s = out[f][:, k]
            tgt = (hs == k).astype(np.float64)
            loss += float((np.logaddexp(0.0, s) - tgt * s).sum())
            dout[f][:, k] = (1.0 / (1.0 + np.exp(-s)) - tgt) / n
            m = np.abs(L - h[k]).max(1) <= OFF_CLIP * OFF_SCALE
            t = np.clip((L - h[k]).astype(np.float64) / OFF_SCALE, -OFF_CLIP, OFF_CLIP)
            e = out[f][:, 2 + 2 * k:4 + 2 * k] - t
            sl = np.where(np.abs(e) < 1.0, 0.5 * e * e, np.abs(e) - 0.5)
            loss += float((sl.sum(1) * m).sum())
            dout[f][:, 2 + 2 * k:4 + 2 * k] = np.clip(e, -1.0, 1.0) * m[:, None] / n
    loss /= n
    dwh = np.einsum("fmj,fmc->jc", dout, pooled)
    dbh = dout.sum(axis=(0, 1))
    dpooled = dout @ wh.astype(np.float64)  # (F, mbs, 32)
    dy = (dpooled / 16.0).reshape(F, mbh, 1, mbw, 1, C)
    dy = np.broadcast_to(dy, (F, mbh, 4, mbw, 4, C)).reshape(F, 4 * mbh, 4 * mbw, C)
    dz = r(np.where(y4 > 0, dy, 0.0).astype(ft))
    grads = [None] * LAYERS
    db_next = dz.astype(np.float64).sum(axis=(0, 1, 2))
    for l in range(LAYERS - 1, -1, -1):
        xin = x0 if l == 0 else acts[l - 1]
        dw = conv_wgrad(xin, dz)
        grads[l] = (dw, db_next)
        if l > 0:
            dxin = conv_dgrad(dz, r(layers[l][0]))
            dz = r(np.where(acts[l - 1] > 0, dxin, 0.0).astype(ft))
            db_next = dz.astype(np.float64).sum(axis=(0, 1, 2))
    return loss, join_grads(grads, dwh, dbh)


def labels_from_mvs(mvs: np.ndarray) -> np.ndarray:
    """Integer-pixel label of a quarter-pel vector: the nearest pixel, ties upward."""
    return (np.asarray(mvs, np.int64) + 2) >> 2
