"""The learned motion-vector proposals on the device against their CPU oracle (oracle/lp_oracle.py).

- the quarter-resolution translation hint and the 16 input channels: exact;
- the loss and the gradient of every parameter from the hand-written backward kernels (tcgen05
  tensor-core convolutions, BF16 operands, FP32 accumulation): within the tolerances below, set by
  the bf16 rounding of the stored activations and gradients (sums are accumulated in another
  order on the tensor cores, so a stored value can land on the neighbouring bf16 number);
- the candidates of inference;
- training on device reduces the loss;
- the learned pass with its plain-search fallback returns legal vectors whose costs are close to
  the plain pass's.
"""
import numpy as np
import pytest

from libvc1_b200 import synth
from libvc1_b200.abi import MV_QPEL, make_params
from libvc1_b200.api import LearnedProposals
from oracle import lp_oracle as lo

pytestmark = pytest.mark.gpu

GRAD_REL_TOL = 3e-2   # per parameter tensor, ||g_device - g_oracle|| / ||g_oracle||
LOSS_REL_TOL = 2e-3


def _clip(w, h, seed, gpx, frames=2):
    return synth.generate(w, h, frames, seed, global_px=gpx, n_objects=3, obj_min=16, obj_max=40, obj_vel=4.0)


def _samples(ctx, net, clips, rng, label_slot0=950):
    """Prepares sample i from clip i's pair (frame 1 against frame 0) and labels it with the plain
    pass; returns the oracle's inputs (features, hints, labels)."""
    xs, hints, labels = [], [], []
    for i, clip in enumerate(clips):
        ctx.upload_frame(600 + 2 * i, *clip.frame(1))
        ctx.upload_frame(601 + 2 * i, *clip.frame(0))
        net.prepare(600 + 2 * i, 601 + 2 * i, i)
        p = make_params(clip.width, clip.height, search_range=rng, local_search_range=min(rng, 32))
        ctx.core_passes(p, [(600 + 2 * i, 601 + 2 * i, MV_QPEL, 0, -1, label_slot0 + i)])
        net.set_labels(i, label_slot0 + i)
        a = ctx.read_result(p, label_slot0 + i)
        f, h, _, _ = net.read_sample(i)
        xs.append(lo.bf16_bits_to_f32(f))
        hints.append((int(h[0]), int(h[1])))
        labels.append(lo.labels_from_mvs(a.mvs))
    return np.stack(xs), hints, np.stack(labels)


@pytest.mark.parametrize("w,h,rng,gpx,seed", [(192, 128, 32, 20.0, 3), (576, 64, 64, 40.0, 5), (96, 64, 0, 3.0, 2),
                                              (322, 242, 128, 90.0, 8)])
def test_hint_and_features_match_oracle(ctx, w, h, rng, gpx, seed):
    clip = _clip(w, h, seed, gpx)
    ctx.upload_frame(0, *clip.frame(1))
    ctx.upload_frame(1, *clip.frame(0))
    net = LearnedProposals(ctx, w, h, rng, capacity=1, max_batch=1)
    try:
        net.prepare(0, 1, 0)
        f, hint, _, _ = net.read_sample(0)
    finally:
        net.close()
    want = lo.hint_search(clip.y[1], clip.y[0], rng)
    assert (int(hint[0]), int(hint[1])) == want
    assert np.array_equal(lo.bf16_bits_to_f32(f), lo.features(clip.y[1], clip.y[0], want))


def _tensor_errors(g, o):
    errs, off = {}, 0
    for l in range(lo.LAYERS):
        for name, n in ((f"W{l}", lo.wcount(l)), (f"b{l}", lo.C)):
            a, b = g[off:off + n], o[off:off + n]
            errs[name] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12))
            off += n
    for name, n in (("Wh", lo.HEAD * lo.C), ("bh", lo.HEAD)):
        a, b = g[off:off + n], o[off:off + n]
        errs[name] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12))
        off += n
    return errs


@pytest.mark.parametrize("w,h,rng", [(128, 96, 32), (576, 64, 64)])
def test_gradients_match_oracle(ctx, w, h, rng):
    """W4 = 32 (one partial tile per row) and W4 = 144 (two tiles per row), batch of two."""
    clips = [_clip(w, h, 11 + k, 0.3 * rng) for k in range(2)]
    net = LearnedProposals(ctx, w, h, rng, capacity=2, max_batch=2, seed=5)
    try:
        x0, hints, labels = _samples(ctx, net, clips, rng)
        loss, g = net.gradients([0, 1])
        params = net.params()
    finally:
        net.close()
    mbw, mbh = (w + 15) // 16, (h + 15) // 16
    eloss, eg = lo.loss_and_grads(params.astype(np.float64), x0, hints, labels, mbw, mbh)
    assert abs(loss - eloss) <= LOSS_REL_TOL * max(1.0, abs(eloss)), (loss, eloss)
    errs = _tensor_errors(g.astype(np.float64), eg)
    assert max(errs.values()) < GRAD_REL_TOL, errs


def test_candidates_match_oracle(ctx):
    w, h, rng = 320, 192, 64
    clips = [_clip(w, h, 21 + k, 30.0) for k in range(2)]
    net = LearnedProposals(ctx, w, h, rng, capacity=2, max_batch=2, seed=9)
    try:
        x0, hints, _ = _samples(ctx, net, clips, rng)
        net.propose(0, 2)
        got = np.stack([net.read_sample(i)[2] for i in range(2)])
        params = net.params()
    finally:
        net.close()
    mbw, mbh = (w + 15) // 16, (h + 15) // 16
    acts = lo.forward(params.astype(np.float64), x0)
    _, out = lo.head(params.astype(np.float64), acts[-1], mbw, mbh)
    want = lo.candidates(out, hints, rng)
    # the raw hints exactly; the refined vectors but where a rounding boundary splits them
    assert np.array_equal(np.sort(got[:, :, 2:], axis=2), np.sort(want[:, :, 2:], axis=2))
    agree = np.mean(np.all(got == want, axis=(2, 3)))
    assert agree >= 0.98, agree


def test_training_on_device_reduces_the_loss(ctx):
    w, h, rng = 256, 160, 64
    clips = [_clip(w, h, 31 + k, 40.0) for k in range(6)]
    net = LearnedProposals(ctx, w, h, rng, capacity=6, max_batch=3, seed=2)
    try:
        _samples(ctx, net, clips, rng)
        first = np.mean([net.gradients([0, 1, 2])[0], net.gradients([3, 4, 5])[0]])
        for step in range(60):
            net.train_step([0, 1, 2] if step % 2 == 0 else [3, 4, 5], 3e-3)
        last = np.mean([net.gradients([0, 1, 2])[0], net.gradients([3, 4, 5])[0]])
    finally:
        net.close()
    assert last < 0.7 * first, (first, last)


LEARNED_CASES = {
    # (w, h, display, range, local range, mode, fallback, global px)
    "cif_qpel": (352, 288, None, 64, 32, MV_QPEL, True, 40.0),
    "odd_hpel": (322, 242, (321, 241), 32, 32, 1, True, 20.0),
    "longrange_bilinear": (192, 128, None, 128, 16, 2, True, 70.0),
    "no_fallback": (256, 160, None, 64, 32, MV_QPEL, False, 30.0),
}


@pytest.mark.parametrize("case", sorted(LEARNED_CASES))
def test_learned_pass_matches_oracle(ctx, oracle, case):
    """Both launches of the learned pass, bit for bit against the oracle's restatement
    (oracle/vc1_oracle.c vo_analyze_p_learned) on the device's own candidates and hint."""
    w, h, disp, rng, local, mode, fallback, gpx = LEARNED_CASES[case]
    clip = _clip(w, h, 51, gpx)
    kw = dict(display_width=disp[0], display_height=disp[1]) if disp else {}
    p = make_params(w, h, search_range=rng, local_search_range=local, **kw)
    ctx.upload_frame(0, *clip.frame(1))
    ctx.upload_frame(1, *clip.frame(0))
    net = LearnedProposals(ctx, w, h, rng, capacity=1, max_batch=1, seed=6)
    try:
        net.prepare(0, 1, 0)
        net.propose(0, 1)
        net.analyze(p, [(0, 1, 0, mode, 970)], fallback=fallback)
        got = ctx.read_result(p, 970)
        _, hint, cands, flags = net.read_sample(0)
    finally:
        net.close()
    want, wflags = oracle.analyze_p_learned(p, clip.frame(1), clip.frame(0), mode, cands, hint, fallback)
    assert np.array_equal(flags, wflags)
    assert got.equal(want) == []


def test_learned_pass_with_fallback(ctx):
    """Every macroblock gets a legal vector; with the plain search as fallback the mean exact
    cost stays close to the plain pass's."""
    w, h, rng = 352, 288, 64
    clip = _clip(w, h, 41, 40.0)
    ctx.upload_frame(0, *clip.frame(1))
    ctx.upload_frame(1, *clip.frame(0))
    p = make_params(w, h, search_range=rng, local_search_range=32)
    ctx.core_passes(p, [(0, 1, MV_QPEL, 0, -1, 960)])
    plain = ctx.read_result(p, 960)
    net = LearnedProposals(ctx, w, h, rng, capacity=1, max_batch=1, seed=4)
    try:
        net.prepare(0, 1, 0)
        net.propose(0, 1)
        net.analyze(p, [(0, 1, 0, MV_QPEL, 961)], fallback=True)
        learned = ctx.read_result(p, 961)
        _, _, cands, fb = net.read_sample(0)
    finally:
        net.close()
    assert learned.mvs.shape == plain.mvs.shape
    assert np.all(np.abs(learned.mvs[:, 0]) <= 4 * rng) and np.all(np.abs(learned.mvs[:, 1]) <= 4 * rng)
    s_plain = plain.screen_sads.astype(np.float64).sum()
    s_learned = learned.screen_sads.astype(np.float64).sum()
    assert s_learned <= 1.10 * s_plain, (s_learned, s_plain, int(fb.sum()))
