"""Intensity compensation on the device (vc1cu_estimate_intensity_comp / _batch,
vc1cu_intensity_compensate) against the reference's outputs (tests/golden/ic_kat.npz) and the
oracle's restatement, bit-exact, through the C ABI."""
import os

import numpy as np
import pytest

from libvc1_b200 import synth
from libvc1_b200.abi import MV_QPEL, make_params
from libvc1_b200.api import Vc1cuError

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# tests/golden/make_golden.py IC_CASES / IC_FIXED
IC_CASES = ((98, 66, dict(search_range=16, local_search_range=16)),
            (130, 98, dict(display_width=125, display_height=93, search_range=16, local_search_range=16)),
            (352, 288, dict(search_range=16, local_search_range=16)),
            (66, 50, dict(search_range=8, local_search_range=8)),
            (16, 16, dict(search_range=8, local_search_range=8)))
IC_FIXED = ((1, 0, 5), (1, 0, 40), (1, 63, 60), (1, 17, 33), (0, 0, 0))


def _frames(g, prefix):
    return tuple(np.ascontiguousarray(g[f"{prefix}.{c}"]) for c in "yuv")


@pytest.mark.parametrize("i", range(len(IC_CASES)))
def test_intensity_matches_reference_fixture(ctx, i):
    g = np.load(os.path.join(GOLDEN, "ic_kat.npz"))
    w, h, kw = IC_CASES[i]
    p = make_params(w, h, **kw)
    ctx.upload_frame(0, *_frames(g, f"c{i}.ref"))
    ctx.upload_frame(1, *_frames(g, f"c{i}.cur"))
    ic = ctx.estimate_intensity_comp(p, 1, 0, g[f"c{i}.mvs"])
    assert ic == tuple(g[f"c{i}.ic"].tolist())
    if f"c{i}.map0.y" in g.files:
        for j, k in enumerate((ic,) + IC_FIXED):
            ctx.intensity_compensate(0, k, 2)
            for got, c in zip(ctx.download_frame(2, w, h), "yuv"):
                assert np.array_equal(got, g[f"c{i}.map{j}.{c}"]), (j, c)


FADES = {
    "cif_darken": (lambda: synth.cif_plain(frames=2, seed=40), 0.75, 12.0),
    "cif_brighten": (lambda: synth.cif_plain(frames=2, seed=41), 1.25, -30.0),
    "cif_none": (lambda: synth.cif_plain(frames=2, seed=42), 1.0, 0.0),
    "odd_strong": (lambda: synth.generate(322, 242, 2, 43), 0.55, 60.0),
    "tiny": (lambda: synth.generate(16, 16, 2, 44, n_objects=0), 0.9, 4.0),
}


def test_intensity_batch_matches_oracle(ctx, oracle):
    """All pictures' estimates in one batch, each along its device quarter-pel pass, then the
    compensated reference of each estimate."""
    for name in sorted(FADES):
        make, a, b = FADES[name]
        clip = make()
        w, h = clip.width, clip.height
        p = make_params(w, h, search_range=16, local_search_range=16, display_width=w - 1 if w > 16 else 0)
        ref, cur = clip.frame(0), synth.fade(clip.frame(1), a, b, 7)
        ctx.upload_frame(0, *ref)
        ctx.upload_frame(1, *cur)
        ctx.core_passes(p, [(1, 0, MV_QPEL, 0, -1, 50)])
        got = ctx.estimate_intensity_batch(p, [(1, 0, 50), (1, 0, 50)])
        q = oracle.analyze_p_core(p, cur, ref, MV_QPEL, False)
        want = oracle.estimate_intensity_comp(p, cur, ref, q.mvs)
        assert got == [want, want], name
        ctx.intensity_compensate(0, want, 3)
        for x, y in zip(ctx.download_frame(3, w, h), oracle.intensity_compensate(ref, want)):
            assert np.array_equal(x, y), name


def test_intensity_1080p_matches_oracle(ctx, oracle):
    clip = synth.hd1080(frames=2, seed=45)
    p = make_params(1920, 1080, search_range=64, local_search_range=64, nonuniform=1)
    ref, cur = clip.frame(0), synth.fade(clip.frame(1), 0.85, 9.0, 45)
    ctx.upload_frame(0, *ref)
    ctx.upload_frame(1, *cur)
    ctx.core_passes(p, [(1, 0, MV_QPEL, 0, -1, 51)])
    a = ctx.read_result(p, 51)
    want = oracle.estimate_intensity_comp(p, cur, ref, a.mvs)
    assert want[0] == 1
    assert ctx.estimate_intensity_batch(p, [(1, 0, 51)]) == [want]
    assert ctx.estimate_intensity_comp(p, 1, 0, a.mvs) == want


def test_intensity_rejects_bad_arguments(ctx):
    clip = synth.generate(64, 48, 2, 46)
    ctx.upload_frame(0, *clip.frame(0))
    with pytest.raises(Vc1cuError, match="6-bit"):
        ctx.intensity_compensate(0, (1, 64, 0), 1)
    with pytest.raises(Vc1cuError, match="output frame"):
        ctx.intensity_compensate(0, (1, 20, 3), 0)
    p = make_params(64, 48, search_range=8, local_search_range=8)
    with pytest.raises(Vc1cuError, match="never uploaded"):
        ctx.estimate_intensity_comp(p, 999, 0, np.zeros((12, 2), np.int32))


def test_intensity_enqueue_collect_matches_batch(ctx):
    """The two-phase form gives the batch form's estimates, with two batches outstanding and
    more work enqueued behind them; a ticket is collectable once."""
    make, a, b = FADES["cif_darken"]
    clip = make()
    w, h = clip.width, clip.height
    p = make_params(w, h, search_range=16, local_search_range=16)
    ref, cur = clip.frame(0), synth.fade(clip.frame(1), a, b, 7)
    ctx.upload_frame(60, *ref)
    ctx.upload_frame(61, *cur)
    ctx.core_passes(p, [(61, 60, MV_QPEL, 0, -1, 62), (60, 61, MV_QPEL, 0, -1, 63)])
    jobs1, jobs2 = [(61, 60, 62)], [(61, 60, 62), (60, 61, 63)]
    want1, want2 = ctx.estimate_intensity_batch(p, jobs1), ctx.estimate_intensity_batch(p, jobs2)
    t1 = ctx.estimate_intensity_enqueue(p, jobs1)
    t2 = ctx.estimate_intensity_enqueue(p, jobs2)
    ctx.core_passes(p, [(61, 60, MV_QPEL, 0, -1, 64)])  # later work on the stream
    assert ctx.estimate_intensity_collect(t2) == want2
    assert ctx.estimate_intensity_collect(t1) == want1
    with pytest.raises(Vc1cuError, match="ticket"):
        ctx.estimate_intensity_collect(t1)
    with pytest.raises(Vc1cuError, match="ticket"):
        ctx.estimate_intensity_collect((123456, 1))
