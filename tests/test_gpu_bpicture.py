"""B-picture analysis on the device (vc1cu_analyze_b_picture / vc1cu_b_decide) against the
oracle's restatement of Vc1Encoder::analyze_b_picture_mode and the reference's own outputs
(tests/golden/b_kat.npz), bit-exact, through the C ABI."""
import os

import numpy as np
import pytest

from libvc1_b200 import synth
from libvc1_b200.abi import MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED, MV_QPEL, make_params
from libvc1_b200.api import Vc1cuError

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# tests/golden/make_golden.py B_CASES
B_GOLDEN = (
    (MV_QPEL, 1, 2, dict(display_width=125, display_height=93, search_range=16, local_search_range=16)),
    (MV_HPEL_BILINEAR, 1, 3, dict(display_width=125, display_height=93, search_range=16, local_search_range=16)),
    (MV_QPEL, 2, 3, dict(search_range=16, local_search_range=16, rnd=1, pqindex=20)),
    (MV_HPEL, 1, 2, dict(display_width=125, display_height=93, search_range=24, local_search_range=8)),
    (MV_MIXED, 1, 3, dict(search_range=16, local_search_range=16, pqindex=3)),
    (MV_QPEL, 1, 2, dict(search_range=16, local_search_range=16, disable_b_intra=1)),
)


def _frames(g, prefix):
    return tuple(np.ascontiguousarray(g[f"{prefix}.{c}"]) for c in "yuv")


@pytest.mark.parametrize("i", range(len(B_GOLDEN)))
def test_b_picture_matches_reference_fixture(ctx, i):
    g = np.load(os.path.join(GOLDEN, "b_kat.npz"))
    mode, num, den, kw = B_GOLDEN[i]
    p = make_params(130, 98, **kw)
    for fid, name in ((0, "past"), (1, "cur"), (2, "future")):
        ctx.upload_frame(fid, *_frames(g, name))
    b = ctx.analyze_b_picture(p, 1, 0, 2, g["anchor.mvs"], g["anchor.use_4mv"], num, den, mode)
    for field in b.ARRAYS:
        got, want = getattr(b, field), g[f"b{i}.{field}"]
        if got.dtype == np.float64:
            assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), field
        else:
            assert np.array_equal(got, want), field
    for k, v in b.totals.items():
        w = g[f"b{i}.total.{k}"]
        assert (np.float64(v).view(np.uint64) == w.view(np.uint64)) if w.dtype == np.float64 else int(v) == int(w), k


def _anchor(oracle, p, clip):
    """The future picture's own P analysis (quarter-pel seed, final Mixed-MV pass with P-intra)."""
    fut, past = clip.frame(2), clip.frame(0)
    q = oracle.analyze_p_core(p, fut, past, MV_QPEL, False)
    a = oracle.analyze_p_core(p, fut, past, MV_MIXED, True, seed=q.mvs, seed_distant=q)
    return a.mvs, a.use_4mv


B_CASES = {
    "cif_qpel_half": (lambda: synth.cif_plain(frames=3, seed=21), MV_QPEL, 1, 2,
                      dict(search_range=16, local_search_range=16)),
    "cif_bilinear_third": (lambda: synth.cif_plain(frames=3, seed=22), MV_HPEL_BILINEAR, 1, 3,
                           dict(search_range=16, local_search_range=16, pqindex=12)),
    "odd_two_thirds_rnd": (lambda: synth.generate(322, 242, 3, 23), MV_QPEL, 2, 3,
                           dict(display_width=321, display_height=241, search_range=24, local_search_range=24, rnd=1)),
    "odd_hpel_crop": (lambda: synth.generate(226, 130, 3, 24, global_px=9.5), MV_HPEL, 1, 2,
                      dict(display_width=219, display_height=121, search_range=16, local_search_range=16)),
    "mixed_pq2": (lambda: synth.generate(194, 146, 3, 25), MV_MIXED, 1, 3,
                  dict(search_range=16, local_search_range=16, pqindex=2)),
    "range0": (lambda: synth.cif_plain(frames=3, seed=26), MV_QPEL, 1, 2, dict(search_range=0, local_search_range=0)),
    "tiny_16x16": (lambda: synth.generate(16, 16, 3, 27, n_objects=0), MV_QPEL, 1, 2,
                   dict(search_range=8, local_search_range=8)),
    "longrange_diamond": (lambda: synth.generate(352, 288, 3, 28, global_px=40.0, n_objects=2), MV_QPEL, 2, 3,
                          dict(search_range=128, local_search_range=16, me_algorithm=1)),
    "no_b_intra": (lambda: synth.generate(322, 242, 3, 29, n_objects=4), MV_QPEL, 1, 2,
                   dict(search_range=16, local_search_range=16, disable_b_intra=1)),
}


@pytest.mark.parametrize("case", sorted(B_CASES))
def test_b_picture_matches_oracle(ctx, oracle, case):
    make, mode, num, den, kw = B_CASES[case]
    clip = make()
    p = make_params(clip.width, clip.height, **kw)
    amv, a4 = _anchor(oracle, p, clip)
    for t in range(3):
        ctx.upload_frame(t, *clip.frame(t))
    g = ctx.analyze_b_picture(p, 1, 0, 2, amv, a4, num, den, mode)
    e = oracle.analyze_b(p, clip.frame(1), clip.frame(0), clip.frame(2), amv, a4, num, den, mode)
    assert g.equal(e) == []
    assert g.totals["mv_mode"] == mode


def test_b_pictures_batched_match_oracle(ctx, oracle):
    """Two B pictures between two anchors, both directions of both pictures in one core launch, the
    anchor read from a result slot, and both decisions in one vc1cu_b_decide call."""
    clip = synth.cif_plain(frames=4, seed=30)
    p = make_params(clip.width, clip.height, search_range=16, local_search_range=16)
    for t in range(4):
        ctx.upload_frame(t, *clip.frame(t))
    # the future anchor (picture 3 against picture 0): seed pass, then the final Mixed-MV pass
    ctx.core_passes(p, [(3, 0, MV_QPEL, 0, -1, 10)])
    ctx.core_passes(p, [(3, 0, MV_MIXED, 1, 10, 11)])
    ctx.core_passes(p, [(1, 0, MV_QPEL, 0, -1, 20), (1, 3, MV_QPEL, 0, -1, 21),
                        (2, 0, MV_QPEL, 0, -1, 22), (2, 3, MV_QPEL, 0, -1, 23)])
    ctx.b_decide(p, [(1, 0, 3, 20, 21, 11, 1, 3, MV_QPEL, 5), (2, 0, 3, 22, 23, 11, 2, 3, MV_QPEL, 6)])
    anc = ctx.read_result(p, 11)
    for t, num, slot in ((1, 1, 5), (2, 2, 6)):
        e = oracle.analyze_b(p, clip.frame(t), clip.frame(0), clip.frame(3), anc.mvs, anc.use_4mv, num, 3, MV_QPEL)
        assert ctx.read_bresult(p, slot).equal(e) == [], t


def test_b_picture_rejects_bad_arguments(ctx):
    clip = synth.generate(64, 48, 3, 31)
    p = make_params(64, 48, search_range=8, local_search_range=8)
    for t in range(3):
        ctx.upload_frame(t, *clip.frame(t))
    amv = np.zeros((12, 2), np.int32)
    a4 = np.zeros(12, np.uint8)
    with pytest.raises(Vc1cuError, match="fraction"):
        ctx.analyze_b_picture(p, 1, 0, 2, amv, a4, 1, 4, MV_QPEL)
    with pytest.raises(Vc1cuError, match="anchor MV"):
        ctx.analyze_b_picture(p, 1, 0, 2, np.full((12, 2), 1 << 20, np.int32), a4, 1, 2, MV_QPEL)
    # a seeded or P-intra pass is not one direction of a B picture
    ctx.core_passes(p, [(1, 0, MV_QPEL, 0, -1, 40), (1, 2, MV_QPEL, 0, -1, 41)])
    ctx.core_passes(p, [(1, 0, MV_HPEL, 0, 40, 42), (1, 2, MV_QPEL, 1, -1, 43)])
    with pytest.raises(Vc1cuError, match="unseeded"):
        ctx.b_decide(p, [(1, 0, 2, 42, 41, 40, 1, 2, MV_HPEL, 7)])
    with pytest.raises(Vc1cuError, match="unseeded"):
        ctx.b_decide(p, [(1, 0, 2, 40, 43, 40, 1, 2, MV_QPEL, 7)])
    with pytest.raises(Vc1cuError, match="share"):
        ctx.b_decide(p, [(1, 0, 2, 40, 41, 40, 1, 2, MV_QPEL, 7), (1, 0, 2, 40, 41, 40, 1, 3, MV_QPEL, 7)])
    with pytest.raises(Vc1cuError, match="empty B-result"):
        ctx.read_bresult(p, 4000)
    # the context stays usable
    ctx.b_decide(p, [(1, 0, 2, 40, 41, 40, 1, 2, MV_QPEL, 7)])
    assert ctx.read_bresult(p, 7).totals["mv_mode"] == MV_QPEL


@pytest.mark.parametrize("i", range(len(B_GOLDEN)))
def test_b_prediction_matches_reference_fixture(ctx, oracle, i):
    """The prediction of the reference's own analysis (decided on the device through the batch
    form, anchor from the fixture), then its transform + quantiser against the oracle's."""
    g = np.load(os.path.join(GOLDEN, "b_kat.npz"))
    mode, num, den, kw = B_GOLDEN[i]
    p = make_params(130, 98, **kw)
    past, cur, fut = _frames(g, "past"), _frames(g, "cur"), _frames(g, "future")
    for fid, fr in ((0, past), (1, cur), (2, fut)):
        ctx.upload_frame(fid, *fr)
    # the anchor's field: the future picture's own passes on the device equal the fixture's anchor
    p0 = make_params(130, 98, search_range=16, local_search_range=16)  # the anchor's own configuration
    ctx.core_passes(p, [(1, 0, mode, 0, -1, 70), (1, 2, mode, 0, -1, 71)])
    ctx.core_passes(p0, [(2, 0, MV_QPEL, 0, -1, 72)])
    ctx.core_passes(p0, [(2, 0, MV_MIXED, 1, 72, 73)])
    anc = ctx.read_result(p0, 73)
    assert np.array_equal(anc.mvs, g["anchor.mvs"]) and np.array_equal(anc.use_4mv, g["anchor.use_4mv"])
    ctx.b_decide(p, [(1, 0, 2, 70, 71, 73, num, den, mode, 9)])
    ctx.b_predict(p, 9, 1, 0, 2, 5)
    pred = ctx.download_frame(5, 130, 98)
    for got, c in zip(pred, "yuv"):
        assert np.array_equal(got, g[f"b{i}.pred.{c}"]), c
    co, lv = ctx.forward_quant(p, 1, 5, 15)
    eco, elv = oracle.forward_quant(p, cur, pred, 15)
    assert np.array_equal(co.view(np.uint64), eco.view(np.uint64)) and np.array_equal(lv, elv)
