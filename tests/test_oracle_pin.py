"""Pins the oracle (our C restatement, oracle/vc1_oracle.c) to the reference (CPU only).

1. Golden vectors produced by the reference's own code (tests/golden/*.npz, written by
   tests/golden/make_golden.py from oracle/_ref) must be reproduced bit-exactly, and the
   properties the reference's tests assert on the same inputs must hold.
2. Where oracle/_ref is built in this tree, the oracle is also compared live with it on
   further seeded inputs.
"""
import os

import numpy as np
import pytest

from libvc1_b200 import synth
from libvc1_b200.abi import BAD_COST, MODES, MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED, MV_QPEL, make_params

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def planes(y, chroma=128):
    h, w = y.shape
    u = np.full((h // 2, w // 2), chroma, np.uint8)
    return (np.ascontiguousarray(y, np.uint8), u, u.copy())


def test_runtime_kat(oracle):
    """tests/vulkan_compute_runtime.cpp:39-98 on the CPU law."""
    g = load("runtime_kat.npz")
    cur, ref = planes(g["cur"]), planes(g["ref"])
    p = make_params(48, 40)
    assert [oracle.block_sad_motion(p, cur, ref, 5, 7, 16, 16, int(a), int(b), MV_QPEL) for a, b in g["mvs"]] == \
        g["sad_qpel"].tolist()
    assert [oracle.block_satd_motion(p, cur, ref, 5, 7, 16, 16, int(a), int(b), MV_QPEL) for a, b in g["mvs"]] == \
        g["satd_qpel"].tolist()
    assert [oracle.block_sad_motion(p, cur, ref, 3, 4, 16, 16, int(a), int(b), MV_HPEL_BILINEAR)
            for a, b in g["half_mvs"]] == g["sad_bilinear"].tolist()
    for s in (2, 4):
        got = [oracle.shader_cost(cur, ref, 5, 7, 16, 16, s, 0, 0, 0, int(a), int(b)) for a, b in g["int_mvs"]]
        assert got == g[f"sad_int_stride{s}"].tolist()


def test_staged_kat(oracle):
    """tests/staged_motion_estimation.cpp:26-39 and :134-147."""
    g = load("staged_kat.npz")
    p16 = make_params(16, 16, search_range=8, local_search_range=8)
    c, f, n = planes(g["cur16"]), planes(g["flat16"]), planes(g["noisy16"])
    sf = oracle.block_sad_motion(p16, c, f, 0, 0, 16, 16, 0, 0, MV_QPEL)
    sn = oracle.block_sad_motion(p16, c, n, 0, 0, 16, 16, 0, 0, MV_QPEL)
    tf = oracle.block_satd_motion(p16, c, f, 0, 0, 16, 16, 0, 0, MV_QPEL)
    tn = oracle.block_satd_motion(p16, c, n, 0, 0, 16, 16, 0, 0, MV_QPEL)
    assert (sf, sn, tf, tn) == (int(g["sad_flat"]), int(g["sad_noisy"]), int(g["satd_flat"]), int(g["satd_noisy"]))
    assert sf == 256 and sn == 256 and tn > tf  # the reference test's own assertions
    p32 = make_params(32, 32, search_range=8, local_search_range=8)
    a, b = planes(g["cur32"]), planes(g["ref32"])
    assert [oracle.block_satd_motion(p32, a, b, 8, 8, 16, 16, int(x), int(y), MV_QPEL) for x, y in g["qgrid"]] == \
        g["satd_qgrid"].tolist()
    assert [oracle.block_satd_motion(p32, a, b, 8, 8, 16, 16, int(x), int(y), MV_HPEL_BILINEAR)
            for x, y in g["bgrid"]] == g["satd_bgrid"].tolist()


def _gradient(w, h, horizontal):
    x = np.arange(w)[None, :].repeat(h, 0)
    y = np.arange(h)[:, None].repeat(w, 1)
    return (20 + 3 * (x if horizontal else y)).astype(np.uint8)


def test_diamond_kat(oracle):
    """tests/diamond_motion.cpp:18-60: exact recovery of a translation, cropped-edge legality."""
    g = load("diamond_kat.npz")
    for i in range(2):
        sx, sy, hor = g[f"shift{i}"].tolist()
        ref = _gradient(64, 48, bool(hor))
        cur = ref[np.clip(np.arange(48) + sy, 0, 47)][:, np.clip(np.arange(64) + sx, 0, 63)]
        p = make_params(64, 48, search_range=12, local_search_range=12, me_algorithm=1)
        got = oracle.integer_motion(p, planes(cur), planes(ref), 1, 1, np.zeros((12, 2), np.int32), 0, 0, 12)
        assert list(got) == g[f"shift{i}.result"].tolist()
        assert got == (sx, sy, 0)
    pe = make_params(64, 48, display_height=42, search_range=8, local_search_range=8, me_algorithm=1)
    f = planes(_gradient(64, 48, True))
    s = oracle.mb_sad(pe, f, f, 1, 2, 0, 4, 1)
    assert s == int(g["edge_mb_sad"]) and s >= (1 << 64) // 8


def _frames(g, prefix):
    return tuple(np.ascontiguousarray(g[f"{prefix}.{c}"]) for c in "yuv")


ANALYSIS = {
    "cif_r8": dict(search_range=8, local_search_range=8),
    "odd_322x242": dict(display_width=321, display_height=241, search_range=16, local_search_range=16, rnd=1,
                        pqindex=12, nonuniform=1),
}


@pytest.mark.parametrize("name", sorted(ANALYSIS))
def test_analysis_chain_golden(oracle, name):
    """Five analyze_p_picture_core passes of one picture against the reference's outputs."""
    g = load(f"analysis_{name}.npz")
    cur, ref = _frames(g, "cur"), _frames(g, "ref")
    p = make_params(cur[0].shape[1], cur[0].shape[0], **ANALYSIS[name])

    def check(pass_name, a):
        for field in a.ARRAYS:
            want = g[f"{pass_name}.{field}"]
            got = getattr(a, field)
            if got.dtype == np.float64:
                assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), (pass_name, field)
            else:
                assert np.array_equal(got, want), (pass_name, field)
        for k, v in a.totals.items():
            w = g[f"{pass_name}.total.{k}"]
            assert (np.float64(v).view(np.uint64) == w.view(np.uint64)) if w.dtype == np.float64 else int(v) == int(w), \
                (pass_name, k)

    q = oracle.analyze_p_core(p, cur, ref, MV_QPEL, False)
    check("qpel", q)
    for m, pn in ((MV_HPEL, "hpel"), (MV_HPEL_BILINEAR, "bilinear"), (MV_MIXED, "mixed")):
        a = oracle.analyze_p_core(p, cur, ref, m, False, seed=q.mvs, seed_distant=q)
        check(pn, a)
    f = oracle.analyze_p_core(p, cur, ref, MV_MIXED, True, seed=a.mvs, seed_distant=a)
    check("final", f)


def test_xform_golden(oracle):
    """Prediction, forward transform (all four sizes) and quantiser at four QP settings."""
    g = load("xform_kat.npz")
    cur, ref = _frames(g, "cur"), _frames(g, "ref")
    for pq, nu, hq in ((3, 0, 1), (8, 1, 1), (17, 1, 0), (31, 0, 0)):
        key = f"pq{pq}_nu{nu}_hq{hq}"
        p = make_params(64, 48, pqindex=pq, nonuniform=nu, halfqp=hq, search_range=8, local_search_range=8)
        q = oracle.analyze_p_core(p, cur, ref, MV_QPEL, False)
        f = oracle.analyze_p_core(p, cur, ref, MV_MIXED, True, seed=q.mvs, seed_distant=q)
        assert np.array_equal(f.mvs, g[f"{key}.mvs"]) and np.array_equal(f.block_mvs, g[f"{key}.block_mvs"])
        pred = oracle.motion_compensate(p, ref, f, MV_MIXED)
        for c, plane in zip("yuv", pred):
            assert np.array_equal(plane, g[f"{key}.pred.{c}"]), (key, c)
        co, lv = oracle.forward_quant(p, cur, pred, 15)
        assert np.array_equal(co.view(np.uint64), g[f"{key}.coeffs"].view(np.uint64)), key
        assert np.array_equal(lv, g[f"{key}.levels"]), key


def test_global_golden(oracle):
    g = load("global_kat.npz")
    for i in range(3):
        cur, ref = planes(g[f"g{i}.cur"]), planes(g[f"g{i}.ref"])
        rng = int(g[f"g{i}.range"])
        p = make_params(352, 288, search_range=rng, local_search_range=rng)
        assert list(oracle.global_motion(p, cur, ref, rng)) == g[f"g{i}.result"].tolist()
        got = [[oracle.frame_sad(cur, ref, int(dx), int(dy), s) for s in (1, 2, 4)]
               for dx, dy in g[f"g{i}.frame_sad_offsets"]]
        assert got == g[f"g{i}.frame_sad"].tolist()


# analyze_b_picture_mode fixtures (tests/golden/make_golden.py B_CASES)
B_CASES = (
    (MV_QPEL, 1, 2, dict(display_width=125, display_height=93, search_range=16, local_search_range=16)),
    (MV_HPEL_BILINEAR, 1, 3, dict(display_width=125, display_height=93, search_range=16, local_search_range=16)),
    (MV_QPEL, 2, 3, dict(search_range=16, local_search_range=16, rnd=1, pqindex=20)),
    (MV_HPEL, 1, 2, dict(display_width=125, display_height=93, search_range=24, local_search_range=8)),
    (MV_MIXED, 1, 3, dict(search_range=16, local_search_range=16, pqindex=3)),
    (MV_QPEL, 1, 2, dict(search_range=16, local_search_range=16, disable_b_intra=1)),
)


@pytest.mark.parametrize("i", range(len(B_CASES)))
def test_b_analysis_golden(oracle, i):
    """B-picture analysis (both core passes + the per-MB mode decision) against the reference."""
    g = load("b_kat.npz")
    past, cur, fut = _frames(g, "past"), _frames(g, "cur"), _frames(g, "future")
    mode, num, den, kw = B_CASES[i]
    p = make_params(130, 98, **kw)
    b = oracle.analyze_b(p, cur, past, fut, g["anchor.mvs"], g["anchor.use_4mv"], num, den, mode)
    for field in b.ARRAYS:
        got, want = getattr(b, field), g[f"b{i}.{field}"]
        if got.dtype == np.float64:
            assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), field
        else:
            assert np.array_equal(got, want), field
    for k, v in b.totals.items():
        w = g[f"b{i}.total.{k}"]
        assert (np.float64(v).view(np.uint64) == w.view(np.uint64)) if w.dtype == np.float64 else int(v) == int(w), k
    for got, c in zip(oracle.b_predict(p, cur, past, fut, b, mode), "yuv"):
        assert np.array_equal(got, g[f"b{i}.pred.{c}"]), c
    # every decision kind the fixture set is meant to cover
    if i == 0:
        modes = set(np.concatenate([g[f"b{j}.modes"] for j in range(len(B_CASES))]).tolist())
        assert modes == {0, 1, 2, 3, 4}


def test_synthetic_clip_is_deterministic():
    a = synth.generate(64, 48, 3, 17)
    b = synth.generate(64, 48, 3, 17)
    for t in range(3):
        for x, y in zip(a.frame(t), b.frame(t)):
            assert np.array_equal(x, y)
    c = synth.generate(64, 48, 3, 18)
    assert not np.array_equal(a.frame(1)[0], c.frame(1)[0])


# ---- live comparison with the reference build (skipped where oracle/_ref is absent) ----

def _ref_or_skip():
    from oracle import ref_available

    if not ref_available():
        pytest.skip("oracle/_ref not built in this tree")
    from oracle import Reference

    return Reference


@pytest.mark.parametrize("rnd", [0, 1])
def test_block_costs_match_reference_live(oracle, rnd):
    Reference = _ref_or_skip()
    clip = synth.generate(66, 50, 2, 3)
    p = make_params(66, 50, display_width=61, display_height=45, search_range=16, local_search_range=16, rnd=rnd)
    R = Reference(p)
    cur, ref = clip.frame(1), clip.frame(0)
    rc, rr = R.frame(cur), R.frame(ref)
    rng = np.random.default_rng(31 + rnd)
    for mode in MODES:
        for (x0, y0, bw, bh) in ((48, 32, 16, 16), (56, 40, 8, 8), (0, 0, 16, 16), (24, 8, 8, 8)):
            for a, b in rng.integers(-30, 31, (40, 2)):
                a, b = int(a), int(b)
                assert oracle.block_sad_motion(p, cur, ref, x0, y0, bw, bh, a, b, mode) == \
                    R.block_sad_motion(rc, rr, x0, y0, bw, bh, a, b, mode)
                assert oracle.block_satd_motion(p, cur, ref, x0, y0, bw, bh, a, b, mode) == \
                    R.block_satd_motion(rc, rr, x0, y0, bw, bh, a, b, mode)
    costs = [oracle.block_sad_motion(p, cur, ref, 48, 32, 16, 16, a, b, MV_QPEL) for a in range(-24, 25, 3)
             for b in range(-24, 25, 3)]
    assert BAD_COST in costs  # the hidden-padding gate is exercised


@pytest.mark.parametrize("kw", [dict(search_range=16, local_search_range=16),
                                dict(search_range=16, local_search_range=16, me_algorithm=1),
                                dict(search_range=16, local_search_range=16, fast_subpel=1, me_quality=0),
                                dict(search_range=24, local_search_range=8, pqindex=5, halfqp=1),
                                dict(search_range=0, local_search_range=0),
                                dict(search_range=96, local_search_range=8),
                                dict(search_range=96, local_search_range=8, long_range_mode=2)])
def test_analysis_matches_reference_live(oracle, kw):
    Reference = _ref_or_skip()
    clip = synth.generate(98, 66, 2, 13)
    p = make_params(98, 66, display_width=97, display_height=65, **kw)
    R = Reference(p)
    cur, ref = clip.frame(1), clip.frame(0)
    rc, rr = R.frame(cur), R.frame(ref)
    e = R.analyze_p_core(rc, rr, MV_QPEL, False)
    assert oracle.analyze_p_core(p, cur, ref, MV_QPEL, False).equal(e) == []
    for mode in (MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED):
        em = R.analyze_p_core(rc, rr, mode, True, seed=e.mvs, seed_distant=e)
        assert oracle.analyze_p_core(p, cur, ref, mode, True, seed=e.mvs, seed_distant=e).equal(em) == [], mode


@pytest.mark.parametrize("case", [(MV_QPEL, 1, 2, 13, dict(display_width=97, display_height=65, search_range=16,
                                                            local_search_range=16)),
                                  (MV_HPEL_BILINEAR, 2, 3, 14, dict(search_range=16, local_search_range=16, rnd=1)),
                                  (MV_QPEL, 1, 3, 17, dict(search_range=0, local_search_range=0)),
                                  (MV_QPEL, 2, 3, 19, dict(search_range=96, local_search_range=8, long_range_mode=1))])
def test_b_analysis_matches_reference_live(oracle, case):
    Reference = _ref_or_skip()
    mode, num, den, seed, kw = case
    clip = synth.generate(98, 66, 3, seed)
    p = make_params(98, 66, **kw)
    R = Reference(p)
    past, cur, fut = clip.frame(0), clip.frame(1), clip.frame(2)
    rp, rc, rf = R.frame(past), R.frame(cur), R.frame(fut)
    anc = R.analyze_p_core(rf, rp, MV_MIXED, True, seed=R.analyze_p_core(rf, rp, MV_QPEL, False).mvs)
    e = R.analyze_b(rc, rp, rf, anc.mvs, anc.use_4mv, num, den, mode)
    assert oracle.analyze_b(p, cur, past, fut, anc.mvs, anc.use_4mv, num, den, mode).equal(e) == []


# ---- intensity compensation (estimate_intensity_comp, intensity_compensated_reference) ----

IC_CASES = ((98, 66), (130, 98), (352, 288), (66, 50), (16, 16))
IC_FIXED = ((1, 0, 5), (1, 0, 40), (1, 63, 60), (1, 17, 33), (0, 0, 0))
IC_PARAMS = (dict(search_range=16, local_search_range=16),
             dict(display_width=125, display_height=93, search_range=16, local_search_range=16),
             dict(search_range=16, local_search_range=16), dict(search_range=8, local_search_range=8),
             dict(search_range=8, local_search_range=8))


@pytest.mark.parametrize("i", range(len(IC_CASES)))
def test_intensity_golden(oracle, i):
    """The fade estimate along the reference's own quarter-pel field, and the compensated planes."""
    g = load("ic_kat.npz")
    w, h = IC_CASES[i]
    p = make_params(w, h, **IC_PARAMS[i])
    ref, cur = _frames(g, f"c{i}.ref"), _frames(g, f"c{i}.cur")
    ic = oracle.estimate_intensity_comp(p, cur, ref, g[f"c{i}.mvs"])
    assert ic == tuple(g[f"c{i}.ic"].tolist())
    if f"c{i}.map0.y" in g.files:
        for j, k in enumerate((ic,) + IC_FIXED):
            for got, c in zip(oracle.intensity_compensate(ref, k), "yuv"):
                assert np.array_equal(got, g[f"c{i}.map{j}.{c}"]), (j, c)


def test_intensity_fixture_covers_both_outcomes():
    g = load("ic_kat.npz")
    states = {int(g[f"c{i}.ic"][0]) for i in range(len(IC_CASES))}
    assert states == {0, 1}


@pytest.mark.parametrize("case", [(98, 66, 11, 0.7, 25.0), (322, 242, 12, 1.15, -12.0), (130, 98, 13, 1.0, 0.0)])
def test_intensity_matches_reference_live(oracle, case):
    Reference = _ref_or_skip()
    w, h, seed, a, b = case
    clip = synth.generate(w, h, 2, seed)
    ref, cur = clip.frame(0), synth.fade(clip.frame(1), a, b, seed)
    p = make_params(w, h, search_range=16, local_search_range=16)
    R = Reference(p)
    rc, rr = R.frame(cur), R.frame(ref)
    q = R.analyze_p_core(rc, rr, MV_QPEL, False)
    ic = R.estimate_intensity_comp(rc, rr, q.mvs)
    assert oracle.estimate_intensity_comp(p, cur, ref, q.mvs) == ic
    for k in (ic, (1, 0, 33), (1, 45, 12)):
        for x, y in zip(oracle.intensity_compensate(ref, k), R.intensity_compensate(rr, k)):
            assert np.array_equal(x, y)


# ---- scene-change score (scene_change_score) ----

@pytest.mark.parametrize("name", ["motion", "cut", "cut_low_threshold", "fade", "fade_no_compensation", "zoom_rescue",
                                  "zoom_rescue_fade", "range0"])
def test_scene_score_golden(oracle, name):
    from scene_cases import scene_pictures

    g = load("scene_kat.npz")
    cur, ref, fade, thr, kw = scene_pictures()[name]
    h, w = cur[0].shape
    got = oracle.scene_change_score(make_params(w, h, **kw), cur, ref, fade, thr)
    assert np.float64(got).view(np.uint64) == g[f"{name}.score"].view(np.uint64)


def test_scene_fixture_covers_every_path():
    """The cases reach the cut, the fade rescue and the zoom rescue (scores below the plain one)."""
    g = load("scene_kat.npz")
    assert float(g["cut.score"]) >= 28.0
    assert float(g["fade.score"]) < float(g["fade_no_compensation.score"])
    assert float(g["zoom_rescue.score"]) < 10.0 * 0.86 and float(g["zoom_rescue_fade.score"]) < 12.0 * 0.86


@pytest.mark.parametrize("case", [(322, 242, 21, 1.0, 0.0, 1, 28.0), (98, 66, 22, 0.7, 20.0, 1, 3.0),
                                  (194, 146, 23, 1.0, 0.0, 0, 0.5)])
def test_scene_score_matches_reference_live(oracle, case):
    Reference = _ref_or_skip()
    w, h, seed, a, b, fade, thr = case
    clip = synth.generate(w, h, 2, seed, global_px=12.0)
    cur = synth.fade(clip.frame(1), a, b, seed) if a != 1.0 else clip.frame(1)
    p = make_params(w, h, search_range=48, local_search_range=16)
    R = Reference(p)
    assert oracle.scene_change_score(p, cur, clip.frame(0), fade, thr) == \
        R.scene_change_score(R.frame(cur), R.frame(clip.frame(0)), fade, thr)


# ---- reconstruction (inverse_partition + add, evaluate_transform_parent) ----

RECON_QP = ((3, 0, 1), (8, 1, 1), (17, 1, 0), (31, 0, 0))


@pytest.mark.parametrize("qp", RECON_QP)
def test_reconstruction_golden(oracle, qp):
    pq, nu, hq = qp
    key = f"pq{pq}_nu{nu}_hq{hq}"
    g, x = load("recon_kat.npz"), load("xform_kat.npz")
    p = make_params(64, 48, pqindex=pq, nonuniform=nu, halfqp=hq, search_range=8, local_search_range=8)
    cur, pred = _frames(x, "cur"), _frames(x, f"{key}.pred")
    _co, lv = oracle.forward_quant(p, cur, pred, 15)
    for name, levels in (("coded", lv), ("random", g[f"{key}.random_levels"])):
        for got, c in zip(oracle.reconstruct(p, pred, levels, 15, g[f"{key}.types"]), "yuv"):
            assert np.array_equal(got, g[f"{key}.{name}.{c}"]), (name, c)


@pytest.mark.parametrize("tm", [1, 2, 4, 8, 6])
def test_reconstruction_matches_reference_live(oracle, tm):
    Reference = _ref_or_skip()
    clip = synth.generate(98, 66, 2, 40 + tm)
    p = make_params(98, 66, search_range=8, local_search_range=8, pqindex=6, nonuniform=1, halfqp=1)
    R = Reference(p)
    cur, ref = clip.frame(1), clip.frame(0)
    q = oracle.analyze_p_core(p, cur, ref, MV_QPEL, False)
    pred = oracle.motion_compensate(p, ref, q, MV_QPEL)
    _co, lv = oracle.forward_quant(p, cur, pred, tm)
    rng = np.random.default_rng(tm)
    types = rng.choice([t for t in range(1, 5) if tm & (1 << (t - 1))], (lv.shape[1], 6)).astype(np.uint8)
    for x, y in zip(oracle.reconstruct(p, pred, lv, tm, types), R.reconstruct(R.frame(pred), lv, tm, types)):
        assert np.array_equal(x, y)


# ---- in-loop deblocking (apply_i_like_loop_filter, apply_p_loop_filter) ----

LF_CASES = ((98, 66, 8), (130, 98, 20), (66, 50, 3), (194, 146, 31))


@pytest.mark.parametrize("i", range(len(LF_CASES)))
def test_loop_filter_golden(oracle, i):
    g = load("lf_kat.npz")
    w, h, pq = LF_CASES[i]
    p = make_params(w, h, pqindex=pq)
    fr = _frames(g, f"c{i}.in")
    for got, c in zip(oracle.loop_filter(p, fr), "yuv"):
        assert np.array_equal(got, g[f"c{i}.i.{c}"]), ("i", c)
    meta = [g[f"c{i}.{k}"] for k in ("bmv", "cbp", "tt", "intra")]
    for got, c in zip(oracle.loop_filter(p, fr, *meta), "yuv"):
        assert np.array_equal(got, g[f"c{i}.p.{c}"]), ("p", c)
    assert not np.array_equal(g[f"c{i}.p.y"], fr[0])  # the filter does change the picture


@pytest.mark.parametrize("seed", [5, 6])
def test_loop_filter_matches_reference_live(oracle, seed):
    from lf_cases import blocky_frame, metadata

    Reference = _ref_or_skip()
    w, h = 322, 242
    p = make_params(w, h, pqindex=10 + seed)
    R = Reference(p)
    fr = blocky_frame(w, h, seed)
    meta = metadata(w, h, seed, dense=seed % 2 == 0)
    for x, y in zip(oracle.loop_filter(p, fr, *meta), R.loop_filter(fr, *meta)):
        assert np.array_equal(x, y)


# ---- overlap smoothing (apply_i_overlap / apply_p_overlap) ----------------------------------

@pytest.mark.parametrize("i", range(6))
def test_overlap_golden(oracle, i):
    from ovl_cases import OVL_CASES, mb_flags, signed_planes

    g = load("ovl_kat.npz")
    w, h, pq, seed = OVL_CASES[i]
    p = make_params(w, h, pqindex=pq)
    planes, flags = signed_planes(w, h, seed), mb_flags(w, h, seed)
    runs = {"all": oracle.overlap_smooth(p, planes, all_edges=True), "sel": oracle.overlap_smooth(p, planes, flags)}
    # apply_p_overlap runs only at PQINDEX >= 9 (with OVERLAP on)
    runs["p"] = oracle.overlap_smooth(p, planes, flags) if pq >= 9 else planes
    for tag, got in runs.items():
        for x, c in zip(got, "yuv"):
            assert np.array_equal(x, g[f"c{i}.{tag}.{c}"]), (tag, c)
    if w >= 32:
        assert not np.array_equal(g[f"c{i}.all.y"], planes[0])  # the filter does change the picture


@pytest.mark.parametrize("seed", [7, 8])
def test_overlap_matches_reference_live(oracle, seed):
    from ovl_cases import mb_flags, signed_planes

    Reference = _ref_or_skip()
    w, h = 322, 242
    p = make_params(w, h, pqindex=9 + seed)
    R = Reference(p)
    planes, flags = signed_planes(w, h, seed), mb_flags(w, h, seed)
    for got, want in ((oracle.overlap_smooth(p, planes, all_edges=True), R.overlap(planes, 1)),
                      (oracle.overlap_smooth(p, planes, flags), R.overlap(planes, 2, flags)),
                      (oracle.overlap_smooth(p, planes, flags), R.overlap(planes, 0, flags, p_picture=True))):
        for x, y in zip(got, want):
            assert np.array_equal(x, y)


def test_store_signed_clamps_and_masks(oracle):
    from ovl_cases import mb_flags, signed_planes

    w, h = 98, 66
    p = make_params(w, h)
    planes, mask = signed_planes(w, h, 9), mb_flags(w, h, 9)
    y, u, v = oracle.store_signed(p, planes, 128)
    assert y.shape == (80, 112) and u.shape == (40, 56)
    assert np.array_equal(y, np.clip(planes[0] + 128, 0, 255))
    base = tuple(np.full(s, 7, np.uint8) for s in ((h, w), (h // 2, w // 2), (h // 2, w // 2)))
    my, mu, _ = oracle.store_signed(p, planes, 128, mask, into=base)
    m = mask.reshape(5, 7).repeat(16, 0).repeat(16, 1)[:h, :w].astype(bool)
    assert np.array_equal(my[m], np.clip(planes[0][:h, :w] + 128, 0, 255)[m]) and (my[~m] == 7).all()
    mc = mask.reshape(5, 7).repeat(8, 0).repeat(8, 1)[:h // 2, :w // 2].astype(bool)
    assert np.array_equal(mu[mc], np.clip(planes[1][:h // 2, :w // 2] + 128, 0, 255)[mc]) and (mu[~mc] == 7).all()


# ---- transform type of the throughput preset (choose_transform_mb, fast transform RDO) ----

TT_CASES = ((98, 66, 4), (130, 98, 12), (322, 242, 6), (16, 16, 1), (354, 290, 3), (98, 66, 10))


@pytest.mark.parametrize("i", range(len(TT_CASES)))
def test_fast_transform_types_golden(oracle, i):
    g = load("tt_kat.npz")
    w, h, pq = TT_CASES[i]
    p = make_params(w, h, search_range=8, local_search_range=8, pqindex=pq)
    got = oracle.fast_transform_types(p, planes(g[f"c{i}.cur"]), planes(g[f"c{i}.pred"]))
    assert np.array_equal(got, g[f"c{i}.types"])


def test_fast_transform_fixture_reaches_every_type():
    g = load("tt_kat.npz")
    assert set(np.concatenate([g[f"c{i}.types"] for i in range(len(TT_CASES))]).tolist()) == {1, 2, 3, 4}


def test_loop_filter_padded_frame_matches_reference_live(oracle):
    """The reference filters the padded reconstruction of its configuration; filtering that frame
    under the padded raster's dimensions gives the same samples."""
    from lf_cases import blocky_frame, metadata

    Reference = _ref_or_skip()
    fr = blocky_frame(336, 256, 25)
    pp = make_params(336, 256, pqindex=13)
    R = Reference(pp)
    meta = metadata(322, 242, 26, True)
    for x, y in zip(oracle.loop_filter(pp, fr, *meta), R.loop_filter(fr, *meta)):
        assert np.array_equal(x, y)
