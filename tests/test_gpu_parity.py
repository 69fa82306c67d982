"""Parity of the CUDA path with the oracle (bit-exact), through the C ABI.

The candidate-scoring cases restate the reference's own GPU parity test,
tests/vulkan_compute_runtime.cpp:31-114 (48x40 LCG frames, 20 quarter-pel vectors, SAD and
SATD at (5,7), bilinear SAD at (3,4), integer SAD at sample strides 2 and 4).
"""
import numpy as np
import pytest

from libvc1_b200 import synth
from libvc1_b200.abi import (BAD_COST, LAW_CPU, LAW_SHADER, METRIC_SAD, METRIC_SATD, MODES, MV_HPEL, MV_HPEL_BILINEAR,
                             MV_MIXED, MV_QPEL, make_params)

pytestmark = pytest.mark.gpu

MVS = [(0, 0), (4, 0), (-4, 0), (0, 4), (0, -4), (3, 1), (-3, 2), (7, -5), (-9, -7), (12, 8), (-16, 11), (1, 3), (2, 2),
       (-1, -3), (20, -12), (-23, 17), (31, 29), (-32, -27), (5, -19), (-21, 6)]


def lcg_frames():
    x = np.arange(48)[None, :]
    y = np.arange(40)[:, None]
    cur = ((x * 13 + y * 29 + (x * y) % 37 + 17) & 255).astype(np.uint8)
    ref = ((x * 7 + y * 19 + (x * y) % 53 + 61) & 255).astype(np.uint8)
    u = np.full((20, 24), 128, np.uint8)
    return (cur, u, u), (ref, u, u)


def test_score_batch_reference_fixture(ctx, oracle):
    cur, ref = lcg_frames()
    p = make_params(48, 40)
    for bil, metric, x0, y0 in ((0, METRIC_SAD, 5, 7), (0, METRIC_SATD, 5, 7)):
        ok, got, err = ctx.score_motion_batch(cur[0], ref[0], 48, 40, x0, y0, 16, 16, 1, bil, 0, metric, MVS)
        assert ok, err
        mode = MV_QPEL
        want = [oracle.block_sad_motion(p, cur, ref, x0, y0, 16, 16, xq, yq, mode) if metric == METRIC_SAD else
                oracle.block_satd_motion(p, cur, ref, x0, y0, 16, 16, xq, yq, mode) for xq, yq in MVS]
        assert got.tolist() == want
    half = [mv for mv in MVS if not (mv[0] & 1) and not (mv[1] & 1)]
    ok, got, err = ctx.score_motion_batch(cur[0], ref[0], 48, 40, 3, 4, 16, 16, 1, 1, 0, METRIC_SAD, half)
    assert ok, err
    assert got.tolist() == [oracle.block_sad_motion(p, cur, ref, 3, 4, 16, 16, xq, yq, MV_HPEL_BILINEAR)
                            for xq, yq in half]
    integer = [mv for mv in MVS if mv[0] % 4 == 0 and mv[1] % 4 == 0]
    for stride in (2, 4):
        ok, got, err = ctx.score_motion_batch(cur[0], ref[0], 48, 40, 5, 7, 16, 16, stride, 0, 0, METRIC_SAD, integer)
        assert ok, err
        want = [oracle.shader_cost(cur, ref, 5, 7, 16, 16, stride, 0, 0, METRIC_SAD, xq, yq) for xq, yq in integer]
        assert got.tolist() == want
    c = ctx.counters()
    assert c["dispatches"] >= 5 and c["candidates"] > 0 and c["frame_uploads"] >= 2


@pytest.mark.parametrize("rnd", [0, 1])
def test_score_batch_shader_law_random(ctx, oracle, rnd):
    rng = np.random.default_rng(5 + rnd)
    cur = rng.integers(0, 256, (50, 66), dtype=np.uint8)
    ref = rng.integers(0, 256, (50, 66), dtype=np.uint8)
    u = np.full((25, 33), 128, np.uint8)
    mvs = rng.integers(-40, 41, (200, 2)).astype(np.int32)
    for bil in (0, 1):
        for metric in (METRIC_SAD, METRIC_SATD):
            for (x0, y0, bw, bh) in ((0, 0, 16, 16), (50, 34, 16, 16), (9, 13, 8, 8), (60, 44, 8, 8)):
                ok, got, err = ctx.score_motion_batch(cur, ref, 66, 50, x0, y0, bw, bh, 1, bil, rnd, metric, mvs)
                assert ok, err
                want = [oracle.shader_cost((cur, u, u), (ref, u, u), x0, y0, bw, bh, 1, bil, rnd, metric, int(a), int(b))
                        for a, b in mvs]
                assert got.tolist() == want


def test_score_batch_cpu_law_hidden_padding(ctx, oracle):
    clip = synth.generate(66, 50, 2, 3)
    p = make_params(66, 50, display_width=61, display_height=45, search_range=16, local_search_range=16, rnd=1)
    cur, ref = clip.frame(1), clip.frame(0)
    rng = np.random.default_rng(9)
    mvs = rng.integers(-30, 31, (300, 2)).astype(np.int32)
    for mode in MODES:
        for (x0, y0, bw, bh) in ((48, 32, 16, 16), (56, 40, 8, 8), (16, 16, 16, 16)):
            got = ctx.score_motion_batch_law(p, LAW_CPU, cur[0], ref[0], x0, y0, bw, bh, 1, mode, METRIC_SAD, mvs)
            want = [oracle.block_sad_motion(p, cur, ref, x0, y0, bw, bh, int(a), int(b), mode) for a, b in mvs]
            assert got.tolist() == want
            got = ctx.score_motion_batch_law(p, LAW_CPU, cur[0], ref[0], x0, y0, bw, bh, 1, mode, METRIC_SATD, mvs)
            want = [oracle.block_satd_motion(p, cur, ref, x0, y0, bw, bh, int(a), int(b), mode) for a, b in mvs]
            assert got.tolist() == want
    ints = (mvs // 4) * 4
    for stride in (1, 2, 4):
        got = ctx.score_motion_batch_law(p, LAW_CPU, cur[0], ref[0], 48, 32, 16, 16, stride, MV_QPEL, METRIC_SAD, ints)
        want = [oracle.mb_sad(p, cur, ref, 3, 2, int(a) // 4, int(b) // 4, stride) for a, b in ints]
        assert got.tolist() == want
    assert BAD_COST in got.tolist()


def _upload(ctx, clip, t0, t1):
    ctx.upload_frame(0, *clip.frame(t0))
    ctx.upload_frame(1, *clip.frame(t1))


CASES = {
    "cif_r8": (lambda: synth.cif_plain(frames=2, seed=1), dict(search_range=8, local_search_range=8)),
    "cif_r32": (lambda: synth.cif_plain(frames=2, seed=3), dict(search_range=32, local_search_range=32, pqindex=4)),
    "odd_321x241": (lambda: synth.generate(322, 242, 2, 4),
                    dict(display_width=321, display_height=241, search_range=32, local_search_range=32, rnd=1)),
    "diamond": (lambda: synth.cif_plain(frames=2, seed=5), dict(search_range=16, local_search_range=16, me_algorithm=1)),
    "fast_subpel": (lambda: synth.cif_plain(frames=2, seed=6), dict(search_range=16, local_search_range=16, fast_subpel=1)),
    "me_rate": (lambda: synth.cif_plain(frames=2, seed=7), dict(search_range=16, local_search_range=16, me_quality=1)),
    "me_sad": (lambda: synth.cif_plain(frames=2, seed=8), dict(search_range=16, local_search_range=16, me_quality=0)),
    "me_sad_fast": (lambda: synth.cif_plain(frames=2, seed=8),
                    dict(search_range=16, local_search_range=16, me_quality=0, fast_subpel=1)),
    "pq20_subpel2": (lambda: synth.cif_plain(frames=2, seed=9),
                     dict(search_range=16, local_search_range=16, pqindex=20, subpel_range=2)),
    "range0": (lambda: synth.cif_plain(frames=2, seed=2), dict(search_range=0, local_search_range=0)),
    "tiny_16x16": (lambda: synth.generate(16, 16, 2, 2, n_objects=0), dict(search_range=8, local_search_range=8)),
    # long-range search (search range beyond the local range): compare, local-good skip, legacy
    "longrange_compare": (lambda: synth.generate(352, 288, 2, 9, global_px=40.0, n_objects=2),
                          dict(search_range=128, local_search_range=16)),
    "longrange_skip": (lambda: synth.generate(352, 288, 2, 9, global_px=40.0, n_objects=2),
                       dict(search_range=128, local_search_range=16, long_range_mode=1)),
    "longrange_legacy": (lambda: synth.generate(352, 288, 2, 9, global_px=40.0, n_objects=2),
                         dict(search_range=128, local_search_range=16, long_range_mode=2)),
    "longrange_odd_diamond": (lambda: synth.generate(322, 242, 2, 31, global_px=60.0, n_objects=3),
                              dict(display_width=321, display_height=241, search_range=96, local_search_range=8,
                                   me_algorithm=1)),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_core_passes_match_oracle(ctx, oracle, case):
    make, kw = CASES[case]
    clip = make()
    p = make_params(clip.width, clip.height, **kw)
    cur, ref = clip.frame(1), clip.frame(0)
    _upload(ctx, clip, 0, 1)
    g = ctx.analyze_p_core(p, 1, 0, MV_QPEL, False)
    e = oracle.analyze_p_core(p, cur, ref, MV_QPEL, False)
    assert g.equal(e) == []
    for mode in (MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED):
        for intra in (False, True):
            gs = ctx.analyze_p_core(p, 1, 0, mode, intra, seed=g.mvs, seed_distant=g)
            es = oracle.analyze_p_core(p, cur, ref, mode, intra, seed=e.mvs, seed_distant=e)
            assert gs.equal(es) == [], (mode, intra)


def test_batched_passes_match_oracle(ctx, oracle):
    """Several pictures in one persistent launch (interleaved work queue)."""
    clip = synth.cif_plain(frames=5, seed=12)
    p = make_params(clip.width, clip.height, search_range=16, local_search_range=16)
    for t in range(5):
        ctx.upload_frame(t, *clip.frame(t))
    ctx.core_passes(p, [(t, t - 1, MV_QPEL, 0, -1, 100 + t) for t in range(1, 5)])
    ctx.core_passes(p, [(t, t - 1, m, 0, 100 + t, 200 + 10 * t + m) for t in range(1, 5)
                        for m in (MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED)])
    ctx.core_passes(p, [(t, t - 1, MV_MIXED, 1, 200 + 10 * t + MV_MIXED, 300 + t) for t in range(1, 5)])
    for t in range(1, 5):
        cur, ref = clip.frame(t), clip.frame(t - 1)
        e = oracle.analyze_p_core(p, cur, ref, MV_QPEL, False)
        assert ctx.read_result(p, 100 + t).equal(e) == []
        for m in (MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED):
            em = oracle.analyze_p_core(p, cur, ref, m, False, seed=e.mvs, seed_distant=e)
            assert ctx.read_result(p, 200 + 10 * t + m).equal(em) == []
        ef = oracle.analyze_p_core(p, cur, ref, MV_MIXED, True, seed=em.mvs, seed_distant=em)
        assert ctx.read_result(p, 300 + t).equal(ef) == []


def test_seeded_passes_in_the_seed_launch_match_oracle(ctx, oracle):
    """Seed pass and seeded passes in ONE launch (per-MB cross-pass dependency), QP per pass."""
    clip = synth.generate(322, 242, 4, 21)
    p = make_params(322, 242, display_width=321, display_height=241, search_range=24, local_search_range=24)
    for t in range(4):
        ctx.upload_frame(t, *clip.frame(t))
    pqs = {1: 4, 2: 9, 3: 13}
    ctx.core_passes(p, [(t, t - 1, MV_QPEL, 0, -1, 400 + t, pqs[t]) for t in range(1, 4)] +
                    [(t, t - 1, m, int(m == MV_MIXED), 400 + t, 500 + 10 * t + m, pqs[t]) for t in range(1, 4)
                     for m in (MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED)])
    for t in range(1, 4):
        q = make_params(322, 242, display_width=321, display_height=241, search_range=24, local_search_range=24,
                        pqindex=pqs[t])
        cur, ref = clip.frame(t), clip.frame(t - 1)
        e = oracle.analyze_p_core(q, cur, ref, MV_QPEL, False)
        assert ctx.read_result(p, 400 + t).equal(e) == []
        for m in (MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED):
            em = oracle.analyze_p_core(q, cur, ref, m, m == MV_MIXED, seed=e.mvs, seed_distant=e)
            assert ctx.read_result(p, 500 + 10 * t + m).equal(em) == [], (t, m)


@pytest.mark.parametrize("pq,nonuniform,halfqp", [(1, 0, 0), (4, 1, 0), (7, 0, 1), (8, 1, 1), (12, 1, 0), (31, 0, 0)])
def test_prediction_and_transform_match_oracle(ctx, oracle, pq, nonuniform, halfqp):
    clip = synth.generate(322, 242, 2, 4)
    p = make_params(322, 242, display_width=321, display_height=241, pqindex=pq, nonuniform=nonuniform, halfqp=halfqp,
                    search_range=16, local_search_range=16)
    _upload(ctx, clip, 0, 1)
    ctx.core_passes(p, [(1, 0, MV_QPEL, 0, -1, 20)])
    ctx.core_passes(p, [(1, 0, MV_MIXED, 1, 20, 21)])
    a = ctx.read_result(p, 21)
    ctx.motion_compensate(p, 0, 21, MV_MIXED, 2)
    pred = ctx.download_frame(2, 322, 242)
    want = oracle.motion_compensate(p, clip.frame(0), a, MV_MIXED)
    for x, y in zip(pred, want):
        assert np.array_equal(x, y)
    co, lv = ctx.forward_quant(p, 1, 2, 15)
    eco, elv = oracle.forward_quant(p, clip.frame(1), want, 15)
    assert np.array_equal(co.view(np.uint64), eco.view(np.uint64))
    assert np.array_equal(lv, elv)


def test_1080p_pass_chain_matches_oracle(ctx, oracle):
    clip = synth.hd1080(frames=2)
    p = make_params(1920, 1080, search_range=64, local_search_range=64, nonuniform=1, pqindex=8)
    cur, ref = clip.frame(1), clip.frame(0)
    _upload(ctx, clip, 0, 1)
    g = ctx.analyze_p_core(p, 1, 0, MV_QPEL, False)
    e = oracle.analyze_p_core(p, cur, ref, MV_QPEL, False)
    assert g.equal(e) == []
    gm = ctx.analyze_p_core(p, 1, 0, MV_MIXED, True, seed=g.mvs, seed_distant=g)
    em = oracle.analyze_p_core(p, cur, ref, MV_MIXED, True, seed=e.mvs, seed_distant=e)
    assert gm.equal(em) == []
