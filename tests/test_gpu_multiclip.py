"""The batched form: many clips of uneven size in one persistent launch per frame step.

Every clip's P picture of a frame step contributes its whole analysis chain (the quarter-pel seed
pass, the three seeded mode passes and the final Mixed-MV pass with P-intra, analyze_p_picture's
passes, encoder_motion.cpp:524-597) to ONE vc1cu_core_passes_multi call; each pass carries its
own raster, display crop, PQINDEX and rounding control. Every result must equal the oracle's
chain for that clip alone, bit for bit.
"""
import pytest

from libvc1_b200 import synth
from libvc1_b200.abi import MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED, MV_QPEL, make_params

pytestmark = pytest.mark.gpu

# (coded width, height, display crop, PQINDEX, rnd, seed, global px)
CLIPS = [
    (96, 64, None, 6, 0, 1, 3.0),
    (160, 96, None, 9, 1, 2, 6.0),
    (322, 242, (321, 241), 5, 0, 3, 10.0),
    (352, 288, None, 12, 1, 4, 12.0),
    (208, 120, (203, 117), 4, 0, 5, 8.0),
    (640, 360, None, 8, 0, 6, 16.0),
]
RANGE = 32
MODES = (MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED)


def _params(c):
    w, h, disp, pq, rnd, _, _ = c
    kw = dict(display_width=disp[0], display_height=disp[1]) if disp else {}
    return make_params(w, h, search_range=RANGE, local_search_range=RANGE, pqindex=pq, rnd=rnd, **kw)


def test_uneven_clips_in_one_launch_per_frame_step(ctx, oracle):
    clips = [synth.generate(c[0], c[1], 3, 40 + c[5], global_px=c[6], n_objects=2, obj_min=16, obj_max=40)
             for c in CLIPS]
    params = [_params(c) for c in CLIPS]
    for k, clip in enumerate(clips):
        for t in range(3):
            ctx.upload_frame(100 * k + t, *clip.frame(t))
    for t in (1, 2):
        plist, passes = [], []
        for k in range(len(clips)):
            cur, ref, base = 100 * k + t, 100 * k + t - 1, 1000 + 10 * k
            plist.append(params[k])
            passes.append((cur, ref, MV_QPEL, 0, -1, base))
            for j, m in enumerate(MODES):
                plist.append(params[k])
                passes.append((cur, ref, m, 0, base, base + 1 + j))
            plist.append(params[k])
            passes.append((cur, ref, MV_MIXED, 1, base + 3, base + 4))
        ctx.core_passes_multi(plist, passes)
        for k, clip in enumerate(clips):
            p, base = params[k], 1000 + 10 * k
            cur, ref = clip.frame(t), clip.frame(t - 1)
            e = oracle.analyze_p_core(p, cur, ref, MV_QPEL, False)
            assert ctx.read_result(p, base).equal(e) == [], (k, t, "seed")
            em = None
            for j, m in enumerate(MODES):
                em = oracle.analyze_p_core(p, cur, ref, m, False, seed=e.mvs, seed_distant=e)
                assert ctx.read_result(p, base + 1 + j).equal(em) == [], (k, t, m)
            ef = oracle.analyze_p_core(p, cur, ref, MV_MIXED, True, seed=em.mvs, seed_distant=em)
            assert ctx.read_result(p, base + 4).equal(ef) == [], (k, t, "final")


def test_multi_launch_rejects_mixed_search_configurations(ctx):
    from libvc1_b200.api import Vc1cuError

    clip = synth.generate(96, 64, 2, 9)
    ctx.upload_frame(0, *clip.frame(1))
    ctx.upload_frame(1, *clip.frame(0))
    a = make_params(96, 64, search_range=16, local_search_range=16)
    b = make_params(96, 64, search_range=32, local_search_range=32)
    with pytest.raises(Vc1cuError) as e:
        ctx.core_passes_multi([a, b], [(0, 1, MV_QPEL, 0, -1, 1100), (0, 1, MV_QPEL, 0, -1, 1101)])
    assert e.value.code == 1


def _step_passes(clips, params, t):
    plist, passes = [], []
    for k in range(len(clips)):
        cur, ref, base = 100 * k + t, 100 * k + t - 1, 1000 + 10 * k
        plist.append(params[k])
        passes.append((cur, ref, MV_QPEL, 0, -1, base))
        for j, m in enumerate(MODES):
            plist.append(params[k])
            passes.append((cur, ref, m, 0, base, base + 1 + j))
        plist.append(params[k])
        passes.append((cur, ref, MV_MIXED, 1, base + 3, base + 4))
    return plist, passes


def _read_all(ctx, clips, params):
    out = []
    for k in range(len(clips)):
        for j in range(5):
            out.append(ctx.read_result(params[k], 1000 + 10 * k + j))
    return out


def test_graph_of_a_gop_replays_the_direct_results(ctx):
    """Two frame steps of every clip captured as one CUDA graph; each replay writes exactly what
    the direct calls wrote."""
    clips = [synth.generate(c[0], c[1], 3, 60 + c[5], global_px=c[6], n_objects=2, obj_min=16, obj_max=40)
             for c in CLIPS]
    params = [_params(c) for c in CLIPS]
    for k, clip in enumerate(clips):
        for t in range(3):
            ctx.upload_frame(100 * k + t, *clip.frame(t))
    steps = [_step_passes(clips, params, t) for t in (1, 2)]
    for plist, passes in steps:  # direct, which also builds every launch's tables
        ctx.core_passes_multi(plist, passes)
    direct = _read_all(ctx, clips, params)
    ctx.graph_begin()
    for plist, passes in steps:
        ctx.core_passes_multi(plist, passes)
    g = ctx.graph_end()
    try:
        for _ in range(2):
            ctx.graph_launch(g)
            got = _read_all(ctx, clips, params)
            assert all(a.equal(b) == [] for a, b in zip(got, direct))
    finally:
        ctx.graph_destroy(g)


def test_autotuned_shape_keeps_results(ctx, oracle):
    clips = [synth.generate(c[0], c[1], 2, 80 + c[5], global_px=c[6], n_objects=2, obj_min=16, obj_max=40)
             for c in CLIPS]
    params = [_params(c) for c in CLIPS]
    for k, clip in enumerate(clips):
        for t in range(2):
            ctx.upload_frame(100 * k + t, *clip.frame(t))
    plist, passes = _step_passes(clips, params, 1)
    warps, blocks, ms = ctx.autotune(plist, passes)
    assert 1 <= warps <= 4 and blocks >= 0 and ms > 0
    ctx.core_passes_multi(plist, passes)
    for k, clip in enumerate(clips):
        e = oracle.analyze_p_core(params[k], clip.frame(1), clip.frame(0), MV_QPEL, False)
        assert ctx.read_result(params[k], 1000 + 10 * k).equal(e) == []
