"""The P picture's motion-mode decision on the device (vc1cu_p_motion_bits, vc1cu_analyze_p_picture)
against the reference's own Vc1Encoder::analyze_p_picture (oracle/_ref, scalar path):

- estimate_p_motion_bits of device analyses in all four modes, plain and with the
  intensity-compensation header, on rasters that take every branch of the MVTYPEMB bitplane's
  NORM-6 coding (2x3 tiles with and without the skip-coded first column, 3x2 tiles with 0, 1 or 2
  lead columns and the skip-coded first row);
- the four candidates' motion bits and sampled mode-RD scores (the reference's long double,
  rounded to double on both sides);
- the whole picture: the chosen mode, the fade-compensation decision, the returned analysis bit
  for bit and its motion bits, under the default presets, scalar quantisation, 8x8-only
  transforms, the fixed-8x8 shortcut and a faded picture whose compensated analysis wins;
- the B picture's quarter-pel versus bilinear choice of analyze_b_picture: both analyses'
  sampled_b_mode_rd scores (B-intra samples included) and the choice, at fractions 1/2, 1/3 and
  2/3, with the same transform configurations."""
import numpy as np
import pytest

from libvc1_b200 import synth
from libvc1_b200.abi import MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED, MV_QPEL, make_params, make_ppic_cfg
from oracle.bindings import Reference, ref_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")]

MODES = (MV_QPEL, MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED)

RASTERS = {
    # (w, h, display): MB raster and the NORM-6 branch it takes
    "11x9_2x3_odd": (176, 144, None),          # h % 3 == 0, w odd: 2x3 tiles + first column
    "10x6_2x3_even": (160, 96, None),          # h % 3 == 0, w even
    "12x8_3x2": (192, 128, None),              # 3x2 tiles, no lead column
    "13x8_3x2_lead1": (208, 128, (203, 121)),  # one lead column, cropped display
    "14x7_3x2_lead2_oddrow": (224, 112, None),  # two lead columns and the first row
}


def _clip(w, h, seed):
    return synth.generate(w, h, 2, seed, global_px=5.0, n_objects=4, obj_min=12, obj_max=40, obj_vel=4.0, sigma=2.0)


@pytest.mark.parametrize("case", sorted(RASTERS))
def test_motion_bits_match_reference(ctx, case):
    w, h, disp = RASTERS[case]
    kw = dict(display_width=disp[0], display_height=disp[1]) if disp else {}
    p = make_params(w, h, search_range=16, local_search_range=16, pqindex=7, **kw)
    clip = _clip(w, h, 400 + w + h)
    ctx.upload_frame(0, *clip.frame(0))
    ctx.upload_frame(1, *clip.frame(1))
    ctx.core_passes(p, [(1, 0, MV_QPEL, 0, -1, 800)])
    ctx.core_passes(p, [(1, 0, m, 0, 800, 801 + i) for i, m in enumerate(MODES[1:])])
    ctx.core_passes(p, [(1, 0, MV_MIXED, 1, 803, 804)])
    ref = Reference(p)
    four = 0
    for slot, mode in ((800, MV_QPEL), (801, MV_HPEL), (802, MV_HPEL_BILINEAR), (803, MV_MIXED), (804, MV_MIXED)):
        a = ctx.read_result(p, slot)
        if mode == MV_MIXED:
            four = max(four, int(a.use_4mv.sum()))
        for intensity in (False, True):
            want = ref.estimate_p_motion_bits(a, mode, intensity)
            assert want is not None
            assert ctx.p_motion_bits(p, slot, mode, intensity) == want, (slot, mode, intensity)
    assert four > 0  # the MVTYPEMB bitplane holds both values


def test_mode_scores_match_reference(ctx):
    w, h = 176, 144
    p = make_params(w, h, search_range=16, local_search_range=16, pqindex=9, nonuniform=1)
    clip = _clip(w, h, 411)
    ctx.upload_frame(0, *clip.frame(0))
    ctx.upload_frame(1, *clip.frame(1))
    cfg = make_ppic_cfg(fade_compensation=0)
    info = ctx.analyze_p_picture(p, cfg, 1, 0, 820, 830, 40)
    bits, scores = Reference(p).p_mode_scores(cfg, clip.frame(1), clip.frame(0))
    assert [int(b) for b in info.cand_bits[:4]] == [int(b) for b in bits]
    got = np.array(info.cand_score[:4], np.float64)
    assert np.array_equal(got.view(np.uint64), scores.astype(np.float64).view(np.uint64)), (got, scores)
    assert MODES[int(np.argmin(scores))] == info.mode or np.sum(scores == scores.min()) > 1


PICTURES = {
    # (w, h, display, pq, nonuniform, cfg overrides, fade)
    "default_presets": (176, 144, None, 8, 0, {}, None),
    "scalar_no_dquant": (208, 128, (203, 121), 11, 1, dict(trd_trellis=0, dquant=0), None),
    "eight_by_eight": (160, 96, None, 5, 0, dict(trd_variable_transforms=0), None),
    "fixed_8x8_shortcut": (160, 96, None, 6, 0, dict(trd_variable_transforms=0, fast_transform_rdo=1, dquant=0,
                                                      trd_trellis=0), None),
    "fade_wins": (176, 144, None, 8, 0, {}, (0.78, 12.0)),
}


@pytest.mark.parametrize("case", sorted(PICTURES))
def test_picture_matches_reference(ctx, case):
    w, h, disp, pq, nu, over, fade = PICTURES[case]
    kw = dict(display_width=disp[0], display_height=disp[1]) if disp else {}
    p = make_params(w, h, search_range=16, local_search_range=16, pqindex=pq, nonuniform=nu, **kw)
    clip = _clip(w, h, 430 + pq)
    cur = clip.frame(1) if fade is None else synth.fade(clip.frame(1), fade[0], fade[1], seed=pq)
    ctx.upload_frame(0, *clip.frame(0))
    ctx.upload_frame(1, *cur)
    cfg = make_ppic_cfg(**over)
    info = ctx.analyze_p_picture(p, cfg, 1, 0, 850, 860, 50)
    want, mode, ic, bits = Reference(p).analyze_p_picture_cfg(cfg, cur, clip.frame(0))
    assert info.mode == mode
    assert bool(info.weighted) == ic
    assert info.motion_bits == bits
    assert ctx.read_result(p, 850).equal(want) == []
    if fade is not None:
        assert info.ic.enabled and info.weighted  # the compensated analysis was kept


B_PICTURES = {
    # (w, h, display, pq, fraction, cfg overrides)
    "cif_half": (176, 144, None, 8, (1, 2), {}),
    "cropped_third_scalar": (208, 128, (203, 121), 11, (1, 3), dict(trd_trellis=0, dquant=0)),
    "two_thirds_8x8": (160, 96, None, 5, (2, 3), dict(trd_variable_transforms=0)),
    "fixed_8x8_shortcut": (160, 96, None, 6, (1, 2), dict(trd_variable_transforms=0, fast_transform_rdo=1, dquant=0,
                                                          trd_trellis=0)),
}


@pytest.mark.parametrize("case", sorted(B_PICTURES))
def test_b_mode_choice_matches_reference(ctx, case):
    """analyze_b_picture's quarter-pel versus bilinear choice (vc1cu_b_mode_rd on two vc1cu_b_decide
    results) against the reference's own two analyses and sampled_b_mode_rd scores."""
    w, h, disp, pq, (num, den), over = B_PICTURES[case]
    kw = dict(display_width=disp[0], display_height=disp[1]) if disp else {}
    p = make_params(w, h, search_range=16, local_search_range=16, pqindex=pq, **kw)
    clip = synth.generate(w, h, 3, 470 + pq, global_px=4.0, n_objects=4, obj_min=12, obj_max=40, obj_vel=4.0, sigma=2.0)
    for t in range(3):
        ctx.upload_frame(t, *clip.frame(t))
    # the future anchor (picture 2 against picture 0), then both modes' B passes and decisions
    ctx.core_passes(p, [(2, 0, MV_QPEL, 0, -1, 870)])
    ctx.core_passes(p, [(2, 0, MV_MIXED, 1, 870, 871)])
    ctx.core_passes(p, [(1, 0, MV_QPEL, 0, -1, 872), (1, 2, MV_QPEL, 0, -1, 873),
                        (1, 0, MV_HPEL_BILINEAR, 0, -1, 874), (1, 2, MV_HPEL_BILINEAR, 0, -1, 875)])
    ctx.b_decide(p, [(1, 0, 2, 872, 873, 871, num, den, MV_QPEL, 60),
                     (1, 0, 2, 874, 875, 871, num, den, MV_HPEL_BILINEAR, 61)])
    cfg = make_ppic_cfg(**over)
    choice, (qs, hs) = ctx.b_mode_rd(p, cfg, 1, 0, 2, 60, 61, 62)
    anc = ctx.read_result(p, 871)
    scores, chosen = Reference(p).b_mode_scores(cfg, clip.frame(1), clip.frame(0), clip.frame(2), anc.mvs,
                                                anc.use_4mv, num, den)
    got = np.array([qs, hs], np.float64)
    assert np.array_equal(got.view(np.uint64), scores.astype(np.float64).view(np.uint64)), (got, scores)
    assert choice == chosen
