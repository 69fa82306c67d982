"""The transform RD of the default presets on the device (vc1cu_choose_transform) against the
reference's own Vc1Encoder::choose_transform_mb (oracle/_ref, scalar path), bit for bit: every
macroblock's type, signaling level, CBP, per-parent types and skip masks, estimated bits,
distortions (by bit pattern) and the chosen quantised levels.

The configurations cover trellis 0 / 1 / 2, the perceptual lambda scale on and off (and a
stronger one), macroblock-only signaling, 8x8-only and frame-level (TTFRM) decisions, every inter
coding set, Escape-3-only coding, per-macroblock MQUANT with DQUANTFRM, HRD, the non-uniform and
half-step quantisers, PQINDEX below 8 (11-bit levels) and cropped rasters whose edge macroblocks
must split."""
import numpy as np
import pytest

from libvc1_b200 import synth
from libvc1_b200.abi import MV_MIXED, MV_QPEL, make_params, make_trd_cfg, tdecisions_differ
from oracle.bindings import Reference, ref_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")]

CASES = {
    # (w, h, display, pq, nonuniform, halfqp, cfg overrides, per-MB mquant)
    "default_cif": (352, 288, None, 8, 0, 0, {}, False),
    "trellis0": (176, 144, None, 6, 0, 0, dict(trellis=0), False),
    "trellis2_nonuniform": (176, 144, None, 10, 1, 0, dict(trellis=2), False),
    "aq_off": (176, 144, None, 5, 0, 1, dict(adaptive_quality=0), False),
    "aq_strong_set3": (176, 144, None, 12, 0, 0, dict(aq_strength=2.5, coding_set=3), False),
    "mb_signaling_set5": (176, 144, None, 9, 0, 0, dict(extended_transform_signaling=0, coding_set=5), False),
    "esc3_only_set7": (176, 144, None, 3, 0, 0, dict(use_vlc=0, coding_set=7), False),
    "odd_crop_lowpq": (322, 242, (321, 241), 2, 0, 0, {}, False),
    "eight_by_eight_only": (176, 144, None, 7, 0, 0, dict(variable_transforms=0), False),
    "frame_level_4x8": (176, 144, None, 8, 1, 0, dict(frame_type=3), False),
    "dquant_mquant": (208, 120, (203, 117), 9, 0, 0, dict(dquantfrm=1), True),
    "hrd_mquant1": (176, 144, None, 1, 0, 0, dict(hrd_enabled=1, trellis=2), False),
}


def _prediction(ctx, p, clip):
    """The device's Mixed-MV prediction of frame 1 from frame 0 (analysis passes, then MC)."""
    ctx.upload_frame(0, *clip.frame(0))
    ctx.upload_frame(1, *clip.frame(1))
    ctx.core_passes(p, [(1, 0, MV_QPEL, 0, -1, 700)])
    ctx.core_passes(p, [(1, 0, MV_MIXED, 1, 700, 701)])
    ctx.motion_compensate(p, 0, 701, MV_MIXED, 2)
    return ctx.download_frame(2, p.width, p.height)


@pytest.mark.parametrize("case", sorted(CASES))
def test_transform_rd_matches_reference(ctx, case):
    w, h, disp, pq, nu, hq, over, per_mb = CASES[case]
    kw = dict(display_width=disp[0], display_height=disp[1]) if disp else {}
    p = make_params(w, h, search_range=16, local_search_range=16, pqindex=pq, nonuniform=nu, halfqp=hq, **kw)
    clip = synth.generate(w, h, 2, 300 + pq, global_px=4.0, n_objects=3, obj_min=16, obj_max=48, obj_vel=3.0,
                          sigma=2.5)
    pred = _prediction(ctx, p, clip)
    cfg = make_trd_cfg(**over)
    mbs = ((w + 15) // 16) * ((h + 15) // 16)
    mquant = None
    if per_mb:
        rng = np.random.default_rng(pq)
        mquant = np.where(rng.random(mbs) < 0.5, pq, rng.integers(1, 32, mbs)).astype(np.uint8)
    got, glv = ctx.choose_transform(p, cfg, 1, 2, mquant=mquant)
    want, wlv = Reference(p).choose_transform(cfg, clip.frame(1), pred, mquant=mquant)
    bad = tdecisions_differ(got, want)
    first = None
    if bad:
        f = bad[0]
        diff = np.nonzero(np.any((got[f] != want[f]).reshape(mbs, -1), axis=1))[0]
        first = (f, int(diff[0]), got[diff[0]], want[diff[0]])
    assert bad == [], first
    assert np.array_equal(glv, wlv)
    # the case exercises a choice: more than one type or signaling level across the picture
    if not over.get("frame_type") and over.get("variable_transforms", 1):
        assert len(set(got["type"].tolist())) > 1 or len(set(got["signal_level"].tolist())) > 1
