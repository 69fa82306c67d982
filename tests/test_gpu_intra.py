"""The I picture's signed intra reconstruction on the device (vc1cu_reconstruct_intra) against the
reference's own Vc1Encoder::reconstruct_i_signed_padded (oracle/_ref, scalar path), bit for bit on
the padded raster: full and cropped rasters, the uniform, non-uniform and half-step quantisers,
PQINDEX 1-2 (the wider DC range), overlap plans none / all / select (the edge source the transform
reads) and a DQUANT plan whose per-MB MQUANT scales the DC predictors; the trellis AC levels
(beams 4 and 8, with and without the perceptual lambda scale, on edge sources of cropped rasters
and under a DQUANT plan); and the I overlap plan (vc1cu_choose_i_overlap) against
choose_i_overlap_plan: every macroblock gaining (ALL), mixed gains scored against the OVERFLAGS
bits, none gaining, PQINDEX above the CONDOVER range, a cropped raster, a DQUANT plan and the
trellis."""
import numpy as np
import pytest

from libvc1_b200 import synth
from libvc1_b200.abi import make_params, make_trd_cfg, mbs_of
from oracle.bindings import Reference, ref_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")]

CASES = {
    # (w, h, display, pq, nonuniform, halfqp, overlap, dquant)
    "cif": (176, 144, None, 8, 0, 0, 0, False),
    "cropped_all": (322, 242, (317, 237), 12, 0, 0, 1, False),
    "cropped_select_nonuniform": (208, 120, (203, 113), 9, 1, 0, 2, False),
    "edge_rem1_halfqp": (130, 98, (129, 97), 5, 0, 1, 1, False),
    "pq1": (96, 64, None, 1, 0, 0, 0, False),
    "pq2_nonuniform": (98, 66, None, 2, 1, 0, 0, False),
    "dquant_plan": (176, 144, None, 10, 0, 0, 0, True),
    "dquant_cropped_all": (322, 242, (319, 239), 14, 1, 0, 1, True),
}

TRELLIS_CASES = {
    # the CASES fields, then (trellis, aq_strength)
    "trellis1_cif": (176, 144, None, 8, 0, 0, 0, False, 1, 1.0),
    "trellis2_cropped_all_nonuniform": (322, 242, (317, 237), 12, 1, 0, 1, False, 2, 1.0),
    "trellis1_cropped_select": (322, 242, (317, 237), 6, 0, 0, 2, False, 1, 1.0),
    "trellis1_no_aq_select": (208, 120, (203, 113), 9, 1, 0, 2, False, 1, 0.0),
    "trellis2_pq1": (96, 64, None, 1, 0, 0, 0, False, 2, 1.0),
    "trellis1_halfqp": (130, 98, (129, 97), 5, 0, 1, 1, False, 1, 0.5),
    "trellis1_dquant": (176, 144, None, 10, 0, 0, 0, True, 1, 1.0),
}


@pytest.mark.parametrize("case", sorted(CASES) + sorted(TRELLIS_CASES))
def test_intra_reconstruction_matches_reference(ctx, case):
    import torch

    if case in CASES:
        w, h, disp, pq, nu, hq, overlap, dquant = CASES[case]
        trellis, aq = 0, (1.0 if dquant else 0.0)
    else:
        w, h, disp, pq, nu, hq, overlap, dquant, trellis, aq = TRELLIS_CASES[case]
    kw = dict(display_width=disp[0], display_height=disp[1]) if disp else {}
    p = make_params(w, h, pqindex=pq, nonuniform=nu, halfqp=hq, **kw)
    mbw, mbh = mbs_of(p)
    clip = synth.generate(w, h, 1, 90 + pq, n_objects=3, obj_min=12, obj_max=40, sigma=3.0)
    flags = (np.random.default_rng(pq).random(mbw * mbh) < 0.5).astype(np.uint8) if overlap == 2 else None
    want, mq, der = Reference(p).reconstruct_intra(clip.frame(0), overlap, flags, dquant=dquant, aq_strength=aq,
                                                   trellis=trellis)
    cfg = make_trd_cfg(trellis=trellis, adaptive_quality=int(aq > 0), aq_strength=aq) if trellis else None
    if trellis:  # the trellis moves levels away from the scalar ones
        scalar, _, _ = Reference(p).reconstruct_intra(clip.frame(0), overlap, flags, dquant=dquant, aq_strength=aq)
        assert any(not np.array_equal(a, b) for a, b in zip(want, scalar))
    if dquant:
        assert len(np.unique(mq)) > 1 and der.any()
    ctx.upload_frame(0, *clip.frame(0))
    d = [torch.zeros((mbh * 16 // s, mbw * 16 // s), dtype=torch.int32, device="cuda") for s in (1, 2, 2)]
    torch.cuda.synchronize()
    ctx.reconstruct_intra(p, 0, *[t.data_ptr() for t in d], overlap=overlap, flags=flags,
                          mquant=mq if dquant else None, derived=der if dquant else None, cfg=cfg)
    ctx.synchronize()
    for got, exp, c in zip(d, want, "yuv"):
        g = got.cpu().numpy()
        assert np.array_equal(g, exp), (c, np.argwhere(g != exp)[:4])


def _overlap_content(kind, w, h):
    yy, xx = np.mgrid[0:h, 0:w]
    g = 40 + 0.8 * xx * 176 / w + 0.5 * yy * 144 / h
    if kind == "gradient":
        y = g
    else:  # a textured quadrant in the gradient: some macroblocks gain from smoothing, some lose
        t = 128 + 60 * np.sin(xx / 2.3) * np.cos(yy / 1.9) + np.random.default_rng(3).normal(0, 10, (h, w))
        y = np.where((xx < w // 2) & (yy < h // 2), t, g)
    y = np.clip(np.rint(y), 0, 255).astype(np.uint8)
    u = np.full((h // 2, w // 2), 128, np.uint8)
    return y, u, u.copy()


OVERLAP_PLANS = {
    # (w, h, display, pq, content, dquant, trellis): the plan the reference takes
    "gradient_all": (176, 144, None, 3, "gradient", False, 0),
    "mixed_scored_none": (176, 144, None, 3, "mixed", False, 0),
    "texture_none": (176, 144, None, 5, "synth", False, 0),
    "above_condover_all": (176, 144, None, 10, "synth", False, 0),
    "cropped_gradient": (322, 242, (317, 237), 3, "gradient", False, 0),
    "dquant_plan": (176, 144, None, 4, "mixed", True, 0),
    "trellis1_gradient": (176, 144, None, 3, "gradient", False, 1),
    "trellis1_mixed": (176, 144, None, 3, "mixed", False, 1),
    "trellis2_cropped_gradient": (322, 242, (317, 237), 3, "gradient", False, 2),
    "trellis1_dquant_texture": (176, 144, None, 5, "synth", True, 1),
}


@pytest.mark.parametrize("case", sorted(OVERLAP_PLANS))
def test_i_overlap_plan_matches_reference(ctx, case):
    """vc1cu_choose_i_overlap against the reference's choose_i_overlap_plan: the mode and flags."""
    w, h, disp, pq, content, dquant, trellis = OVERLAP_PLANS[case]
    kw = dict(display_width=disp[0], display_height=disp[1]) if disp else {}
    p = make_params(w, h, pqindex=pq, **kw)
    frame = synth.generate(w, h, 1, 7).frame(0) if content == "synth" else _overlap_content(content, w, h)
    R = Reference(p)
    aq = 1.0 if (dquant or trellis) else 0.0
    want_mode, want_flags = R.choose_i_overlap(frame, dquant=dquant, aq_strength=aq, trellis=trellis)
    _, mq, der = R.reconstruct_intra(frame, 0, None, dquant=dquant, aq_strength=aq, trellis=trellis)
    cfg = make_trd_cfg(trellis=trellis, adaptive_quality=1, aq_strength=aq) if trellis else None
    ctx.upload_frame(0, *frame)
    mode, flags = ctx.choose_i_overlap(p, 0, mquant=mq if dquant else None, derived=der if dquant else None, cfg=cfg)
    assert mode == want_mode
    assert np.array_equal(flags, want_flags)
