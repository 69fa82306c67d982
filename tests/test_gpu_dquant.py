"""The DQUANT MQUANT search on the device (vc1cu_choose_dquant) against the reference's own
Vc1Encoder::choose_dquant_transform_mb (oracle/_ref, scalar path), bit for bit: each macroblock's
MQUANT, its transform decision and its levels. The base MQUANT the reference forms from its
rate-control hooks is handed to the device as the caller would. The cases reach the finer
absolute MQUANT (adjacency, bright-on-dark, predictable texture), the coarser candidates with
their 0.05% acceptance, base MQUANTs below PQINDEX (per-MB DQUANTFRM), HALFQP's repeated
candidates, DQUANT off, the perceptual scale off and trellis 0 / 2."""
import numpy as np
import pytest

from libvc1_b200.abi import make_params, make_trd_cfg, tdecisions_differ
from oracle.bindings import Reference, ref_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")]

CASES = {
    # (content, pq, halfqp, trd overrides, search switches)
    "adjacency": ("adjacency", 14, 0, {}, {}),
    "bright_on_dark": ("bright_on_dark", 12, 0, {}, {}),
    "coarser": ("coarser", 4, 0, {}, {}),
    "coarser_halfqp": ("coarser", 5, 1, {}, {}),
    "boosted_base": ("dark_detail", 6, 0, {}, {}),
    "boosted_base_trellis2": ("dark_detail", 10, 0, dict(trellis=2), {}),
    "predictable": ("natural", 14, 0, {}, dict(predictable=True)),
    "dquant_off": ("natural", 10, 0, {}, dict(dquant=False)),
    "aq_off_scalar": ("dark_detail", 13, 0, dict(adaptive_quality=0, trellis=0), {}),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_dquant_search_matches_reference(ctx, case):
    from dq_cases import frames

    kind, pq, hq, over, sw = CASES[case]
    w, h = 176, 144
    p = make_params(w, h, pqindex=pq, halfqp=hq)
    src, pred = frames(kind, w, h, pq)
    cfg = make_trd_cfg(**over)
    rb, want, wmq, wlv = Reference(p).choose_dquant(cfg, src, pred, **sw)
    ctx.upload_frame(0, *src)
    ctx.upload_frame(1, *pred)
    got, gmq, glv = ctx.choose_dquant(p, cfg, 0, 1, rb, dquant=sw.get("dquant", True),
                                      predictable_texture=sw.get("predictable", False))
    assert np.array_equal(gmq, wmq), np.nonzero(gmq != wmq)[0][:8]
    assert tdecisions_differ(got, want) == []
    assert np.array_equal(glv, wlv)
    if case in ("adjacency", "bright_on_dark", "predictable"):
        assert (wmq < rb).any()
    if case.startswith("coarser") or case == "boosted_base":
        assert (wmq > rb).any()
    if case.startswith("boosted"):
        assert (rb != pq).any()
