"""The padded-raster motion compensation of the picture coder's reconstruction loop
(motion_compensate_mb_padded / _4mv_padded / bi_mb_padded, src/encoder_motion_compensation.cpp:573-763,
called by encoder_encode.cpp:1183-1195 and :1679-1688) on the device: vc1cu_motion_compensate and
vc1cu_b_predict given the padded raster (mbw*16 x mbh*16) and padded frames predict every whole
macroblock with the samples clamped to the padded reference, as the reference does. Checked
against the reference's own padded functions (oracle/_ref) on cropped rasters, for 1-MV modes,
Mixed-MV with 4-MV macroblocks and every B macroblock mode."""
import numpy as np
import pytest

from libvc1_b200 import synth
from libvc1_b200.abi import MV_HPEL_BILINEAR, MV_MIXED, MV_QPEL, make_params, mbs_of
from oracle.bindings import Reference, ref_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")]

RASTERS = [(322, 242, 61), (208, 120, 62), (98, 66, 63)]


def _padded(p, seed):
    mbw, mbh = mbs_of(p)
    return synth.generate(mbw * 16, mbh * 16, 3, seed, global_px=6.0, n_objects=3, obj_min=12, obj_max=40,
                          obj_vel=5.0, sigma=2.0)


@pytest.mark.parametrize("raster", RASTERS)
@pytest.mark.parametrize("mode", [MV_QPEL, MV_HPEL_BILINEAR, MV_MIXED])
def test_p_padded_prediction_matches_reference(ctx, raster, mode):
    w, h, seed = raster
    p = make_params(w, h, search_range=24, local_search_range=24)
    mbw, mbh = mbs_of(p)
    pp = make_params(mbw * 16, mbh * 16)  # the padded raster
    big = _padded(p, seed)
    cur, ref = (tuple(pl[: (h if i == 0 else h // 2), : (w if i == 0 else w // 2)] for i, pl in enumerate(big.frame(t)))
                for t in (1, 0))
    ctx.upload_frame(0, *[np.ascontiguousarray(a) for a in ref])
    ctx.upload_frame(1, *[np.ascontiguousarray(a) for a in cur])
    ctx.core_passes(p, [(1, 0, MV_QPEL, 0, -1, 900)])
    ctx.core_passes(p, [(1, 0, mode, mode == MV_MIXED, 900, 901)])
    a = ctx.read_result(p, 901)
    if mode == MV_MIXED:
        assert a.use_4mv.sum() > 0
    ctx.upload_frame(10, *big.frame(0))  # the padded reconstruction of the reference
    ctx.motion_compensate(pp, 10, 901, mode, 11)
    got = ctx.download_frame(11, mbw * 16, mbh * 16)
    want = Reference(p).motion_compensate_padded(big.frame(0), a, mode)
    for g, e, c in zip(got, want, "yuv"):
        assert np.array_equal(g, e), c


@pytest.mark.parametrize("raster", RASTERS)
@pytest.mark.parametrize("mode", [MV_QPEL, MV_HPEL_BILINEAR])
def test_b_padded_prediction_matches_reference(ctx, raster, mode):
    w, h, seed = raster
    p = make_params(w, h, search_range=24, local_search_range=24)
    mbw, mbh = mbs_of(p)
    pp = make_params(mbw * 16, mbh * 16)
    big = _padded(p, seed + 10)
    crop = [tuple(np.ascontiguousarray(pl[: (h if i == 0 else h // 2), : (w if i == 0 else w // 2)])
                  for i, pl in enumerate(big.frame(t))) for t in range(3)]
    for t in range(3):
        ctx.upload_frame(t, *crop[t])
    ctx.core_passes(p, [(2, 0, MV_QPEL, 0, -1, 910)])
    ctx.core_passes(p, [(2, 0, MV_MIXED, 1, 910, 911)])
    ctx.core_passes(p, [(1, 0, mode, 0, -1, 912), (1, 2, mode, 0, -1, 913)])
    ctx.b_decide(p, [(1, 0, 2, 912, 913, 911, 1, 2, mode, 70)])
    b = ctx.read_bresult(p, 70)
    assert len(set(b.modes.tolist()) - {4}) >= 2  # several inter modes
    for t in range(3):
        ctx.upload_frame(20 + t, *big.frame(t))
    ctx.b_predict(pp, 70, 21, 20, 22, 23)
    got = ctx.download_frame(23, mbw * 16, mbh * 16)
    want = Reference(p).b_predict_padded(big.frame(0), big.frame(2), b, mode)
    inter = (b.modes != 4).reshape(mbh, mbw)
    for g, e, s in zip(got, want, (16, 8, 8)):
        m = np.kron(inter, np.ones((s, s), bool))
        assert np.array_equal(g[m], e[m])
