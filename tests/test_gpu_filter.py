"""In-loop deblocking on the device (vc1cu_loop_filter_i / _p) against the reference's
filtered pictures (tests/golden/lf_kat.npz) and the oracle, bit-exact, through the C ABI."""
import os

import numpy as np
import pytest

from libvc1_b200.abi import make_params
from libvc1_b200.api import Vc1cuError

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
LF_CASES = ((98, 66, 8), (130, 98, 20), (66, 50, 3), (194, 146, 31))


def _frames(g, prefix):
    return tuple(np.ascontiguousarray(g[f"{prefix}.{c}"]) for c in "yuv")


@pytest.mark.parametrize("i", range(len(LF_CASES)))
def test_loop_filter_matches_reference_fixture(ctx, i):
    g = np.load(os.path.join(GOLDEN, "lf_kat.npz"))
    w, h, pq = LF_CASES[i]
    p = make_params(w, h, pqindex=pq)
    fr = _frames(g, f"c{i}.in")
    ctx.upload_frame(0, *fr)
    ctx.loop_filter(p, 0)
    for got, c in zip(ctx.download_frame(0, w, h), "yuv"):
        assert np.array_equal(got, g[f"c{i}.i.{c}"]), ("i", c)
    ctx.upload_frame(0, *fr)
    ctx.loop_filter(p, 0, *[g[f"c{i}.{k}"] for k in ("bmv", "cbp", "tt", "intra")])
    for got, c in zip(ctx.download_frame(0, w, h), "yuv"):
        assert np.array_equal(got, g[f"c{i}.p.{c}"]), ("p", c)


@pytest.mark.parametrize("case", [(1920, 1080, 11, 9, True), (322, 242, 12, 25, False), (16, 16, 13, 5, True),
                                  (354, 290, 14, 14, True)])
def test_loop_filter_matches_oracle(ctx, oracle, case):
    from lf_cases import blocky_frame, metadata

    w, h, seed, pq, dense = case
    p = make_params(w, h, pqindex=pq)
    fr = blocky_frame(w, h, seed)
    meta = metadata(w, h, seed, dense)
    ctx.upload_frame(0, *fr)
    ctx.loop_filter(p, 0, *meta)
    for got, want in zip(ctx.download_frame(0, w, h), oracle.loop_filter(p, fr, *meta)):
        assert np.array_equal(got, want)
    ctx.upload_frame(0, *fr)
    ctx.loop_filter(p, 0)
    for got, want in zip(ctx.download_frame(0, w, h), oracle.loop_filter(p, fr)):
        assert np.array_equal(got, want)


def test_loop_filter_rejects_bad_codes(ctx):
    from lf_cases import blocky_frame, metadata

    p = make_params(64, 48, pqindex=8)
    ctx.upload_frame(0, *blocky_frame(64, 48, 15))
    bmv, cbp, tt, intra = metadata(64, 48, 15)
    tt[0, 0] = 5
    with pytest.raises(Vc1cuError, match="transform kinds"):
        ctx.loop_filter(p, 0, bmv, cbp, tt, intra)


def test_loop_filter_of_padded_reconstruction(ctx, oracle):
    """The padded raster the reference's reconstruction holds (whole macroblocks): both filters
    cover the frame's own extent, and an I picture stored by vc1cu_store_signed filters in place."""
    import torch

    from lf_cases import blocky_frame, metadata
    from ovl_cases import signed_planes

    w, h = 322, 242
    p = make_params(w, h, pqindex=14)
    pw, ph = 336, 256
    pp = make_params(pw, ph, pqindex=14)  # the oracle filters whatever frame it is given
    fr = blocky_frame(pw, ph, 21)
    ctx.upload_frame(0, *fr)
    ctx.loop_filter(p, 0)
    for got, want in zip(ctx.download_frame(0, pw, ph), oracle.loop_filter(pp, fr)):
        assert np.array_equal(got, want)
    meta = metadata(w, h, 22, True)
    ctx.upload_frame(0, *fr)
    ctx.loop_filter(p, 0, *meta)
    for got, want in zip(ctx.download_frame(0, pw, ph), oracle.loop_filter(pp, fr, *meta)):
        assert np.array_equal(got, want)
    planes = signed_planes(w, h, 23)
    d = [torch.from_numpy(a).cuda() for a in planes]
    torch.cuda.synchronize()
    ctx.overlap_smooth(p, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), None, True)
    ctx.store_signed(p, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), 128, 12)
    ctx.loop_filter(p, 12)
    want = oracle.loop_filter(pp, oracle.store_signed(p, oracle.overlap_smooth(p, planes, all_edges=True), 128))
    for got, x in zip(ctx.download_frame(12, pw, ph), want):
        assert np.array_equal(got, x)
    ctx.upload_frame(0, *blocky_frame(330, 250, 24))
    with pytest.raises(Vc1cuError, match="padded raster"):
        ctx.loop_filter(p, 0)


@pytest.mark.parametrize("case", [(98, 66, 21, 8, False, False), (322, 242, 22, 12, True, False),
                                  (130, 98, 23, 25, True, True), (354, 290, 24, 4, False, True)])
def test_main_profile_p_filter_matches_reference(ctx, case):
    """vc1cu_loop_filter_p_main against the reference's own apply_p_loop_filter under WMV9 Main
    syntax (oracle/_ref): block 0 of the first macroblock intra or not (exception 1), every
    transform kind (exceptions 2 and 3), and block vectors long enough to hit the chroma range
    limit of exception 4."""
    from lf_cases import blocky_frame, metadata
    from oracle.bindings import Reference, ref_available

    if not ref_available():
        pytest.skip("oracle/_ref not built")
    w, h, seed, pq, first_intra, long_mvs = case
    p = make_params(w, h, pqindex=pq)
    fr = blocky_frame(w, h, seed)
    bmv, cbp, tt, intra = metadata(w, h, seed, True)
    intra[0] = (int(intra[0]) | 1) if first_intra else (int(intra[0]) & 0xFE)
    if long_mvs:
        # one vector per 2x2 macroblocks, many pointing far outside the picture: neighbours share
        # a luma vector while their range-limited chroma vectors differ
        mbw, mbh = (w + 15) // 16, (h + 15) // 16
        rng = np.random.default_rng(seed)
        g = rng.integers(-4 * (w + 40), 4 * (w + 40), ((mbh + 1) // 2, (mbw + 1) // 2, 2))
        bmv = np.repeat(np.repeat(g, 2, 0), 2, 1)[:mbh, :mbw].reshape(-1, 1, 2).repeat(4, 1).astype(np.int32)
    ctx.upload_frame(0, *fr)
    ctx.loop_filter(p, 0, bmv, cbp, tt, intra, main_profile=True)
    want = Reference(p).loop_filter(fr, bmv, cbp, tt, intra, main_profile=True)
    for got, exp, c in zip(ctx.download_frame(0, w, h), want, "yuv"):
        assert np.array_equal(got, exp), c
    # the Main rules change the picture against the Advanced filter on these inputs
    adv = Reference(p).loop_filter(fr, bmv, cbp, tt, intra)
    assert any(not np.array_equal(a, b) for a, b in zip(adv, want))
