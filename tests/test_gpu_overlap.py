"""Overlap smoothing on the device (vc1cu_overlap_smooth) and the signed store
(vc1cu_store_signed) against the reference's outputs (tests/golden/ovl_kat.npz) and the oracle,
bit for bit, through the C ABI."""
import os

import numpy as np
import pytest

from libvc1_b200.abi import make_params, mbs_of
from libvc1_b200.api import Vc1cuError

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _device(planes):
    import torch

    d = [torch.from_numpy(np.ascontiguousarray(a, np.int32)).cuda() for a in planes]
    torch.cuda.synchronize()  # the library's stream does not wait for torch's
    return d


def _host(ctx, d):
    ctx.synchronize()
    return [t.cpu().numpy() for t in d]


def _smooth(ctx, p, planes, flags=None, all_edges=False):
    d = _device(planes)
    ctx.overlap_smooth(p, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), flags, all_edges)
    return _host(ctx, d)


@pytest.mark.parametrize("i", range(6))
def test_overlap_matches_reference_fixture(ctx, i):
    from ovl_cases import OVL_CASES, mb_flags, signed_planes

    g = np.load(os.path.join(GOLDEN, "ovl_kat.npz"))
    w, h, pq, seed = OVL_CASES[i]
    p = make_params(w, h, pqindex=pq)
    planes, flags = signed_planes(w, h, seed), mb_flags(w, h, seed)
    runs = {"all": _smooth(ctx, p, planes, all_edges=True), "sel": _smooth(ctx, p, planes, flags)}
    if pq >= 9:  # apply_p_overlap's picture condition
        runs["p"] = _smooth(ctx, p, planes, flags)
    for tag, got in runs.items():
        for x, c in zip(got, "yuv"):
            assert np.array_equal(x, g[f"c{i}.{tag}.{c}"]), (tag, c)


def test_overlap_1080p_matches_oracle(ctx, oracle):
    from ovl_cases import mb_flags, signed_planes

    p = make_params(1920, 1080, pqindex=12)
    planes, flags = signed_planes(1920, 1080, 11), mb_flags(1920, 1080, 11)
    for fl, al in ((None, True), (flags, False), (np.zeros_like(flags), False)):
        got = _smooth(ctx, p, planes, fl, al)
        for x, y in zip(got, oracle.overlap_smooth(p, planes, fl, al)):
            assert np.array_equal(x, y)


def test_store_signed_matches_oracle(ctx, oracle):
    """The I path (smooth, then store every sample with the +128 bias) and the P path (smooth with
    the intra map, then write back only the intra macroblocks over an inter reconstruction)."""
    from ovl_cases import mb_flags, signed_planes

    w, h = 322, 242
    p = make_params(w, h, pqindex=10)
    mbw, mbh = mbs_of(p)
    planes, intra = signed_planes(w, h, 12), mb_flags(w, h, 12)
    d = _device(planes)
    ptrs = [t.data_ptr() for t in d]
    ctx.overlap_smooth(p, *ptrs, None, True)
    ctx.store_signed(p, *ptrs, 128, 5)
    sm = oracle.overlap_smooth(p, planes, all_edges=True)
    for x, y in zip(ctx.download_frame(5, mbw * 16, mbh * 16), oracle.store_signed(p, sm, 128)):
        assert np.array_equal(x, y)
    # P: an inter reconstruction of the raster's size, intra macroblocks written over it
    rng = np.random.default_rng(13)
    inter = (rng.integers(0, 256, (h, w), np.uint8), rng.integers(0, 256, (h // 2, w // 2), np.uint8),
             rng.integers(0, 256, (h // 2, w // 2), np.uint8))
    ctx.upload_frame(6, *inter)
    d = _device(planes)
    ptrs = [t.data_ptr() for t in d]
    ctx.overlap_smooth(p, *ptrs, intra, False)
    ctx.store_signed(p, *ptrs, 128, 6, intra)
    sp = oracle.overlap_smooth(p, planes, intra)
    for x, y in zip(ctx.download_frame(6, w, h), oracle.store_signed(p, sp, 128, intra, into=inter)):
        assert np.array_equal(x, y)


def test_overlap_rejects_bad_arguments(ctx):
    p = make_params(64, 48)
    d = _device((np.zeros((48, 64)), np.zeros((24, 32)), np.zeros((24, 32))))
    ptrs = [t.data_ptr() for t in d]
    with pytest.raises(Vc1cuError, match="flags"):
        ctx.overlap_smooth(p, *ptrs, None, False)
    with pytest.raises(Vc1cuError, match="output frame slot"):
        ctx.store_signed(p, *ptrs, 128, -1)
    with pytest.raises(Vc1cuError, match="never uploaded"):
        ctx.store_signed(p, *ptrs, 128, 977, np.ones(12, np.uint8))
