"""Reconstruction on the device (vc1cu_reconstruct: dequantisation, VC-1 inverse transforms, add
to the prediction) against the reference's reconstructions (tests/golden/recon_kat.npz) and the
oracle, bit-exact, through the C ABI."""
import os

import numpy as np
import pytest

from libvc1_b200 import synth
from libvc1_b200.abi import MV_MIXED, MV_QPEL, make_params
from libvc1_b200.api import Vc1cuError

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RECON_QP = ((3, 0, 1), (8, 1, 1), (17, 1, 0), (31, 0, 0))


def _frames(g, prefix):
    return tuple(np.ascontiguousarray(g[f"{prefix}.{c}"]) for c in "yuv")


def _device(levels):
    import torch

    return torch.from_numpy(np.ascontiguousarray(levels, np.int16)).cuda()


@pytest.mark.parametrize("qp", RECON_QP)
def test_reconstruction_matches_reference_fixture(ctx, qp):
    import torch

    pq, nu, hq = qp
    key = f"pq{pq}_nu{nu}_hq{hq}"
    g = np.load(os.path.join(GOLDEN, "recon_kat.npz"))
    x = np.load(os.path.join(GOLDEN, "xform_kat.npz"))
    p = make_params(64, 48, pqindex=pq, nonuniform=nu, halfqp=hq, search_range=8, local_search_range=8)
    ctx.upload_frame(0, *_frames(x, "cur"))
    ctx.upload_frame(1, *_frames(x, f"{key}.pred"))
    coded = torch.empty((4, 12, 6, 64), dtype=torch.int16, device="cuda")
    ctx.forward_quant_device(p, 0, 1, 15, 0, coded.data_ptr())
    for name, lv in (("coded", coded), ("random", _device(g[f"{key}.random_levels"]))):
        ctx.reconstruct(p, 1, lv.data_ptr(), 15, g[f"{key}.types"], 2)
        for got, c in zip(ctx.download_frame(2, 64, 48), "yuv"):
            assert np.array_equal(got, g[f"{key}.{name}.{c}"]), (name, c)


@pytest.mark.parametrize("tm", [1, 2, 4, 8, 15])
def test_reconstruction_matches_oracle(ctx, oracle, tm):
    """A Mixed-MV prediction of an odd, cropped raster; levels of the selected types; a seeded
    type per block."""
    import torch

    clip = synth.generate(322, 242, 2, 60 + tm)
    p = make_params(322, 242, display_width=321, display_height=241, search_range=16, local_search_range=16,
                    pqindex=5, nonuniform=tm & 1, halfqp=1)
    cur, ref = clip.frame(1), clip.frame(0)
    ctx.upload_frame(0, *ref)
    ctx.upload_frame(1, *cur)
    ctx.core_passes(p, [(1, 0, MV_QPEL, 0, -1, 80)])
    ctx.core_passes(p, [(1, 0, MV_MIXED, 1, 80, 81)])
    ctx.motion_compensate(p, 0, 81, MV_MIXED, 2)
    pred = ctx.download_frame(2, 322, 242)
    nt = bin(tm).count("1")
    mbs = 21 * 16
    lv = torch.empty((nt, mbs, 6, 64), dtype=torch.int16, device="cuda")
    ctx.forward_quant_device(p, 1, 2, tm, 0, lv.data_ptr())
    rng = np.random.default_rng(tm)
    types = rng.choice([t for t in range(1, 5) if tm & (1 << (t - 1))], (mbs, 6)).astype(np.uint8)
    ctx.reconstruct(p, 2, lv.data_ptr(), tm, types, 3)
    want = oracle.reconstruct(p, pred, lv.cpu().numpy(), tm, types)
    for got, w in zip(ctx.download_frame(3, 322, 242), want):
        assert np.array_equal(got, w)


def test_reconstruction_rejects_a_type_outside_the_mask(ctx):
    import torch

    clip = synth.generate(64, 48, 2, 70)
    p = make_params(64, 48)
    ctx.upload_frame(1, *clip.frame(0))
    lv = torch.zeros((1, 12, 6, 64), dtype=torch.int16, device="cuda")
    types = np.full((12, 6), 2, np.uint8)
    with pytest.raises(Vc1cuError, match="type_mask"):
        ctx.reconstruct(p, 1, lv.data_ptr(), 1, types, 2)
    ctx.reconstruct(p, 1, lv.data_ptr(), 1, np.ones((12, 6), np.uint8), 2)
    for got, want in zip(ctx.download_frame(2, 64, 48), clip.frame(0)):
        assert np.array_equal(got, want)  # zero levels reproduce the prediction


DQUANT_RASTERS = [(176, 144, 7, 0, 1), (98, 66, 6, 1, 0), (130, 98, 14, 0, 0)]


@pytest.mark.parametrize("raster", DQUANT_RASTERS)
def test_reconstruction_under_dquant_matches_reference(ctx, raster):
    """vc1cu_reconstruct_dquant against the reference's inverse_partition at each MB's MQUANT
    (derived flags drop the HALFQP half step), every transform type, random sparse levels."""
    import torch

    from oracle.bindings import Reference, ref_available

    if not ref_available():
        pytest.skip("oracle/_ref not built")
    w, h, pq, nu, hq = raster
    p = make_params(w, h, pqindex=pq, nonuniform=nu, halfqp=hq)
    mbw, mbh = (w + 15) // 16, (h + 15) // 16
    mbs = mbw * mbh
    rng = np.random.default_rng(w + pq)
    pred = synth.generate(w, h, 1, pq).frame(0)
    levels = (rng.integers(-24, 25, (4, mbs, 6, 64)) * (rng.random((4, mbs, 6, 64)) < 0.15)).astype(np.int16)
    levels[:, :, :, 0] = rng.integers(-60, 61, (4, mbs, 6))
    dc_only = rng.random((4, mbs, 6)) < 0.2  # the DC-only shortcut
    levels[:, :, :, 1:][dc_only] = 0
    types = rng.integers(1, 5, (mbs, 6)).astype(np.uint8)
    mq = rng.integers(1, 32, mbs).astype(np.uint8)
    mq[::5] = pq  # PQINDEX, with and without the derived flag
    der = (rng.random(mbs) < 0.5).astype(np.uint8)
    ctx.upload_frame(1, *pred)
    lv = _device(levels)
    ctx.reconstruct(p, 1, lv.data_ptr(), 15, types, 2, mquant=mq, derived=der)
    got = ctx.download_frame(2, w, h)
    want = Reference(p).reconstruct(pred, levels, 15, types, mq, der)
    for g, e, c in zip(got, want, "yuv"):
        assert np.array_equal(g, e), (c, np.argwhere(g != e)[:4])
    plain = Reference(p).reconstruct(pred, levels, 15, types)
    assert any(not np.array_equal(a, b) for a, b in zip(want, plain))


def test_dquant_reconstruction_rejects_mquant_outside_1_to_31(ctx):
    p = make_params(64, 48, pqindex=8, search_range=8, local_search_range=8)
    ctx.upload_frame(1, *synth.generate(64, 48, 1, 3).frame(0))
    lv = _device(np.zeros((1, 12, 6, 64), np.int16))
    mq = np.full(12, 8, np.uint8)
    mq[5] = 0
    with pytest.raises(Vc1cuError):
        ctx.reconstruct(p, 1, lv.data_ptr(), 1, np.ones((12, 6), np.uint8), 2, mquant=mq)
    mq[5] = 32
    with pytest.raises(Vc1cuError):
        ctx.reconstruct(p, 1, lv.data_ptr(), 1, np.ones((12, 6), np.uint8), 2, mquant=mq)
    mq[5] = 31
    ctx.reconstruct(p, 1, lv.data_ptr(), 1, np.ones((12, 6), np.uint8), 2, mquant=mq)
    ctx.synchronize()
