"""Seeded random configurations of the whole analysis path on the device against the oracle:
raster sizes and display crops, search and local ranges (long range included), UMH and diamond,
the three me_quality laws, sub-pel settings, quantiser settings and rounding control. Every
configuration runs the P chain (quarter-pel seed pass, the three seeded modes, the final Mixed-MV
pass with P-intra), the prediction and transform, one B picture in quarter-pel and bilinear
mode, and the fade estimate; everything is compared bit for bit."""
import numpy as np
import pytest

from libvc1_b200 import synth
from libvc1_b200.abi import MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED, MV_QPEL, make_params

pytestmark = pytest.mark.gpu


def random_config(seed):
    rng = np.random.default_rng(1000 + seed)
    w = int(rng.integers(1, 26)) * 16 - int(rng.choice([0, 0, 2, 6, 10]))
    h = int(rng.integers(1, 19)) * 16 - int(rng.choice([0, 0, 2, 4, 12]))
    w, h = max(w, 16), max(h, 16)
    search = int(rng.choice([0, 4, 8, 16, 24, 32, 48, 96]))
    local = int(rng.choice([search, search, max(0, search // 3), 8])) if search else 0
    kw = dict(search_range=search, local_search_range=min(local, search),
              display_width=w - int(rng.integers(0, 2)) if w > 16 else 0,
              display_height=h - int(rng.integers(0, 2)) if h > 16 else 0,
              me_algorithm=int(rng.integers(0, 2)), me_quality=int(rng.integers(0, 3)),
              fast_subpel=int(rng.integers(0, 2)), subpel_range=int(rng.choice([1, 2, 1024])),
              long_range_mode=int(rng.integers(0, 3)), pqindex=int(rng.integers(1, 32)),
              nonuniform=int(rng.integers(0, 2)), rnd=int(rng.integers(0, 2)))
    kw["halfqp"] = int(rng.integers(0, 2)) if kw["pqindex"] <= 8 else 0
    motion = float(rng.choice([1.5, 6.75, 20.0]))
    return w, h, kw, motion


@pytest.mark.parametrize("seed", range(12))
def test_random_configuration_matches_oracle(ctx, oracle, seed):
    w, h, kw, motion = random_config(seed)
    p = make_params(w, h, **kw)
    clip = synth.generate(w, h, 3, 500 + seed, global_px=motion, n_objects=2, obj_min=8, obj_max=32)
    past, cur, fut = clip.frame(0), clip.frame(1), clip.frame(2)
    for fid, fr in ((0, past), (1, cur), (2, fut)):
        ctx.upload_frame(fid, *fr)
    # P chain of the future picture against the past one (it is the B picture's anchor)
    ctx.core_passes(p, [(2, 0, MV_QPEL, 0, -1, 200)])
    ctx.core_passes(p, [(2, 0, m, 0, 200, 201 + m) for m in (MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED)])
    ctx.core_passes(p, [(2, 0, MV_MIXED, 1, 201 + MV_MIXED, 210)])
    e = oracle.analyze_p_core(p, fut, past, MV_QPEL, False)
    assert ctx.read_result(p, 200).equal(e) == [], (seed, "qpel", kw)
    em = None
    for m in (MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED):
        em = oracle.analyze_p_core(p, fut, past, m, False, seed=e.mvs, seed_distant=e)
        assert ctx.read_result(p, 201 + m).equal(em) == [], (seed, m, kw)
    ef = oracle.analyze_p_core(p, fut, past, MV_MIXED, True, seed=em.mvs, seed_distant=em)
    assert ctx.read_result(p, 210).equal(ef) == [], (seed, "final", kw)
    # prediction + transform of the final pass
    ctx.motion_compensate(p, 0, 210, MV_MIXED, 3)
    pred = ctx.download_frame(3, w, h)
    want = oracle.motion_compensate(p, past, ef, MV_MIXED)
    assert all(np.array_equal(a, b) for a, b in zip(pred, want)), seed
    co, lv = ctx.forward_quant(p, 2, 3, 15)
    eco, elv = oracle.forward_quant(p, fut, want, 15)
    assert np.array_equal(co.view(np.uint64), eco.view(np.uint64)) and np.array_equal(lv, elv), seed
    # the fade estimate along the final field
    assert ctx.estimate_intensity_batch(p, [(2, 0, 210)]) == [oracle.estimate_intensity_comp(p, fut, past, ef.mvs)]
    # a B picture between them in both modes, anchored on the final pass
    for mode in (MV_QPEL, MV_HPEL_BILINEAR):
        g = ctx.analyze_b_picture(p, 1, 0, 2, ef.mvs, ef.use_4mv, 1, 2, mode)
        eb = oracle.analyze_b(p, cur, past, fut, ef.mvs, ef.use_4mv, 1, 2, mode)
        assert g.equal(eb) == [], (seed, "B", mode, kw)


@pytest.mark.parametrize("seed", range(12))
def test_random_configuration_reconstruction_matches_oracle(ctx, oracle, seed):
    """The same random configurations through the rest of the path: a B picture decided from
    passes in result slots and its prediction, the reconstruction of the P picture's levels with
    a random transform type per block, the P loop filter with random block metadata, overlap
    smoothing of a signed picture and the compensated reference of a random fade code."""
    import torch

    from lf_cases import metadata
    from ovl_cases import mb_flags, signed_planes

    w, h, kw, motion = random_config(seed)
    p = make_params(w, h, **kw)
    mbw, mbh = (w + 15) // 16, (h + 15) // 16
    clip = synth.generate(w, h, 3, 700 + seed, global_px=motion, n_objects=2, obj_min=8, obj_max=32)
    past, cur, fut = clip.frame(0), clip.frame(1), clip.frame(2)
    for fid, fr in ((0, past), (1, cur), (2, fut)):
        ctx.upload_frame(fid, *fr)
    ctx.core_passes(p, [(2, 0, MV_QPEL, 0, -1, 230)])
    ctx.core_passes(p, [(2, 0, MV_MIXED, 1, 230, 231)])
    q = oracle.analyze_p_core(p, fut, past, MV_QPEL, False)
    ef = oracle.analyze_p_core(p, fut, past, MV_MIXED, True, seed=q.mvs, seed_distant=q)
    assert ctx.read_result(p, 231).equal(ef) == [], (seed, kw)
    # B picture from user slots: forward / backward quarter-pel passes, the decision, the prediction
    ctx.core_passes(p, [(1, 0, MV_QPEL, 0, -1, 232), (1, 2, MV_QPEL, 0, -1, 233)])
    ctx.b_decide(p, [(1, 0, 2, 232, 233, 231, 1, 2, MV_QPEL, 7, 0)])
    eb = oracle.analyze_b(p, cur, past, fut, ef.mvs, ef.use_4mv, 1, 2, MV_QPEL)
    assert ctx.read_bresult(p, 7).equal(eb) == [], (seed, kw)
    ctx.b_predict(p, 7, 1, 0, 2, 8)
    for x, y in zip(ctx.download_frame(8, w, h), oracle.b_predict(p, cur, past, fut, eb, MV_QPEL)):
        assert np.array_equal(x, y), seed
    # reconstruction of the P picture from all four types' levels, a random type per block
    ctx.motion_compensate(p, 0, 231, MV_MIXED, 3)
    pred = ctx.download_frame(3, w, h)
    lv = torch.empty((4, mbw * mbh, 6, 64), dtype=torch.int16, device="cuda")
    ctx.forward_quant_device(p, 2, 3, 15, 0, lv.data_ptr())
    types = np.random.default_rng(seed).integers(1, 5, (mbw * mbh, 6)).astype(np.uint8)
    ctx.reconstruct(p, 3, lv.data_ptr(), 15, types, 4)
    ctx.synchronize()
    rec = oracle.reconstruct(p, pred, lv.cpu().numpy(), 15, types)
    assert all(np.array_equal(x, y) for x, y in zip(ctx.download_frame(4, w, h), rec)), seed
    # the P loop filter of the reconstruction
    meta = metadata(w, h, seed, seed % 2 == 0)
    ctx.loop_filter(p, 4, *meta)
    assert all(np.array_equal(x, y) for x, y in zip(ctx.download_frame(4, w, h), oracle.loop_filter(p, rec, *meta))), seed
    # overlap smoothing of a signed picture of the padded raster (select flags)
    planes, flags = signed_planes(w, h, seed), mb_flags(w, h, seed)
    d = [torch.from_numpy(a).cuda() for a in planes]
    torch.cuda.synchronize()
    ctx.overlap_smooth(p, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), flags, False)
    ctx.synchronize()
    for x, y in zip(d, oracle.overlap_smooth(p, planes, flags)):
        assert np.array_equal(x.cpu().numpy(), y), seed
    # the compensated reference of a random fade code
    rng = np.random.default_rng(900 + seed)
    ic = (1, int(rng.integers(0, 64)), int(rng.integers(0, 64)))
    ctx.intensity_compensate(0, ic, 9)
    for x, y in zip(ctx.download_frame(9, w, h), oracle.intensity_compensate(past, ic)):
        assert np.array_equal(x, y), (seed, ic)


@pytest.mark.parametrize("seed", range(12))
def test_paired_passes_match_oracle(ctx, oracle, seed):
    """A B picture's four unseeded passes in one call, as an encoder batches them: the two modes
    run as two launches sharing each picture pair's global search; every pass equals the
    oracle's."""
    w, h, kw, motion = random_config(seed)
    p = make_params(w, h, **kw)
    clip = synth.generate(w, h, 3, 800 + seed, global_px=motion, n_objects=2, obj_min=8, obj_max=32)
    frames = [clip.frame(f) for f in range(3)]
    for f in range(3):
        ctx.upload_frame(f, *frames[f])
    passes = [(1, r, m, 0, -1, 260 + 2 * j + (r == 2), 0)
              for j, m in enumerate((MV_QPEL, MV_HPEL_BILINEAR)) for r in (0, 2)]
    ctx.core_passes(p, passes)
    for t, r, m, _a, _s, slot, _q in passes:
        e = oracle.analyze_p_core(p, frames[t], frames[r], m, False)
        assert ctx.read_result(p, slot).equal(e) == [], (seed, m, r, kw)
