"""The index-checked build (libvc1cu_checked.so, -DVC1CU_INDEX_CHECK): every guarded access of the
analysis kernels (search-window reads, stage key slots, first-visit bitsets, neighbour, candidate
and signature tables, work items, window staging) is tested against its buffer; a violation is
counted and skipped instead of touching memory. The cases that stress the index arithmetic most
run on it: a 16x16 picture, odd and cropped rasters, long-range searches, a B picture, the
learned pass with its fallback and a batch of uneven clips. Each must leave the record empty and
still equal the oracle bit for bit."""
import os

import numpy as np
import pytest

from libvc1_b200 import synth
from libvc1_b200.abi import MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED, MV_QPEL, make_params
from libvc1_b200.api import CHECKED_LIB_PATH, CudaComputeContext, LearnedProposals

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(CHECKED_LIB_PATH), reason="index-checked build missing")]


@pytest.fixture(scope="module")
def cctx():
    c, err = CudaComputeContext.create(0, library=CHECKED_LIB_PATH)
    if c is None:
        pytest.fail(f"index-checked backend unavailable: {err}")
    c.index_faults(reset=True)
    yield c
    c.close()


def _clean(c):
    n, site, index = c.index_faults(reset=True)
    assert n == 0, f"{n} index violations, first at site {site} index {index}"


CHAINS = {
    # (w, h, display, range, local, algorithm, long-range policy)
    "16x16": (16, 16, None, 16, 16, 0, 0),
    "odd_cropped": (322, 242, (321, 241), 32, 32, 0, 0),
    "longrange_compare": (192, 128, None, 128, 16, 0, 0),
    "longrange_legacy_diamond": (208, 120, (203, 117), 96, 16, 1, 2),
}


@pytest.mark.parametrize("case", sorted(CHAINS))
def test_p_chain_clean_and_exact(cctx, oracle, case):
    w, h, disp, rng, local, alg, pol = CHAINS[case]
    clip = synth.generate(w, h, 2, 33, global_px=min(0.4 * rng, 40.0), n_objects=2, obj_min=8, obj_max=24)
    kw = dict(display_width=disp[0], display_height=disp[1]) if disp else {}
    p = make_params(w, h, search_range=rng, local_search_range=local, me_algorithm=alg, long_range_mode=pol, **kw)
    cur, ref = clip.frame(1), clip.frame(0)
    cctx.upload_frame(0, *ref)
    cctx.upload_frame(1, *cur)
    g = cctx.analyze_p_core(p, 1, 0, MV_QPEL, False)
    e = oracle.analyze_p_core(p, cur, ref, MV_QPEL, False)
    assert g.equal(e) == []
    for m in (MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED):
        gm = cctx.analyze_p_core(p, 1, 0, m, m == MV_MIXED, seed=g.mvs, seed_distant=g)
        em = oracle.analyze_p_core(p, cur, ref, m, m == MV_MIXED, seed=e.mvs, seed_distant=e)
        assert gm.equal(em) == [], m
    _clean(cctx)


def test_b_picture_clean_and_exact(cctx, oracle):
    w, h = 98, 66
    clip = synth.generate(w, h, 3, 12, global_px=5.0, n_objects=2, obj_min=8, obj_max=24)
    p = make_params(w, h, display_width=97, display_height=65, search_range=16, local_search_range=16)
    for t in range(3):
        cctx.upload_frame(t, *clip.frame(t))
    a = oracle.analyze_p_core(p, clip.frame(2), clip.frame(0), MV_MIXED, True)
    for mode in (MV_QPEL, MV_HPEL_BILINEAR):
        g = cctx.analyze_b_picture(p, 1, 0, 2, a.mvs, a.use_4mv, 1, 2, mode)
        e = oracle.analyze_b(p, clip.frame(1), clip.frame(0), clip.frame(2), a.mvs, a.use_4mv, 1, 2, mode)
        assert g.equal(e) == [], mode
    _clean(cctx)


def test_learned_pass_clean_and_exact(cctx, oracle):
    w, h, rng = 322, 242, 64
    clip = synth.generate(w, h, 2, 51, global_px=30.0, n_objects=3, obj_min=16, obj_max=40, obj_vel=4.0)
    p = make_params(w, h, display_width=321, display_height=241, search_range=rng, local_search_range=32)
    cctx.upload_frame(0, *clip.frame(1))
    cctx.upload_frame(1, *clip.frame(0))
    net = LearnedProposals(cctx, w, h, rng, capacity=1, max_batch=1, seed=6)
    try:
        net.prepare(0, 1, 0)
        net.propose(0, 1)
        net.analyze(p, [(0, 1, 0, MV_QPEL, 970)], fallback=True)
        got = cctx.read_result(p, 970)
        _, hint, cands, flags = net.read_sample(0)
    finally:
        net.close()
    want, wflags = oracle.analyze_p_learned(p, clip.frame(1), clip.frame(0), MV_QPEL, cands, hint, True)
    assert np.array_equal(flags, wflags)
    assert got.equal(want) == []
    _clean(cctx)


def test_uneven_batch_clean_and_exact(cctx, oracle):
    sizes = [(96, 64, None), (162, 98, (161, 97)), (48, 32, None)]
    clips = [synth.generate(w, h, 2, 70 + k, global_px=6.0, n_objects=1, obj_min=8, obj_max=16)
             for k, (w, h, _) in enumerate(sizes)]
    params = []
    for w, h, disp in sizes:
        kw = dict(display_width=disp[0], display_height=disp[1]) if disp else {}
        params.append(make_params(w, h, search_range=24, local_search_range=24, **kw))
    plist, passes = [], []
    for k, clip in enumerate(clips):
        cctx.upload_frame(100 + 2 * k, *clip.frame(1))
        cctx.upload_frame(101 + 2 * k, *clip.frame(0))
        plist += [params[k], params[k]]
        passes += [(100 + 2 * k, 101 + 2 * k, MV_QPEL, 0, -1, 500 + 2 * k),
                   (100 + 2 * k, 101 + 2 * k, MV_MIXED, 1, 500 + 2 * k, 501 + 2 * k)]
    cctx.core_passes_multi(plist, passes)
    for k, clip in enumerate(clips):
        e = oracle.analyze_p_core(params[k], clip.frame(1), clip.frame(0), MV_QPEL, False)
        assert cctx.read_result(params[k], 500 + 2 * k).equal(e) == [], k
        ef = oracle.analyze_p_core(params[k], clip.frame(1), clip.frame(0), MV_MIXED, True, seed=e.mvs, seed_distant=e)
        assert cctx.read_result(params[k], 501 + 2 * k).equal(ef) == [], k
    _clean(cctx)
