"""Long-range pans at the extended MV ranges (MVRANGE 2 and 3, search ranges 512 and 1024;
motion_search_bounds_px, encoder_motion.cpp:1236-1291): camera pans of up to 200 px/frame
horizontally and 60 vertically with four independent objects, local search range 32, so most
vectors come from the long-range searches (propagated distant candidates and the content-signature
index, encoder_motion.cpp:1578-1779). The seed pass and the final Mixed-MV pass against the
oracle, bit for bit, under the three long-range policies; and the learned form at range 1024,
two pictures in one call, with the plain search as its fallback."""
import os

import numpy as np
import pytest

from libvc1_b200 import synth
from libvc1_b200.abi import MV_MIXED, MV_QPEL, make_params

pytestmark = pytest.mark.gpu

CASES = {
    # (w, h, search range, long-range policy)
    "640x360_r512_compare": (640, 360, 512, 0),
    "640x360_r1024_legacy": (640, 360, 1024, 2),
    "1080p_r1024_compare": (1920, 1080, 1024, 0),
    "1080p_r512_local_good_skip": (1920, 1080, 512, 1),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_long_range_pans_match_oracle(ctx, oracle, case):
    w, h, rng, policy = CASES[case]
    clip = synth.generate(w, h, 2, 77, global_px=200.0, global_py=60.0, n_objects=4, obj_vel=8.0)
    p = make_params(w, h, search_range=rng, local_search_range=32, long_range_mode=policy)
    cur, ref = clip.frame(1), clip.frame(0)
    ctx.upload_frame(0, *ref)
    ctx.upload_frame(1, *cur)
    g = ctx.analyze_p_core(p, 1, 0, MV_QPEL, False)
    e = oracle.analyze_p_core(p, cur, ref, MV_QPEL, False)
    assert g.equal(e) == []
    # most vectors lie beyond the local range: the long-range searches found them
    assert (np.abs(e.mvs) > 4 * 33).any(axis=1).mean() > 0.5
    gf = ctx.analyze_p_core(p, 1, 0, MV_MIXED, True, seed=g.mvs, seed_distant=g)
    ef = oracle.analyze_p_core(p, cur, ref, MV_MIXED, True, seed=e.mvs, seed_distant=e)
    assert gf.equal(ef) == []


def test_learned_long_pans_batched_match_oracle(ctx, oracle):
    """The long-range learned form: two 1080p long-pan pairs at search range 1024 (MVRANGE 3) in
    one vc1cu_lp_analyze call, with the plain search (long-range searches included) as fallback;
    each pass bit for bit against the oracle's learned pass on the device's candidates and hint."""
    from libvc1_b200.api import LearnedProposals
    from libvc1_b200 import learned as lw

    w, h, rng = 1920, 1080, 1024
    clips = [synth.generate(w, h, 2, 90 + k, global_px=200.0, global_py=60.0, n_objects=4, obj_vel=8.0)
             for k in range(2)]
    p = make_params(w, h, search_range=rng, local_search_range=32)
    for k, clip in enumerate(clips):
        ctx.upload_frame(10 + 2 * k, *clip.frame(1))
        ctx.upload_frame(11 + 2 * k, *clip.frame(0))
    net = LearnedProposals(ctx, w, h, rng, capacity=2, max_batch=2, seed=3)
    try:
        if os.path.exists(lw.WEIGHTS):
            net.set_params(np.load(lw.WEIGHTS))
        for k in range(2):
            net.prepare(10 + 2 * k, 11 + 2 * k, k)
        net.propose(0, 2)
        net.analyze(p, [(10 + 2 * k, 11 + 2 * k, k, MV_QPEL, 980 + k) for k in range(2)], fallback=True)
        got = [ctx.read_result(p, 980 + k) for k in range(2)]
        samples = [net.read_sample(k) for k in range(2)]
    finally:
        net.close()
    for k, clip in enumerate(clips):
        _, hint, cands, flags = samples[k]
        want, wflags = oracle.analyze_p_learned(p, clip.frame(1), clip.frame(0), MV_QPEL, cands, hint, True)
        assert np.array_equal(flags, wflags)
        assert got[k].equal(want) == []
        # the pans reach beyond the local range: the hint and the vectors carry them
        assert abs(int(hint[0])) > 32 or abs(int(hint[1])) > 32
