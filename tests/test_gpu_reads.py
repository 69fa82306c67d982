"""Result reads wait for the launch that last wrote their slot only: a slot read while later
launches are still queued returns that writer's result, and a slot written again before the read
returns the newest write (compared with the oracle, bit for bit)."""
import pytest

from libvc1_b200 import synth
from libvc1_b200.abi import MV_HPEL_BILINEAR, MV_QPEL, make_params

pytestmark = pytest.mark.gpu


def test_read_waits_for_its_writer_only(ctx, oracle):
    clip = synth.generate(322, 242, 3, 71)
    p = make_params(322, 242, search_range=24, local_search_range=24)
    for f in range(3):
        ctx.upload_frame(f, *clip.frame(f))
    ctx.core_passes(p, [(1, 0, MV_QPEL, 0, -1, 700)])
    # later work on the stream: more passes into other slots, and a B picture
    ctx.core_passes(p, [(2, 0, MV_QPEL, 0, -1, 701), (2, 1, MV_HPEL_BILINEAR, 0, -1, 702)])
    ctx.core_passes(p, [(1, 2, MV_QPEL, 0, -1, 703)])
    want = {700: (1, 0, MV_QPEL), 701: (2, 0, MV_QPEL), 702: (2, 1, MV_HPEL_BILINEAR), 703: (1, 2, MV_QPEL)}
    for slot in (700, 703, 701, 702):
        t, r, m = want[slot]
        e = oracle.analyze_p_core(p, clip.frame(t), clip.frame(r), m, False)
        assert ctx.read_result(p, slot).equal(e) == [], slot
    # a slot written again before its read holds the newest write
    ctx.core_passes(p, [(2, 1, MV_QPEL, 0, -1, 700)])
    ctx.core_passes(p, [(1, 0, MV_QPEL, 0, -1, 704)])
    e = oracle.analyze_p_core(p, clip.frame(2), clip.frame(1), MV_QPEL, False)
    assert ctx.read_result(p, 700).equal(e) == []
