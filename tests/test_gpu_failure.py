"""Failure detection of the wavefront waits, without a GPU fault.

A core pass's macroblock waits for its left, top-left, top and top-right neighbours' done
flags. Every wait is bounded: once it gives up, the launch aborts and the call that reads the
pass fails with VC1CU_ERR_TIMEOUT, naming the first waiting work item. Here one macroblock's
flag is withheld on purpose (a host-side hook of the launch descriptor, nothing faults) with a
short poll limit, and the context must serve the next call normally.
"""
import re

import pytest

from libvc1_b200 import synth
from libvc1_b200.abi import MV_HPEL, MV_QPEL, make_params
from libvc1_b200.api import Vc1cuError

pytestmark = pytest.mark.gpu

_MSG = re.compile(r"pass (\d+) of its launch, macroblock (\d+), lanes still waiting 0x([0-9a-f]+)")


def _descends(mb, from_mb, mbw):
    """Whether macroblock mb waits, directly or through other waits, on from_mb's flag: a
    macroblock waits for its left, top-left, top and top-right neighbours, so the blocked region
    is the rest of from_mb's row and, on each row below, everything right of a boundary that moves
    one macroblock left per row. The first wait to give up can be any of them (each wait counts
    its own polls)."""
    x, y = mb % mbw, mb // mbw
    fx, fy = from_mb % mbw, from_mb // mbw
    return (y == fy and x > fx) or (y > fy and x >= fx - (y - fy))


def test_withheld_done_flag_times_out_and_context_recovers(ctx, oracle):
    clip = synth.cif_plain(frames=2, seed=14)
    p = make_params(clip.width, clip.height, search_range=16, local_search_range=16)
    ctx.upload_frame(0, *clip.frame(0))
    ctx.upload_frame(1, *clip.frame(1))
    mbw = (clip.width + 15) // 16
    withheld = 5 * mbw + 7
    ctx.debug_set_wait_limit(16)
    try:
        ctx.debug_withhold_publish(0, withheld)
        ctx.core_passes(p, [(1, 0, MV_QPEL, 0, -1, 900)])
        with pytest.raises(Vc1cuError) as e:
            ctx.read_result(p, 900)
        assert e.value.code == 3, str(e.value)
        m = _MSG.search(str(e.value))
        assert m, str(e.value)
        assert int(m.group(1)) == 0
        waiting, mask = int(m.group(2)), int(m.group(3), 16)
        assert mask and _descends(waiting, withheld, mbw), (waiting, hex(mask))
    finally:
        ctx.debug_withhold_publish(-1, -1)
        ctx.debug_set_wait_limit(24)
    # the context serves the next calls normally: the same pass and a seeded one match the oracle
    g = ctx.analyze_p_core(p, 1, 0, MV_QPEL, False)
    e = oracle.analyze_p_core(p, clip.frame(1), clip.frame(0), MV_QPEL, False)
    assert g.equal(e) == []
    gs = ctx.analyze_p_core(p, 1, 0, MV_HPEL, True, seed=g.mvs, seed_distant=g)
    es = oracle.analyze_p_core(p, clip.frame(1), clip.frame(0), MV_HPEL, True, seed=e.mvs, seed_distant=e)
    assert gs.equal(es) == []


def test_withheld_seed_flag_in_one_launch_times_out(ctx, oracle):
    """A seeded pass that takes its seed from a pass of the same launch waits for the seed
    macroblock's flag (lane 0); withholding it makes that wait (or a neighbour wait of the seed
    pass) give up."""
    clip = synth.generate(96, 64, 2, 3, global_px=3.0, n_objects=1, obj_min=16, obj_max=32)
    p = make_params(96, 64, search_range=8, local_search_range=8)
    ctx.upload_frame(0, *clip.frame(0))
    ctx.upload_frame(1, *clip.frame(1))
    mbw = 6
    withheld = 1 * mbw + 2
    ctx.debug_set_wait_limit(16)
    try:
        ctx.debug_withhold_publish(0, withheld)
        ctx.core_passes(p, [(1, 0, MV_QPEL, 0, -1, 920), (1, 0, MV_HPEL, 0, 920, 921)])
        with pytest.raises(Vc1cuError) as e:
            ctx.read_result(p, 921)
        assert e.value.code == 3, str(e.value)
        m = _MSG.search(str(e.value))
        assert m, str(e.value)
        pas, waiting, mask = int(m.group(1)), int(m.group(2)), int(m.group(3), 16)
        # the seeded pass's own macroblock waits for the seed (lane 0); the seed pass's
        # dependents, and the seeded pass's, wait behind it
        assert pas in (0, 1) and mask
        assert waiting == withheld or _descends(waiting, withheld, mbw), (pas, waiting, hex(mask))
    finally:
        ctx.debug_withhold_publish(-1, -1)
        ctx.debug_set_wait_limit(24)
    g = ctx.analyze_p_core(p, 1, 0, MV_QPEL, False)
    assert g.equal(oracle.analyze_p_core(p, clip.frame(1), clip.frame(0), MV_QPEL, False)) == []


def test_debug_hooks_check_their_arguments(ctx):
    with pytest.raises(Vc1cuError) as e:
        ctx.debug_set_wait_limit(3)
    assert e.value.code == 1
    with pytest.raises(Vc1cuError) as e:
        ctx.debug_withhold_publish(0, -5)
    assert e.value.code == 1
