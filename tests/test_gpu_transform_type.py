"""The throughput preset's transform type on the device (vc1cu_fast_transform_types) against the
reference's choices (tests/golden/tt_kat.npz) and the oracle, through the C ABI."""
import os

import numpy as np
import pytest

from libvc1_b200 import synth
from libvc1_b200.abi import MV_MIXED, MV_QPEL, make_params

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TT_CASES = ((98, 66, 4), (130, 98, 12), (322, 242, 6), (16, 16, 1), (354, 290, 3), (98, 66, 10))


def _planes(y):
    h, w = y.shape
    u = np.full((h // 2, w // 2), 128, np.uint8)
    return np.ascontiguousarray(y), u, u.copy()


@pytest.mark.parametrize("i", range(len(TT_CASES)))
def test_fast_transform_types_match_reference_fixture(ctx, i):
    g = np.load(os.path.join(GOLDEN, "tt_kat.npz"))
    w, h, pq = TT_CASES[i]
    p = make_params(w, h, search_range=8, local_search_range=8, pqindex=pq)
    ctx.upload_frame(0, *_planes(g[f"c{i}.cur"]))
    ctx.upload_frame(1, *_planes(g[f"c{i}.pred"]))
    assert np.array_equal(ctx.fast_transform_types(p, 0, 1), g[f"c{i}.types"])


def test_fast_transform_types_1080p_match_oracle(ctx, oracle):
    clip = synth.hd1080(frames=2, seed=47)
    p = make_params(1920, 1080, search_range=32, local_search_range=32, pqindex=5, nonuniform=1)
    cur, ref = clip.frame(1), clip.frame(0)
    ctx.upload_frame(0, *ref)
    ctx.upload_frame(1, *cur)
    ctx.core_passes(p, [(1, 0, MV_QPEL, 0, -1, 90)])
    ctx.core_passes(p, [(1, 0, MV_MIXED, 1, 90, 91)])
    ctx.motion_compensate(p, 0, 91, MV_MIXED, 2)
    pred = ctx.download_frame(2, 1920, 1080)
    got = ctx.fast_transform_types(p, 1, 2)
    assert np.array_equal(got, oracle.fast_transform_types(p, cur, pred))
    assert len(set(got.tolist())) >= 2
