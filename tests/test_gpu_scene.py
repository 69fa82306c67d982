"""The scene-change score on the device (vc1cu_scene_change_score) against the reference's
scores (tests/golden/scene_kat.npz) and the oracle, bit-exact (doubles by bit pattern)."""
import os

import numpy as np
import pytest

from libvc1_b200 import synth
from libvc1_b200.abi import make_params
from libvc1_b200.api import Vc1cuError

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _bits(x):
    return np.float64(x).view(np.uint64)


@pytest.mark.parametrize("name", ["motion", "cut", "cut_low_threshold", "fade", "fade_no_compensation", "zoom_rescue",
                                  "zoom_rescue_fade", "range0"])
def test_scene_score_matches_reference_fixture(ctx, name):
    from scene_cases import scene_pictures

    g = np.load(os.path.join(GOLDEN, "scene_kat.npz"))
    cur, ref, fade, thr, kw = scene_pictures()[name]
    h, w = cur[0].shape
    p = make_params(w, h, **kw)
    ctx.upload_frame(0, *ref)
    ctx.upload_frame(1, *cur)
    assert _bits(ctx.scene_change_score(p, 1, 0, bool(fade), thr)) == g[f"{name}.score"].view(np.uint64)


@pytest.mark.parametrize("case", [(1920, 1080, 31, 1.0, 0.0, 1, 28.0), (322, 242, 32, 0.75, 25.0, 1, 6.0),
                                  (16, 16, 33, 1.0, 0.0, 1, 0.0)])
def test_scene_score_matches_oracle(ctx, oracle, case):
    w, h, seed, a, b, fade, thr = case
    clip = synth.generate(w, h, 2, seed, global_px=12.0, n_objects=0 if w == 16 else 4)
    cur = synth.fade(clip.frame(1), a, b, seed) if a != 1.0 else clip.frame(1)
    p = make_params(w, h, search_range=64, local_search_range=32)
    ctx.upload_frame(0, *clip.frame(0))
    ctx.upload_frame(1, *cur)
    want = oracle.scene_change_score(p, cur, clip.frame(0), fade, thr)
    assert _bits(ctx.scene_change_score(p, 1, 0, bool(fade), thr)) == _bits(want)


def test_scene_score_rejects_bad_threshold(ctx):
    clip = synth.generate(64, 48, 2, 34)
    p = make_params(64, 48)
    ctx.upload_frame(0, *clip.frame(0))
    ctx.upload_frame(1, *clip.frame(1))
    with pytest.raises(Vc1cuError, match="threshold"):
        ctx.scene_change_score(p, 1, 0, True, 300.0)
