"""The device-side clip generator (vc1cu_synth_frames) against the host generator: the same
bytes for the benchmark configurations' content (pans, zoom, objects, noise)."""
import numpy as np
import pytest

from libvc1_b200 import synth

pytestmark = pytest.mark.gpu

CASES = {
    "cif": dict(width=352, height=288, frames=3, seed=1),
    "hd_learned": dict(width=1920, height=1080, frames=2, seed=7, global_px=128.0, n_objects=8, obj_vel=8.0, sigma=2.5),
    "odd_zoom": dict(width=322, height=242, frames=5, seed=9, zoom=1.002, n_objects=6),
    "no_noise": dict(width=64, height=48, frames=2, seed=3, sigma=0.0, n_objects=0),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_device_generator_matches_host(ctx, case):
    kw = dict(CASES[case])
    w, h, t, seed = kw.pop("width"), kw.pop("height"), kw.pop("frames"), kw.pop("seed")
    clip = synth.generate(w, h, t, seed, **kw)
    cfg = synth.make_cfg(w, h, t, seed, **kw)
    # all frames in one call, and the last frame alone (its own global track and zoom)
    ctx.synth_frames(cfg, 0, t, 700)
    ctx.synth_frames(cfg, t - 1, 1, 800)
    for i in range(t):
        got = ctx.download_frame(700 + i, w, h)
        assert all(np.array_equal(a, b) for a, b in zip(got, clip.frame(i))), (case, i)
    got = ctx.download_frame(800, w, h)
    assert all(np.array_equal(a, b) for a, b in zip(got, clip.frame(t - 1)))


def test_device_generator_checks_arguments(ctx):
    from libvc1_b200.api import Vc1cuError

    cfg = synth.make_cfg(64, 48, 2, 1)
    with pytest.raises(Vc1cuError):
        ctx.synth_frames(cfg, 1, 2, 0)  # beyond the clip
    with pytest.raises(Vc1cuError):
        ctx.synth_frames(cfg, 0, 65, 0)  # more than 64 frames per call
