"""The scene-change-score cases shared by the fixture generator and the tests: seeded synthetic
pictures (motion, a cut, a fade, camera zooms) with the switches each case runs under."""
from libvc1_b200 import synth


def scene_pictures():
    """name -> (cur, ref, fade_compensation, scene_threshold, params)."""
    a, b = synth.generate(130, 98, 2, 1), synth.generate(130, 98, 2, 99)
    z = synth.generate(352, 288, 2, 5, zoom=1.04, global_px=0.0, n_objects=0)
    z2 = synth.generate(352, 288, 2, 7, zoom=1.05, global_px=0.0, n_objects=0)
    wide = dict(search_range=64, local_search_range=32)
    faded = synth.fade(a.frame(1), 0.6, 40.0, 3)
    return {
        "motion": (a.frame(1), a.frame(0), 1, 28.0, wide),
        "cut": (b.frame(0), a.frame(0), 1, 28.0, wide),
        "cut_low_threshold": (b.frame(0), a.frame(0), 1, 5.0, wide),
        "fade": (faded, a.frame(0), 1, 28.0, wide),
        "fade_no_compensation": (faded, a.frame(0), 0, 28.0, wide),
        "zoom_rescue": (z.frame(1), z.frame(0), 0, 10.0, dict(search_range=8, local_search_range=8)),
        "zoom_rescue_fade": (z2.frame(1), z2.frame(0), 1, 12.0, dict(search_range=32, local_search_range=32)),
        "range0": (a.frame(1), a.frame(0), 1, 28.0, dict(search_range=0, local_search_range=0)),
    }
