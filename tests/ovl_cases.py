"""Seeded inputs for the overlap-smoothing tests: signed padded reconstructions (a synthetic
picture minus 128 with per-8x8-block offsets, as an intra reconstruction before its +128 store,
plus sample noise) and per-macroblock OVERFLAGS / intra maps."""
import numpy as np

from libvc1_b200 import synth

# (width, height, PQINDEX, seed); tests/golden/make_golden.py writes ovl_kat.npz from them
OVL_CASES = ((64, 48, 10, 1), (130, 98, 12, 2), (16, 16, 9, 3), (176, 144, 20, 4), (98, 66, 4, 5), (34, 18, 9, 6))


def signed_planes(w, h, seed):
    """int32 planes of the padded raster: (mbh*16, mbw*16) luma, (mbh*8, mbw*8) chroma."""
    mbw, mbh = (w + 15) // 16, (h + 15) // 16
    clip = synth.generate(mbw * 16, mbh * 16, 1, seed)
    rng = np.random.default_rng(seed)
    out = []
    for pl in clip.frame(0):
        ph, pw = pl.shape
        offs = rng.integers(-40, 41, (ph // 8, pw // 8)).repeat(8, 0).repeat(8, 1)
        out.append((pl.astype(np.int32) - 128 + offs + rng.integers(-6, 7, pl.shape)).astype(np.int32))
    return tuple(out)


def mb_flags(w, h, seed):
    mbw, mbh = (w + 15) // 16, (h + 15) // 16
    return (np.random.default_rng(seed + 100).random(mbw * mbh) < 0.5).astype(np.uint8)
