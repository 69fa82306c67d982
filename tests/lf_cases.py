"""Seeded inputs for the loop-filter tests: a blocky picture (noise added to a synthetic frame)
and random coded-block metadata (block vectors, loop_filter_pattern / loop_filter_tt codes, intra
bits) in the layout the reference's apply_p_loop_filter takes."""
import numpy as np

from libvc1_b200 import synth

TT_OF_TYPE = {1: 0, 2: 3, 3: 6, 4: 7}  # loop_filter_tt (encoder_filter.cpp)


def pattern(skip: int, t: int) -> int:
    """loop_filter_pattern (encoder_filter.cpp): the filtered sub-blocks of a transform type."""
    if t == 1:
        return 0x0F
    if t == 4:
        return (~skip) & 0x0F
    if t == 2:
        return (~(((skip & 2) * 6) + ((skip & 1) * 3))) & 0x0F
    return (~(skip * 5)) & 0x0F


def blocky_frame(w, h, seed):
    clip = synth.generate(w, h, 1, seed)
    rng = np.random.default_rng(seed)
    out = []
    for pl in clip.frame(0):
        ph, pw = pl.shape
        offs = rng.integers(-10, 11, ((ph + 7) // 8, (pw + 7) // 8)).repeat(8, 0).repeat(8, 1)[:ph, :pw]
        out.append(np.clip(pl.astype(int) + offs, 0, 255).astype(np.uint8))
    return tuple(out)


def metadata(w, h, seed, dense=True):
    rng = np.random.default_rng(seed + 1000)
    mbs = ((w + 15) // 16) * ((h + 15) // 16)
    bmv = rng.integers(-3, 4, (mbs, 4, 2)).astype(np.int32)
    if not dense:
        bmv[:] = bmv[:, :1, :]
    types = rng.integers(1, 5, (mbs, 6))
    skips = rng.integers(0, 16, (mbs, 6))
    cbp = np.array([[pattern(int(s) & (3 if t in (2, 3) else 15), int(t)) for s, t in zip(sr, tr)]
                    for sr, tr in zip(skips, types)], np.uint8)
    tt = np.vectorize(TT_OF_TYPE.get)(types).astype(np.uint8)
    intra = ((rng.random(mbs) < 0.08) * rng.integers(1, 64, mbs)).astype(np.uint8)
    return bmv, cbp, tt, intra
