"""Algorithmic op count of the analysis path per macroblock, from the instrumented oracle.

Runs the oracle's core passes over P pictures of the 1080p benchmark clip and weights the
evaluation counters (vo_counts) with the per-kind integer costs of the path:

    integer-MV sample (SAD / prediction copy)   3 ops  (sub, abs, add)
    one-axis bicubic sample                      15 ops (4-tap filter 12 + 3)
    two-axis bicubic sample                      55 ops (5 column filters 52 amortised + 3)
    bilinear half-pel sample                     11 ops
    4x4 Hadamard SATD tile                       114 ops
    whole-frame SAD sample (global search)       3 ops
    FP64 transform: 2*(bh*bw*bh + bh*bw*bw) flops per partition; quantiser 10 flops/coefficient

Usage: python oracle/count_ops.py [pictures]   (prints JSON; takes about a minute)
This is measurement infrastructure: bench.py embeds the resulting per-MB constants.
"""
from __future__ import annotations

import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from libvc1_b200 import synth  # noqa: E402
from libvc1_b200.abi import MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED, MV_QPEL, make_params  # noqa: E402
from oracle import Oracle  # noqa: E402

W_INT, W_1D, W_2D, W_BIL, W_SATD, W_FRAME = 3, 15, 55, 11, 114, 3


def int_ops(c: dict) -> float:
    return (W_INT * c["int_sad_samples"] + W_1D * c["qpel1d_samples"] + W_2D * c["qpel2d_samples"] +
            W_BIL * c["bilinear_samples"] + W_SATD * c["satd_tiles"])


def main(pictures: int = 2) -> dict:
    clip = synth.hd1080(frames=3 * pictures + 1)
    o = Oracle()
    res = {"unseeded": [], "seeded_hpel": [], "seeded_bilinear": [], "seeded_mixed": [], "final_mixed_intra": [],
           "global_frame_ops_per_picture": [], "xform_flops_per_mb": []}
    mbs = 120 * 68
    for k in range(pictures):
        t = 3 * (k + 1)
        cur, ref = clip.frame(t), clip.frame(t - 3)
        p = make_params(1920, 1080, search_range=64, local_search_range=64, nonuniform=1, pqindex=4 + 2 * k)
        o.reset_counts()
        q = o.analyze_p_core(p, cur, ref, MV_QPEL, False)
        c = o.counts()
        res["unseeded"].append(int_ops(c) / mbs)
        res["global_frame_ops_per_picture"].append(W_FRAME * c["frame_sad_samples"])
        seeds = {}
        for name, m in (("seeded_hpel", MV_HPEL), ("seeded_bilinear", MV_HPEL_BILINEAR), ("seeded_mixed", MV_MIXED)):
            o.reset_counts()
            seeds[m] = o.analyze_p_core(p, cur, ref, m, False, seed=q.mvs, seed_distant=q)
            res[name].append(int_ops(o.counts()) / mbs)
        o.reset_counts()
        f = o.analyze_p_core(p, cur, ref, MV_MIXED, True, seed=seeds[MV_MIXED].mvs, seed_distant=seeds[MV_MIXED])
        res["final_mixed_intra"].append(int_ops(o.counts()) / mbs)
        pred = o.motion_compensate(p, ref, f, MV_MIXED)
        o.reset_counts()
        o.forward_quant(p, cur, pred, 15)
        c = o.counts()
        res["xform_flops_per_mb"].append((c["xform_flops"] + 10 * c["quant_coeffs"]) / mbs)
    out = {k: sum(v) / len(v) for k, v in res.items()}
    out["pictures"] = pictures
    out["weights"] = {"int": W_INT, "qpel1d": W_1D, "qpel2d": W_2D, "bilinear": W_BIL, "satd_tile": W_SATD,
                      "frame_sample": W_FRAME}
    return out


if __name__ == "__main__":
    print(json.dumps(main(int(sys.argv[1]) if len(sys.argv) > 1 else 2), indent=1))
