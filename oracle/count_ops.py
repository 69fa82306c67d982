"""Algorithmic op count of the analysis path per macroblock, from the instrumented oracle.

Runs the oracle's core passes over pictures of the first GOP of the 1080p benchmark clip (P
pictures 3 and 11 against their past anchors 0 and 9; the forward and backward passes, in
quarter-pel and half-pel bilinear mode, of B pictures 1 (anchors 0, 3) and 10 (anchors 9,
11)) and weights the evaluation counters (vo_counts) with the per-kind integer costs:

    integer-MV sample (SAD / prediction copy)   3 ops  (sub, abs, add)
    one-axis bicubic sample                      15 ops (4-tap filter 12 + 3)
    two-axis bicubic sample                      55 ops (5 column filters 52 amortised + 3)
    bilinear half-pel sample                     11 ops
    4x4 Hadamard SATD tile                       114 ops
    whole-frame SAD sample (global search)       3 ops
    FP64 transform: 2*(bh*bw*bh + bh*bw*bw) flops per partition; quantiser 10 flops/coefficient

Usage: python oracle/count_ops.py   (prints JSON; takes a few minutes)
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


P_PICTURES = ((3, 0), (11, 9))
B_PICTURES = ((1, 0, 3), (10, 9, 11))


def main() -> dict:
    clip = synth.hd1080(frames=12)
    o = Oracle()
    res = {"unseeded": [], "seeded_hpel": [], "seeded_bilinear": [], "seeded_mixed": [], "final_mixed_intra": [],
           "global_frame_ops_per_picture": [], "xform_flops_per_mb": [], "b_qpel_forward": [], "b_qpel_backward": [],
           "b_bilinear_forward": [], "b_bilinear_backward": []}
    mbs = 120 * 68
    p = make_params(1920, 1080, search_range=64, local_search_range=64, nonuniform=1, pqindex=4)
    for t, r in P_PICTURES:
        cur, ref = clip.frame(t), clip.frame(r)
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
    for t, past, fut in B_PICTURES:
        for mode, mname in ((MV_QPEL, "qpel"), (MV_HPEL_BILINEAR, "bilinear")):
            for ref, dname in ((past, "forward"), (fut, "backward")):
                o.reset_counts()
                o.analyze_p_core(p, clip.frame(t), clip.frame(ref), mode, False)
                res[f"b_{mname}_{dname}"].append(int_ops(o.counts()) / mbs)
    out = {k: sum(v) / len(v) for k, v in res.items()}
    out["pictures"] = {"p": P_PICTURES, "b": B_PICTURES}
    out["weights"] = {"int": W_INT, "qpel1d": W_1D, "qpel2d": W_2D, "bilinear": W_BIL, "satd_tile": W_SATD,
                      "frame_sample": W_FRAME}
    return out


if __name__ == "__main__":
    print(json.dumps(main(), indent=1))
