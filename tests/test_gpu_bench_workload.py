"""The benchmarked workload, one GOP, against the reference build itself.

bench.py times a step of the 1080p IBBP workload (search +/-64, non-uniform quantiser): per P
picture the quarter-pel seed pass, the three seeded mode passes, the final Mixed-MV pass with
P-intra, the fade estimate along its field, the prediction and the transform + quantiser of all
four transform types; per B picture analyze_b_picture_mode in quarter-pel and in half-pel
bilinear mode against the future anchor's final pass. Here the first GOP of that workload
(4 P + 7 B pictures) runs through bench.Runner exactly as timed, at PQINDEX 4 and 12, and every
result is compared bit for bit with the reference's own functions (oracle/_ref, compiled from
the reference's sources, scalar path):

- every P pass: Vc1Encoder::analyze_p_picture_core (encoder_motion.cpp:47-442) as
  analyze_p_picture chains it (:524-597);
- the fade estimate: estimate_intensity_comp (encoder_motion_compensation.cpp:296-348);
- the prediction: motion_compensate_* (encoder_motion_compensation.cpp:474-600);
- coefficients' levels of the four types: forward_transform_residual_part + scalar_quantize_level
  (encoder_transform.cpp:935-1171);
- both B modes: analyze_b_picture_mode (encoder_motion.cpp:753-1005).
"""
import concurrent.futures
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402
from libvc1_b200 import synth  # noqa: E402
from libvc1_b200.abi import MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED, MV_QPEL  # noqa: E402
from libvc1_b200.replicas import clip_seed  # noqa: E402
from oracle.bindings import Reference, ref_available  # noqa: E402

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")]

_THREADS = max(1, min(16, os.cpu_count() or 1))


def _ref_p_chain(pq, cur, ref):
    """analyze_p_picture's passes for one picture, its fade estimate, prediction and levels."""
    r = Reference(bench.params(pq))
    seed = r.analyze_p_core(cur, ref, MV_QPEL, False)
    modes = {m: r.analyze_p_core(cur, ref, m, False, seed=seed.mvs, seed_distant=seed)
             for m in (MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED)}
    mixed = modes[MV_MIXED]
    final = r.analyze_p_core(cur, ref, MV_MIXED, True, seed=mixed.mvs, seed_distant=mixed)
    ic = r.estimate_intensity_comp(cur, ref, final.mvs)
    pred = r.motion_compensate(ref, final, MV_MIXED)
    _, levels = r.forward_quant(cur, pred, 15)
    return seed, modes, final, ic, pred, levels


def _ref_b(pq, cur, past, fut, anchor, num, den, mode):
    return Reference(bench.params(pq)).analyze_b(cur, past, fut, anchor.mvs, anchor.use_4mv, num, den, mode)


@pytest.mark.parametrize("pq", [4, 12])
def test_bench_gop_matches_reference(ctx, pq):
    torch = pytest.importorskip("torch")
    clip = synth.hd1080(frames=bench.GOP, seed=clip_seed(0))
    run = bench.Runner(ctx, clip, gops=1)
    run.pics = [(t, r, pq) for t, r, _ in run.pics]
    run.bpics = [(t, past, fut, num, den, pq, a) for t, past, fut, num, den, _, a in run.bpics]
    run.upload_all()
    run.step()
    ctx.synchronize()
    F = clip.frame
    with concurrent.futures.ThreadPoolExecutor(_THREADS) as ex:
        pj = [ex.submit(_ref_p_chain, pq, F(t), F(r)) for t, r, _ in run.pics]
        want_p = [j.result() for j in pj]
        bj = {(k, j): ex.submit(_ref_b, pq, F(t), F(past), F(fut), want_p[a][2], num, den, m)
              for k, (t, past, fut, num, den, _, a) in enumerate(run.bpics)
              for j, m in enumerate((MV_QPEL, MV_HPEL_BILINEAR))}
        want_b = {key: j.result() for key, j in bj.items()}
    bad = []
    levels = run.levels.cpu().numpy()
    p = run.p0
    for i, (t, r, _) in enumerate(run.pics):
        seed, modes, final, ic, pred, lv = want_p[i]
        bad += [(t, "seed", f) for f in ctx.read_result(p, run.seed_slot(i)).equal(seed)]
        for m, e in modes.items():
            bad += [(t, f"mode{m}", f) for f in ctx.read_result(p, run.mode_slot(i, m)).equal(e)]
        bad += [(t, "final", f) for f in ctx.read_result(p, run.final_slot(i)).equal(final)]
        if tuple(run.ic[i]) != tuple(ic):
            bad.append((t, "fade", (run.ic[i], ic)))
        g = ctx.download_frame(3500 + i, bench.W, bench.H)
        if not all(np.array_equal(a, b) for a, b in zip(g, pred)):
            bad.append((t, "prediction", None))
        if not np.array_equal(levels[i], lv):
            bad.append((t, "levels", int((levels[i] != lv).sum())))
    for (k, j), e in want_b.items():
        bad += [(run.bpics[k][0], f"b{j}", f) for f in ctx.read_bresult(p, run.bresult_slot(k, j)).equal(e)]
    assert bad == []
    # the comparison covered every result slot of the step
    assert len(want_p) == 4 and len(want_b) == 14
