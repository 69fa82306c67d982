"""The learned-proposal workload: 1080p picture pairs with camera pans of up to +-128 pixels.

Everything runs on the device through the C ABI (include/vc1cu.h, vc1cu_lp_* and vc1cu_synth_frames):

- pairs: the seeded clip generator (global translation drawn in +-128 px at quarter-pel, 8 moving
  textured rectangles of 32-96 px at up to 8 px/frame, Irwin-Hall noise with sigma in [1, 4]),
  generated in device memory;
- labels: the plain unseeded quarter-pel pass at search range 128 (local range 32, UMH, the
  long-range searches beyond it), the reference's analyze_p_picture_core seed pass;
- training: the network's own forward and backward kernels and Adam, on the device;
- evaluation: on held-out pairs, the plain pass against the learned pass (the network's four
  candidates, an exact descent and refinement, the plain search where the best candidate is not a
  good match) by exact SAD of the chosen vectors, luma PSNR of the QP-6 reconstruction, and the
  share of macroblocks that fell back.

The shipped parameters (learned_weights.npy beside this file) come from `python -m
libvc1_b200.learned train`.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import synth
from .abi import MV_QPEL, make_params

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "learned_weights.npy")

W, H = 1920, 1080
RANGE, LOCAL = 128, 32
QP = 6
TRAIN_SEED0 = 100_000   # training pairs: seeds TRAIN_SEED0 + i
HELD_SEED0 = 900_000    # held-out pairs: seeds HELD_SEED0 + i (disjoint)
GROUP = 8               # pairs per batch of device work

# frame-slot and result-slot ranges this module uses on its context
_F0 = 2000              # frame slots _F0 .. _F0 + 2 * GROUP - 1 (pairs), then predictions / reconstructions
_R0 = 2000              # result slots


def pair_cfg(seed: int):
    """The generator configuration of one picture pair."""
    sigma = 1.0 + 3.0 * (((seed * 2654435761) >> 7) % 1000) / 1000.0
    return synth.make_cfg(W, H, 2, seed, global_px=128.0, n_objects=8, obj_min=32, obj_max=96, obj_vel=8.0,
                          sigma=sigma)


def params(pq: int = QP):
    return make_params(W, H, search_range=RANGE, local_search_range=LOCAL, pqindex=pq)


def make_pairs(ctx, seeds, slot0=_F0):
    """Generates the pairs on the device: pair k in frame slots slot0 + 2k (current) and
    slot0 + 2k + 1 (reference)."""
    for k, s in enumerate(seeds):
        cfg = pair_cfg(s)
        ctx.synth_frames(cfg, 1, 1, slot0 + 2 * k)
        ctx.synth_frames(cfg, 0, 1, slot0 + 2 * k + 1)


def build_dataset(ctx, net, seeds, first_sample=0, label=True):
    """Samples first_sample.. of `net` := the features, hints and (label) plain-pass labels of the
    pairs of `seeds`."""
    p = params()
    for g in range(0, len(seeds), GROUP):
        grp = seeds[g:g + GROUP]
        make_pairs(ctx, grp)
        for k in range(len(grp)):
            net.prepare(_F0 + 2 * k, _F0 + 2 * k + 1, first_sample + g + k)
        if label:
            ctx.core_passes(p, [(_F0 + 2 * k, _F0 + 2 * k + 1, MV_QPEL, 0, -1, _R0 + k) for k in range(len(grp))])
            for k in range(len(grp)):
                net.set_labels(first_sample + g + k, _R0 + k)
    ctx.synchronize()


def train(net, n_samples, epochs=8, batch=8, lr=2e-3, seed=0, log=None):
    """Adam over shuffled batches with a cosine-decayed learning rate; returns the loss curve."""
    rng = np.random.default_rng(seed)
    steps = epochs * (n_samples // batch)
    curve, step = [], 0
    for _ in range(epochs):
        perm = rng.permutation(n_samples)
        for b in range(0, n_samples - batch + 1, batch):
            a = lr * 0.5 * (1.0 + np.cos(np.pi * step / max(1, steps)))
            loss = net.train_step(perm[b:b + batch], float(max(a, 0.02 * lr)))
            curve.append(loss)
            step += 1
            if log and step % 100 == 0:
                log(f"step {step}/{steps} loss {np.mean(curve[-100:]):.4f}")
    return curve


def _psnr(a, b):
    mse = np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2)
    return 99.0 if mse == 0 else 10.0 * np.log10(255.0 * 255.0 / mse)


def evaluate(ctx, net, seeds, sample0=0, fallback=True, psnr=True):
    """Plain against learned on the pairs of `seeds` (samples sample0.. of `net` are overwritten).
    Returns per-pair exact SAD sums, PSNRs, fallback counts, and device milliseconds of both forms."""
    import torch

    p = params()
    mbs = ((W + 15) // 16) * ((H + 15) // 16)
    levels = torch.empty((mbs, 6, 64), dtype=torch.int16, device="cuda")
    types = np.ones(mbs * 6, np.uint8)
    out = {"sad_plain": [], "sad_learned": [], "psnr_plain": [], "psnr_learned": [], "fallback": [],
           "ms_plain": 0.0, "ms_learned": 0.0, "ms_prepare": 0.0, "ms_propose": 0.0, "ms_analyze": 0.0}
    stream = torch.cuda.ExternalStream(ctx.stream_handle())
    for g in range(0, len(seeds), GROUP):
        grp = seeds[g:g + GROUP]
        n = len(grp)
        make_pairs(ctx, grp)
        ctx.synchronize()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
        e[0].record(stream)
        ctx.core_passes(p, [(_F0 + 2 * k, _F0 + 2 * k + 1, MV_QPEL, 0, -1, _R0 + k) for k in range(n)])
        e[1].record(stream)
        e[2].record(stream)
        for k in range(n):
            net.prepare(_F0 + 2 * k, _F0 + 2 * k + 1, sample0 + k)
        e[3].record(stream)
        net.propose(sample0, n)
        e[4].record(stream)
        net.analyze(p, [(_F0 + 2 * k, _F0 + 2 * k + 1, sample0 + k, MV_QPEL, _R0 + 100 + k) for k in range(n)],
                    fallback=fallback)
        e[5].record(stream)
        e[5].synchronize()
        out["ms_plain"] += e[0].elapsed_time(e[1])
        out["ms_learned"] += e[2].elapsed_time(e[5])
        out["ms_prepare"] += e[2].elapsed_time(e[3])
        out["ms_propose"] += e[3].elapsed_time(e[4])
        out["ms_analyze"] += e[4].elapsed_time(e[5])
        for k in range(n):
            a = ctx.read_result(p, _R0 + k)
            b = ctx.read_result(p, _R0 + 100 + k)
            out["sad_plain"].append(int(a.screen_sads.astype(np.uint64).sum()))
            out["sad_learned"].append(int(b.screen_sads.astype(np.uint64).sum()))
            out["fallback"].append(int(net.read_sample(sample0 + k)[3].sum()))
            if psnr:
                cur = ctx.download_frame(_F0 + 2 * k, W, H)[0]
                for key, slot in (("psnr_plain", _R0 + k), ("psnr_learned", _R0 + 100 + k)):
                    ctx.motion_compensate(p, _F0 + 2 * k + 1, slot, MV_QPEL, _F0 + 40)
                    ctx.forward_quant_device(p, _F0 + 2 * k, _F0 + 40, 1, 0, levels.data_ptr())
                    ctx.reconstruct(p, _F0 + 40, levels.data_ptr(), 1, types, _F0 + 41)
                    rec = ctx.download_frame(_F0 + 41, W, H)[0]
                    out[key].append(_psnr(rec, cur))
    return out


def summarize(ev, mbs_per_pair):
    sp = np.array(ev["sad_plain"], np.float64)
    sl = np.array(ev["sad_learned"], np.float64)
    gap = (sl - sp) / np.maximum(sp, 1.0)
    n = len(sp)
    s = {"pairs": n, "cost_gap_mean": float(gap.mean()), "cost_gap_p99": float(np.percentile(gap, 99)),
         "fallback_rate": float(np.sum(ev["fallback"]) / (n * mbs_per_pair)),
         "mbs_per_s_plain": n * mbs_per_pair / (ev["ms_plain"] / 1e3) if ev["ms_plain"] else None,
         "mbs_per_s_learned": n * mbs_per_pair / (ev["ms_learned"] / 1e3) if ev["ms_learned"] else None,
         "ms_per_pair": {k[3:]: ev[k] / max(n, 1) for k in ("ms_plain", "ms_learned", "ms_prepare", "ms_propose",
                                                            "ms_analyze")}}
    if s["mbs_per_s_plain"] and s["mbs_per_s_learned"]:
        s["speedup"] = s["mbs_per_s_learned"] / s["mbs_per_s_plain"]
    if ev["psnr_plain"]:
        s["psnr_plain"] = float(np.mean(ev["psnr_plain"]))
        s["psnr_learned"] = float(np.mean(ev["psnr_learned"]))
        s["psnr_delta_db"] = s["psnr_learned"] - s["psnr_plain"]
    return s


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("cmd", choices=["train", "eval"])
    ap.add_argument("--pairs", type=int, default=2000)
    ap.add_argument("--held", type=int, default=300)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--weights", default=WEIGHTS)
    ap.add_argument("--out", default=None, help="where train writes the parameters (default --weights)")
    ap.add_argument("--report", default=None, help="JSON summary path")
    ap.add_argument("--no-psnr", action="store_true")
    a = ap.parse_args(argv)
    from .api import CudaComputeContext, LearnedProposals

    ctx, err = CudaComputeContext.create(0)
    if ctx is None:
        raise SystemExit(f"CUDA backend unavailable: {err}")
    mbs = ((W + 15) // 16) * ((H + 15) // 16)
    log = lambda m: print(m, flush=True)  # noqa: E731
    report = {}
    if a.cmd == "train":
        net = LearnedProposals(ctx, W, H, RANGE, a.pairs, max_batch=8, seed=1)
        t0 = time.time()
        build_dataset(ctx, net, [TRAIN_SEED0 + i for i in range(a.pairs)])
        log(f"dataset: {a.pairs} pairs in {time.time() - t0:.1f} s")
        t0 = time.time()
        curve = train(net, a.pairs, epochs=a.epochs, lr=a.lr, log=log)
        log(f"training: {len(curve)} steps in {time.time() - t0:.1f} s, loss {np.mean(curve[:50]):.4f} -> "
            f"{np.mean(curve[-50:]):.4f}")
        np.save(a.out or a.weights, net.params())
        report["train"] = {"pairs": a.pairs, "steps": len(curve), "loss_first": float(np.mean(curve[:50])),
                           "loss_last": float(np.mean(curve[-50:]))}
        net.close()
    net = LearnedProposals(ctx, W, H, RANGE, GROUP, max_batch=GROUP, seed=1)
    net.set_params(np.load(a.out or a.weights))
    t0 = time.time()
    ev = evaluate(ctx, net, [HELD_SEED0 + i for i in range(a.held)], psnr=not a.no_psnr)
    report["eval"] = summarize(ev, mbs)
    log(f"evaluation ({time.time() - t0:.1f} s): {json.dumps(report['eval'])}")
    if a.report:
        with open(a.report, "w") as f:
            json.dump(report, f, indent=1)
    net.close()
    ctx.close()


if __name__ == "__main__":
    main()
