#!/usr/bin/env python
"""Encoder-analysis throughput of libvc1's analysis hot path on B200, in macroblocks/s.

Workload (the 1080p configuration): 1920x1080 8-bit 4:2:0, 60 seeded synthetic frames
(value-noise texture, zoom 1.002/frame, 8 objects at up to 8 px/frame, sigma 2), GOP 12
IBBP planned the way the reference's encoder plans it (encoder_core.cpp:928-962: segments
start at each I picture, anchors every 3 frames, the segment's last frame an anchor), so per
GOP P pictures at 3, 6, 9, 11 and B pictures at 1, 2, 4, 5, 7, 8, 10: 20 P and 35 B
pictures per clip. Search range +/-64, Mixed-MV, non-uniform quantiser at QP 4/6/8/10/12
(one per GOP; a B picture takes its GOP's QP).

One step = every picture of the clip analysed:
  P pictures: the quarter-pel seed pass, the three seeded mode passes (half-pel, half-pel
    bilinear, Mixed-MV), the final Mixed-MV pass with P-intra, the fade (intensity
    compensation) estimate along its vectors, the decoder-equivalent prediction, and the
    forward transform + quantiser of that prediction for all four transform sizes (Vc1Encoder::analyze_p_picture_core x5 and quantize_inter_part,
    src/encoder_motion.cpp:47-597, src/encoder_transform.cpp:935-1171). The final pass is
    timed in Mixed-MV mode, the most expensive of the reference's four candidates (the
    reference chooses it on the host by sampled RD).
  B pictures: analyze_b_picture_mode in quarter-pel and in half-pel bilinear mode (the two
    modes analyze_b_picture compares, encoder_motion.cpp:1062-1095): per mode the forward
    and backward core passes and the per-macroblock Direct / Forward / Backward /
    Interpolated / Intra decision against the future P anchor's final-pass vectors
    (src/encoder_motion.cpp:753-1005).

  value : MB/s with the clip resident in HBM (CUDA events on the library's stream, L2
          flushed between steps)
  e2e   : MB/s through the C ABI from pinned host frames, including the H2D upload of the
          step's frames and the D2H read of every result (MVs, decisions, levels)
  --impl reference : the reference's own CPU code (oracle/_ref, SIMD dispatch on) on the
          host's cores, same workload and unit

Multi-GPU: one process per GPU (torchrun); each rank analyses its own clip (seeded by
rank), no collective on the data path; value = all ranks' MBs / max rank time.
Profiling: --gops N analyses only the pictures of the first N GOPs.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

W, H = 1920, 1080
FRAMES, GOP, BFRAMES = 60, 12, 2
MBS = ((W + 15) // 16) * ((H + 15) // 16)
METRIC = "1080p ME+qpel+xform MB/s on 1 B200: plain (bit-exact) vs learned @<=1% cost gap"
UNIT = "MB/s"

# Algorithmic integer ops per macroblock of each core pass on this workload, from the
# instrumented oracle (oracle/count_ops.py over pictures of the clip's first GOP; weights there).
OPS_PER_MB = {"unseeded": 286137.3, "seeded_hpel": 56261.4, "seeded_bilinear": 25321.8, "seeded_mixed": 471920.4,
              "final_mixed_intra": 472178.7, "b_qpel_forward": 286981.1, "b_qpel_backward": 289317.5,
              "b_bilinear_forward": 121400.1, "b_bilinear_backward": 122512.3}
WORKLOAD = ("1080p IBBP analysis: 1920x1080 4:2:0, 60 frames, GOP 12 IBBP as the reference plans it -> 20 P + 35 B "
            "pictures/step; P: 5 core passes + fade estimate + prediction + 4-size transform/quant; B: forward+backward "
            "core passes and "
            "the MB decision in qpel and hpel-bilinear mode; search +/-64, Mixed-MV, nonuniform QP 4-12")
# DRAM bytes (read + write) of core_pass_kernel per launch on this workload, with the sub-pel
# plane builds that precede each launch: an ncu capture of the first GOP's six core launches and
# their plane builds (709.7 MB in all; the core launches re-read the 15 phase planes of each
# reference) scaled by macroblocks to the five GOPs of a step and divided over the step's six
# launches.
CORE_DRAM_BYTES_PER_LAUNCH = 709.7e6 * 5 / 6  # ncu, first GOP (6 launches + planes), scaled to the 5 GOPs of a step
P_PASSES = ("unseeded", "seeded_hpel", "seeded_bilinear", "seeded_mixed", "final_mixed_intra")
B_PASSES = ("b_qpel_forward", "b_qpel_backward", "b_bilinear_forward", "b_bilinear_backward")
XFORM_FLOPS_PER_MB = 51911.5


def gop_plan(gops=None):
    """P pictures [(frame, past anchor, PQINDEX)] and B pictures [(frame, past, future,
    fraction_num, fraction_den, PQINDEX, index of the future anchor in the P list)] of GOP 12
    IBBP over FRAMES frames, planned like the reference's encoder (encoder_core.cpp:928-962)."""
    ps, bs = [], []
    for seg in range(0, FRAMES, GOP):
        if gops is not None and seg // GOP >= gops:
            break
        end = min(seg + GOP, FRAMES)
        pq = 4 + 2 * ((seg // GOP) % 5)
        prev = seg
        while prev + 1 < end:
            nxt = min(prev + BFRAMES + 1, end - 1)
            ps.append((nxt, prev, pq))
            for j in range(prev + 1, nxt):
                bs.append((j, prev, nxt, j - prev, nxt - prev, pq, len(ps) - 1))
            prev = nxt
    return ps, bs


def make_clip(rank: int):
    from libvc1_b200 import synth
    from libvc1_b200.replicas import clip_seed

    return synth.hd1080(frames=FRAMES, seed=clip_seed(rank))


def params(pq: int):
    from libvc1_b200.abi import make_params

    return make_params(W, H, search_range=64, local_search_range=64, nonuniform=1, pqindex=pq)


# ---------------------------------------------------------------------------------------
def sample_clocks(stop_path: str):
    cmd = ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
           "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
           "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
           "--format=csv,noheader,nounits", "-lms", "200"]
    try:
        return subprocess.Popen(cmd, stdout=open(stop_path, "w"), stderr=subprocess.DEVNULL)
    except Exception:
        return None


def parse_clocks(path: str, device: int):
    sm, mx, reasons = [], 0.0, set()
    try:
        for line in open(path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9 or int(f[0]) != device:
                continue
            sm.append(float(f[1]))
            mx = max(mx, float(f[2]))
            for name, val in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
    except Exception:
        pass
    return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None, "reasons": sorted(reasons),
            "samples": len(sm)}


# ---------------------------------------------------------------------------------------
class Runner:
    """Drives one step of the analysis path through the C ABI."""

    def __init__(self, ctx, clip, gops=None):
        from libvc1_b200.abi import MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED, MV_QPEL

        self.ctx, self.clip = ctx, clip
        self.pics, self.bpics = gop_plan(gops)
        self.frames = sorted({f for p in self.pics for f in p[:2]} | {f for b in self.bpics for f in b[:3]})
        self.p0 = params(8)
        self.modes = (MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED)
        self.QPEL, self.MIXED, self.BIL = MV_QPEL, MV_MIXED, MV_HPEL_BILINEAR
        import torch

        self.torch = torch
        n = len(self.pics)
        # device-side levels of every picture: [pic][type][mb][parent][64] int16
        self.levels = torch.empty((n, 4, MBS, 6, 64), dtype=torch.int16, device="cuda")
        self.frame_bytes = W * H * 3 // 2

    @staticmethod
    def fid(f, b=0):
        """Frame slot of clip frame f in frame set b (two sets let a pipelined run upload one
        step's frames while the previous step reads the other set)."""
        return f + 100 * b

    def upload_all(self, pinned=None, b=0):
        for f in self.frames:
            if pinned is None:
                self.ctx.upload_frame(self.fid(f, b), *self.clip.frame(f))
            else:
                y, u, v = pinned[f]
                self.ctx.upload_frame_ptr(self.fid(f, b), y.data_ptr(), u.data_ptr(), v.data_ptr(), W, H)

    # Result-slot ids of the step's passes; `b` selects one of two sets, so that a pipelined run
    # can read one step's results while the next step writes the other set.
    @staticmethod
    def seed_slot(i, b=0):
        return 1000 * b + i

    @staticmethod
    def mode_slot(i, m, b=0):
        return 1000 * b + 100 + 4 * i + m

    @staticmethod
    def final_slot(i, b=0):
        return 1000 * b + 200 + i

    @staticmethod
    def bpass_slot(k, bil, fut, b=0):
        return 1000 * b + 300 + 4 * k + 2 * bil + fut

    @staticmethod
    def bresult_slot(k, j, b=0):
        return 100 * b + 2 * k + j

    def step(self, levels=None, mark=None, b=0):
        """Enqueues one step on the library's stream and runs its fade estimates (which wait for
        the step's device work); levels go to `levels` (default self.levels). mark(stage), when
        given, is called after each stage (to record a timing event)."""
        self.launch(levels, mark, b)
        self.finish(mark, b)

    def launch(self, levels=None, mark=None, b=0):
        """The step's device work up to the B decisions, enqueued without waiting."""
        levels = self.levels if levels is None else levels
        c, F = self.ctx, lambda f: self.fid(f, b)
        pics = [(F(t), F(r), pq) for t, r, pq in self.pics]
        bpics = [(F(t), F(past), F(fut), num, den, pq, a) for t, past, fut, num, den, pq, a in self.bpics]
        mark = mark or (lambda stage: None)
        # every P picture's quarter-pel seed pass and the four unseeded core passes of every B
        # picture (forward / backward in quarter-pel and in half-pel bilinear mode); the library
        # runs one launch per pass kind
        c.core_passes(self.p0, [(t, r, self.QPEL, 0, -1, self.seed_slot(i, b), pq) for i, (t, r, pq) in enumerate(pics)] +
                      [(t, ref, m, 0, -1, self.bpass_slot(k, m == self.BIL, ref == fut, b), pq)
                       for k, (t, past, fut, _n, _d, pq, _a) in enumerate(bpics)
                       for m in (self.QPEL, self.BIL) for ref in (past, fut)])
        mark("unseeded passes")
        # the three seeded mode passes of every picture (the library runs one launch per mode)
        c.core_passes(self.p0, [(t, r, m, 0, self.seed_slot(i, b), self.mode_slot(i, m, b), pq)
                                for i, (t, r, pq) in enumerate(pics) for m in self.modes])
        mark("seeded mode passes")
        # the final pass (after the host's mode decision over whole passes)
        c.core_passes(self.p0, [(t, r, self.MIXED, 1, self.mode_slot(i, self.MIXED, b), self.final_slot(i, b), pq)
                                for i, (t, r, pq) in enumerate(pics)])
        mark("final passes")
        for i, (t, r, pq) in enumerate(pics):
            p = params(pq)
            c.motion_compensate(p, r, self.final_slot(i, b), self.MIXED, 3500 + i)
            c.forward_quant_device(p, t, 3500 + i, 15, 0, levels[i].data_ptr())
        mark("prediction + transform")
        # the B decisions of both modes against the future anchor's final pass
        if bpics:
            c.b_decide(self.p0, [(t, past, fut, self.bpass_slot(k, j, 0, b), self.bpass_slot(k, j, 1, b),
                                  self.final_slot(a, b), num, den, m, self.bresult_slot(k, j, b), pq)
                                 for k, (t, past, fut, num, den, pq, a) in enumerate(bpics)
                                 for j, m in enumerate((self.QPEL, self.BIL))])
        mark("B decisions")

    def tune(self, b=0):
        """The library's launch-shape autotuner on each of the step's launch kinds (unseeded
        passes, seeded half-pel modes, seeded Mixed-MV, final passes); later launches of those
        kinds use the fastest shape. Returns the shapes found."""
        c, F = self.ctx, lambda f: self.fid(f, b)
        pics = [(F(t), F(r), pq) for t, r, pq in self.pics]
        bpics = [(F(t), F(past), F(fut), pq) for t, past, fut, _n, _d, pq, _a in self.bpics]
        groups = {
            "unseeded": [(t, r, self.QPEL, 0, -1, self.seed_slot(i, b), pq) for i, (t, r, pq) in enumerate(pics)] +
                        [(t, ref, m, 0, -1, self.bpass_slot(k, m == self.BIL, ref == fut, b), pq)
                         for k, (t, past, fut, pq) in enumerate(bpics) for m in (self.QPEL, self.BIL) for ref in (past, fut)],
            "seeded_hpel": [(t, r, m, 0, self.seed_slot(i, b), self.mode_slot(i, m, b), pq)
                            for i, (t, r, pq) in enumerate(pics) for m in self.modes[:2]],
            "seeded_mixed": [(t, r, self.MIXED, 0, self.seed_slot(i, b), self.mode_slot(i, self.MIXED, b), pq)
                             for i, (t, r, pq) in enumerate(pics)],
            "final": [(t, r, self.MIXED, 1, self.mode_slot(i, self.MIXED, b), self.final_slot(i, b), pq)
                      for i, (t, r, pq) in enumerate(pics)],
        }
        out = {}
        for name, passes in groups.items():
            w, blk, ms = c.autotune(self.p0, passes)
            out[name] = {"warps_per_block": w, "blocks_per_sm": blk or "occupancy limit", "ms": round(ms, 3)}
        return out

    def finish(self, mark=None, b=0):
        """The fade estimate analyze_p_picture runs on its final pass when fade compensation is on
        (the default; encoder_motion.cpp:570-573); it waits for the step's device work."""
        mark = mark or (lambda stage: None)
        self.ic = self.ctx.estimate_intensity_batch(
            self.p0, [(self.fid(t, b), self.fid(r, b), self.final_slot(i, b)) for i, (t, r, pq) in enumerate(self.pics)])
        mark("fade estimates")

    def enqueue_ic(self, b=0):
        """finish() in two phases for a pipelined run: the estimates' device work, enqueued
        without waiting; returns the ticket collect_ic takes."""
        return self.ctx.estimate_intensity_enqueue(
            self.p0, [(self.fid(t, b), self.fid(r, b), self.final_slot(i, b)) for i, (t, r, pq) in enumerate(self.pics)])

    def collect_ic(self, ticket):
        self.ic = self.ctx.estimate_intensity_collect(ticket)

    def read_results(self, b=0):
        """D2H of every P picture's final-pass analysis and every B analysis of slot set b; each
        read waits only for the launch that wrote its slot."""
        return ([self.ctx.read_result(self.p0, self.final_slot(i, b)) for i in range(len(self.pics))] +
                [self.ctx.read_bresult(self.p0, self.bresult_slot(k, j, b))
                 for k in range(len(self.bpics)) for j in range(2)])

    def mbs_per_step(self):
        return (len(self.pics) + len(self.bpics)) * MBS

    def result_bytes(self):
        per_mb = 8 + 32 + 1 + 1 + 8 + 8 + 8 + 8 + 1
        per_b_mb = 1 + 8 + 8 + 8 + 2 * (8 + 8 + 1)
        return len(self.pics) * (MBS * per_mb) + 2 * len(self.bpics) * MBS * per_b_mb + self.levels.numel() * 2


def learned_leg(ctx, torch, l2, steps, warmup, pairs=16):
    """The learned-proposal form against the plain form on the learned workload (1080p pairs with
    pans of up to +-128 px, search range 128, local range 32; libvc1_b200/learned.py), both as
    ME + quarter-pel refinement + prediction + the four transform sizes' forward transform and
    quantiser, over `pairs` held-out pairs generated on the device. Device time per rep with CUDA
    events on the library stream, L2 flushed between reps; the exact-SAD cost gap and fallback
    rate of the same pairs."""
    from libvc1_b200 import learned as lw
    from libvc1_b200.abi import MV_QPEL
    from libvc1_b200.api import LearnedProposals

    if not os.path.exists(lw.WEIGHTS):
        return {"unavailable": "no trained parameters (libvc1_b200/learned_weights.npy)"}
    p = lw.params()
    mbs = ((lw.W + 15) // 16) * ((lw.H + 15) // 16)
    net = LearnedProposals(ctx, lw.W, lw.H, lw.RANGE, pairs, max_batch=pairs, seed=1)
    net.set_params(np.load(lw.WEIGHTS))
    seeds = [lw.HELD_SEED0 + 5000 + i for i in range(pairs)]
    F0, R0, P0 = 3000, 3000, 3200
    for k, s in enumerate(seeds):
        cfg = lw.pair_cfg(s)
        ctx.synth_frames(cfg, 1, 1, F0 + 2 * k)
        ctx.synth_frames(cfg, 0, 1, F0 + 2 * k + 1)
    levels = torch.empty((pairs, 4, mbs, 6, 64), dtype=torch.int16, device="cuda")
    ext = torch.cuda.ExternalStream(ctx.stream_handle())
    plain_passes = [(F0 + 2 * k, F0 + 2 * k + 1, MV_QPEL, 0, -1, R0 + k) for k in range(pairs)]
    learned_passes = [(F0 + 2 * k, F0 + 2 * k + 1, k, MV_QPEL, R0 + 100 + k) for k in range(pairs)]

    def xform(slot0):
        for k in range(pairs):
            ctx.motion_compensate(p, F0 + 2 * k + 1, slot0 + k, MV_QPEL, P0 + k)
            ctx.forward_quant_device(p, F0 + 2 * k, P0 + k, 15, 0, levels[k].data_ptr())

    def plain():
        ctx.core_passes(p, plain_passes)
        xform(R0)

    def learned_form():
        for k in range(pairs):
            net.prepare(F0 + 2 * k, F0 + 2 * k + 1, k)
        net.propose(0, pairs)
        net.analyze(p, learned_passes, fallback=True)
        xform(R0 + 100)

    ms = {}
    for name, fn in (("plain", plain), ("learned", learned_form)):
        for _ in range(warmup):
            fn()
        ctx.synchronize()
        t = 0.0
        for _ in range(steps):
            with torch.cuda.stream(ext):
                l2.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(ext)
            fn()
            b.record(ext)
            b.synchronize()
            t += a.elapsed_time(b)
        ms[name] = t / steps
    sp = np.array([ctx.read_result(p, R0 + k).screen_sads.astype(np.float64).sum() for k in range(pairs)])
    sl = np.array([ctx.read_result(p, R0 + 100 + k).screen_sads.astype(np.float64).sum() for k in range(pairs)])
    gap = (sl - sp) / np.maximum(sp, 1.0)
    fb = sum(int(net.read_sample(k)[3].sum()) for k in range(pairs))
    net.close()
    mb = pairs * mbs
    return {"workload": f"{pairs} held-out 1080p pairs, pans up to +-128 px, 8 objects, sigma 1-4; search range "
                        f"{lw.RANGE}, local {lw.LOCAL}; ME + qpel + prediction + 4-size transform/quant, QP {lw.QP}",
            "mb_per_s_plain": round(mb / (ms["plain"] * 1e-3), 1), "mb_per_s_learned": round(mb / (ms["learned"] * 1e-3), 1),
            "speedup": round(ms["plain"] / ms["learned"], 3), "ms_per_rep_plain": round(ms["plain"], 3),
            "ms_per_rep_learned": round(ms["learned"], 3), "cost_gap_mean": round(float(gap.mean()), 5),
            "cost_gap_p99": round(float(np.percentile(gap, 99)), 5), "fallback_rate": round(fb / mb, 4),
            "cost_gap_definition": "per pair (sum of the chosen vectors' exact SAD, learned - plain) / plain"}


def longrange_leg(ctx, torch, reps, clips=8, frames=12):
    """Long-range pans (1920x1080, pans up to 200 px/frame horizontal and 60 vertical, 4 objects;
    search range 1024 = MVRANGE 3, local 32, QP 6): `clips` clips of `frames` frames, every frame
    step's P pictures of all clips as one batch. The plain batched form (one launch of the
    unseeded quarter-pel passes per frame step) against the learned form (hint + features +
    network for every clip, one learned launch and one fallback launch per frame step), each GOP
    captured as one CUDA graph and replayed; then the exact-SAD cost gap, fallback rate and the
    luma PSNR of the QP-6 reconstruction of every pair."""
    from libvc1_b200 import learned as lw
    from libvc1_b200 import synth
    from libvc1_b200.abi import MV_QPEL, make_params
    from libvc1_b200.api import LearnedProposals

    if not os.path.exists(lw.WEIGHTS):
        return {"unavailable": "no trained parameters (libvc1_b200/learned_weights.npy)"}
    p = make_params(W, H, search_range=1024, local_search_range=32, pqindex=lw.QP)
    F0, R0 = 200, 2000
    fid = lambda k, t: F0 + 64 * k + t  # noqa: E731
    for k in range(clips):
        cfg = synth.make_cfg(W, H, frames, 700 + k, global_px=200.0, global_py=60.0, n_objects=4, obj_vel=8.0,
                             sigma=2.0)
        ctx.synth_frames(cfg, 0, frames, fid(k, 0))
    net = LearnedProposals(ctx, W, H, 1024, clips, max_batch=clips, seed=1)
    net.set_params(np.load(lw.WEIGHTS))
    steps = range(1, frames)
    pslot = lambda k, t: R0 + 2 * (frames * k + t)  # noqa: E731
    lslot = lambda k, t: pslot(k, t) + 1  # noqa: E731

    def plain_gop():
        for t in steps:
            ctx.core_passes(p, [(fid(k, t), fid(k, t - 1), MV_QPEL, 0, -1, pslot(k, t)) for k in range(clips)])

    def learned_gop():
        for t in steps:
            for k in range(clips):
                net.prepare(fid(k, t), fid(k, t - 1), k)
            net.propose(0, clips)
            net.analyze(p, [(fid(k, t), fid(k, t - 1), k, MV_QPEL, lslot(k, t)) for k in range(clips)], fallback=True)

    ext = torch.cuda.ExternalStream(ctx.stream_handle())
    out = {}
    for name, gop in (("plain", plain_gop), ("learned", learned_gop)):
        gop()  # direct: builds the launches' tables and slots
        ctx.synchronize()
        ctx.graph_begin()
        gop()
        g = ctx.graph_end()
        ctx.graph_launch(g)
        ctx.synchronize()
        t = 0.0
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(ext)
            ctx.graph_launch(g)
            b.record(ext)
            b.synchronize()
            t += a.elapsed_time(b)
        ctx.graph_destroy(g)
        out[name] = t / reps
    # quality of every pair (the last replay's results)
    gaps, psnr_p, psnr_l = [], [], []
    levels = torch.empty((MBS, 6, 64), dtype=torch.int16, device="cuda")
    types = np.ones(MBS * 6, np.uint8)
    for k in range(clips):
        for t in steps:
            a, b = ctx.read_result(p, pslot(k, t)), ctx.read_result(p, lslot(k, t))
            sp, sl = float(a.screen_sads.astype(np.float64).sum()), float(b.screen_sads.astype(np.float64).sum())
            gaps.append((sl - sp) / max(sp, 1.0))
        for t in (1, frames - 1):
            cur = ctx.download_frame(fid(k, t), W, H)[0]
            for acc, slot in ((psnr_p, pslot(k, t)), (psnr_l, lslot(k, t))):
                ctx.motion_compensate(p, fid(k, t - 1), slot, MV_QPEL, 3900)
                ctx.forward_quant_device(p, fid(k, t), 3900, 1, 0, levels.data_ptr())
                ctx.reconstruct(p, 3900, levels.data_ptr(), 1, types, 3901)
                rec = ctx.download_frame(3901, W, H)[0]
                mse = np.mean((rec.astype(np.float64) - cur.astype(np.float64)) ** 2)
                acc.append(99.0 if mse == 0 else 10.0 * np.log10(255.0 ** 2 / mse))
    # fallback share of the last frame step (the network's per-sample flags)
    fb = sum(int(net.read_sample(k)[3].sum()) for k in range(clips))
    net.close()
    gaps = np.array(gaps)
    mb_gop = clips * len(steps) * MBS
    return {"workload": f"{clips} clips x {frames} frames 1920x1080, pans up to 200 px/frame horizontal and 60 vertical, "
                        "4 objects, sigma 2; search range 1024 (MVRANGE 3), local 32; ME + qpel per P picture; "
                        "every frame step's pictures of all clips in one batch; a CUDA graph per GOP",
            "mb_per_s_plain": round(mb_gop / (out["plain"] * 1e-3), 1),
            "mb_per_s_learned": round(mb_gop / (out["learned"] * 1e-3), 1),
            "speedup": round(out["plain"] / out["learned"], 3), "ms_per_gop_plain": round(out["plain"], 2),
            "ms_per_gop_learned": round(out["learned"], 2), "cost_gap_mean": round(float(gaps.mean()), 5),
            "cost_gap_p99": round(float(np.percentile(gaps, 99)), 5),
            "fallback_rate_last_step": round(fb / (clips * MBS), 4),
            "psnr_plain": round(float(np.mean(psnr_p)), 4), "psnr_learned": round(float(np.mean(psnr_l)), 4),
            "psnr_delta_db": round(float(np.mean(psnr_l) - np.mean(psnr_p)), 4),
            "psnr_sample": "QP-6 luma reconstruction of frame steps 1 and last of every clip"}


def transform_rd_leg(ctx, run, clip, pictures=4):
    """The default presets' transform RD (vc1cu_choose_transform: candidate types, trellis with
    the perceptual lambda scale, bit estimates, macroblock/block signaling) on the step's first
    P pictures against their final Mixed-MV predictions (frame slots the step left), through the
    C ABI with the decisions and levels copied back; and the reference's choose_transform_mb on
    one of those pictures on one host thread, compared bit for bit."""
    import time

    from libvc1_b200.abi import make_trd_cfg, tdecisions_differ

    cfg = make_trd_cfg()
    pics = run.pics[:pictures]
    ctx.choose_transform(params(pics[0][2]), cfg, pics[0][0], 3500)  # tables and buffers
    t0 = time.perf_counter()
    results = [ctx.choose_transform(params(pq), cfg, t, 3500 + i) for i, (t, _r, pq) in enumerate(pics)]
    dt = time.perf_counter() - t0
    out = {"workload": f"{len(pics)} 1080p P pictures of the step against their Mixed-MV predictions; trellis 1, "
                       "AQ strength 1, variable transforms with TTBLK signaling, coding set 1",
           "mb_per_s": round(len(pics) * MBS / dt, 1), "ms_per_picture": round(1e3 * dt / len(pics), 2),
           "timing": "wall clock of synchronous C-ABI calls, decisions and levels copied to the host"}
    try:
        from oracle import Reference, ref_available
    except Exception:  # pragma: no cover
        return out
    if not ref_available():
        return out
    t, _r, pq = pics[0]
    pred = ctx.download_frame(3500, W, H)
    R = Reference(params(pq), simd_auto=True)
    t0 = time.perf_counter()
    want, wlv = R.choose_transform(cfg, clip.frame(t), pred)
    dt_ref = time.perf_counter() - t0
    got, glv = results[0]
    out["reference_one_thread_mb_per_s"] = round(MBS / dt_ref, 1)
    out["matches_reference"] = tdecisions_differ(got, want) == [] and bool(np.array_equal(glv, wlv))
    return out


def mode_decision_leg(ctx, run, clip, pictures=4):
    """The P picture's whole motion-mode decision (vc1cu_analyze_p_picture: quarter-pel seed pass,
    three seeded mode passes, each candidate's motion bits and sampled transform RD, the final
    pass in the chosen mode, the fade estimate and, when it is enabled, the compensated candidates)
    on the step's first P pictures with the reference's default presets, through the C ABI; and
    the reference's analyze_p_picture on one of those pictures on one host thread, compared."""
    import time

    from libvc1_b200.abi import make_ppic_cfg

    cfg = make_ppic_cfg()
    pics = run.pics[:pictures]
    t, r, pq = pics[0]
    ctx.analyze_p_picture(params(pq), cfg, t, r, 3600, 3610, 3600)  # buffers and tuned shapes
    t0 = time.perf_counter()
    infos = [ctx.analyze_p_picture(params(pq), cfg, t, r, 3600 + i, 3610, 3600) for i, (t, r, pq) in enumerate(pics)]
    dt = time.perf_counter() - t0
    out = {"workload": f"{len(pics)} 1080p P pictures of the step against their references; the reference's default "
                       "presets (trellis 1, DQUANT on, variable transforms with TTBLK signaling, fade compensation)",
           "mb_per_s": round(len(pics) * MBS / dt, 1), "ms_per_picture": round(1e3 * dt / len(pics), 2),
           "modes": [int(i.mode) for i in infos], "weighted": [int(i.weighted) for i in infos],
           "timing": "wall clock of synchronous C-ABI calls (every pass, score and decision of the picture)"}
    try:
        from oracle import Reference, ref_available
    except Exception:  # pragma: no cover
        return out
    if not ref_available():
        return out
    t, r, pq = pics[0]
    R = Reference(params(pq), simd_auto=True)
    t0 = time.perf_counter()
    want, mode, ic, bits = R.analyze_p_picture_cfg(cfg, clip.frame(t), clip.frame(r))
    dt_ref = time.perf_counter() - t0
    got = ctx.read_result(params(pq), 3600)
    out["reference_one_thread_mb_per_s"] = round(MBS / dt_ref, 1)
    out["matches_reference"] = (got.equal(want) == [] and infos[0].mode == mode and bool(infos[0].weighted) == ic
                                and infos[0].motion_bits == bits)
    return out


def batched_clips(n_odd_seed=7):
    """The batched workload's 48 clips: (coded width, height, display width, height, seed):
    16 at 640x360, 16 at 1280x720, 8 at 1920x1080 and 8 of odd display sizes with widths in
    322..1918 and heights in 242..1078 (coded raster rounded up to even)."""
    rng = np.random.default_rng(n_odd_seed)
    out = [(640, 360, 640, 360)] * 16 + [(1280, 720, 1280, 720)] * 16 + [(1920, 1080, 1920, 1080)] * 8
    for _ in range(8):
        dw, dh = int(rng.integers(161, 960)) * 2 + 1, int(rng.integers(121, 540)) * 2 + 1  # odd, 323..1919
        dw, dh = min(dw, 1917), min(dh, 1077)
        out.append((dw + 1, dh + 1, dw, dh))
    return [c + (500 + k,) for k, c in enumerate(out)]


def batched_leg(ctx, torch, reps, frames=31):
    """The batched plain form: 48 clips of uneven size, every clip's P picture of a frame step
    analysed (quarter-pel seed pass, three seeded mode passes, final Mixed-MV pass with P-intra,
    search range 32, QP 8 uniform) in ONE persistent launch per frame step; the 30 frame steps of
    the GOP captured as one CUDA graph and replayed; the launch shape chosen by the autotuner.
    Bit-exactness per clip is what tests/test_gpu_multiclip.py checks."""
    from libvc1_b200 import synth
    from libvc1_b200.abi import make_params

    clips = batched_clips()
    params, mbs_step = [], 0
    for k, (w, h, dw, dh, seed) in enumerate(clips):
        cfg = synth.make_cfg(w, h, frames, seed, global_px=16.0, n_objects=4, obj_vel=3.0, sigma=2.0)
        for t0 in range(0, frames, 16):
            ctx.synth_frames(cfg, t0, min(16, frames - t0), 200 + 64 * k + t0)
        params.append(make_params(w, h, display_width=dw, display_height=dh, search_range=32, local_search_range=32,
                                  pqindex=8))
        mbs_step += ((w + 15) // 16) * ((h + 15) // 16)

    def step(t):
        ctx.core_passes_multi(*_batched_step_args(params, clips, t))

    ext = torch.cuda.ExternalStream(ctx.stream_handle())
    step(1)  # builds the launch's tables and slots
    ctx.synchronize()
    warps, blocks, tune_ms = ctx.autotune(*_batched_step_args(params, clips))

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(ext)
        fn()
        b.record(ext)
        b.synchronize()
        return a.elapsed_time(b)

    direct_ms = timed(lambda: [step(t) for t in range(1, frames)])
    ctx.graph_begin()
    for t in range(1, frames):
        step(t)
    g = ctx.graph_end()
    ctx.graph_launch(g)  # warm-up replay
    ctx.synchronize()
    graph_ms = sum(timed(lambda: ctx.graph_launch(g)) for _ in range(reps)) / reps
    ctx.graph_destroy(g)
    mb_gop = mbs_step * (frames - 1)
    return {"workload": "48 clips (16x 640x360, 16x 1280x720, 8x 1920x1080, 8 odd sizes 323-1917 x 243-1077), "
                        f"{frames - 1} P frames each, global +-16 px; P analysis (5 passes) per picture, range 32, QP 8",
            "mb_per_gop": mb_gop, "launches_per_frame_step": 1,
            "mb_per_s_graph": round(mb_gop / (graph_ms * 1e-3), 1), "mb_per_s_direct": round(mb_gop / (direct_ms * 1e-3), 1),
            "ms_per_gop_graph": round(graph_ms, 2), "ms_per_gop_direct": round(direct_ms, 2),
            "autotuned_shape": {"warps_per_block": warps, "blocks_per_sm": blocks or "occupancy limit",
                                "ms_per_launch": round(tune_ms, 3)}}


def _batched_step_args(params, clips, t=1):
    from libvc1_b200.abi import MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED, MV_QPEL

    plist, passes = [], []
    for k in range(len(clips)):
        cur, ref, base = 200 + 64 * k + t, 200 + 64 * k + t - 1, 2000 + 5 * k
        plist += [params[k]] * 5
        passes += [(cur, ref, MV_QPEL, 0, -1, base)]
        passes += [(cur, ref, m, 0, base, base + 1 + j) for j, m in enumerate((MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED))]
        passes += [(cur, ref, MV_MIXED, 1, base + 3, base + 4)]
    return plist, passes


def flush_l2(torch, buf):
    buf.zero_()
    torch.cuda.synchronize()


def run_ours(args, rank, world, device):
    import torch

    from libvc1_b200.api import CudaComputeContext
    from libvc1_b200.replicas import slowest, whole_job_rate

    torch.cuda.set_device(device)
    ctx, err = CudaComputeContext.create(device)
    if ctx is None:
        raise RuntimeError(f"CUDA backend unavailable: {err}")
    clip = make_clip(rank)
    run = Runner(ctx, clip, args.gops)
    run.upload_all()
    ext = torch.cuda.ExternalStream(ctx.stream_handle(), device=device)
    l2 = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    for _ in range(args.warmup):
        run.step()
    ctx.synchronize()
    shapes = None if args.no_autotune else run.tune()
    run.step()
    ctx.synchronize()
    # ---- value: resident inputs, device time per step, L2 flushed between steps
    ctx.reset_counters()
    ctx.set_timing(True)
    clock_log = os.path.join(tempfile.gettempdir(), f"vc1cu_clocks_{os.getpid()}.csv")
    sampler = sample_clocks(clock_log)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    step_ms = []
    stage_ms = {}
    for _ in range(args.steps):
        flush_l2(torch, l2)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        marks = []

        def mark(stage):
            e = torch.cuda.Event(enable_timing=True)
            e.record(ext)
            marks.append((stage, e))

        a.record(ext)
        run.step(mark=mark)
        b.record(ext)
        b.synchronize()
        step_ms.append(a.elapsed_time(b))
        prev = a
        for stage, e in marks:
            stage_ms[stage] = stage_ms.get(stage, 0.0) + prev.elapsed_time(e)
            prev = e
    ctx.synchronize()
    torch.cuda.synchronize()
    if sampler:
        sampler.terminate()
        sampler.wait()
    timing = ctx.timing()
    counters = ctx.counters()
    ctx.set_timing(False)
    total_ms = float(sum(step_ms))
    mbs_per_step = run.mbs_per_step()
    max_ms = 1e3 * slowest(total_ms * 1e-3, world, "cuda")
    value = whole_job_rate(mbs_per_step * args.steps, max_ms * 1e-3, world)
    clocks = parse_clocks(clock_log, device)
    # ---- e2e: pinned host frames -> upload -> analysis -> results back, wall clock
    pinned = {}
    for f in run.frames:
        y, u, v = clip.frame(f)
        pinned[f] = tuple(torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in (y, u, v))
    # Every step: upload the step's frames from pinned memory, analyse, read every P final-pass
    # and B analysis back, and copy all levels to pinned host memory. Steps are pipelined over
    # two sets of frame slots, result slots and level buffers, so the device always has the
    # next step queued: while step i computes, the library's upload stream brings step i+1's
    # frames and step i+1 is enqueued behind it; the host then collects step i's fade
    # estimates (waiting for step i alone), a copy stream moves step i's levels and the host
    # reads step i's results (each read waits only for the launch that wrote its slot), all
    # beside step i+1's compute. A run ends when its last step's results are read and its
    # levels have landed.
    lev = [run.levels, torch.empty_like(run.levels)]
    host_levels = [torch.empty(run.levels.shape, dtype=torch.int16).pin_memory() for _ in range(2)]
    copy_stream = torch.cuda.Stream()
    copied = [None, None]

    def copy_levels(b, after):
        copy_stream.wait_event(after)
        with torch.cuda.stream(copy_stream):
            host_levels[b].copy_(lev[b], non_blocking=True)
            copied[b] = torch.cuda.Event()
            copied[b].record(copy_stream)

    def start(i):
        """Enqueues step i (frames already uploaded into set i % 2) without waiting."""
        b = i % 2
        if copied[b] is not None:
            ext.wait_event(copied[b])  # the previous copy out of this level buffer is done
        with torch.cuda.stream(ext):
            l2.zero_()  # L2 flush between steps, on the library's stream
        run.launch(lev[b], b=b)  # waits on the device for its frames' uploads
        ticket = run.enqueue_ic(b)
        done = torch.cuda.Event()
        done.record(ext)
        return b, ticket, done

    def e2e_run(n):
        if not n:
            return
        run.upload_all(pinned, 0)
        cur = start(0)
        for i in range(n):
            b, ticket, done = cur
            if i + 1 < n:
                run.upload_all(pinned, 1 - b)  # step i+1's frames, beside step i's compute
                cur = start(i + 1)
            run.collect_ic(ticket)  # step i's fade estimates (waits for step i alone)
            copy_levels(b, done)  # step i's levels, beside step i+1's compute
            run.read_results(b)
        copy_stream.synchronize()
        ctx.synchronize()

    e2e_s = []
    if not args.no_e2e:
        e2e_run(args.warmup)
        flush_l2(torch, l2)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        t0 = time.perf_counter()
        e2e_run(args.steps)
        e2e_s.append(time.perf_counter() - t0)
    e2e_worst = slowest(sum(e2e_s), world, "cuda")
    e2e_value = world * mbs_per_step * args.steps / e2e_worst if e2e_s else None
    # ---- roofline of the dominant kernel (core_pass_kernel), INT32-bound
    n = len(run.pics)
    ops_step = n * MBS * sum(OPS_PER_MB[k] for k in P_PASSES) + len(run.bpics) * MBS * sum(OPS_PER_MB[k] for k in B_PASSES)
    core_launches = max(1, timing["core_launches"])
    core_ms = timing["core_ms"]
    achieved_ops = ops_step * args.steps / (core_ms * 1e-3) if core_ms > 0 else 0.0
    peak_ops = ctx.measure_int32_peak()
    peak_fp64 = ctx.measure_fp64_peak()
    xform_ms = timing["xform_ms"]
    xform_flops = n * MBS * XFORM_FLOPS_PER_MB * args.steps
    learned = None
    if not args.no_learned and world == 1:
        learned = learned_leg(ctx, torch, l2, args.steps, args.warmup)
    batched = None
    if not args.no_batched and world == 1:
        batched = batched_leg(ctx, torch, reps=min(args.steps, 2))
    longrange = None
    if not args.no_longrange and world == 1:
        longrange = longrange_leg(ctx, torch, reps=min(args.steps, 2))
    transform_rd = None
    if not args.no_transform_rd and world == 1:
        run.step()  # the step's predictions back in their frame slots
        ctx.synchronize()
        transform_rd = transform_rd_leg(ctx, run, clip)
    mode_decision = None
    if not args.no_mode_decision and world == 1:
        mode_decision = mode_decision_leg(ctx, run, clip)
    out = None
    if rank == 0:
        cpu = cpu_baseline(args, clip) if (world == 1 and not args.no_cpu_baseline) else None
        out = {
            "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(max_ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32 (integer SAD/SATD/interpolation) + f64 transform",
            "data": "synthetic (seeded value-noise clip with the 1080p config's motion, zoom, objects and noise)",
            "config": step_config(len(run.pics), len(run.bpics), world),
            "e2e": {"value": round(e2e_value, 1) if e2e_value else None, "unit": UNIT,
                    "h2d_bytes_per_step": len(run.frames) * run.frame_bytes,
                    "d2h_bytes_per_step": run.result_bytes()},
            "gpu_launches": counters["kernel_launches"],
            "roofline": {"bound": "int32", "kernel": "core_pass_kernel (+ its subpel_plane_kernel builds, timed with it)",
                         "achieved": round(achieved_ops / 1e9, 1),
                         "peak": round(peak_ops / 1e9, 1), "unit": "Gop/s (int32 lane ops)",
                         "frac": round(achieved_ops / peak_ops, 4) if peak_ops else None,
                         "peak_source": "measured live: vc1cu_measure_int32_peak add/xor kernel",
                         "ops_per_p_mb": round(sum(OPS_PER_MB[k] for k in P_PASSES), 1),
                         "ops_per_b_mb": round(sum(OPS_PER_MB[k] for k in B_PASSES), 1),
                         "core_ms_per_launch": round(core_ms / core_launches, 3),
                         "traffic": round(CORE_DRAM_BYTES_PER_LAUNCH) if args.gops is None else None,
                         "traffic_unit": "DRAM bytes per launch (ncu, first GOP scaled by macroblocks)"},
            "stage_ms_per_step": {k: round(v / args.steps, 3) for k, v in stage_ms.items()},
            "autotuned_shapes": shapes,
            "pass_mb_per_s": {
                "unseeded (P seed + B forward/backward)": round((len(run.pics) + 4 * len(run.bpics)) * MBS * args.steps
                                                              / (stage_ms["unseeded passes"] * 1e-3), 1),
                "seeded mode passes": round(3 * len(run.pics) * MBS * args.steps / (stage_ms["seeded mode passes"] * 1e-3), 1),
                "final Mixed-MV + intra": round(len(run.pics) * MBS * args.steps / (stage_ms["final passes"] * 1e-3), 1),
            } if stage_ms else None,
            "kernel_ms_per_step": {k: round(timing[k] / args.steps, 3)
                                   for k in ("core_ms", "global_ms", "totals_ms", "mc_ms", "xform_ms", "b_ms", "ic_ms")},
            "xform_roofline": xform_roofline(xform_flops, xform_ms, peak_fp64),
            "clocks": clocks,
            "cpu_baseline": cpu,
            "mpixel_per_s": round(value * 256 / 1e6, 1),
            "learned": learned,
            "batched": batched,
            "longrange": longrange,
            "transform_rd": transform_rd,
            "mode_decision": mode_decision,
        }
    ctx.close()
    return out


def reference_jobs(clip):
    """The reference's jobs of one step: P jobs (Reference at the picture's PQINDEX, cur, ref)
    and B jobs (Reference, cur, past, future, future anchor's P index, num, den)."""
    from oracle import Reference

    ps, bs = gop_plan()
    refs = {pq: Reference(params(pq), simd_auto=True) for pq in sorted({p[2] for p in ps} | {b[5] for b in bs})}
    any_ref = next(iter(refs.values()))
    frames = {}

    def fr(t):
        if t not in frames:
            frames[t] = any_ref.frame(clip.frame(t))
        return frames[t]

    pjobs = [(refs[pq], fr(t), fr(r)) for t, r, pq in ps]
    bjobs = [(refs[pq], fr(t), fr(past), fr(fut), a, num, den) for t, past, fut, num, den, pq, a in bs]
    return any_ref, pjobs, bjobs


REF_SAMPLE = ("every picture of the clip once (one step), the same work as the GPU arm on the reference's own "
              "functions: per P picture the five analyze_p_picture_core passes (qpel seed, hpel, bilinear, Mixed-MV, "
              "final Mixed-MV + P-intra), estimate_intensity_comp, the prediction and quantize_inter_part of all four "
              "transform types; per B picture analyze_b_picture_mode in qpel and bilinear mode; P and B pictures in one "
              "job pool (a B job waits for its anchor), one picture per thread, SIMD dispatch auto")
REF_FULL_RD = ("the reference's whole picture analysis instead: analyze_p_picture (sampled mode RD, final pass in the "
               "chosen mode) + choose_transform_mb RD of every MB, then analyze_b_picture (both modes + sampled B mode "
               "RD), P phase then B phase")


def xform_roofline(flops, ms, peak):
    """The transform kernel against the FP64 peak measured live (FMA kernel, an FMA counted as
    two flops). The transform rounds every product and sum separately (no contraction, for the
    reference's bits), so its instruction-rate ceiling is half the FMA peak."""
    if not ms or ms <= 0:
        return None
    achieved = flops / (ms * 1e-3)
    return {"bound": "fp64", "kernel": "xform_kernel", "achieved_gflops": round(achieved / 1e9, 1),
            "peak_gflops": round(peak / 1e9, 1) if peak else None,
            "frac": round(achieved / peak, 4) if peak else None,
            "frac_of_unfused_ceiling": round(2 * achieved / peak, 4) if peak else None,
            "peak_source": "measured live: vc1cu_measure_fp64_peak FMA kernel"}


def step_config(n_p, n_b, world):
    """The workload's config block, the same in both arms' lines."""
    return {"workload": WORKLOAD, "mb_per_step_per_gpu": (n_p + n_b) * MBS, "p_pictures": n_p, "b_pictures": n_b,
            "core_passes_per_step": 5 * n_p + 4 * n_b,
            "l2": "inputs larger than L2 (60 frames x 3.1 MB read per step); the GPU arm also flushes L2 (256 MB "
                  "write) between timed steps",
            "parallelism": f"replicas x{world}"}


def cpu_baseline(args, clip):
    """The reference's own CPU path (oracle/_ref, SIMD dispatch on) over a bounded sample of
    the same workload: every picture of the clip once, one picture per host thread."""
    try:
        from oracle import ref_available
    except Exception as e:  # pragma: no cover
        return {"unavailable": f"oracle import failed: {e}"}
    if not ref_available():
        return {"unavailable": "oracle/_ref/libvc1ref.so not built"}
    cores = os.cpu_count() or 1
    anyref, pjobs, bjobs = reference_jobs(clip)
    threads = min(len(pjobs) + len(bjobs), cores)
    ns = anyref.bench_gop_same(pjobs, bjobs, threads)
    out = {"value": round((len(pjobs) + len(bjobs)) * MBS / (ns * 1e-9), 1), "unit": UNIT, "cores": threads,
           "kind": "reference", "sample": REF_SAMPLE}
    ns_rd = anyref.bench_gop_multi(pjobs, bjobs, threads)
    out["full_rd"] = {"value": round((len(pjobs) + len(bjobs)) * MBS / (ns_rd * 1e-9), 1), "unit": UNIT,
                      "sample": REF_FULL_RD}
    # one core: the first P picture and the first B picture anchored on it, with the SIMD dispatch
    # on and with the scalar path (the reference's parity configuration)
    from oracle import Reference

    one = {}
    for name, simd in (("simd_auto", True), ("simd_none", False)):
        R = Reference(params(pjobs[0][0].p.pqindex), simd_auto=simd)
        pj = [(R, pjobs[0][1], pjobs[0][2])]
        bj = [(R,) + tuple(bjobs[0][1:])]
        ns1 = R.bench_gop_same(pj, bj, 1)
        one[name] = round(2 * MBS / (ns1 * 1e-9), 1)
    out["one_thread"] = dict(one, sample="P picture 3 and B picture 1 of the clip on one host thread")
    return out


def run_reference(args, rank, world):
    if rank != 0:
        return None
    try:
        from oracle import ref_available
    except Exception as e:
        return {"impl": "reference", "unavailable": f"oracle package import failed: {e}"}
    if not ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libvc1ref.so was not built (reference tree absent)"}
    clip = make_clip(0)
    cores = os.cpu_count() or 1
    anyref, pjobs, bjobs = reference_jobs(clip)
    threads = min(len(pjobs) + len(bjobs), cores)
    per = []
    for i in range(args.warmup + args.steps):
        ns = anyref.bench_gop_same(pjobs, bjobs, threads)
        if i >= args.warmup:
            per.append(ns * 1e-9)
    value = (len(pjobs) + len(bjobs)) * MBS * len(per) / sum(per)
    return {"metric": METRIC, "value": round(value, 1), "unit": UNIT, "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * sum(per) / len(per), 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32 + f64 (CPU)",
            "data": "synthetic (same seeded clip as ours)",
            "config": step_config(len(pjobs), len(bjobs), world),
            "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": REF_SAMPLE},
            "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-proposal leg")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched multi-clip leg")
    ap.add_argument("--no-longrange", action="store_true", help="skip the long-range pan leg")
    ap.add_argument("--no-transform-rd", action="store_true", help="skip the transform RD leg")
    ap.add_argument("--no-mode-decision", action="store_true", help="skip the P motion-mode decision leg")
    ap.add_argument("--no-autotune", action="store_true", help="default launch shapes (no autotuning)")
    ap.add_argument("--gops", type=int, default=None, help="analyse only the pictures of the first N GOPs (profiling)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        # the reference's CPU path runs on rank 0 alone; other ranks exit without work
        out = run_reference(args, rank, world)
        if out is not None and rank == 0:
            print(json.dumps(out), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    out = run_ours(args, rank, world, local)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if out is not None and rank == 0:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
