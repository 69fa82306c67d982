#!/usr/bin/env python
"""Encoder-analysis throughput of libvc1's P-picture hot path on B200, in macroblocks/s.

Workload (the 1080p configuration): 1920x1080 8-bit 4:2:0, 60 seeded synthetic frames
(value-noise texture, zoom 1.002/frame, 8 objects at up to 8 px/frame, sigma 2), GOP 12
IBBP, so 15 P pictures per clip, each analysed against the previous anchor (3 frames back)
with search range +/-64, Mixed-MV, non-uniform quantiser at QP 4/6/8/10/12 (one per GOP).

One step = every P picture of the clip fully analysed: the quarter-pel seed pass, the three
seeded mode passes (half-pel, half-pel bilinear, Mixed-MV), the final Mixed-MV pass with
P-intra, the decoder-equivalent prediction, and the forward transform + quantiser of that
prediction for all four transform sizes (Vc1Encoder::analyze_p_picture_core x5 and
quantize_inter_part, src/encoder_motion.cpp:47-597, src/encoder_transform.cpp:935-1171).
The final pass is timed in Mixed-MV mode, the most expensive of the reference's four
candidates (the reference chooses it on the host by sampled RD).

  value : MB/s with the clip resident in HBM (CUDA events on the library's stream, L2
          flushed between steps)
  e2e   : MB/s through the C ABI from pinned host frames, including the H2D upload of the
          step's frames and the D2H read of every result (MVs, decisions, levels)
  --impl reference : the reference's own CPU code (oracle/_ref, SIMD dispatch on) on the
          host's cores, same workload and unit

Multi-GPU: one process per GPU (torchrun); each rank analyses its own clip (seeded by
rank), no collective on the data path; value = all ranks' MBs / max rank time.
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
# instrumented oracle (oracle/count_ops.py over two P pictures of the clip; weights there).
OPS_PER_MB = {"unseeded": 286531.9, "seeded_hpel": 56280.0, "seeded_bilinear": 25312.1, "seeded_mixed": 474288.5,
              "final_mixed_intra": 474771.4}
XFORM_FLOPS_PER_MB = 51911.5


def anchors_and_pictures():
    """(P frame, reference anchor, PQINDEX) of GOP 12 IBBP over FRAMES frames."""
    pics = []
    for t in range(0, FRAMES, BFRAMES + 1):
        if t % GOP == 0:
            continue  # I picture
        pics.append((t, t - (BFRAMES + 1), 4 + 2 * ((t // GOP) % 5)))
    return pics


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

    def __init__(self, ctx, clip, pictures=None):
        from libvc1_b200.abi import MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED, MV_QPEL

        self.ctx, self.clip = ctx, clip
        self.pics = anchors_and_pictures()[:pictures]
        self.frames = sorted({f for p in self.pics for f in p[:2]})
        self.p0 = params(8)
        self.modes = (MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED)
        self.QPEL, self.MIXED = MV_QPEL, MV_MIXED
        import torch

        self.torch = torch
        n = len(self.pics)
        # device-side levels of every picture: [pic][type][mb][parent][64] int16
        self.levels = torch.empty((n, 4, MBS, 6, 64), dtype=torch.int16, device="cuda")
        self.frame_bytes = W * H * 3 // 2

    def upload_all(self, pinned=None):
        for f in self.frames:
            if pinned is None:
                self.ctx.upload_frame(f, *self.clip.frame(f))
            else:
                y, u, v = pinned[f]
                self.ctx.upload_frame_ptr(f, y.data_ptr(), u.data_ptr(), v.data_ptr(), W, H)

    def step(self, levels=None):
        """Enqueues one step on the library's stream; levels go to `levels` (default self.levels)."""
        levels = self.levels if levels is None else levels
        c, pics = self.ctx, self.pics
        # every picture's quarter-pel seed pass (full search window per warp)
        c.core_passes(self.p0, [(t, r, self.QPEL, 0, -1, 1000 + i, pq) for i, (t, r, pq) in enumerate(pics)])
        # the three seeded mode passes of every picture (the library runs one launch per mode)
        c.core_passes(self.p0, [(t, r, m, 0, 1000 + i, 2000 + 4 * i + m, pq) for i, (t, r, pq) in enumerate(pics)
                                for m in self.modes])
        # the final pass (after the host's mode decision over whole passes)
        c.core_passes(self.p0, [(t, r, self.MIXED, 1, 2000 + 4 * i + self.MIXED, 3000 + i, pq)
                                for i, (t, r, pq) in enumerate(pics)])
        for i, (t, r, pq) in enumerate(pics):
            p = params(pq)
            c.motion_compensate(p, r, 3000 + i, self.MIXED, 3500 + i)
            c.forward_quant_device(p, t, 3500 + i, 15, 0, levels[i].data_ptr())

    def read_results(self):
        """D2H of the final-pass analysis of every picture (waits for the step)."""
        return [self.ctx.read_result(self.p0, 3000 + i) for i in range(len(self.pics))]

    def result_bytes(self):
        per_mb = 8 + 32 + 1 + 1 + 8 + 8 + 8 + 8 + 1
        return len(self.pics) * (MBS * per_mb) + self.levels.numel() * 2


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
    run = Runner(ctx, clip, args.pictures)
    run.upload_all()
    ext = torch.cuda.ExternalStream(ctx.stream_handle(), device=device)
    l2 = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    for _ in range(args.warmup):
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
    for _ in range(args.steps):
        flush_l2(torch, l2)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(ext)
        run.step()
        b.record(ext)
        b.synchronize()
        step_ms.append(a.elapsed_time(b))
    ctx.synchronize()
    torch.cuda.synchronize()
    if sampler:
        sampler.terminate()
        sampler.wait()
    timing = ctx.timing()
    counters = ctx.counters()
    ctx.set_timing(False)
    total_ms = float(sum(step_ms))
    mbs_per_step = len(run.pics) * MBS
    max_ms = 1e3 * slowest(total_ms * 1e-3, world, "cuda")
    value = whole_job_rate(mbs_per_step * args.steps, max_ms * 1e-3, world)
    clocks = parse_clocks(clock_log, device)
    # ---- e2e: pinned host frames -> upload -> analysis -> results back, wall clock
    pinned = {}
    for f in run.frames:
        y, u, v = clip.frame(f)
        pinned[f] = tuple(torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in (y, u, v))
    # Every step: upload the step's frames from pinned memory, analyse, read the final-pass
    # analysis back, and copy all levels to pinned host memory. The level copy of step i runs
    # on a copy stream while step i+1 computes (two level buffers); the timed region ends
    # when the last step's copy has landed.
    lev = [run.levels, torch.empty_like(run.levels)]
    host_levels = [torch.empty(run.levels.shape, dtype=torch.int16).pin_memory() for _ in range(2)]
    copy_stream = torch.cuda.Stream()
    copied = [None, None]
    e2e_s = []
    n_e2e = 0 if args.no_e2e else args.warmup + args.steps
    t0 = None
    for i in range(n_e2e):
        if i == args.warmup:
            copy_stream.synchronize()
            ctx.synchronize()
            flush_l2(torch, l2)
            if world > 1:
                torch.distributed.barrier()
            t0 = time.perf_counter()
        b = i % 2
        if copied[b] is not None:
            ext.wait_event(copied[b])  # the previous copy out of this buffer is done
        with torch.cuda.stream(ext):
            l2.zero_()  # L2 flush between steps, on the library's stream
        run.upload_all(pinned)
        run.step(lev[b])
        done = torch.cuda.Event()
        done.record(ext)
        copy_stream.wait_event(done)
        with torch.cuda.stream(copy_stream):
            host_levels[b].copy_(lev[b], non_blocking=True)
            copied[b] = torch.cuda.Event()
            copied[b].record(copy_stream)
        run.read_results()
    if n_e2e:
        copy_stream.synchronize()
        ctx.synchronize()
        e2e_s.append(time.perf_counter() - t0)
    e2e_worst = slowest(sum(e2e_s), world, "cuda")
    e2e_value = world * mbs_per_step * args.steps / e2e_worst if e2e_s else None
    # ---- roofline of the dominant kernel (core_pass_kernel), INT32-bound
    n = len(run.pics)
    ops_step = n * MBS * (OPS_PER_MB["unseeded"] + OPS_PER_MB["seeded_hpel"] + OPS_PER_MB["seeded_bilinear"] +
                          OPS_PER_MB["seeded_mixed"] + OPS_PER_MB["final_mixed_intra"])
    core_launches = max(1, timing["core_launches"])
    core_ms = timing["core_ms"]
    achieved_ops = ops_step * args.steps / (core_ms * 1e-3) if core_ms > 0 else 0.0
    peak_ops = ctx.measure_int32_peak()
    xform_ms = timing["xform_ms"]
    xform_flops = n * MBS * XFORM_FLOPS_PER_MB * args.steps
    out = None
    if rank == 0:
        cpu = cpu_baseline(args, clip) if (world == 1 and not args.no_cpu_baseline) else None
        out = {
            "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(max_ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32 (integer SAD/SATD/interpolation) + f64 transform",
            "data": "synthetic (seeded value-noise clip with the 1080p config's motion, zoom, objects and noise)",
            "config": {"workload": "1080p P-picture analysis: 1920x1080 4:2:0, 60 frames, GOP 12 IBBP -> 15 P "
                                   "pictures/step, search +/-64, Mixed-MV, nonuniform QP 4-12, 4 transform sizes",
                       "mb_per_step_per_gpu": mbs_per_step, "passes_per_picture": 5,
                       "l2": "flushed between timed steps (256 MB write)", "parallelism": f"replicas x{world}"},
            "e2e": {"value": round(e2e_value, 1) if e2e_value else None, "unit": UNIT,
                    "h2d_bytes_per_step": len(run.frames) * run.frame_bytes,
                    "d2h_bytes_per_step": run.result_bytes()},
            "gpu_launches": counters["kernel_launches"],
            "roofline": {"bound": "int32", "kernel": "core_pass_kernel", "achieved": round(achieved_ops / 1e9, 1),
                         "peak": round(peak_ops / 1e9, 1), "unit": "Gop/s (int32 lane ops)",
                         "frac": round(achieved_ops / peak_ops, 4) if peak_ops else None,
                         "peak_source": "measured live: vc1cu_measure_int32_peak add/xor kernel",
                         "ops_per_mb": round(sum(OPS_PER_MB.values()), 1),
                         "core_ms_per_launch": round(core_ms / core_launches, 3), "traffic": None},
            "kernel_ms_per_step": {k: round(timing[k] / args.steps, 3)
                                   for k in ("core_ms", "global_ms", "totals_ms", "mc_ms", "xform_ms")},
            "xform_roofline": {"bound": "fp64", "achieved_gflops": round(xform_flops / (xform_ms * 1e-3) / 1e9, 1)
                               if xform_ms > 0 else None},
            "clocks": clocks,
            "cpu_baseline": cpu,
            "mpixel_per_s": round(value * 256 / 1e6, 1),
        }
    ctx.close()
    return out


def reference_jobs(clip, pics):
    """One (Reference, cur, ref) job per P picture, each encoder at the picture's PQINDEX."""
    from oracle import Reference

    refs = {pq: Reference(params(pq), simd_auto=True) for pq in sorted({p[2] for p in pics})}
    any_ref = next(iter(refs.values()))
    jobs = [(refs[pq], any_ref.frame(clip.frame(t)), any_ref.frame(clip.frame(r))) for t, r, pq in pics]
    return any_ref, jobs


def cpu_baseline(args, clip):
    """The reference's own CPU path (oracle/_ref, SIMD dispatch on) over a bounded sample of
    the same workload: every P picture of the clip once, one picture per host thread."""
    try:
        from oracle import ref_available
    except Exception as e:  # pragma: no cover
        return {"unavailable": f"oracle import failed: {e}"}
    if not ref_available():
        return {"unavailable": "oracle/_ref/libvc1ref.so not built"}
    pics = anchors_and_pictures()
    cores = os.cpu_count() or 1
    anyref, jobs = reference_jobs(clip, pics)
    threads = min(len(jobs), cores)
    ns = anyref.bench_analysis_multi(jobs, threads)
    return {"value": round(len(jobs) * MBS / (ns * 1e-9), 1), "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"{len(jobs)} P pictures of the 1080p clip (one step), one per thread: analyze_p_picture + "
                      f"choose_transform_mb of the chosen prediction, SIMD dispatch auto"}


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
    pics = anchors_and_pictures()
    cores = os.cpu_count() or 1
    anyref, jobs = reference_jobs(clip, pics)
    threads = min(len(jobs), cores)
    per = []
    for i in range(args.warmup + args.steps):
        ns = anyref.bench_analysis_multi(jobs, threads)
        if i >= args.warmup:
            per.append(ns * 1e-9)
    value = len(jobs) * MBS * len(per) / sum(per)
    return {"metric": METRIC, "value": round(value, 1), "unit": UNIT, "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * sum(per) / len(per), 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32 + f64 (CPU)",
            "data": "synthetic (same seeded clip as ours)",
            "config": {"workload": "1080p P-picture analysis: 1920x1080 4:2:0, 60 frames, GOP 12 IBBP -> 15 P "
                                   "pictures/step, search +/-64, Mixed-MV, nonuniform QP 4-12, 4 transform sizes"},
            "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": "every P picture of the clip per step, one per thread: analyze_p_picture + "
                                       "choose_transform_mb, SIMD dispatch auto"},
            "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    ap.add_argument("--pictures", type=int, default=None, help="analyse only the first N P pictures (profiling)")
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
