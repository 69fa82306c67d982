"""Regenerates the golden vectors in this directory from the reference's own code.

The vectors are outputs of libvc1 v0.2.69 itself: oracle/_ref/libvc1ref.so is compiled from
the reference sources by oracle/Makefile (`make -C oracle ref`, scalar SIMD tiers), and this
script calls it through oracle.Reference on inputs restated from the reference's tests:

  runtime_kat.npz   tests/vulkan_compute_runtime.cpp:17-98 (48x40 LCG frames, 20 quarter-pel
                    vectors: SAD/SATD at (5,7), bilinear SAD at (3,4), sampled integer SAD)
  staged_kat.npz    tests/staged_motion_estimation.cpp:26-39 (flat vs noisy residual) and
                    :134-147 (32x32 LCG pair, SATD over a quarter-pel and a bilinear grid)
  diamond_kat.npz   tests/diamond_motion.cpp:8-60 (gradient shifts, cropped-edge legality)
  analysis_*.npz    analyze_p_core chains (quarter-pel seed pass, three seeded mode passes,
                    final Mixed-MV pass with P-intra) on seeded synthetic pictures
  xform_kat.npz     forward transform + quantiser of a motion-compensated prediction
  global_kat.npz    whole-frame translation search and frame SADs
  ic_kat.npz        estimate_intensity_comp along each picture's quarter-pel field on seeded
                    synthetic fades, and (small pictures) intensity_compensated_reference with
                    the estimate and fixed LUMSCALE/LUMSHIFT codes covering the LUMSCALE 0 law
  recon_kat.npz     the reconstruction of xform_kat's pictures (levels of all four types, a
                    seeded transform type per block) and of seeded random levels, through the
                    reference's inverse_partition
  lf_kat.npz        the reference's apply_i_like_loop_filter and apply_p_loop_filter of blocky
                    seeded pictures with seeded coded-block metadata (tests/lf_cases.py), at
                    four PQINDEX values, dense 4-MV and 1-MV fields
  tt_kat.npz        the transform type choose_transform_mb picks with the throughput preset for
                    noisy seeded pictures against a quarter-pel prediction (cropped rasters
                    included, every type reached)
  scene_kat.npz     scene_change_score on seeded pictures: motion, a cut (two thresholds),
                    a fade with and without fade compensation, two camera zooms that the
                    local-motion fit rescues, and search range 0
  b_kat.npz         analyze_b_picture_mode (two core passes + the per-MB B mode decision) of a
                    seeded three-picture group, anchor vectors from the future picture's own
                    Mixed-MV analysis, several fractions, modes and parameter sets, and the
                    B prediction of each analysis (motion_compensate_mb / _bi_mb, intra means)

Run it where the reference tree is present (it is not needed to run the tests):
    python tests/golden/make_golden.py            # every fixture
    python tests/golden/make_golden.py b_kat      # only the named ones
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from libvc1_b200 import synth  # noqa: E402
from libvc1_b200.abi import MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED, MV_QPEL, make_params  # noqa: E402

RUNTIME_MVS = [(0, 0), (4, 0), (-4, 0), (0, 4), (0, -4), (3, 1), (-3, 2), (7, -5), (-9, -7), (12, 8), (-16, 11),
               (1, 3), (2, 2), (-1, -3), (20, -12), (-23, 17), (31, 29), (-32, -27), (5, -19), (-21, 6)]

# analysis fixtures: name -> (clip factory, params)
ANALYSIS = {
    "cif_r8": (lambda: synth.cif_plain(frames=2, seed=1), dict(search_range=8, local_search_range=8)),
    "odd_322x242": (lambda: synth.generate(322, 242, 2, 4),
                    dict(display_width=321, display_height=241, search_range=16, local_search_range=16, rnd=1,
                         pqindex=12, nonuniform=1)),
}


def planes(y, chroma=128):
    h, w = y.shape
    u = np.full((h // 2, w // 2), chroma, np.uint8)
    return (np.ascontiguousarray(y, np.uint8), u, u.copy())


def runtime_frames():
    x = np.arange(48)[None, :]
    y = np.arange(40)[:, None]
    cur = ((x * 13 + y * 29 + (x * y) % 37 + 17) & 255).astype(np.uint8)
    ref = ((x * 7 + y * 19 + (x * y) % 53 + 61) & 255).astype(np.uint8)
    return planes(cur), planes(ref)


def integer_sampled_sad(cur, ref, x0, y0, bw, bh, dx, dy, stride):
    """The reference test's own helper (tests/vulkan_compute_runtime.cpp:17-29)."""
    H, W = cur.shape
    aw, ah = max(0, min(bw, W - x0)), max(0, min(bh, H - y0))
    s = 0
    for y in range(0, ah, stride):
        for x in range(0, aw, stride):
            rx = min(max(x0 + x + dx, 0), W - 1)
            ry = min(max(y0 + y + dy, 0), H - 1)
            s += abs(int(cur[y0 + y, x0 + x]) - int(ref[ry, rx]))
    return s * stride * stride


def lcg_bytes(n, state, twice=False):
    out = np.zeros(n, np.uint8)
    out2 = np.zeros(n, np.uint8)
    for i in range(n):
        state = (state * 1664525 + 1013904223) & 0xFFFFFFFF
        out[i] = state >> 24
        if twice:
            state = (state * 1664525 + 1013904223) & 0xFFFFFFFF
            out2[i] = state >> 24
    return out, out2


def staged_frames():
    cur = np.full((16, 16), 128, np.uint8)
    flat = np.full((16, 16), 127, np.uint8)
    noisy = np.zeros(256, np.uint8)
    state = 1
    for i in range(256):
        state = (state * 1664525 + 1013904223) & 0xFFFFFFFF
        noisy[i] = 127 if state & 0x80000000 else 129
    c32, r32 = lcg_bytes(32 * 32, 7, twice=True)
    return cur, flat, noisy.reshape(16, 16), c32.reshape(32, 32), r32.reshape(32, 32)


def gradient(w, h, horizontal):
    x = np.arange(w)[None, :].repeat(h, 0)
    y = np.arange(h)[:, None].repeat(w, 1)
    return (20 + 3 * (x if horizontal else y)).astype(np.uint8)


def shifted(ref, sx, sy):
    h, w = ref.shape
    yy = np.clip(np.arange(h) + sy, 0, h - 1)
    xx = np.clip(np.arange(w) + sx, 0, w - 1)
    return ref[yy][:, xx]


def analysis_chain(run_pass, p, cur, ref):
    """qseed, the three seeded mode passes, final Mixed-MV + intra: {pass name: Analysis}."""
    out = {}
    q = run_pass(p, cur, ref, MV_QPEL, False, None, None)
    out["qpel"] = q
    for m, name in ((MV_HPEL, "hpel"), (MV_HPEL_BILINEAR, "bilinear"), (MV_MIXED, "mixed")):
        out[name] = run_pass(p, cur, ref, m, False, q.mvs, q)
    out["final"] = run_pass(p, cur, ref, MV_MIXED, True, out["mixed"].mvs, out["mixed"])
    return out


def flatten(prefix, a, d):
    for name in a.ARRAYS:
        d[f"{prefix}.{name}"] = getattr(a, name)
    for k, v in a.totals.items():
        d[f"{prefix}.total.{k}"] = np.array(v)


# B-picture fixtures: (mode, fraction_num, fraction_den, params)
B_CASES = (
    (MV_QPEL, 1, 2, dict(display_width=125, display_height=93, search_range=16, local_search_range=16)),
    (MV_HPEL_BILINEAR, 1, 3, dict(display_width=125, display_height=93, search_range=16, local_search_range=16)),
    (MV_QPEL, 2, 3, dict(search_range=16, local_search_range=16, rnd=1, pqindex=20)),
    (MV_HPEL, 1, 2, dict(display_width=125, display_height=93, search_range=24, local_search_range=8)),
    (MV_MIXED, 1, 3, dict(search_range=16, local_search_range=16, pqindex=3)),
    (MV_QPEL, 1, 2, dict(search_range=16, local_search_range=16, disable_b_intra=1)),
)


def make_b_kat():
    from oracle import Reference

    clip = synth.generate(130, 98, 3, 15)
    past, cur, fut = clip.frame(0), clip.frame(1), clip.frame(2)
    d = {}
    for c, pl in zip("yuv", past):
        d[f"past.{c}"] = pl
    for c, pl in zip("yuv", cur):
        d[f"cur.{c}"] = pl
    for c, pl in zip("yuv", fut):
        d[f"future.{c}"] = pl
    p0 = make_params(130, 98, search_range=16, local_search_range=16)
    R = Reference(p0)
    rp, rf = R.frame(past), R.frame(fut)
    q = R.analyze_p_core(rf, rp, MV_QPEL, False)
    anc = R.analyze_p_core(rf, rp, MV_MIXED, True, seed=q.mvs, seed_distant=q)
    d["anchor.mvs"], d["anchor.use_4mv"] = anc.mvs, anc.use_4mv
    for i, (mode, num, den, kw) in enumerate(B_CASES):
        p = make_params(130, 98, **kw)
        R = Reference(p)
        b = R.analyze_b(R.frame(cur), R.frame(past), R.frame(fut), anc.mvs, anc.use_4mv, num, den, mode)
        flatten(f"b{i}", b, d)
        for c, pl in zip("yuv", R.b_predict(R.frame(cur), R.frame(past), R.frame(fut), b, mode)):
            d[f"b{i}.pred.{c}"] = pl
    np.savez_compressed(os.path.join(HERE, "b_kat.npz"), **d)


# intensity fixtures: (width, height, seed, fade scale, fade offset, params)
IC_CASES = (
    (98, 66, 1, 0.8, 10.0, dict(search_range=16, local_search_range=16)),
    (130, 98, 2, 1.2, -20.0, dict(display_width=125, display_height=93, search_range=16, local_search_range=16)),
    (352, 288, 4, 0.6, 30.0, dict(search_range=16, local_search_range=16)),
    (66, 50, 5, 1.0, 0.0, dict(search_range=8, local_search_range=8)),
    (16, 16, 6, 0.9, 5.0, dict(search_range=8, local_search_range=8)),
)
IC_FIXED = ((1, 0, 5), (1, 0, 40), (1, 63, 60), (1, 17, 33), (0, 0, 0))


def make_ic_kat():
    from oracle import Reference

    d = {}
    for i, (w, h, seed, a, b, kw) in enumerate(IC_CASES):
        clip = synth.generate(w, h, 2, seed)
        ref, cur = clip.frame(0), synth.fade(clip.frame(1), a, b, seed)
        p = make_params(w, h, **kw)
        R = Reference(p)
        rc, rr = R.frame(cur), R.frame(ref)
        q = R.analyze_p_core(rc, rr, MV_QPEL, False)
        for c, pl in zip("yuv", ref):
            d[f"c{i}.ref.{c}"] = pl
        for c, pl in zip("yuv", cur):
            d[f"c{i}.cur.{c}"] = pl
        d[f"c{i}.mvs"] = q.mvs
        ic = R.estimate_intensity_comp(rc, rr, q.mvs)
        d[f"c{i}.ic"] = np.array(ic, np.int32)
        if w * h > 130 * 98:
            continue  # the mapped planes of the small pictures cover the law; keep the file small
        for j, k in enumerate((ic,) + IC_FIXED):
            for c, pl in zip("yuv", R.intensity_compensate(rr, k)):
                d[f"c{i}.map{j}.{c}"] = pl
    np.savez_compressed(os.path.join(HERE, "ic_kat.npz"), **d)


def make_recon_kat():
    from oracle import Oracle, Reference

    g = np.load(os.path.join(HERE, "xform_kat.npz"))
    cur = tuple(np.ascontiguousarray(g[f"cur.{c}"]) for c in "yuv")
    d = {}
    for pq, nu, hq in ((3, 0, 1), (8, 1, 1), (17, 1, 0), (31, 0, 0)):
        key = f"pq{pq}_nu{nu}_hq{hq}"
        p = make_params(64, 48, pqindex=pq, nonuniform=nu, halfqp=hq, search_range=8, local_search_range=8)
        R = Reference(p)
        pred = tuple(np.ascontiguousarray(g[f"{key}.pred.{c}"]) for c in "yuv")
        _co, lv = Oracle().forward_quant(p, cur, pred, 15)
        rng = np.random.default_rng(pq)
        types = rng.integers(1, 5, (lv.shape[1], 6)).astype(np.uint8)
        rand = (rng.integers(-60, 61, lv.shape) * (rng.random(lv.shape) < 0.1)).astype(np.int16)
        rand[..., 0] = rng.integers(-400, 401, rand.shape[:-1])
        d[f"{key}.types"], d[f"{key}.random_levels"] = types, rand
        for name, levels in (("coded", lv), ("random", rand)):
            for c, pl in zip("yuv", R.reconstruct(R.frame(pred), levels, 15, types)):
                d[f"{key}.{name}.{c}"] = pl
    np.savez_compressed(os.path.join(HERE, "recon_kat.npz"), **d)


LF_CASES = ((98, 66, 1, 8, True), (130, 98, 2, 20, False), (66, 50, 3, 3, True), (194, 146, 4, 31, True))


def make_lf_kat():
    from oracle import Reference

    sys.path.insert(0, os.path.dirname(HERE))
    from lf_cases import blocky_frame, metadata

    d = {}
    for i, (w, h, seed, pq, dense) in enumerate(LF_CASES):
        R = Reference(make_params(w, h, pqindex=pq))
        fr = blocky_frame(w, h, seed)
        for c, pl in zip("yuv", fr):
            d[f"c{i}.in.{c}"] = pl
        for c, pl in zip("yuv", R.loop_filter(fr)):
            d[f"c{i}.i.{c}"] = pl
        bmv, cbp, tt, intra = metadata(w, h, seed, dense)
        d[f"c{i}.bmv"], d[f"c{i}.cbp"], d[f"c{i}.tt"], d[f"c{i}.intra"] = bmv, cbp, tt, intra
        for c, pl in zip("yuv", R.loop_filter(fr, bmv, cbp, tt, intra)):
            d[f"c{i}.p.{c}"] = pl
    np.savez_compressed(os.path.join(HERE, "lf_kat.npz"), **d)


TT_CASES = ((98, 66, 1, 4, 30), (130, 98, 2, 12, 8), (322, 242, 4, 6, 25), (16, 16, 5, 1, 60), (354, 290, 6, 3, 50),
            (98, 66, 7, 10, 0))


def make_tt_kat():
    from oracle import Oracle, Reference

    d = {}
    for i, (w, h, seed, pq, noise) in enumerate(TT_CASES):
        clip = synth.generate(w, h, 2, seed)
        p = make_params(w, h, search_range=8, local_search_range=8, pqindex=pq)
        R = Reference(p)
        cur, ref = clip.frame(1), clip.frame(0)
        rng = np.random.default_rng(seed)
        cur = tuple(np.clip(pl.astype(int) + rng.integers(-noise, noise + 1, pl.shape), 0, 255).astype(np.uint8)
                    for pl in cur)
        q = R.analyze_p_core(R.frame(cur), R.frame(ref), MV_QPEL, False)
        pred = R.motion_compensate(R.frame(ref), q, MV_QPEL)
        d[f"c{i}.cur"], d[f"c{i}.pred"] = cur[0], pred[0]
        d[f"c{i}.types"] = R.fast_transform_types(R.frame(cur), R.frame(pred))
    np.savez_compressed(os.path.join(HERE, "tt_kat.npz"), **d)


def make_scene_kat():
    from oracle import Reference

    sys.path.insert(0, os.path.dirname(HERE))
    from scene_cases import scene_pictures

    d = {}
    for name, (cur, ref, fade, thr, kw) in scene_pictures().items():
        h, w = cur[0].shape
        R = Reference(make_params(w, h, **kw))
        d[f"{name}.score"] = np.float64(R.scene_change_score(R.frame(cur), R.frame(ref), fade, thr))
    np.savez_compressed(os.path.join(HERE, "scene_kat.npz"), **d)


def make_ovl_kat():
    """Overlap smoothing by the reference: apply_i_overlap with CONDOVER ALL and with a SELECT
    plan, and apply_p_overlap with an intra map, of tests/ovl_cases.py's signed planes."""
    from oracle import Reference

    sys.path.insert(0, os.path.dirname(HERE))
    from ovl_cases import OVL_CASES, mb_flags, signed_planes

    d = {}
    for i, (w, h, pq, seed) in enumerate(OVL_CASES):
        R = Reference(make_params(w, h, pqindex=pq))
        planes, flags = signed_planes(w, h, seed), mb_flags(w, h, seed)
        for tag, out in (("all", R.overlap(planes, 1)), ("sel", R.overlap(planes, 2, flags)),
                         ("p", R.overlap(planes, 0, flags, p_picture=True))):
            for c, pl in zip("yuv", out):
                d[f"c{i}.{tag}.{c}"] = pl.astype(np.int16)
    np.savez_compressed(os.path.join(HERE, "ovl_kat.npz"), **d)


def main(only=()):
    if only:
        for name in only:
            {"b_kat": make_b_kat, "ic_kat": make_ic_kat, "scene_kat": make_scene_kat,
             "recon_kat": make_recon_kat, "lf_kat": make_lf_kat, "tt_kat": make_tt_kat,
             "ovl_kat": make_ovl_kat}[name]()
        return
    from oracle import Reference, ref_available

    if not ref_available():
        raise SystemExit("oracle/_ref/libvc1ref.so is missing: run `make -C oracle ref` first")

    # ---- runtime_kat
    cur, ref = runtime_frames()
    p = make_params(48, 40)
    R = Reference(p)
    rc, rr = R.frame(cur), R.frame(ref)
    mvs = np.array(RUNTIME_MVS, np.int32)
    half = np.array([mv for mv in RUNTIME_MVS if not (mv[0] & 1) and not (mv[1] & 1)], np.int32)
    ints = np.array([mv for mv in RUNTIME_MVS if mv[0] % 4 == 0 and mv[1] % 4 == 0], np.int32)
    d = {"cur": cur[0], "ref": ref[0], "mvs": mvs, "half_mvs": half, "int_mvs": ints,
         "sad_qpel": np.array([R.block_sad_motion(rc, rr, 5, 7, 16, 16, a, b, MV_QPEL) for a, b in mvs], np.uint64),
         "satd_qpel": np.array([R.block_satd_motion(rc, rr, 5, 7, 16, 16, a, b, MV_QPEL) for a, b in mvs], np.uint64),
         "sad_bilinear": np.array([R.block_sad_motion(rc, rr, 3, 4, 16, 16, a, b, MV_HPEL_BILINEAR) for a, b in half],
                                  np.uint64)}
    for s in (2, 4):
        d[f"sad_int_stride{s}"] = np.array([integer_sampled_sad(cur[0], ref[0], 5, 7, 16, 16, a // 4, b // 4, s)
                                            for a, b in ints], np.uint64)
    np.savez_compressed(os.path.join(HERE, "runtime_kat.npz"), **d)

    # ---- staged_kat
    c16, flat, noisy, c32, r32 = staged_frames()
    p16 = make_params(16, 16, search_range=8, local_search_range=8)
    R = Reference(p16)
    fc, ff, fn = R.frame(planes(c16)), R.frame(planes(flat)), R.frame(planes(noisy))
    d = {"cur16": c16, "flat16": flat, "noisy16": noisy,
         "sad_flat": np.uint64(R.block_sad_motion(fc, ff, 0, 0, 16, 16, 0, 0, MV_QPEL)),
         "sad_noisy": np.uint64(R.block_sad_motion(fc, fn, 0, 0, 16, 16, 0, 0, MV_QPEL)),
         "satd_flat": np.uint64(R.block_satd_motion(fc, ff, 0, 0, 16, 16, 0, 0, MV_QPEL)),
         "satd_noisy": np.uint64(R.block_satd_motion(fc, fn, 0, 0, 16, 16, 0, 0, MV_QPEL))}
    p32 = make_params(32, 32, search_range=8, local_search_range=8)
    R = Reference(p32)
    a32, b32 = R.frame(planes(c32)), R.frame(planes(r32))
    qgrid = np.array([(x, y) for y in range(-7, 8) for x in range(-7, 8)], np.int32)
    bgrid = np.array([(x, y) for y in range(-6, 7, 2) for x in range(-6, 7, 2)], np.int32)
    d.update({"cur32": c32, "ref32": r32, "qgrid": qgrid, "bgrid": bgrid,
              "satd_qgrid": np.array([R.block_satd_motion(a32, b32, 8, 8, 16, 16, x, y, MV_QPEL) for x, y in qgrid],
                                     np.uint64),
              "satd_bgrid": np.array([R.block_satd_motion(a32, b32, 8, 8, 16, 16, x, y, MV_HPEL_BILINEAR)
                                      for x, y in bgrid], np.uint64)})
    np.savez_compressed(os.path.join(HERE, "staged_kat.npz"), **d)

    # ---- diamond_kat
    d = {}
    for i, (sx, sy, hor) in enumerate(((4, 0, True), (0, -3, False))):
        pd = make_params(64, 48, search_range=12, local_search_range=12, me_algorithm=1)
        R = Reference(pd)
        g = gradient(64, 48, hor)
        c = shifted(g, sx, sy)
        field = np.zeros((4 * 3, 2), np.int32)
        d[f"shift{i}"] = np.array([sx, sy, int(hor)], np.int32)
        d[f"shift{i}.result"] = np.array(R.integer_motion(R.frame(planes(c)), R.frame(planes(g)), 1, 1, field, 0, 0, 12),
                                         np.int64)
    pe = make_params(64, 48, display_height=42, search_range=8, local_search_range=8, me_algorithm=1)
    R = Reference(pe)
    g = R.frame(planes(gradient(64, 48, True)))
    d["edge_mb_sad"] = np.uint64(R.mb_sad(g, g, 1, 2, 0, 4, 1))
    np.savez_compressed(os.path.join(HERE, "diamond_kat.npz"), **d)

    # ---- analysis chains
    for name, (make, kw) in ANALYSIS.items():
        clip = make()
        p = make_params(clip.width, clip.height, **kw)
        R = Reference(p)
        cur, ref = clip.frame(1), clip.frame(0)
        rc, rr = R.frame(cur), R.frame(ref)

        def run_pass(_p, _c, _r, mode, intra, seed, sd):
            return R.analyze_p_core(rc, rr, mode, intra, seed=seed, seed_distant=sd)

        d = {"cur.y": cur[0], "cur.u": cur[1], "cur.v": cur[2], "ref.y": ref[0], "ref.u": ref[1], "ref.v": ref[2]}
        for k, a in analysis_chain(run_pass, p, cur, ref).items():
            flatten(k, a, d)
        np.savez_compressed(os.path.join(HERE, f"analysis_{name}.npz"), **d)

    # ---- xform_kat: prediction of the final pass of cif_r8, transform + quantiser at four QPs
    clip = synth.generate(64, 48, 2, 11)
    d = {"cur.y": clip.frame(1)[0], "cur.u": clip.frame(1)[1], "cur.v": clip.frame(1)[2],
         "ref.y": clip.frame(0)[0], "ref.u": clip.frame(0)[1], "ref.v": clip.frame(0)[2]}
    for pq, nu, hq in ((3, 0, 1), (8, 1, 1), (17, 1, 0), (31, 0, 0)):
        p = make_params(64, 48, pqindex=pq, nonuniform=nu, halfqp=hq, search_range=8, local_search_range=8)
        R = Reference(p)
        rc, rr = R.frame(clip.frame(1)), R.frame(clip.frame(0))
        q = R.analyze_p_core(rc, rr, MV_QPEL, False)
        f = R.analyze_p_core(rc, rr, MV_MIXED, True, seed=q.mvs, seed_distant=q)
        pred = R.motion_compensate(rr, f, MV_MIXED)
        co, lv = R.forward_quant(rc, R.frame(pred), 15)
        key = f"pq{pq}_nu{nu}_hq{hq}"
        d[f"{key}.mvs"], d[f"{key}.block_mvs"] = f.mvs, f.block_mvs
        d[f"{key}.use_4mv"], d[f"{key}.use_intra"] = f.use_4mv, f.use_intra
        d[f"{key}.pred.y"], d[f"{key}.pred.u"], d[f"{key}.pred.v"] = pred
        d[f"{key}.coeffs"], d[f"{key}.levels"] = co, lv
    np.savez_compressed(os.path.join(HERE, "xform_kat.npz"), **d)

    # ---- global_kat
    d = {}
    for i, (make, rng) in enumerate(((lambda: synth.cif_plain(frames=2, seed=3), 8),
                                     (lambda: synth.cif_plain(frames=2, seed=3), 31),
                                     (lambda: synth.generate(352, 288, 2, 9, global_px=20.0, n_objects=2), 32))):
        clip = make()
        p = make_params(352, 288, search_range=rng, local_search_range=rng)
        R = Reference(p)
        rc, rr = R.frame(clip.frame(1)), R.frame(clip.frame(0))
        d[f"g{i}.cur"], d[f"g{i}.ref"] = clip.frame(1)[0], clip.frame(0)[0]
        d[f"g{i}.range"] = np.int32(rng)
        d[f"g{i}.result"] = np.array(R.global_motion(rc, rr, rng), np.int64)
        offs = [(0, 0), (3, -2), (-17, 9), (40, 31), (-60, -50)]
        d[f"g{i}.frame_sad_offsets"] = np.array(offs, np.int32)
        d[f"g{i}.frame_sad"] = np.array([[R.frame_sad(rc, rr, dx, dy, s) for s in (1, 2, 4)] for dx, dy in offs],
                                        np.uint64)
    np.savez_compressed(os.path.join(HERE, "global_kat.npz"), **d)
    make_b_kat()
    make_ic_kat()
    make_scene_kat()
    make_recon_kat()
    make_lf_kat()
    make_tt_kat()
    make_ovl_kat()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
