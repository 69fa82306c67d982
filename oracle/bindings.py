"""ctypes bindings of the two CPU checkers (see oracle/__init__.py)."""
from __future__ import annotations

import collections
import ctypes as C
import os

import numpy as np

from libvc1_b200.abi import Analysis, BAnalysis, BAnalysisC, Intensity, Mv, PAnalysisC, Params, PpicCfg, mbs_of

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_oracle", "libvc1oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libvc1ref.so")
P = C.POINTER(Params)
u64, i32, vp = C.c_uint64, C.c_int, C.c_void_p


def ref_available() -> bool:
    return os.path.exists(REF_SO)


class VoFrame(C.Structure):
    _fields_ = [("w", C.c_int32), ("h", C.c_int32), ("y", vp), ("u", vp), ("v", vp)]


class Counts(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("int_sad_samples", "qpel1d_samples", "qpel2d_samples",
                                          "bilinear_samples", "satd_tiles", "frame_sad_samples",
                                          "xform_flops", "quant_coeffs", "macroblocks")]


def _planes(frame):
    y, u, v = frame
    y = np.ascontiguousarray(y, np.uint8)
    u = np.ascontiguousarray(u, np.uint8)
    v = np.ascontiguousarray(v, np.uint8)
    return y, u, v


def _seed_ptr(seed):
    if seed is None:
        return None, None
    s = np.ascontiguousarray(seed, np.int32).reshape(-1, 2)
    return s, s.ctypes.data


class Oracle:
    """Our C restatement of the reference path."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: build it with `make -C oracle oracle`")
        L = self.lib = C.CDLL(path)
        L.vo_mb_sad.argtypes = [P, vp, vp, i32, i32, i32, i32, i32]
        L.vo_mb_sad.restype = u64
        L.vo_block_sad_qpel.argtypes = [P, vp, vp, i32, i32, i32, i32, i32, i32]
        L.vo_block_sad_qpel.restype = u64
        L.vo_block_sad_motion.argtypes = [P, vp, vp, i32, i32, i32, i32, i32, i32, i32]
        L.vo_block_sad_motion.restype = u64
        L.vo_block_satd_motion.argtypes = [P, vp, vp, i32, i32, i32, i32, i32, i32, i32]
        L.vo_block_satd_motion.restype = u64
        L.vo_frame_sad.argtypes = [vp, vp, i32, i32, i32]
        L.vo_frame_sad.restype = u64
        L.vo_shader_cost.argtypes = [vp, vp, i32, i32, i32, i32, i32, i32, i32, i32, i32, i32]
        L.vo_shader_cost.restype = u64
        L.vo_hidden_padding.argtypes = [P, i32, i32, i32, i32, i32, i32, i32, i32]
        L.vo_predict_luma.argtypes = [P, vp, i32, i32, i32, i32, i32, i32, i32, vp, i32]
        L.vo_analyze_p_learned.argtypes = [P, vp, vp, i32, vp, i32, i32, i32, vp, C.POINTER(PAnalysisC)]
        L.vo_analyze_p_learned.restype = i32
        L.vo_global_motion.argtypes = [P, vp, vp, i32, C.POINTER(i32), C.POINTER(i32), C.POINTER(u64)]
        L.vo_integer_motion.argtypes = [P, vp, vp, i32, i32, vp, i32, i32, i32, C.POINTER(i32),
                                        C.POINTER(i32), C.POINTER(u64)]
        L.vo_analyze_p_core.argtypes = [P, vp, vp, i32, i32, vp, C.POINTER(PAnalysisC), C.POINTER(PAnalysisC)]
        L.vo_motion_compensate.argtypes = [P, vp, vp, vp, vp, i32, vp, vp, vp]
        L.vo_forward_part.argtypes = [vp, vp, i32, i32, i32, i32, i32, i32, vp]
        L.vo_quantize_level.argtypes = [P, C.c_double]
        L.vo_forward_quant.argtypes = [P, vp, vp, i32, vp, vp]
        L.vo_estimate_intensity_comp.argtypes = [P, vp, vp, vp, C.POINTER(Intensity)]
        L.vo_intensity_compensate.argtypes = [vp, C.POINTER(Intensity), vp, vp, vp]
        L.vo_scene_change_score.argtypes = [P, vp, vp, i32, C.c_double]
        L.vo_scene_change_score.restype = C.c_double
        L.vo_zoom_coherent.argtypes = [vp, i32, i32]
        L.vo_b_predict.argtypes = [P, vp, vp, vp, vp, vp, vp, i32, vp, vp, vp]
        L.vo_reconstruct.argtypes = [P, vp, vp, i32, vp, vp, vp, vp]
        L.vo_loop_filter_i.argtypes = [P, vp, vp, vp]
        L.vo_loop_filter_p.argtypes = [P, vp, vp, vp, vp, vp, vp, vp]
        L.vo_overlap_smooth.argtypes = [i32, i32, vp, vp, vp, vp, i32]
        L.vo_store_signed.argtypes = [i32, i32, vp, vp, vp, i32, vp, i32, i32, vp, vp, vp]
        L.vo_fast_transform_types.argtypes = [P, vp, vp, vp]
        L.vo_analyze_b.argtypes = [P, vp, vp, vp, vp, vp, i32, i32, i32, C.POINTER(BAnalysisC)]
        L.vo_b_costs.argtypes = [P, vp, vp, vp, i32, i32, Mv, Mv, Mv, Mv, i32, vp]
        L.vo_score_key.argtypes = [u64, C.c_double, u64, i32, C.POINTER(u64), C.POINTER(u64)]
        L.vo_counts_get.argtypes = [C.POINTER(Counts)]
        self._keep = []

    def frame(self, frame) -> VoFrame:
        y, u, v = _planes(frame)
        f = VoFrame(y.shape[1], y.shape[0], y.ctypes.data, u.ctypes.data, v.ctypes.data)
        f._arrays = (y, u, v)
        return f

    def _f(self, fr):
        return C.byref(fr if isinstance(fr, VoFrame) else self.frame(fr))

    def counts(self) -> dict:
        c = Counts()
        self.lib.vo_counts_get(C.byref(c))
        return {f[0]: getattr(c, f[0]) for f in Counts._fields_}

    def reset_counts(self):
        self.lib.vo_counts_reset()

    def mb_sad(self, p, cur, ref, mx, my, dx, dy, stride=1):
        return self.lib.vo_mb_sad(C.byref(p), self._f(cur), self._f(ref), mx, my, dx, dy, stride)

    def block_sad_qpel(self, p, cur, ref, x0, y0, bw, bh, xq, yq):
        return self.lib.vo_block_sad_qpel(C.byref(p), self._f(cur), self._f(ref), x0, y0, bw, bh, xq, yq)

    def block_sad_motion(self, p, cur, ref, x0, y0, bw, bh, xq, yq, mode):
        return self.lib.vo_block_sad_motion(C.byref(p), self._f(cur), self._f(ref), x0, y0, bw, bh, xq, yq, mode)

    def block_satd_motion(self, p, cur, ref, x0, y0, bw, bh, xq, yq, mode):
        return self.lib.vo_block_satd_motion(C.byref(p), self._f(cur), self._f(ref), x0, y0, bw, bh, xq, yq, mode)

    def frame_sad(self, cur, ref, dx, dy, stride=1):
        return self.lib.vo_frame_sad(self._f(cur), self._f(ref), dx, dy, stride)

    def shader_cost(self, cur, ref, x0, y0, bw, bh, stride, bilinear, rnd, metric, xq, yq):
        return self.lib.vo_shader_cost(self._f(cur), self._f(ref), x0, y0, bw, bh, stride, bilinear, rnd,
                                       metric, xq, yq)

    def hidden(self, p, x0, y0, bw, bh, xq, yq, mode, chroma):
        return bool(self.lib.vo_hidden_padding(C.byref(p), x0, y0, bw, bh, xq, yq, mode, chroma))

    def predict_luma(self, p, ref, x0, y0, bw, bh, xq, yq, mode):
        out = np.zeros((bh, bw), np.uint8)
        self.lib.vo_predict_luma(C.byref(p), self._f(ref), x0, y0, bw, bh, xq, yq, mode, out.ctypes.data, bw)
        return out

    def global_motion(self, p, cur, ref, rng):
        dx, dy, s = i32(), i32(), u64()
        self.lib.vo_global_motion(C.byref(p), self._f(cur), self._f(ref), rng, C.byref(dx), C.byref(dy), C.byref(s))
        return dx.value, dy.value, s.value

    def integer_motion(self, p, cur, ref, mx, my, field, gdx, gdy, rng):
        fld = np.ascontiguousarray(field, np.int32).reshape(-1, 2)
        dx, dy, s = i32(), i32(), u64()
        self.lib.vo_integer_motion(C.byref(p), self._f(cur), self._f(ref), mx, my, fld.ctypes.data, gdx, gdy, rng,
                                   C.byref(dx), C.byref(dy), C.byref(s))
        return dx.value, dy.value, s.value

    def analyze_p_core(self, p, cur, ref, mode, allow_intra, seed=None, seed_distant: Analysis | None = None):
        mbw, mbh = mbs_of(p)
        out = Analysis.empty(mbw * mbh)
        oc = out.as_c()
        s, sp = _seed_ptr(seed)
        sd = seed_distant.as_c() if seed_distant is not None else None
        rc = self.lib.vo_analyze_p_core(C.byref(p), self._f(cur), self._f(ref), mode, int(allow_intra), sp,
                                        C.byref(sd) if sd is not None else None, C.byref(oc))
        if rc:
            raise RuntimeError("oracle analyze_p_core failed")
        return out.take_totals(oc)

    def analyze_p_learned(self, p, cur, ref, mode, cands, hint, fallback=True):
        """This library's learned pass (vo_analyze_p_learned): cands (mbs, 4, 2) integer pixels,
        hint (dx, dy). Returns (Analysis, fallback flags)."""
        mbw, mbh = mbs_of(p)
        out = Analysis.empty(mbw * mbh)
        oc = out.as_c()
        cc = np.ascontiguousarray(cands, np.int32).reshape(-1, 2)
        flags = np.zeros(mbw * mbh, np.uint8)
        rc = self.lib.vo_analyze_p_learned(C.byref(p), self._f(cur), self._f(ref), mode, cc.ctypes.data, int(hint[0]),
                                           int(hint[1]), int(fallback), flags.ctypes.data, C.byref(oc))
        if rc:
            raise RuntimeError("oracle analyze_p_learned failed")
        return out.take_totals(oc), flags

    def scene_change_score(self, p, cur, ref, fade_compensation=True, scene_threshold=28.0):
        return self.lib.vo_scene_change_score(C.byref(p), self._f(cur), self._f(ref), int(fade_compensation),
                                              float(scene_threshold))

    def zoom_coherent(self, mvs, mbw, mbh):
        m = np.ascontiguousarray(mvs, np.int32).reshape(-1, 2)
        return bool(self.lib.vo_zoom_coherent(m.ctypes.data, mbw, mbh))

    def estimate_intensity_comp(self, p, cur, ref, mvs):
        m = np.ascontiguousarray(mvs, np.int32).reshape(-1, 2)
        out = Intensity()
        self.lib.vo_estimate_intensity_comp(C.byref(p), self._f(cur), self._f(ref), m.ctypes.data, C.byref(out))
        return out.as_tuple()

    def intensity_compensate(self, ref, ic):
        y, u, v = _planes(ref)
        h, w = y.shape
        k = Intensity(*ic)
        oy, ou, ov = np.zeros_like(y), np.zeros_like(u), np.zeros_like(v)
        self.lib.vo_intensity_compensate(self._f(ref), C.byref(k), oy.ctypes.data, ou.ctypes.data, ov.ctypes.data)
        return oy, ou, ov

    def loop_filter(self, p, frame, block_mvs=None, cbp=None, tt=None, intra=None):
        """A filtered copy of frame: the I-like filter when block_mvs is None, else the P filter."""
        y, u, v = (np.array(a, np.uint8, copy=True) for a in _planes(frame))
        if block_mvs is None:
            self.lib.vo_loop_filter_i(C.byref(p), y.ctypes.data, u.ctypes.data, v.ctypes.data)
        else:
            b = np.ascontiguousarray(block_mvs, np.int32)
            cb, t, i = (np.ascontiguousarray(a, np.uint8) for a in (cbp, tt, intra))
            self.lib.vo_loop_filter_p(C.byref(p), y.ctypes.data, u.ctypes.data, v.ctypes.data, b.ctypes.data,
                                      cb.ctypes.data, t.ctypes.data, i.ctypes.data)
        return y, u, v

    def overlap_smooth(self, p, planes, flags=None, all_edges=False):
        """Overlap-smoothed copies of a signed padded reconstruction (int32 planes
        (mbh*16, mbw*16), (mbh*8, mbw*8) x 2); flags per MB, or all_edges."""
        mbw, mbh = mbs_of(p)
        y, u, v = (np.array(a, np.int32, copy=True, order="C") for a in planes)
        f = None if flags is None else np.ascontiguousarray(flags, np.uint8)
        self.lib.vo_overlap_smooth(mbw, mbh, y.ctypes.data, u.ctypes.data, v.ctypes.data,
                                   None if f is None else f.ctypes.data, int(all_edges))
        return y, u, v

    def store_signed(self, p, planes, bias, mask=None, into=None):
        """clamp(s + bias) of the signed planes: the padded raster when into is None, else written
        over a copy of the frame `into` (masked MBs only when mask is given)."""
        mbw, mbh = mbs_of(p)
        sy, su, sv = (np.ascontiguousarray(a, np.int32) for a in planes)
        if into is None:
            y = np.zeros((mbh * 16, mbw * 16), np.uint8)
            u, v = np.zeros((mbh * 8, mbw * 8), np.uint8), np.zeros((mbh * 8, mbw * 8), np.uint8)
        else:
            y, u, v = (np.array(a, np.uint8, copy=True) for a in _planes(into))
        m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        self.lib.vo_store_signed(mbw, mbh, sy.ctypes.data, su.ctypes.data, sv.ctypes.data, int(bias),
                                 None if m is None else m.ctypes.data, y.shape[1], y.shape[0], y.ctypes.data,
                                 u.ctypes.data, v.ctypes.data)
        return y, u, v

    def fast_transform_types(self, p, src, pred):
        mbw, mbh = mbs_of(p)
        out = np.zeros(mbw * mbh, np.uint8)
        self.lib.vo_fast_transform_types(C.byref(p), self._f(src), self._f(pred), out.ctypes.data)
        return out

    def reconstruct(self, p, pred, levels, type_mask, block_types):
        h, w = p.height, p.width
        y = np.zeros((h, w), np.uint8)
        u = np.zeros((h // 2, w // 2), np.uint8)
        v = np.zeros_like(u)
        lv = np.ascontiguousarray(levels, np.int16)
        bt = np.ascontiguousarray(block_types, np.uint8)
        self.lib.vo_reconstruct(C.byref(p), self._f(pred), lv.ctypes.data, type_mask, bt.ctypes.data, y.ctypes.data,
                                u.ctypes.data, v.ctypes.data)
        return y, u, v

    def b_predict(self, p, cur, past, future, b: BAnalysis, mode):
        h, w = p.height, p.width
        y = np.zeros((h, w), np.uint8)
        u = np.zeros((h // 2, w // 2), np.uint8)
        v = np.zeros_like(u)
        self.lib.vo_b_predict(C.byref(p), self._f(cur), self._f(past), self._f(future), b.modes.ctypes.data,
                              b.forward_mvs.ctypes.data, b.backward_mvs.ctypes.data, mode, y.ctypes.data,
                              u.ctypes.data, v.ctypes.data)
        return y, u, v

    def analyze_b(self, p, cur, past, future, anchor_mvs, anchor_4mv, num, den, mode):
        mbw, mbh = mbs_of(p)
        out = BAnalysis.empty(mbw * mbh)
        oc = out.as_c()
        am = np.ascontiguousarray(anchor_mvs, np.int32).reshape(-1, 2)
        a4 = np.ascontiguousarray(anchor_4mv, np.uint8)
        rc = self.lib.vo_analyze_b(C.byref(p), self._f(cur), self._f(past), self._f(future), am.ctypes.data,
                                   a4.ctypes.data, num, den, mode, C.byref(oc))
        if rc:
            raise RuntimeError("oracle analyze_b failed")
        return out.take_totals(oc)

    def motion_compensate(self, p, ref, a: Analysis, mode):
        h, w = p.height, p.width
        y = np.zeros((h, w), np.uint8)
        u = np.full((h // 2, w // 2), 128, np.uint8)
        v = u.copy()
        self.lib.vo_motion_compensate(C.byref(p), self._f(ref), a.mvs.ctypes.data, a.block_mvs.ctypes.data,
                                      a.use_4mv.ctypes.data, mode, y.ctypes.data, u.ctypes.data, v.ctypes.data)
        return y, u, v

    def forward_quant(self, p, src, pred, type_mask=1):
        mbw, mbh = mbs_of(p)
        nt = bin(type_mask & 15).count("1")
        co = np.zeros((nt, mbw * mbh, 6, 64), np.float64)
        lv = np.zeros((nt, mbw * mbh, 6, 64), np.int16)
        self.lib.vo_forward_quant(C.byref(p), self._f(src), self._f(pred), type_mask, co.ctypes.data, lv.ctypes.data)
        return co, lv

    def quantize_level(self, p, c):
        return self.lib.vo_quantize_level(C.byref(p), c)

    def score_key(self, sad, lam, rate, bits=64):
        hi, lo = u64(), u64()
        self.lib.vo_score_key(sad, lam, rate, bits, C.byref(hi), C.byref(lo))
        return (hi.value << 64) | lo.value


class RefFrame:
    def __init__(self, lib, frame):
        y, u, v = _planes(frame)
        self._lib = lib
        self.h = lib.ref_frame_new(y.ctypes.data, u.ctypes.data, v.ctypes.data, y.shape[1], y.shape[0])

    def __del__(self):
        try:
            self._lib.ref_frame_free(self.h)
        except Exception:
            pass


class Reference:
    """The reference's own functions (compiled from its sources; scalar or SIMD-dispatched)."""

    def __init__(self, p: Params, simd_auto: bool = False, path: str = REF_SO):
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: build it with `make -C oracle ref`")
        L = self.lib = C.CDLL(path)
        L.ref_frame_new.argtypes = [vp, vp, vp, i32, i32]
        L.ref_frame_new.restype = vp
        L.ref_frame_free.argtypes = [vp]
        L.ref_frame_read.argtypes = [vp, vp, vp, vp]
        L.ref_encoder_new.argtypes = [P, i32]
        L.ref_encoder_new.restype = vp
        L.ref_encoder_free.argtypes = [vp]
        for n in ("ref_block_sad_motion", "ref_block_satd_motion"):
            getattr(L, n).argtypes = [vp, vp, vp, i32, i32, i32, i32, i32, i32, i32]
            getattr(L, n).restype = u64
        L.ref_block_sad_qpel.argtypes = [vp, vp, vp, i32, i32, i32, i32, i32, i32]
        L.ref_block_sad_qpel.restype = u64
        L.ref_mb_sad.argtypes = [vp, vp, vp, i32, i32, i32, i32, i32]
        L.ref_mb_sad.restype = u64
        L.ref_frame_sad.argtypes = [vp, vp, vp, i32, i32, i32]
        L.ref_frame_sad.restype = u64
        L.ref_global_motion.argtypes = [vp, vp, vp, i32, C.POINTER(i32), C.POINTER(i32), C.POINTER(u64)]
        L.ref_predict_luma.argtypes = [vp, vp, i32, i32, i32, i32, i32, i32, i32, vp, i32]
        L.ref_integer_motion.argtypes = [vp, vp, vp, i32, i32, vp, i32, i32, i32, C.POINTER(i32), C.POINTER(i32),
                                         C.POINTER(u64)]
        L.ref_analyze_p_core.argtypes = [vp, vp, vp, i32, i32, vp, C.POINTER(PAnalysisC), C.POINTER(PAnalysisC)]
        L.ref_analyze_p_core.restype = i32
        L.ref_analyze_p_picture.argtypes = [vp, vp, vp, C.POINTER(PAnalysisC), C.POINTER(i32), C.POINTER(i32)]
        L.ref_analyze_p_picture.restype = i32
        L.ref_analyze_p_picture_cfg.argtypes = [vp, C.POINTER(PpicCfg), vp, vp, C.POINTER(PAnalysisC), C.POINTER(i32),
                                                C.POINTER(i32), C.POINTER(u64)]
        L.ref_analyze_p_picture_cfg.restype = i32
        L.ref_p_mode_scores.argtypes = [vp, C.POINTER(PpicCfg), vp, vp, vp, vp]
        L.ref_p_mode_scores.restype = i32
        L.ref_b_mode_scores.argtypes = [vp, C.POINTER(PpicCfg), vp, vp, vp, vp, vp, i32, i32, vp, C.POINTER(i32)]
        L.ref_b_mode_scores.restype = i32
        L.ref_reconstruct_intra.argtypes = [vp, i32, C.c_double, i32, vp, i32, vp, vp, vp, vp, vp, vp]
        L.ref_choose_i_overlap.argtypes = [vp, i32, C.c_double, i32, vp, C.POINTER(i32), vp]
        L.ref_estimate_p_motion_bits.argtypes = [vp, vp, vp, vp, vp, i32, i32]
        L.ref_estimate_p_motion_bits.restype = u64
        L.ref_motion_compensate.argtypes = [vp, vp, vp, vp, vp, i32, vp]
        L.ref_motion_compensate_padded.argtypes = [vp, vp, vp, vp, vp, i32, vp]
        L.ref_b_predict_padded.argtypes = [vp, vp, vp, vp, vp, vp, i32, vp]
        L.ref_forward_quant.argtypes = [vp, vp, vp, i32, vp, vp]
        L.ref_scalar_quantize_level.argtypes = [vp, C.c_double]
        L.ref_estimate_ic.argtypes = [vp, vp, vp, vp, C.POINTER(Intensity)]
        L.ref_ic_reference.argtypes = [vp, vp, C.POINTER(Intensity), vp]
        L.ref_scene_change_score.argtypes = [vp, vp, vp, i32, C.c_double]
        L.ref_scene_change_score.restype = C.c_double
        L.ref_b_predict.argtypes = [vp, vp, vp, vp, vp, vp, vp, i32, vp]
        L.ref_reconstruct.argtypes = [vp, vp, vp, i32, vp, vp, vp, vp]
        L.ref_loop_filter_i.argtypes = [vp, vp]
        L.ref_loop_filter_p.argtypes = [vp, vp, vp, vp, vp, vp, i32]
        L.ref_overlap.argtypes = [vp, C.c_int, C.c_int, vp, vp, vp, vp]
        L.ref_fast_transform_types.argtypes = [vp, vp, vp, vp]
        L.ref_analyze_b.argtypes = [vp, vp, vp, vp, vp, vp, i32, i32, i32, C.POINTER(BAnalysisC)]
        L.ref_bench_analysis.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), i32, i32]
        L.ref_bench_analysis.restype = u64
        L.ref_bench_analysis_multi.argtypes = [C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), i32, i32]
        L.ref_bench_analysis_multi.restype = u64
        L.ref_bench_gop_multi.argtypes = [C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), i32, C.POINTER(vp),
                                          C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(i32), C.POINTER(i32),
                                          C.POINTER(i32), i32, i32]
        L.ref_bench_gop_multi.restype = u64
        L.ref_bench_gop_same.argtypes = L.ref_bench_gop_multi.argtypes
        L.ref_bench_gop_same.restype = u64
        L.ref_choose_transform.argtypes = [vp, vp, vp, vp, vp, vp, vp]
        L.ref_choose_dquant.argtypes = [vp, vp, i32, i32, C.c_double, C.c_double, vp, vp, vp, vp, vp, vp]
        L.ref_choose_transform.restype = None
        L.ref_ac_direct_bits.argtypes = [i32, i32, i32, i32]
        L.ref_ac_direct_bits.restype = i32
        L.ref_ac_rate_bits.argtypes = [vp, i32, i32, i32, i32]
        L.ref_ac_rate_bits.restype = i32
        self.p = p
        self._recent = collections.deque(maxlen=8)
        self.h = L.ref_encoder_new(C.byref(p), int(simd_auto))

    def __del__(self):
        try:
            self.lib.ref_encoder_free(self.h)
        except Exception:
            pass

    def frame(self, frame) -> RefFrame:
        return RefFrame(self.lib, frame)

    def _f(self, fr):
        if isinstance(fr, RefFrame):
            return fr.h
        # a frame converted for this call: kept alive for the next few calls (the C++ side reads it
        # during the call; freeing it as soon as its handle is taken would leave the handle dangling)
        rf = self.frame(fr)
        self._recent.append(rf)
        return rf.h

    def mb_sad(self, cur, ref, mx, my, dx, dy, stride=1):
        return self.lib.ref_mb_sad(self.h, self._f(cur), self._f(ref), mx, my, dx, dy, stride)

    def block_sad_qpel(self, cur, ref, x0, y0, bw, bh, xq, yq):
        return self.lib.ref_block_sad_qpel(self.h, self._f(cur), self._f(ref), x0, y0, bw, bh, xq, yq)

    def block_sad_motion(self, cur, ref, x0, y0, bw, bh, xq, yq, mode):
        return self.lib.ref_block_sad_motion(self.h, self._f(cur), self._f(ref), x0, y0, bw, bh, xq, yq, mode)

    def block_satd_motion(self, cur, ref, x0, y0, bw, bh, xq, yq, mode):
        return self.lib.ref_block_satd_motion(self.h, self._f(cur), self._f(ref), x0, y0, bw, bh, xq, yq, mode)

    def frame_sad(self, cur, ref, dx, dy, stride=1):
        return self.lib.ref_frame_sad(self.h, self._f(cur), self._f(ref), dx, dy, stride)

    def global_motion(self, cur, ref, rng):
        dx, dy, s = i32(), i32(), u64()
        self.lib.ref_global_motion(self.h, self._f(cur), self._f(ref), rng, C.byref(dx), C.byref(dy), C.byref(s))
        return dx.value, dy.value, s.value

    def predict_luma(self, ref, x0, y0, bw, bh, xq, yq, mode):
        out = np.zeros((bh, bw), np.uint8)
        self.lib.ref_predict_luma(self.h, self._f(ref), x0, y0, bw, bh, xq, yq, mode, out.ctypes.data, bw)
        return out

    def integer_motion(self, cur, ref, mx, my, field, gdx, gdy, rng):
        fld = np.ascontiguousarray(field, np.int32).reshape(-1, 2)
        dx, dy, s = i32(), i32(), u64()
        self.lib.ref_integer_motion(self.h, self._f(cur), self._f(ref), mx, my, fld.ctypes.data, gdx, gdy, rng,
                                    C.byref(dx), C.byref(dy), C.byref(s))
        return dx.value, dy.value, s.value

    def analyze_p_core(self, cur, ref, mode, allow_intra, seed=None, seed_distant: Analysis | None = None):
        mbw, mbh = mbs_of(self.p)
        out = Analysis.empty(mbw * mbh)
        oc = out.as_c()
        s, sp = _seed_ptr(seed)
        sd = seed_distant.as_c() if seed_distant is not None else None
        rc = self.lib.ref_analyze_p_core(self.h, self._f(cur), self._f(ref), mode, int(allow_intra), sp,
                                         C.byref(sd) if sd is not None else None, C.byref(oc))
        if rc:
            raise RuntimeError("reference analyze_p_picture_core threw")
        return out.take_totals(oc)

    def scene_change_score(self, cur, ref, fade_compensation=True, scene_threshold=28.0):
        return self.lib.ref_scene_change_score(self.h, self._f(cur), self._f(ref), int(fade_compensation),
                                               float(scene_threshold))

    def estimate_intensity_comp(self, cur, ref, mvs):
        m = np.ascontiguousarray(mvs, np.int32).reshape(-1, 2)
        out = Intensity()
        self.lib.ref_estimate_ic(self.h, self._f(cur), self._f(ref), m.ctypes.data, C.byref(out))
        return out.as_tuple()

    def intensity_compensate(self, ref, ic):
        h, w = self.p.height, self.p.width
        dst = self.frame((np.zeros((h, w), np.uint8), np.zeros((h // 2, w // 2), np.uint8),
                          np.zeros((h // 2, w // 2), np.uint8)))
        k = Intensity(*ic)
        self.lib.ref_ic_reference(self.h, self._f(ref), C.byref(k), dst.h)
        y = np.zeros((h, w), np.uint8)
        u = np.zeros((h // 2, w // 2), np.uint8)
        v = np.zeros_like(u)
        self.lib.ref_frame_read(dst.h, y.ctypes.data, u.ctypes.data, v.ctypes.data)
        return y, u, v

    def loop_filter(self, frame, block_mvs=None, cbp=None, tt=None, intra=None, main_profile=False):
        h, w = self.p.height, self.p.width
        f = self.frame(frame)
        if block_mvs is None:
            self.lib.ref_loop_filter_i(self.h, f.h)
        else:
            b = np.ascontiguousarray(block_mvs, np.int32)
            cb, t, i = (np.ascontiguousarray(a, np.uint8) for a in (cbp, tt, intra))
            self.lib.ref_loop_filter_p(self.h, f.h, b.ctypes.data, cb.ctypes.data, t.ctypes.data, i.ctypes.data,
                                       int(main_profile))
        y = np.zeros((h, w), np.uint8)
        u = np.zeros((h // 2, w // 2), np.uint8)
        v = np.zeros_like(u)
        self.lib.ref_frame_read(f.h, y.ctypes.data, u.ctypes.data, v.ctypes.data)
        return y, u, v

    def overlap(self, planes, mode=1, flags=None, p_picture=False):
        """apply_i_overlap with plan mode (0 None, 1 All, 2 Select with flags), or with p_picture
        apply_p_overlap with flags as the intra map, on copies of the signed padded planes."""
        y, u, v = (np.array(a, np.int32, copy=True, order="C") for a in planes)
        f = None if flags is None else np.ascontiguousarray(flags, np.uint8)
        self.lib.ref_overlap(self.h, int(p_picture), int(mode), None if f is None else f.ctypes.data, y.ctypes.data,
                             u.ctypes.data, v.ctypes.data)
        return y, u, v

    def fast_transform_types(self, src, pred):
        mbw, mbh = mbs_of(self.p)
        out = np.zeros(mbw * mbh, np.uint8)
        self.lib.ref_fast_transform_types(self.h, self._f(src), self._f(pred), out.ctypes.data)
        return out

    def reconstruct(self, pred, levels, type_mask, block_types, mquant=None, derived=None):
        h, w = self.p.height, self.p.width
        dst = self.frame((np.zeros((h, w), np.uint8), np.zeros((h // 2, w // 2), np.uint8),
                          np.zeros((h // 2, w // 2), np.uint8)))
        lv = np.ascontiguousarray(levels, np.int16)
        bt = np.ascontiguousarray(block_types, np.uint8)
        mq, der = [None if a is None else np.ascontiguousarray(a, np.uint8) for a in (mquant, derived)]
        self.lib.ref_reconstruct(self.h, self._f(pred), lv.ctypes.data, type_mask, bt.ctypes.data,
                                 None if mq is None else mq.ctypes.data, None if der is None else der.ctypes.data, dst.h)
        y = np.zeros((h, w), np.uint8)
        u = np.zeros((h // 2, w // 2), np.uint8)
        v = np.zeros_like(u)
        self.lib.ref_frame_read(dst.h, y.ctypes.data, u.ctypes.data, v.ctypes.data)
        return y, u, v

    def b_predict(self, cur, past, future, b: BAnalysis, mode):
        h, w = self.p.height, self.p.width
        dst = self.frame((np.zeros((h, w), np.uint8), np.zeros((h // 2, w // 2), np.uint8),
                          np.zeros((h // 2, w // 2), np.uint8)))
        self.lib.ref_b_predict(self.h, self._f(cur), self._f(past), self._f(future), b.modes.ctypes.data,
                               b.forward_mvs.ctypes.data, b.backward_mvs.ctypes.data, mode, dst.h)
        y = np.zeros((h, w), np.uint8)
        u = np.zeros((h // 2, w // 2), np.uint8)
        v = np.zeros_like(u)
        self.lib.ref_frame_read(dst.h, y.ctypes.data, u.ctypes.data, v.ctypes.data)
        return y, u, v

    def analyze_b(self, cur, past, future, anchor_mvs, anchor_4mv, num, den, mode):
        mbw, mbh = mbs_of(self.p)
        out = BAnalysis.empty(mbw * mbh)
        oc = out.as_c()
        am = np.ascontiguousarray(anchor_mvs, np.int32).reshape(-1, 2)
        a4 = np.ascontiguousarray(anchor_4mv, np.uint8)
        rc = self.lib.ref_analyze_b(self.h, self._f(cur), self._f(past), self._f(future), am.ctypes.data,
                                    a4.ctypes.data, num, den, mode, C.byref(oc))
        if rc:
            raise RuntimeError("reference analyze_b_picture_mode threw")
        return out.take_totals(oc)

    def analyze_p_picture(self, cur, ref):
        mbw, mbh = mbs_of(self.p)
        out = Analysis.empty(mbw * mbh)
        oc = out.as_c()
        mode, ic = i32(), i32()
        rc = self.lib.ref_analyze_p_picture(self.h, self._f(cur), self._f(ref), C.byref(oc), C.byref(mode), C.byref(ic))
        if rc:
            raise RuntimeError("reference analyze_p_picture threw")
        out.take_totals(oc)
        return out, mode.value, bool(ic.value)

    def analyze_p_picture_cfg(self, cfg: PpicCfg, cur, ref):
        """analyze_p_picture under cfg: (analysis, chosen mode, IC enabled, motion bits)."""
        mbw, mbh = mbs_of(self.p)
        out = Analysis.empty(mbw * mbh)
        oc = out.as_c()
        mode, ic, bits = i32(), i32(), u64()
        rc = self.lib.ref_analyze_p_picture_cfg(self.h, C.byref(cfg), self._f(cur), self._f(ref), C.byref(oc),
                                                C.byref(mode), C.byref(ic), C.byref(bits))
        if rc:
            raise RuntimeError("reference analyze_p_picture threw")
        out.take_totals(oc)
        return out, mode.value, bool(ic.value), bits.value

    def p_mode_scores(self, cfg: PpicCfg, cur, ref):
        """The four plain candidates' motion bits and sampled mode-RD scores (long double values,
        returned as numpy longdouble)."""
        bits = np.zeros(4, np.uint64)
        scores = np.zeros(4, np.longdouble)
        assert C.sizeof(C.c_longdouble) == scores.itemsize
        rc = self.lib.ref_p_mode_scores(self.h, C.byref(cfg), self._f(cur), self._f(ref), bits.ctypes.data,
                                        scores.ctypes.data)
        if rc:
            raise RuntimeError("reference mode scoring threw")
        return bits, scores

    def b_mode_scores(self, cfg: PpicCfg, cur, past, future, anchor_mvs, anchor_4mv, num, den):
        """analyze_b_picture's quarter-pel and bilinear sampled_b_mode_rd scores (numpy longdouble)
        and its choice (1: bilinear)."""
        am = np.ascontiguousarray(anchor_mvs, np.int32).reshape(-1, 2)
        a4 = np.ascontiguousarray(anchor_4mv, np.uint8)
        scores = np.zeros(2, np.longdouble)
        chosen = i32()
        rc = self.lib.ref_b_mode_scores(self.h, C.byref(cfg), self._f(cur), self._f(past), self._f(future),
                                        am.ctypes.data, a4.ctypes.data, num, den, scores.ctypes.data, C.byref(chosen))
        if rc:
            raise RuntimeError("reference B mode scoring threw")
        return scores, chosen.value

    def reconstruct_intra(self, frame, overlap=0, flags=None, dquant=False, aq_strength=0.0, trellis=0):
        """reconstruct_i_signed_padded (AQ on when aq_strength > 0): the signed int32 planes of the
        padded raster and the DQUANT plan's per-MB MQUANT and derived flags."""
        mbw, mbh = mbs_of(self.p)
        pw, ph = mbw * 16, mbh * 16
        y = np.zeros((ph, pw), np.int32)
        u = np.zeros((ph // 2, pw // 2), np.int32)
        v = np.zeros_like(u)
        mq = np.zeros(mbw * mbh, np.uint8)
        der = np.zeros(mbw * mbh, np.uint8)
        fl = None if flags is None else np.ascontiguousarray(flags, np.uint8)
        self.lib.ref_reconstruct_intra(self.h, int(dquant), aq_strength, int(trellis), self._f(frame), overlap,
                                       None if fl is None else fl.ctypes.data, y.ctypes.data, u.ctypes.data,
                                       v.ctypes.data, mq.ctypes.data, der.ctypes.data)
        return (y, u, v), mq, der

    def choose_i_overlap(self, frame, dquant=False, aq_strength=0.0, trellis=0):
        """choose_i_overlap_plan with OVERLAP on: (mode 0 none / 1 all / 2 select, per-MB flags)."""
        mbw, mbh = mbs_of(self.p)
        flags = np.zeros(mbw * mbh, np.uint8)
        mode = i32()
        self.lib.ref_choose_i_overlap(self.h, int(dquant), aq_strength, int(trellis), self._f(frame), C.byref(mode),
                                      flags.ctypes.data)
        return mode.value, flags

    def estimate_p_motion_bits(self, a: Analysis, mode: int, intensity: bool = False) -> int:
        """estimate_p_motion_bits of analysis a made in mode (None when the reference throws)."""
        v = self.lib.ref_estimate_p_motion_bits(self.h, a.mvs.ctypes.data, a.block_mvs.ctypes.data,
                                                np.ascontiguousarray(a.use_4mv, np.uint8).ctypes.data,
                                                np.ascontiguousarray(a.use_intra, np.uint8).ctypes.data, mode,
                                                int(intensity))
        return None if v == 2 ** 64 - 1 else int(v)

    def motion_compensate(self, ref, a: Analysis, mode):
        h, w = self.p.height, self.p.width
        dst = self.frame((np.zeros((h, w), np.uint8), np.full((h // 2, w // 2), 128, np.uint8),
                          np.full((h // 2, w // 2), 128, np.uint8)))
        self.lib.ref_motion_compensate(self.h, self._f(ref), a.mvs.ctypes.data, a.block_mvs.ctypes.data,
                                       a.use_4mv.ctypes.data, mode, dst.h)
        y = np.zeros((h, w), np.uint8)
        u = np.zeros((h // 2, w // 2), np.uint8)
        v = np.zeros_like(u)
        self.lib.ref_frame_read(dst.h, y.ctypes.data, u.ctypes.data, v.ctypes.data)
        return y, u, v

    def _padded_call(self, fn):
        mbw, mbh = mbs_of(self.p)
        pw, ph = mbw * 16, mbh * 16
        dst = self.frame((np.zeros((ph, pw), np.uint8), np.full((ph // 2, pw // 2), 128, np.uint8),
                          np.full((ph // 2, pw // 2), 128, np.uint8)))
        fn(dst)
        y = np.zeros((ph, pw), np.uint8)
        u = np.zeros((ph // 2, pw // 2), np.uint8)
        v = np.zeros_like(u)
        self.lib.ref_frame_read(dst.h, y.ctypes.data, u.ctypes.data, v.ctypes.data)
        return y, u, v

    def motion_compensate_padded(self, ref, a: Analysis, mode):
        """motion_compensate_{mb,4mv}_padded of every macroblock from the padded reference frame
        `ref` (mbw*16 x mbh*16 planes) into a padded destination."""
        r = self.frame(ref)
        return self._padded_call(lambda dst: self.lib.ref_motion_compensate_padded(
            self.h, r.h, a.mvs.ctypes.data, a.block_mvs.ctypes.data, a.use_4mv.ctypes.data, mode, dst.h))

    def b_predict_padded(self, past, future, b, mode):
        """The B picture's padded prediction (Backward / Forward / bi) from padded references;
        B-intra macroblocks stay zero (luma) and 128 (chroma)."""
        pa, fu = self.frame(past), self.frame(future)
        return self._padded_call(lambda dst: self.lib.ref_b_predict_padded(
            self.h, pa.h, fu.h, np.ascontiguousarray(b.modes, np.uint8).ctypes.data, b.forward_mvs.ctypes.data,
            b.backward_mvs.ctypes.data, mode, dst.h))

    def forward_quant(self, src, pred, type_mask=1):
        mbw, mbh = mbs_of(self.p)
        nt = bin(type_mask & 15).count("1")
        co = np.zeros((nt, mbw * mbh, 6, 64), np.float64)
        lv = np.zeros((nt, mbw * mbh, 6, 64), np.int16)
        self.lib.ref_forward_quant(self.h, self._f(src), self._f(pred), type_mask, co.ctypes.data, lv.ctypes.data)
        return co, lv

    def quantize_level(self, c):
        return self.lib.ref_scalar_quantize_level(self.h, c)

    def bench_gop_multi(self, pjobs, bjobs, threads):
        """Wall ns of every P job (Reference, cur, ref) and then every B job (Reference, cur, past,
        future, index of its future anchor in pjobs, fraction_num, fraction_den)."""
        vpa = lambda xs: (vp * max(1, len(xs)))(*xs)  # noqa: E731
        ia = lambda xs: (i32 * max(1, len(xs)))(*xs)  # noqa: E731
        return self.lib.ref_bench_gop_multi(vpa([j[0].h for j in pjobs]), vpa([j[1].h for j in pjobs]),
                                            vpa([j[2].h for j in pjobs]), len(pjobs), vpa([j[0].h for j in bjobs]),
                                            vpa([j[1].h for j in bjobs]), vpa([j[2].h for j in bjobs]),
                                            vpa([j[3].h for j in bjobs]), ia([j[4] for j in bjobs]),
                                            ia([j[5] for j in bjobs]), ia([j[6] for j in bjobs]), len(bjobs), threads)

    def choose_transform(self, cfg, src, pred, mquant=None):
        """Vc1Encoder::choose_transform_mb of every MB (ref_choose_transform): decisions as a
        TDECISION_DTYPE array and the chosen levels int16 [mb][6][64]. cfg: abi.TrdCfg."""
        from libvc1_b200.abi import TDECISION_DTYPE

        mbw, mbh = mbs_of(self.p)
        out = np.zeros(mbw * mbh, TDECISION_DTYPE)
        lv = np.zeros((mbw * mbh, 6, 64), np.int16)
        mq = None if mquant is None else np.ascontiguousarray(mquant, np.uint8).reshape(-1)
        self.lib.ref_choose_transform(self.h, C.addressof(cfg), self._f(src), self._f(pred),
                                      None if mq is None else mq.ctypes.data, out.ctypes.data, lv.ctypes.data)
        return out, lv

    def choose_dquant(self, cfg, src, pred, dquant=True, predictable=False, block_weight=1.0, residual_mean=0.0):
        """Vc1Encoder::choose_dquant_transform_mb of every MB (ref_choose_dquant): (base MQUANT the
        function starts from, decisions, chosen MQUANT, levels)."""
        from libvc1_b200.abi import TDECISION_DTYPE

        mbw, mbh = mbs_of(self.p)
        n = mbw * mbh
        rb = np.zeros(n, np.uint8)
        out = np.zeros(n, TDECISION_DTYPE)
        mq = np.zeros(n, np.uint8)
        lv = np.zeros((n, 6, 64), np.int16)
        self.lib.ref_choose_dquant(self.h, C.addressof(cfg), int(dquant), int(predictable), block_weight, residual_mean,
                                   self._f(src), self._f(pred), rb.ctypes.data, out.ctypes.data, mq.ctypes.data,
                                   lv.ctypes.data)
        return rb, out, mq, lv

    def ac_direct_bits(self, coding_set, run, level, last):
        return self.lib.ref_ac_direct_bits(coding_set, run, level, int(last))

    def ac_rate_bits(self, coding_set, run, level, last):
        return self.lib.ref_ac_rate_bits(self.h, coding_set, run, level, int(last))

    def bench_gop_same(self, pjobs, bjobs, threads):
        """Wall ns of the GPU arm's work on the reference's functions (ref_bench_gop_same): per P
        job the five core passes, the fade estimate, the prediction and all four types' levels;
        per B job analyze_b_picture_mode in quarter-pel and bilinear mode; one pool for both."""
        vpa = lambda xs: (vp * max(1, len(xs)))(*xs)  # noqa: E731
        ia = lambda xs: (i32 * max(1, len(xs)))(*xs)  # noqa: E731
        return self.lib.ref_bench_gop_same(vpa([j[0].h for j in pjobs]), vpa([j[1].h for j in pjobs]),
                                           vpa([j[2].h for j in pjobs]), len(pjobs), vpa([j[0].h for j in bjobs]),
                                           vpa([j[1].h for j in bjobs]), vpa([j[2].h for j in bjobs]),
                                           vpa([j[3].h for j in bjobs]), ia([j[4] for j in bjobs]),
                                           ia([j[5] for j in bjobs]), ia([j[6] for j in bjobs]), len(bjobs), threads)

    def bench_analysis_multi(self, jobs, threads):
        """Wall ns over (Reference, cur RefFrame, ref RefFrame) jobs, each with its own config."""
        hs = (vp * len(jobs))(*[j[0].h for j in jobs])
        curs = (vp * len(jobs))(*[j[1].h for j in jobs])
        refs = (vp * len(jobs))(*[j[2].h for j in jobs])
        return self.lib.ref_bench_analysis_multi(hs, curs, refs, len(jobs), threads)

    def bench_analysis(self, pairs, threads):
        """Wall ns of analyze_p_picture + choose_transform_mb over (cur, ref) RefFrame pairs."""
        curs = (vp * len(pairs))(*[c.h for c, _ in pairs])
        refs = (vp * len(pairs))(*[r.h for _, r in pairs])
        return self.lib.ref_bench_analysis(self.h, curs, refs, len(pairs), threads)
