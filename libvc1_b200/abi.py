"""ctypes mirror of include/vc1cu.h: parameter, motion-vector and result structures.

The structures match the C declarations field for field; `Analysis` owns numpy arrays for
one core pass's per-macroblock results (the layout of libvc1's Vc1Encoder::PAnalysis,
src/encoder_internal.h:346-370) and exposes them to C through a `vc1cu_panalysis`.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

VC1CU_OK = 0
ERRORS = {1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_TIMEOUT", 4: "ERR_OOM", 5: "ERR_STATE", 6: "ERR_UNSUPPORTED"}

METRIC_SAD, METRIC_SATD = 0, 1
MV_QPEL, MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED = 0, 1, 2, 3
MODES = (MV_QPEL, MV_HPEL, MV_HPEL_BILINEAR, MV_MIXED)
LAW_SHADER, LAW_CPU = 0, 1
BAD_COST = (2**64 - 1) // 4


class Mv(C.Structure):
    _fields_ = [("xq", C.c_int32), ("yq", C.c_int32)]


class Params(C.Structure):
    _fields_ = [
        ("width", C.c_int32), ("height", C.c_int32),
        ("display_width", C.c_int32), ("display_height", C.c_int32),
        ("pqindex", C.c_int32), ("halfqp", C.c_int32), ("nonuniform", C.c_int32),
        ("search_range", C.c_int32), ("local_search_range", C.c_int32),
        ("me_algorithm", C.c_int32), ("me_quality", C.c_int32),
        ("subpel", C.c_int32), ("fast_subpel", C.c_int32), ("subpel_range", C.c_int32),
        ("long_range_mode", C.c_int32), ("rnd", C.c_int32), ("disable_p_intra", C.c_int32),
        ("disable_b_intra", C.c_int32),
        ("distant_match_max_mae", C.c_double), ("inter_intra_threshold", C.c_double),
    ]


class PAnalysisC(C.Structure):
    _fields_ = [
        ("mvs", C.c_void_p), ("block_mvs", C.c_void_p), ("use_4mv", C.c_void_p),
        ("use_intra", C.c_void_p), ("screen_sads", C.c_void_p),
        ("inter_intra_cost_ratio", C.c_void_p), ("distant_local_mae", C.c_void_p),
        ("distant_candidate_mae", C.c_void_p), ("distant_match_decision", C.c_void_p),
        ("mean_abs_residual", C.c_double), ("rate_complexity", C.c_double),
        ("motion_sad", C.c_uint64), ("moved_macroblocks", C.c_uint64),
        ("fractional_chroma_macroblocks", C.c_uint64), ("four_mv_macroblocks", C.c_uint64),
        ("intra_macroblocks", C.c_uint64),
        ("global_dx", C.c_int32), ("global_dy", C.c_int32), ("global_full_sad", C.c_uint64),
    ]


class Counters(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("dispatches", "candidates", "frame_uploads",
                                          "frame_upload_bytes", "submit_wait_nanoseconds",
                                          "macroblocks_analysed", "kernel_launches")]


class Timing(C.Structure):
    _fields_ = [("core_ms", C.c_double), ("global_ms", C.c_double), ("totals_ms", C.c_double),
                ("mc_ms", C.c_double), ("xform_ms", C.c_double), ("core_launches", C.c_uint64),
                ("xform_launches", C.c_uint64), ("b_ms", C.c_double), ("ic_ms", C.c_double)]


def make_params(width: int, height: int, **kw) -> Params:
    """Defaults of vc1_param_default (src/encoder_api_helpers.cpp:27-52) for the fields the
    analysis path reads; `width`/`height` are the even internal coding raster."""
    p = Params()
    p.width, p.height = width, height
    p.display_width, p.display_height = 0, 0
    p.pqindex, p.halfqp, p.nonuniform = 8, 0, 0
    p.search_range, p.local_search_range = 1024, 32
    p.me_algorithm, p.me_quality = 0, 2
    p.subpel, p.fast_subpel, p.subpel_range = 1, 0, 1024
    p.long_range_mode, p.rnd, p.disable_p_intra = 0, 0, 0
    p.distant_match_max_mae, p.inter_intra_threshold = 255.0, 0.80
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p


def params_dict(p: Params) -> dict:
    return {f[0]: getattr(p, f[0]) for f in Params._fields_}


def mbs_of(p: Params) -> tuple[int, int]:
    return (p.width + 15) // 16, (p.height + 15) // 16


@dataclass
class Analysis:
    """One core pass's results (host numpy arrays) plus picture totals."""
    mvs: np.ndarray            # (mbs, 2) int32
    block_mvs: np.ndarray      # (mbs, 4, 2) int32
    use_4mv: np.ndarray        # (mbs,) uint8
    use_intra: np.ndarray      # (mbs,) uint8
    screen_sads: np.ndarray    # (mbs,) uint64
    inter_intra_cost_ratio: np.ndarray  # (mbs,) float64
    distant_local_mae: np.ndarray
    distant_candidate_mae: np.ndarray
    distant_match_decision: np.ndarray  # uint8
    totals: dict

    ARRAYS = ("mvs", "block_mvs", "use_4mv", "use_intra", "screen_sads", "inter_intra_cost_ratio",
              "distant_local_mae", "distant_candidate_mae", "distant_match_decision")

    @classmethod
    def empty(cls, mbs: int) -> "Analysis":
        return cls(
            mvs=np.zeros((mbs, 2), np.int32), block_mvs=np.zeros((mbs, 4, 2), np.int32),
            use_4mv=np.zeros(mbs, np.uint8), use_intra=np.zeros(mbs, np.uint8),
            screen_sads=np.zeros(mbs, np.uint64), inter_intra_cost_ratio=np.zeros(mbs, np.float64),
            distant_local_mae=np.zeros(mbs, np.float64), distant_candidate_mae=np.zeros(mbs, np.float64),
            distant_match_decision=np.zeros(mbs, np.uint8), totals={})

    def as_c(self) -> PAnalysisC:
        s = PAnalysisC()
        for name in self.ARRAYS:
            setattr(s, name, getattr(self, name).ctypes.data)
        return s

    def take_totals(self, s: PAnalysisC) -> "Analysis":
        self.totals = {f[0]: getattr(s, f[0]) for f in PAnalysisC._fields_[9:]}
        return self

    def equal(self, other: "Analysis") -> list[str]:
        """Names of fields that differ (bit-exact comparison, doubles by bit pattern)."""
        bad = []
        for name in self.ARRAYS:
            a, b = getattr(self, name), getattr(other, name)
            if a.dtype == np.float64:
                if not np.array_equal(a.view(np.uint64), b.view(np.uint64)):
                    bad.append(name)
            elif not np.array_equal(a, b):
                bad.append(name)
        for k, v in self.totals.items():
            w = other.totals.get(k)
            if isinstance(v, float):
                if np.float64(v).view(np.uint64) != np.float64(w).view(np.uint64):
                    bad.append(k)
            elif v != w:
                bad.append(k)
        return bad


BMB_FORWARD, BMB_BACKWARD, BMB_INTERPOLATED, BMB_DIRECT, BMB_INTRA = 0, 1, 2, 3, 4


class BAnalysisC(C.Structure):
    _fields_ = [
        ("modes", C.c_void_p), ("forward_mvs", C.c_void_p), ("backward_mvs", C.c_void_p),
        ("inter_intra_cost_ratio", C.c_void_p),
        ("forward_distant_local_mae", C.c_void_p), ("forward_distant_candidate_mae", C.c_void_p),
        ("forward_distant_match_decision", C.c_void_p),
        ("backward_distant_local_mae", C.c_void_p), ("backward_distant_candidate_mae", C.c_void_p),
        ("backward_distant_match_decision", C.c_void_p),
        ("forward_macroblocks", C.c_uint64), ("backward_macroblocks", C.c_uint64),
        ("interpolated_macroblocks", C.c_uint64), ("direct_macroblocks", C.c_uint64),
        ("intra_macroblocks", C.c_uint64), ("moved_macroblocks", C.c_uint64),
        ("fractional_chroma_macroblocks", C.c_uint64),
        ("mean_abs_residual", C.c_double), ("rate_complexity", C.c_double),
        ("motion_sad", C.c_uint64), ("motion_bits", C.c_uint64),
        ("mv_mode", C.c_int32), ("reserved", C.c_int32),
    ]


class BPass(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("cur_id", "past_id", "future_id", "fwd_slot", "bwd_slot", "anchor_slot",
                                         "fraction_num", "fraction_den", "mode", "out_bslot", "pqindex")]


@dataclass
class BAnalysis:
    """One B-picture analysis (Vc1Encoder::BAnalysis, src/encoder_internal.h:408-434)."""
    modes: np.ndarray                   # (mbs,) uint8, BMB_*
    forward_mvs: np.ndarray             # (mbs, 2) int32
    backward_mvs: np.ndarray            # (mbs, 2) int32
    inter_intra_cost_ratio: np.ndarray  # (mbs,) float64
    forward_distant_local_mae: np.ndarray
    forward_distant_candidate_mae: np.ndarray
    forward_distant_match_decision: np.ndarray
    backward_distant_local_mae: np.ndarray
    backward_distant_candidate_mae: np.ndarray
    backward_distant_match_decision: np.ndarray
    totals: dict

    ARRAYS = ("modes", "forward_mvs", "backward_mvs", "inter_intra_cost_ratio",
              "forward_distant_local_mae", "forward_distant_candidate_mae", "forward_distant_match_decision",
              "backward_distant_local_mae", "backward_distant_candidate_mae", "backward_distant_match_decision")

    @classmethod
    def empty(cls, mbs: int) -> "BAnalysis":
        f64 = lambda: np.zeros(mbs, np.float64)  # noqa: E731
        return cls(modes=np.zeros(mbs, np.uint8), forward_mvs=np.zeros((mbs, 2), np.int32),
                   backward_mvs=np.zeros((mbs, 2), np.int32), inter_intra_cost_ratio=f64(),
                   forward_distant_local_mae=f64(), forward_distant_candidate_mae=f64(),
                   forward_distant_match_decision=np.zeros(mbs, np.uint8),
                   backward_distant_local_mae=f64(), backward_distant_candidate_mae=f64(),
                   backward_distant_match_decision=np.zeros(mbs, np.uint8), totals={})

    def as_c(self) -> BAnalysisC:
        s = BAnalysisC()
        for name in self.ARRAYS:
            setattr(s, name, getattr(self, name).ctypes.data)
        return s

    def take_totals(self, s: BAnalysisC) -> "BAnalysis":
        self.totals = {f[0]: getattr(s, f[0]) for f in BAnalysisC._fields_[10:-1]}
        return self

    def equal(self, other: "BAnalysis") -> list[str]:
        """Names of fields that differ (bit-exact comparison, doubles by bit pattern)."""
        bad = []
        for name in self.ARRAYS:
            a, b = getattr(self, name), getattr(other, name)
            if a.dtype == np.float64:
                if not np.array_equal(a.view(np.uint64), b.view(np.uint64)):
                    bad.append(name)
            elif not np.array_equal(a, b):
                bad.append(name)
        for k, v in self.totals.items():
            w = other.totals.get(k)
            if isinstance(v, float):
                if np.float64(v).view(np.uint64) != np.float64(w).view(np.uint64):
                    bad.append(k)
            elif v != w:
                bad.append(k)
        return bad


class Intensity(C.Structure):
    """vc1cu_intensity: Vc1Encoder::IntensityComp (enabled, LUMSCALE, LUMSHIFT codes)."""
    _fields_ = [("enabled", C.c_int32), ("lumscale", C.c_int32), ("lumshift", C.c_int32)]

    def as_tuple(self):
        return (int(self.enabled), int(self.lumscale), int(self.lumshift))


class IcPass(C.Structure):
    _fields_ = [("cur_id", C.c_int32), ("ref_id", C.c_int32), ("mv_slot", C.c_int32)]


class TrdCfg(C.Structure):
    """vc1cu_trd_cfg: the transform RD's configuration (EncoderConfig fields and picture choices)."""
    _fields_ = [("trellis", C.c_int32), ("adaptive_quality", C.c_int32), ("aq_strength", C.c_double),
                ("variable_transforms", C.c_int32), ("extended_transform_signaling", C.c_int32),
                ("coding_set", C.c_int32), ("use_vlc", C.c_int32), ("dquantfrm", C.c_int32), ("hrd_enabled", C.c_int32),
                ("frame_type", C.c_int32)]


def make_trd_cfg(**kw) -> TrdCfg:
    """The default presets' values (trellis 1, AQ on at strength 1, variable transforms with
    extended signaling, VLC coding) unless overridden; coding set 1 (high-motion inter)."""
    c = TrdCfg()
    c.trellis, c.adaptive_quality, c.aq_strength = 1, 1, 1.0
    c.variable_transforms, c.extended_transform_signaling = 1, 1
    c.coding_set, c.use_vlc, c.dquantfrm, c.hrd_enabled, c.frame_type = 1, 1, 0, 0, 0
    for k, v in kw.items():
        if not hasattr(c, k):
            raise KeyError(k)
        setattr(c, k, v)
    return c


class PpicCfg(C.Structure):
    """vc1cu_ppic_cfg: the EncoderConfig fields analyze_p_picture reads beyond the parameters."""
    _fields_ = [("trd", TrdCfg), ("fast_transform_rdo", C.c_int32), ("dquant", C.c_int32), ("n_modes", C.c_int32),
                ("fade_compensation", C.c_int32), ("fade_min_gain", C.c_double)]


def make_ppic_cfg(**kw) -> PpicCfg:
    """The reference's EncoderConfig defaults (trellis 1, variable transforms with extended
    signaling, VLC coding, DQUANT on, fast transform RDO off, fade compensation on with a 0.04
    minimum gain) and the four Advanced Profile candidate modes, unless overridden; trd_* keys set
    fields of the transform RD configuration."""
    c = PpicCfg()
    c.trd = make_trd_cfg(adaptive_quality=0, aq_strength=0.0)
    c.fast_transform_rdo, c.dquant, c.n_modes, c.fade_compensation, c.fade_min_gain = 0, 1, 4, 1, 0.04
    for k, v in kw.items():
        if k.startswith("trd_"):
            if not hasattr(c.trd, k[4:]):
                raise KeyError(k)
            setattr(c.trd, k[4:], v)
        elif hasattr(c, k):
            setattr(c, k, v)
        else:
            raise KeyError(k)
    return c


class PpicInfo(C.Structure):
    """vc1cu_ppic_info: what analyze_p_picture decided (mode, fade use, motion bits, candidates)."""
    _fields_ = [("mode", C.c_int32), ("weighted", C.c_int32), ("ic", Intensity), ("motion_bits", C.c_uint64),
                ("cand_bits", C.c_uint64 * 8), ("cand_score", C.c_double * 8)]


class TDecisionC(C.Structure):
    """vc1cu_tdecision: one macroblock's MbTransformDecision."""
    _fields_ = [("type", C.c_uint8), ("signal_level", C.c_uint8), ("cbp", C.c_uint8), ("parent_type", C.c_uint8 * 6),
                ("skip_mask", C.c_uint8 * 6), ("reserved", C.c_uint8), ("estimated_bits", C.c_uint32),
                ("parent_bits", C.c_uint32 * 6), ("distortion", C.c_double), ("parent_distortion", C.c_double * 6)]


# numpy view of an array of vc1cu_tdecision
TDECISION_DTYPE = np.dtype({"names": ["type", "signal_level", "cbp", "parent_type", "skip_mask", "reserved",
                                      "estimated_bits", "parent_bits", "distortion", "parent_distortion"],
                            "formats": [np.uint8, np.uint8, np.uint8, (np.uint8, 6), (np.uint8, 6), np.uint8, np.uint32,
                                        (np.uint32, 6), np.float64, (np.float64, 6)],
                            "offsets": [TDecisionC.type.offset, TDecisionC.signal_level.offset, TDecisionC.cbp.offset,
                                        TDecisionC.parent_type.offset, TDecisionC.skip_mask.offset,
                                        TDecisionC.reserved.offset, TDecisionC.estimated_bits.offset,
                                        TDecisionC.parent_bits.offset, TDecisionC.distortion.offset,
                                        TDecisionC.parent_distortion.offset],
                            "itemsize": C.sizeof(TDecisionC)})


def tdecisions_differ(a: np.ndarray, b: np.ndarray) -> list[str]:
    """Fields of two decision arrays that differ (doubles by bit pattern)."""
    bad = []
    for name in TDECISION_DTYPE.names:
        if name == "reserved":
            continue
        x, y = a[name], b[name]
        if x.dtype == np.float64:
            if not np.array_equal(np.ascontiguousarray(x).view(np.uint64), np.ascontiguousarray(y).view(np.uint64)):
                bad.append(name)
        elif not np.array_equal(x, y):
            bad.append(name)
    return bad
