"""Host-side mirror of libvc1's motion-compute backend interface over the vc1cu C ABI.

`CudaComputeContext` has the shape of libvc1's VulkanComputeContext
(src/vulkan_compute.h:26-60): create / device_name / device_index / score_motion_batch /
counters / reset_counters, with the same argument meaning and the same error behaviour
(`score_motion_batch` returns False plus an error string on a recoverable failure; `create`
returns None plus an error string). On top of that interface it exposes the whole-picture
analysis path that the C ABI adds: frames resident in HBM, `analyze_p_core` (one
Vc1Encoder::analyze_p_picture_core pass, src/encoder_motion.cpp:47-442), batched
`core_passes`, `motion_compensate` and `forward_quant`.

There is no CPU fallback: the library must load (libvc1_b200/libvc1cu.so, built by
__graft_entry__.build()) and every device failure is raised.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .abi import (Analysis, BAnalysis, BAnalysisC, BPass, Counters, ERRORS, IcPass, Intensity, Timing, MV_QPEL,
                  METRIC_SAD, METRIC_SATD, Mv, PAnalysisC, Params, PpicCfg, PpicInfo, TDECISION_DTYPE, TrdCfg,
                  mbs_of)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libvc1cu.so")
CHECKED_LIB_PATH = os.path.join(_HERE, "libvc1cu_checked.so")  # the index-checked build
_LIBS = {}

# Every entry point declared in include/vc1cu.h.
EXPORTS = (
    "vc1cu_open", "vc1cu_close", "vc1cu_device_name", "vc1cu_device_index", "vc1cu_last_error",
    "vc1cu_counters_get", "vc1cu_reset_counters", "vc1cu_params_default", "vc1cu_score_motion_batch",
    "vc1cu_score_motion_batch_law", "vc1cu_upload_frame", "vc1cu_download_frame", "vc1cu_analyze_p_core",
    "vc1cu_core_passes", "vc1cu_read_result", "vc1cu_synchronize", "vc1cu_motion_compensate",
    "vc1cu_forward_quant", "vc1cu_forward_quant_device", "vc1cu_set_timing", "vc1cu_timing_get", "vc1cu_stream",
    "vc1cu_measure_int32_peak", "vc1cu_measure_fp64_peak", "vc1cu_debug_index_faults", "vc1cu_global_motion_noalloc", "vc1cu_analyze_b_picture", "vc1cu_b_decide",
    "vc1cu_read_bresult", "vc1cu_estimate_intensity_comp", "vc1cu_estimate_intensity_batch",
    "vc1cu_intensity_compensate", "vc1cu_scene_change_score", "vc1cu_b_predict", "vc1cu_reconstruct",
    "vc1cu_loop_filter_i", "vc1cu_loop_filter_p", "vc1cu_overlap_smooth", "vc1cu_store_signed",
    "vc1cu_estimate_intensity_enqueue", "vc1cu_estimate_intensity_collect",
    "vc1cu_fast_transform_types", "vc1cu_choose_transform", "vc1cu_debug_set_wait_limit", "vc1cu_debug_withhold_publish",
    "vc1cu_synth_frames", "vc1cu_lp_param_count", "vc1cu_lp_create", "vc1cu_lp_destroy", "vc1cu_lp_get_params",
    "vc1cu_lp_set_params", "vc1cu_lp_prepare", "vc1cu_lp_set_labels", "vc1cu_lp_train_step", "vc1cu_lp_gradients",
    "vc1cu_lp_propose", "vc1cu_lp_read_sample", "vc1cu_lp_analyze", "vc1cu_core_passes_multi",
    "vc1cu_graph_begin", "vc1cu_graph_end", "vc1cu_graph_launch", "vc1cu_graph_destroy", "vc1cu_autotune",
    "vc1cu_p_motion_bits", "vc1cu_analyze_p_picture", "vc1cu_b_mode_rd", "vc1cu_loop_filter_p_main",
    "vc1cu_choose_dquant", "vc1cu_reconstruct_intra", "vc1cu_choose_i_overlap",
    "vc1cu_reconstruct_dquant",
)


class LpPass(C.Structure):
    _fields_ = [("cur_id", C.c_int32), ("ref_id", C.c_int32), ("sample", C.c_int32), ("mode", C.c_int32),
                ("out_slot", C.c_int32), ("pqindex", C.c_int32)]


class Pass(C.Structure):
    _fields_ = [("cur_id", C.c_int32), ("ref_id", C.c_int32), ("mode", C.c_int32), ("allow_intra", C.c_int32),
                ("seed_slot", C.c_int32), ("out_slot", C.c_int32), ("pqindex", C.c_int32)]


def load_library(path: str = LIB_PATH):
    """Loads libvc1cu.so (or another build of it, e.g. CHECKED_LIB_PATH) and declares its C
    signatures (no device work)."""
    if path in _LIBS:
        return _LIBS[path]
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: the CUDA backend must be built (__graft_entry__.build())")
    L = C.CDLL(path)
    vp, i32, sz = C.c_void_p, C.c_int, C.c_size_t
    PP = C.POINTER(Params)
    L.vc1cu_open.argtypes = [i32, C.POINTER(vp)]
    L.vc1cu_close.argtypes = [vp]
    L.vc1cu_device_name.argtypes = [vp]
    L.vc1cu_device_name.restype = C.c_char_p
    L.vc1cu_device_index.argtypes = [vp]
    L.vc1cu_last_error.argtypes = [vp]
    L.vc1cu_last_error.restype = C.c_char_p
    L.vc1cu_counters_get.argtypes = [vp, C.POINTER(Counters)]
    L.vc1cu_reset_counters.argtypes = [vp]
    L.vc1cu_params_default.argtypes = [PP, i32, i32]
    L.vc1cu_params_default.restype = None
    L.vc1cu_score_motion_batch.argtypes = [vp, vp, vp, i32, i32, i32, i32, i32, i32, i32, i32, i32, i32, vp, sz, vp]
    L.vc1cu_score_motion_batch_law.argtypes = [vp, PP, i32, vp, vp, i32, i32, i32, i32, i32, i32, i32, vp, sz, vp]
    L.vc1cu_upload_frame.argtypes = [vp, i32, vp, vp, vp, i32, i32]
    L.vc1cu_download_frame.argtypes = [vp, i32, vp, vp, vp]
    L.vc1cu_analyze_p_core.argtypes = [vp, PP, i32, i32, i32, i32, vp, C.POINTER(PAnalysisC), C.POINTER(PAnalysisC)]
    L.vc1cu_core_passes.argtypes = [vp, PP, C.POINTER(Pass), i32]
    L.vc1cu_core_passes_multi.argtypes = [vp, PP, C.POINTER(Pass), i32]
    L.vc1cu_graph_begin.argtypes = [vp]
    L.vc1cu_graph_end.argtypes = [vp, C.POINTER(i32)]
    L.vc1cu_graph_launch.argtypes = [vp, i32]
    L.vc1cu_graph_destroy.argtypes = [vp, i32]
    L.vc1cu_autotune.argtypes = [vp, PP, C.POINTER(Pass), i32, i32, C.POINTER(i32), C.POINTER(i32),
                                 C.POINTER(C.c_double)]
    L.vc1cu_read_result.argtypes = [vp, i32, C.POINTER(PAnalysisC)]
    L.vc1cu_synchronize.argtypes = [vp]
    L.vc1cu_motion_compensate.argtypes = [vp, PP, i32, i32, i32, i32]
    L.vc1cu_forward_quant.argtypes = [vp, PP, i32, i32, i32, vp, vp]
    L.vc1cu_forward_quant_device.argtypes = [vp, PP, i32, i32, i32, vp, vp]
    L.vc1cu_set_timing.argtypes = [vp, i32]
    L.vc1cu_synth_frames.argtypes = [vp, vp, i32, i32, i32]
    L.vc1cu_lp_param_count.argtypes = []
    L.vc1cu_lp_create.argtypes = [vp, i32, i32, i32, i32, i32, C.c_uint64, C.POINTER(vp)]
    L.vc1cu_lp_destroy.argtypes = [vp]
    L.vc1cu_lp_get_params.argtypes = [vp, vp]
    L.vc1cu_lp_set_params.argtypes = [vp, vp]
    L.vc1cu_lp_prepare.argtypes = [vp, i32, i32, i32]
    L.vc1cu_lp_set_labels.argtypes = [vp, i32, i32]
    L.vc1cu_lp_train_step.argtypes = [vp, vp, i32, C.c_float, C.POINTER(C.c_float)]
    L.vc1cu_lp_gradients.argtypes = [vp, vp, i32, vp, C.POINTER(C.c_float)]
    L.vc1cu_lp_propose.argtypes = [vp, i32, i32]
    L.vc1cu_lp_read_sample.argtypes = [vp, i32, vp, vp, vp, vp]
    L.vc1cu_lp_analyze.argtypes = [vp, PP, C.POINTER(LpPass), i32, i32]
    L.vc1cu_debug_set_wait_limit.argtypes = [vp, i32]
    L.vc1cu_debug_withhold_publish.argtypes = [vp, i32, i32]
    L.vc1cu_timing_get.argtypes = [vp, C.POINTER(Timing)]
    L.vc1cu_stream.argtypes = [vp]
    L.vc1cu_stream.restype = vp
    L.vc1cu_measure_int32_peak.argtypes = [vp, C.POINTER(C.c_double)]
    L.vc1cu_measure_fp64_peak.argtypes = [vp, C.POINTER(C.c_double)]
    L.vc1cu_debug_index_faults.argtypes = [C.POINTER(C.c_uint), C.POINTER(C.c_ulonglong), i32]
    L.vc1cu_choose_transform.argtypes = [vp, PP, C.POINTER(TrdCfg), i32, i32, vp, vp, vp]
    L.vc1cu_choose_dquant.argtypes = [vp, PP, C.POINTER(TrdCfg), i32, i32, i32, i32, vp, vp, vp, vp]
    L.vc1cu_reconstruct_dquant.argtypes = [vp, PP, i32, vp, i32, vp, vp, vp, i32]
    L.vc1cu_reconstruct_intra.argtypes = [vp, PP, C.POINTER(TrdCfg), i32, i32, vp, vp, vp, vp, vp, vp]
    L.vc1cu_choose_i_overlap.argtypes = [vp, PP, C.POINTER(TrdCfg), i32, vp, vp, C.POINTER(i32), vp]
    L.vc1cu_p_motion_bits.argtypes = [vp, PP, i32, i32, i32, C.POINTER(C.c_uint64)]
    L.vc1cu_analyze_p_picture.argtypes = [vp, PP, C.POINTER(PpicCfg), i32, i32, i32, i32, i32, C.POINTER(PpicInfo)]
    L.vc1cu_b_mode_rd.argtypes = [vp, PP, C.POINTER(PpicCfg), i32, i32, i32, i32, i32, i32, C.POINTER(i32),
                                  C.POINTER(C.c_double)]
    L.vc1cu_analyze_b_picture.argtypes = [vp, PP, i32, i32, i32, vp, vp, i32, i32, i32, C.POINTER(BAnalysisC)]
    L.vc1cu_b_decide.argtypes = [vp, PP, C.POINTER(BPass), i32]
    L.vc1cu_read_bresult.argtypes = [vp, i32, C.POINTER(BAnalysisC)]
    L.vc1cu_estimate_intensity_comp.argtypes = [vp, PP, i32, i32, vp, C.POINTER(Intensity)]
    L.vc1cu_estimate_intensity_batch.argtypes = [vp, PP, C.POINTER(IcPass), i32, C.POINTER(Intensity)]
    L.vc1cu_intensity_compensate.argtypes = [vp, i32, C.POINTER(Intensity), i32]
    L.vc1cu_b_predict.argtypes = [vp, PP, i32, i32, i32, i32, i32]
    L.vc1cu_reconstruct.argtypes = [vp, PP, i32, vp, i32, vp, i32]
    L.vc1cu_loop_filter_i.argtypes = [vp, PP, i32]
    L.vc1cu_fast_transform_types.argtypes = [vp, PP, i32, i32, vp]
    L.vc1cu_loop_filter_p.argtypes = [vp, PP, i32, vp, vp, vp, vp]
    L.vc1cu_loop_filter_p_main.argtypes = [vp, PP, i32, vp, vp, vp, vp]
    L.vc1cu_overlap_smooth.argtypes = [vp, PP, vp, vp, vp, vp, i32]
    L.vc1cu_estimate_intensity_enqueue.argtypes = [vp, PP, vp, i32, C.POINTER(C.c_int64)]
    L.vc1cu_estimate_intensity_collect.argtypes = [vp, C.c_int64, vp, i32]
    L.vc1cu_store_signed.argtypes = [vp, PP, vp, vp, vp, i32, vp, i32]
    L.vc1cu_scene_change_score.argtypes = [vp, PP, i32, i32, i32, C.c_double, C.POINTER(C.c_double)]
    for name in EXPORTS:
        getattr(L, name)  # AttributeError if the library lacks a declared entry point
    _LIBS[path] = L
    return L


class Vc1cuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def _u8(a):
    return np.ascontiguousarray(a, dtype=np.uint8)


class CudaComputeContext:
    """VulkanComputeContext's shape over the CUDA backend (one context per device)."""

    def __init__(self, handle, lib):
        self._h = handle
        self._L = lib

    # --- VulkanComputeContext::create / device_name / device_index -----------------------
    @staticmethod
    def create(requested_device: int = -1, library: str | None = None):
        """Returns (context, "") or (None, error) like VulkanComputeContext::create. `library`
        selects another build of the backend (e.g. CHECKED_LIB_PATH)."""
        L = load_library(library or LIB_PATH)
        h = C.c_void_p()
        rc = L.vc1cu_open(requested_device, C.byref(h))
        if rc:
            return None, L.vc1cu_last_error(None).decode()
        return CudaComputeContext(h, L), ""

    def close(self):
        if self._h:
            self._L.vc1cu_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def device_name(self) -> str:
        return self._L.vc1cu_device_name(self._h).decode()

    def device_index(self) -> int:
        return self._L.vc1cu_device_index(self._h)

    def last_error(self) -> str:
        return self._L.vc1cu_last_error(self._h).decode()

    def _check(self, rc):
        if rc:
            raise Vc1cuError(rc, self.last_error())

    # --- VulkanComputeContext::score_motion_batch ----------------------------------------
    def score_motion_batch(self, cur, ref, width, height, x0, y0, bw, bh, sample_stride, bilinear, rnd, metric,
                           candidates):
        """Returns (ok, costs, error) with the semantics of score_motion_batch
        (src/vulkan_compute.h:42-51): costs are uint64 per candidate."""
        cand = np.ascontiguousarray(candidates, np.int32).reshape(-1, 2)
        costs = np.zeros(len(cand), np.uint64)
        cur, ref = _u8(cur), _u8(ref)
        rc = self._L.vc1cu_score_motion_batch(self._h, cur.ctypes.data, ref.ctypes.data, width, height, x0, y0, bw, bh,
                                             sample_stride, int(bilinear), int(rnd), metric, cand.ctypes.data,
                                             len(cand), costs.ctypes.data)
        if rc:
            return False, np.zeros(0, np.uint64), self.last_error()
        return True, costs, ""

    def score_motion_batch_law(self, params: Params, law, cur, ref, x0, y0, bw, bh, sample_stride, mode, metric,
                               candidates):
        cand = np.ascontiguousarray(candidates, np.int32).reshape(-1, 2)
        costs = np.zeros(len(cand), np.uint64)
        cur, ref = _u8(cur), _u8(ref)
        self._check(self._L.vc1cu_score_motion_batch_law(self._h, C.byref(params), law, cur.ctypes.data,
                                                         ref.ctypes.data, x0, y0, bw, bh, sample_stride, mode,
                                                         metric, cand.ctypes.data, len(cand), costs.ctypes.data))
        return costs

    # --- VulkanComputeContext::counters / reset_counters ---------------------------------
    def counters(self) -> dict:
        c = Counters()
        self._check(self._L.vc1cu_counters_get(self._h, C.byref(c)))
        return {f[0]: getattr(c, f[0]) for f in Counters._fields_}

    def reset_counters(self):
        self._check(self._L.vc1cu_reset_counters(self._h))

    def synth_frames(self, cfg, first: int, count: int, frame_id0: int):
        """Frames first..first+count-1 of the synthetic clip `cfg` (libvc1_b200.synth.make_cfg)
        generated on the device into frame slots frame_id0.. (asynchronous)."""
        self._check(self._L.vc1cu_synth_frames(self._h, C.byref(cfg), first, count, frame_id0))

    def debug_set_wait_limit(self, log2_polls: int):
        """Wavefront waits give up after 2**log2_polls polls (6..24) in later core launches."""
        self._check(self._L.vc1cu_debug_set_wait_limit(self._h, int(log2_polls)))

    def debug_withhold_publish(self, pass_index: int, mb: int):
        """The next core launch does not publish the done flag of (pass_index, mb)."""
        self._check(self._L.vc1cu_debug_withhold_publish(self._h, int(pass_index), int(mb)))

    def set_timing(self, enable: bool):
        self._check(self._L.vc1cu_set_timing(self._h, int(enable)))

    def timing(self) -> dict:
        t = Timing()
        self._check(self._L.vc1cu_timing_get(self._h, C.byref(t)))
        return {f[0]: getattr(t, f[0]) for f in Timing._fields_}

    def measure_int32_peak(self) -> float:
        """32-bit integer lane-ops per second of this device (calibration kernel)."""
        v = C.c_double()
        self._check(self._L.vc1cu_measure_int32_peak(self._h, C.byref(v)))
        return v.value

    def index_faults(self, reset: bool = True):
        """(count, first site, first index) of the index-checked build's record; raises
        Vc1cuError (VC1CU_ERR_UNSUPPORTED) on other builds."""
        n, first = C.c_uint(), C.c_ulonglong()
        rc = self._L.vc1cu_debug_index_faults(C.byref(n), C.byref(first), int(reset))
        if rc:
            raise Vc1cuError(rc, self._L.vc1cu_last_error(None).decode())
        return n.value, first.value >> 40, first.value & ((1 << 40) - 1)

    def measure_fp64_peak(self) -> float:
        """FP64 flops per second of this device (FMA calibration kernel, an FMA counted as two)."""
        v = C.c_double()
        self._check(self._L.vc1cu_measure_fp64_peak(self._h, C.byref(v)))
        return v.value

    def stream_handle(self) -> int:
        """cudaStream_t of this context (every launch is ordered on it)."""
        return self._L.vc1cu_stream(self._h) or 0

    # --- the analysis path -------------------------------------------------------------
    def upload_frame(self, frame_id: int, y, u=None, v=None):
        """Copies one 4:2:0 frame into frame slot `frame_id`. With pinned host arrays the copy
        is asynchronous: keep them unchanged until synchronize()."""
        y = _u8(y)
        h, w = y.shape
        uu = _u8(u) if u is not None else None
        vv = _u8(v) if v is not None else None
        self._check(self._L.vc1cu_upload_frame(self._h, frame_id, y.ctypes.data,
                                               uu.ctypes.data if uu is not None else None,
                                               vv.ctypes.data if vv is not None else None, w, h))

    def upload_frame_ptr(self, frame_id: int, y_ptr: int, u_ptr: int, v_ptr: int, w: int, h: int):
        self._check(self._L.vc1cu_upload_frame(self._h, frame_id, y_ptr, u_ptr, v_ptr, w, h))

    def download_frame(self, frame_id: int, w: int, h: int):
        y = np.zeros((h, w), np.uint8)
        u = np.zeros((h // 2, w // 2), np.uint8)
        v = np.zeros_like(u)
        self._check(self._L.vc1cu_download_frame(self._h, frame_id, y.ctypes.data, u.ctypes.data, v.ctypes.data))
        return y, u, v

    def analyze_p_core(self, params: Params, cur_id: int, ref_id: int, mode: int = MV_QPEL, allow_intra=False,
                       seed=None, seed_distant: Analysis | None = None) -> Analysis:
        mbw, mbh = mbs_of(params)
        out = Analysis.empty(mbw * mbh)
        oc = out.as_c()
        s = None
        if seed is not None:
            s = np.ascontiguousarray(seed, np.int32).reshape(-1, 2)
            if len(s) != mbw * mbh:
                raise ValueError("shared P motion seed has the wrong macroblock count")
        sd = seed_distant.as_c() if seed_distant is not None else None
        self._check(self._L.vc1cu_analyze_p_core(self._h, C.byref(params), cur_id, ref_id, mode, int(allow_intra),
                                                 s.ctypes.data if s is not None else None,
                                                 C.byref(sd) if sd is not None else None, C.byref(oc)))
        return out.take_totals(oc)

    def core_passes(self, params: Params, passes):
        """passes: iterable of (cur_id, ref_id, mode, allow_intra, seed_slot, out_slot[, pqindex])."""
        arr = (Pass * len(passes))(*[Pass(*p) for p in passes])
        self._check(self._L.vc1cu_core_passes(self._h, C.byref(params), arr, len(passes)))

    def core_passes_multi(self, params_list, passes):
        """Passes over pictures of different sizes in one launch: params_list[i] is pass i's
        parameter block; passes as for core_passes."""
        arr = (Pass * len(passes))(*[Pass(*p) for p in passes])
        pp = (Params * len(params_list))(*params_list)
        self._check(self._L.vc1cu_core_passes_multi(self._h, pp, arr, len(passes)))

    def graph_begin(self):
        self._check(self._L.vc1cu_graph_begin(self._h))

    def graph_end(self) -> int:
        g = C.c_int()
        self._check(self._L.vc1cu_graph_end(self._h, C.byref(g)))
        return g.value

    def graph_launch(self, graph_id: int):
        self._check(self._L.vc1cu_graph_launch(self._h, graph_id))

    def graph_destroy(self, graph_id: int):
        self._check(self._L.vc1cu_graph_destroy(self._h, graph_id))

    def autotune(self, params, passes):
        """params: one Params (one raster) or a list with one per pass (vc1cu_core_passes_multi).
        Returns (warps per block, blocks per SM or 0, ms per launch) of the fastest shape."""
        arr = (Pass * len(passes))(*[Pass(*p) for p in passes])
        multi = isinstance(params, (list, tuple))
        pp = (Params * len(params))(*params) if multi else C.byref(params)
        w, b, ms = C.c_int(), C.c_int(), C.c_double()
        self._check(self._L.vc1cu_autotune(self._h, pp, arr, len(passes), int(multi), C.byref(w), C.byref(b),
                                           C.byref(ms)))
        return w.value, b.value, ms.value

    def read_result(self, params: Params, slot: int) -> Analysis:
        mbw, mbh = mbs_of(params)
        out = Analysis.empty(mbw * mbh)
        oc = out.as_c()
        self._check(self._L.vc1cu_read_result(self._h, slot, C.byref(oc)))
        return out.take_totals(oc)

    def synchronize(self):
        self._check(self._L.vc1cu_synchronize(self._h))

    def estimate_intensity_comp(self, params: Params, cur_id: int, ref_id: int, mvs) -> tuple:
        """Vc1Encoder::estimate_intensity_comp (src/encoder_motion_compensation.cpp:296-348) along a
        host 1-MV field: (enabled, LUMSCALE, LUMSHIFT)."""
        mbw, mbh = mbs_of(params)
        m = np.ascontiguousarray(mvs, np.int32).reshape(-1, 2)
        if len(m) != mbw * mbh:
            raise ValueError("MV field has the wrong macroblock count")
        out = Intensity()
        self._check(self._L.vc1cu_estimate_intensity_comp(self._h, C.byref(params), cur_id, ref_id, m.ctypes.data,
                                                          C.byref(out)))
        return out.as_tuple()

    def estimate_intensity_batch(self, params: Params, passes) -> list:
        """passes: iterable of (cur_id, ref_id, mv_slot); one estimate per picture."""
        arr = (IcPass * max(1, len(passes)))(*[IcPass(*q) for q in passes])
        out = (Intensity * max(1, len(passes)))()
        self._check(self._L.vc1cu_estimate_intensity_batch(self._h, C.byref(params), arr, len(passes), out))
        return [out[i].as_tuple() for i in range(len(passes))]

    def estimate_intensity_enqueue(self, params: Params, passes) -> tuple:
        """The batch's device work, enqueued without waiting; returns (ticket, n) for
        estimate_intensity_collect."""
        arr = (IcPass * max(1, len(passes)))(*[IcPass(*q) for q in passes])
        t = C.c_int64()
        self._check(self._L.vc1cu_estimate_intensity_enqueue(self._h, C.byref(params), arr, len(passes), C.byref(t)))
        return t.value, len(passes)

    def estimate_intensity_collect(self, ticket) -> list:
        """Waits for an enqueued batch alone and returns its estimates."""
        t, n = ticket
        out = (Intensity * max(1, n))()
        self._check(self._L.vc1cu_estimate_intensity_collect(self._h, t, out, n))
        return [out[i].as_tuple() for i in range(n)]

    def scene_change_score(self, params: Params, cur_id: int, ref_id: int, fade_compensation: bool = True,
                           scene_threshold: float = 28.0) -> float:
        """Vc1Encoder::scene_change_score (src/encoder_motion.cpp:599-676): the scene-cut score of
        cur_id against ref_id (a cut when it reaches the encoder's scene threshold)."""
        out = C.c_double()
        self._check(self._L.vc1cu_scene_change_score(self._h, C.byref(params), cur_id, ref_id, int(fade_compensation),
                                                     float(scene_threshold), C.byref(out)))
        return out.value

    def intensity_compensate(self, ref_id: int, ic, out_id: int):
        """Frame slot out_id = the intensity-compensated reference of ref_id (intensity_compensated_reference)."""
        k = Intensity(*ic)
        self._check(self._L.vc1cu_intensity_compensate(self._h, ref_id, C.byref(k), out_id))

    def analyze_b_picture(self, params: Params, cur_id: int, past_id: int, future_id: int, anchor_mvs, anchor_4mv,
                          fraction_num: int, fraction_den: int, mode: int = MV_QPEL) -> BAnalysis:
        """One Vc1Encoder::analyze_b_picture_mode (src/encoder_motion.cpp:753-1005): forward and
        backward core passes plus the per-macroblock B mode decision. anchor_mvs / anchor_4mv are
        the future P anchor's MVs and Mixed-MV flags."""
        mbw, mbh = mbs_of(params)
        am = np.ascontiguousarray(anchor_mvs, np.int32).reshape(-1, 2)
        a4 = np.ascontiguousarray(anchor_4mv, np.uint8).reshape(-1)
        if len(am) != mbw * mbh or len(a4) != mbw * mbh:
            raise ValueError("B analysis needs the future anchor's collocated P MV/type fields")
        out = BAnalysis.empty(mbw * mbh)
        oc = out.as_c()
        self._check(self._L.vc1cu_analyze_b_picture(self._h, C.byref(params), cur_id, past_id, future_id,
                                                    am.ctypes.data, a4.ctypes.data, fraction_num, fraction_den,
                                                    mode, C.byref(oc)))
        return out.take_totals(oc)

    def b_decide(self, params: Params, bpasses):
        """bpasses: iterable of (cur_id, past_id, future_id, fwd_slot, bwd_slot, anchor_slot,
        fraction_num, fraction_den, mode, out_bslot[, pqindex])."""
        arr = (BPass * len(bpasses))(*[BPass(*b) for b in bpasses])
        self._check(self._L.vc1cu_b_decide(self._h, C.byref(params), arr, len(bpasses)))

    def b_predict(self, params: Params, bslot: int, cur_id: int, past_id: int, future_id: int, pred_id: int):
        """Frame slot pred_id = the prediction of the B analysis in bslot (Forward / Backward /
        Direct / Interpolated motion compensation, block means for B-intra)."""
        self._check(self._L.vc1cu_b_predict(self._h, C.byref(params), bslot, cur_id, past_id, future_id, pred_id))

    def read_bresult(self, params: Params, bslot: int) -> BAnalysis:
        mbw, mbh = mbs_of(params)
        out = BAnalysis.empty(mbw * mbh)
        oc = out.as_c()
        self._check(self._L.vc1cu_read_bresult(self._h, bslot, C.byref(oc)))
        return out.take_totals(oc)

    def motion_compensate(self, params: Params, ref_id: int, mv_slot: int, mv_mode: int, pred_id: int):
        self._check(self._L.vc1cu_motion_compensate(self._h, C.byref(params), ref_id, mv_slot, mv_mode, pred_id))

    def forward_quant(self, params: Params, src_id: int, pred_id: int, type_mask: int = 1):
        mbw, mbh = mbs_of(params)
        nt = bin(type_mask & 15).count("1")
        co = np.zeros((nt, mbw * mbh, 6, 64), np.float64)
        lv = np.zeros((nt, mbw * mbh, 6, 64), np.int16)
        self._check(self._L.vc1cu_forward_quant(self._h, C.byref(params), src_id, pred_id, type_mask,
                                                co.ctypes.data, lv.ctypes.data))
        return co, lv

    def choose_transform(self, params: Params, cfg: TrdCfg, src_id: int, pred_id: int, mquant=None, levels=True):
        """Vc1Encoder::choose_transform_mb for every MB (vc1cu_choose_transform): a structured array of
        TDECISION_DTYPE per MB and, with levels, the chosen levels int16 [mb][6][64]."""
        mbw, mbh = mbs_of(params)
        out = np.zeros(mbw * mbh, TDECISION_DTYPE)
        lv = np.zeros((mbw * mbh, 6, 64), np.int16) if levels else None
        mq = None if mquant is None else np.ascontiguousarray(mquant, np.uint8).reshape(-1)
        if mq is not None and mq.size != mbw * mbh:
            raise ValueError("mquant needs one value per macroblock")
        self._check(self._L.vc1cu_choose_transform(self._h, C.byref(params), C.byref(cfg), src_id, pred_id,
                                                   None if mq is None else mq.ctypes.data, out.ctypes.data,
                                                   None if lv is None else lv.ctypes.data))
        return out, lv

    def choose_dquant(self, params: Params, cfg: TrdCfg, src_id: int, pred_id: int, rate_base, dquant: bool = True,
                      predictable_texture: bool = False, levels: bool = True):
        """Vc1Encoder::choose_dquant_transform_mb for every MB (vc1cu_choose_dquant) from the base
        MQUANTs rate_base: (decisions as TDECISION_DTYPE, chosen MQUANT, levels [mb][6][64] or None)."""
        mbw, mbh = mbs_of(params)
        n = mbw * mbh
        rb = np.ascontiguousarray(rate_base, np.uint8).reshape(-1)
        if rb.size != n:
            raise ValueError("rate_base needs one value per macroblock")
        out = np.zeros(n, TDECISION_DTYPE)
        mq = np.zeros(n, np.uint8)
        lv = np.zeros((n, 6, 64), np.int16) if levels else None
        self._check(self._L.vc1cu_choose_dquant(self._h, C.byref(params), C.byref(cfg), int(dquant),
                                                int(predictable_texture), src_id, pred_id, rb.ctypes.data,
                                                out.ctypes.data, mq.ctypes.data, None if lv is None else lv.ctypes.data))
        return out, mq, lv

    def p_motion_bits(self, params: Params, slot: int, mode: int, intensity: bool = False) -> int:
        """Vc1Encoder::estimate_p_motion_bits of the analysis in result slot `slot` (made in mode)."""
        out = C.c_uint64()
        self._check(self._L.vc1cu_p_motion_bits(self._h, C.byref(params), slot, mode, int(intensity), C.byref(out)))
        return out.value

    def analyze_p_picture(self, params: Params, cfg: PpicCfg, cur_id: int, ref_id: int, out_slot: int,
                          scratch_slot: int, scratch_frame: int) -> PpicInfo:
        """Vc1Encoder::analyze_p_picture on the device (vc1cu_analyze_p_picture): the final analysis
        lands in out_slot (read it with read_result); returns the decision record."""
        info = PpicInfo()
        self._check(self._L.vc1cu_analyze_p_picture(self._h, C.byref(params), C.byref(cfg), cur_id, ref_id, out_slot,
                                                    scratch_slot, scratch_frame, C.byref(info)))
        return info

    def b_mode_rd(self, params: Params, cfg: PpicCfg, cur_id: int, past_id: int, future_id: int, bslot_qpel: int,
                  bslot_bilinear: int, pred_id: int):
        """analyze_b_picture's quarter-pel versus bilinear choice (vc1cu_b_mode_rd) for two B-result
        slots: (1 when the bilinear analysis wins else 0, (quarter-pel score, bilinear score))."""
        choice = C.c_int32()
        scores = (C.c_double * 2)()
        self._check(self._L.vc1cu_b_mode_rd(self._h, C.byref(params), C.byref(cfg), cur_id, past_id, future_id,
                                            bslot_qpel, bslot_bilinear, pred_id, C.byref(choice), scores))
        return choice.value, (scores[0], scores[1])

    def fast_transform_types(self, params: Params, src_id: int, pred_id: int):
        """The throughput preset's transform type (1..4) of every MB of src_id against pred_id."""
        mbw, mbh = mbs_of(params)
        out = np.zeros(mbw * mbh, np.uint8)
        self._check(self._L.vc1cu_fast_transform_types(self._h, C.byref(params), src_id, pred_id, out.ctypes.data))
        return out

    def loop_filter(self, params: Params, frame_id: int, block_mvs=None, cbp=None, tt=None, intra=None,
                    main_profile: bool = False):
        """In-place deblocking of frame slot frame_id: the I-like filter when block_mvs is None, else
        the P filter of the coded blocks (per MB: 4 block vectors, 6 patterns, 6 kinds, intra bits),
        with the Main Profile exceptions when main_profile."""
        if block_mvs is None:
            self._check(self._L.vc1cu_loop_filter_i(self._h, C.byref(params), frame_id))
            return
        b = np.ascontiguousarray(block_mvs, np.int32)
        cb, t, i = (np.ascontiguousarray(a, np.uint8) for a in (cbp, tt, intra))
        fn = self._L.vc1cu_loop_filter_p_main if main_profile else self._L.vc1cu_loop_filter_p
        self._check(fn(self._h, C.byref(params), frame_id, b.ctypes.data, cb.ctypes.data, t.ctypes.data, i.ctypes.data))

    def reconstruct_intra(self, params: Params, src_id: int, d_y: int, d_u: int, d_v: int, overlap: int = 0,
                          flags=None, mquant=None, derived=None, cfg: TrdCfg = None):
        """The signed intra reconstruction of I picture src_id into DEVICE int32 planes of the padded
        raster (vc1cu_reconstruct_intra): overlap 0 none / 1 all / 2 select with per-MB flags; the
        DQUANT plan's per-MB MQUANT and derived flags, or None for PQINDEX; cfg's trellis,
        adaptive_quality, aq_strength and hrd_enabled (None: scalar levels)."""
        arrs = [None if a is None else np.ascontiguousarray(a, np.uint8) for a in (flags, mquant, derived)]
        self._check(self._L.vc1cu_reconstruct_intra(self._h, C.byref(params), None if cfg is None else C.byref(cfg),
                                                    src_id, overlap,
                                                    *[None if a is None else a.ctypes.data for a in arrs], d_y, d_u,
                                                    d_v))

    def choose_i_overlap(self, params: Params, src_id: int, mquant=None, derived=None, cfg: TrdCfg = None):
        """The I picture's overlap plan (vc1cu_choose_i_overlap): (mode 0 none / 1 all / 2 select,
        per-MB flags); cfg as for reconstruct_intra."""
        mbw, mbh = mbs_of(params)
        flags = np.zeros(mbw * mbh, np.uint8)
        mode = C.c_int32()
        arrs = [None if a is None else np.ascontiguousarray(a, np.uint8) for a in (mquant, derived)]
        self._check(self._L.vc1cu_choose_i_overlap(self._h, C.byref(params), None if cfg is None else C.byref(cfg),
                                                   src_id,
                                                   *[None if a is None else a.ctypes.data for a in arrs],
                                                   C.byref(mode), flags.ctypes.data))
        return mode.value, flags

    def overlap_smooth(self, params: Params, d_y: int, d_u: int, d_v: int, flags=None, all_edges: bool = False):
        """In-place overlap smoothing of DEVICE int32 signed planes (padded raster, rows packed):
        every 8x8 edge when all_edges, else the edges the per-MB flags enable."""
        f = None if flags is None else np.ascontiguousarray(flags, np.uint8)
        self._check(self._L.vc1cu_overlap_smooth(self._h, C.byref(params), d_y, d_u, d_v,
                                                 None if f is None else f.ctypes.data, int(all_edges)))

    def store_signed(self, params: Params, d_y: int, d_u: int, d_v: int, bias: int, out_id: int, mask=None):
        """Frame slot out_id = clamp(s + bias) of DEVICE int32 signed planes: the whole padded
        raster, or with a per-MB mask only those macroblocks of an existing slot."""
        m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        self._check(self._L.vc1cu_store_signed(self._h, C.byref(params), d_y, d_u, d_v, int(bias),
                                               None if m is None else m.ctypes.data, out_id))

    def reconstruct(self, params: Params, pred_id: int, d_levels: int, type_mask: int, block_types, out_id: int,
                    mquant=None, derived=None):
        """Frame slot out_id = pred_id + the inverse-transformed levels of each block's type
        (device levels in forward_quant_device's layout; block_types: (mbs, 6) TransformType codes),
        dequantised at PQINDEX or at the per-MB MQUANT and derived flags of a DQUANT plan
        (vc1cu_reconstruct_dquant)."""
        bt = np.ascontiguousarray(block_types, np.uint8)
        if mquant is not None:
            mq = np.ascontiguousarray(mquant, np.uint8)
            der = None if derived is None else np.ascontiguousarray(derived, np.uint8)
            self._check(self._L.vc1cu_reconstruct_dquant(self._h, C.byref(params), pred_id, d_levels, type_mask,
                                                          bt.ctypes.data, mq.ctypes.data,
                                                          None if der is None else der.ctypes.data, out_id))
            return
        self._check(self._L.vc1cu_reconstruct(self._h, C.byref(params), pred_id, d_levels, type_mask, bt.ctypes.data,
                                              out_id))

    def forward_quant_device(self, params: Params, src_id: int, pred_id: int, type_mask: int, d_coeffs: int,
                             d_levels: int):
        self._check(self._L.vc1cu_forward_quant_device(self._h, C.byref(params), src_id, pred_id, type_mask,
                                                       d_coeffs, d_levels))


def global_motion_noalloc(cur_ptrs, ref_ptrs, pitch: int, width: int, height: int, search_range: int,
                          d_dxdy: int, d_sad: int, stream: int = 0):
    """Whole-frame translation search of len(cur_ptrs) pictures without any device allocation.

    For callers that cannot allocate device memory while they run: every pointer is a
    device address the caller already owns (luma planes, int32[2n] and uint64[n] outputs),
    and the search state lives in a fixed array inside the library (at most 16 pictures
    per call, search_range 0..32). Enqueued on `stream` (a cudaStream_t handle); the
    results are ready once that stream is synchronised. Calls on one device must not
    overlap on the GPU: they share that array.
    """
    L = load_library()
    n = len(cur_ptrs)
    cur = (C.c_void_p * max(n, 1))(*cur_ptrs)
    ref = (C.c_void_p * max(n, 1))(*ref_ptrs)
    err = C.create_string_buffer(256)
    L.vc1cu_global_motion_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                               C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t]
    L.vc1cu_global_motion_noalloc.restype = C.c_int
    rc = L.vc1cu_global_motion_noalloc(cur, ref, pitch, width, height, search_range, n, d_dxdy, d_sad, stream or None,
                                       err, 256)
    if rc:
        raise Vc1cuError(rc, err.value.decode())


class LearnedProposals:
    """The learned motion-vector proposals of one context (vc1cu_lp_*, include/vc1cu.h): a
    network for one raster and search range holding `capacity` samples (a picture pair's
    features, translation hint, labels, candidates and fallback flags)."""

    def __init__(self, ctx: "CudaComputeContext", width: int, height: int, search_range: int, capacity: int,
                 max_batch: int = 8, seed: int = 1):
        self._L = ctx._L
        self.ctx = ctx
        self.width, self.height, self.range = width, height, search_range
        self.mbw, self.mbh = (width + 15) // 16, (height + 15) // 16
        self.w4, self.h4 = 4 * self.mbw, 4 * self.mbh
        self.capacity, self.max_batch = capacity, max_batch
        h = C.c_void_p()
        ctx._check(self._L.vc1cu_lp_create(ctx._h, width, height, search_range, capacity, max_batch, seed, C.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            self._L.vc1cu_lp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def param_count() -> int:
        return int(load_library().vc1cu_lp_param_count())

    def params(self) -> np.ndarray:
        out = np.zeros(self.param_count(), np.float32)
        self.ctx._check(self._L.vc1cu_lp_get_params(self._h, out.ctypes.data))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        self.ctx._check(self._L.vc1cu_lp_set_params(self._h, p.ctypes.data))

    def prepare(self, cur_id: int, ref_id: int, sample: int):
        self.ctx._check(self._L.vc1cu_lp_prepare(self._h, cur_id, ref_id, sample))

    def set_labels(self, sample: int, result_slot: int):
        self.ctx._check(self._L.vc1cu_lp_set_labels(self._h, sample, result_slot))

    def train_step(self, samples, lr: float) -> float:
        s = np.ascontiguousarray(samples, np.int32)
        loss = C.c_float()
        self.ctx._check(self._L.vc1cu_lp_train_step(self._h, s.ctypes.data, len(s), lr, C.byref(loss)))
        return float(loss.value)

    def gradients(self, samples):
        s = np.ascontiguousarray(samples, np.int32)
        g = np.zeros(self.param_count(), np.float32)
        loss = C.c_float()
        self.ctx._check(self._L.vc1cu_lp_gradients(self._h, s.ctypes.data, len(s), g.ctypes.data, C.byref(loss)))
        return float(loss.value), g

    def propose(self, first_sample: int, n: int = 1):
        self.ctx._check(self._L.vc1cu_lp_propose(self._h, first_sample, n))

    def read_sample(self, sample: int):
        """(features (H4, W4, 16) bf16 bit patterns, hint (2,), candidates (mbs, 4, 2), fallback (mbs,))."""
        mbs = self.mbw * self.mbh
        f = np.zeros((self.h4, self.w4, 16), np.uint16)
        h = np.zeros(2, np.int32)
        c = np.zeros((mbs, 4, 2), np.int32)
        fb = np.zeros(mbs, np.uint8)
        self.ctx._check(self._L.vc1cu_lp_read_sample(self._h, sample, f.ctypes.data, h.ctypes.data, c.ctypes.data,
                                                     fb.ctypes.data))
        return f, h, c, fb

    def analyze(self, params: Params, passes, fallback: bool = True):
        """passes: (cur_id, ref_id, sample, mode, out_slot[, pqindex]) tuples."""
        arr = (LpPass * len(passes))(*[LpPass(*(tuple(q) + (0,) * (6 - len(q)))) for q in passes])
        self.ctx._check(self._L.vc1cu_lp_analyze(self._h, C.byref(params), arr, len(passes), int(fallback)))


__all__ = ["CudaComputeContext", "Vc1cuError", "Pass", "load_library", "EXPORTS", "METRIC_SAD", "METRIC_SATD",
           "global_motion_noalloc", "LearnedProposals"]
