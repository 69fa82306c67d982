"""The C-ABI library loads and exports every entry point include/vc1cu.h declares (no GPU)."""
import ctypes as C
import os
import re

from libvc1_b200 import abi, api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "vc1cu.h")).read()
    return sorted(set(re.findall(r"\b(vc1cu_[a-z_0-9]+)\s*\(", text)))


def test_header_and_python_export_lists_agree():
    assert declared_functions() == sorted(api.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(api.LIB_PATH)
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_struct_layouts_match_header():
    # vc1cu_params: 18 int32 + 2 double; vc1cu_panalysis: 9 pointers + 2 double + 5 u64 + 2 i32 + u64
    assert C.sizeof(abi.Params) == 18 * 4 + 2 * 8
    assert C.sizeof(abi.Mv) == 8
    assert C.sizeof(abi.PAnalysisC) == 9 * 8 + 2 * 8 + 5 * 8 + 2 * 4 + 8
    assert C.sizeof(abi.Counters) == 7 * 8
    assert C.sizeof(abi.Timing) == 5 * 8 + 2 * 8
    assert C.sizeof(api.Pass) == 7 * 4


def test_params_default_matches_reference_defaults():
    lib = api.load_library()
    p = abi.Params()
    lib.vc1cu_params_default(C.byref(p), 1920, 1080)
    mine = abi.make_params(1920, 1080)
    for name, _ in abi.Params._fields_:
        assert getattr(p, name) == getattr(mine, name), name


def test_open_without_device_reports_error_not_crash():
    import torch

    if torch.cuda.is_available():
        return
    ctx, err = api.CudaComputeContext.create(0)
    assert ctx is None and err
