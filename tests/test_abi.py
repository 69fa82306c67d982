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


# ctypes mirror -> C struct name in include/vc1cu.h
STRUCTS = {"Params": (abi.Params, "vc1cu_params"), "Mv": (abi.Mv, "vc1cu_mv"),
           "PAnalysisC": (abi.PAnalysisC, "vc1cu_panalysis"), "Counters": (abi.Counters, "vc1cu_counters"),
           "Timing": (abi.Timing, "vc1cu_timing"), "Pass": (api.Pass, "vc1cu_pass"),
           "BAnalysisC": (abi.BAnalysisC, "vc1cu_banalysis"), "BPass": (abi.BPass, "vc1cu_bpass"),
           "Intensity": (abi.Intensity, "vc1cu_intensity"), "IcPass": (abi.IcPass, "vc1cu_icpass"),
           "TrdCfg": (abi.TrdCfg, "vc1cu_trd_cfg"), "TDecisionC": (abi.TDecisionC, "vc1cu_tdecision"),
           "PpicCfg": (abi.PpicCfg, "vc1cu_ppic_cfg"), "PpicInfo": (abi.PpicInfo, "vc1cu_ppic_info")}


def test_struct_layouts_match_header(tmp_path):
    """Size and every field offset of the ctypes mirrors equal the C compiler's for the header."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        import pytest

        pytest.skip("no C compiler")
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "vc1cu.h"', "int main(void) {"]
    for key, (cls, cname) in STRUCTS.items():
        lines.append(f'printf("{key} size %zu\\n", sizeof({cname}));')
        for f in cls._fields_:
            lines.append(f'printf("{key} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    want = []
    for key, (cls, _) in STRUCTS.items():
        want.append(f"{key} size {C.sizeof(cls)}")
        want += [f"{key} {f[0]} {getattr(cls, f[0]).offset}" for f in cls._fields_]
    assert [g for g in got if g] == want


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


def test_checked_build_exports_the_same_symbols():
    """The index-checked build is a full copy of the library."""
    lib = C.CDLL(api.CHECKED_LIB_PATH)
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_index_fault_record_only_in_the_checked_build():
    lib = api.load_library()
    n, first = C.c_uint(), C.c_ulonglong()
    assert lib.vc1cu_debug_index_faults(C.byref(n), C.byref(first), 0) == 6  # VC1CU_ERR_UNSUPPORTED
    assert b"index-checked" in lib.vc1cu_last_error(None)
