"""Builds the native parts in place: libvc1cu.so (CUDA, sm_100a) and libvc1synth.so (C).

The CUDA library is compiled with nvcc for sm_100a only, with --fmad=false so that the FP64
transform keeps the reference's separately rounded products and sums. Outputs are written
next to this file so that they travel with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
CU_SOURCES = ["vc1cu_api.cu", "vc1cu_core.cu", "vc1cu_global.cu", "vc1cu_xform.cu", "vc1cu_score.cu", "vc1cu_bpic.cu", "vc1cu_ic.cu", "vc1cu_filter.cu",
              "vc1cu_synth.cu", "vc1cu_lp.cu", "vc1cu_moderd.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


# Library variants: name -> (file, extra nvcc defines). "checked" is the index-checked build:
# every guarded shared-memory, frame and table access of the analysis kernels is bounds-checked,
# a violation is counted with its site and skipped (vc1cu_debug_index_faults reads the record).
VARIANTS = {"default": ("libvc1cu.so", ()), "checked": ("libvc1cu_checked.so", ("-DVC1CU_INDEX_CHECK",))}


def build_cuda(force: bool = False, verbose: bool = False, variant: str = "default", out: str | None = None,
               defines=()) -> str:
    name, vdefs = VARIANTS[variant]
    out = out or os.path.join(HERE, name)
    defines = tuple(vdefs) + tuple(defines)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh"))]
    deps.append(os.path.join(HERE, "..", "include", "vc1cu.h"))
    if not force and not _stale(out, deps):
        return out
    objs = []
    procs = []
    tag = os.path.splitext(os.path.basename(out))[0]
    for src in CU_SOURCES:
        obj = os.path.join(CSRC, f"_{tag}_" + src.replace(".cu", ".o"))
        cmd = [_nvcc(), *ARCH, "-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC", *defines,
               "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(-4, "-Xptxas=-v")
        procs.append((subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT), cmd))
        objs.append(obj)
    for p, cmd in procs:
        o, _ = p.communicate()
        if p.returncode:
            raise RuntimeError(f"nvcc failed: {' '.join(cmd)}\n{o.decode()}")
        if verbose:
            sys.stdout.write(o.decode())
    link = [_nvcc(), *ARCH, "-shared", "-o", out, *objs]
    subprocess.run(link, check=True)
    for o in objs:
        os.remove(o)
    return out


def build_synth(force: bool = False) -> str:
    out = os.path.join(HERE, "libvc1synth.so")
    src = os.path.join(CSRC, "vc1synth.c")
    if force or _stale(out, [src, os.path.join(CSRC, "vc1synth.h")]):
        subprocess.run(["gcc", "-std=gnu11", "-O2", "-fPIC", "-ffp-contract=off", "-fopenmp", "-shared", "-o", out, src,
                        "-lm"], check=True)
    return out


def build_all(force: bool = False, verbose: bool = False):
    build_synth(force)
    build_cuda(force, verbose)
    build_cuda(force, verbose, variant="checked")


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose="-v" in sys.argv)
