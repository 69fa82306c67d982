"""Elementary-stream parity: the reference encoder with its analysis on the CUDA backend.

oracle/_ref/vc1enc_cuda is the reference's own CLI and library built from a copy of its
sources with libvc1_b200/binding/libvc1_cuda.patch applied and libvc1_b200/binding/
encoder_cuda.cpp linked in: with `--compute cuda`, every analyze_p_picture_core,
analyze_b_picture_mode, estimate_intensity_comp and scene_change_score call runs on the device
through the C ABI, while the mode RD, transform RD, entropy coder and rate control stay the
reference's and consume the device's results. The output must be byte-identical to the
unpatched reference CLI (oracle/_ref/vc1enc) on its scalar path (`--simd none`), which is the
reference's bit-exact oracle path.

The clips are the seeded synthetic workloads (libvc1_b200/synth.py) with the benchmark
configurations' shapes: CIF 8 frames IPPPPPPP, and the first 12 frames (one GOP, IBBP) of the
1080p clip.
"""
import os
import subprocess

import pytest

from libvc1_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ENC = os.path.join(ROOT, "oracle", "_ref", "vc1enc")
ENC_CUDA = os.path.join(ROOT, "oracle", "_ref", "vc1enc_cuda")

needs_encoders = pytest.mark.skipif(not (os.path.exists(ENC) and os.path.exists(ENC_CUDA)),
                                    reason="reference encoders not built (make -C oracle ref)")

# The benchmark configurations' encoder knobs.
C1_ARGS = ("--cq 8 --quantizer-type uniform --bframes 0 --keyint 8 --no-scene-cut --fixed-8x8 --no-trellis "
           "--no-aq --no-dquant --threads 1 --search-range 8 --local-search-range 8").split()
C2_ARGS = ("--keyint 12 --bframes 2 --quantizer-type nonuniform --cq 6 --search-range 64 --local-search-range 64 "
           "--no-trellis --no-aq --no-dquant --threads 1").split()
# The encoder's defaults (scene cuts, fade compensation, variable transforms, trellis, AQ, DQUANT,
# search range 1024 with local range 32, B pictures) at a fixed quantiser.
DEFAULT_ARGS = "--cq 5 --keyint 9 --threads 1".split()


def write_y4m(path, clip, fps=30):
    with open(path, "wb") as f:
        f.write(f"YUV4MPEG2 W{clip.width} H{clip.height} F{fps}:1 Ip A1:1 C420jpeg\n".encode())
        for t in range(clip.frames):
            f.write(b"FRAME\n")
            f.write(clip.y[t].tobytes())
            f.write(clip.u[t].tobytes())
            f.write(clip.v[t].tobytes())


def _encode(exe, y4m, out, args, compute):
    return subprocess.Popen([exe, "-i", y4m, "-o", out, *args, "--simd", "none", "--compute", compute],
                            stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)


def _both(tmp_path, clip, args):
    """Encodes the clip with the unpatched reference (CPU) and with the CUDA backend, side by
    side; returns both streams and the CUDA run's log."""
    y4m = str(tmp_path / "in.y4m")
    write_y4m(y4m, clip)
    ref_out, cuda_out = str(tmp_path / "ref.vc1"), str(tmp_path / "cuda.vc1")
    pr = _encode(ENC, y4m, ref_out, args, "cpu")
    pc = _encode(ENC_CUDA, y4m, cuda_out, args, "cuda")
    _, err_c = pc.communicate(timeout=900)
    _, err_r = pr.communicate(timeout=900)
    assert pr.returncode == 0, err_r[-2000:]
    assert pc.returncode == 0, err_c[-2000:]
    with open(ref_out, "rb") as f:
        ref = f.read()
    with open(cuda_out, "rb") as f:
        cud = f.read()
    return ref, cud, err_c


@needs_encoders
def test_patch_leaves_the_cpu_path_unchanged(tmp_path):
    """The patched encoder with --compute cpu writes the unpatched encoder's bytes."""
    clip = synth.generate(96, 64, 6, 21, global_px=3.0, n_objects=1, obj_min=16, obj_max=32)
    y4m = str(tmp_path / "in.y4m")
    write_y4m(y4m, clip)
    outs = []
    for exe in (ENC, ENC_CUDA):
        out = str(tmp_path / (os.path.basename(exe) + ".vc1"))
        p = _encode(exe, y4m, out, "--cq 6 --keyint 6 --bframes 2 --threads 1".split(), "cpu")
        _, err = p.communicate(timeout=300)
        assert p.returncode == 0, err[-2000:]
        with open(out, "rb") as f:
            outs.append(f.read())
    assert len(outs[0]) > 0 and outs[0] == outs[1]


@needs_encoders
def test_cuda_backend_without_a_device_fails_loudly(tmp_path):
    """--compute cuda has no CPU fallback: without a usable device the encode stops with the
    library's error."""
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    clip = synth.generate(64, 48, 2, 3, n_objects=0)
    y4m = str(tmp_path / "in.y4m")
    write_y4m(y4m, clip)
    p = _encode(ENC_CUDA, y4m, str(tmp_path / "x.vc1"), ["--cq", "6"], "cuda")
    _, err = p.communicate(timeout=120)
    assert p.returncode != 0 and "CUDA compute unavailable" in err


@pytest.mark.gpu
@needs_encoders
def test_stream_cif_plain_matches_reference(tmp_path):
    ref, cud, log = _both(tmp_path, synth.cif_plain(frames=8, seed=1), C1_ARGS)
    assert "compute=cuda" in log, log[-2000:]
    assert len(ref) > 0 and cud == ref


@pytest.mark.gpu
@needs_encoders
def test_stream_cif_default_preset_matches_reference(tmp_path):
    """Default knobs: scene-cut scores, fade estimates, Mixed-MV mode RD, variable transforms
    with trellis / AQ / DQUANT on the device's analysis, B pictures at search range 1024."""
    clip = synth.generate(352, 288, 9, 44, global_px=24.0, n_objects=4)
    ref, cud, log = _both(tmp_path, clip, DEFAULT_ARGS)
    assert "compute=cuda" in log, log[-2000:]
    assert len(ref) > 0 and cud == ref


@pytest.mark.gpu
@needs_encoders
def test_stream_1080p_ibbp_gop_matches_reference(tmp_path):
    ref, cud, log = _both(tmp_path, synth.hd1080(frames=12, seed=2), C2_ARGS)
    assert "compute=cuda" in log, log[-2000:]
    assert len(ref) > 0 and cud == ref
