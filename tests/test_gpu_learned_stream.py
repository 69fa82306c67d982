"""The learned proposals inside the reference encoder: a valid VC-1 stream at fixed QP.

The reference CLI built with the CUDA analysis backend (oracle/_ref/vc1enc_cuda, see
tests/test_stream_parity.py) runs the unseeded 1-MV analysis passes of P pictures through the
learned pass when LIBVC1_CUDA_LEARNED names the trained parameters; everything else (mode RD,
transform RD, entropy coding, rate control, reconstruction) stays the reference's. On a held-out
1080p clip with pans of up to +-128 px at QP 6 the test compares the stream's size and the luma
PSNR of the encoder's reconstruction (--recon-out) with the plain backend's, and writes them to
$LIBVC1_LEARNED_REPORT (a JSON file) when that is set.
"""
import json
import os
import subprocess
import time

import numpy as np
import pytest

from libvc1_b200 import learned as lw
from libvc1_b200 import synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ENC_CUDA = os.path.join(ROOT, "oracle", "_ref", "vc1enc_cuda")
FRAMES = 12


def _y4m(path, clip):
    with open(path, "wb") as f:
        f.write(f"YUV4MPEG2 W{clip.width} H{clip.height} F30:1 Ip A1:1 C420jpeg\n".encode())
        for t in range(clip.frames):
            f.write(b"FRAME\n")
            for a in clip.frame(t):
                f.write(a.tobytes())


def _psnr_y(rec_path, clip):
    w, h = clip.width, clip.height
    per = w * h * 3 // 2
    data = np.fromfile(rec_path, np.uint8)
    assert data.size == per * clip.frames
    out = []
    for t in range(clip.frames):
        y = data[t * per:t * per + w * h].reshape(h, w).astype(np.float64)
        mse = np.mean((y - clip.y[t].astype(np.float64)) ** 2)
        out.append(99.0 if mse == 0 else 10.0 * np.log10(255.0 ** 2 / mse))
    return float(np.mean(out))


@pytest.mark.skipif(not (os.path.exists(ENC_CUDA) and os.path.exists(lw.WEIGHTS)),
                    reason="needs oracle/_ref/vc1enc_cuda and the trained parameters")
def test_learned_stream_at_fixed_qp(tmp_path):
    clip = synth.generate(lw.W, lw.H, FRAMES, lw.HELD_SEED0 + 77, global_px=128.0, n_objects=8, obj_min=32, obj_max=96,
                          obj_vel=8.0, sigma=2.5)
    y4m = str(tmp_path / "in.y4m")
    _y4m(y4m, clip)
    weights = str(tmp_path / "weights.f32")
    np.load(lw.WEIGHTS).astype("<f4").tofile(weights)
    args = (f"--cq {lw.QP} --bframes 0 --keyint {FRAMES} --search-range {lw.RANGE} --local-search-range {lw.LOCAL} "
            "--threads 1 --simd auto --compute cuda").split()
    res = {}
    for name in ("plain", "learned"):
        env = dict(os.environ)
        env.pop("LIBVC1_CUDA_LEARNED", None)
        if name == "learned":
            env["LIBVC1_CUDA_LEARNED"] = weights
        out, rec = str(tmp_path / f"{name}.vc1"), str(tmp_path / f"{name}.yuv")
        t0 = time.time()
        r = subprocess.run([ENC_CUDA, "-i", y4m, "-o", out, "--recon-out", rec, *args], env=env, capture_output=True,
                           text=True, timeout=1200)
        assert r.returncode == 0, r.stderr[-2000:]
        res[name] = {"bits": os.path.getsize(out) * 8, "psnr_y": _psnr_y(rec, clip), "encode_s": time.time() - t0}
    res["bits_delta"] = res["learned"]["bits"] / res["plain"]["bits"] - 1.0
    res["psnr_delta_db"] = res["learned"]["psnr_y"] - res["plain"]["psnr_y"]
    res["clip"] = f"{FRAMES} frames 1920x1080, pans up to +-128 px, 8 objects, sigma 2.5, QP {lw.QP}, IPPP"
    if os.environ.get("LIBVC1_LEARNED_REPORT"):
        with open(os.environ["LIBVC1_LEARNED_REPORT"], "w") as f:
            json.dump(res, f, indent=1)
    # a valid stream whose quality stays within a few tenths of a dB of the plain search
    assert res["learned"]["bits"] > 0
    assert res["psnr_delta_db"] > -0.3, res
