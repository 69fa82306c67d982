"""Seeded synthetic clips for the analysis workloads (bindings of csrc/vc1synth.c).

Each named workload restates one configuration of the benchmark suite with its shapes,
motion and noise statistics: the content is generated, never read from a dataset.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class SynthCfg(C.Structure):
    _fields_ = [
        ("width", C.c_int32), ("height", C.c_int32), ("frames", C.c_int32), ("n_objects", C.c_int32),
        ("seed", C.c_uint64), ("global_range_x_px", C.c_double), ("global_range_y_px", C.c_double),
        ("obj_min", C.c_int32), ("obj_max", C.c_int32), ("obj_vel_px", C.c_double),
        ("zoom", C.c_double), ("noise_sigma", C.c_double),
    ]


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libvc1synth.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing; run __graft_entry__.build() first")
        lib = C.CDLL(path)
        lib.vc1synth_default.argtypes = [C.POINTER(SynthCfg), C.c_int, C.c_int, C.c_int, C.c_uint64]
        lib.vc1synth_generate.argtypes = [C.POINTER(SynthCfg), C.c_void_p, C.c_void_p, C.c_void_p]
        lib.vc1synth_generate.restype = C.c_int
        _LIB = lib
    return _LIB


@dataclass
class Clip:
    width: int
    height: int
    y: np.ndarray  # (frames, h, w) uint8
    u: np.ndarray  # (frames, h/2, w/2)
    v: np.ndarray

    @property
    def frames(self) -> int:
        return self.y.shape[0]

    def frame(self, t: int):
        return self.y[t], self.u[t], self.v[t]


def make_cfg(width: int, height: int, frames: int, seed: int, *, global_px=6.75, global_py=None,
             n_objects=4, obj_min=32, obj_max=96, obj_vel=3.0, zoom=1.0, sigma=2.0) -> SynthCfg:
    """The generator configuration of a clip (the layout of vc1synth_cfg / vc1cu_synth_cfg)."""
    if width % 2 or height % 2:
        raise ValueError("the internal coding raster is even (libvc1 copy_input_picture)")
    cfg = SynthCfg()
    _lib().vc1synth_default(C.byref(cfg), width, height, frames, seed)
    cfg.global_range_x_px = global_px
    cfg.global_range_y_px = global_px if global_py is None else global_py
    cfg.n_objects, cfg.obj_min, cfg.obj_max, cfg.obj_vel_px = n_objects, obj_min, obj_max, obj_vel
    cfg.zoom, cfg.noise_sigma = zoom, sigma
    return cfg


def generate(width: int, height: int, frames: int, seed: int, **kw) -> Clip:
    cfg = make_cfg(width, height, frames, seed, **kw)
    y = np.empty((frames, height, width), np.uint8)
    u = np.empty((frames, height // 2, width // 2), np.uint8)
    v = np.empty_like(u)
    rc = _lib().vc1synth_generate(C.byref(cfg), y.ctypes.data, u.ctypes.data, v.ctypes.data)
    if rc:
        raise RuntimeError(f"vc1synth_generate failed ({rc})")
    return Clip(width, height, y, u, v)


# Named workloads (shapes, motion and noise of each benchmark configuration).
def cif_plain(frames=8, seed=1):
    """352x288, 4 rectangles 32-96 px at +/-3 px/frame, global +/-6.75 px, sigma 2."""
    return generate(352, 288, frames, seed, global_px=6.75, n_objects=4, obj_vel=3.0, sigma=2.0)


def hd1080(frames=60, seed=2):
    """1920x1080 (coded raster 1920x1080, MB raster 120x68), zoom 1.002/frame, 8 objects +/-8 px/frame."""
    return generate(1920, 1080, frames, seed, global_px=6.75, n_objects=8, obj_vel=8.0, zoom=1.002, sigma=2.0)


def long_pan(frames=60, seed=5):
    """1920x1080 camera pans up to 200 px/frame horizontal, 60 px vertical, 4 objects."""
    return generate(1920, 1080, frames, seed, global_px=200.0, global_py=60.0, n_objects=4, obj_vel=8.0,
                    sigma=2.0)


def fade(frame, scale: float, offset: float, seed: int, sigma: float = 1.0):
    """A brightness fade of one picture: luma scale*y + offset plus Gaussian noise (sigma), chroma
    scaled about 128, rounded and clipped to 8 bits (content for the intensity-compensation
    estimate; seeded, so repeatable)."""
    y, u, v = frame
    rng = np.random.default_rng(seed)
    yy = np.clip(np.rint(y.astype(np.float64) * scale + offset + rng.normal(0.0, sigma, y.shape)), 0, 255)
    uu = np.clip(np.rint((u.astype(np.float64) - 128.0) * scale + 128.0), 0, 255)
    vv = np.clip(np.rint((v.astype(np.float64) - 128.0) * scale + 128.0), 0, 255)
    return yy.astype(np.uint8), uu.astype(np.uint8), vv.astype(np.uint8)
