"""The allocation-free translation search (vc1cu_global_motion_noalloc) through the C ABI.

Callers that cannot allocate device memory while they run (for example an encoder worker
held to a fixed device-memory budget) use this entry point: it takes device buffers the
caller owns and keeps its search state in a fixed array inside the library. Its results
must be exactly those of the unseeded analysis pass (vc1cu_analyze_p_core's global_dx,
global_dy, global_full_sad), on two calls in a row that share that array.

This file is named to be collected last.
"""
import numpy as np
import pytest

from libvc1_b200 import synth
from libvc1_b200.abi import MV_QPEL, make_params

pytestmark = pytest.mark.gpu


def _noalloc(torch, clip, pairs, rng, width=None, height=None):
    """Runs the entry point on device copies of the pairs' luma planes (pitch = the clip's
    width; width/height may crop them). Returns (dx, dy) per pair, the SADs and the device's
    free memory just before and just after the call."""
    from libvc1_b200.api import global_motion_noalloc

    w = width or clip.width
    h = height or clip.height
    planes = {t: torch.from_numpy(np.ascontiguousarray(clip.frame(t)[0])).cuda() for pair in pairs for t in pair}
    n = len(pairs)
    dxdy = torch.full((2 * n,), -999, dtype=torch.int32, device="cuda")
    sad = torch.full((n,), -1, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream()
    stream.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    global_motion_noalloc([planes[c].data_ptr() for c, _ in pairs], [planes[r].data_ptr() for _, r in pairs],
                          clip.width, w, h, rng, dxdy.data_ptr(), sad.data_ptr(), stream.cuda_stream)
    stream.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    return dxdy.cpu().numpy().reshape(n, 2), sad.cpu().numpy().view(np.uint64), (free_before, free_after)


def _existing(ctx, clip, pairs, **kw):
    p = make_params(clip.width, clip.height, **kw)
    out = []
    for c, r in pairs:
        ctx.upload_frame(0, *clip.frame(c))
        ctx.upload_frame(1, *clip.frame(r))
        t = ctx.analyze_p_core(p, 0, 1, MV_QPEL, False).totals
        out.append((t["global_dx"], t["global_dy"], t["global_full_sad"]))
    return out


def test_noalloc_global_search_matches_analysis_pass_twice(ctx):
    torch = pytest.importorskip("torch")
    # call 1: three CIF pictures, search range 8
    clip = synth.generate(352, 288, 4, 9, global_px=6.0, n_objects=2)
    pairs = [(1, 0), (2, 1), (3, 2)]
    dxdy, sad, _ = _noalloc(torch, clip, pairs, 8)
    want = _existing(ctx, clip, pairs, search_range=8, local_search_range=8)
    assert [(int(a), int(b), int(s)) for (a, b), s in zip(dxdy, sad)] == want
    # call 2, right after it on the same scratch: two pictures of another size, range 32
    clip2 = synth.generate(322, 242, 3, 4, global_px=20.0, n_objects=1)
    pairs2 = [(1, 0), (2, 1)]
    dxdy2, sad2, mem = _noalloc(torch, clip2, pairs2, 32)
    want2 = _existing(ctx, clip2, pairs2, search_range=32, local_search_range=32)
    assert [(int(a), int(b), int(s)) for (a, b), s in zip(dxdy2, sad2)] == want2
    # the call itself took no device memory (the scratch is the library's fixed array)
    assert mem[0] == mem[1]


def test_noalloc_global_search_odd_size_matches_oracle():
    """An odd coding size (a 321x241 crop of the planes, pitch 322) against the oracle's
    global_motion_search restatement, at a short and at the extended range."""
    torch = pytest.importorskip("torch")
    from oracle import Oracle

    o = Oracle()
    clip = synth.generate(322, 242, 3, 12, global_px=9.0, n_objects=1)
    pairs = [(1, 0), (2, 1)]
    p = make_params(322, 242)
    dummy = np.full((121, 161), 128, np.uint8)
    for rng in (12, 32):
        want = []
        for c, r in pairs:
            cur = (np.ascontiguousarray(clip.frame(c)[0][:241, :321]), dummy, dummy)
            ref = (np.ascontiguousarray(clip.frame(r)[0][:241, :321]), dummy, dummy)
            want.append(o.global_motion(p, cur, ref, rng))
        # two calls in a row; the first may load the search kernels into the context (lazy
        # module loading takes device memory), the second must take none
        for call in range(2):
            dxdy, sad, mem = _noalloc(torch, clip, pairs, rng, width=321, height=241)
            assert [(int(a), int(b), int(s)) for (a, b), s in zip(dxdy, sad)] == want
        assert mem[0] == mem[1]


def test_noalloc_rejects_requests_beyond_its_fixed_scratch():
    from libvc1_b200.api import Vc1cuError, global_motion_noalloc

    ptrs = [1] * 17
    with pytest.raises(Vc1cuError) as e:
        global_motion_noalloc(ptrs, ptrs, 64, 64, 48, 8, 8, 8, 0)
    assert e.value.code == 1 and "16 pictures" in str(e.value)
    with pytest.raises(Vc1cuError) as e:
        global_motion_noalloc([1], [1], 64, 64, 48, 33, 8, 8, 0)
    assert e.value.code == 1 and "range" in str(e.value)
