"""The I picture's signed intra reconstruction on the device (vc1cu_reconstruct_intra) against the
reference's own Vc1Encoder::reconstruct_i_signed_padded (oracle/_ref, scalar path, trellis 0),
bit for bit on the padded raster: full and cropped rasters, the uniform, non-uniform and half-step
quantisers, PQINDEX 1-2 (the wider DC range), overlap plans none / all / select (the edge source
the transform reads) and a DQUANT plan whose per-MB MQUANT scales the DC predictors."""
import numpy as np
import pytest

from libvc1_b200 import synth
from libvc1_b200.abi import make_params, mbs_of
from oracle.bindings import Reference, ref_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")]

CASES = {
    # (w, h, display, pq, nonuniform, halfqp, overlap, dquant)
    "cif": (176, 144, None, 8, 0, 0, 0, False),
    "cropped_all": (322, 242, (317, 237), 12, 0, 0, 1, False),
    "cropped_select_nonuniform": (208, 120, (203, 113), 9, 1, 0, 2, False),
    "edge_rem1_halfqp": (130, 98, (129, 97), 5, 0, 1, 1, False),
    "pq1": (96, 64, None, 1, 0, 0, 0, False),
    "pq2_nonuniform": (98, 66, None, 2, 1, 0, 0, False),
    "dquant_plan": (176, 144, None, 10, 0, 0, 0, True),
    "dquant_cropped_all": (322, 242, (319, 239), 14, 1, 0, 1, True),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_intra_reconstruction_matches_reference(ctx, case):
    import torch

    w, h, disp, pq, nu, hq, overlap, dquant = CASES[case]
    kw = dict(display_width=disp[0], display_height=disp[1]) if disp else {}
    p = make_params(w, h, pqindex=pq, nonuniform=nu, halfqp=hq, **kw)
    mbw, mbh = mbs_of(p)
    clip = synth.generate(w, h, 1, 90 + pq, n_objects=3, obj_min=12, obj_max=40, sigma=3.0)
    flags = (np.random.default_rng(pq).random(mbw * mbh) < 0.5).astype(np.uint8) if overlap == 2 else None
    want, mq, der = Reference(p).reconstruct_intra(clip.frame(0), overlap, flags, dquant=dquant,
                                                   aq_strength=1.0 if dquant else 0.0)
    if dquant:
        assert len(np.unique(mq)) > 1 and der.any()
    ctx.upload_frame(0, *clip.frame(0))
    d = [torch.zeros((mbh * 16 // s, mbw * 16 // s), dtype=torch.int32, device="cuda") for s in (1, 2, 2)]
    torch.cuda.synchronize()
    ctx.reconstruct_intra(p, 0, *[t.data_ptr() for t in d], overlap=overlap, flags=flags,
                          mquant=mq if dquant else None, derived=der if dquant else None)
    ctx.synchronize()
    for got, exp, c in zip(d, want, "yuv"):
        g = got.cpu().numpy()
        assert np.array_equal(g, exp), (c, np.argwhere(g != exp)[:4])
