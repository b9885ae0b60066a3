"""tdv_stereo_sgm_frames: the fused path over a frame sequence on two lanes
(each with its own planes, volumes and streams).  Every map must equal the
one-call-per-frame result bit for bit, and the oracle's on a sample frame;
frames of a sequence must not leak into one another (the lanes alternate and
reuse their volumes)."""
import numpy as np
import pytest
import torch

from thundervision_b200 import _lib as L
from thundervision_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def frames(W, H, D, n, seed):
    out = []
    for t in range(n):
        l, r = syn.make_pair(W, H, D, seed + 17 * t, n_rects=4, slanted=True)[:2]
        out.append((torch.from_numpy(l).cuda(), torch.from_numpy(r).cuda()))
    return out


@pytest.mark.parametrize("sem,table", [("ref_cpu", "ref"), ("standard", "full"), ("ref_gpu", "ref")])
@pytest.mark.parametrize("n", [1, 2, 3, 6])
def test_sequence_equals_single_calls(ctx, sem, table, n):
    fr = frames(640, 480, 64, n, 5)
    kw = dict(table=table, semantics=sem)
    outs = ctx.stereo_sgm_frames([f[0] for f in fr], [f[1] for f in fr], 64, 10, 120, lr=1, norm=True,
                                 right_disp=True, **kw)
    torch.cuda.synchronize()
    for (l, r), o in zip(fr, outs):
        ref = ctx.stereo_sgm(l, r, 64, 10, 120, lr=1, norm=True, right_disp=True, **kw)
        for key in ("disp", "disp_norm", "disp_right"):
            assert torch.equal(o[key], ref[key]), key


def test_sequence_matches_oracle(ctx, orc):
    """One frame of a sequence against the oracle's reference CPU recurrence
    over the reference table (WTA + left-right check)."""
    fr = frames(384, 288, 16, 3, 9)
    outs = ctx.stereo_sgm_frames([f[0] for f in fr], [f[1] for f in fr], 16, 10, 120, lr=1, table="ref",
                                 semantics="ref_cpu")
    torch.cuda.synchronize()
    l, r = fr[1][0].cpu().numpy(), fr[1][1].cpu().numpy()
    Lf, Rf = orc.u8_to_f32(l), orc.u8_to_f32(r)
    d, _, S = orc.sgm(orc.bt_cost(Lf, Rf, 16), Lf, 10, 120, paths=8, table=1, semantics=1)
    dl, _ = orc.lr_check(S, d, thr=1)
    np.testing.assert_array_equal(outs[1]["disp"].cpu().numpy(), dl)


def test_outputs_rewritten_in_place(ctx):
    """A second call with the first call's outputs writes the same maps into
    them, after other frames ran in between."""
    fr = frames(320, 240, 64, 4, 21)
    ls, rs = [f[0] for f in fr], [f[1] for f in fr]
    outs = ctx.stereo_sgm_frames(ls, rs, 64, 10, 120, lr=1, table="ref", semantics="ref_cpu")
    first = [o["disp"].clone() for o in outs]
    other = frames(320, 240, 64, 3, 99)
    ctx.stereo_sgm_frames([f[0] for f in other], [f[1] for f in other], 64, 10, 120, lr=1, table="ref",
                          semantics="ref_cpu")
    for o in outs:
        o["disp"].fill_(7)
    ctx.stereo_sgm_frames(ls, rs, 64, 10, 120, lr=1, table="ref", semantics="ref_cpu", outs=outs)
    torch.cuda.synchronize()
    for a, o in zip(first, outs):
        assert torch.equal(a, o["disp"])


def test_full_hd_sequence(ctx):
    """Four full-HD D=256 frames under the reference semantics: the headline
    workload's sequence call against one call per frame."""
    vs = syn.VideoStream(seed=3)
    fr = [vs.frame(t)[:2] for t in range(4)]
    ls = [torch.from_numpy(f[0]).cuda() for f in fr]
    rs = [torch.from_numpy(f[1]).cuda() for f in fr]
    outs = ctx.stereo_sgm_frames(ls, rs, 256, 10, 120, lr=1, table="ref", semantics="ref_cpu")
    torch.cuda.synchronize()
    for l, r, o in zip(ls, rs, outs):
        ref = ctx.stereo_sgm(l, r, 256, 10, 120, lr=1, table="ref", semantics="ref_cpu")
        assert torch.equal(o["disp"], ref["disp"])


def test_rejections(ctx):
    fr = frames(64, 48, 16, 2, 1)
    ls, rs = [f[0] for f in fr], [f[1] for f in fr]
    with pytest.raises(L.TdvError) as e:  # float images leave the fused path
        ctx.stereo_sgm_frames([x.float() for x in ls], [x.float() for x in rs], 16, 10, 120)
    assert e.value.status == L.TDV_ERR_UNSUPPORTED
    with pytest.raises(L.TdvError) as e:  # P2 not a multiple of 1/2
        ctx.stereo_sgm_frames(ls, rs, 16, 10, 120.3)
    assert e.value.status == L.TDV_ERR_UNSUPPORTED
    small = torch.zeros((40, 64), dtype=torch.uint8, device="cuda")
    with pytest.raises(L.TdvError) as e:  # frames of different sizes
        ctx.stereo_sgm_frames([ls[0], small], [rs[0], small], 16, 10, 120)
    assert e.value.status == L.TDV_ERR_INVALID_ARG
