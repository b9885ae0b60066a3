"""16-bit cost DSIs (TDV_U16): BT of u8 images at scale 1 in half-units.
The 16-bit DSI must hold exactly twice the float DSI's values (+INF as
0xFFFF), and every consumer -- SGM (each semantics and table, with the
left-right check), WTA, DP -- must give the same maps from it as from the
float DSI, in both layouts."""
import numpy as np
import pytest
import torch

from thundervision_b200 import _lib as L
from thundervision_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def pair(W, H, D, seed):
    l, r = syn.make_pair(W, H, D, seed, n_rects=4, slanted=True)[:2]
    return torch.from_numpy(l).cuda(), torch.from_numpy(r).cuda()


def decode(c16):
    v = c16.cpu().numpy().astype(np.float32) * np.float32(0.5)
    v[c16.cpu().numpy() == 0xFFFF] = np.inf
    return v


@pytest.mark.parametrize("layout", ["hwd", "ref"])
@pytest.mark.parametrize("W,H,D", [(640, 480, 64), (97, 41, 130), (33, 20, 600)])
def test_u16_dsi_is_twice_the_float_dsi(ctx, layout, W, H, D):
    l, r = pair(W, H, D, W + H)
    c32 = ctx.cost(l, r, D, kind="bt", layout=layout)
    c16 = ctx.cost(l, r, D, kind="bt", layout=layout, dtype="u16")
    torch.cuda.synchronize()
    np.testing.assert_array_equal(decode(c16), c32.cpu().numpy())


@pytest.mark.parametrize("sem,table", [("ref_cpu", "ref"), ("ref_gpu", "ref"), ("standard", "full")])
@pytest.mark.parametrize("layout", ["hwd", "ref"])
def test_sgm_from_u16_equals_float(ctx, sem, table, layout):
    """640x480 D=64 (the plain GPU config): SGM-8 + WTA + left-right check."""
    l, r = pair(640, 480, 64, 5)
    lf = l.float()
    c32 = ctx.cost(l, r, 64, kind="bt", layout=layout)
    c16 = ctx.cost(l, r, 64, kind="bt", layout=layout, dtype="u16")
    a = ctx.sgm(c32, 10.0, 120.0, guide=lf, table=table, semantics=sem, layout=layout, lr=1, right=True)
    b = ctx.sgm(c16, 10.0, 120.0, guide=lf, table=table, semantics=sem, layout=layout, lr=1, right=True)
    torch.cuda.synchronize()
    assert torch.equal(a["disp"], b["disp"])
    assert torch.equal(a["disp_right"], b["disp_right"])


def test_sgm_adjusted_p2_from_u16(ctx):
    """P2 divided by the guide's intensity step, 4 paths."""
    l, r = pair(320, 240, 32, 8)
    lf = l.float()
    c32 = ctx.cost(l, r, 32, kind="bt")
    c16 = ctx.cost(l, r, 32, kind="bt", dtype="u16")
    a = ctx.sgm(c32, 10.0, 120.0, guide=lf, p2_mode="adjust", paths=4, table="ref", semantics="ref_cpu")
    b = ctx.sgm(c16, 10.0, 120.0, guide=lf, p2_mode="adjust", paths=4, table="ref", semantics="ref_cpu")
    torch.cuda.synchronize()
    assert torch.equal(a["disp"], b["disp"])


@pytest.mark.parametrize("D", [16, 64, 67, 300])
def test_wta_and_dp_from_u16(ctx, D):
    l, r = pair(200, 64, D, D)
    c32 = ctx.cost(l, r, D, kind="bt")
    c16 = ctx.cost(l, r, D, kind="bt", dtype="u16")
    for fn in (lambda c: ctx.wta(c, lr=1, right=True), lambda c: ctx.dp(c)):
        a, b = fn(c32), fn(c16)
        torch.cuda.synchronize()
        for k in a:
            assert torch.equal(a[k], b[k]), k


def test_u16_matches_oracle(ctx, orc):
    """384x288 D=16: SGM over the 16-bit DSI against the oracle's reference
    CPU recurrence over the reference table."""
    l, r = pair(384, 288, 16, 1)
    c16 = ctx.cost(l, r, 16, kind="bt", dtype="u16")
    out = ctx.sgm(c16, 10.0, 120.0, guide=l.float(), table="ref", semantics="ref_cpu")
    torch.cuda.synchronize()
    Lf, Rf = orc.u8_to_f32(l.cpu().numpy()), orc.u8_to_f32(r.cpu().numpy())
    d, _, _ = orc.sgm(orc.bt_cost(Lf, Rf, 16), Lf, 10.0, 120.0, paths=8, table=1, semantics=1)
    np.testing.assert_array_equal(out["disp"].cpu().numpy(), d)


def test_u16_rejections(ctx):
    l, r = pair(64, 48, 16, 3)
    with pytest.raises(L.TdvError) as e:  # SSD values are not half-units
        ctx.cost(l, r, 16, kind="ssd", dtype="u16")
    assert e.value.status == L.TDV_ERR_UNSUPPORTED
    with pytest.raises(L.TdvError) as e:  # [0,1] intensities
        ctx.cost(l, r, 16, kind="bt", dtype="u16", scale=1.0 / 255.0)
    assert e.value.status == L.TDV_ERR_UNSUPPORTED
    c16 = ctx.cost(l, r, 16, kind="bt", dtype="u16")
    agg = torch.empty(c16.shape, dtype=torch.uint16, device="cuda")
    with pytest.raises(L.TdvError) as e:  # the aggregation stays float
        ctx.sgm(c16, 10.0, 120.0, aggreg=agg)
    assert e.value.status == L.TDV_ERR_INVALID_ARG
