"""The plain-method configuration at its full size, 640x480, D=64 (8
rectangles + a slanted plane + 2 % salt-and-pepper), through the general
float path (cost DSI, scheduled aggregation passes, WTA, left-right check,
DP), bit-exact to the oracle: the three costs at the configuration's windows
(SSD 5x5, NCC 9x9) and the reference's (SSD 7x7, NCC 3x3); the reference's
CPU and GPU recurrences over its path table in the integer domain (P1 = 10,
P2 = 120) and in the reference's own domain (intensities / 255, P1 = 30/255,
P2 = 150/255 divided by |dI|); WTA + left-right check (threshold 1); DP.
Float costs and sums in the [0,1] domain within 1e-5 relative (the kernels
follow the oracle's rounding order and match exactly in practice); integer
costs, sums and every disparity bit-exact."""
import numpy as np
import pytest
import torch

from thundervision_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

W, H, D = 640, 480, 64
REL = 1e-5


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def close(got, ref):
    np.testing.assert_array_equal(np.isinf(got), np.isinf(ref))
    np.testing.assert_array_equal(np.isnan(got), np.isnan(ref))
    m = np.isfinite(ref)
    np.testing.assert_allclose(got[m], ref[m], rtol=REL, atol=0)


@pytest.fixture(scope="module")
def pair():
    L, R, _, _ = syn.pair_medium(5)
    assert L.shape == (H, W)
    return L, R


@pytest.mark.parametrize("domain", ["integer", "reference"])
@pytest.mark.parametrize("kind,radius", [("bt", 0), ("ssd", 2), ("ssd", 3), ("ncc", 4), ("ncc", 1)])
def test_costs(ctx, orc, pair, domain, kind, radius):
    L, R = pair
    s = np.float32(1) if domain == "integer" else np.float32(1) / np.float32(255)
    Lf, Rf = orc.u8_to_f32(L, s), orc.u8_to_f32(R, s)
    got = host(ctx.cost(dev(L), dev(R), D, kind=kind, radius=radius, scale=float(s)))
    ref = {"bt": lambda: orc.bt_cost(Lf, Rf, D), "ssd": lambda: orc.ssd_cost(Lf, Rf, D, radius),
           "ncc": lambda: orc.ncc_cost(Lf, Rf, D, radius)}[kind]()
    if domain == "integer" and kind != "ncc":
        np.testing.assert_array_equal(got, ref)
    else:
        close(got, ref)


@pytest.mark.parametrize("sem", ["ref_cpu", "ref_gpu"])
@pytest.mark.parametrize("domain", ["integer", "reference"])
def test_sgm_reference_table_wta_lr(ctx, orc, pair, sem, domain):
    L, R = pair
    if domain == "integer":
        s, p1, p2, mode = np.float32(1), np.float32(10), np.float32(120), "const"
    else:
        s = np.float32(1) / np.float32(255)
        p1, p2, mode = np.float32(30) / np.float32(255), np.float32(150) / np.float32(255), "adjust"
    Lf, Rf = orc.u8_to_f32(L, s), orc.u8_to_f32(R, s)
    C = orc.bt_cost(Lf, Rf, D)
    d_ref, dn_ref, S_ref = orc.sgm(C, Lf, p1, p2, p2_mode=1 if mode == "adjust" else 0, paths=8, table=1,
                                   semantics={"ref_cpu": 1, "ref_gpu": 2}[sem], threads=8)
    agg = torch.empty(C.shape, dtype=torch.float32, device="cuda")
    out = ctx.sgm(dev(C), float(p1), float(p2), guide=dev(L), guide_scale=float(s), p2_mode=mode, table="ref",
                  semantics=sem, aggreg=agg, lr=1, right=True)
    S = host(agg)
    if domain == "integer":
        np.testing.assert_array_equal(S, S_ref)
    else:
        close(S, S_ref)
    dl, dr = orc.lr_check(S_ref, d_ref, thr=1)
    np.testing.assert_array_equal(host(out["disp_right"]), dr)
    np.testing.assert_array_equal(host(out["disp"]), dl)


@pytest.mark.parametrize("kind,radius", [("bt", 0), ("ssd", 2), ("ncc", 4)])
def test_dp(ctx, orc, pair, kind, radius):
    L, R = pair
    Lf, Rf = orc.u8_to_f32(L), orc.u8_to_f32(R)
    C = {"bt": lambda: orc.bt_cost(Lf, Rf, D), "ssd": lambda: orc.ssd_cost(Lf, Rf, D, radius),
         "ncc": lambda: orc.ncc_cost(Lf, Rf, D, radius)}[kind]()
    d_ref, dn_ref = orc.dp(C)
    out = ctx.dp(dev(C), norm=True)
    np.testing.assert_array_equal(host(out["disp"]), d_ref)
    np.testing.assert_array_equal(host(out["disp_norm"]), dn_ref)


def test_wta_lr(ctx, orc, pair):
    L, R = pair
    C = orc.ssd_cost(orc.u8_to_f32(L), orc.u8_to_f32(R), D, 2)
    d_ref, _ = orc.wta(C)
    dl, dr = orc.lr_check(C, d_ref, thr=1)
    out = ctx.wta(dev(C), lr=1, right=True)
    np.testing.assert_array_equal(host(out["disp"]), dl)
    np.testing.assert_array_equal(host(out["disp_right"]), dr)
