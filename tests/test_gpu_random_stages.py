"""Seeded random sweeps of the stand-alone stages against the oracle: the
cost DSI (BT, SSD and NCC at random window radii, both layouts, u8 or float
images of different sizes), WTA with the left-right check and DP on random
volumes full of ties and +INF, and FastWTA.  Every value and map bit-exact."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

KINDS = {0: "bt", 1: "ssd", 2: "ncc"}


def lay(orc, name):
    return orc.LAYOUT_HWD if name == "hwd" else orc.LAYOUT_REF_WHD


def images(rng, W, H):
    L = rng.integers(0, 256, (H, W)).astype(np.uint8)
    s = int(rng.integers(0, 8))
    R = np.clip(np.roll(L, -s, axis=1).astype(int) + rng.integers(-4, 5, (H, W)), 0, 255).astype(np.uint8)
    return L, R


@pytest.mark.parametrize("i", range(40))
def test_random_cost(ctx, orc, i):
    rng = np.random.default_rng(7000 + i)
    W, H = int(rng.integers(1, 160)), int(rng.integers(1, 90))
    D = int(rng.choice([1, 3, 8, 16, 33, 64, 100]))
    kind = int(rng.integers(0, 3))
    radius = 0 if kind == 0 else int(rng.integers(0, 7))
    layout = "hwd" if rng.random() < 0.5 else "ref"
    L, R = images(rng, W, H)
    if rng.random() < 0.3:  # a right image of another size: the DSI is the smaller one
        R = R[: max(1, H - int(rng.integers(0, 5))), : max(1, W - int(rng.integers(0, 9)))].copy()
    unit = rng.random() < 0.5  # [0,1] float intensities, else u8 values
    scale = np.float32(1) / np.float32(255) if unit else np.float32(1)
    Lf, Rf = orc.u8_to_f32(L, scale), orc.u8_to_f32(R, scale)
    want = orc.cost_pair(Lf, Rf, D, kind, radius, layout=lay(orc, layout))
    if unit:
        got = ctx.cost(torch.from_numpy(Lf).cuda(), torch.from_numpy(Rf).cuda(), D, kind=KINDS[kind],
                       radius=radius, layout=layout)
    else:
        got = ctx.cost(torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda(), D, kind=KINDS[kind],
                       radius=radius, layout=layout)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(got.cpu().numpy(), want)


def volume(rng, W, H, D, layout):
    v = rng.integers(0, 6, (H, W, D)).astype(np.float32)  # many ties
    v[rng.random(v.shape) < 0.05] = np.inf
    v[rng.random((H, W)) < 0.02] = np.inf  # pixels with no finite cost
    if layout == "ref":
        v = np.ascontiguousarray(v.transpose(1, 0, 2))
    return v


@pytest.mark.parametrize("i", range(24))
def test_random_wta_lr_dp(ctx, orc, i):
    rng = np.random.default_rng(7500 + i)
    W, H = int(rng.integers(1, 200)), int(rng.integers(1, 60))
    D = int(rng.choice([1, 2, 5, 32, 64, 77, 128, 300]))
    layout = "hwd" if rng.random() < 0.5 else "ref"
    v = volume(rng, W, H, D, layout)
    dv = torch.from_numpy(v).cuda()
    thr = int(rng.integers(0, 3))
    out = ctx.wta(dv, layout=layout, lr=thr, right=True)
    torch.cuda.synchronize()
    d, _ = orc.wta(v, layout=lay(orc, layout))
    dl, dr = orc.lr_check(v, d, thr=thr, layout=lay(orc, layout))
    np.testing.assert_array_equal(out["disp"].cpu().numpy(), dl)
    np.testing.assert_array_equal(out["disp_right"].cpu().numpy(), dr)
    got = ctx.dp(dv, layout=layout)["disp"]
    torch.cuda.synchronize()
    np.testing.assert_array_equal(got.cpu().numpy(), orc.dp(v, layout=lay(orc, layout))[0])


@pytest.mark.parametrize("i", range(12))
def test_random_fast_wta(ctx, orc, i):
    rng = np.random.default_rng(7800 + i)
    W, H = int(rng.integers(8, 200)), int(rng.integers(8, 80))
    D = int(rng.choice([4, 16, 48, 64, 130]))
    radius = int(rng.integers(1, 6))
    L, R = images(rng, W, H)
    scale = np.float32(1) / np.float32(255)
    Lf, Rf = orc.u8_to_f32(L, scale), orc.u8_to_f32(R, scale)
    got = ctx.fast_wta(torch.from_numpy(Lf).cuda(), torch.from_numpy(Rf).cuda(), D, radius=radius)["disp"]
    torch.cuda.synchronize()
    np.testing.assert_array_equal(got.cpu().numpy(), orc.fastwta(Lf, Rf, D, radius=radius)[0])
