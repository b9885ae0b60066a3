"""Image stages either side of the path on the GPU: every kernel bit-identical
to oracle/image_ops.py (itself pinned to OpenCV, tests/test_image_ops_cpu.py)
on sizes that cut the 32x8 tiles unevenly, padded row pitches, each dtype and
channel count, and the golden inputs."""
import os

import numpy as np
import pytest
import torch

from oracle import image_ops as io

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "image_ops.npz")
SIZES = [(1, 1), (7, 31), (9, 33), (97, 200), (480, 640)]


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def padded(a, extra=5):
    """A device copy of `a` whose rows are padded by `extra` elements."""
    H, W = a.shape[:2]
    big = torch.zeros((H, W + extra) + a.shape[2:], dtype=dev(a[:1]).dtype, device="cuda")
    big[:, :W] = dev(a)
    return big[:, :W]


def host(t):
    return t.cpu().numpy()


@pytest.fixture(scope="module")
def g():
    return np.load(GOLDEN)


@pytest.mark.parametrize("H,W", SIZES)
@pytest.mark.parametrize("u8", [False, True])
def test_prefilters(ctx, H, W, u8):
    rng = np.random.default_rng(H * 1000 + W)
    a = rng.integers(0, 256, (H, W), dtype=np.uint8) if u8 else rng.random((H, W), dtype=np.float32)
    scale = 1.0 / 255.0 if u8 else 1.0
    for kind, ref in (("gauss5", io.gauss5), ("median7", io.median7)):
        out = ctx.prefilter(padded(a), kind, scale=scale)
        np.testing.assert_array_equal(host(out), ref(a, scale), err_msg=kind)


def test_prefilters_on_golden(ctx, g):
    np.testing.assert_array_equal(host(ctx.prefilter(dev(g["img"]), "gauss5")), io.gauss5(g["img"]))
    np.testing.assert_array_equal(host(ctx.prefilter(dev(g["u8"]), "median7")), g["median7_u8"].astype(np.float32))


@pytest.mark.parametrize("H,W", SIZES)
@pytest.mark.parametrize("dt", [np.float32, np.uint16])
def test_postfilters(ctx, H, W, dt):
    rng = np.random.default_rng(7 * H + W)
    if dt == np.uint16:
        a = rng.integers(0, 300, (H, W)).astype(np.uint16)
        a[rng.random((H, W)) < 0.05] = 0xFFFF
    else:
        a = rng.random((H, W), dtype=np.float32)
    t = padded(a) if dt == np.float32 else dev(a)
    np.testing.assert_array_equal(host(ctx.postfilter(t, "open7")), io.open7(a))
    np.testing.assert_array_equal(host(ctx.postfilter(t, "median3")), io.median3(a))


def test_postfilters_on_golden(ctx, g):
    for dt in ("f32", "u16"):
        np.testing.assert_array_equal(host(ctx.postfilter(dev(g["disp_" + dt]), "open7")), g["open7_" + dt])
        np.testing.assert_array_equal(host(ctx.postfilter(dev(g["disp_" + dt]), "median3")), g["median3_" + dt])


@pytest.mark.parametrize("H,W", SIZES)
def test_gray(ctx, H, W):
    rng = np.random.default_rng(H + 3 * W)
    c = rng.integers(0, 256, (H, W, 3), dtype=np.uint8)
    np.testing.assert_array_equal(host(ctx.to_gray(padded(c))), io.to_gray(c))


@pytest.mark.parametrize("H,W", [(1, 1), (9, 33), (97, 200), (480, 640)])
def test_remap(ctx, H, W):
    rng = np.random.default_rng(H * W + 1)
    Hs, Ws = H + 3, W - 1 if W > 1 else 1
    mx = (rng.random((H, W), dtype=np.float32) * (Ws + 8) - 4).astype(np.float32)
    my = (rng.random((H, W), dtype=np.float32) * (Hs + 8) - 4).astype(np.float32)
    mx.flat[::17] = np.round(mx.flat[::17] * 64) / 64  # ties of the 1/32 rounding
    for src in (rng.random((Hs, Ws), dtype=np.float32), rng.integers(0, 256, (Hs, Ws, 3), dtype=np.uint8),
                rng.integers(0, 256, (Hs, Ws), dtype=np.uint8), rng.random((Hs, Ws, 3), dtype=np.float32)):
        out = ctx.remap(padded(src), dev(mx), dev(my))
        np.testing.assert_array_equal(host(out), io.remap(src, mx, my))


@pytest.mark.parametrize("n", ["5", "8"])
def test_rectify_maps(ctx, g, n):
    H, W = g["img"].shape
    mx, my = ctx.rectify_maps(g["K"], g["dist" + n], g["R"], g["P"], W, H)
    np.testing.assert_array_equal(host(mx), g["rmapx" + n])
    np.testing.assert_array_equal(host(my), g["rmapy" + n])
    # a full-size camera, against the oracle, then remapping with those maps
    K = [[1400.0, 0, 961.3], [0, 1395.5, 539.2], [0, 0, 1]]
    P = [[1380.0, 0, 955.0], [0, 1380.0, 541.0], [0, 0, 1]]
    mx, my = ctx.rectify_maps(K, g["dist" + n], g["R"], P, 1920, 1080)
    rx, ry = io.rectify_maps(K, g["dist" + n], g["R"], P, 1920, 1080)
    np.testing.assert_array_equal(host(mx), rx)
    np.testing.assert_array_equal(host(my), ry)


def test_remap_on_golden(ctx, g):
    np.testing.assert_array_equal(host(ctx.remap(dev(g["img"]), dev(g["mapx"]), dev(g["mapy"]))), g["remap_f32"])
    np.testing.assert_array_equal(host(ctx.remap(dev(g["color"]), dev(g["mapx"]), dev(g["mapy"]))), g["remap_u8c3"])


@pytest.mark.parametrize("H,W,D", [(1, 1, 3), (9, 33, 16), (97, 200, 64)])
def test_subpixel(ctx, H, W, D):
    rng = np.random.default_rng(H + W + D)
    S = rng.random((H, W, D), dtype=np.float32) * np.float32(100)
    disp = rng.integers(0, D, (H, W)).astype(np.uint16)
    disp[rng.random((H, W)) < 0.1] = 0xFFFF
    out = ctx.subpixel(dev(S), dev(disp))
    np.testing.assert_array_equal(host(out), io.subpixel(S, disp))


@pytest.mark.parametrize("H,W", [(1, 1), (9, 33), (97, 200)])
@pytest.mark.parametrize("dt", [np.float32, np.uint16])
def test_reproject(ctx, H, W, dt):
    rng = np.random.default_rng(5 * H + W)
    d = (rng.random((H, W), dtype=np.float32) if dt == np.float32 else rng.integers(0, 256, (H, W)).astype(np.uint16))
    c = rng.integers(0, 256, (H, W, 3), dtype=np.uint8)
    v, cols = ctx.reproject(dev(d), padded(c), "direct", zscale=3.0)
    rv, rc = io.reproject(d, c, "direct", 3.0)
    np.testing.assert_array_equal(host(v), rv)
    np.testing.assert_array_equal(host(cols), rc)
    Q = [1, 0, 0, -W / 2, 0, 1, 0, -H / 2, 0, 0, 0, 500.0, 0, 0, -0.25, 0.5]
    if H == 1:  # w vanishes on every pixel: vertices (0, 0, 0)
        Q[14] = Q[15] = 0.0
    v, none = ctx.reproject(dev(d), None, "q", q=Q)
    assert none is None
    np.testing.assert_array_equal(host(v), io.reproject(d, None, "q", q=Q)[0])


def test_reproject_on_golden_and_ply(ctx, g, tmp_path):
    from thundervision_b200 import api
    v, _ = ctx.reproject(dev(g["disp_f32"]), None, "q", q=g["Q"].ravel().tolist())
    p = g["persp"].copy()
    p[..., 2] = p[..., 2] * np.float32(24.0)
    np.testing.assert_array_equal(host(v), p)
    vd, cd = ctx.reproject(dev(g["disp_f32"][:6, :7]), dev(g["color"][:6, :7]), "direct")
    path = tmp_path / "m.ply"
    api.write_ply(path, vd, cd)
    rv, rc = io.reproject(g["disp_f32"][:6, :7], g["color"][:6, :7], "direct")
    assert path.read_text() == io.ply_text(rv, rc)
