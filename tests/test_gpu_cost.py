"""The matching-cost DSI kernels (tdv_cost: BT, SSD, NCC) against the oracle,
bit for bit (NaN where the oracle has NaN, +INF where x - d < 0), over the
shapes that exercise the banded kernels' edges: tiles cut by the image,
disparity ranges below, at and above a warp, both DSI layouts, u8 images with
the 1/255 scale and float images with padded rows, and left / right images of
different sizes (each clamps to its own edges).  Radius 5 takes the per-cell
kernel and is checked the same way."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

KINDS = [("bt", 0), ("ssd", 1), ("ssd", 2), ("ssd", 3), ("ssd", 4), ("ssd", 5),
         ("ncc", 1), ("ncc", 2), ("ncc", 4), ("ncc", 5)]
KIND_ID = {"bt": 0, "ssd": 1, "ncc": 2}
SHAPES = [((1, 1), (1, 1)), ((5, 7), (5, 7)), ((9, 70), (12, 75)), ((37, 130), (35, 129))]


def padded(a, extra=3):
    H, W = a.shape
    t = torch.zeros((H, W + extra), dtype=torch.from_numpy(a[:1]).dtype, device="cuda")
    t[:, :W] = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return t[:, :W]


@pytest.mark.parametrize("kind,radius", KINDS)
@pytest.mark.parametrize("D", [1, 3, 8, 16, 17, 33, 64, 100])
def test_cost_bit_exact(ctx, orc, kind, radius, D):
    rng = np.random.default_rng(D * 100 + radius * 10 + KIND_ID[kind])
    for i, ((lh, lw), (rh, rw)) in enumerate(SHAPES):
        L8 = rng.integers(0, 256, (lh, lw), dtype=np.uint8)
        R8 = rng.integers(0, 256, (rh, rw), dtype=np.uint8)
        if i == 2:
            L8[:, :5] = 0  # all-zero NCC windows: NaN
            R8[:, :9] = 0
        for layout in ("hwd", "ref"):
            lay = orc.LAYOUT_HWD if layout == "hwd" else orc.LAYOUT_REF_WHD
            if (i + (layout == "ref")) % 2 == 0:
                s = np.float32(1.0) / np.float32(255.0)
                C = ctx.cost(torch.from_numpy(L8).cuda(), torch.from_numpy(R8).cuda(), D, kind=kind, radius=radius,
                             layout=layout, scale=float(s))
                Lf, Rf = orc.u8_to_f32(L8, s), orc.u8_to_f32(R8, s)
            else:
                Lf = rng.random((lh, lw), dtype=np.float32)
                Rf = rng.random((rh, rw), dtype=np.float32)
                C = ctx.cost(padded(Lf), padded(Rf), D, kind=kind, radius=radius, layout=layout)
            ref = orc.cost_pair(Lf, Rf, D, KIND_ID[kind], radius, lay)
            torch.cuda.synchronize()
            got = C.cpu().numpy()
            assert got.shape == ref.shape
            assert np.array_equal(got, ref, equal_nan=True), f"{kind} r={radius} D={D} shape={i} {layout}"


@pytest.mark.parametrize("kind,radius", [("bt", 0), ("ssd", 3), ("ncc", 4)])
def test_cost_large_d(ctx, orc, kind, radius):
    # D = 256 over a frame wider than four tiles: every band column offset
    rng = np.random.default_rng(3)
    L8 = rng.integers(0, 256, (21, 300), dtype=np.uint8)
    R8 = rng.integers(0, 256, (21, 300), dtype=np.uint8)
    C = ctx.cost(torch.from_numpy(L8).cuda(), torch.from_numpy(R8).cuda(), 256, kind=kind, radius=radius)
    ref = orc.cost_pair(orc.u8_to_f32(L8), orc.u8_to_f32(R8), 256, KIND_ID[kind], radius)
    torch.cuda.synchronize()
    assert np.array_equal(C.cpu().numpy(), ref, equal_nan=True)


@pytest.mark.parametrize("radius", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("D", [1, 3, 16, 17, 33, 64, 100])
def test_fast_wta_bit_exact(ctx, orc, radius, D):
    # the fused SSD + argmin (lowest d on ties, NaN and +INF never win, d = 0
    # when no cost is finite) against the oracle's scan, both outputs
    rng = np.random.default_rng(1000 + D * 10 + radius)
    for i, ((h, w), _) in enumerate(SHAPES):
        if i % 2 == 0:
            L8 = rng.integers(0, 256, (h, w), dtype=np.uint8)
            R8 = np.roll(L8, 2, axis=1) if w > 4 else rng.integers(0, 256, (h, w), dtype=np.uint8)
            s = np.float32(1.0) / np.float32(255.0)
            out = ctx.fast_wta(torch.from_numpy(L8).cuda(), torch.from_numpy(R8).cuda(), D, radius=radius,
                               scale=float(s), norm=True)
            Lf, Rf = orc.u8_to_f32(L8, s), orc.u8_to_f32(R8, s)
        else:
            Lf = rng.random((h, w), dtype=np.float32)
            Rf = rng.random((h, w), dtype=np.float32)
            Lf[:, : w // 3] = Lf[:, :1]  # flat runs: ties
            Rf[:, : w // 3] = Lf[:, :1]
            if i == 3:
                Lf[h // 2, w // 2] = np.nan  # windows over it give NaN costs
            out = ctx.fast_wta(padded(Lf), padded(Rf), D, radius=radius, norm=True)
        d_ref, dn_ref = orc.fastwta(Lf, Rf, D, radius=radius)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out["disp"].cpu().numpy(), d_ref, err_msg=f"shape {i}")
        np.testing.assert_array_equal(out["disp_norm"].cpu().numpy(), dn_ref, err_msg=f"shape {i}")


@pytest.mark.parametrize("D", [1, 5, 31, 32, 33, 300, 600])
@pytest.mark.parametrize("layout", ["hwd", "ref"])
def test_dp_bit_exact(ctx, orc, D, layout):
    # the DP scanline matcher over disparity ranges that fill one to
    # nineteen lanes per warp slot, rows wider than one backtrack stage
    rng = np.random.default_rng(7 * D + (layout == "ref"))
    lay = orc.LAYOUT_HWD if layout == "hwd" else orc.LAYOUT_REF_WHD
    for (h, w) in ((1, 1), (3, 45), (6, 131)):
        L8 = rng.integers(0, 256, (h, w), dtype=np.uint8)
        R8 = rng.integers(0, 256, (h, w), dtype=np.uint8)
        C = orc.bt_cost(orc.u8_to_f32(L8), orc.u8_to_f32(R8), D, layout=lay)
        C[rng.random(C.shape) < 0.01] = np.float32(np.nan)
        d_ref, dn_ref = orc.dp(C, layout=lay)
        out = ctx.dp(torch.from_numpy(C).cuda(), layout=layout, norm=True)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out["disp"].cpu().numpy(), d_ref, err_msg=f"{h}x{w}")
        np.testing.assert_array_equal(out["disp_norm"].cpu().numpy(), dn_ref, err_msg=f"{h}x{w}")


@pytest.mark.parametrize("D", [1, 3, 4, 8, 33, 64, 100, 256])
@pytest.mark.parametrize("layout", ["hwd", "ref"])
def test_wta_and_lr_bit_exact(ctx, orc, D, layout):
    # WTA (thread per pixel when D is a multiple of 4, warp per pixel
    # otherwise) and the left-right check (right-view argmin tiled through
    # shared memory) on volumes with ties, NaN and +INF cells, rows wider
    # than one 256-pixel tile
    rng = np.random.default_rng(11 * D + (layout == "ref"))
    lay = orc.LAYOUT_HWD if layout == "hwd" else orc.LAYOUT_REF_WHD
    for (h, w) in ((1, 1), (4, 37), (3, 600)):
        shape = (h, w, D) if layout == "hwd" else (w, h, D)
        V = (rng.integers(0, 8, shape) / np.float32(4.0)).astype(np.float32)  # many ties
        V[rng.random(shape) < 0.02] = np.float32(np.nan)
        V[rng.random(shape) < 0.02] = np.float32(np.inf)
        d_ref, dn_ref = orc.wta(V, layout=lay)
        out = ctx.wta(torch.from_numpy(V).cuda(), layout=layout, norm=True)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out["disp"].cpu().numpy(), d_ref, err_msg=f"wta {h}x{w}")
        np.testing.assert_array_equal(out["disp_norm"].cpu().numpy(), dn_ref, err_msg=f"wta {h}x{w}")
        dl, dr = orc.lr_check(V, d_ref, thr=1, layout=lay)
        out = ctx.wta(torch.from_numpy(V).cuda(), layout=layout, lr=1, right=True)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out["disp"].cpu().numpy(), dl, err_msg=f"lr {h}x{w}")
        np.testing.assert_array_equal(out["disp_right"].cpu().numpy(), dr, err_msg=f"lr right {h}x{w}")


@pytest.mark.parametrize("kind,radius,D", [("ssd", 4, 1000), ("ncc", 4, 1000), ("bt", 0, 1500)])
def test_cost_bands_past_48kb(ctx, orc, kind, radius, D):
    # disparity ranges whose bands need more than 48 KB of shared memory (the
    # kernels raise their limit per device), on an image wider than one tile
    rng = np.random.default_rng(D + radius)
    L8 = rng.integers(0, 256, (9, 1100), dtype=np.uint8)
    R8 = rng.integers(0, 256, (9, 1100), dtype=np.uint8)
    C = ctx.cost(torch.from_numpy(L8).cuda(), torch.from_numpy(R8).cuda(), D, kind=kind, radius=radius)
    ref = orc.cost_pair(orc.u8_to_f32(L8), orc.u8_to_f32(R8), D, KIND_ID[kind], radius)
    torch.cuda.synchronize()
    assert np.array_equal(C.cpu().numpy(), ref, equal_nan=True)
    if kind == "ssd":
        out = ctx.fast_wta(torch.from_numpy(L8).cuda(), torch.from_numpy(R8).cuda(), D, radius=radius)
        d_ref, _ = orc.fastwta(orc.u8_to_f32(L8), orc.u8_to_f32(R8), D, radius=radius)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out["disp"].cpu().numpy(), d_ref)


@pytest.mark.parametrize("kind,radius", [("bt", 0), ("ssd", 1), ("ssd", 3), ("ssd", 4), ("ssd", 5), ("ncc", 2),
                                         ("ncc", 4)])
@pytest.mark.parametrize("D", [1, 16, 33, 100])
def test_cost_filtered_bit_exact(ctx, orc, kind, radius, D):
    # the Gaussian fused into the cost kernel's staging (radius 5 takes the
    # filter-then-cost path) against tdv_prefilter + tdv_cost on the GPU and
    # against the oracle's gauss5 + cost; the filtered left image too
    from oracle import image_ops as io
    rng = np.random.default_rng(500 + D * 10 + radius + KIND_ID[kind])
    for i, ((lh, lw), (rh, rw)) in enumerate(SHAPES):
        L8 = rng.integers(0, 256, (lh, lw), dtype=np.uint8)
        R8 = rng.integers(0, 256, (rh, rw), dtype=np.uint8)
        layout = "hwd" if i % 2 == 0 else "ref"
        lay = orc.LAYOUT_HWD if layout == "hwd" else orc.LAYOUT_REF_WHD
        if i % 2 == 0:
            s = float(np.float32(1.0) / np.float32(255.0))
            Lt, Rt, Lh, Rh = torch.from_numpy(L8).cuda(), torch.from_numpy(R8).cuda(), L8, R8
        else:
            s = 1.0
            Lh = rng.random((lh, lw), dtype=np.float32)
            Rh = rng.random((rh, rw), dtype=np.float32)
            Lt, Rt = padded(Lh), padded(Rh)
        C, fl = ctx.cost_filtered(Lt, Rt, D, kind=kind, radius=radius, layout=layout, scale=s)
        FL, FR = ctx.prefilter(Lt, "gauss5", scale=s), ctx.prefilter(Rt, "gauss5", scale=s)
        C2 = ctx.cost(FL, FR, D, kind=kind, radius=radius, layout=layout)
        ref = orc.cost_pair(io.gauss5(Lh, s), io.gauss5(Rh, s), D, KIND_ID[kind], radius, lay)
        torch.cuda.synchronize()
        H, W = min(lh, rh), min(lw, rw)
        got = C.cpu().numpy()
        assert np.array_equal(got, C2.cpu().numpy(), equal_nan=True), f"vs two-step, shape {i}"
        assert np.array_equal(got, ref, equal_nan=True), f"vs oracle, shape {i}"
        np.testing.assert_array_equal(fl.cpu().numpy(), FL.cpu().numpy()[:H, :W])


def test_cost_filtered_median_and_validation(ctx, orc):
    from oracle import image_ops as io
    from thundervision_b200 import _lib as L
    rng = np.random.default_rng(9)
    L8 = rng.integers(0, 256, (20, 90), dtype=np.uint8)
    R8 = rng.integers(0, 256, (20, 90), dtype=np.uint8)
    s = float(np.float32(1.0) / np.float32(255.0))
    C, fl = ctx.cost_filtered(torch.from_numpy(L8).cuda(), torch.from_numpy(R8).cuda(), 24, kind="ssd", radius=2,
                              scale=s, prefilter="median7")
    ref = orc.cost_pair(io.median7(L8, s), io.median7(R8, s), 24, 1, 2)
    torch.cuda.synchronize()
    assert np.array_equal(C.cpu().numpy(), ref)
    np.testing.assert_array_equal(fl.cpu().numpy(), io.median7(L8, s))
    with pytest.raises(L.TdvError):
        ctx.check(L.lib().tdv_cost_filtered(ctx.handle, None, None, None, 0, None, None, None))
