"""sm_100a kernels vs the CPU oracle on seeded synthetic pairs, through the C ABI.

Tolerances (stated per test):
  * disparity maps, DP/WTA outputs and integer-domain costs / sums: bit-exact;
  * float32 SSD / NCC costs and aggregated sums in the reference [0,1]
    domain: within 1e-5 relative (the kernels follow the oracle's rounding
    order, so in practice they match exactly);
  * +INF / NaN cells must coincide.
"""
import numpy as np
import pytest
import torch

from thundervision_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

REL = 1e-5


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def assert_close_f32(got, ref, rel=REL):
    gi, ri = np.isinf(got), np.isinf(ref)
    np.testing.assert_array_equal(gi, ri)
    np.testing.assert_array_equal(np.isnan(got), np.isnan(ref))
    m = np.isfinite(ref)
    np.testing.assert_allclose(got[m], ref[m], rtol=rel, atol=0)


@pytest.fixture(scope="module")
def small_pair():
    L, R, gt, occ = syn.pair_small(11)
    return L, R


@pytest.fixture(scope="module")
def medium_pair():
    L, R, gt, occ = syn.pair_medium(5)
    return L, R


# ------------------------------------------------------------------ costs
@pytest.mark.parametrize("layout", ["hwd", "ref"])
def test_bt_cost_integer_domain(ctx, orc, small_pair, layout):
    L, R = small_pair
    C = host(ctx.cost(dev(L), dev(R), 16, kind="bt", layout=layout))
    ref = orc.bt_cost(orc.u8_to_f32(L), orc.u8_to_f32(R), 16,
                      layout=orc.LAYOUT_HWD if layout == "hwd" else orc.LAYOUT_REF_WHD)
    np.testing.assert_array_equal(C, ref)


@pytest.mark.parametrize("kind,radius", [("bt", 0), ("ssd", 3), ("ssd", 2), ("ncc", 1), ("ncc", 4)])
def test_costs_reference_domain(ctx, orc, medium_pair, kind, radius):
    L, R = medium_pair
    L, R = L[:96, :160], R[:96, :160]
    s = np.float32(1.0) / np.float32(255.0)
    C = host(ctx.cost(dev(L), dev(R), 32, kind=kind, radius=radius, scale=float(s)))
    Lf, Rf = orc.u8_to_f32(L, s), orc.u8_to_f32(R, s)
    fn = {"bt": lambda: orc.bt_cost(Lf, Rf, 32), "ssd": lambda: orc.ssd_cost(Lf, Rf, 32, radius),
          "ncc": lambda: orc.ncc_cost(Lf, Rf, 32, radius)}[kind]
    assert_close_f32(C, fn())


@pytest.mark.parametrize("kind,radius", [("ssd", 3), ("ssd", 2)])
def test_ssd_integer_domain_exact(ctx, orc, small_pair, kind, radius):
    L, R = small_pair
    C = host(ctx.cost(dev(L), dev(R), 16, kind=kind, radius=radius))
    np.testing.assert_array_equal(C, orc.ssd_cost(orc.u8_to_f32(L), orc.u8_to_f32(R), 16, radius))


# --------------------------------------------------------- general SGM path
@pytest.mark.parametrize("sem", ["standard", "ref_cpu", "ref_gpu"])
@pytest.mark.parametrize("table", ["full", "ref"])
@pytest.mark.parametrize("paths", [8, 4])
def test_sgm_integer_domain(ctx, orc, small_pair, sem, table, paths):
    L, R = small_pair
    Lf, Rf = orc.u8_to_f32(L), orc.u8_to_f32(R)
    C = orc.bt_cost(Lf, Rf, 16)
    semi = {"standard": 0, "ref_cpu": 1, "ref_gpu": 2}[sem]
    d_ref, dn_ref, S_ref = orc.sgm(C, Lf, 10, 120, paths=paths, table=1 if table == "ref" else 0,
                                   semantics=semi)
    agg = torch.empty(C.shape, dtype=torch.float32, device="cuda")
    out = ctx.sgm(dev(C), 10, 120, paths=paths, table=table, semantics=sem, norm=True, aggreg=agg)
    np.testing.assert_array_equal(host(agg), S_ref)
    np.testing.assert_array_equal(host(out["disp"]), d_ref)
    np.testing.assert_array_equal(host(out["disp_norm"]), dn_ref)


@pytest.mark.parametrize("sem", ["ref_cpu", "ref_gpu", "standard"])
@pytest.mark.parametrize("shape", [(96, 64), (64, 96), (80, 80)])
def test_sgm_reference_domain(ctx, orc, medium_pair, sem, shape):
    """The reference's literal configuration: [0,1] intensities, P1=30/255,
    P2=150/255 divided by |dI|, the reference path table, its layout."""
    W, H = shape
    L, R = medium_pair
    L, R = L[:H, :W], R[:H, :W]
    s = np.float32(1) / np.float32(255)
    Lf, Rf = orc.u8_to_f32(L, s), orc.u8_to_f32(R, s)
    p1, p2 = np.float32(30) / np.float32(255), np.float32(150) / np.float32(255)
    C = orc.bt_cost(Lf, Rf, 32, layout=orc.LAYOUT_REF_WHD)
    semi = {"standard": 0, "ref_cpu": 1, "ref_gpu": 2}[sem]
    d_ref, dn_ref, S_ref = orc.sgm(C, Lf, p1, p2, p2_mode=1, table=1, semantics=semi,
                                   layout=orc.LAYOUT_REF_WHD)
    agg = torch.empty(C.shape, dtype=torch.float32, device="cuda")
    out = ctx.sgm(dev(C), float(p1), float(p2), guide=dev(L), guide_scale=float(s), p2_mode="adjust",
                  table="ref", semantics=sem, layout="ref", norm=True, aggreg=agg)
    assert_close_f32(host(agg), S_ref)
    np.testing.assert_array_equal(host(out["disp"]), d_ref)
    np.testing.assert_array_equal(host(out["disp_norm"]), dn_ref)


@pytest.mark.parametrize("kind,radius", [("ssd", 2), ("ncc", 4)])
def test_sgm_on_window_costs(ctx, orc, medium_pair, kind, radius):
    L, R = medium_pair
    L, R = L[:120, :200], R[:120, :200]
    Lf, Rf = orc.u8_to_f32(L), orc.u8_to_f32(R)
    C = orc.ssd_cost(Lf, Rf, 64, radius) if kind == "ssd" else orc.ncc_cost(Lf, Rf, 64, radius)
    d_ref, _, S_ref = orc.sgm(C, Lf, 10, 120)
    agg = torch.empty(C.shape, dtype=torch.float32, device="cuda")
    out = ctx.sgm(dev(C), 10, 120, aggreg=agg)
    assert_close_f32(host(agg), S_ref)
    np.testing.assert_array_equal(host(out["disp"]), d_ref)


# ------------------------------------------------------------- fused path
@pytest.mark.parametrize("paths", [8, 4])
@pytest.mark.parametrize("lr", [None, 1])
def test_fused_small(ctx, orc, small_pair, paths, lr):
    L, R = small_pair
    _check_fused(ctx, orc, L, R, 16, 10, 120, paths, lr)


@pytest.mark.parametrize("paths", [8, 4])
def test_fused_medium(ctx, orc, medium_pair, paths):
    L, R = medium_pair
    _check_fused(ctx, orc, L, R, 64, 10, 120, paths, 1)


@pytest.mark.parametrize("W,H,D", [(640, 96, 128), (640, 96, 256), (1001, 37, 200),
                                   (257, 64, 129), (1920, 24, 256), (777, 19, 65)])
@pytest.mark.parametrize("lr", [None, 1])
@pytest.mark.parametrize("paths", [8, 4])
def test_fused_wide_large_d(ctx, orc, W, H, D, lr, paths):
    """Disparity ranges above 64 (two or four disparity pairs per lane) on
    rows many right-plane chunks long, including widths that are not chunk
    multiples (a partial last pixel group in the horizontal passes) and
    ranges that are not multiples of 64 pairs (lanes holding d >= D)."""
    L, R, _, _ = syn.make_pair(W, H, D, W + 7 * H + D, n_rects=4, slanted=True)
    _check_fused(ctx, orc, L, R, D, 10, 120, paths, lr)


def _check_fused(ctx, orc, L, R, D, p1, p2, paths, lr):
    Lf, Rf = orc.u8_to_f32(L), orc.u8_to_f32(R)
    C = orc.bt_cost(Lf, Rf, D)
    d_ref, dn_ref, S_ref = orc.sgm(C, Lf, p1, p2, paths=paths, threads=8)
    out = ctx.stereo_sgm(dev(L), dev(R), D, p1, p2, paths=paths, lr=lr, norm=True,
                         right_disp=lr is not None)
    if lr is None:
        np.testing.assert_array_equal(host(out["disp"]), d_ref)
        np.testing.assert_array_equal(host(out["disp_norm"]), dn_ref)
    else:
        dl, dr = orc.lr_check(S_ref, d_ref, thr=lr)
        np.testing.assert_array_equal(host(out["disp_right"]), dr)
        np.testing.assert_array_equal(host(out["disp"]), dl)
        dn = np.where(dl == 0xFFFF, np.float32(-1), dl.astype(np.float32) / np.float32(D))
        np.testing.assert_array_equal(host(out["disp_norm"]), dn)


def test_fused_matches_general_path(ctx, orc, medium_pair):
    L, R = medium_pair
    fused = ctx.stereo_sgm(dev(L), dev(R), 64, 10, 120, lr=1)
    C = ctx.cost(dev(L), dev(R), 64)
    gen = ctx.sgm(C, 10, 120, lr=1)
    np.testing.assert_array_equal(host(fused["disp"]), host(gen["disp"]))


def test_non_integer_inputs_take_general_path(ctx, orc, small_pair):
    L, R = small_pair
    s = np.float32(1) / np.float32(255)
    p1, p2 = np.float32(30) / np.float32(255), np.float32(150) / np.float32(255)
    out = ctx.stereo_sgm(dev(L), dev(R), 16, float(p1), float(p2), scale=float(s),
                         p2_mode="adjust", table="ref", semantics="ref_cpu")
    Lf, Rf = orc.u8_to_f32(L, s), orc.u8_to_f32(R, s)
    C = orc.bt_cost(Lf, Rf, 16)
    d_ref, _, _ = orc.sgm(C, Lf, p1, p2, p2_mode=1, table=1, semantics=1)
    np.testing.assert_array_equal(host(out["disp"]), d_ref)


# ---------------------------------------------------------- other stages
@pytest.mark.parametrize("layout", ["hwd", "ref"])
def test_wta(ctx, orc, small_pair, layout):
    L, R = small_pair
    lay = orc.LAYOUT_HWD if layout == "hwd" else orc.LAYOUT_REF_WHD
    C = orc.bt_cost(orc.u8_to_f32(L), orc.u8_to_f32(R), 16, layout=lay)
    C[..., 3] = C[..., 2]  # planted ties
    d_ref, dn_ref = orc.wta(C, layout=lay)
    out = ctx.wta(dev(C), layout=layout, norm=True)
    np.testing.assert_array_equal(host(out["disp"]), d_ref)
    np.testing.assert_array_equal(host(out["disp_norm"]), dn_ref)


def test_wta_lr(ctx, orc, small_pair):
    L, R = small_pair
    C = orc.bt_cost(orc.u8_to_f32(L), orc.u8_to_f32(R), 16)
    d_ref, _ = orc.wta(C)
    dl, dr = orc.lr_check(C, d_ref, thr=1)
    out = ctx.wta(dev(C), lr=1, right=True)
    np.testing.assert_array_equal(host(out["disp"]), dl)
    np.testing.assert_array_equal(host(out["disp_right"]), dr)


@pytest.mark.parametrize("D", [16, 64, 100])
@pytest.mark.parametrize("layout", ["hwd", "ref"])
def test_dp(ctx, orc, medium_pair, D, layout):
    L, R = medium_pair
    L, R = L[:64, :200], R[:64, :200]
    lay = orc.LAYOUT_HWD if layout == "hwd" else orc.LAYOUT_REF_WHD
    C = orc.bt_cost(orc.u8_to_f32(L), orc.u8_to_f32(R), D, layout=lay)
    d_ref, dn_ref = orc.dp(C, layout=lay)
    out = ctx.dp(dev(C), layout=layout, norm=True)
    np.testing.assert_array_equal(host(out["disp"]), d_ref)
    np.testing.assert_array_equal(host(out["disp_norm"]), dn_ref)


@pytest.mark.parametrize("scale", [1.0, 1.0 / 255.0])
def test_fast_wta(ctx, orc, small_pair, scale):
    L, R = small_pair
    s = np.float32(scale)
    d_ref, dn_ref = orc.fastwta(orc.u8_to_f32(L, s), orc.u8_to_f32(R, s), 16, 3)
    out = ctx.fast_wta(dev(L), dev(R), 16, 3, scale=float(s), norm=True)
    np.testing.assert_array_equal(host(out["disp"]), d_ref)
    np.testing.assert_array_equal(host(out["disp_norm"]), dn_ref)


# ------------------------------------------------------------- edge sweep
@pytest.mark.parametrize("W", [1, 2, 3, 17, 33])
@pytest.mark.parametrize("H", [1, 2, 3, 17, 33])
def test_edge_sizes(ctx, orc, W, H):
    rng = np.random.default_rng(W * 1000 + H)
    L = rng.integers(0, 256, size=(H, W), dtype=np.uint8)
    R = rng.integers(0, 256, size=(H, W), dtype=np.uint8)
    Lf, Rf = orc.u8_to_f32(L), orc.u8_to_f32(R)
    for D in (1, 2, 3, 16, 33, 64, 256):
        C = orc.bt_cost(Lf, Rf, D)
        for paths in (8, 4):
            d_ref, _, S_ref = orc.sgm(C, Lf, 10, 120, paths=paths)
            out = ctx.stereo_sgm(dev(L), dev(R), D, 10, 120, paths=paths)
            np.testing.assert_array_equal(host(out["disp"]), d_ref, err_msg=f"fused D={D} P={paths}")
        agg = torch.empty(C.shape, dtype=torch.float32, device="cuda")
        for sem in (0, 1, 2):
            d_ref, _, S_ref = orc.sgm(C, Lf, 10, 120, table=1, semantics=sem)
            o = ctx.sgm(dev(C), 10, 120, table="ref", semantics=["standard", "ref_cpu", "ref_gpu"][sem],
                        aggreg=agg)
            assert_close_f32(host(agg), S_ref)
            np.testing.assert_array_equal(host(o["disp"]), d_ref, err_msg=f"general D={D} sem={sem}")
        d_ref, _ = orc.dp(C)
        np.testing.assert_array_equal(host(ctx.dp(dev(C))["disp"]), d_ref)


def test_deterministic(ctx, medium_pair):
    L, R = medium_pair
    a = host(ctx.stereo_sgm(dev(L), dev(R), 64, 10, 120, lr=1)["disp"])
    b = host(ctx.stereo_sgm(dev(L), dev(R), 64, 10, 120, lr=1)["disp"])
    np.testing.assert_array_equal(a, b)
    C = ctx.cost(dev(L), dev(R), 64)
    s1 = torch.empty_like(C)
    s2 = torch.empty_like(C)
    ctx.sgm(C, 10, 120, aggreg=s1)
    ctx.sgm(C, 10, 120, aggreg=s2)
    assert torch.equal(s1, s2)


@pytest.mark.slow
def test_full_hd_d256_bit_exact(ctx, orc):
    """The headline configuration, 1920x1080, D=256, 8 paths, left-right
    check: fused kernels vs the oracle (all host cores), bit-exact."""
    vs = syn.VideoStream(seed=2)
    L, R, gt, occ = vs.frame(0)
    Lf, Rf = orc.u8_to_f32(L), orc.u8_to_f32(R)
    C = orc.bt_cost(Lf, Rf, 256)
    import os
    d_ref, _, S_ref = orc.sgm(C, Lf, 10, 120, threads=os.cpu_count() or 8)
    dl, dr = orc.lr_check(S_ref, d_ref, thr=1)
    out = ctx.stereo_sgm(dev(L), dev(R), 256, 10, 120, lr=1, right_disp=True)
    np.testing.assert_array_equal(host(out["disp_right"]), dr)
    np.testing.assert_array_equal(host(out["disp"]), dl)
