"""Image stages either side of the path, on the CPU: the oracle against
OpenCV's own outputs (tests/golden/image_ops.npz, made by
tests/golden/make_golden.py), the C PLY writer against the oracle's text, and
argument validation of the new C-ABI entry points (no device work)."""
import ctypes
import os

import numpy as np
import pytest

from oracle import image_ops as io

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "image_ops.npz")
ULP_1 = 2.0 ** -23  # one ulp of values in [1, 2): the float sums OpenCV orders its own way


@pytest.fixture(scope="module")
def g():
    return np.load(GOLDEN)


def test_gauss5_matches_opencv(g):
    # cvSmooth(CV_GAUSSIAN, 5), tdvision/medianfiltercpu.cpp:15
    d = np.abs(io.gauss5(g["img"]).astype(np.float64) - g["gauss5"])
    assert d.max() <= 2 * ULP_1


def test_gauss5_of_a_constant_and_a_step():
    a = np.full((9, 11), 0.25, np.float32)
    assert np.array_equal(io.gauss5(a), a)
    s = np.zeros((7, 12), np.float32)
    s[:, 6:] = 1.0
    row = io.gauss5(s)[3]
    np.testing.assert_allclose(row[4:8], [1 / 16, 5 / 16, 11 / 16, 15 / 16], atol=1e-7)


def test_median7_matches_opencv_on_u8(g):
    assert np.array_equal(io.median7(g["u8"]), g["median7_u8"].astype(np.float32))


@pytest.mark.parametrize("dt", ["f32", "u16"])
def test_open7_matches_opencv(g, dt):
    # Dilate: cvErode + cvDilate, 3 iterations (tdvision/dilate.cpp:18-19)
    assert np.array_equal(io.open7(g["disp_" + dt]), g["open7_" + dt])


@pytest.mark.parametrize("dt", ["f32", "u16"])
def test_median3_matches_opencv(g, dt):
    assert np.array_equal(io.median3(g["disp_" + dt]), g["median3_" + dt])


def test_gray_matches_opencv(g):
    # tdvision/misc.cpp:31-32
    assert np.array_equal(io.scale255()[g["color"]], g["scaled"])
    d = np.abs(io.to_gray(g["color"]).astype(np.float64) - g["gray"])
    assert d.max() <= 2 * ULP_1


def test_remap_matches_opencv(g):
    # cvRemap, tdvision/rectificationcv.cpp:298-310
    assert np.array_equal(io.remap(g["img"], g["mapx"], g["mapy"]), g["remap_f32"])
    assert np.array_equal(io.remap(g["color"], g["mapx"], g["mapy"]), g["remap_u8c3"])


@pytest.mark.parametrize("n", ["5", "8"])
def test_rectify_maps_match_opencv(g, n):
    # cvInitUndistortRectifyMap, tdvision/rectificationcv.cpp:114-117
    H, W = g["img"].shape
    mx, my = io.rectify_maps(g["K"], g["dist" + n], g["R"], g["P"], W, H)
    assert np.array_equal(mx, g["rmapx" + n]) and np.array_equal(my, g["rmapy" + n])


def test_reprojection_q_matches_opencv(g):
    # CVReprojector::reproject, tdvision/cvreprojector.cpp:45-60
    v, _ = io.reproject(g["disp_f32"], mode="q", q=g["Q"].ravel())
    p = g["persp"].copy()
    p[..., 2] = p[..., 2] * np.float32(24.0)
    assert np.array_equal(v, p)


def test_reprojection_direct_and_colors():
    d = np.array([[0.5, 0.25], [0.0, 1.0]], np.float32)
    c = np.array([[[255, 0, 1], [2, 3, 4]], [[5, 6, 7], [8, 9, 10]]], np.uint8)
    v, cols = io.reproject(d, c, mode="direct", zscale=2.0)
    assert v[0, 0].tolist() == [0.0, 2.0, 1.0] and v[1, 1].tolist() == [1.0, 1.0, 2.0]
    assert cols[0, 0, 0] == np.float32(255) * (np.float32(1) / np.float32(255))


def test_subpixel_parabola():
    S = np.zeros((1, 3, 5), np.float32)
    S[0, 0] = [9, 4, 1, 2, 7]  # minimum at 2, neighbours 4 and 2
    S[0, 1] = [1, 5, 6, 7, 8]  # minimum at 0: kept
    S[0, 2] = [3, 3, 3, 3, 3]  # flat: kept
    disp = np.array([[2, 0, 0xFFFF]], np.uint16)
    out = io.subpixel(S, disp)
    assert out[0, 0] == np.float32(2 + (4 - 2) / (2 * (4 + 2 - 2)))
    assert out[0, 1] == 0.0 and out[0, 2] == -1.0


def test_ply_writer_matches_the_reference_format(tmp_path):
    from thundervision_b200 import _lib as L
    lib = L.lib()
    v = np.array([[[0, 3, 0.125], [1, 3, 1e-7]], [[0, 2, 123456.7], [1, 2, -2.5]], [[0, 1, 0], [1, 1, 7]]],
                 np.float32)
    c = np.array([[[1, 0, 0.5], [0.2, 0.4, 0.6]], [[0, 0, 0], [1, 1, 1]], [[0.1, 0.2, 0.3], [0.9, 0.8, 0.7]]],
                 np.float32)
    for cols in (c, None):
        path = tmp_path / "mesh.ply"
        st = lib.tdv_write_ply(str(path).encode(), v.ctypes.data, cols.ctypes.data if cols is not None else None,
                               2, 3)
        assert st == L.TDV_OK
        assert path.read_text() == io.ply_text(v, cols)
    assert "element face 2" in io.ply_text(v, c)


def test_image_stage_arguments_are_validated():
    from thundervision_b200 import _lib as L
    lib = L.lib()
    h = ctypes.c_void_p()
    assert lib.tdv_ctx_create(0, ctypes.byref(h)) == L.TDV_OK
    try:
        bad = L.tdv_raster(None, 4, 4, 16, L.F32, 1)
        assert lib.tdv_postfilter(h, ctypes.byref(bad), L.POST_OPEN7, ctypes.byref(bad), None) == L.TDV_ERR_INVALID_ARG
        r = L.tdv_raster(1 << 20, 4, 4, 8, L.F32, 1)  # pitch below the row
        assert lib.tdv_postfilter(h, ctypes.byref(r), L.POST_OPEN7, ctypes.byref(r), None) == L.TDV_ERR_INVALID_ARG
        r = L.tdv_raster(1 << 20, 4, 4, 16, L.U8, 1)  # opening takes F32 or U16
        o = L.tdv_raster(2 << 20, 4, 4, 16, L.U8, 1)
        assert lib.tdv_postfilter(h, ctypes.byref(r), L.POST_OPEN7, ctypes.byref(o), None) == L.TDV_ERR_INVALID_ARG
        r = L.tdv_raster(1 << 20, 4, 4, 16, L.F32, 1)
        o = L.tdv_raster(2 << 20, 4, 4, 16, L.F32, 1)
        assert lib.tdv_postfilter(h, ctypes.byref(r), 7, ctypes.byref(o), None) == L.TDV_ERR_INVALID_ARG
        assert lib.tdv_postfilter(h, ctypes.byref(r), L.POST_OPEN7, ctypes.byref(r), None) == L.TDV_ERR_INVALID_ARG
        c1 = L.tdv_raster(1 << 20, 4, 4, 16, L.U8, 1)  # grey conversion needs 3 channels
        assert lib.tdv_to_gray(h, ctypes.byref(c1), 1 << 21, None) == L.TDV_ERR_INVALID_ARG
        s3 = L.tdv_raster(1 << 20, 4, 4, 12, L.U8, 3)
        d1 = L.tdv_raster(2 << 20, 4, 4, 4, L.U8, 1)  # channel mismatch
        assert lib.tdv_remap(h, ctypes.byref(s3), 1 << 22, 1 << 23, ctypes.byref(d1), None) == L.TDV_ERR_INVALID_ARG
        img = L.tdv_image(1 << 20, 4, 4, 4, L.U8, 1.0)
        assert lib.tdv_prefilter(h, ctypes.byref(img), 9, 1 << 21, None) == L.TDV_ERR_INVALID_ARG
        prm = L.tdv_reproject_params()
        prm.mode = 5
        dr = L.tdv_raster(1 << 20, 4, 4, 16, L.F32, 1)
        assert lib.tdv_reproject(h, ctypes.byref(dr), None, ctypes.byref(prm), 1 << 21, None, None) == L.TDV_ERR_INVALID_ARG
        vol = L.tdv_volume(1 << 20, 4, 4, 8, L.LAYOUT_REF_WHD, L.F32)  # sub-pixel reads HWD
        assert lib.tdv_subpixel(h, ctypes.byref(vol), 1 << 21, 1 << 22, None) == L.TDV_ERR_INVALID_ARG
        assert lib.tdv_write_ply(None, 1, None, 2, 2) == L.TDV_ERR_INVALID_ARG
        z = (ctypes.c_double * 9)()  # a singular P R
        d8 = (ctypes.c_double * 8)()
        assert lib.tdv_rectify_maps(h, z, d8, z, z, 4, 4, 1 << 21, 1 << 22, None) == L.TDV_ERR_INVALID_ARG
    finally:
        lib.tdv_ctx_destroy(h)


def test_reconstruction_chain_with_identity_rectification(orc):
    # K = P, R = I, no distortion: the maps are the pixel grid and the remap
    # the identity, so the chain is gauss5 -> SSD -> WTA -> opening -> direct
    rng = np.random.default_rng(3)
    H, W, D = 12, 20, 4
    lc = rng.integers(0, 256, (H, W, 3), dtype=np.uint8)
    rc = np.roll(lc, -2, axis=1)
    K = np.array([[50.0, 0, 9.5], [0, 50.0, 6.0], [0, 0, 1]])
    cam = (K, [0.0] * 5, np.eye(3), K)
    mx, my = io.rectify_maps(*cam, W, H)
    assert np.array_equal(mx, np.broadcast_to(np.arange(W, dtype=np.float32), (H, W)))
    cl, dn, v, c = io.reconstruction(lc, rc, (cam, cam), D, zscale=2.0)
    assert np.array_equal(cl, lc)
    _, dref = orc.wta(orc.ssd_cost(io.gauss5(io.to_gray(lc)), io.gauss5(io.to_gray(rc)), D))
    assert np.array_equal(dn, io.open7(dref))
    assert np.array_equal(v[..., 2], dn * np.float32(2.0))
    assert np.all(dn[:, 6:] == np.float32(2 / D))  # the 2-pixel shift, away from the left border


def test_reconstruction_arguments():
    from thundervision_b200 import reconstruction as rc
    with pytest.raises(ValueError):
        rc.StereoMatcher(None, cost="census")
    with pytest.raises(ValueError):
        rc.StereoMatcher(None, optimizer="graphcut")
    with pytest.raises(ValueError):
        rc.Camera(np.eye(3), [0.0] * 9, np.eye(3), np.eye(3))


def test_cost_filtered_arguments_are_validated():
    from thundervision_b200 import _lib as L
    lib = L.lib()
    h = ctypes.c_void_p()
    assert lib.tdv_ctx_create(0, ctypes.byref(h)) == L.TDV_OK
    try:
        img = L.tdv_image(1 << 20, 8, 4, 8, L.U8, 1.0)
        vol = L.tdv_volume(1 << 21, 8, 4, 4, L.LAYOUT_HWD, L.F32)
        prm = L.tdv_cost_params(L.COST_SSD, 2)
        assert lib.tdv_cost_filtered(None, ctypes.byref(img), ctypes.byref(img), ctypes.byref(prm), L.FILTER_GAUSS5,
                                     ctypes.byref(vol), None, None) == L.TDV_ERR_INVALID_ARG
        assert lib.tdv_cost_filtered(h, ctypes.byref(img), ctypes.byref(img), ctypes.byref(prm), 7,
                                     ctypes.byref(vol), None, None) == L.TDV_ERR_INVALID_ARG  # filter kind
        bad = L.tdv_volume(1 << 21, 9, 4, 4, L.LAYOUT_HWD, L.F32)  # not the images' size
        assert lib.tdv_cost_filtered(h, ctypes.byref(img), ctypes.byref(img), ctypes.byref(prm), L.FILTER_GAUSS5,
                                     ctypes.byref(bad), None, None) == L.TDV_ERR_INVALID_ARG
        wide = L.tdv_cost_params(L.COST_NCC, 16)  # radius past 15
        assert lib.tdv_cost_filtered(h, ctypes.byref(img), ctypes.byref(img), ctypes.byref(wide), L.FILTER_GAUSS5,
                                     ctypes.byref(vol), None, None) == L.TDV_ERR_INVALID_ARG
        assert lib.tdv_cost_filtered(h, ctypes.byref(img), ctypes.byref(img), None, L.FILTER_GAUSS5,
                                     ctypes.byref(vol), None, None) == L.TDV_ERR_INVALID_ARG
    finally:
        lib.tdv_ctx_destroy(h)
