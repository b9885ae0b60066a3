"""The oracle pinned to the reference's own code: oracle/_ref/libtdvref.so is
LibThunderVision's semiglobalcpu.cpp, wtacpu.cpp and semiglobal.cu compiled
from the reference tree by `make -C oracle ref` (see oracle/Makefile).  The
oracle's reference CPU recurrence (tdv_oracle.cpp cost_path, REF_CPU), its
reference path table and its WTA must equal that code bit for bit:

  * SGPaths::getDescCPU's table, stale diagonal ends included, for landscape,
    portrait, square and one-pixel images;
  * the aggregated volume of costPath over that table in updateImpl's order,
    its WTACPU::wta disparity map (d/D), and on square images the map
    updateImpl itself leaves, in the reference's literal
    configuration (intensities / 255, P1 = 30/255, P2 = 150/255 divided by
    |dI|, semiglobalcpu.cpp:36-37,99-102) and with 0..255 intensities, on the
    configurations' shapes and on noise;
  * WTACPU::wta on volumes with ties, +INF and NaN.

The reference's penalties are compile-time constants with the |dI| adjust, so
the integer-domain configuration (P1 = 10, P2 = 120, constant) is not run by
the reference's code; the oracle computes it with the same recurrence and a
constant penalty term."""
import ctypes
import os

import numpy as np
import pytest

import oracle
from thundervision_b200 import synthetic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libtdvref.so")


@pytest.fixture(scope="module")
def ref():
    if os.path.isdir(os.path.join(oracle.REFERENCE_TREE, "LibThunderVision")):
        oracle.build_ref()  # make: rebuilt only when a source changed
    if not os.path.exists(REF_LIB):
        pytest.skip("oracle/_ref/libtdvref.so not built (the reference tree is not on this machine)")
    lib = ctypes.CDLL(REF_LIB)
    f32p = ctypes.POINTER(ctypes.c_float)
    lib.ref_path_table.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int32)]
    lib.ref_path_table.restype = ctypes.c_int
    for n in ("ref_semiglobal_cpu", "ref_semiglobal_cpu_volume"):
        getattr(lib, n).argtypes = [f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, f32p, f32p]
    lib.ref_wta.argtypes = [f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, f32p]
    return lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


@pytest.mark.parametrize("W,H", [(1, 1), (1, 7), (7, 1), (2, 5), (5, 2), (17, 3), (3, 17), (64, 48), (48, 64),
                                 (50, 50), (384, 288), (288, 384), (1920, 1080)])
def test_path_table(ref, W, H):
    n = ref.ref_path_table(W, H, None)
    got = np.empty((n, 7), np.int32)
    ref.ref_path_table(W, H, got.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    np.testing.assert_array_equal(oracle.path_table(W, H, oracle.TABLE_REF), got)


def _ref_sgm(ref, C, guide):
    """(S, d/D) of the reference code: S from costPath over SGPaths in
    updateImpl's order into a zeroed volume, d/D from WTACPU::wta on it, and,
    for square images, d/D from updateImpl itself as well (it must agree).
    updateImpl zeroes its volume with x and y swapped
    (tdvision/semiglobalcpu.cpp:44-54): only for W == H does that clear every
    cell; for W > H some cells keep what the allocator left there, for W < H
    it writes past the end of the volume."""
    W, H, D = C.shape
    C = np.ascontiguousarray(C, np.float32)
    g = np.ascontiguousarray(guide, np.float32)
    S = np.empty_like(C)
    ref.ref_semiglobal_cpu_volume(_p(C), W, H, D, _p(g), _p(S))
    dn = np.empty((H, W), np.float32)
    ref.ref_wta(_p(S), W, H, D, _p(dn))
    if W == H:
        dn_upd = np.empty((H, W), np.float32)
        ref.ref_semiglobal_cpu(_p(C), W, H, D, _p(g), _p(dn_upd))
        np.testing.assert_array_equal(dn_upd, dn)
    return S, dn


def _same(a, b):
    np.testing.assert_array_equal(np.isnan(a), np.isnan(b))
    m = ~np.isnan(a)
    np.testing.assert_array_equal(a[m], b[m])


CASES = [("small", 384, 288, 16), ("medium", 640, 480, 64), ("portrait", 120, 200, 32), ("wide", 301, 45, 100),
         ("square", 160, 160, 48)]


@pytest.mark.parametrize("name,W,H,D", CASES)
@pytest.mark.parametrize("domain", ["reference", "integer"])
def test_semiglobal_cpu(ref, name, W, H, D, domain):
    if name == "small":
        L, R = synthetic.pair_small(11)[:2]
    elif name == "medium":
        L, R = synthetic.pair_medium(5)[:2]
    else:
        L, R = synthetic.make_pair(W, H, D, W + H, n_rects=4, slanted=True, salt_pepper=0.02)[:2]
    s = np.float32(1) / np.float32(255) if domain == "reference" else np.float32(1)
    Lf, Rf = oracle.u8_to_f32(L, s), oracle.u8_to_f32(R, s)
    C = oracle.bt_cost(Lf, Rf, D, layout=oracle.LAYOUT_REF_WHD)
    p1, p2 = np.float32(30) / np.float32(255), np.float32(150) / np.float32(255)
    d, dn, S = oracle.sgm(C, Lf, p1, p2, p2_mode=oracle.P2_ADJUST, paths=8, table=oracle.TABLE_REF,
                          semantics=oracle.SEM_REF_CPU, layout=oracle.LAYOUT_REF_WHD, threads=8)
    S_ref, dn_ref = _ref_sgm(ref, C, Lf)
    _same(S, S_ref)
    np.testing.assert_array_equal(dn, dn_ref)


@pytest.mark.parametrize("W,H,D", [(33, 21, 8), (21, 33, 16), (40, 40, 5)])
def test_semiglobal_cpu_noise(ref, W, H, D):
    """Uniform noise: ties, equal neighbours (|dI| = 0 gives an infinite P2
    term) and the excluded d = D-1 winning the minimum often."""
    rng = np.random.default_rng(W * H + D)
    L = rng.integers(0, 256, (H, W)).astype(np.uint8)
    R = rng.integers(0, 256, (H, W)).astype(np.uint8)
    L[:, ::3] = L[:, :1]  # runs of equal intensities
    s = np.float32(1) / np.float32(255)
    Lf, Rf = oracle.u8_to_f32(L, s), oracle.u8_to_f32(R, s)
    C = oracle.bt_cost(Lf, Rf, D, layout=oracle.LAYOUT_REF_WHD)
    p1, p2 = np.float32(30) / np.float32(255), np.float32(150) / np.float32(255)
    d, dn, S = oracle.sgm(C, Lf, p1, p2, p2_mode=oracle.P2_ADJUST, paths=8, table=oracle.TABLE_REF,
                          semantics=oracle.SEM_REF_CPU, layout=oracle.LAYOUT_REF_WHD)
    S_ref, dn_ref = _ref_sgm(ref, C, Lf)
    _same(S, S_ref)
    np.testing.assert_array_equal(dn, dn_ref)


def test_wta(ref):
    rng = np.random.default_rng(3)
    W, H, D = 37, 23, 19
    V = rng.integers(0, 6, (W, H, D)).astype(np.float32)  # many ties
    V[rng.random(V.shape) < 0.05] = np.inf
    V[rng.random(V.shape) < 0.05] = np.nan
    V[0, 0, :] = np.inf
    V[1, 0, :] = np.nan
    dn_ref = np.empty((H, W), np.float32)
    ref.ref_wta(_p(V), W, H, D, _p(dn_ref))
    _, dn = oracle.wta(V, layout=oracle.LAYOUT_REF_WHD)
    np.testing.assert_array_equal(dn, dn_ref)
