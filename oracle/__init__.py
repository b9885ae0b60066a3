"""CPU oracle for the dense-stereo hot path -- TEST INFRASTRUCTURE ONLY.

numpy front end over ``liborc.so`` (``tdv_oracle.cpp``), a C++ restatement of
LibThunderVision's BT/SSD/NCC costs, ``SGPaths`` table, ``costPath`` SGM
recurrence, ``WTACPU::wta`` and the DP scanline matcher.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arm
import this module, and only as the checker or the timed CPU baseline.

Volumes are numpy arrays indexed like the chosen layout: REF_WHD arrays have
shape (W, H, D) (the reference DSI, tdvision/dsimem.cpp:34-35), HWD arrays
shape (H, W, D).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liborc.so")
_lib = None

LAYOUT_REF_WHD, LAYOUT_HWD = 0, 1
SEM_STANDARD, SEM_REF_CPU, SEM_REF_GPU = 0, 1, 2
TABLE_FULL, TABLE_REF = 0, 1
P2_CONST, P2_ADJUST = 0, 1

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_u16p = ctypes.POINTER(ctypes.c_uint16)
_i32p = ctypes.POINTER(ctypes.c_int32)


# where the reference tree lies on the machine that builds oracle/_ref
REFERENCE_TREE = os.environ.get("TDV_REFERENCE_TREE", "/root/reference")


def build(force=False):
    """Compile liborc.so with the recipe in oracle/Makefile (make rebuilds it
    when tdv_oracle.cpp is newer)."""
    subprocess.check_call(["make", "-s", "-C", _HERE] + (["-B"] if force else []))


def build_ref():
    """Compile the reference's own CPU aggregation (semiglobalcpu.cpp,
    wtacpu.cpp, semiglobal.cu from the reference tree) into
    _ref/libtdvref.so, the code the oracle is checked against
    (tests/test_oracle_ref.py)."""
    subprocess.check_call(["make", "-s", "-C", _HERE, "ref", "REF=" + REFERENCE_TREE])


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(_LIB)
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def u8_to_f32(img, scale=1.0):
    img = np.ascontiguousarray(img, dtype=np.uint8)
    out = np.empty(img.shape, np.float32)
    lib().orc_u8_to_f32(_p(img, ctypes.POINTER(ctypes.c_uint8)), ctypes.c_size_t(img.size),
                        ctypes.c_float(scale), _p(out, _f32p))
    return out


def _vol(W, H, D, layout):
    shape = (W, H, D) if layout == LAYOUT_REF_WHD else (H, W, D)
    return np.empty(shape, np.float32)


def _img(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def bt_cost(L, R, D, layout=LAYOUT_HWD):
    L, R = _img(L), _img(R)
    H, W = L.shape
    out = _vol(W, H, D, layout)
    lib().orc_bt_cost(_p(L, _f32p), _p(R, _f32p), W, H, D, layout, _p(out, _f32p))
    return out


def ssd_cost(L, R, D, radius=3, layout=LAYOUT_HWD):
    L, R = _img(L), _img(R)
    H, W = L.shape
    out = _vol(W, H, D, layout)
    lib().orc_ssd_cost(_p(L, _f32p), _p(R, _f32p), W, H, D, radius, layout, _p(out, _f32p))
    return out


def ncc_cost(L, R, D, radius=1, layout=LAYOUT_HWD):
    L, R = _img(L), _img(R)
    H, W = L.shape
    out = _vol(W, H, D, layout)
    lib().orc_ncc_cost(_p(L, _f32p), _p(R, _f32p), W, H, D, radius, layout, _p(out, _f32p))
    return out


def cost_pair(L, R, D, kind, radius=0, layout=LAYOUT_HWD):
    """BT / SSD / NCC (kind 0 / 1 / 2) for images of different sizes: the
    DSI is the smaller size, each image's taps clamp to its own edges."""
    L, R = _img(L), _img(R)
    W, H = min(L.shape[1], R.shape[1]), min(L.shape[0], R.shape[0])
    out = _vol(W, H, D, layout)
    lib().orc_cost_pair(_p(L, _f32p), L.shape[1], L.shape[0], _p(R, _f32p), R.shape[1], R.shape[0], D, kind,
                        radius, layout, _p(out, _f32p))
    return out


def path_table(W, H, table=TABLE_REF):
    n = lib().orc_path_count(W, H)
    out = np.empty((n, 7), np.int32)
    lib().orc_path_table(W, H, table, _p(out, _i32p))
    return out


def _dims(vol, layout):
    if layout == LAYOUT_REF_WHD:
        W, H, D = vol.shape
    else:
        H, W, D = vol.shape
    return W, H, D


def wta(vol, layout=LAYOUT_HWD):
    vol = np.ascontiguousarray(vol, dtype=np.float32)
    W, H, D = _dims(vol, layout)
    dn = np.empty((H, W), np.float32)
    d = np.empty((H, W), np.uint16)
    lib().orc_wta(_p(vol, _f32p), layout, W, H, D, _p(dn, _f32p), _p(d, _u16p))
    return d, dn


def sgm(cost, guide, p1, p2, p2_mode=P2_CONST, paths=8, table=TABLE_FULL,
        semantics=SEM_STANDARD, layout=LAYOUT_HWD, threads=1, want_S=True):
    """Aggregate + WTA.  Returns (disp u16, disp/D f32, S or None)."""
    cost = np.ascontiguousarray(cost, dtype=np.float32)
    guide = _img(guide)
    W, H, D = _dims(cost, layout)
    S = np.empty_like(cost) if want_S else None
    dn = np.empty((H, W), np.float32)
    d = np.empty((H, W), np.uint16)
    lib().orc_sgm(_p(cost, _f32p), layout, _p(guide, _f32p), W, H, D,
                  ctypes.c_float(p1), ctypes.c_float(p2), p2_mode, paths, table, semantics,
                  threads, _p(S, _f32p) if S is not None else None, _p(dn, _f32p), _p(d, _u16p))
    return d, dn, S


def lr_check(S, disp, thr=1, layout=LAYOUT_HWD):
    S = np.ascontiguousarray(S, dtype=np.float32)
    W, H, D = _dims(S, layout)
    dl = np.array(disp, dtype=np.uint16, copy=True, order="C")
    dr = np.empty((H, W), np.uint16)
    lib().orc_lr_check(_p(S, _f32p), layout, W, H, D, thr, _p(dl, _u16p), _p(dr, _u16p))
    return dl, dr


def dp(cost, layout=LAYOUT_HWD):
    cost = np.ascontiguousarray(cost, dtype=np.float32)
    W, H, D = _dims(cost, layout)
    dn = np.empty((H, W), np.float32)
    d = np.empty((H, W), np.uint16)
    lib().orc_dp(_p(cost, _f32p), layout, W, H, D, _p(dn, _f32p), _p(d, _u16p))
    return d, dn


def fastwta(L, R, D, radius=3):
    L, R = _img(L), _img(R)
    H, W = L.shape
    dn = np.empty((H, W), np.float32)
    d = np.empty((H, W), np.uint16)
    lib().orc_fastwta(_p(L, _f32p), _p(R, _f32p), W, H, D, radius, _p(dn, _f32p), _p(d, _u16p))
    return d, dn


def soft_sgm_fwd(cost, p1, p2, tau=1.0, paths=8):
    """FP64 soft-argmin SGM on an HWD volume: returns (S, dhat)."""
    cost = np.ascontiguousarray(cost, dtype=np.float64)
    H, W, D = cost.shape
    S = np.empty_like(cost)
    dh = np.empty((H, W), np.float64)
    lib().orc_soft_sgm_fwd(_p(cost, _f64p), W, H, D, ctypes.c_double(p1), ctypes.c_double(p2),
                           paths, ctypes.c_double(tau), _p(S, _f64p), _p(dh, _f64p))
    return S, dh


def soft_sgm_bwd(cost, p1, p2, g_dhat, tau=1.0, paths=8):
    """FP64 adjoint: returns (dC, dP1, dP2) for upstream gradient g_dhat."""
    cost = np.ascontiguousarray(cost, dtype=np.float64)
    g = np.ascontiguousarray(g_dhat, dtype=np.float64)
    H, W, D = cost.shape
    dC = np.empty_like(cost)
    d1 = ctypes.c_double()
    d2 = ctypes.c_double()
    lib().orc_soft_sgm_bwd(_p(cost, _f64p), W, H, D, ctypes.c_double(p1), ctypes.c_double(p2),
                           paths, ctypes.c_double(tau), _p(g, _f64p), _p(dC, _f64p),
                           ctypes.byref(d1), ctypes.byref(d2))
    return dC, d1.value, d2.value
