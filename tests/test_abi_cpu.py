"""C-ABI checks that need no GPU: the library builds and loads, exports every
symbol include/tdv_stereo.h declares, and rejects bad arguments before any
CUDA call (the reference's stages raise CUException instead,
tdvision/cuerr.hpp:73-78)."""
import ctypes
import os
import re
import subprocess

import pytest

from thundervision_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "tdv_stereo.h")
FAKE = 0x10000  # never dereferenced: every call below fails validation first


@pytest.fixture(scope="module")
def lib():
    L.build()
    return L.lib()


@pytest.fixture()
def hctx(lib):
    h = ctypes.c_void_p()
    assert lib.tdv_ctx_create(0, ctypes.byref(h)) == L.TDV_OK
    yield h
    lib.tdv_ctx_destroy(h)


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set()
    for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(tdv_[a-z0-9_]+)\s*\(", src, flags=re.M):
        line = src[src.rfind("\n", 0, m.start()) + 1:m.end()]
        if "typedef" in line:
            continue
        names.add(m.group(1))
    return names


def test_header_declares_what_the_binding_lists():
    assert declared_functions() == set(L.EXPORTS)


def test_every_declared_symbol_is_exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    for name in declared_functions():
        assert name in exported, name
        assert hasattr(lib, name)


def test_library_is_sm100a_only():
    # the build recipe compiles one target: sm_100a (no other arch, no PTX JIT)
    mk = open(os.path.join(ROOT, "thundervision_b200", "csrc", "Makefile")).read()
    assert "arch=compute_100a,code=sm_100a" in mk
    assert "compute_90" not in mk and "sm_80" not in mk


def test_version_and_strings(lib):
    assert lib.tdv_version() == 1
    assert lib.tdv_status_string(L.TDV_ERR_OOM) == b"out of memory"
    assert lib.tdv_volume_bytes(640, 480, 64, L.F32) == 640 * 480 * 64 * 4
    assert lib.tdv_volume_bytes(0, 480, 64, L.F32) == 0


def _img(w=8, h=4, dt=L.U8, ptr=FAKE, pitch=None, scale=1.0):
    return L.tdv_image(ptr, w, h, w if pitch is None else pitch, dt, scale)


def _vol(w=8, h=4, d=4, layout=L.LAYOUT_HWD, ptr=FAKE, dt=L.F32):
    return L.tdv_volume(ptr, w, h, d, layout, dt)


def _params(**kw):
    p = dict(p1=10.0, p2=120.0, p2_mode=L.P2_CONST, paths=8, table=L.TABLE_FULL,
             semantics=L.SEM_STANDARD)
    p.update(kw)
    return L.tdv_sgm_params(**p)


def _out(lr=-1, disp=FAKE):
    return L.tdv_disparity(disp, None, None, lr)


B = ctypes.byref


def test_null_context(lib):
    assert lib.tdv_sgm(None, None, None, None, None, None, None) == L.TDV_ERR_INVALID_ARG
    assert lib.tdv_last_error_string(None) == b"null context"
    assert lib.tdv_ctx_create(0, None) == L.TDV_ERR_INVALID_ARG


def test_sgm_argument_validation(lib, hctx):
    v, o = _vol(), _out()
    cases = [
        (_vol(ptr=0), _params(), "null data pointer"),
        (_vol(w=0), _params(), "bad size"),
        (_vol(layout=7), _params(), "bad layout"),
        (_vol(dt=L.F64), _params(), "dtype"),
        (v, _params(paths=6), "paths"),
        (v, _params(table=3), "bad table"),
        (v, _params(semantics=9), "bad semantics"),
        (v, _params(p2_mode=5), "bad p2_mode"),
        (v, _params(p1=float("inf")), "finite"),
        (v, _params(p2_mode=L.P2_ADJUST), "guide"),
    ]
    for vol, prm, msg in cases:
        st = lib.tdv_sgm(hctx, B(vol), None, B(prm), None, B(o), None)
        assert st == L.TDV_ERR_INVALID_ARG, msg
        assert msg in lib.tdv_last_error_string(hctx).decode()
    big = _vol(d=300)
    assert lib.tdv_sgm(hctx, B(big), None, B(_params()), None, B(o), None) == L.TDV_ERR_UNSUPPORTED
    none_out = L.tdv_disparity(None, None, None, -1)
    assert lib.tdv_sgm(hctx, B(v), None, B(_params()), None, B(none_out), None) == L.TDV_ERR_INVALID_ARG
    bad_agg = _vol(w=9)
    assert lib.tdv_sgm(hctx, B(v), None, B(_params()), B(bad_agg), B(o), None) == L.TDV_ERR_INVALID_ARG
    small_guide = _img(w=4)
    assert lib.tdv_sgm(hctx, B(v), B(small_guide), B(_params()), None, B(o), None) == L.TDV_ERR_INVALID_ARG


def test_cost_argument_validation(lib, hctx):
    li, ri, v = _img(), _img(), _vol()
    p = L.tdv_cost_params(L.COST_SSD, 3)
    assert lib.tdv_cost(hctx, B(_img(pitch=3)), B(ri), B(p), B(v), None) == L.TDV_ERR_INVALID_ARG
    assert lib.tdv_cost(hctx, B(_img(dt=L.U16)), B(ri), B(p), B(v), None) == L.TDV_ERR_INVALID_ARG
    assert lib.tdv_cost(hctx, B(li), B(ri), B(L.tdv_cost_params(5, 1)), B(v), None) == L.TDV_ERR_INVALID_ARG
    assert lib.tdv_cost(hctx, B(li), B(ri), B(L.tdv_cost_params(L.COST_NCC, 99)), B(v),
                        None) == L.TDV_ERR_INVALID_ARG
    # DSI must be sized to the smaller image (tdvision/matchingcost.cpp:20-24)
    assert lib.tdv_cost(hctx, B(li), B(_img(w=6)), B(p), B(v), None) == L.TDV_ERR_INVALID_ARG
    assert lib.tdv_cost(hctx, B(li), B(ri), None, B(v), None) == L.TDV_ERR_INVALID_ARG
    assert lib.tdv_cost(hctx, B(_img(scale=float("nan"))), B(ri), B(p), B(v), None) == L.TDV_ERR_INVALID_ARG


def test_other_entry_points_validate(lib, hctx):
    li, ri, v, o = _img(), _img(), _vol(), _out()
    assert lib.tdv_wta(hctx, B(_vol(ptr=0)), B(o), None) == L.TDV_ERR_INVALID_ARG
    assert lib.tdv_wta(hctx, B(v), B(L.tdv_disparity(None, FAKE, None, 1)), None) == L.TDV_ERR_INVALID_ARG
    assert lib.tdv_dp_scanline(hctx, B(_vol(d=2000)), B(o), None) == L.TDV_ERR_UNSUPPORTED
    assert lib.tdv_dp_scanline(hctx, B(v), B(_out(lr=1)), None) == L.TDV_ERR_UNSUPPORTED
    assert lib.tdv_fast_wta(hctx, B(li), B(ri), 0, 3, B(o), None) == L.TDV_ERR_INVALID_ARG
    assert lib.tdv_fast_wta(hctx, B(li), B(ri), 16, 40, B(o), None) == L.TDV_ERR_INVALID_ARG
    assert lib.tdv_fast_wta(hctx, B(li), B(_img(h=5)), 16, 3, B(o), None) == L.TDV_ERR_INVALID_ARG
    assert lib.tdv_stereo_sgm(hctx, B(li), B(ri), 300, B(_params()), B(o), None) == L.TDV_ERR_UNSUPPORTED
    assert lib.tdv_stereo_sgm(hctx, B(li), B(_img(w=7)), 16, B(_params()), B(o), None) == L.TDV_ERR_INVALID_ARG
    assert lib.tdv_stereo_sgm(hctx, B(_img(w=20000)), B(ri), 16, B(_params()), B(o), None) == L.TDV_ERR_INVALID_ARG


def test_frame_sequence_validation(lib, hctx):
    """tdv_stereo_sgm_frames rejects bad sequences before any CUDA call."""
    n = 3
    ls = (L.tdv_image * n)(*[_img() for _ in range(n)])
    rs = (L.tdv_image * n)(*[_img() for _ in range(n)])
    os_ = (L.tdv_disparity * n)(*[_out() for _ in range(n)])
    f = lib.tdv_stereo_sgm_frames
    assert f(None, n, ls, rs, 16, B(_params()), os_, None) == L.TDV_ERR_INVALID_ARG
    assert f(hctx, 0, ls, rs, 16, B(_params()), os_, None) == L.TDV_ERR_INVALID_ARG
    assert f(hctx, n, None, rs, 16, B(_params()), os_, None) == L.TDV_ERR_INVALID_ARG
    assert f(hctx, n, ls, rs, 300, B(_params()), os_, None) == L.TDV_ERR_UNSUPPORTED
    assert f(hctx, n, ls, rs, 16, B(_params(paths=5)), os_, None) == L.TDV_ERR_INVALID_ARG
    # a frame of another size
    odd = (L.tdv_image * n)(_img(), _img(w=10), _img())
    assert f(hctx, n, odd, rs, 16, B(_params()), os_, None) == L.TDV_ERR_INVALID_ARG
    assert "frame 1" in lib.tdv_last_error_string(hctx).decode()
    # outside the fused path: float images, a P2 that is not a multiple of 1/2
    fl = (L.tdv_image * n)(*[_img(dt=L.F32) for _ in range(n)])
    assert f(hctx, n, fl, fl, 16, B(_params()), os_, None) == L.TDV_ERR_UNSUPPORTED
    assert f(hctx, n, ls, rs, 16, B(_params(p2=120.3)), os_, None) == L.TDV_ERR_UNSUPPORTED
    # an output with every pointer null
    bad = (L.tdv_disparity * n)(_out(), L.tdv_disparity(None, None, None, -1), _out())
    assert f(hctx, n, ls, rs, 16, B(_params()), bad, None) == L.TDV_ERR_INVALID_ARG


def test_u16_dsi_validation(lib, hctx):
    """A 16-bit DSI: BT of u8 images at scale 1 only; never an aggregation."""
    li, ri = _img(), _img()
    v16 = _vol(dt=L.U16)
    assert lib.tdv_cost(hctx, B(li), B(ri), B(L.tdv_cost_params(L.COST_SSD, 1)), B(v16),
                        None) == L.TDV_ERR_UNSUPPORTED
    assert lib.tdv_cost(hctx, B(_img(scale=0.5)), B(_img(scale=0.5)), B(L.tdv_cost_params(L.COST_BT, 0)), B(v16),
                        None) == L.TDV_ERR_UNSUPPORTED
    assert lib.tdv_cost(hctx, B(_img(dt=L.F32)), B(_img(dt=L.F32)), B(L.tdv_cost_params(L.COST_BT, 0)), B(v16),
                        None) == L.TDV_ERR_UNSUPPORTED
    assert lib.tdv_sgm(hctx, B(v16), None, B(_params()), B(_vol(dt=L.U16)), B(_out()),
                       None) == L.TDV_ERR_INVALID_ARG
    assert "aggreg" in lib.tdv_last_error_string(hctx).decode()
    assert lib.tdv_volume_bytes(640, 480, 64, L.U16) == 640 * 480 * 64 * 2


def test_injected_allocator_failure(lib, hctx):
    calls = []

    def alloc(n, user):
        calls.append(n)
        return None  # out of memory

    def release(p, user):
        raise AssertionError("nothing was allocated")

    a, r = L.ALLOC_FN(alloc), L.FREE_FN(release)
    assert lib.tdv_ctx_set_allocator(hctx, a, r, None) == L.TDV_OK
    assert lib.tdv_ctx_reserve(hctx, 640, 480, 64) == L.TDV_ERR_OOM
    assert calls and "scratch" in lib.tdv_last_error_string(hctx).decode()
    # a half-specified allocator is rejected
    assert lib.tdv_ctx_set_allocator(hctx, a, L.FREE_FN(), None) == L.TDV_ERR_INVALID_ARG
    assert lib.tdv_ctx_reserve(hctx, 0, 480, 64) == L.TDV_ERR_INVALID_ARG


def test_injected_allocator_success_is_used(lib):
    h = ctypes.c_void_p()
    assert lib.tdv_ctx_create(0, ctypes.byref(h)) == L.TDV_OK
    blocks, freed = {}, []

    def alloc(n, user):
        buf = ctypes.create_string_buffer(n)  # host memory: never handed to a kernel
        blocks[ctypes.addressof(buf)] = buf
        return ctypes.addressof(buf)

    def release(p, user):
        freed.append(p)

    a, r = L.ALLOC_FN(alloc), L.FREE_FN(release)
    assert lib.tdv_ctx_set_allocator(h, a, r, None) == L.TDV_OK
    assert lib.tdv_ctx_reserve(h, 64, 32, 16) == L.TDV_OK
    n = len(blocks)
    assert n >= 2
    lib.tdv_ctx_destroy(h)
    assert sorted(freed) == sorted(blocks)


def test_batch_argument_validation(lib, hctx):
    def pairs(*specs):
        arr = (L.tdv_batch_pair * len(specs))()
        for i, (li, ri, D) in enumerate(specs):
            arr[i] = L.tdv_batch_pair(li, ri, D, _out())
        return arr

    h = ctypes.c_void_p()
    ok = pairs((_img(), _img(), 16), (_img(w=32, h=9), _img(w=32, h=9), 64))
    assert lib.tdv_batch_create(None, ok, 2, B(_params()), B(h)) == L.TDV_ERR_INVALID_ARG
    assert lib.tdv_batch_create(hctx, ok, 0, B(_params()), B(h)) == L.TDV_ERR_INVALID_ARG
    assert lib.tdv_batch_create(hctx, None, 2, B(_params()), B(h)) == L.TDV_ERR_INVALID_ARG
    assert lib.tdv_batch_create(hctx, ok, 2, B(_params()), None) == L.TDV_ERR_INVALID_ARG
    # only the integer-domain fused path batches
    for prm in (_params(semantics=L.SEM_REF_CPU), _params(table=L.TABLE_REF), _params(p2_mode=L.P2_ADJUST),
                _params(p1=10.25), _params(p2=1300.0)):
        st = lib.tdv_batch_create(hctx, ok, 2, B(prm), B(h))
        assert st in (L.TDV_ERR_UNSUPPORTED, L.TDV_ERR_INVALID_ARG)
    cases = [
        (pairs((_img(dt=L.F32), _img(dt=L.F32), 16)), L.TDV_ERR_UNSUPPORTED, "u8"),
        (pairs((_img(scale=0.5), _img(scale=0.5), 16)), L.TDV_ERR_UNSUPPORTED, "scale"),
        (pairs((_img(), _img(), 300)), L.TDV_ERR_UNSUPPORTED, "max_disp"),
        (pairs((_img(), _img(), 0)), L.TDV_ERR_UNSUPPORTED, "max_disp"),
        (pairs((_img(), _img(w=9), 16)), L.TDV_ERR_INVALID_ARG, "differ"),
        (pairs((_img(), _img(ptr=0), 16)), L.TDV_ERR_INVALID_ARG, "pair 0 right"),
        (pairs((_img(), _img(), 16), (_img(pitch=2), _img(), 16)), L.TDV_ERR_INVALID_ARG, "pair 1 left"),
    ]
    for arr, want, msg in cases:
        assert lib.tdv_batch_create(hctx, arr, len(arr), B(_params()), B(h)) == want, msg
        assert msg in lib.tdv_last_error_string(hctx).decode()
    none_out = (L.tdv_batch_pair * 1)()
    none_out[0] = L.tdv_batch_pair(_img(), _img(), 16, L.tdv_disparity(None, None, None, -1))
    assert lib.tdv_batch_create(hctx, none_out, 1, B(_params()), B(h)) == L.TDV_ERR_INVALID_ARG
    t = L.tdv_batch_tiles(8, 8, 0, 0)
    for fn, args in (("tdv_batch_set_tiles", (B(t),)), ("tdv_batch_get_tiles", (B(t),)),
                     ("tdv_batch_run", (None,)), ("tdv_batch_graph_launch", (None,)),
                     ("tdv_batch_status", (None,)), ("tdv_batch_set_wait_limit", (1.0,))):
        assert getattr(lib, fn)(None, *args) == L.TDV_ERR_INVALID_ARG, fn
    lib.tdv_batch_destroy(None)
