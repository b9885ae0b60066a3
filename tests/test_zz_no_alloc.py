"""tdv_stereo_sgm_static: the entry point for callers that may not allocate
device memory while they run (a control loop with a memory budget fixed at
start-up, a plugin whose host owns all allocations).  Its scratch lives in a
static device array inside the library; these checks call it through the C
ABI and compare it with tdv_stereo_sgm, which allocates its scratch in a
context.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest
import torch

from thundervision_b200 import _lib as L
from thundervision_b200 import api, synthetic

pytestmark = pytest.mark.gpu

STATIC_BYTES = 64 << 20


def _r256(v):
    return (v + 255) & ~255


def _static_need(W, H, D):
    """Scratch bytes the header documents for one pair: BT planes
    16*(W + 9*ceil(W/8)) per row, the volume 128*ppl per pixel, each rounded
    to 256, plus 256."""
    ppl = 1 if D <= 64 else (2 if D <= 128 else 4)
    planes = 16 * (W + 9 * ((W + 7) // 8)) * H
    return _r256(planes) + _r256(W * H * 128 * ppl) + 256


def _static_call(left, right, D, p1, p2, paths, lr, p2_mode=L.P2_CONST, table=L.TABLE_FULL,
                 sem=L.SEM_STANDARD):
    H, W = left.shape
    li = L.tdv_image(left.data_ptr(), W, H, W, L.U8, 1.0)
    ri = L.tdv_image(right.data_ptr(), right.shape[1], right.shape[0], right.shape[1], L.U8, 1.0)
    prm = L.tdv_sgm_params(p1, p2, p2_mode, paths, table, sem)
    disp = torch.full((H, W), 7, dtype=torch.uint16, device=left.device)
    dright = torch.full((H, W), 7, dtype=torch.uint16, device=left.device)
    out = L.tdv_disparity(disp.data_ptr(), None, dright.data_ptr(), lr)
    st = L.lib().tdv_stereo_sgm_static(ctypes.byref(li), ctypes.byref(ri), D, ctypes.byref(prm),
                                       ctypes.byref(out),
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return st, disp, dright


def _check_against_context(ctx, l_np, r_np, D, paths):
    left, right = torch.from_numpy(l_np).cuda(), torch.from_numpy(r_np).cuda()
    st, disp, dright = _static_call(left, right, D, 10.0, 120.0, paths, 1)
    assert st == L.TDV_OK
    ref = ctx.stereo_sgm(left, right, D, 10.0, 120.0, paths=paths, lr=1, right_disp=True)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(disp.cpu().numpy(), ref["disp"].cpu().numpy())
    np.testing.assert_array_equal(dright.cpu().numpy(), ref["disp_right"].cpu().numpy())


def test_static_scratch_matches_context_path_in_sequence():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L.build()
    ctx = api.Context(0)
    try:
        # calls in a row share the static array, which keeps each call's
        # contents: a large pair then a smaller one, a large disparity range
        # then a smaller one on the same size (a full volume of leftover data
        # under the second call), and small before large
        l64, r64 = synthetic.make_pair(160, 96, 256, 31, n_rects=4)[:2]
        cases = [(synthetic.pair_medium(21)[:2], 64, 8),
                 (synthetic.pair_small(22)[:2], 16, 4),
                 ((l64, r64), 256, 8),
                 ((l64, r64), 200, 8),
                 ((l64, r64), 96, 4),
                 ((l64, r64), 256, 4),
                 (synthetic.pair_medium(23)[:2], 64, 8)]
        for (l_np, r_np), D, paths in cases:
            _check_against_context(ctx, l_np, r_np, D, paths)
    finally:
        ctx.close()


def test_static_scratch_size_limit_boundary():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    W, D = 256, 256
    H = 1
    while _static_need(W, H + 1, D) <= STATIC_BYTES:
        H += 1
    assert _static_need(W, H, D) <= STATIC_BYTES < _static_need(W, H + 1, D)
    ctx = api.Context(0)
    try:
        l_np, r_np = synthetic.make_pair(W, H, D, 41, n_rects=4)[:2]
        _check_against_context(ctx, l_np, r_np, D, 8)  # just under the limit: runs
    finally:
        ctx.close()
    over = torch.zeros((H + 1, W), dtype=torch.uint8, device="cuda")
    st, _, _ = _static_call(over, over, D, 10.0, 120.0, 8, 1)
    assert st == L.TDV_ERR_UNSUPPORTED  # one row more: rejected


def test_static_scratch_rejections():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    left = torch.zeros((1080, 1920), dtype=torch.uint8, device="cuda")
    st, _, _ = _static_call(left, left, 256, 10.0, 120.0, 8, 1)
    assert st == L.TDV_ERR_UNSUPPORTED  # needs about 1.1 GB of scratch
    small = torch.zeros((48, 64), dtype=torch.uint8, device="cuda")
    st, _, _ = _static_call(small, small, 16, 10.25, 120.0, 8, 1)
    assert st == L.TDV_ERR_UNSUPPORTED  # P1 not a multiple of 1/2: not the fused path
    st, _, _ = _static_call(small, small, 16, -2.0, 120.0, 8, 1)
    assert st == L.TDV_ERR_UNSUPPORTED  # a negative penalty: not the fused path either
    st, _, _ = _static_call(small, small, 16, 10.0, 120.0, 8, 1, sem=L.SEM_REF_CPU)
    assert st == L.TDV_ERR_UNSUPPORTED
    for bad in (dict(p1=float("nan")), dict(p2=float("inf")), dict(p2_mode=7), dict(table=3), dict(sem=9),
                dict(paths=6)):
        kw = dict(p1=10.0, p2=120.0, paths=8)
        kw.update(bad)
        st, _, _ = _static_call(small, small, 16, kw.pop("p1"), kw.pop("p2"), kw.pop("paths"), 1, **kw)
        assert st == L.TDV_ERR_INVALID_ARG, bad
    other = torch.zeros((48, 80), dtype=torch.uint8, device="cuda")
    st, _, _ = _static_call(small, other, 16, 10.0, 120.0, 8, 1)
    assert st == L.TDV_ERR_INVALID_ARG  # left and right sizes differ
