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


def _static_call(left, right, D, p1, p2, paths, lr):
    H, W = left.shape
    li = L.tdv_image(left.data_ptr(), W, H, W, L.U8, 1.0)
    ri = L.tdv_image(right.data_ptr(), W, H, W, L.U8, 1.0)
    prm = L.tdv_sgm_params(p1, p2, L.P2_CONST, paths, L.TABLE_FULL, L.SEM_STANDARD)
    disp = torch.full((H, W), 7, dtype=torch.uint16, device=left.device)
    dright = torch.full((H, W), 7, dtype=torch.uint16, device=left.device)
    out = L.tdv_disparity(disp.data_ptr(), None, dright.data_ptr(), lr)
    st = L.lib().tdv_stereo_sgm_static(ctypes.byref(li), ctypes.byref(ri), D, ctypes.byref(prm),
                                       ctypes.byref(out),
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return st, disp, dright


def test_static_scratch_matches_context_path_twice():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L.build()
    ctx = api.Context(0)
    try:
        # two calls in a row on different pairs and sizes: the second must not
        # see anything of the first in the shared static array
        cases = [(synthetic.pair_medium(21)[:2], 64, 8), (synthetic.pair_small(22)[:2], 16, 4)]
        for (l_np, r_np), D, paths in cases:
            left, right = torch.from_numpy(l_np).cuda(), torch.from_numpy(r_np).cuda()
            st, disp, dright = _static_call(left, right, D, 10.0, 120.0, paths, 1)
            assert st == L.TDV_OK
            ref = ctx.stereo_sgm(left, right, D, 10.0, 120.0, paths=paths, lr=1, right_disp=True)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(disp.cpu().numpy(), ref["disp"].cpu().numpy())
            np.testing.assert_array_equal(dright.cpu().numpy(), ref["disp_right"].cpu().numpy())
    finally:
        ctx.close()


def test_static_scratch_rejects_what_does_not_fit():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    left = torch.zeros((1080, 1920), dtype=torch.uint8, device="cuda")
    st, _, _ = _static_call(left, left, 256, 10.0, 120.0, 8, 1)
    assert st == L.TDV_ERR_UNSUPPORTED  # needs about 1.1 GB of scratch
    small = torch.zeros((48, 64), dtype=torch.uint8, device="cuda")
    st, _, _ = _static_call(small, small, 16, 10.25, 120.0, 8, 1)
    assert st == L.TDV_ERR_UNSUPPORTED  # P1 not a multiple of 1/2: not the fused path
