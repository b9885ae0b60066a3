"""The fused 16-bit path computing the reference's own aggregation: the CPU
recurrence of tdvision/semiglobalcpu.cpp:56-126 (start-assign, minimum over
d < D-1), and its GPU recurrence (tdvision/semiglobal.cu:283-466), over the
reference path table of tdvision/semiglobal.cu:57-230 (stale diagonal ends),
in the integer domain (u8 intensities unscaled, P1/P2
multiples of 1/2, constant P2).  Every map is compared bit-for-bit with the
oracle's WTA (+ left-right check), and each test asserts that the fused
kernels ran (not the general float path)."""
import os

import numpy as np
import pytest
import torch

from thundervision_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

SEMS = {"standard": 0, "ref_cpu": 1, "ref_gpu": 2}
TABLES = {"full": 0, "ref": 1}


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def check(ctx, orc, L, R, D, p1, p2, paths, lr, sem="ref_cpu", table="ref", threads=8):
    Lf, Rf = orc.u8_to_f32(L), orc.u8_to_f32(R)
    C = orc.bt_cost(Lf, Rf, D)
    d_ref, dn_ref, S_ref = orc.sgm(C, Lf, p1, p2, paths=paths, table=TABLES[table], semantics=SEMS[sem],
                                   threads=threads)
    outs = []

    def call():
        outs.append(ctx.stereo_sgm(dev(L), dev(R), D, p1, p2, paths=paths, table=table, semantics=sem, lr=lr,
                                   norm=True, right_disp=lr is not None))

    # with per-kernel timing (the two pass chains in sequence), then without
    # (concurrent chains on two streams)
    names = [n for n, _ in ctx.kernel_times(call)]
    assert any(n.startswith("fused_pass_H-") for n in names), names
    assert not any(n.startswith("sgm") for n in names), names
    call()
    if lr is not None:
        dl, dr = orc.lr_check(S_ref, d_ref, thr=lr)
        dn = np.where(dl == 0xFFFF, np.float32(-1), dl.astype(np.float32) / np.float32(D))
    for out in outs:
        if lr is None:
            np.testing.assert_array_equal(host(out["disp"]), d_ref)
            np.testing.assert_array_equal(host(out["disp_norm"]), dn_ref)
        else:
            np.testing.assert_array_equal(host(out["disp_right"]), dr)
            np.testing.assert_array_equal(host(out["disp"]), dl)
            np.testing.assert_array_equal(host(out["disp_norm"]), dn)


@pytest.mark.parametrize("paths", [8, 4])
@pytest.mark.parametrize("lr", [None, 1])
def test_plain_small_config(ctx, orc, paths, lr):
    """384x288, D=16, BT, SGM P1=10 P2=120, WTA: the CPU-sized plain config."""
    L, R, _, _ = syn.pair_small(11)
    check(ctx, orc, L, R, 16, 10, 120, paths, lr)


@pytest.mark.parametrize("sem,table", [("ref_cpu", "ref"), ("ref_cpu", "full"), ("standard", "ref"),
                                       ("ref_gpu", "ref"), ("ref_gpu", "full")])
@pytest.mark.parametrize("paths", [8, 4])
def test_plain_gpu_config(ctx, orc, sem, table, paths):
    """640x480, D=64, 8 rectangles + slanted plane + 2 % salt-and-pepper,
    WTA + left-right check (threshold 1)."""
    L, R, _, _ = syn.pair_medium(5)
    check(ctx, orc, L, R, 64, 10, 120, paths, 1, sem=sem, table=table)


@pytest.mark.parametrize("W,H,D", [(1001, 37, 200), (37, 200, 64), (257, 64, 129), (64, 257, 32),
                                   (1920, 24, 256), (24, 300, 16), (101, 61, 48), (61, 101, 100),
                                   (640, 96, 256), (777, 19, 65)])
@pytest.mark.parametrize("lr", [None, 1])
def test_shapes(ctx, orc, W, H, D, lr):
    """Landscape and portrait (the stale ends differ), one cell on both
    repeated lines (101x61: x-y = W-H and x+y = H-1 meet at (50, 10)), D above
    the width, ranges that are not multiples of 64."""
    L, R, _, _ = syn.make_pair(W, H, D, W + 7 * H + D, n_rects=4, slanted=True)
    check(ctx, orc, L, R, D, 10, 120, 8, lr)


@pytest.mark.parametrize("W,H,D", [(1001, 37, 200), (37, 200, 64), (101, 61, 48), (640, 96, 256), (3, 2, 16),
                                   (17, 2, 8), (1, 1, 4)])
@pytest.mark.parametrize("paths", [8, 4])
def test_reference_gpu_recurrence(ctx, orc, W, H, D, paths):
    """The reference's GPU recurrence (tdvision/semiglobal.cu:283-466 without
    its race: starts accumulate, the second step sees C + P1 with the minimum
    of C) over its path table, on the fused path."""
    L, R, _, _ = syn.make_pair(W, H, D, W + 3 * H + D, n_rects=3, slanted=True)
    check(ctx, orc, L, R, D, 10, 120, paths, 1, sem="ref_gpu", table="ref")


@pytest.mark.parametrize("p1,p2", [(30.0, 20.0), (7.5, 300.0), (100.0, 640.0), (0.0, 0.0), (0.5, 1.0)])
def test_noise_and_penalties(ctx, orc, p1, p2):
    """Uniform noise makes the excluded d = D-1 the smallest path cost often,
    so path costs go below zero; large penalties stretch the 16-bit ranges."""
    rng = np.random.default_rng(int(10 * p2 + p1))
    for (W, H, D) in ((133, 71, 16), (71, 133, 64), (300, 40, 256)):
        L = rng.integers(0, 256, (H, W)).astype(np.uint8)
        R = rng.integers(0, 256, (H, W)).astype(np.uint8)
        check(ctx, orc, L, R, D, p1, p2, 8, 1)


@pytest.mark.parametrize("W", [1, 2, 3, 17])
@pytest.mark.parametrize("H", [1, 2, 3, 17])
def test_edge_sizes(ctx, orc, W, H):
    rng = np.random.default_rng(W * 100 + H)
    L = rng.integers(0, 256, size=(H, W), dtype=np.uint8)
    R = rng.integers(0, 256, size=(H, W), dtype=np.uint8)
    for D in (2, 3, 16, 64, 256):
        for paths in (8, 4):
            check(ctx, orc, L, R, D, 10, 120, paths, 1)


def test_d1_takes_the_general_path(ctx, orc):
    """With D = 1 the reference's minimum over d < D-1 is empty: the general
    path reproduces it."""
    L, R, _, _ = syn.pair_small(3)
    Lf, Rf = orc.u8_to_f32(L), orc.u8_to_f32(R)
    d_ref, _, _ = orc.sgm(orc.bt_cost(Lf, Rf, 1), Lf, 10, 120, table=1, semantics=1)
    out = ctx.stereo_sgm(dev(L), dev(R), 1, 10, 120, table="ref", semantics="ref_cpu")
    np.testing.assert_array_equal(host(out["disp"]), d_ref)


def test_deterministic_and_graph_safe(ctx):
    L, R, _, _ = syn.pair_medium(9)
    a = host(ctx.stereo_sgm(dev(L), dev(R), 64, 10, 120, table="ref", semantics="ref_cpu", lr=1)["disp"])
    b = host(ctx.stereo_sgm(dev(L), dev(R), 64, 10, 120, table="ref", semantics="ref_cpu", lr=1)["disp"])
    np.testing.assert_array_equal(a, b)
    # another size in between, then the first again: the cached weights follow the size
    L2, R2, _, _ = syn.pair_small(9)
    ctx.stereo_sgm(dev(L2), dev(R2), 16, 10, 120, table="ref", semantics="ref_cpu", lr=1)
    c = host(ctx.stereo_sgm(dev(L), dev(R), 64, 10, 120, table="ref", semantics="ref_cpu", lr=1)["disp"])
    np.testing.assert_array_equal(a, c)


@pytest.mark.slow
def test_full_hd_d256_reference_semantics(ctx, orc):
    """1920x1080, D=256, 8 paths, reference CPU recurrence and table, WTA +
    left-right check: fused kernels vs the oracle on all host cores."""
    vs = syn.VideoStream(seed=2)
    L, R, _, _ = vs.frame(0)
    check(ctx, orc, L, R, 256, 10, 120, 8, 1, threads=os.cpu_count() or 8)
