"""Differentiable soft-argmin SGM: forward and hand-written adjoint kernels.

Tolerances:
  * FP64 kernels vs the FP64 oracle (same recurrence, same direction order):
    dhat within 1e-12 relative, dC / dP1 / dP2 within 1e-9 relative (sums
    over disparities are reduced in a different order);
  * torch.autograd.gradcheck in FP64 (finite differences, eps 1e-6,
    atol 1e-5, rtol 1e-4);
  * FP32 kernels vs FP64 kernels at 960x540, D=128: gradients within 1e-4
    relative (norm-wise) -- the bar the path is held to.
"""
import numpy as np
import pytest
import torch

from thundervision_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def _bt_volume(orc, W, H, D, seed):
    L, R, gt, occ = syn.make_pair(W, H, D, seed, n_rects=3, slanted=True)
    C = orc.bt_cost(orc.u8_to_f32(L), orc.u8_to_f32(R), D).astype(np.float64)
    # break the ties of integer-valued BT costs so min-plus choices are unique
    rng = np.random.default_rng(seed)
    C = C + rng.uniform(0, 0.25, size=C.shape)
    return C, gt.astype(np.float64)


@pytest.mark.parametrize("W,H,D,paths", [(13, 9, 6, 8), (9, 13, 5, 4), (20, 11, 16, 8), (7, 1, 3, 8)])
def test_fp64_matches_oracle(ctx, orc, W, H, D, paths):
    from thundervision_b200.soft import soft_sgm
    C, _ = _bt_volume(orc, W, H, D, W * H + D)
    g = np.random.default_rng(1).normal(size=(H, W))
    _, dh_ref = orc.soft_sgm_fwd(C, 1.5, 7.25, tau=0.8, paths=paths)
    dC_ref, d1_ref, d2_ref = orc.soft_sgm_bwd(C, 1.5, 7.25, g, tau=0.8, paths=paths)
    for ck in (0, 3):
        c = torch.tensor(C, device="cuda", requires_grad=True)
        p1 = torch.tensor(1.5, dtype=torch.float64, device="cuda", requires_grad=True)
        p2 = torch.tensor(7.25, dtype=torch.float64, device="cuda", requires_grad=True)
        dh = soft_sgm(c, p1, p2, tau=0.8, paths=paths, checkpoint=ck, ctx=ctx)
        (dh * torch.tensor(g, device="cuda")).sum().backward()
        np.testing.assert_allclose(dh.detach().cpu().numpy(), dh_ref, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(c.grad.cpu().numpy(), dC_ref, rtol=1e-9, atol=1e-11)
        assert p1.grad.item() == pytest.approx(d1_ref, rel=1e-9, abs=1e-11)
        assert p2.grad.item() == pytest.approx(d2_ref, rel=1e-9, abs=1e-11)


def test_gradcheck_fp64_crop(ctx, orc):
    """FP64 gradcheck on a 64x48, D=16 crop (cost, P1 and P2)."""
    from thundervision_b200.soft import soft_sgm
    C, _ = _bt_volume(orc, 64, 48, 16, 5)
    c = torch.tensor(C, device="cuda", requires_grad=True)
    p1 = torch.tensor(10.0, dtype=torch.float64, device="cuda", requires_grad=True)
    p2 = torch.tensor(120.0, dtype=torch.float64, device="cuda", requires_grad=True)
    f = lambda cc, a, b: soft_sgm(cc, a, b, tau=1.0, paths=8, ctx=ctx)
    assert torch.autograd.gradcheck(f, (c, p1, p2), eps=1e-6, atol=1e-5, rtol=1e-4, fast_mode=True)


def test_gradcheck_fp64_full_jacobian_small(ctx, orc):
    from thundervision_b200.soft import soft_sgm
    C, _ = _bt_volume(orc, 6, 5, 4, 9)
    c = torch.tensor(C, device="cuda", requires_grad=True)
    p1 = torch.tensor(1.25, dtype=torch.float64, device="cuda", requires_grad=True)
    p2 = torch.tensor(3.5, dtype=torch.float64, device="cuda", requires_grad=True)
    for ck in (0, 2):
        f = lambda cc, a, b: soft_sgm(cc, a, b, tau=0.5, paths=8, checkpoint=ck, ctx=ctx)
        assert torch.autograd.gradcheck(f, (c, p1, p2), eps=1e-6, atol=1e-5, rtol=1e-4)


def test_checkpoint_equals_codes(ctx, orc):
    from thundervision_b200.soft import soft_sgm
    C, _ = _bt_volume(orc, 120, 70, 32, 3)
    grads = []
    for ck in (0, 32, 7):
        c = torch.tensor(C, device="cuda", requires_grad=True)
        p = torch.tensor([10.0, 120.0], dtype=torch.float64, device="cuda", requires_grad=True)
        dh = soft_sgm(c, p[0], p[1], tau=1.0, checkpoint=ck, ctx=ctx)
        dh.sum().backward()
        grads.append((c.grad.cpu().numpy(), p.grad.cpu().numpy()))
    for gc, gp in grads[1:]:
        np.testing.assert_array_equal(gc, grads[0][0])
        np.testing.assert_allclose(gp, grads[0][1], rtol=1e-12)


@pytest.mark.slow
def test_fp32_within_1e4_of_fp64_config2(ctx, orc):
    """960x540, D=128 BT volume, 8 paths, tau=1, L1 loss vs ground truth:
    FP32 gradients within 1e-4 (relative, norm-wise) of FP64."""
    from thundervision_b200.soft import soft_sgm
    L, R, gt, occ = syn.make_pair(960, 540, 128, 17, n_rects=8, slanted=True, salt_pepper=0.02)
    C32 = torch.from_numpy(orc.bt_cost(orc.u8_to_f32(L), orc.u8_to_f32(R), 128)).cuda()
    gt_t = torch.from_numpy(gt.astype(np.float64)).cuda()
    out = {}
    for dt in (torch.float64, torch.float32):
        c = C32.to(dt).clone().requires_grad_(True)
        p = torch.tensor([10.0, 120.0], dtype=dt, device="cuda", requires_grad=True)
        dh = soft_sgm(c, p[0], p[1], tau=1.0, checkpoint=32, ctx=ctx)
        loss = (dh.double() - gt_t).abs().mean()
        loss.backward()
        out[dt] = (c.grad.double(), p.grad.double(), loss.item())
    g64, p64, l64 = out[torch.float64]
    g32, p32, l32 = out[torch.float32]
    assert abs(l32 - l64) <= 1e-4 * abs(l64)
    rel = (torch.linalg.vector_norm(g32 - g64) / torch.linalg.vector_norm(g64)).item()
    assert rel <= 1e-4, rel
    prel = (torch.linalg.vector_norm(p32 - p64) / torch.linalg.vector_norm(p64)).item()
    assert prel <= 1e-4, prel
