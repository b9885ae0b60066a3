"""Seeded random sweep of tdv_stereo_sgm against the oracle: sizes from 1x1
to 300x200, D from 1 to 256, 4 and 8 paths, every recurrence and table,
penalties in half-units (large ones push the call onto the general path),
with and without the left-right check.  Every map must be bit-exact, on
whichever path the call takes."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

SEMS = ["standard", "ref_cpu", "ref_gpu"]
SEM_ID = {"standard": 0, "ref_cpu": 1, "ref_gpu": 2}


def case(i):
    rng = np.random.default_rng(9000 + i)
    W = int(rng.integers(1, 301))
    H = int(rng.integers(1, 201))
    D = int(rng.choice([1, 2, 3, 7, 16, 31, 64, 65, 100, 128, 129, 200, 256]))
    paths = int(rng.choice([4, 8]))
    sem = SEMS[int(rng.integers(0, 3))]
    table = "ref" if rng.random() < 0.6 else "full"
    p1 = float(rng.integers(0, 101)) / 2
    p2 = float(rng.integers(0, 1601)) / 2
    lr = [None, 0, 1, 3][int(rng.integers(0, 4))]
    L = rng.integers(0, 256, (H, W)).astype(np.uint8)
    if rng.random() < 0.7:  # a shifted copy with noise: a pair with structure
        s = int(rng.integers(0, max(1, min(D, W))))
        R = np.roll(L, -s, axis=1)
        R = np.clip(R.astype(int) + rng.integers(-3, 4, R.shape), 0, 255).astype(np.uint8)
    else:
        R = rng.integers(0, 256, (H, W)).astype(np.uint8)
    return W, H, D, paths, sem, table, p1, p2, lr, L, R


@pytest.mark.parametrize("i", range(160))
def test_random_case(ctx, orc, i):
    W, H, D, paths, sem, table, p1, p2, lr, L, R = case(i)
    Lf, Rf = orc.u8_to_f32(L), orc.u8_to_f32(R)
    d, _, S = orc.sgm(orc.bt_cost(Lf, Rf, D), Lf, p1, p2, paths=paths, table=1 if table == "ref" else 0,
                      semantics=SEM_ID[sem])
    out = ctx.stereo_sgm(torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda(), D, p1, p2, paths=paths,
                         table=table, semantics=sem, lr=lr, right_disp=lr is not None)
    torch.cuda.synchronize()
    if lr is None:
        np.testing.assert_array_equal(out["disp"].cpu().numpy(), d)
    else:
        dl, dr = orc.lr_check(S, d, thr=lr)
        np.testing.assert_array_equal(out["disp"].cpu().numpy(), dl)
        np.testing.assert_array_equal(out["disp_right"].cpu().numpy(), dr)


@pytest.mark.parametrize("seed", range(4))
def test_random_batch_equals_per_pair(ctx, seed):
    """A random uneven batch (one persistent launch) against per-pair calls."""
    from thundervision_b200 import Batch
    rng = np.random.default_rng(9900 + seed)
    pairs, ref = [], []
    for i in range(int(rng.integers(3, 13))):
        W, H = int(rng.integers(1, 400)), int(rng.integers(1, 160))
        D = int(rng.choice([1, 5, 16, 32, 64, 65, 128, 200, 256]))
        lr = [None, 0, 1, 2][int(rng.integers(0, 4))]
        L = rng.integers(0, 256, (H, W)).astype(np.uint8)
        R = np.clip(np.roll(L, -int(rng.integers(0, 6)), axis=1).astype(int) + rng.integers(-3, 4, (H, W)),
                    0, 255).astype(np.uint8)
        l, r = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
        pairs.append((l, r, D, lr))
        ref.append(ctx.stereo_sgm(l, r, D, 10, 120, lr=lr, right_disp=lr is not None))
    b = Batch(ctx, pairs, 10, 120, right_disp="lr")
    b.run()
    b.status()
    for i, (o, want) in enumerate(zip(b.outputs, ref)):
        for k in want:
            assert torch.equal(o[k], want[k]), (i, k)
    b.close()


@pytest.mark.parametrize("seed", range(6))
def test_random_frame_sequence(ctx, orc, seed):
    """A random frame sequence (two lanes) against the oracle, frame by frame."""
    rng = np.random.default_rng(9950 + seed)
    W, H = int(rng.integers(2, 260)), int(rng.integers(2, 120))
    D = int(rng.choice([2, 16, 64, 100, 256]))
    sem = SEMS[int(rng.integers(0, 3))]
    table = "ref" if rng.random() < 0.7 else "full"
    n = int(rng.integers(2, 6))
    frames = []
    for t in range(n):
        L = rng.integers(0, 256, (H, W)).astype(np.uint8)
        R = np.clip(np.roll(L, -int(rng.integers(0, 5)), axis=1).astype(int) + rng.integers(-3, 4, (H, W)),
                    0, 255).astype(np.uint8)
        frames.append((L, R))
    outs = ctx.stereo_sgm_frames([torch.from_numpy(f[0]).cuda() for f in frames],
                                 [torch.from_numpy(f[1]).cuda() for f in frames], D, 10, 120, lr=1,
                                 table=table, semantics=sem)
    torch.cuda.synchronize()
    for (L, R), o in zip(frames, outs):
        Lf, Rf = orc.u8_to_f32(L), orc.u8_to_f32(R)
        d, _, S = orc.sgm(orc.bt_cost(Lf, Rf, D), Lf, 10, 120, paths=8, table=1 if table == "ref" else 0,
                          semantics=SEM_ID[sem])
        dl, _ = orc.lr_check(S, d, thr=1)
        np.testing.assert_array_equal(o["disp"].cpu().numpy(), dl)
