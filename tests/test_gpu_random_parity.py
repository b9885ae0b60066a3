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
