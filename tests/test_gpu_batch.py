"""Batched fused stereo (tdv_batch_*): one persistent launch over pairs of
uneven size and disparity range.

Parity bar: every pair's disparities (and normalised / right-view maps)
bit-identical to a per-pair ``stereo_sgm`` call on the same inputs, which the
fused parity tests tie to the oracle; small pairs are also checked against the
oracle directly.  Faults are planted in the device work queue only as items
the kernel rejects (an index out of range) or a dependency nothing satisfies
(bounded wait), never as memory the kernel would touch.
"""
import numpy as np
import pytest
import torch

from thundervision_b200 import synthetic as syn
from thundervision_b200 import _lib as L

pytestmark = pytest.mark.gpu

SHAPES = [  # (W, H, D, lr)
    (96, 64, 16, None), (257, 31, 100, 1), (64, 96, 64, None), (333, 17, 256, 1),
    (33, 33, 1, None), (400, 120, 128, 1), (129, 80, 65, None), (200, 48, 32, 2),
]


def _pairs(shapes, seed=0):
    out = []
    for i, (W, H, D, lr) in enumerate(shapes):
        Lh, Rh, _, _ = syn.make_pair(W, H, D, syn.pair_seed(seed, i) % (2 ** 31), n_rects=4, slanted=True)
        out.append((torch.from_numpy(Lh).cuda(), torch.from_numpy(Rh).cuda(), D, lr))
    return out


def _per_pair(ctx, pairs, paths=8):
    res = []
    for (l, r, D, lr) in pairs:
        res.append(ctx.stereo_sgm(l, r, D, 10, 120, paths=paths, lr=lr, norm=True,
                                  right_disp=lr is not None))
    return res


def _same(batch_out, ref):
    for i, (a, b) in enumerate(zip(batch_out, ref)):
        for key in b:
            assert key in a, (i, key)
            np.testing.assert_array_equal(a[key].cpu().numpy(), b[key].cpu().numpy(),
                                          err_msg=f"pair {i} {key}")


def _batch(ctx, pairs, paths=8):
    from thundervision_b200 import Batch
    return Batch(ctx, pairs, 10, 120, paths=paths, norm=True, right_disp="lr")


@pytest.mark.parametrize("paths", [8, 4])
@pytest.mark.parametrize("tiles", [
    {},
    {"lines_per_cta": 3, "rows_per_cta": 1, "order": 1},
    {"split_disparity": 1, "rows_per_cta": 5},
    {"lines_per_cta": 24, "rows_per_cta": 25, "split_disparity": 1},
    {"lines_per_cta": 7, "rows_per_cta": 12, "split_disparity": 0},
    {"ctas_per_sm": 2},
    {"ctas_per_sm": 2, "lines_per_cta": 24, "rows_per_cta": 25, "split_disparity": 1},
])
def test_batch_matches_per_pair(ctx, paths, tiles):
    pairs = _pairs(SHAPES, seed=paths)
    ref = _per_pair(ctx, pairs, paths)
    b = _batch(ctx, pairs, paths)
    if tiles:
        b.set_tiles(**tiles)
    b.run()
    b.status()
    _same(b.outputs, ref)
    # a second run over the same buffers gives the same maps
    b.run()
    b.status()
    _same(b.outputs, ref)
    b.close()


def test_batch_small_pairs_match_oracle(ctx, orc):
    pairs = _pairs([(96, 64, 16, None), (120, 40, 64, 1), (70, 50, 100, None)], seed=3)
    b = _batch(ctx, pairs)
    b.run()
    b.status()
    for (l, r, D, lr), out in zip(pairs, b.outputs):
        Lf, Rf = orc.u8_to_f32(l.cpu().numpy()), orc.u8_to_f32(r.cpu().numpy())
        C = orc.bt_cost(Lf, Rf, D)
        d_ref, dn_ref, S_ref = orc.sgm(C, Lf, 10, 120, threads=8)
        if lr is None:
            np.testing.assert_array_equal(out["disp"].cpu().numpy(), d_ref)
            np.testing.assert_array_equal(out["disp_norm"].cpu().numpy(), dn_ref)
        else:
            dl, dr = orc.lr_check(S_ref, d_ref, thr=lr)
            np.testing.assert_array_equal(out["disp"].cpu().numpy(), dl)
            np.testing.assert_array_equal(out["disp_right"].cpu().numpy(), dr)
    b.close()


def test_batch_trace(ctx):
    """The diagnostic trace: every queue item recorded once, taken before its
    dependency was met and ended after it, with its own pair and pass; maps
    unchanged with the trace on; runs after it record nothing."""
    pairs = _pairs(SHAPES, seed=3)
    ref = _per_pair(ctx, pairs)
    b = _batch(ctx, pairs)
    tr = b.trace().numpy()
    _same(b.outputs, ref)
    n = b.work_queue()[1]
    assert tr.shape == (n, 4)
    take, go, end = tr[:, 0], tr[:, 1], tr[:, 2]
    assert (take > 0).all() and (go >= take).all() and (end >= go).all()
    _, q = _queue(b)
    pp = tr[:, 3] & 0xFFFFFFFF
    np.testing.assert_array_equal(pp, q[:, 0])
    # the first item of a pair's pass never starts before its pass's dependency ended
    for pair in range(len(pairs)):
        for ps in range(2, 9):
            cur = (pp >> 4 == pair) & (pp & 15 == ps)
            prev = (pp >> 4 == pair) & (pp & 15 == ps - 1)
            if cur.any() and prev.any():
                assert go[cur].min() >= end[prev].max() - 1000  # timer granularity
    b.run()
    b.status()
    _same(b.outputs, ref)
    b.close()


def test_batch_graph_replay_video(ctx):
    """Graph replays read the inputs again: rewrite them between replays."""
    shapes = [(160, 96, 64, 1), (320, 48, 128, None), (80, 80, 256, 1)]
    pairs = _pairs(shapes, seed=11)
    b = _batch(ctx, pairs)
    for frame in range(3):
        if frame:
            for i, (l, r, D, lr) in enumerate(pairs):
                W, H = l.shape[1], l.shape[0]
                Lh, Rh, _, _ = syn.make_pair(W, H, D, 1000 * frame + i, n_rects=3, slanted=True)
                l.copy_(torch.from_numpy(Lh))
                r.copy_(torch.from_numpy(Rh))
        ref = _per_pair(ctx, pairs)
        b.graph_launch()
        b.status()
        _same(b.outputs, ref)
    b.close()


def test_batch_autotune_keeps_results(ctx):
    pairs = _pairs([(300, 100, 256, 1), (200, 150, 32, None), (640, 40, 128, None), (64, 200, 64, 1)], seed=5)
    ref = _per_pair(ctx, pairs)
    b = _batch(ctx, pairs)
    tiles, ms = b.autotune(reps=1)
    assert ms > 0 and np.isfinite(ms)
    assert b.tiles == tiles
    b.run()
    b.status()
    _same(b.outputs, ref)
    b.close()


def _queue(b):
    from cuda.bindings import runtime as rt
    p, n, nb = b.work_queue()
    assert nb == 8
    host = np.empty((n, 2), dtype=np.int32)
    torch.cuda.synchronize()
    err, = rt.cudaMemcpy(host.ctypes.data, p, host.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert int(err) == 0
    return p, host


def _write_queue(p, host):
    from cuda.bindings import runtime as rt
    torch.cuda.synchronize()
    err, = rt.cudaMemcpy(p, host.ctypes.data, host.nbytes, rt.cudaMemcpyKind.cudaMemcpyHostToDevice)
    assert int(err) == 0


def test_batch_queue_layout(ctx):
    pairs = _pairs(SHAPES[:4], seed=1)
    b = _batch(ctx, pairs)
    _, q = _queue(b)
    passes = q[:, 0] & 15
    assert np.all(np.diff(passes) >= 0), "queue must be pass-major"
    assert set(np.unique(q[:, 0] >> 4)) == set(range(len(pairs)))
    b.close()


def test_batch_bad_work_item_is_rejected(ctx):
    pairs = _pairs(SHAPES[:3], seed=2)
    ref = _per_pair(ctx, pairs)
    b = _batch(ctx, pairs)
    p, q = _queue(b)
    bad = q.copy()
    bad[len(bad) // 2, 0] = (len(pairs) << 4) | 1  # pair index out of range
    _write_queue(p, bad)
    b.run()
    with pytest.raises(L.TdvError) as ei:
        b.status()
    assert ei.value.status == L.TDV_ERR_BAD_WORK
    bad = q.copy()
    bad[-1, 1] = 1 << 20  # block index out of range
    _write_queue(p, bad)
    b.run()
    with pytest.raises(L.TdvError) as ei:
        b.status()
    assert ei.value.status == L.TDV_ERR_BAD_WORK
    # the context and the batch stay usable
    _write_queue(p, q)
    b.run()
    b.status()
    _same(b.outputs, ref)
    b.close()


def test_batch_unsatisfied_dependency_times_out(ctx):
    """Pair 0's prep items replaced by copies of pair 1's: pair 0's first
    aggregation pass waits for a counter nothing completes and must give up
    within the wait limit, recording TDV_ERR_TIMEOUT."""
    import time
    pairs = _pairs(SHAPES[:3], seed=4)
    ref = _per_pair(ctx, pairs)
    b = _batch(ctx, pairs)
    b.set_wait_limit(0.2)
    p, q = _queue(b)
    bad = q.copy()
    prep1 = np.nonzero(bad[:, 0] == ((1 << 4) | 0))[0]
    prep0 = np.nonzero(bad[:, 0] == ((0 << 4) | 0))[0]
    assert len(prep0) and len(prep1)
    bad[prep0] = bad[prep1[0]]
    _write_queue(p, bad)
    t0 = time.time()
    b.run()
    with pytest.raises(L.TdvError) as ei:
        b.status()
    assert ei.value.status == L.TDV_ERR_TIMEOUT
    assert time.time() - t0 < 10.0
    _write_queue(p, q)
    b.set_wait_limit(2.0)
    b.run()
    b.status()
    _same(b.outputs, ref)
    b.close()
