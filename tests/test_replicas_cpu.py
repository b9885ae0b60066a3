"""Multi-GPU host logic (replicas only: each rank its own frames or pairs, no
collective on the data path, time = max over ranks), exercised with two
`gloo` ranks on CPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from thundervision_b200.replicas import max_over_ranks, shard_indices


def test_shard_covers_every_item_once_and_balances():
    weights = [1920 * 1080 * 256, 320 * 240 * 32, 640 * 480 * 64, 1280 * 720 * 128, 5, 5, 7, 900 * 300 * 256]
    for world in (1, 2, 3, 8):
        parts = [shard_indices(weights, r, world) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(weights)))
        loads = [sum(weights[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(weights)
    assert shard_indices(weights, 0, 2) == shard_indices(list(weights), 0, 2)
    with pytest.raises(ValueError):
        shard_indices(weights, 2, 2)


def test_max_over_ranks_without_a_group():
    assert max_over_ranks([1.5, 2.0]) == [1.5, 2.0]


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist

    from thundervision_b200 import synthetic
    from thundervision_b200.replicas import shard_pairs
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        got = max_over_ranks([10.0 * (rank + 1), 5.0 - rank])
        mine = shard_indices([3, 1, 4, 1, 5, 9, 2, 6], rank, world)
        # the uneven 64-pair batch: each rank its own share of the pairs
        # (stand-in image arrays of each pair's shape), loads gathered
        shapes = synthetic.batch_shapes(seed=0, n=64)
        pairs = [(np.empty((h, w), np.uint8), np.empty((h, w), np.uint8), d) for (w, h, d) in shapes]
        idx, share = shard_pairs(pairs, rank, world)
        load = sum(p[0].size * p[2] for p in share)
        gathered = [None] * world
        dist.all_gather_object(gathered, (idx, load))
        with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as f:
            f.write(repr((got, mine, gathered)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_to_the_max(tmp_path):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.spawn(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    res = [eval(open(tmp_path / f"r{r}.txt").read()) for r in range(2)]
    for got, _, _ in res:
        assert got == [20.0, 5.0]
    assert sorted(res[0][1] + res[1][1]) == list(range(8))
    # both ranks saw the same split of the 64 pairs: disjoint, complete, balanced
    assert res[0][2] == res[1][2]
    (i0, l0), (i1, l1) = res[0][2]
    assert sorted(i0 + i1) == list(range(64)) and not set(i0) & set(i1)
    assert abs(l0 - l1) <= 1920 * 1080 * 256
