"""Video loop (double-buffered frames from pinned host memory): every frame's
disparity map, read back to the host, is bit-identical to a ``stereo_sgm``
call on the same frame, for both engines (one persistent batch launch per
frame; the per-frame fused kernels captured as a CUDA graph), with graph
replay on and off, and with consecutive frames on one context or overlapped
on two (one per buffer set, each on its own stream)."""
import numpy as np
import pytest
import torch

from thundervision_b200 import synthetic as syn
from thundervision_b200 import video

pytestmark = pytest.mark.gpu


def _frames(W, H, D, n, seed=3):
    out = []
    for t in range(n):
        Lh, Rh, _, _ = syn.make_pair(W, H, D, syn.pair_seed(seed, t) % (2 ** 31), n_rects=3, slanted=True)
        out.append((torch.from_numpy(Lh).pin_memory(), torch.from_numpy(Rh).pin_memory()))
    return out


@pytest.mark.parametrize("engine,overlap", [("persistent", False), ("launches", False), ("launches", True)])
@pytest.mark.parametrize("graph", [True, False])
@pytest.mark.parametrize("paths", [8, 4])
def test_video_loop_matches_per_frame(ctx, engine, overlap, graph, paths):
    W, H, D, lr = 240, 96, 64, 1
    frames = _frames(W, H, D, 7)
    loop = video.VideoLoop(ctx, W, H, D, 10, 120, paths=paths, lr=lr, graph=graph, autotune=False,
                           engine=engine, overlap=overlap)
    out = [torch.empty((H, W), dtype=torch.uint16).pin_memory() for _ in frames]
    ms = loop.run(frames, out)
    assert ms > 0
    for t, (hl, hr) in enumerate(frames):
        ref = ctx.stereo_sgm(hl.cuda(), hr.cuda(), D, 10, 120, paths=paths, lr=lr)
        np.testing.assert_array_equal(out[t].numpy(), ref["disp"].cpu().numpy(), err_msg=f"frame {t}")
    loop.close()


def test_video_loop_rejects_unknown_engine(ctx):
    with pytest.raises(ValueError):
        video.VideoLoop(ctx, 64, 32, 16, 10, 120, engine="cpu")


def test_video_loop_graphs_survive_caller_context_growth(ctx):
    """The captured kernels keep their scratch while the caller's context
    grows for a larger pair between two runs of the loop."""
    W, H, D = 200, 64, 32
    frames = _frames(W, H, D, 3, seed=9)
    loop = video.VideoLoop(ctx, W, H, D, 10, 120, paths=8, lr=1)
    out = [torch.empty((H, W), dtype=torch.uint16).pin_memory() for _ in frames]
    loop.run(frames, out)
    big = _frames(640, 256, 256, 1, seed=10)[0]
    ctx.stereo_sgm(big[0].cuda(), big[1].cuda(), 256, 10, 120, paths=8, lr=1)
    out2 = [torch.empty((H, W), dtype=torch.uint16).pin_memory() for _ in frames]
    loop.run(frames, out2)
    for t, (hl, hr) in enumerate(frames):
        ref = ctx.stereo_sgm(hl.cuda(), hr.cuda(), D, 10, 120, paths=8, lr=1)["disp"].cpu().numpy()
        np.testing.assert_array_equal(out[t].numpy(), ref, err_msg=f"frame {t}")
        np.testing.assert_array_equal(out2[t].numpy(), ref, err_msg=f"frame {t} after growth")
    loop.close()
