"""The reference's reconstruction chain (tdvision/reconstruction.cpp:9-55) on
the device, through thundervision_b200.reconstruction and through the C++
stage classes of include/tdv_stages.hpp, against the oracle's restatement of
the same chain (oracle/image_ops.reconstruction): every stage bit-exact, so
the rectified colors, the d/D map after the opening, the vertices, the colors
and the PLY text are equal."""
import os
import subprocess

import numpy as np
import pytest
import torch

from oracle import image_ops as io
from thundervision_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

W, H, D = 96, 64, 16


def scene(seed):
    """A color pair: the synthetic grey pair spread over three channels."""
    L, R, _, _ = syn.make_pair(W, H, D, seed, n_rects=4)
    col = lambda g: np.stack([g, (g // 2 + 64).astype(np.uint8), (255 - g).astype(np.uint8)], -1)
    return col(L), col(R)


def cameras():
    """Two cameras with mild distortion and rectifying rotations, and the Q
    of the rectified pair (baseline 3.5 units, focal 90)."""
    K = np.array([[95.0, 0, W / 2 + 0.3], [0, 94.0, H / 2 - 0.2], [0, 0, 1]])
    P = np.array([[90.0, 0, W / 2, 0], [0, 90.0, H / 2, 0], [0, 0, 1, 0]])
    def rot(a):
        c, s = np.cos(a), np.sin(a)
        return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])
    left = (K, [-0.05, 0.01, 0.001, -0.0005, 0.0], rot(0.004), P)
    right = (K, [-0.04, 0.008, -0.0008, 0.0004, 0.0], rot(-0.004), P)
    Q = np.array([[1, 0, 0, -W / 2], [0, 1, 0, -H / 2], [0, 0, 0, 90.0], [0, 0, -1 / 3.5, 0]], np.float32)
    return left, right, Q


def host(t):
    return t.cpu().numpy()


def check(out, ref):
    cl, dn, v, c = ref
    np.testing.assert_array_equal(host(out["rect_left"]), cl)
    np.testing.assert_array_equal(host(out["disp"]), dn)
    np.testing.assert_array_equal(host(out["vertices"]), v)
    np.testing.assert_array_equal(host(out["colors"]), c)


@pytest.mark.parametrize("cost,optimizer", [("ssd", "wta"), ("ncc", "dp"), ("bt", "sgm")])
@pytest.mark.parametrize("graph", [False, True])
def test_reconstruction_matches_oracle_chain(ctx, orc, cost, optimizer, graph):
    from thundervision_b200 import reconstruction as rc
    left, right, Q = cameras()
    m = rc.StereoMatcher(ctx, max_disp=D, cost=cost, optimizer=optimizer)
    rec = rc.Reconstruction(ctx, W, H, rc.Camera(*left), rc.Camera(*right), Q=Q, matcher=m, graph=graph)
    try:
        for t in range(3):  # later frames replay the graph on new inputs
            lc, rcol = scene(40 + t)
            out = rec.update(torch.from_numpy(lc).pin_memory(), torch.from_numpy(rcol).pin_memory())
            torch.cuda.synchronize()
            check(out, io.reconstruction(lc, rcol, (left, right), D, q=Q.ravel(), cost=cost, optimizer=optimizer))
    finally:
        rec.close()


def test_reconstruction_direct_no_filter_and_ply(ctx, orc, tmp_path):
    from thundervision_b200 import reconstruction as rc
    left, right, _ = cameras()
    m = rc.StereoMatcher(ctx, max_disp=D, median_filter=False)
    rec = rc.Reconstruction(ctx, W, H, rc.Camera(*left), rc.Camera(*right), zscale=5.0, matcher=m, dilate=False)
    lc, rcol = scene(7)
    out = rec.update(torch.from_numpy(lc).cuda(), torch.from_numpy(rcol).cuda())
    torch.cuda.synchronize()
    ref = io.reconstruction(lc, rcol, (left, right), D, zscale=5.0, median_filter=False, dilate=False)
    check(out, ref)
    path = tmp_path / "mesh.ply"
    rec.export_ply(path)
    assert path.read_text() == io.ply_text(ref[2], ref[3])
    rec.close()


def test_cpp_reconstruct_matches_oracle_chain(orc, tmp_path):
    from test_cpp_stages import build_demo
    demo = build_demo(str(tmp_path / "stages_demo"))
    left, right, Q = cameras()
    lc, rcol = scene(11)
    lc.tofile(tmp_path / "l.rgb")
    rcol.tofile(tmp_path / "r.rgb")
    cams = []
    for K, dist, R, P in (left, right):
        d8 = np.zeros(8)
        d8[:len(dist)] = dist
        cams += [np.ravel(K), d8, np.ravel(R), np.asarray(P)[:, :3].ravel()]
    np.concatenate(cams + [Q.astype(np.float64).ravel()]).astype(np.float64).tofile(tmp_path / "cams.f64")
    prefix = str(tmp_path / "out")
    r = subprocess.run([demo, "reconstruct", str(W), str(H), str(D), str(tmp_path / "l.rgb"),
                        str(tmp_path / "r.rgb"), str(tmp_path / "cams.f64"), prefix], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    cl, dn, v, c = io.reconstruction(lc, rcol, (left, right), D, q=Q.ravel())
    np.testing.assert_array_equal(np.fromfile(prefix + ".disp.f32", np.float32).reshape(H, W), dn)
    np.testing.assert_array_equal(np.fromfile(prefix + ".verts.f32", np.float32).reshape(H, W, 3), v)
    np.testing.assert_array_equal(np.fromfile(prefix + ".cols.f32", np.float32).reshape(H, W, 3), c)
    with open(prefix + ".ply") as f:
        assert f.read() == io.ply_text(v, c)


@pytest.mark.parametrize("optimizer", ["wta", "sgm"])
def test_reconstruction_stream_overlapped(ctx, orc, optimizer):
    # frames alternate between two contexts on two streams; every map read
    # back equals the oracle chain's for its frame
    from thundervision_b200 import reconstruction as rc
    left, right, Q = cameras()
    cost = "ssd" if optimizer == "wta" else "bt"
    m = rc.StereoMatcher(ctx, max_disp=D, cost=cost, optimizer=optimizer)
    rec = rc.Reconstruction(ctx, W, H, rc.Camera(*left), rc.Camera(*right), Q=Q, matcher=m)
    try:
        scenes = [scene(60 + t) for t in range(5)]
        frames = [(torch.from_numpy(a).pin_memory(), torch.from_numpy(b).pin_memory()) for a, b in scenes]
        out = [torch.empty((H, W), dtype=torch.float32).pin_memory() for _ in frames]
        assert rec.stream(frames, out) > 0
        for t, (a, b) in enumerate(scenes):
            ref = io.reconstruction(a, b, (left, right), D, q=Q.ravel(), cost=cost, optimizer=optimizer)[1]
            np.testing.assert_array_equal(out[t].numpy(), ref, err_msg=f"frame {t}")
    finally:
        rec.close()
