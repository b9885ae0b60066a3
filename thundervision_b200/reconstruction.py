"""The reference's reconstruction chain on the device, frame by frame.

LibThunderVision's ``Reconstruction`` (tdvision/reconstruction.cpp:9-55)
wires worker-thread stages through pipes:

  color frames -> RectificationCV (grey [0,1] + cvRemap of the grey frames
  and of the left color frame, rectificationcv.cpp:258-310)
  -> DevStereoMatcher (5x5 Gaussian pre-filter, matching cost, optimizer,
  devstereomatcher.cpp:13-48, as CommonStereoMatcherFactory builds it,
  commonstereomatcherfactory.cpp:16-80)
  -> Dilate (erode + dilate, dilate.cpp:11-22)
  -> ReprojectProcess (one vertex and one color per pixel through the
  rectification's CVReprojector, reprojectprocess.cpp:6-19).

Here the stages are device kernels of libtdvb200.so on one CUDA stream; the
pipes and threads become stream order.  After the first frame the whole chain
is captured as one CUDA graph per input buffer set, so a frame is one graph
launch.  The matcher's output is the reference's d/D float map, and that is
the value the dilation and the reprojection see.
"""
import math

import numpy as np
import torch

from . import api


class Camera:
    """One calibrated camera: intrinsics K (3x3), distortion (k1, k2, p1,
    p2[, k3[, k4, k5, k6]]), rectifying rotation R (3x3) and rectified camera
    P (3x3 or 3x4), as cvStereoRectify gives them (rectificationcv.cpp:
    131-160)."""

    def __init__(self, K, dist, R, P):
        self.K = np.asarray(K, np.float64).reshape(3, 3)
        self.dist = np.asarray(dist, np.float64).ravel()
        if self.dist.size > 8:
            raise ValueError("at most 8 distortion coefficients")
        self.R = np.asarray(R, np.float64).reshape(3, 3)
        self.P = np.asarray(P, np.float64).reshape(3, -1)


class StereoMatcher:
    """DevStereoMatcher as CommonStereoMatcherFactory configures it: cost
    "ssd" (the factory default, 7x7), "ncc" (3x3) or "bt"; optimizer "wta"
    (default), "dp" or "sgm" (SemiGlobalDev: P1 = 30/255, P2 = 150/255
    divided by the intensity step, the reference's path table and its device
    semantics); ``median_filter`` runs the 5x5 Gaussian on both inputs first
    (DevStereoMatcher's default).  ``max_disp`` defaults to the factory's 64.
    Returns the d/D float map (H, W)."""

    COSTS = ("ssd", "ncc", "bt")
    OPTIMIZERS = ("wta", "dp", "sgm")

    def __init__(self, ctx, max_disp=64, cost="ssd", optimizer="wta", median_filter=True):
        if cost not in self.COSTS:
            raise ValueError(f"cost must be one of {self.COSTS}")
        if optimizer not in self.OPTIMIZERS:
            raise ValueError(f"optimizer must be one of {self.OPTIMIZERS}")
        self.ctx, self.max_disp = ctx, int(max_disp)
        self.cost, self.optimizer, self.median_filter = cost, optimizer, bool(median_filter)

    def __call__(self, left, right):
        if self.median_filter:
            # the Gaussian runs inside the cost kernel; the filtered left
            # image is kept as the SGM's P2 guide
            C, left = self.ctx.cost_filtered(left, right, self.max_disp, kind=self.cost, prefilter="gauss5",
                                             left_filtered=self.optimizer == "sgm")
        else:
            C = self.ctx.cost(left, right, self.max_disp, kind=self.cost)
        if self.optimizer == "wta":
            return self.ctx.wta(C, norm=True)["disp_norm"]
        if self.optimizer == "dp":
            return self.ctx.dp(C, norm=True)["disp_norm"]
        return self.ctx.sgm(C, 30.0 / 255.0, 150.0 / 255.0, guide=left, p2_mode="adjust", table="ref",
                            semantics="ref_gpu", norm=True)["disp_norm"]


class Reconstruction:
    """Color stereo frames -> rectified grey pair -> disparity (d/D) ->
    dilation -> one vertex and one color per pixel.

    ``Q`` (4x4, cvStereoRectify's reprojection matrix) selects the
    CVReprojector the reference reprojects through (cvreprojector.cpp:45-60);
    without it, DirectReprojector (x, H - y, d * zscale).  ``dilate`` runs the
    7x7 opening the reference chains after the matcher
    (reconstruction.cpp:30-31).  Frames are (H, W, 3) uint8 tensors on this
    context's device, or host tensors (pinned for an asynchronous copy).

    ``update`` returns a dict with "rect_left" (rectified left color),
    "disp" (d/D after the dilation), "vertices" and "colors"; with
    ``graph=True`` these are the graph's own buffers, overwritten by the next
    frame.
    """

    def __init__(self, ctx, width, height, left_cam, right_cam, Q=None, zscale=1.0, matcher=None,
                 dilate=True, graph=True):
        self._args = (width, height, left_cam, right_cam, Q, zscale, dilate, graph)
        self._twin = None
        self.ctx, self.W, self.H = ctx, int(width), int(height)
        self.matcher = matcher if matcher is not None else StereoMatcher(ctx)
        self.dilate, self.graph = bool(dilate), bool(graph)
        self.dev = torch.device("cuda", ctx.device)
        self.maps = [ctx.rectify_maps(c.K, c.dist, c.R, c.P, self.W, self.H, device=self.dev)
                     for c in (left_cam, right_cam)]
        if Q is None:
            self.mode, self.q = "direct", None
        else:
            q = np.asarray(Q, np.float64).ravel()
            if q.size != 16 or not all(math.isfinite(v) for v in q):
                raise ValueError("Q must be 4x4 and finite")
            self.mode, self.q = "q", [float(v) for v in q]
        self.zscale = float(zscale)
        self._in = None
        self._g = None
        self._out = None
        self.last = None

    def _frame(self, left, right):
        ctx = self.ctx
        (mxl, myl), (mxr, myr) = self.maps
        gl = ctx.remap(ctx.to_gray(left), mxl, myl)
        gr = ctx.remap(ctx.to_gray(right), mxr, myr)
        cl = ctx.remap(left, mxl, myl)
        d = self.matcher(gl, gr)
        if self.dilate:
            d = ctx.postfilter(d, "open7")
        v, c = ctx.reproject(d, cl, self.mode, zscale=self.zscale, q=self.q)
        return {"rect_left": cl, "disp": d, "vertices": v, "colors": c}

    def _check(self, t):
        if tuple(t.shape) != (self.H, self.W, 3) or t.dtype != torch.uint8:
            raise ValueError(f"frames must be ({self.H}, {self.W}, 3) uint8")

    def update(self, left, right):
        self._check(left)
        self._check(right)
        if not self.graph:
            self.last = self._frame(left.to(self.dev, non_blocking=True), right.to(self.dev, non_blocking=True))
            return self.last
        if self._in is None:
            self._in = [torch.empty((self.H, self.W, 3), dtype=torch.uint8, device=self.dev) for _ in range(2)]
        self._in[0].copy_(left, non_blocking=True)
        self._in[1].copy_(right, non_blocking=True)
        if self._g is None:
            # the first frame runs uncaptured: it sizes the context's scratch
            # and path schedules, which the captured frames then reuse
            out = self._frame(*self._in)
            torch.cuda.current_stream(self.dev).synchronize()
            s = torch.cuda.Stream(self.dev)
            s.wait_stream(torch.cuda.current_stream(self.dev))
            g = torch.cuda.CUDAGraph()
            with torch.cuda.stream(s), torch.cuda.graph(g, stream=s):
                self._out = self._frame(*self._in)
            torch.cuda.current_stream(self.dev).wait_stream(s)
            self._g = g
            self.last = out
            return out
        self._g.replay()
        self.last = self._out
        return self._out

    def export_ply(self, path, out=None):
        """Writes the last frame's mesh as the reference's PLY
        (PLYMeshExporter::exportMesh, plymeshexporter.cpp:8-76)."""
        out = out if out is not None else self.last
        if out is None:
            raise RuntimeError("no frame reconstructed yet")
        api.write_ply(path, out["vertices"], out["colors"])

    def stream(self, frames, out_disp):
        """Runs a stream of frames and returns the device milliseconds from
        the first copy in to the last map read back.  ``frames``: list of
        (left, right) pinned host (H, W, 3) uint8 tensors; ``out_disp``: list
        of pinned host (H, W) float32 tensors receiving each frame's d/D map.
        Frames alternate between this object and a twin with its own context
        (its own scratch), input buffers, graph and CUDA stream, so
        consecutive frames overlap on the GPU, as the video loop runs them;
        each frame's map is the one ``update`` gives for it."""
        if self._twin is None:
            W, H, L, R, Q, z, dil, graph = self._args
            m = self.matcher
            ctx2 = api.Context(self.ctx.device)
            self._twin = Reconstruction(ctx2, W, H, L, R, Q=Q, zscale=z, dilate=dil, graph=graph,
                                        matcher=StereoMatcher(ctx2, m.max_disp, m.cost, m.optimizer,
                                                              m.median_filter))
            self._twin_ctx = ctx2
        lanes = [self, self._twin]
        streams = [torch.cuda.Stream(self.dev), torch.cuda.Stream(self.dev)]
        main = torch.cuda.current_stream(self.dev)
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(main)
        for st in streams:
            st.wait_stream(main)
        for t, (left, right) in enumerate(frames):
            k = t % 2
            with torch.cuda.stream(streams[k]):
                out = lanes[k].update(left, right)
                out_disp[t].copy_(out["disp"], non_blocking=True)
        for st in streams:
            main.wait_stream(st)
        t1.record(main)
        t1.synchronize()
        return t0.elapsed_time(t1)

    def close(self):
        self._g = None
        self._out = None
        self._in = None
        self.last = None
        if self._twin is not None:
            torch.cuda.synchronize()
            self._twin.close()
            self._twin_ctx.close()
            self._twin = None
