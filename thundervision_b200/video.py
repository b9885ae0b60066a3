"""Video-stream form of the fused path, and the P1/P2 refit through the
soft-SGM adjoint (no reference counterpart: the reference matches one frame
per pipeline update, tdvision/devstereomatcher.cpp:36-48).

* ``DeviceVideoStream`` -- the frames of ``synthetic.VideoStream`` (slanted
  background, moving rectangles, sensor noise) generated on the GPU: the same
  texture, rectangle tracks and forward warp, with torch's seeded generators
  for the per-frame noise, so 300 full-HD frames take seconds instead of
  minutes of host time.
* ``VideoLoop`` -- frames from pinned host memory through one CUDA graph
  replay per frame (a persistent batch launch, or the per-frame fused kernels
  of tdv_stereo_sgm with their two concurrent chains): the copy of frame t+1
  runs on a copy stream while frame t is aggregated (two input buffer sets),
  and each frame's disparity map is copied back to pinned host memory.
* ``refit_penalties`` -- fits P1, P2 by gradient steps on the soft-argmin L1
  loss against ground truth (tdv_soft_sgm_forward / _backward).
* ``accuracy`` -- bad-pixel rate and density of a disparity map against
  ground truth.
"""
import math

import torch

from . import api, soft, synthetic


class DeviceVideoStream:
    """``synthetic.VideoStream`` restated with torch on a CUDA device."""

    def __init__(self, W=1920, H=1080, D=256, seed=0, n_rects=12, device="cuda"):
        base = synthetic.VideoStream(W, H, D, seed=seed, n_rects=n_rects)
        self.W, self.H, self.D = W, H, D
        self.device = torch.device(device)
        self.tex = torch.from_numpy(base.left_tex).to(self.device, torch.float32)
        self.rects = [list(r) for r in base.rects]
        self.bg = torch.from_numpy(base.bg).to(self.device)
        self.ys = torch.arange(H, device=self.device).view(H, 1).expand(H, W)
        self.xs = torch.arange(W, device=self.device).view(1, W).expand(H, W)

    def frame(self, t):
        """(left u8, right u8, ground-truth disparity int64, occluded bool)."""
        W, H = self.W, self.H
        g = torch.Generator(device=self.device)
        g.manual_seed(synthetic.pair_seed(12345, t) & ((1 << 63) - 1))
        s = (t * 2) % 512
        left = self.tex[:, s:s + W]
        disp = self.bg.view(1, W).expand(H, W).clone()
        for (x0, y0, rw, rh, d, vx, vy) in self.rects:
            x = (x0 + vx * t) % max(1, W - rw)
            y = (y0 + vy * t) % max(1, H - rh)
            disp[y:y + rh, x:x + rw] = d
        # forward warp x_r = x - d, the larger disparity winning a target
        xr = self.xs - disp
        ok = xr >= 0
        key = torch.full((H * W,), -1, dtype=torch.int64, device=self.device)
        tgt = (self.ys * W + xr)[ok]
        val = (disp * 65536 + self.xs)[ok]
        key.scatter_reduce_(0, tgt, val, reduce="amax", include_self=True)
        key = key.view(H, W)
        hit = key >= 0
        src = torch.where(hit, key % 65536, torch.zeros_like(key))
        holes = torch.rand((H, W), generator=g, device=self.device) * 255.0
        right = torch.where(hit, left.gather(1, src), holes)
        zbuf = torch.where(hit, key // 65536, torch.full_like(key, -1))
        visible = ok & (zbuf.gather(1, xr.clamp(min=0)) == disp)
        right = right + torch.randn((H, W), generator=g, device=self.device) * 2.0
        left = left + torch.randn((H, W), generator=g, device=self.device) * 2.0
        to_u8 = lambda v: torch.clamp(torch.round(v), 0, 255).to(torch.uint8)
        return to_u8(left), to_u8(right), disp, ~visible


def accuracy(disp, gt, occl, thr=1):
    """Bad-pixel rate (|d - gt| > thr) over non-occluded pixels the map keeps,
    the density of kept non-occluded pixels, and the mean absolute error."""
    d = disp.to(torch.int64)
    kept = d != 0xFFFF
    nonocc = ~occl
    m = kept & nonocc
    err = (d - gt).abs()
    n = int(m.sum())
    return {"bad_rate": float(((err > thr) & m).sum()) / max(n, 1),
            "density": n / max(int(nonocc.sum()), 1),
            "mae": float(err[m].float().mean()) if n else float("nan")}


class VideoLoop:
    """Double-buffered frame loop, one CUDA graph replay per frame.

    ``engine="launches"`` (default): each frame is the per-frame fused
    kernels of tdv_stereo_sgm (two concurrent pass chains), captured into one
    CUDA graph per buffer set.  ``engine="persistent"``: each frame is one
    persistent batch launch (tdv_batch_graph_launch, tiles autotuned once).
    ``paths`` 4 or 8; P1/P2 must be multiples of 1/2 (the integer-domain
    fused path).  ``semantics`` / ``table`` (launches engine): "standard" /
    "full", or "ref_cpu" / "ref" for the reference's own CPU recurrence over
    its path table (tdvision/semiglobalcpu.cpp:173-230), which the fused
    kernels also run; the persistent engine takes the standard ones only.

    ``overlap=True`` (launches engine): each buffer set has its own private
    context (its own aggregation volumes) and its own compute stream, so
    frame t+1's passes can run while frame t finishes: the last horizontal
    pass, bound by its instruction stream, overlaps the next frame's
    DRAM-bound passes.  Maps are the same as with one context.
    """

    def __init__(self, ctx, W, H, D, p1, p2, paths=8, lr=1, graph=True, autotune=True, device="cuda",
                 engine="launches", overlap=True, semantics="standard", table="full"):
        self.ctx, self.graph, self.engine = ctx, graph, engine
        if engine == "persistent" and (semantics, table) != ("standard", "full"):
            raise ValueError("the persistent engine runs the standard recurrence over the full table")
        self.bufs = [(torch.empty((H, W), dtype=torch.uint8, device=device),
                      torch.empty((H, W), dtype=torch.uint8, device=device)) for _ in range(2)]
        self.copy_stream = torch.cuda.Stream(device=device)
        self.overlap = bool(overlap) and engine == "launches"
        self.compute_streams = [torch.cuda.Stream(device=device) for _ in range(2)] if self.overlap else None
        self.tiles = None
        if engine == "persistent":
            self.batches = [api.Batch(ctx, [(l, r, D, lr)], p1, p2, paths=paths) for (l, r) in self.bufs]
            if autotune:
                tiles, _ = self.batches[0].autotune(reps=5)
                self.batches[1].set_tiles(**tiles)
                self.tiles = tiles
            else:
                self.tiles = self.batches[0].tiles
            self.outputs = [b.outputs[0]["disp"] for b in self.batches]
        elif engine == "launches":
            # the graphs hold the context's scratch pointers: a private
            # context keeps other callers from growing (reallocating) them
            self.batches = []
            idx = torch.device(device).index
            dev_index = torch.cuda.current_device() if idx is None else idx
            self._ctxs = [api.Context(dev_index) for _ in range(2 if self.overlap else 1)]
            for c in self._ctxs:
                c.reserve(W, H, D)
            self.ctx = self._own_ctx = self._ctxs[0]
            self.outputs = [torch.empty((H, W), dtype=torch.uint16, device=device) for _ in range(2)]
            prm = api.L.tdv_sgm_params(float(p1), float(p2), api.L.P2_CONST, paths, api._TABLES[table],
                                       api._SEMS[semantics])
            calls = []
            for (l, r), o in zip(self.bufs, self.outputs):
                calls.append((api._image(l), api._image(r), api.L.tdv_disparity(o.data_ptr(), None, None,
                                                                                 -1 if lr is None else lr)))
            self._prm, self._calls, self._D = prm, calls, D
            self._graphs = [None, None]
            if graph:
                cs = torch.cuda.Stream(device=device)
                for b in range(2):
                    with torch.cuda.stream(cs):
                        self._call(b)  # first use: kernel attributes, scratch (outside the capture)
                    torch.cuda.synchronize()
                    g = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(g, stream=cs):
                        self._call(b)
                    self._graphs[b] = g
        else:
            raise ValueError("engine must be 'persistent' or 'launches'")
        # first launches (graph captures) now, outside any timed loop
        for b in range(2):
            self._launch(b)
        torch.cuda.synchronize()

    def _call(self, b):
        import ctypes
        li, ri, o = self._calls[b]
        ctx = self._ctxs[b % len(self._ctxs)]
        ctx.check(api.L.lib().tdv_stereo_sgm(ctx.handle, ctypes.byref(li), ctypes.byref(ri), self._D,
                                             ctypes.byref(self._prm), ctypes.byref(o), api._stream()))

    def close(self):
        for b in self.batches:
            b.close()
        if self.engine == "launches":
            torch.cuda.synchronize()
            self._graphs = [None, None]
            for c in self._ctxs:
                c.close()

    def _launch(self, b):
        if self.engine == "persistent":
            (self.batches[b].graph_launch if self.graph else self.batches[b].run)()
        elif self._graphs[b] is not None:
            self._graphs[b].replay()
        else:
            self._call(b)

    def run(self, host_frames, host_out):
        """host_frames: list of pinned (left, right) uint8 tensors; host_out:
        list of pinned uint16 tensors receiving each frame's disparity.
        Returns the device milliseconds from the first copy to the last
        disparity read-back."""
        ks = torch.cuda.current_stream()
        cs = self.copy_stream
        copied = [torch.cuda.Event() for _ in range(2)]
        done = [torch.cuda.Event() for _ in range(2)]
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(ks)
        cs.wait_stream(ks)

        def upload(t):
            b = t % 2
            with torch.cuda.stream(cs):
                if t >= 2:
                    cs.wait_event(done[b])
                hl, hr = host_frames[t]
                self.bufs[b][0].copy_(hl, non_blocking=True)
                self.bufs[b][1].copy_(hr, non_blocking=True)
                copied[b].record(cs)

        n = len(host_frames)
        streams = self.compute_streams if self.overlap else [ks, ks]
        if self.overlap:
            for st in streams:
                st.wait_stream(ks)
        upload(0)
        for t in range(n):
            b = t % 2
            if t + 1 < n:
                upload(t + 1)
            st = streams[b]
            st.wait_event(copied[b])
            with torch.cuda.stream(st):
                self._launch(b)
                host_out[t].copy_(self.outputs[b], non_blocking=True)
            done[b].record(st)
        if self.overlap:
            for st in streams:
                ks.wait_stream(st)
        t1.record(ks)
        t1.synchronize()
        for b in self.batches:
            b.status()
        if self.engine == "launches":
            for c in self._ctxs:
                c.device_status()
        return t0.elapsed_time(t1)

    def disparity(self, left, right):
        """One frame from device tensors (untimed helper for accuracy runs)."""
        self.bufs[0][0].copy_(left)
        self.bufs[0][1].copy_(right)
        self._launch(0)
        return self.outputs[0]


def refit_penalties(ctx, frames, max_disp, p1, p2, steps=50, lr=0.05, tau=1.0, paths=8, checkpoint=32):
    """Fit P1, P2 by `steps` Adam steps (in log space, so both stay positive)
    on the L1 loss between the soft-argmin disparity of the FP32 BT cost
    volume and ground truth over non-occluded pixels, one frame per step
    (cycling through `frames`, a list of (left, right, gt, occl) device
    tensors).  Returns (p1, p2, history)."""
    dev = frames[0][0].device
    theta = torch.tensor([math.log(p1), math.log(p2)], dtype=torch.float64, device=dev, requires_grad=True)
    opt = torch.optim.Adam([theta], lr=lr)
    hist = []
    for it in range(steps):
        left, right, gt, occl = frames[it % len(frames)]
        cost = ctx.cost(left, right, max_disp)
        pen = theta.exp().to(torch.float32)
        dh = soft.soft_sgm(cost, pen[0], pen[1], tau=tau, paths=paths, checkpoint=checkpoint, ctx=ctx)
        loss = (dh - gt.to(torch.float32)).abs()[~occl].mean()
        opt.zero_grad()
        loss.backward()
        opt.step()
        hist.append({"step": it, "loss": loss.item(), "p1": pen[0].item(), "p2": pen[1].item()})
        del cost, dh, loss
    p = theta.detach().exp().tolist()
    return p[0], p[1], hist
