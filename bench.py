#!/usr/bin/env python
"""Throughput of the dense-stereo hot path on the full-HD configuration:
1920x1080 rectified u8 pair, D = 256, Birchfield-Tomasi cost, 8-path SGM
(P1 = 10, P2 = 120), WTA + left-right check (threshold 1).

One step = one stereo frame through tdv_stereo_sgm.  Prints one JSON line.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm (default): `value` is frames/s with the pair already in HBM, timed
per step with CUDA events on the launch stream, L2 flushed (256 MiB write)
between steps; `e2e` is the same frames run as a stream through the public
video API (video.VideoLoop): every frame copied from pinned host memory and
its disparity map copied back inside the timed region, with two buffer sets,
each with its own context and compute stream, so that the copies of one frame
and the kernels of the next overlap the kernels of the previous one;
`e2e_sequential` runs copy-in, tdv_stereo_sgm and copy-out of each step in
sequence on one stream.  Under torchrun every rank processes its own frames (weak scaling, no
collective on the data path); the time is the max over ranks.

Reference arm (--impl reference): the reference's CPU path restated in C++
(the oracle: BT cost + SemiGlobalCPU with its table and start-assign
recurrence + WTACPU) on all host threads, each step a band of rows of the
same frame sized so the run stays within a few minutes; rank 0 only.
"""
import argparse
import datetime
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W, H, D = 1920, 1080, 256
P1, P2, PATHS, LR = 10.0, 120.0, 8, 1
METRIC = "1080p D=256 8-path SGM fps"
UNIT = "frames/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--frames", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batch and soft-SGM measurements")
    ap.add_argument("--profile-case", choices=["general", "cost1080"],
                    help="general: one launch of each general-path kernel on 1280x720, D=64; cost1080: "
                         "one BT cost DSI at 1920x1080, D=256 (HWD); then exit (the cases the ncu "
                         "summaries are captured on)")
    return ap.parse_args()


def config(extra=None):
    c = {"workload": f"BT + SGM-{PATHS} + WTA + LR, {W}x{H}, D={D}", "width": W, "height": H,
         "max_disp": D, "paths": PATHS, "p1": P1, "p2": P2, "lr_threshold": LR,
         "l2": "flushed between timed steps (256 MiB write)",
         "inputs": "seeded synthetic video frames (moving rectangles over a slanted plane)"}
    if extra:
        c.update(extra)
    return c


# ------------------------------------------------------------------ clocks
class Clocks:
    """SM clocks and clock-event (throttle) reasons of the benchmark's own GPU
    (found by UUID), sampled on a thread through NVML every 20 ms while a
    timed region runs; falls back to `nvidia-smi -lms 200` without NVML."""

    REASON_BITS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
                   0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, gpu_index, period=0.02):
        import threading
        self.rows, self.p, self.nv = [], None, None
        self.stop_ev = threading.Event()
        uuid = None
        try:
            import torch
            uuid = "GPU-" + str(torch.cuda.get_device_properties(gpu_index).uuid)
        except Exception:
            pass
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByUUID(uuid) if uuid else pynvml.nvmlDeviceGetHandleByIndex(gpu_index)
            self.nv, self.h = pynvml, h
            self.max_sm = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                pynvml.nvmlDeviceGetCurrentClocksThrottleReasons

            def run():
                while not self.stop_ev.is_set():
                    try:
                        self.rows.append((pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM), reasons(h)))
                    except Exception:
                        pass
                    self.stop_ev.wait(period)

            self.t = threading.Thread(target=run, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nv = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", uuid or str(gpu_index),
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.nv is not None:
            self.stop_ev.set()
            self.t.join(timeout=5)
            rows = self.rows
            mx = self.max_sm
        elif self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
            self.f.flush()
            rows, mx = [], None
            with open(self.f.name) as fh:
                for ln in fh:
                    parts = [x.strip() for x in ln.split(",")]
                    if len(parts) >= 3 and parts[0].replace(".", "").isdigit():
                        rows.append((float(parts[0]), int(parts[2], 16) if parts[2].startswith("0x") else 0))
                        mx = float(parts[1]) if parts[1].replace(".", "").isdigit() else mx
            os.unlink(self.f.name)
        else:
            return None
        if not rows:
            return None
        sm = sorted(float(r[0]) for r in rows)
        reasons = sorted({name for r in rows for bit, name in self.REASON_BITS.items() if int(r[1]) & bit})
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------- CPU arms
def cpu_reference_run(steps, warmup, budget_s=150.0):
    """Times the oracle's restatement of the reference CPU path on bands of a
    full-HD frame; returns (frames/s, description, threads)."""
    import numpy as np

    import oracle
    from thundervision_b200 import synthetic
    threads = os.cpu_count() or 1
    L, R, _, _ = synthetic.VideoStream(seed=0).frame(0)
    Lf, Rf = oracle.u8_to_f32(L), oracle.u8_to_f32(R)

    def band(h):
        t0 = time.perf_counter()
        C = oracle.bt_cost(Lf[:h], Rf[:h], D, layout=oracle.LAYOUT_REF_WHD)
        oracle.sgm(C, Lf[:h], P1, P2, paths=PATHS, table=oracle.TABLE_REF,
                   semantics=oracle.SEM_REF_CPU, layout=oracle.LAYOUT_REF_WHD, threads=threads,
                   want_S=False)
        return time.perf_counter() - t0

    t_probe = band(32)
    per_row = t_probe / 32
    total_steps = max(1, steps + warmup)
    h = int(max(16, min(H, (budget_s / total_steps) / per_row)))
    for _ in range(warmup):
        band(h)
    ts = [band(h) for _ in range(steps)]
    t = sum(ts) / len(ts)
    fps = (h / H) / t
    desc = (f"rows 0..{h - 1} of a {W}x{H} frame ({h / H:.3f} frame) per step, D={D}, {PATHS} paths,"
            f" reference CPU semantics (start-assign, stale-end table), {threads} threads;"
            f" frames/s scaled by rows")
    return fps, desc, threads


def cpu_baseline_sample(budget_s=20.0):
    fps, desc, threads = cpu_reference_run(1, 0, budget_s=budget_s)
    return {"value": fps, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    fps, desc, threads = cpu_reference_run(args.steps, args.warmup)
    line = {"metric": METRIC, "value": fps, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 / fps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference", "config": config(),
            "cpu_baseline": {"value": fps, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": desc},
            "e2e": {"value": fps, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------- extra metrics
def _event_ms(fn, reps, warm, st):
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        fn()
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def measure_batch(ctx, dev, reps=3):
    """Uneven batch: 64 seeded pairs, W ~ U[320,1920], H ~ U[240,1080] (multiples
    of 16), D in {32,64,128,256}; BT + SGM-8 + WTA.  One graph-captured
    persistent launch with autotuned tiles vs (a) 64 per-pair launches of the
    plain method -- BT cost DSI (tdv_cost, FP32) then SGM + WTA (tdv_sgm) --
    and (b) 64 per-pair launches of the fused path (tdv_stereo_sgm); outputs
    and the DSI preallocated, all on one stream, device time."""
    import ctypes

    import torch

    from thundervision_b200 import _lib, api, synthetic
    shapes = synthetic.batch_shapes(seed=0, n=64)
    pairs = []
    for i, (w, h, d) in enumerate(shapes):
        l, r, _, _ = synthetic.pair_sized(w, h, d, synthetic.pair_seed(0, i) % (2 ** 31))
        pairs.append((torch.from_numpy(l).to(dev), torch.from_numpy(r).to(dev), d))
    cells = sum(w * h * d * 8 for (w, h, d) in shapes)
    st = torch.cuda.current_stream()
    lib = _lib.lib()
    prm = _lib.tdv_sgm_params(P1, P2, _lib.P2_CONST, 8, _lib.TABLE_FULL, _lib.SEM_STANDARD)
    outs = [torch.empty(l.shape, dtype=torch.uint16, device=dev) for (l, r, d) in pairs]
    calls = [(api._image(l), api._image(r), d, _lib.tdv_disparity(o.data_ptr(), None, None, -1))
             for (l, r, d), o in zip(pairs, outs)]
    ctx.reserve(max(s[0] for s in shapes), max(s[1] for s in shapes), 256)

    def per_pair():
        sp = api._stream()
        for li, ri, d, o in calls:
            ctx.check(lib.tdv_stereo_sgm(ctx.handle, ctypes.byref(li), ctypes.byref(ri), d,
                                         ctypes.byref(prm), ctypes.byref(o), sp))

    t_pair = _event_ms(per_pair, reps, 1, st)
    fused_ref = [o.clone() for o in outs]

    maxc = max(w * h * d for (w, h, d) in shapes)
    dsi = torch.empty(maxc, dtype=torch.float32, device=dev)
    cprm = _lib.tdv_cost_params(_lib.COST_BT, 0)
    plain_calls = []
    for (l, r, d), o in zip(pairs, outs):
        h, w = l.shape
        plain_calls.append((api._image(l), api._image(r), _lib.tdv_volume(dsi.data_ptr(), w, h, d, _lib.LAYOUT_HWD,
                                                                           _lib.F32),
                            _lib.tdv_disparity(o.data_ptr(), None, None, -1)))

    def per_pair_plain():
        sp = api._stream()
        for li, ri, v, o in plain_calls:
            ctx.check(lib.tdv_cost(ctx.handle, ctypes.byref(li), ctypes.byref(ri), ctypes.byref(cprm),
                                   ctypes.byref(v), sp))
            ctx.check(lib.tdv_sgm(ctx.handle, ctypes.byref(v), None, ctypes.byref(prm), None, ctypes.byref(o),
                                  sp))

    t_plain = _event_ms(per_pair_plain, 1, 1, st)
    plain_equal = all(torch.equal(o, ref) for o, ref in zip(outs, fused_ref))
    del dsi
    b = api.Batch(ctx, pairs, P1, P2, paths=8)
    t_default = _event_ms(b.run, reps, 1, st)
    tiles, t_tune = b.autotune(reps=2)
    t_run = _event_ms(b.run, reps, 1, st)
    t_graph = _event_ms(b.graph_launch, reps, 1, st)
    b.status()
    equal = all(torch.equal(o["disp"], ref) for o, ref in zip(b.outputs, fused_ref))
    n_items = b.work_queue()[1]
    b.close()
    return {"workload": "64 pairs, W~U[320,1920], H~U[240,1080] (x16), D in {32,64,128,256}, "
                        "BT + SGM-8 + WTA, seed 0",
            "pairs": len(shapes), "cells": cells, "work_items": n_items,
            "per_pair_plain_ms": t_plain, "per_pair_fused_ms": t_pair, "batch_default_tiles_ms": t_default,
            "batch_tuned_ms": t_run, "batch_graph_ms": t_graph, "tiles": tiles,
            "pairs_per_s": len(shapes) / (t_graph / 1000.0),
            "gcells_per_s": cells / (t_graph / 1000.0) / 1e9,
            "per_pair_fused_gcells_per_s": cells / (t_pair / 1000.0) / 1e9,
            "speedup_vs_per_pair_plain": t_plain / t_graph, "speedup_vs_per_pair_fused": t_pair / t_graph,
            "bit_identical_to_per_pair": equal and plain_equal}


def measure_soft(ctx, dev, reps=5):
    """Soft-argmin SGM at 960x540, D=128, FP32 BT volume, 8 paths, tau=1,
    checkpoint every 32 steps: forward (recording the tape) + adjoint vs the
    plain forward (no tape) and vs the hard SGM + WTA on the same volume."""
    import torch

    from thundervision_b200 import soft, synthetic
    l, r, gt, _ = synthetic.make_pair(960, 540, 128, 17, n_rects=8, slanted=True, salt_pepper=0.02)
    cost = ctx.cost(torch.from_numpy(l).to(dev), torch.from_numpy(r).to(dev), 128)
    gt_t = torch.from_numpy(gt.astype("float32")).to(dev)
    st = torch.cuda.current_stream()
    p = torch.tensor([P1, P2], dtype=torch.float32, device=dev, requires_grad=True)
    c = cost.clone().requires_grad_(True)

    def fwd_bwd():
        dh = soft.soft_sgm(c, p[0], p[1], tau=1.0, paths=8, checkpoint=32, ctx=ctx)
        (dh - gt_t).abs().mean().backward()

    def fwd_plain():
        soft.soft_sgm_infer(cost, P1, P2, tau=1.0, paths=8, ctx=ctx)

    def hard():
        ctx.sgm(cost, P1, P2)

    t_fb = _event_ms(fwd_bwd, reps, 2, st)
    t_f = _event_ms(fwd_plain, reps, 2, st)
    t_h = _event_ms(hard, reps, 2, st)
    return {"workload": "960x540, D=128, FP32 BT cost, 8 paths, tau=1, L1 loss, checkpoint 32",
            "fwd_adjoint_ms": t_fb, "plain_soft_forward_ms": t_f, "hard_sgm_wta_ms": t_h,
            "ratio_vs_plain_forward": t_fb / t_f, "ratio_vs_hard_sgm": t_fb / t_h}


def measure_plain(ctx, dev, reps=3):
    """The drop-in stage chain a reference user calls (the plain method):
    BT cost DSI in the reference's layout from [0,1] float images (tdv_cost),
    then SGM + WTA with the reference's path table, GPU semantics and P2
    divided by the intensity step (tdv_sgm, P1 = 30/255, P2 = 150/255), at
    640x480, D=64 and 1920x1080, D=256; device time per pair."""
    import torch

    from thundervision_b200 import synthetic
    st = torch.cuda.current_stream()
    out = {}
    for (w, h, d) in ((640, 480, 64), (1920, 1080, 256)):
        l, r, _, _ = synthetic.pair_sized(w, h, d, 3)
        lf = torch.from_numpy(l).to(dev).float() * (1.0 / 255.0)
        rf = torch.from_numpy(r).to(dev).float() * (1.0 / 255.0)
        dsi = torch.empty((w, h, d), dtype=torch.float32, device=dev)

        def run():
            ctx.cost(lf, rf, d, layout="ref", out=dsi)
            ctx.sgm(dsi, 30.0 / 255.0, 150.0 / 255.0, guide=lf, p2_mode="adjust", table="ref",
                    semantics="ref_gpu", layout="ref")

        ms = _event_ms(run, reps, 1, st)
        out[f"{w}x{h}_D{d}"] = {"ms": ms, "fps": 1000.0 / ms, "gcells_per_s": w * h * d * 8 / (ms / 1000.0) / 1e9}
        del dsi
    out["workload"] = ("tdv_cost (BT, REF_WHD, [0,1] floats) + tdv_sgm (REF table, REF_GPU semantics, "
                       "P2 adjusted, 8 paths) + WTA")
    # every stage of the 640x480, D=64 configuration timed alone: the three
    # costs at the configuration's windows (SSD 5x5, NCC 9x9) and the
    # reference's (SSD 7x7, NCC 3x3), 8-path SGM with WTA + left-right check,
    # DP, WTA + left-right check, and the 8-path fused SGM on u8 intensities
    l, r, _, _ = synthetic.pair_sized(640, 480, 64, 1)
    lf = torch.from_numpy(l).to(dev).float() * (1.0 / 255.0)
    rf = torch.from_numpy(r).to(dev).float() * (1.0 / 255.0)
    l8, r8 = torch.from_numpy(l).to(dev), torch.from_numpy(r).to(dev)
    dsi = torch.empty((480, 640, 64), dtype=torch.float32, device=dev)
    c1 = {"workload": "640x480, D=64, [0,1] float images, HWD DSI; device ms per call (mean of 10 after 2)"}
    for name, kind, rad in (("cost_bt", "bt", 0), ("cost_ssd5x5", "ssd", 2), ("cost_ssd7x7", "ssd", 3),
                            ("cost_ncc9x9", "ncc", 4), ("cost_ncc3x3", "ncc", 1)):
        c1[name] = _event_ms(lambda: ctx.cost(lf, rf, 64, kind=kind, radius=rad, out=dsi), 10, 2, st)
    ctx.cost(lf, rf, 64, out=dsi)
    c1["sgm8_ref_gpu_wta_lr"] = _event_ms(
        lambda: ctx.sgm(dsi, 30.0 / 255.0, 150.0 / 255.0, guide=lf, p2_mode="adjust", table="ref",
                        semantics="ref_gpu", lr=1), 10, 2, st)
    c1["sgm8_standard_wta_lr"] = _event_ms(lambda: ctx.sgm(dsi, 10.0 / 255.0, 120.0 / 255.0, lr=1), 10, 2, st)
    c1["dp"] = _event_ms(lambda: ctx.dp(dsi), 10, 2, st)
    c1["wta_lr"] = _event_ms(lambda: ctx.wta(dsi, lr=1), 10, 2, st)
    c1["fused_bt_sgm8_wta_lr_u8"] = _event_ms(lambda: ctx.stereo_sgm(l8, r8, 64, 10, 120, paths=8, lr=1), 10, 2, st)
    out["640x480_D64_stages"] = c1
    del dsi
    return out


def measure_image(ctx, dev, reps=10):
    """The image stages either side of the path at 1920x1080: rectification
    maps, grey conversion, remap (grey F32 and color U8x3), the two pre-filters, the
    opening and the 3x3 median of a disparity map, sub-pixel refinement from
    a D=256 F32 volume and Q reprojection with colors.  Each call timed alone
    with CUDA events (median of `reps`, L2 flushed before each), against the
    bytes it must read and write."""
    import torch

    g = torch.Generator(device=dev)
    g.manual_seed(5)
    color = torch.randint(0, 256, (H, W, 3), dtype=torch.uint8, device=dev, generator=g)
    gray = torch.rand((H, W), device=dev, generator=g)
    yy, xx = torch.meshgrid(torch.arange(H, device=dev, dtype=torch.float32),
                            torch.arange(W, device=dev, dtype=torch.float32), indexing="ij")
    # a mild rectifying warp: small rotation and scale about the centre
    mapx = (0.999 * (xx - W / 2) - 0.01 * (yy - H / 2) + W / 2 + 0.37).contiguous()
    mapy = (0.01 * (xx - W / 2) + 0.999 * (yy - H / 2) + H / 2 - 0.21).contiguous()
    dispf = torch.rand((H, W), device=dev, generator=g)
    disp16 = torch.randint(0, D, (H, W), device=dev, generator=g).to(torch.uint16)
    S = torch.rand((H, W, D), device=dev, generator=g)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    Q = [1, 0, 0, -W / 2, 0, 1, 0, -H / 2, 0, 0, 0, 1400.0, 0, 0, -1 / 0.12, 0]
    K = [[1400.0, 0, W / 2 + 0.3], [0, 1398.0, H / 2 - 0.7], [0, 0, 1]]
    dist = [-0.28, 0.09, 0.0012, -0.0007, -0.011]
    Rr = [[0.9998, -0.0175, 0.0087], [0.0175, 0.9998, 0.0], [-0.0087, 0.0002, 0.99996]]
    px = W * H
    cases = [
        ("rectify_maps", lambda: ctx.rectify_maps(K, dist, Rr, K, W, H), 8 * px),
        ("to_gray", lambda: ctx.to_gray(color), 3 * px + 4 * px),
        ("remap_gray_f32", lambda: ctx.remap(gray, mapx, mapy), 4 * px + 8 * px + 4 * px),
        ("remap_color_u8x3", lambda: ctx.remap(color, mapx, mapy), 3 * px + 8 * px + 3 * px),
        ("prefilter_gauss5", lambda: ctx.prefilter(gray, "gauss5"), 8 * px),
        ("prefilter_median7", lambda: ctx.prefilter(gray, "median7"), 8 * px),
        ("postfilter_open7_f32", lambda: ctx.postfilter(dispf, "open7"), 16 * px),
        ("postfilter_median3_u16", lambda: ctx.postfilter(disp16, "median3"), 4 * px),
        ("subpixel_d256", lambda: ctx.subpixel(S, disp16), (2 + 12 + 4) * px),
        ("reproject_q_color", lambda: ctx.reproject(dispf, color, "q", q=Q), 4 * px + 3 * px + 24 * px),
    ]
    st = torch.cuda.current_stream()
    res = {"workload": f"{W}x{H} frame; sub-pixel from a D={D} F32 volume; bytes = what each stage must read "
                       "and write (maps 8 B/px, F32 4 B/px, U8x3 3 B/px)"}
    for name, fn, nbytes in cases:
        fn()
        ts = []
        for _ in range(reps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            fn()
            e1.record(st)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        ms = sorted(ts)[len(ts) // 2]
        res[name] = {"ms": ms, "gb_per_s": nbytes / (ms / 1000.0) / 1e9}
    del S
    return res


def measure_reconstruction(ctx, dev, frames=20, warmup=3):
    """The reference's reconstruction chain (color frames -> grey -> remap ->
    Gaussian -> cost -> optimizer -> opening -> Q reprojection with colors) at
    1920x1080 through reconstruction.Reconstruction, one CUDA graph per frame;
    each frame's two color frames are copied from pinned host memory inside
    the timed region.  Two matchers: the factory default (SSD + WTA, D=64)
    and BT + SGM (the reference's SemiGlobalDev) at D=256."""
    import numpy as np
    import torch

    from thundervision_b200 import reconstruction as rc
    from thundervision_b200 import synthetic

    K = np.array([[1400.0, 0, W / 2 + 0.3], [0, 1398.0, H / 2 - 0.7], [0, 0, 1]])
    P = np.array([[1380.0, 0, W / 2, 0], [0, 1380.0, H / 2, 0], [0, 0, 1, 0]])
    cams = [rc.Camera(K, [-0.28, 0.09, 0.0012, -0.0007, -0.011], np.eye(3), P),
            rc.Camera(K, [-0.27, 0.085, -0.001, 0.0006, -0.01], np.eye(3), P)]
    Q = [1, 0, 0, -W / 2, 0, 1, 0, -H / 2, 0, 0, 0, 1380.0, 0, 0, -1 / 0.12, 0]
    Lh, Rh, _, _ = synthetic.make_pair(W, H, D, 17, n_rects=12)
    col = lambda g: torch.from_numpy(np.stack([g, g // 2 + 64, 255 - g], -1).astype(np.uint8)).pin_memory()
    lc, rcol = col(Lh), col(Rh)
    st = torch.cuda.current_stream()
    res = {"workload": f"{W}x{H} color pair per frame, pinned host -> device inside the timed region; "
                       f"median of {frames} frames after {warmup}"}
    for name, cost, opt, d in (("ssd_wta_d64", "ssd", "wta", 64), ("bt_sgm_d256", "bt", "sgm", D)):
        rec = rc.Reconstruction(ctx, W, H, cams[0], cams[1], Q=Q,
                                matcher=rc.StereoMatcher(ctx, max_disp=d, cost=cost, optimizer=opt))
        try:
            ts = []
            for i in range(warmup + frames):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
                rec.update(lc, rcol)
                e1.record(st)
                e1.synchronize()
                if i >= warmup:
                    ts.append(e0.elapsed_time(e1))
            ms = sorted(ts)[len(ts) // 2]
            res[name] = {"ms_per_frame": ms, "fps": 1000.0 / ms}
            # the same frames as a stream, consecutive frames overlapped on two
            # contexts, each map read back to pinned host memory
            outs = [torch.empty((H, W), dtype=torch.float32).pin_memory() for _ in range(frames)]
            pairs = [(lc, rcol)] * frames
            rec.stream(pairs[:4], outs[:4])
            sms = rec.stream(pairs, outs) / frames
            res[name + "_stream"] = {"ms_per_frame": sms, "fps": 1000.0 / sms}
        finally:
            rec.close()
    return res


def measure_video(ctx, dev, n_frames=300, refit_steps=50):
    """Full-HD video: 300 frames (12 moving rectangles over a slanted plane,
    sensor noise sigma 2), D=256, fused BT + SGM + WTA + L-R check, through a
    double-buffered loop of per-frame graph replays (the fused kernels, and
    beside them the persistent batch kernel) with every frame copied from
    pinned host memory and its map copied back (timed), 4-path vs 8-path; then P1/P2 fitted by 50 Adam steps on the soft-argmin L1
    loss (FP32 BT volume, adjoint kernels) and the refit vs default accuracy
    of the 8-path maps over all frames."""
    import torch

    from thundervision_b200 import video
    vs = video.DeviceVideoStream(W, H, D, seed=7, device=dev)
    frames = []
    for t in range(n_frames):
        l, r, gt, occ = vs.frame(t)
        frames.append((l, r, gt.to(torch.int16), occ))
    host = [(l.cpu().pin_memory(), r.cpu().pin_memory()) for (l, r, _, _) in frames]
    out_host = [torch.empty((H, W), dtype=torch.uint16).pin_memory() for _ in range(n_frames)]

    def mean_acc(maps):
        accs = [video.accuracy(m, f[2], f[3]) for m, f in zip(maps, frames)]
        return {k: sum(a[k] for a in accs) / len(accs) for k in accs[0]}

    res = {"workload": f"{n_frames} frames {W}x{H}, D={D}, moving rectangles, noise sigma 2, "
                       "pinned host in/out, double-buffered, graph replay"}
    for paths in (4, 8):
        for engine, key in (("launches", f"paths{paths}"), ("persistent", f"paths{paths}_persistent")):
            loop = video.VideoLoop(ctx, W, H, D, P1, P2, paths=paths, lr=LR, engine=engine)
            ms = loop.run(host, out_host)
            maps = [o.to(dev) for o in out_host]
            res[key] = {"engine": engine, "fps": n_frames / (ms / 1000.0), "ms_per_frame": ms / n_frames,
                        **({"tiles": loop.tiles} if loop.tiles else {}), **mean_acc(maps)}
            loop.close()
    # P1/P2 refit through the adjoint, then the 8-path maps with both settings
    fit_frames = [(l, r, gt.to(torch.int64), occ) for (l, r, gt, occ) in frames[:refit_steps]]
    p1r, p2r, hist = video.refit_penalties(ctx, fit_frames, D, P1, P2, steps=refit_steps)
    # the fused path takes penalties in halves
    p1h = max(0.5, round(p1r * 2) / 2)
    p2h = min(1280.0, max(p1h, round(p2r * 2) / 2))
    acc = {}
    for name, (a, b) in (("default", (P1, P2)), ("refit", (p1h, p2h))):
        maps = [ctx.stereo_sgm(f[0], f[1], D, a, b, paths=8, lr=LR)["disp"] for f in frames]
        acc[name] = {"p1": a, "p2": b, **mean_acc(maps)}
    res["refit"] = {"steps": refit_steps, "tau": 1.0, "p1": p1r, "p2": p2r,
                    "loss_first": hist[0]["loss"], "loss_last": hist[-1]["loss"],
                    "accuracy_8path": acc}
    return res


# ------------------------------------------------------------------ ours
# the compiled kernel behind each timed pass (PPL = 4 at D = 256), as ncu names it
KERNEL_OF = {
    "fused_prep": "prep_kernel",
    "fused_pass_V+": "vd_pass<4, 0, 0>",
    "fused_pass_D1-": "vd_pass<4, 0, 1>",
    "fused_pass_V-": "vd_pass<4, 1, 0>",
    "fused_pass_D1+": "vd_pass<4, 1, 1>",
    "fused_pass_D2+": "vd_pass<4, 1, 1>",
    "fused_pass_D2-": "vd_pass<4, 1, 1>",
    "fused_pass_H+": "hp_pass<4, 1, 1>",
    "fused_pass_H-_wta": "hp_pass<4, 2, 0>",
}


def alg_bytes(name):
    """Algorithmic HBM bytes of one launch of a fused kernel at this size:
    the u16 aggregation volumes (256 disparities = 512 B per pixel) read
    and/or written once, plus the 16-byte BT planes of both images once.  At
    8 paths the passes run as two concurrent chains on two volumes (V+ V- D1+
    and D1- D2+ D2-): V+ and D1- only store their volume, the other chain
    passes read and write it, H+ reads both and writes the first, H- reads it
    and writes the maps."""
    pix = W * H
    s_vol = pix * 256 * 2
    planes = 2 * pix * 16
    if name == "fused_prep":
        return 2 * pix + planes
    if name in ("fused_pass_V+", "fused_pass_D1-"):
        return s_vol + planes
    if name == "fused_pass_H+":
        return 3 * s_vol + planes
    if name.endswith("_wta"):
        return s_vol + planes + 3 * pix * 2
    return 2 * s_vol + planes


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    from thundervision_b200 import api, synthetic

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    ctx = api.Context(local)
    ctx.reserve(W, H, D)

    vs = synthetic.VideoStream(seed=1000 + rank)
    host_frames = [vs.frame(t)[:2] for t in range(args.frames)]
    dev_frames = [(torch.from_numpy(l).to(dev), torch.from_numpy(r).to(dev)) for l, r in host_frames]
    pinned = [(torch.from_numpy(l).pin_memory(), torch.from_numpy(r).pin_memory())
              for l, r in host_frames]
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    st = torch.cuda.current_stream()

    def step(i):
        l, r = dev_frames[i % len(dev_frames)]
        return ctx.stereo_sgm(l, r, D, P1, P2, paths=PATHS, lr=LR)

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()

    # ---- device-resident timed region (the headline): one event pair per step ----
    import ctypes

    from thundervision_b200 import _lib
    lib = _lib.lib()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk = Clocks(local)
    total_ms = 0.0
    for i in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        step(i)
        e1.record(st)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
    torch.cuda.synchronize()
    clocks = clk.stop()

    # ---- per-kernel device time (events around every kernel inside the ABI;
    #      work that runs on two streams runs in sequence while timing is on,
    #      so each kernel is timed alone, as in the ncu launch list) ----
    lib.tdv_ctx_enable_timing(ctx.handle, 1)
    kbuf = (ctypes.c_float * 64)()
    ksum, kcnt = {}, {}
    launches_per_step = 0
    for i in range(args.steps):
        flush.zero_()
        step(i)
        n = lib.tdv_ctx_timings(ctx.handle, kbuf, 64)
        launches_per_step = n
        for j in range(n):
            nm = lib.tdv_ctx_timing_name(ctx.handle, j).decode()
            ksum[nm] = ksum.get(nm, 0.0) + kbuf[j]
            kcnt[nm] = kcnt.get(nm, 0) + 1
    torch.cuda.synchronize()
    lib.tdv_ctx_enable_timing(ctx.handle, 0)
    launches = launches_per_step * args.steps

    # ---- end-to-end through the public API, host buffers ----
    host_out = torch.empty((H, W), dtype=torch.uint16).pin_memory()
    dl = torch.empty((H, W), dtype=torch.uint8, device=dev)
    dr = torch.empty((H, W), dtype=torch.uint8, device=dev)
    e2e_ms = 0.0
    e2e_steps = []
    parts = [0.0, 0.0, 0.0]
    clk2 = Clocks(local)
    for i in range(args.steps):
        flush.zero_()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        pl, pr = pinned[i % len(pinned)]
        ev[0].record(st)
        dl.copy_(pl, non_blocking=True)
        dr.copy_(pr, non_blocking=True)
        ev[1].record(st)
        out = ctx.stereo_sgm(dl, dr, D, P1, P2, paths=PATHS, lr=LR)
        ev[2].record(st)
        host_out.copy_(out["disp"], non_blocking=True)
        ev[3].record(st)
        ev[3].synchronize()
        step_ms = ev[0].elapsed_time(ev[3])
        e2e_steps.append(step_ms)
        e2e_ms += step_ms
        for j in range(3):
            parts[j] += ev[j].elapsed_time(ev[j + 1])
    clocks_e2e = clk2.stop()

    # ---- end-to-end over a frame stream through the public video API:
    #      every frame copied from pinned host memory and its map copied back,
    #      double-buffered so that copies overlap the previous frame's kernels,
    #      each frame one CUDA graph replay of the per-frame kernels ----
    from thundervision_b200 import video
    loop = video.VideoLoop(ctx, W, H, D, P1, P2, paths=PATHS, lr=LR, engine="launches")
    stream_in = [pinned[i % len(pinned)] for i in range(args.steps)]
    stream_out = [torch.empty((H, W), dtype=torch.uint16).pin_memory() for _ in range(args.steps)]
    loop.run(stream_in[:min(len(stream_in), args.warmup)], stream_out[:min(len(stream_in), args.warmup)])
    flush.zero_()
    clk3 = Clocks(local)
    stream_ms = loop.run(stream_in, stream_out)
    clocks_stream = clk3.stop()
    stream_ok = bool(torch.equal(stream_out[-1], ctx.stereo_sgm(*dev_frames[(args.steps - 1) % len(dev_frames)], D, P1,
                                                                  P2, paths=PATHS, lr=LR)["disp"].cpu()))
    loop.close()

    from thundervision_b200.replicas import max_over_ranks
    total_ms, e2e_ms, stream_ms = max_over_ranks([total_ms, e2e_ms, stream_ms], device=dev)
    if world > 1:
        dist.barrier()
    if rank != 0:
        ctx.close()
        if world > 1:
            dist.destroy_process_group()
        return

    frames = args.steps * world
    fps = frames / (total_ms / 1000.0)
    e2e_fps = frames / (e2e_ms / 1000.0)
    stream_fps = frames / (stream_ms / 1000.0)
    cells = W * H * D * PATHS
    # dominant kernel: the compiled kernel (as ncu names it) with the largest
    # share of the per-kernel device time
    fsum, fcnt, fbytes = {}, {}, {}
    for k in ksum:
        f = KERNEL_OF.get(k, k)
        fsum[f] = fsum.get(f, 0.0) + ksum[k]
        fcnt[f] = fcnt.get(f, 0) + kcnt[k]
        fbytes[f] = fbytes.get(f, 0) + alg_bytes(k) * kcnt[k]
    dom = max(fsum, key=lambda f: fsum[f])
    avg_ms = fsum[dom] / fcnt[dom]
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    dom_bytes = fbytes[dom] / fcnt[dom]
    achieved = dom_bytes / (avg_ms / 1000.0) / 1e9
    traffic = None
    try:
        tr = json.load(open(os.path.join(ROOT, "profiles", "fused_traffic_1080p_d256.json")))
        traffic = tr.get("per_launch_bytes", {}).get(dom)
    except OSError:
        pass
    kernels = {k: {"launches": kcnt[k], "avg_ms": ksum[k] / kcnt[k],
                   "share": ksum[k] / sum(ksum.values())} for k in sorted(ksum)}
    frame_alg = W * H * D * 4 * (PATHS + 3) + W * H * (2 * 1 + 2)
    frame_own = sum(alg_bytes(k) * kcnt[k] for k in kcnt) / args.steps
    line = {
        "metric": METRIC, "value": fps, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic",
        "config": config({"parallelism": f"replicas x{world}, frames sharded by rank"}),
        "gcells_per_s": cells * fps / 1e9,
        "e2e": {"value": stream_fps, "unit": UNIT, "h2d_bytes_per_step": 2 * W * H,
                "d2h_bytes_per_step": 2 * W * H, "ms_per_step": stream_ms / args.steps,
                "path": "video.VideoLoop: pinned host frames in, maps out to pinned host, two buffer sets, "
                        "each with its own context and compute stream so consecutive frames overlap, "
                        "one CUDA graph replay of the tdv_stereo_sgm kernels per frame",
                "last_map_equals_stereo_sgm": stream_ok, "clocks": clocks_stream},
        "e2e_sequential": {"value": e2e_fps, "unit": UNIT, "h2d_bytes_per_step": 2 * W * H,
                           "d2h_bytes_per_step": 2 * W * H,
                           "path": "per step: copy in, tdv_stereo_sgm, copy out, in sequence on one stream",
                           "ms_per_step": {"h2d": parts[0] / args.steps, "stereo_sgm": parts[1] / args.steps,
                                           "d2h": parts[2] / args.steps},
                           "median_ms_per_step": sorted(e2e_steps)[len(e2e_steps) // 2],
                           "max_ms_per_step": max(e2e_steps), "clocks": clocks_e2e},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "alg_bytes_per_launch": dom_bytes, "avg_launch_ms": avg_ms,
                     "share": fsum[dom] / sum(fsum.values()),
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if "hbm_gbs" in peaks
                     else "fallback 6.65 TB/s"},
        "frame_roofline": {"model": "stage-interface bytes W*H*D*4*(P+3)+W*H*4 per frame",
                           "achieved_gbs": frame_alg * fps / world / 1e9,
                           "frac": frame_alg * fps / world / 1e9 / peak},
        "frame_alg_roofline": {"model": "sum of the frame's kernels' algorithmic bytes",
                               "bytes": frame_own, "achieved_gbs": frame_own * fps / world / 1e9,
                               "frac": frame_own * fps / world / 1e9 / peak},
        "kernels": kernels,
        "kernel_functions": {f: {"launches": fcnt[f], "avg_ms": fsum[f] / fcnt[f],
                                 "share": fsum[f] / sum(fsum.values())} for f in sorted(fsum)},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if not args.no_extras:
        for key, fn in (("batch", measure_batch), ("soft", measure_soft), ("plain", measure_plain),
                        ("image_stages", measure_image), ("reconstruction", measure_reconstruction),
                        ("video", measure_video)):
            try:
                line[key] = fn(ctx, dev)
            except Exception as exc:  # an extra never hides the headline line
                line[key] = {"error": f"{type(exc).__name__}: {exc}"}
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample()
    print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


def profile_case_general():
    """One launch of each general-path kernel on a 1280x720 pair, D=64 (a
    236 MB DSI, larger than L2): BT cost, SGM with the reference table and
    REF_GPU semantics, DP, FastWTA, SSD 7x7 cost."""
    import torch

    from thundervision_b200 import api, synthetic
    ctx = api.Context(0)
    dev = torch.device("cuda", 0)
    w, h, d = 1280, 720, 64
    l, r, _, _ = synthetic.pair_sized(w, h, d, 3)
    lf = torch.from_numpy(l).to(dev).float() * (1.0 / 255.0)
    rf = torch.from_numpy(r).to(dev).float() * (1.0 / 255.0)
    C = ctx.cost(lf, rf, d)
    ctx.sgm(C, 30 / 255, 150 / 255, guide=lf, p2_mode="adjust", table="ref", semantics="ref_gpu")
    ctx.dp(C)
    ctx.fast_wta(lf, rf, d)
    ctx.cost(lf, rf, d, kind="ssd", radius=3)
    torch.cuda.synchronize()
    ctx.close()
    print(json.dumps({"profile_case": "general", "ok": True}))


def profile_case_cost1080():
    """One BT cost DSI (HWD, 2.12 GB) of a 1920x1080 pair at D=256 after
    one warm-up call."""
    import torch

    from thundervision_b200 import api, synthetic
    ctx = api.Context(0)
    dev = torch.device("cuda", 0)
    l, r, _, _ = synthetic.pair_sized(W, H, D, 3)
    lf = torch.from_numpy(l).to(dev).float() * (1.0 / 255.0)
    rf = torch.from_numpy(r).to(dev).float() * (1.0 / 255.0)
    out = torch.empty((H, W, D), dtype=torch.float32, device=dev)
    for _ in range(2):
        ctx.cost(lf, rf, D, out=out)
    torch.cuda.synchronize()
    ctx.close()
    print(json.dumps({"profile_case": "cost1080", "ok": True}))


def main():
    args = parse()
    if args.profile_case == "general":
        profile_case_general()
        return
    if args.profile_case == "cost1080":
        profile_case_cost1080()
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
