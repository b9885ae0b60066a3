#!/usr/bin/env python
"""Throughput of the dense-stereo hot path on the full-HD configuration:
1920x1080 rectified u8 pair, D = 256, Birchfield-Tomasi cost, 8-path SGM
(P1 = 10, P2 = 120, constant), WTA + left-right check (threshold 1).  By
default the aggregation is the reference's own: the CPU recurrence of
tdvision/semiglobalcpu.cpp:56-126 (start-assign, minimum over d < D-1) over
the reference's path table (tdvision/semiglobal.cu:57-230, stale diagonal
ends); --semantics standard runs the textbook recurrence over the full table.

One step = one stereo frame through tdv_stereo_sgm.  Prints one JSON line.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--semantics reference|standard] [--cpu-matrix]

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

Reference arm (--impl reference): the same computation on the host cores, rank
0 only: the oracle's restatement of the reference's CPU path (BT, the
aggregation of the chosen semantics, WTACPU, the left-right check) on all host
threads, each step a band of rows of the same frame sized so the run stays
within a few minutes.  The reference's own compiled code (oracle/_ref, built
from its sources) is timed beside it on the same band: it hard-wires its
penalties (P1 = 30/255, P2 = 150/255 divided by |dI|,
tdvision/semiglobalcpu.cpp:36-37,99-102) and runs on one thread as written, so
it cannot run this configuration itself; the restatement equals it bit for bit
in its own configuration (tests/test_oracle_ref.py).
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
# recurrence and path table per --semantics: stereo_sgm keywords, the
# oracle's constants, and the fused kernels' variant at D = 256 (0 standard
# over the full table; 2 reference weights with the minimum over d < D-1)
SEMANTICS = {
    "reference": {"kw": {"semantics": "ref_cpu", "table": "ref"}, "orc": (1, 1), "var": 2,
                  "recurrence": "reference CPU (tdvision/semiglobalcpu.cpp:56-126: start-assign, min over d < D-1)",
                  "table": "reference (tdvision/semiglobal.cu:57-230, stale diagonal ends)"},
    "standard": {"kw": {"semantics": "standard", "table": "full"}, "orc": (0, 0), "var": 0,
                 "recurrence": "standard (S += C at path starts, min over all d)",
                 "table": "full (every line walked once each way)"},
    "reference_gpu": {"kw": {"semantics": "ref_gpu", "table": "ref"}, "orc": (2, 1), "var": 1,
                      "recurrence": "reference GPU (tdvision/semiglobal.cu:283-466 without its race: "
                                    "the second step from C + P1)",
                      "table": "reference (tdvision/semiglobal.cu:57-230, stale diagonal ends)"},
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--semantics", choices=sorted(SEMANTICS), default="reference")
    ap.add_argument("--frames", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batch and soft-SGM measurements")
    ap.add_argument("--cpu-matrix", action="store_true",
                    help="time the CPU baselines (reference code, restatement on one and on all threads; "
                         "384x288 D=16, 640x480 D=64, 1080p D=256; 8 and 4 paths), print one JSON line, exit")
    ap.add_argument("--profile-case", choices=["general", "cost1080"],
                    help="general: one launch of each general-path kernel on 1280x720, D=64; cost1080: "
                         "one BT cost DSI at 1920x1080, D=256 (HWD); then exit (the cases the ncu "
                         "summaries are captured on)")
    return ap.parse_args()


def config(sem):
    """The workload both arms run (identical dicts for one --semantics)."""
    s = SEMANTICS[sem]
    return {"workload": f"BT + SGM-{PATHS} + WTA + LR, {W}x{H}, D={D}", "width": W, "height": H,
            "max_disp": D, "paths": PATHS, "p1": P1, "p2": P2, "p2_mode": "constant",
            "recurrence": s["recurrence"], "path_table": s["table"],
            "domain": "u8 intensities used unscaled", "lr_threshold": LR,
            "l2": "a timed frame sequence has no flush between frames: every frame streams 15.5 GB of "
                  "aggregation volumes through HBM (126 MB L2) and an input pair recurs only after three "
                  "other frames; one-frame-per-call legs flush L2 (256 MiB write) before each call",
            "inputs": "seeded synthetic video frames (moving rectangles over a slanted plane)"}


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
def _band(h, frame_seed=1000):
    """Rows 0..h-1 of the first frame rank 0 times, as a W x h pair."""
    from thundervision_b200 import synthetic
    L, R = synthetic.VideoStream(seed=frame_seed).frame(0)[:2]
    return L[:h].copy(), R[:h].copy()


def port_run(L, R, sem, threads, paths=PATHS, d=D):
    """The oracle's restatement of the reference CPU path on a u8 pair: BT
    cost, SGM of the semantics, WTA, left-right check; (seconds, dl, dr)."""
    import oracle
    sm, tb = SEMANTICS[sem]["orc"]
    t0 = time.perf_counter()
    Lf, Rf = oracle.u8_to_f32(L), oracle.u8_to_f32(R)
    C = oracle.bt_cost(Lf, Rf, d)
    dd, _, S = oracle.sgm(C, Lf, P1, P2, paths=paths, table=tb, semantics=sm, threads=threads)
    dl, dr = oracle.lr_check(S, dd, thr=LR)
    return time.perf_counter() - t0, dl, dr


def ref_code_lib():
    """The reference's own CPU aggregation compiled from its sources
    (oracle/_ref/libtdvref.so), or None where it was not built."""
    import ctypes
    path = os.path.join(ROOT, "oracle", "_ref", "libtdvref.so")
    if not os.path.exists(path):
        return None
    lib = ctypes.CDLL(path)
    f32p = ctypes.POINTER(ctypes.c_float)
    lib.ref_semiglobal_cpu.argtypes = [f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, f32p, f32p]
    return lib


def ref_code_run(lib, L, R, d=D):
    """SemiGlobalCPU::updateImpl + WTACPU of the reference (one thread, as
    written; TBB disabled, tdvision/semiglobalcpu.cpp:191-222) on the BT cost
    of a u8 pair in the reference's own configuration ([0,1] intensities,
    P1 = 30/255, P2 = 150/255 divided by |dI|); the cost DSI is computed
    before the timed call (the reference computes it on the GPU).  Returns
    (seconds, d/D map)."""
    import ctypes

    import numpy as np

    import oracle
    s = np.float32(1) / np.float32(255)
    Lf, Rf = oracle.u8_to_f32(L, s), oracle.u8_to_f32(R, s)
    C = np.ascontiguousarray(oracle.bt_cost(Lf, Rf, d, layout=oracle.LAYOUT_REF_WHD))
    h, w = L.shape
    dn = np.empty((h, w), np.float32)
    p = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    # the reference prints its own timer to stdout (semiglobalcpu.cpp:229,
    # wtacpu.cpp:54): send it to stderr so that stdout stays one JSON line
    libc = ctypes.CDLL(None)
    sys.stdout.flush()
    saved = os.dup(1)
    os.dup2(2, 1)
    try:
        t0 = time.perf_counter()
        lib.ref_semiglobal_cpu(p(C), w, h, d, p(Lf), p(dn))
        t = time.perf_counter() - t0
        libc.fflush(None)
    finally:
        os.dup2(saved, 1)
        os.close(saved)
    return t, dn


def _rows_for(seconds_per_step, sem, threads, lo=16):
    """Band height whose restatement run takes about `seconds_per_step`."""
    L, R = _band(lo)
    t, _, _ = port_run(L, R, sem, threads)
    return int(max(lo, min(H, seconds_per_step / (t / lo))))


def cpu_reference_run(steps, warmup, sem, budget_s=60.0):
    """Times the restatement on bands of a full-HD frame on every host thread;
    returns (frames/s, seconds per step, rows, threads, description)."""
    threads = os.cpu_count() or 1
    total_steps = max(1, steps + warmup)
    h = _rows_for(budget_s / total_steps, sem, threads)
    L, R = _band(h)
    for _ in range(warmup):
        port_run(L, R, sem, threads)
    ts = [port_run(L, R, sem, threads)[0] for _ in range(steps)]
    t = sum(ts) / len(ts)
    desc = (f"rows 0..{h - 1} of a {W}x{H} frame (a {W}x{h} pair, {h / H:.3f} frame) per step, D={D}, "
            f"{PATHS} paths, BT + {SEMANTICS[sem]['recurrence']} over the {SEMANTICS[sem]['table']} table + "
            f"WTACPU + left-right check, the oracle's restatement (pinned to the reference's compiled code) "
            f"on {threads} threads; frames/s scaled by rows")
    return (h / H) / t, t, h, threads, desc


def reference_code_sample(rows=48, reps=1):
    """The reference's compiled SemiGlobalCPU (one thread) on a band, its own
    configuration; frames/s scaled by rows, or None without oracle/_ref."""
    lib = ref_code_lib()
    if lib is None:
        return None
    L, R = _band(rows)
    t = min(ref_code_run(lib, L, R)[0] for _ in range(reps))
    return {"value": (rows / H) / t, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"rows 0..{rows - 1} of the {W}x{H} frame ({W}x{rows} pair), D={D}, 8 paths: "
                      "LibThunderVision's SemiGlobalCPU::updateImpl + WTACPU compiled from its sources "
                      "(oracle/_ref), one thread as written, its compile-time penalties (P1 = 30/255, "
                      "P2 = 150/255 / |dI|, [0,1] intensities; the same operations per cell as this "
                      "configuration's constant P2); cost DSI precomputed; frames/s scaled by rows"}


def cpu_baseline_sample(sem, budget_s=20.0):
    fps, t, h, threads, desc = cpu_reference_run(1, 0, sem, budget_s=budget_s)
    out = {"value": fps, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc,
           "seconds_per_sample": t}
    rc = reference_code_sample()
    if rc is not None:
        out["reference_code"] = rc
    return out


def band_parity(ctx, dev, sem, rows=64):
    """Our GPU path against the CPU path on the same band (as its own W x
    rows pair): the fused kernels vs the restatement for this configuration,
    and the general float path in the reference's own configuration vs the
    reference's compiled SemiGlobalCPU (d/D maps), bit for bit."""
    import numpy as np
    import torch
    L, R = _band(rows)
    threads = os.cpu_count() or 1
    _, dl, dr = port_run(L, R, sem, threads)
    out = ctx.stereo_sgm(torch.from_numpy(L).to(dev), torch.from_numpy(R).to(dev), D, P1, P2, paths=PATHS,
                         lr=LR, right_disp=True, **SEMANTICS[sem]["kw"])
    res = {"rows": rows, "fused_vs_restatement_bit_exact":
           bool(np.array_equal(out["disp"].cpu().numpy(), dl) and np.array_equal(out["disp_right"].cpu().numpy(), dr))}
    lib = ref_code_lib()
    if lib is not None:
        _, dn = ref_code_run(lib, L, R)
        s = float(np.float32(1) / np.float32(255))
        g = ctx.stereo_sgm(torch.from_numpy(L).to(dev), torch.from_numpy(R).to(dev), D,
                           float(np.float32(30) / np.float32(255)), float(np.float32(150) / np.float32(255)),
                           paths=8, p2_mode="adjust", table="ref", semantics="ref_cpu", scale=s, norm=True)
        res["general_literal_vs_reference_code_bit_exact"] = bool(np.array_equal(g["disp_norm"].cpu().numpy(), dn))
    return res


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    fps, t, h, threads, desc = cpu_reference_run(args.steps, args.warmup, args.semantics)
    line = {"metric": METRIC, "value": fps, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * t, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference", "config": config(args.semantics),
            "sample_rows": h, "sample_frame_fraction": h / H,
            "cpu_baseline": {"value": fps, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc},
            "e2e": {"value": fps, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    rc = reference_code_sample()
    if rc is not None:
        line["reference_code"] = rc
    print(json.dumps(line), flush=True)


def cpu_matrix():
    """CPU baselines on this host: the reference's compiled code (one thread,
    its own configuration, 8 paths only: its table always holds the diagonals)
    and the restatement (this configuration) on one and on all threads, 8 and 4
    paths; 384x288 D=16 and 640x480 D=64 as whole frames, 1080p D=256 as a
    64-row band scaled by rows; median of 5 after one warm-up."""
    import numpy as np

    from thundervision_b200 import synthetic
    threads = os.cpu_count() or 1
    model = ""
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                model = ln.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    lib = ref_code_lib()
    cases = [("384x288_D16", synthetic.pair_small(1)[:2], 16, 1.0),
             ("640x480_D64", synthetic.pair_medium(1)[:2], 64, 1.0),
             ("1920x1080_D256_band64", _band(64), 256, 64 / H)]
    res = {"host_threads": threads, "cpu_model": model, "repeats": "median of 5 after 1 warm-up",
           "note": "seconds per frame (band runs scaled by rows); the reference code runs its own penalties "
                   "(P1 = 30/255, P2 = 150/255 / |dI| on [0,1] intensities), the restatement this configuration "
                   "(P1 = 10, P2 = 120 constant, 0..255 intensities, reference CPU recurrence and table); "
                   "the cost DSI is outside the reference code's time (it computes it on the GPU); the "
                   "reference's toCpuMem (a device-to-host copy per DSI row) has no host-only counterpart and is "
                   "not timed"}

    def med(fn):
        fn()
        return float(np.median([fn() for _ in range(5)]))

    for name, (L, R), d, frac in cases:
        row = {}
        if lib is not None:
            row["reference_code_1thread_8path"] = med(lambda: ref_code_run(lib, L, R, d)[0]) / frac
        for paths in (8, 4):
            for th in (1, threads):
                row[f"restatement_{th}threads_{paths}path"] = med(
                    lambda: port_run(L, R, "reference", th, paths=paths, d=d)[0]) / frac
        res[name] = row
    print(json.dumps({"cpu_matrix": res}), flush=True)


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


def batch_trace_summary(tr, shapes, per_sm):
    """Where one persistent batch run spends its block-time, from the per-item
    trace (taken, dependency met, ended, smid << 32 | pair * 16 + pass): work,
    dependency waits (per pass), the gaps a block spends between items, and
    the tail each SM idles after its last item (per_sm blocks per SM take
    items in turn; the tail is counted per SM); the time of the items of the
    pairs below 0.25 Mpixel."""
    import numpy as np
    t = tr.numpy().astype(np.int64)
    take, go, end = t[:, 0], t[:, 1], t[:, 2]
    ok = (take > 0) & (go >= take) & (end >= go)
    take, go, end, info = take[ok], go[ok], end[ok], t[ok, 3]
    sm = info >> 32
    pp = info & 0xFFFFFFFF
    pair, ps = pp >> 4, pp & 15
    t0, t1 = take.min(), end.max()
    span = float(t1 - t0)
    slots = len(np.unique(sm)) * per_sm
    busy = float((end - go).sum())
    wait = float((go - take).sum())
    last_end = {}
    for s_, e_ in zip(sm, end):
        last_end[s_] = max(last_end.get(s_, 0), e_)
    tail = float(sum(t1 - e for e in last_end.values())) * per_sm
    total = span * slots
    small = np.array([w * h < 250000 for (w, h, d) in shapes])[pair]
    names = ["prep", "V+", "V-", "D1+", "D1-", "D2+", "D2-", "H+", "H-"]
    return {"span_ms": span / 1e6, "block_slots": int(slots),
            "work_frac": busy / total, "dependency_wait_frac": wait / total, "tail_idle_frac": tail / total,
            "other_frac": max(0.0, 1.0 - (busy + wait + tail) / total),
            "wait_ms_by_pass": {names[p]: float((go - take)[ps == p].sum()) / 1e6 for p in range(9)},
            "small_pairs_work_frac": float((end - go)[small].sum()) / max(busy, 1.0)}


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
    # algorithmic bytes of the fused kernels: each pair's 16-bit volume holds
    # 64 * ceil-to-{1,2,4}(D / 64) disparities per pixel and is touched 14 times
    # (two first stores, four read-modify-writes, the join's two reads and one
    # write, the last pass's read), plus the BT planes (34 B per pixel) per pass
    span = lambda d: 64 if d <= 64 else (128 if d <= 128 else 256)
    batch_bytes = sum(w * h * (2 * span(d) * 14 + 34 * 8) for (w, h, d) in shapes)
    peak = 6650.0
    try:
        peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
    except (OSError, KeyError, ValueError):
        pass
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
    trace = batch_trace_summary(b.trace(), shapes, int(tiles.get("ctas_per_sm", 1)) if isinstance(tiles, dict) else 1)
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
            "roofline": {"alg_bytes": batch_bytes, "hbm_floor_ms": batch_bytes / (peak * 1e9) * 1e3,
                         "batch_frac": batch_bytes / (peak * 1e9) / (t_graph / 1000.0),
                         "per_pair_fused_frac": batch_bytes / (peak * 1e9) / (t_pair / 1000.0),
                         "max_speedup_vs_per_pair_fused": t_pair / (batch_bytes / (peak * 1e9) * 1e3)},
            "bit_identical_to_per_pair": equal and plain_equal, "trace": trace}


def measure_batch_sharded(ctx, dev, rank, world, reps=3):
    """The 64-pair uneven batch split over the ranks (replicas.shard_pairs:
    largest pairs first, each to the least-loaded rank): every rank runs one
    graph-replayed persistent batch over its share with autotuned tiles, no
    collective on the data path; returns this rank's (ms per run, pairs)."""
    import torch

    from thundervision_b200 import api, replicas, synthetic
    shapes = synthetic.batch_shapes(seed=0, n=64)
    pairs = []
    for i, (w, h, d) in enumerate(shapes):
        l, r, _, _ = synthetic.pair_sized(w, h, d, synthetic.pair_seed(0, i) % (2 ** 31))
        pairs.append((l, r, d))
    idx, mine = replicas.shard_pairs(pairs, rank, world)
    dev_pairs = [(torch.from_numpy(l).to(dev), torch.from_numpy(r).to(dev), d) for (l, r, d) in mine]
    b = api.Batch(ctx, dev_pairs, P1, P2, paths=8)
    try:
        b.autotune(reps=2)
        ms = _event_ms(b.graph_launch, reps, 1, torch.cuda.current_stream())
        b.status()
    finally:
        b.close()
    return ms, len(idx)


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


def measure_configs(ctx, dev, sem, reps=20):
    """The fused call (tdv_stereo_sgm: BT + SGM + WTA + L-R, threshold 1) on
    each plain-method configuration under the bench's semantics: 384x288
    D=16 and 640x480 D=64 (8 paths), 1920x1080 D=256 with 8 and 4 paths;
    device ms per pair, L2 flushed before each call (mean of `reps`)."""
    import torch

    from thundervision_b200 import synthetic
    st = torch.cuda.current_stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    out = {"semantics": sem, "l2": "flushed before each call"}
    cases = [("384x288_D16_P8", synthetic.pair_small(1)[:2], 16, 8),
             ("640x480_D64_P8", synthetic.pair_medium(1)[:2], 64, 8),
             ("1920x1080_D256_P8", _band(H), 256, 8),
             ("1920x1080_D256_P4", _band(H), 256, 4)]
    for name, (L, R), d, paths in cases:
        l, r = torch.from_numpy(L).to(dev), torch.from_numpy(R).to(dev)
        h, w = L.shape

        def call():
            return ctx.stereo_sgm(l, r, d, P1, P2, paths=paths, lr=LR, **SEMANTICS[sem]["kw"])

        for _ in range(3):
            call()
        torch.cuda.synchronize()
        tot = 0.0
        for _ in range(reps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            call()
            e1.record(st)
            e1.synchronize()
            tot += e0.elapsed_time(e1)
        ms = tot / reps
        out[name] = {"ms": ms, "fps": 1000.0 / ms, "gcells_per_s": w * h * d * paths / (ms / 1000.0) / 1e9}
    return out


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
    # the same stage chain on u8 intensities (the integer domain: P1 = 10,
    # P2 = 120, reference CPU recurrence and table, WTA + left-right check)
    # with the DSI as F32 and as the exact 16-bit half-unit DSI
    l, r, _, _ = synthetic.pair_sized(1920, 1080, 256, 3)
    l8, r8 = torch.from_numpy(l).to(dev), torch.from_numpy(r).to(dev)
    ints = {"workload": "1920x1080, D=256, u8 images: tdv_cost BT (HWD) + tdv_sgm (reference CPU recurrence "
                        "and table, P1 = 10, P2 = 120, 8 paths) + WTA + left-right check; device ms per pair"}
    for dt in ("f32", "u16"):
        dsi = torch.empty((1080, 1920, 256), dtype=torch.float32 if dt == "f32" else torch.uint16, device=dev)

        def run_int():
            ctx.cost(l8, r8, 256, kind="bt", out=dsi)
            return ctx.sgm(dsi, 10.0, 120.0, table="ref", semantics="ref_cpu", lr=1)

        ints[f"dsi_{dt}_ms"] = _event_ms(run_int, reps, 1, st)
        ints[f"dsi_{dt}_map"] = run_int()["disp"].clone()
        del dsi
    ints["maps_equal"] = bool(torch.equal(ints.pop("dsi_f32_map"), ints.pop("dsi_u16_map")))
    out["1920x1080_D256_integer_domain"] = ints
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
def kernel_of(sem):
    """The compiled kernel behind each timed pass (PPL = 4 at D = 256), as
    ncu names it; the last template argument is the kernel variant."""
    e = SEMANTICS[sem]["var"]
    return {
        "fused_prep": "prep_kernel",
        "fused_pass_V+": f"vd_pass<4, 0, 0, {e}>",
        "fused_pass_D1-": f"vd_pass<4, 0, 1, {e}>",
        "fused_pass_V-": f"vd_pass<4, 1, 0, {e}>",
        "fused_pass_D1+": f"vd_pass<4, 1, 1, {e}>",
        "fused_pass_D2+": f"vd_pass<4, 1, 1, {e}>",
        "fused_pass_D2-": f"vd_pass<4, 1, 1, {e}>",
        "fused_pass_H+": f"hp_pass<4, 1, 1, {e}>",
        "fused_pass_H-_wta": f"hp_wta_pass<4, 0, {e}>",
    }


def time_frames(ctx, frames, kw, steps, flush, st):
    """Device ms per frame of tdv_stereo_sgm over device-resident frames, L2
    flushed before each, and the per-kernel means (events around each kernel,
    the two pass chains in sequence)."""
    import ctypes

    import torch

    from thundervision_b200 import _lib
    lib = _lib.lib()

    def step(i):
        l, r = frames[i % len(frames)]
        return ctx.stereo_sgm(l, r, D, P1, P2, paths=PATHS, lr=LR, **kw)

    for i in range(3):
        step(i)
    total = 0.0
    for i in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        step(i)
        e1.record(st)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    lib.tdv_ctx_enable_timing(ctx.handle, 1)
    kbuf = (ctypes.c_float * 64)()
    ksum, kcnt = {}, {}
    for i in range(steps):
        flush.zero_()
        step(i)
        n = lib.tdv_ctx_timings(ctx.handle, kbuf, 64)
        for j in range(n):
            nm = lib.tdv_ctx_timing_name(ctx.handle, j).decode()
            ksum[nm] = ksum.get(nm, 0.0) + kbuf[j]
            kcnt[nm] = kcnt.get(nm, 0) + 1
    torch.cuda.synchronize()
    lib.tdv_ctx_enable_timing(ctx.handle, 0)
    return total / steps, {k: ksum[k] / kcnt[k] for k in sorted(ksum)}


def measure_reference_literal(ctx, dev, frames, flush, reps=5):
    """What the reference's own compiled code computes, on the GPU: BT on
    [0,1] intensities, its CPU recurrence over its path table with P1 =
    30/255 and P2 = 150/255 divided by |dI|, WTA (the general float path:
    cost DSI + scheduled passes), 1080p D=256, device ms per frame."""
    import numpy as np
    import torch
    st = torch.cuda.current_stream()
    s = float(np.float32(1) / np.float32(255))
    p1, p2 = float(np.float32(30) / np.float32(255)), float(np.float32(150) / np.float32(255))

    def run(i):
        l, r = frames[i % len(frames)]
        ctx.stereo_sgm(l, r, D, p1, p2, paths=8, p2_mode="adjust", table="ref", semantics="ref_cpu", scale=s,
                       norm=True)

    run(0)
    ts = []
    for i in range(reps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        run(i)
        e1.record(st)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    ms = sorted(ts)[len(ts) // 2]
    return {"workload": f"{W}x{H}, D={D}: BT on [0,1] intensities + reference CPU recurrence and path table, "
                        "P1 = 30/255, P2 = 150/255 / |dI| + WTA, through tdv_stereo_sgm (general float path)",
            "ms": ms, "fps": 1000.0 / ms}


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

    SEM = SEMANTICS[args.semantics]["kw"]
    KERNEL_OF = kernel_of(args.semantics)

    def step(i):
        l, r = dev_frames[i % len(dev_frames)]
        return ctx.stereo_sgm(l, r, D, P1, P2, paths=PATHS, lr=LR, **SEM)

    # the frame sequence of the headline: `steps` frames, cycling through the
    # device-resident frames, in one tdv_stereo_sgm_frames call
    seq_l = [dev_frames[i % len(dev_frames)][0] for i in range(args.steps)]
    seq_r = [dev_frames[i % len(dev_frames)][1] for i in range(args.steps)]

    def sequence(outs=None):
        return ctx.stereo_sgm_frames(seq_l, seq_r, D, P1, P2, paths=PATHS, lr=LR, outs=outs, **SEM)

    for i in range(args.warmup):
        step(i)
    seq_outs = sequence()  # allocates the second lane and the output maps
    for _ in range(max(0, args.warmup - 1)):
        sequence(seq_outs)
    torch.cuda.synchronize()

    # ---- device-resident timed region (the headline): K frames in one call,
    #      consecutive frames on two lanes; one event pair around the call ----
    import ctypes

    from thundervision_b200 import _lib
    lib = _lib.lib()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    flush.zero_()
    clk = Clocks(local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    sequence(seq_outs)
    e1.record(st)
    e1.synchronize()
    total_ms = e0.elapsed_time(e1)
    clocks = clk.stop()
    seq_ok = all(bool(torch.equal(seq_outs[i]["disp"], step(i)["disp"])) for i in range(min(args.steps, 4)))

    # ---- one frame per call, L2 flushed before each: the per-frame latency ----
    torch.cuda.synchronize()
    clk1 = Clocks(local)
    single_ms = 0.0
    for i in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        step(i)
        e1.record(st)
        e1.synchronize()
        single_ms += e0.elapsed_time(e1)
    torch.cuda.synchronize()
    clocks_single = clk1.stop()

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
        out = ctx.stereo_sgm(dl, dr, D, P1, P2, paths=PATHS, lr=LR, **SEM)
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
    loop = video.VideoLoop(ctx, W, H, D, P1, P2, paths=PATHS, lr=LR, engine="launches", **SEM)
    stream_in = [pinned[i % len(pinned)] for i in range(args.steps)]
    stream_out = [torch.empty((H, W), dtype=torch.uint16).pin_memory() for _ in range(args.steps)]
    loop.run(stream_in[:min(len(stream_in), args.warmup)], stream_out[:min(len(stream_in), args.warmup)])
    flush.zero_()
    clk3 = Clocks(local)
    stream_ms = loop.run(stream_in, stream_out)
    clocks_stream = clk3.stop()
    stream_ok = bool(torch.equal(stream_out[-1], ctx.stereo_sgm(*dev_frames[(args.steps - 1) % len(dev_frames)], D, P1,
                                                                  P2, paths=PATHS, lr=LR, **SEM)["disp"].cpu()))
    loop.close()

    from thundervision_b200.replicas import max_over_ranks
    sharded = None
    if world > 1 and not args.no_extras:
        # every rank takes part: the batch split over the ranks, time = max over ranks
        b_ms, b_n = measure_batch_sharded(ctx, dev, rank, world)
        b_max, b_min = max_over_ranks([b_ms, -b_ms], device=dev)
        sharded = {"workload": "the 64-pair uneven batch split over the ranks by cell count, one persistent "
                               "graph-replayed batch per rank, autotuned per rank",
                   "ranks": world, "pairs_on_rank0": b_n, "ms_max_over_ranks": b_max, "ms_min_over_ranks": -b_min,
                   "pairs_per_s": 64 / (b_max / 1000.0)}
    total_ms, e2e_ms, stream_ms, single_ms = max_over_ranks([total_ms, e2e_ms, stream_ms, single_ms], device=dev)
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
        "config": config(args.semantics), "replicas": f"{world}, frames sharded by rank",
        "gcells_per_s": cells * fps / 1e9,
        "timed": f"{args.steps} frames per rank in one tdv_stereo_sgm_frames call (consecutive frames on two "
                 "lanes with their own volumes and streams), device-resident inputs",
        "sequence_maps_equal_single_calls": seq_ok,
        "single_frame": {"value": frames / (single_ms / 1000.0), "unit": UNIT,
                         "ms_per_frame": single_ms / args.steps, "clocks": clocks_single,
                         "path": "one tdv_stereo_sgm call per frame, L2 flushed before each; the per-frame "
                                 "latency (the two pass chains of a frame run concurrently)"},
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
                     "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum per launch of this kernel "
                                       "from the ncu capture in profiles/fused_traffic_1080p_d256.json (not "
                                       "measured in this run)",
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
    if sharded is not None:
        line["batch_sharded"] = sharded
    if not args.no_extras:
        # the other recurrences / tables on the same frames and kernels
        for other in [o for o in SEMANTICS if o != args.semantics]:
            try:
                oms, okern = time_frames(ctx, dev_frames, SEMANTICS[other]["kw"], args.steps, flush, st)
                okw = SEMANTICS[other]["kw"]
                oouts = ctx.stereo_sgm_frames(seq_l, seq_r, D, P1, P2, paths=PATHS, lr=LR, **okw)
                torch.cuda.synchronize()
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
                ctx.stereo_sgm_frames(seq_l, seq_r, D, P1, P2, paths=PATHS, lr=LR, outs=oouts, **okw)
                e1.record(st)
                e1.synchronize()
                sms = e0.elapsed_time(e1) / args.steps
                line[f"semantics_{other}"] = {"recurrence": SEMANTICS[other]["recurrence"],
                                              "path_table": SEMANTICS[other]["table"],
                                              "fps": 1000.0 / sms, "ms_per_step": sms,
                                              "frame_alg_roofline_frac": frame_own / (sms / 1000.0) / 1e9 / peak,
                                              "single_frame": {"fps": 1000.0 / oms, "ms_per_frame": oms},
                                              "kernel_avg_ms": okern}
            except Exception as exc:
                line[f"semantics_{other}"] = {"error": f"{type(exc).__name__}: {exc}"}
        try:
            line["reference_literal"] = measure_reference_literal(ctx, dev, dev_frames, flush)
        except Exception as exc:
            line["reference_literal"] = {"error": f"{type(exc).__name__}: {exc}"}
        try:
            line["configs"] = measure_configs(ctx, dev, args.semantics)
        except Exception as exc:
            line["configs"] = {"error": f"{type(exc).__name__}: {exc}"}
        for key, fn in (("batch", measure_batch), ("soft", measure_soft), ("plain", measure_plain),
                        ("image_stages", measure_image), ("reconstruction", measure_reconstruction),
                        ("video", measure_video)):
            try:
                line[key] = fn(ctx, dev)
            except Exception as exc:  # an extra never hides the headline line
                line[key] = {"error": f"{type(exc).__name__}: {exc}"}
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample(args.semantics)
        line["cpu_baseline"]["band_parity"] = band_parity(ctx, dev, args.semantics)
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
    if args.cpu_matrix:
        cpu_matrix()
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
