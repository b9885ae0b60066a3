"""Python front end of the C ABI on torch CUDA tensors.

Images are (H, W) uint8 or float32 CUDA tensors (row stride may exceed W);
cost / aggregation volumes are float32 CUDA tensors shaped (H, W, D) for the
HWD layout or (W, H, D) for the reference layout ((x*H)+y)*D+d
(tdvision/dsimem.cpp:34-35).  Every call runs on torch's current stream.
Disparities come back as uint16 (0xFFFF = rejected by the left-right check)
and, on request, float32 d/D -- the reference's output format
(tdvision/wtacpu.cpp:35-36).
"""
import ctypes

import torch

from . import _lib as L

_LAYOUTS = {"hwd": L.LAYOUT_HWD, "ref": L.LAYOUT_REF_WHD, "whd": L.LAYOUT_REF_WHD}
_COSTS = {"bt": L.COST_BT, "ssd": L.COST_SSD, "ncc": L.COST_NCC}
_SEMS = {"standard": L.SEM_STANDARD, "ref_cpu": L.SEM_REF_CPU, "ref_gpu": L.SEM_REF_GPU}
_TABLES = {"full": L.TABLE_FULL, "ref": L.TABLE_REF}
_P2 = {"const": L.P2_CONST, "adjust": L.P2_ADJUST}


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _image(t, scale=1.0):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError("images must be CUDA tensors")
    if t.dim() != 2 or t.stride(1) != 1:
        raise ValueError("images must be (H, W) with unit column stride")
    if t.dtype == torch.uint8:
        dt = L.U8
    elif t.dtype == torch.float32:
        dt = L.F32
    else:
        raise TypeError("images must be uint8 or float32")
    return L.tdv_image(t.data_ptr(), t.shape[1], t.shape[0], t.stride(0), dt, float(scale))


_RASTER_DTYPES = {torch.uint8: (L.U8, 1), torch.uint16: (L.U16, 2), torch.float32: (L.F32, 4)}


def _raster(t):
    """tdv_raster of an (H, W) or (H, W, C) CUDA tensor whose rows may be
    padded but whose pixels and channels are dense."""
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError("rasters must be CUDA tensors")
    if t.dtype not in _RASTER_DTYPES:
        raise TypeError("rasters must be uint8, uint16 or float32")
    dt, size = _RASTER_DTYPES[t.dtype]
    if t.dim() == 2:
        ch = 1
        dense = t.stride(1) == 1
    elif t.dim() == 3:
        ch = t.shape[2]
        dense = t.stride(2) == 1 and t.stride(1) == ch
    else:
        raise ValueError("rasters must be (H, W) or (H, W, C)")
    if not dense:
        raise ValueError("raster pixels must be dense within a row")
    return L.tdv_raster(t.data_ptr(), t.shape[1], t.shape[0], t.stride(0) * size, dt, ch)


_U16_TYPES = (torch.uint16, torch.int16)


def _volume(t, layout):
    """A float32 volume, or a 16-bit cost DSI (uint16 or int16 storage: BT of
    integer intensities in half-units, 0xFFFF = +INF)."""
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype not in (torch.float32,) + _U16_TYPES:
        raise TypeError("volumes must be float32 (or 16-bit cost) CUDA tensors")
    if t.dim() != 3 or not t.is_contiguous():
        raise ValueError("volumes must be contiguous 3-d tensors")
    lay = _LAYOUTS[layout]
    if lay == L.LAYOUT_HWD:
        H, W, D = t.shape
    else:
        W, H, D = t.shape
    return L.tdv_volume(t.data_ptr(), W, H, D, lay, L.U16 if t.dtype in _U16_TYPES else L.F32)


def _vol_dims(t, layout):
    if _LAYOUTS[layout] == L.LAYOUT_HWD:
        H, W, D = t.shape
    else:
        W, H, D = t.shape
    return W, H, D


class Context:
    """Owns a tdv_ctx (scratch buffers, path schedules) for one device."""

    def __init__(self, device=None):
        if device is None:
            device = torch.cuda.current_device()
        self.device = int(device)
        h = ctypes.c_void_p()
        st = L.lib().tdv_ctx_create(self.device, ctypes.byref(h))
        if st != L.TDV_OK:
            raise L.TdvError(st, "tdv_ctx_create")
        self.handle = h
        self._keep = []

    def close(self):
        if self.handle:
            L.lib().tdv_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, status):
        if status != L.TDV_OK:
            msg = L.lib().tdv_last_error_string(self.handle).decode()
            raise L.TdvError(status, msg)

    def device_status(self):
        """Synchronise and raise if a kernel recorded an error (e.g. a timed-out wait)."""
        self.check(L.lib().tdv_ctx_device_status(self.handle, _stream()))

    def reserve(self, W, H, D):
        self.check(L.lib().tdv_ctx_reserve(self.handle, W, H, D))

    def set_allocator(self, alloc, release, user=None):
        a, r = L.ALLOC_FN(alloc), L.FREE_FN(release)
        self._keep += [a, r]
        self.check(L.lib().tdv_ctx_set_allocator(self.handle, a, r, user))

    # ---- outputs --------------------------------------------------------
    def _outputs(self, W, H, dev, norm, right, lr):
        disp = torch.empty((H, W), dtype=torch.uint16, device=dev)
        dn = torch.empty((H, W), dtype=torch.float32, device=dev) if norm else None
        dr = torch.empty((H, W), dtype=torch.uint16, device=dev) if right else None
        o = L.tdv_disparity(disp.data_ptr(), dn.data_ptr() if dn is not None else None,
                            dr.data_ptr() if dr is not None else None,
                            -1 if lr is None else int(lr))
        return o, disp, dn, dr

    @staticmethod
    def _result(disp, dn, dr):
        out = {"disp": disp}
        if dn is not None:
            out["disp_norm"] = dn
        if dr is not None:
            out["disp_right"] = dr
        return out

    # ---- stages ---------------------------------------------------------
    def cost(self, left, right, max_disp, kind="bt", radius=None, layout="hwd", scale=1.0,
             out=None, dtype="f32"):
        """Matching-cost DSI (BirchfieldCostRun / SSDDevRun / CrossCorrelationDevRun).
        ``dtype="u16"``: BT of uint8 images at scale 1 as a 16-bit DSI in
        half-units (0xFFFF = +INF), exact and half the bytes."""
        if radius is None:
            radius = {"bt": 0, "ssd": 3, "ncc": 1}[kind]
        H = min(left.shape[0], right.shape[0])
        W = min(left.shape[1], right.shape[1])
        if out is None:
            shape = (H, W, max_disp) if _LAYOUTS[layout] == L.LAYOUT_HWD else (W, H, max_disp)
            out = torch.empty(shape, dtype=torch.uint16 if dtype == "u16" else torch.float32, device=left.device)
        li, ri = _image(left, scale), _image(right, scale)
        vol = _volume(out, layout)
        p = L.tdv_cost_params(_COSTS[kind], radius)
        self.check(L.lib().tdv_cost(self.handle, ctypes.byref(li), ctypes.byref(ri), ctypes.byref(p),
                                    ctypes.byref(vol), _stream()))
        return out

    def cost_filtered(self, left, right, max_disp, kind="bt", radius=None, layout="hwd", scale=1.0,
                      prefilter="gauss5", out=None, left_filtered=True):
        """Cost DSI of the pre-filtered pair, DevStereoMatcher's default chain
        (the 5x5 Gaussian fused into the cost kernel): bit-identical to
        ``cost(prefilter(left), prefilter(right))``.  Returns (DSI, filtered
        left image of the DSI's size, or None)."""
        if radius is None:
            radius = {"bt": 0, "ssd": 3, "ncc": 1}[kind]
        f = {"gauss5": L.FILTER_GAUSS5, "median7": L.FILTER_MEDIAN7}[prefilter]
        H = min(left.shape[0], right.shape[0])
        W = min(left.shape[1], right.shape[1])
        if out is None:
            shape = (H, W, max_disp) if _LAYOUTS[layout] == L.LAYOUT_HWD else (W, H, max_disp)
            out = torch.empty(shape, dtype=torch.float32, device=left.device)
        fl = torch.empty((H, W), dtype=torch.float32, device=left.device) if left_filtered else None
        li, ri = _image(left, scale), _image(right, scale)
        vol = _volume(out, layout)
        p = L.tdv_cost_params(_COSTS[kind], radius)
        self.check(L.lib().tdv_cost_filtered(self.handle, ctypes.byref(li), ctypes.byref(ri), ctypes.byref(p), f,
                                             ctypes.byref(vol), fl.data_ptr() if fl is not None else None,
                                             _stream()))
        return out, fl

    def sgm(self, cost, p1, p2, guide=None, guide_scale=1.0, p2_mode="const", paths=8,
            table="full", semantics="standard", layout="hwd", lr=None, norm=False, right=False,
            aggreg=None):
        """SGM aggregation + WTA (SemiGlobalDevRun / SemiGlobalCPU::updateImpl)."""
        W, H, D = _vol_dims(cost, layout)
        cv = _volume(cost, layout)
        gi = _image(guide, guide_scale) if guide is not None else None
        prm = L.tdv_sgm_params(p1, p2, _P2[p2_mode], paths, _TABLES[table], _SEMS[semantics])
        av = _volume(aggreg, layout) if aggreg is not None else None
        o, disp, dn, dr = self._outputs(W, H, cost.device, norm, right, lr)
        self.check(L.lib().tdv_sgm(self.handle, ctypes.byref(cv),
                                   ctypes.byref(gi) if gi is not None else None, ctypes.byref(prm),
                                   ctypes.byref(av) if av is not None else None, ctypes.byref(o),
                                   _stream()))
        return self._result(disp, dn, dr)

    def wta(self, vol, layout="hwd", norm=False, lr=None, right=False):
        """Winner-take-all (WTARunDev / WTACPU::wta)."""
        W, H, D = _vol_dims(vol, layout)
        v = _volume(vol, layout)
        o, disp, dn, dr = self._outputs(W, H, vol.device, norm, right, lr)
        self.check(L.lib().tdv_wta(self.handle, ctypes.byref(v), ctypes.byref(o), _stream()))
        return self._result(disp, dn, dr)

    def dp(self, cost, layout="hwd", norm=False):
        """Dynamic-programming scanline matcher (DynamicProgDevRun)."""
        W, H, D = _vol_dims(cost, layout)
        v = _volume(cost, layout)
        o, disp, dn, dr = self._outputs(W, H, cost.device, norm, False, None)
        self.check(L.lib().tdv_dp_scanline(self.handle, ctypes.byref(v), ctypes.byref(o), _stream()))
        return self._result(disp, dn, dr)

    def fast_wta(self, left, right, max_disp, radius=3, scale=1.0, norm=False):
        """SSD window + WTA without a DSI (FastWTADevRun)."""
        H, W = left.shape
        li, ri = _image(left, scale), _image(right, scale)
        o, disp, dn, dr = self._outputs(W, H, left.device, norm, False, None)
        self.check(L.lib().tdv_fast_wta(self.handle, ctypes.byref(li), ctypes.byref(ri), max_disp,
                                        radius, ctypes.byref(o), _stream()))
        return self._result(disp, dn, dr)

    # ---- image stages either side of the path ------------------------
    def to_gray(self, color):
        """(H, W, 3) uint8 -> (H, W) float32 grey in [0, 1] (channel 0 weighted
        as red, as tdvision/misc.cpp:29-32 converts its frames)."""
        out = torch.empty(color.shape[:2], dtype=torch.float32, device=color.device)
        self.check(L.lib().tdv_to_gray(self.handle, ctypes.byref(_raster(color)), out.data_ptr(), _stream()))
        return out

    def rectify_maps(self, K, dist, R, P, width, height, device=None):
        """Rectification maps ((H, W) float32 mapx, mapy) of one camera from
        its intrinsics K (3x3), distortion (k1, k2, p1, p2, k3[, k4, k5, k6]),
        rectifying rotation R (3x3) and new camera P (3x3 or 3x4)."""
        import numpy as np
        K = np.ascontiguousarray(np.asarray(K, np.float64).reshape(3, 3))
        R = np.ascontiguousarray(np.asarray(R, np.float64).reshape(3, 3))
        P = np.ascontiguousarray(np.asarray(P, np.float64).reshape(3, -1)[:, :3])
        d = np.zeros(8)
        d[:len(dist)] = np.asarray(dist, np.float64)
        dev = torch.device("cuda", self.device) if device is None else device
        mx = torch.empty((height, width), dtype=torch.float32, device=dev)
        my = torch.empty((height, width), dtype=torch.float32, device=dev)
        self.check(L.lib().tdv_rectify_maps(self.handle, K.ctypes.data, d.ctypes.data, R.ctypes.data, P.ctypes.data,
                                            width, height, mx.data_ptr(), my.data_ptr(), _stream()))
        return mx, my

    def remap(self, src, mapx, mapy):
        """Rectification remap: src sampled bilinearly at (mapx, mapy), the
        maps (H, W) float32 of the output's size; src (H', W') or (H', W', 3),
        uint8 or float32."""
        if mapx.shape != mapy.shape or mapx.dtype != torch.float32 or mapy.dtype != torch.float32:
            raise ValueError("maps must be float32 of one shape")
        mapx, mapy = mapx.contiguous(), mapy.contiguous()
        out = torch.empty(tuple(mapx.shape) + tuple(src.shape[2:]), dtype=src.dtype, device=src.device)
        self.check(L.lib().tdv_remap(self.handle, ctypes.byref(_raster(src)), mapx.data_ptr(), mapy.data_ptr(),
                                     ctypes.byref(_raster(out)), _stream()))
        return out

    def prefilter(self, img, kind="gauss5", scale=1.0):
        """Pre-filter before the cost: "gauss5" (DevStereoMatcher's default
        5x5 Gaussian) or "median7"; returns (H, W) float32 of value * scale."""
        k = {"gauss5": L.FILTER_GAUSS5, "median7": L.FILTER_MEDIAN7}[kind]
        out = torch.empty(img.shape, dtype=torch.float32, device=img.device)
        self.check(L.lib().tdv_prefilter(self.handle, ctypes.byref(_image(img, scale)), k, out.data_ptr(),
                                         _stream()))
        return out

    def postfilter(self, disp, kind="open7"):
        """Disparity clean-up: "open7" (the reference's erode + dilate) or
        "median3"; float32 or uint16 maps."""
        k = {"open7": L.POST_OPEN7, "median3": L.POST_MEDIAN3}[kind]
        out = torch.empty_like(disp)
        self.check(L.lib().tdv_postfilter(self.handle, ctypes.byref(_raster(disp)), k, ctypes.byref(_raster(out)),
                                          _stream()))
        return out

    def subpixel(self, S, disp):
        """Parabola sub-pixel refinement of a uint16 disparity map from the
        aggregated volume S ((H, W, D) float32)."""
        out = torch.empty(disp.shape, dtype=torch.float32, device=disp.device)
        self.check(L.lib().tdv_subpixel(self.handle, ctypes.byref(_volume(S, "hwd")), disp.contiguous().data_ptr(),
                                        out.data_ptr(), _stream()))
        return out

    def reproject(self, disp, color=None, mode="direct", zscale=1.0, q=None):
        """One vertex per pixel ((H, W, 3) float32) and, with a (H, W, 3)
        uint8 color image, its color in [0, 1]; mode "direct" or "q" (q: 16
        floats, row-major)."""
        prm = L.tdv_reproject_params()
        prm.mode = {"direct": L.REPROJECT_DIRECT, "q": L.REPROJECT_Q}[mode]
        prm.zscale = float(zscale)
        qq = [1.0 if i % 5 == 0 else 0.0 for i in range(16)] if q is None else [float(v) for v in q]
        if len(qq) != 16:
            raise ValueError("q must hold 16 values")
        for i, v in enumerate(qq):
            prm.q[i] = v
        H, W = disp.shape
        verts = torch.empty((H, W, 3), dtype=torch.float32, device=disp.device)
        cols = torch.empty((H, W, 3), dtype=torch.float32, device=disp.device) if color is not None else None
        craster = ctypes.byref(_raster(color)) if color is not None else None
        self.check(L.lib().tdv_reproject(self.handle, ctypes.byref(_raster(disp)), craster, ctypes.byref(prm),
                                         verts.data_ptr(), cols.data_ptr() if cols is not None else None,
                                         _stream()))
        return verts, cols

    def kernel_times(self, fn):
        """Runs fn() with per-kernel timing on (tdv_ctx_enable_timing) and
        returns [(kernel name, device ms)] of the last ABI call fn made."""
        self.check(L.lib().tdv_ctx_enable_timing(self.handle, 1))
        try:
            fn()
            torch.cuda.synchronize()
            buf = (ctypes.c_float * 256)()
            n = L.lib().tdv_ctx_timings(self.handle, buf, 256)
            return [(L.lib().tdv_ctx_timing_name(self.handle, i).decode(), buf[i]) for i in range(n)]
        finally:
            L.lib().tdv_ctx_enable_timing(self.handle, 0)

    def stereo_sgm(self, left, right, max_disp, p1, p2, paths=8, p2_mode="const", table="full",
                   semantics="standard", scale=1.0, lr=None, norm=False, right_disp=False):
        """BT + SGM + WTA with the cost recomputed inside the aggregation."""
        H, W = left.shape
        li, ri = _image(left, scale), _image(right, scale)
        prm = L.tdv_sgm_params(p1, p2, _P2[p2_mode], paths, _TABLES[table], _SEMS[semantics])
        o, disp, dn, dr = self._outputs(W, H, left.device, norm, right_disp, lr)
        self.check(L.lib().tdv_stereo_sgm(self.handle, ctypes.byref(li), ctypes.byref(ri), max_disp,
                                          ctypes.byref(prm), ctypes.byref(o), _stream()))
        return self._result(disp, dn, dr)

    def stereo_sgm_frames(self, lefts, rights, max_disp, p1, p2, paths=8, table="full", semantics="standard",
                          lr=None, norm=False, right_disp=False, outs=None):
        """``stereo_sgm``'s fused path over a sequence of equal-size uint8
        frame pairs (tdv_stereo_sgm_frames): consecutive frames run on two
        lanes, so one frame's passes overlap the other's last pass.  Returns
        one result dict per frame; ``outs`` (the dicts a previous call
        returned) are written again instead of allocating new maps."""
        n = len(lefts)
        if n != len(rights) or n == 0:
            raise ValueError("need as many right frames as left frames, at least one")
        H, W = lefts[0].shape
        li = (L.tdv_image * n)(*[_image(x) for x in lefts])
        ri = (L.tdv_image * n)(*[_image(x) for x in rights])
        prm = L.tdv_sgm_params(p1, p2, L.P2_CONST, paths, _TABLES[table], _SEMS[semantics])
        oa = (L.tdv_disparity * n)()
        results = []
        for i in range(n):
            if outs is not None:
                r = outs[i]
                dn, dr = r.get("disp_norm"), r.get("disp_right")
                oa[i] = L.tdv_disparity(r["disp"].data_ptr(), dn.data_ptr() if dn is not None else None,
                                        dr.data_ptr() if dr is not None else None, -1 if lr is None else int(lr))
                results.append(r)
            else:
                o, disp, dn, dr = self._outputs(W, H, lefts[i].device, norm, right_disp, lr)
                oa[i] = o
                results.append(self._result(disp, dn, dr))
        self.check(L.lib().tdv_stereo_sgm_frames(self.handle, n, li, ri, max_disp, ctypes.byref(prm), oa,
                                                 _stream()))
        return results


class Batch:
    """Many uint8 pairs of uneven size and disparity range aggregated by one
    persistent launch (tdv_batch_*): BT + SGM + WTA (+ left-right check) with
    results bit-identical to per-pair ``Context.stereo_sgm`` calls.

    ``pairs`` is a list of ``(left, right, max_disp)`` or
    ``(left, right, max_disp, lr)`` with (H, W) uint8 CUDA tensors; the
    tensors are kept alive and read again by every run, so a video loop
    copies new frames into them and relaunches.  ``outputs[i]`` holds pair
    i's result tensors (rewritten by every run).  ``right_disp``: False, True,
    or "lr" (right-view maps for the pairs that run the left-right check).
    """

    def __init__(self, ctx, pairs, p1, p2, paths=8, lr=None, norm=False, right_disp=False):
        self.ctx = ctx
        self.handle = None
        n = len(pairs)
        arr = (L.tdv_batch_pair * n)()
        self.outputs = []
        self._inputs = []
        for i, pr in enumerate(pairs):
            left, right, D = pr[0], pr[1], int(pr[2])
            lr_i = pr[3] if len(pr) > 3 else lr
            H, W = left.shape
            want_right = (lr_i is not None) if right_disp == "lr" else bool(right_disp)
            o, disp, dn, dr = ctx._outputs(W, H, left.device, norm, want_right, lr_i)
            arr[i] = L.tdv_batch_pair(_image(left), _image(right), D, o)
            self.outputs.append(Context._result(disp, dn, dr))
            self._inputs.append((left, right))
        prm = L.tdv_sgm_params(p1, p2, L.P2_CONST, paths, L.TABLE_FULL, L.SEM_STANDARD)
        h = ctypes.c_void_p()
        ctx.check(L.lib().tdv_batch_create(ctx.handle, arr, n, ctypes.byref(prm), ctypes.byref(h)))
        self.handle = h

    def close(self):
        if self.handle:
            L.lib().tdv_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self):
        """One persistent launch on torch's current stream."""
        self.ctx.check(L.lib().tdv_batch_run(self.handle, _stream()))
        return self.outputs

    def trace(self):
        """One run with the per-item trace on (tdv_batch_set_trace); returns
        an (n_items, 4) int64 CPU tensor: global-timer ns when a block took
        the item, when its dependency was met, when it ended, and
        smid << 32 | (pair * 16 + pass)."""
        n = self.work_queue()[1]
        buf = torch.zeros((n, 4), dtype=torch.int64, device="cuda")
        self.ctx.check(L.lib().tdv_batch_set_trace(self.handle, buf.data_ptr(), n))
        try:
            self.run()
            self.status()
        finally:
            self.ctx.check(L.lib().tdv_batch_set_trace(self.handle, None, 0))
        return buf.cpu()

    def graph_launch(self):
        """The same run replayed from a CUDA graph (captured on first use)."""
        self.ctx.check(L.lib().tdv_batch_graph_launch(self.handle, _stream()))
        return self.outputs

    def status(self):
        """Synchronise; raise TdvError if the last run recorded a device error."""
        self.ctx.check(L.lib().tdv_batch_status(self.handle, _stream()))

    @property
    def tiles(self):
        t = L.tdv_batch_tiles()
        self.ctx.check(L.lib().tdv_batch_get_tiles(self.handle, ctypes.byref(t)))
        return {f: getattr(t, f) for f, _ in L.tdv_batch_tiles._fields_}

    def set_tiles(self, **kw):
        cur = self.tiles
        cur.update(kw)
        t = L.tdv_batch_tiles(**cur)
        self.ctx.check(L.lib().tdv_batch_set_tiles(self.handle, ctypes.byref(t)))

    def autotune(self, reps=3):
        """Time candidate tile shapes, keep the fastest; returns (tiles, ms)."""
        t = L.tdv_batch_tiles()
        ms = ctypes.c_double()
        self.ctx.check(L.lib().tdv_batch_autotune(self.handle, reps, _stream(), ctypes.byref(t),
                                                  ctypes.byref(ms)))
        return {f: getattr(t, f) for f, _ in L.tdv_batch_tiles._fields_}, ms.value

    def set_wait_limit(self, seconds):
        self.ctx.check(L.lib().tdv_batch_set_wait_limit(self.handle, float(seconds)))

    def work_queue(self):
        """(device pointer, item count, bytes per item) of the work queue."""
        p = ctypes.c_void_p()
        n = ctypes.c_int32()
        b = ctypes.c_int32()
        self.ctx.check(L.lib().tdv_batch_work_queue(self.handle, ctypes.byref(p), ctypes.byref(n),
                                                    ctypes.byref(b)))
        return p.value, n.value, b.value


_default = {}


def default_context(device=None):
    if device is None:
        device = torch.cuda.current_device()
    if device not in _default:
        _default[device] = Context(device)
    return _default[device]


def write_ply(path, vertices, colors=None):
    """Writes a grid mesh ((H, W, 3) float32 vertices, optional (H, W, 3)
    float32 colors in [0, 1], host or device tensors) as the reference's
    ASCII PLY (tdvision/plymeshexporter.cpp:8-76)."""
    v = vertices.detach().to("cpu", torch.float32).contiguous()
    c = colors.detach().to("cpu", torch.float32).contiguous() if colors is not None else None
    H, W = v.shape[0], v.shape[1]
    st = L.lib().tdv_write_ply(str(path).encode(), v.data_ptr(), c.data_ptr() if c is not None else None, W, H)
    if st != L.TDV_OK:
        raise L.TdvError(st, f"writing {path}")
