"""ctypes binding of the C ABI declared in include/tdv_stereo.h.

The shared library ``libtdvb200.so`` is built in-tree by
``thundervision_b200/csrc/Makefile``; nothing here falls back to another
implementation: if the library is missing or a call fails, an exception is
raised (the reference's stages throw ``CUException``, tdvision/cuerr.hpp:73-78).
"""
import ctypes
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtdvb200.so")
CSRC = os.path.join(_HERE, "csrc")

TDV_OK, TDV_ERR_INVALID_ARG, TDV_ERR_UNSUPPORTED, TDV_ERR_OOM = 0, 1, 2, 3
TDV_ERR_CUDA, TDV_ERR_TIMEOUT, TDV_ERR_BAD_WORK = 4, 5, 6
LAYOUT_REF_WHD, LAYOUT_HWD = 0, 1
F32, U16, U8, F64 = 0, 1, 2, 3
COST_BT, COST_SSD, COST_NCC = 0, 1, 2
SEM_STANDARD, SEM_REF_CPU, SEM_REF_GPU = 0, 1, 2
TABLE_FULL, TABLE_REF = 0, 1
P2_CONST, P2_ADJUST = 0, 1

# every symbol include/tdv_stereo.h declares
EXPORTS = [
    "tdv_cost", "tdv_cost_filtered", "tdv_sgm", "tdv_wta", "tdv_dp_scanline", "tdv_fast_wta", "tdv_stereo_sgm",
    "tdv_ctx_create", "tdv_ctx_destroy", "tdv_ctx_set_allocator", "tdv_ctx_reserve",
    "tdv_last_error_string", "tdv_status_string", "tdv_version", "tdv_volume_bytes",
    "tdv_ctx_enable_timing", "tdv_ctx_timings", "tdv_ctx_timing_name", "tdv_ctx_device_status",
    "tdv_soft_sgm_tape_bytes", "tdv_soft_sgm_forward", "tdv_soft_sgm_backward",
    "tdv_stereo_sgm_static", "tdv_stereo_sgm_frames",
    "tdv_batch_create", "tdv_batch_destroy", "tdv_batch_set_tiles", "tdv_batch_get_tiles",
    "tdv_batch_autotune", "tdv_batch_run", "tdv_batch_graph_launch", "tdv_batch_status",
    "tdv_batch_set_wait_limit", "tdv_batch_set_trace", "tdv_batch_work_queue",
    "tdv_to_gray", "tdv_rectify_maps", "tdv_remap", "tdv_prefilter", "tdv_postfilter", "tdv_subpixel", "tdv_reproject",
    "tdv_write_ply",
]
F32, U16, U8, F64 = 0, 1, 2, 3
FILTER_GAUSS5, FILTER_MEDIAN7 = 0, 1
POST_OPEN7, POST_MEDIAN3 = 0, 1
REPROJECT_DIRECT, REPROJECT_Q = 0, 1
BATCH_ORDER_LONGEST_FIRST, BATCH_ORDER_INPUT = 0, 1


class tdv_image(ctypes.Structure):
    _fields_ = [("ptr", ctypes.c_void_p), ("width", ctypes.c_int32), ("height", ctypes.c_int32),
                ("pitch", ctypes.c_int32), ("dtype", ctypes.c_int32), ("scale", ctypes.c_float)]


class tdv_raster(ctypes.Structure):
    _fields_ = [("ptr", ctypes.c_void_p), ("width", ctypes.c_int32), ("height", ctypes.c_int32),
                ("pitch_bytes", ctypes.c_int32), ("dtype", ctypes.c_int32), ("channels", ctypes.c_int32)]


class tdv_reproject_params(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int32), ("zscale", ctypes.c_float), ("q", ctypes.c_float * 16)]


class tdv_volume(ctypes.Structure):
    _fields_ = [("ptr", ctypes.c_void_p), ("width", ctypes.c_int32), ("height", ctypes.c_int32),
                ("depth", ctypes.c_int32), ("layout", ctypes.c_int32), ("dtype", ctypes.c_int32)]


class tdv_disparity(ctypes.Structure):
    _fields_ = [("disp", ctypes.c_void_p), ("disp_norm", ctypes.c_void_p),
                ("disp_right", ctypes.c_void_p), ("lr_threshold", ctypes.c_int32)]


class tdv_cost_params(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("radius", ctypes.c_int32)]


class tdv_sgm_params(ctypes.Structure):
    _fields_ = [("p1", ctypes.c_float), ("p2", ctypes.c_float), ("p2_mode", ctypes.c_int32),
                ("paths", ctypes.c_int32), ("table", ctypes.c_int32), ("semantics", ctypes.c_int32)]


class tdv_soft_params(ctypes.Structure):
    _fields_ = [("p1", ctypes.c_double), ("p2", ctypes.c_double), ("paths", ctypes.c_int32),
                ("tau", ctypes.c_double), ("checkpoint", ctypes.c_int32)]


class tdv_batch_pair(ctypes.Structure):
    _fields_ = [("left", tdv_image), ("right", tdv_image), ("max_disp", ctypes.c_int32),
                ("out", tdv_disparity)]


class tdv_batch_tiles(ctypes.Structure):
    _fields_ = [("lines_per_cta", ctypes.c_int32), ("rows_per_cta", ctypes.c_int32),
                ("split_disparity", ctypes.c_int32), ("order", ctypes.c_int32),
                ("ctas_per_sm", ctypes.c_int32)]


ALLOC_FN = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p)
FREE_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p)

_lib = None


def build(force=False):
    """Compile libtdvb200.so for sm_100a (nvcc cross-compiles without a GPU)."""
    if force:
        subprocess.check_call(["make", "-s", "-C", CSRC, "clean"])
    subprocess.check_call(["make", "-s", "-C", CSRC])


def _declare(lib):
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    st = ctypes.c_int
    sig = {
        "tdv_cost": (st, [vp, P(tdv_image), P(tdv_image), P(tdv_cost_params), P(tdv_volume), vp]),
        "tdv_cost_filtered": (st, [vp, P(tdv_image), P(tdv_image), P(tdv_cost_params), ctypes.c_int32,
                                   P(tdv_volume), vp, vp]),
        "tdv_sgm": (st, [vp, P(tdv_volume), P(tdv_image), P(tdv_sgm_params), P(tdv_volume),
                         P(tdv_disparity), vp]),
        "tdv_wta": (st, [vp, P(tdv_volume), P(tdv_disparity), vp]),
        "tdv_dp_scanline": (st, [vp, P(tdv_volume), P(tdv_disparity), vp]),
        "tdv_fast_wta": (st, [vp, P(tdv_image), P(tdv_image), ctypes.c_int32, ctypes.c_int32,
                              P(tdv_disparity), vp]),
        "tdv_stereo_sgm": (st, [vp, P(tdv_image), P(tdv_image), ctypes.c_int32, P(tdv_sgm_params),
                                P(tdv_disparity), vp]),
        "tdv_stereo_sgm_static": (st, [P(tdv_image), P(tdv_image), ctypes.c_int32, P(tdv_sgm_params),
                                       P(tdv_disparity), vp]),
        "tdv_stereo_sgm_frames": (st, [vp, ctypes.c_int32, P(tdv_image), P(tdv_image), ctypes.c_int32,
                                       P(tdv_sgm_params), P(tdv_disparity), vp]),
        "tdv_ctx_create": (st, [ctypes.c_int32, P(vp)]),
        "tdv_ctx_destroy": (None, [vp]),
        "tdv_ctx_set_allocator": (st, [vp, ALLOC_FN, FREE_FN, vp]),
        "tdv_ctx_reserve": (st, [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
        "tdv_last_error_string": (ctypes.c_char_p, [vp]),
        "tdv_status_string": (ctypes.c_char_p, [ctypes.c_int]),
        "tdv_version": (ctypes.c_int32, []),
        "tdv_ctx_enable_timing": (st, [vp, ctypes.c_int32]),
        "tdv_ctx_timings": (ctypes.c_int32, [vp, P(ctypes.c_float), ctypes.c_int32]),
        "tdv_ctx_timing_name": (ctypes.c_char_p, [vp, ctypes.c_int32]),
        "tdv_ctx_device_status": (st, [vp, vp]),
        "tdv_volume_bytes": (ctypes.c_size_t, [ctypes.c_int32] * 4),
        "tdv_soft_sgm_tape_bytes": (ctypes.c_size_t, [ctypes.c_int32] * 4 + [P(tdv_soft_params)]),
        "tdv_soft_sgm_forward": (st, [vp, P(tdv_volume), P(tdv_soft_params), vp, vp, ctypes.c_size_t, vp]),
        "tdv_soft_sgm_backward": (st, [vp, P(tdv_volume), P(tdv_soft_params), vp, ctypes.c_size_t, vp,
                                       P(tdv_volume), vp, vp]),
        "tdv_batch_create": (st, [vp, P(tdv_batch_pair), ctypes.c_int32, P(tdv_sgm_params), P(vp)]),
        "tdv_batch_destroy": (None, [vp]),
        "tdv_batch_set_tiles": (st, [vp, P(tdv_batch_tiles)]),
        "tdv_batch_get_tiles": (st, [vp, P(tdv_batch_tiles)]),
        "tdv_batch_autotune": (st, [vp, ctypes.c_int32, vp, P(tdv_batch_tiles), P(ctypes.c_double)]),
        "tdv_batch_run": (st, [vp, vp]),
        "tdv_batch_graph_launch": (st, [vp, vp]),
        "tdv_batch_status": (st, [vp, vp]),
        "tdv_batch_set_wait_limit": (st, [vp, ctypes.c_double]),
        "tdv_batch_set_trace": (st, [vp, vp, ctypes.c_int64]),
        "tdv_batch_work_queue": (st, [vp, P(vp), P(ctypes.c_int32), P(ctypes.c_int32)]),
        "tdv_to_gray": (st, [vp, P(tdv_raster), vp, vp]),
        "tdv_rectify_maps": (st, [vp, vp, vp, vp, vp, ctypes.c_int32, ctypes.c_int32, vp, vp, vp]),
        "tdv_remap": (st, [vp, P(tdv_raster), vp, vp, P(tdv_raster), vp]),
        "tdv_prefilter": (st, [vp, P(tdv_image), ctypes.c_int32, vp, vp]),
        "tdv_postfilter": (st, [vp, P(tdv_raster), ctypes.c_int32, P(tdv_raster), vp]),
        "tdv_subpixel": (st, [vp, P(tdv_volume), vp, vp, vp]),
        "tdv_reproject": (st, [vp, P(tdv_raster), P(tdv_raster), P(tdv_reproject_params), vp, vp, vp]),
        "tdv_write_ply": (st, [ctypes.c_char_p, vp, vp, ctypes.c_int32, ctypes.c_int32]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args


def lib():
    """The loaded C-ABI library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                "libtdvb200.so not built: run thundervision_b200._lib.build() (or make -C "
                "thundervision_b200/csrc)")
        l = ctypes.CDLL(LIB_PATH)
        _declare(l)
        _lib = l
    return _lib


class TdvError(RuntimeError):
    """A non-OK tdv_status (the reference raises tdv::CUException)."""

    def __init__(self, status, message):
        self.status = status
        super().__init__(f"{lib().tdv_status_string(status).decode()}: {message}")
