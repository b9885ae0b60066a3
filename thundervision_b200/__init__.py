"""B200 (sm_100a) dense-stereo hot path of LibThunderVision: matching-cost DSI
-> SGM / DP aggregation -> WTA, behind the C ABI in include/tdv_stereo.h.

The compute runs only in libtdvb200.so (hand-written CUDA); this package is
its Python front end.  ``Context`` wraps one tdv_ctx (``api``); ``Batch``
runs many pairs per launch; ``video`` streams frames through graph replays;
``soft`` is the differentiable SGM; ``reconstruction`` chains the stages
either side of the matcher as the reference's Reconstruction does.  The C++
stage classes mirroring the reference's plugins are in include/tdv_stages.hpp.
"""
from ._lib import TdvError, build, lib  # noqa: F401

__all__ = ["TdvError", "build", "lib", "Context", "Batch", "default_context"]


def __getattr__(name):
    # torch is imported lazily so that the ABI layer loads without it
    if name in ("Context", "Batch", "default_context"):
        from . import api
        return getattr(api, name)
    raise AttributeError(name)
