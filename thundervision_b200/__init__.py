"""B200 (sm_100a) dense-stereo hot path of LibThunderVision: matching-cost DSI
-> SGM / DP aggregation -> WTA, behind the C ABI in include/tdv_stereo.h.

The compute runs only in libtdvb200.so (hand-written CUDA); this package is
its Python front end.  ``Context`` wraps one tdv_ctx; ``stages`` mirrors the
reference's MatchingCost / Optimizer plugin classes.
"""
from ._lib import TdvError, build, lib  # noqa: F401

__all__ = ["TdvError", "build", "lib", "Context", "Batch", "default_context"]


def __getattr__(name):
    # torch is imported lazily so that the ABI layer loads without it
    if name in ("Context", "Batch", "default_context"):
        from . import api
        return getattr(api, name)
    raise AttributeError(name)
