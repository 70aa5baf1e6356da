"""ctypes binding of the batched analysis (gjxl_b200_batch_*, include/gjxl_b200.h):
many images of uneven sizes, one call, per-image queue / service / ready times."""

from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_float, c_int, c_size_t, c_void_p

import numpy as np

from . import _lib
from .session import AnalysisSession, Options, _bind as _bind_session


class Request(ctypes.Structure):
    _fields_ = [("pixels", c_void_p), ("width", c_size_t), ("height", c_size_t),
                ("row_stride", c_size_t), ("channels", c_int), ("butteraugli_target", c_float)]


class Result(ctypes.Structure):
    _fields_ = [("status", c_int), ("session", c_void_p), ("lane", c_int),
                ("queue_ms", c_double), ("service_ms", c_double), ("ready_ms", c_double)]


def _check(code: int, name: str) -> None:
    if code != 0:
        raise _lib.GjxlB200Error(code, name, _lib.load().gjxl_b200_last_error().decode())


def schedule(pixels, lanes: int, largest_first: bool) -> tuple[np.ndarray, np.ndarray]:
    """The batch's placement rule: (lane of each request, placement order)."""
    px = np.ascontiguousarray(pixels, np.uint64)
    lane_of = np.zeros(px.size, np.int32)
    order = np.zeros(px.size, np.uint64)
    _check(_lib.load().gjxl_b200_batch_schedule(px.size, px.ctypes.data, lanes,
                                                int(largest_first), lane_of.ctypes.data,
                                                order.ctypes.data), "gjxl_b200_batch_schedule")
    return lane_of, order.astype(np.int64)


class BatchAnalyzer:
    """Runs many images per call over `max_in_flight` concurrent lanes."""

    def __init__(self, max_in_flight: int = 0, effort: int = 7, precision: int = 0,
                 tokenize: bool = True, proposal_weights: int = 0, learned_iterations: int = 1):
        _bind_session()
        lib = _lib.load()
        opts = Options()
        lib.gjxl_b200_default_options(ctypes.byref(opts))
        opts.effort = effort
        opts.precision = precision
        opts.tokenize = int(tokenize)
        opts.proposal_weights = proposal_weights or None
        opts.learned_iterations = learned_iterations
        handle = c_void_p()
        _check(lib.gjxl_b200_batch_create(max_in_flight, ctypes.byref(opts), ctypes.byref(handle)),
               "gjxl_b200_batch_create")
        self.handle = handle

    def close(self):
        if self.handle:
            _lib.load().gjxl_b200_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def requests(images) -> ctypes.Array:
        """images: sequence of (pixels pointer, width, height, butteraugli target),
        packed 3-channel rows."""
        arr = (Request * len(images))()
        for r, (ptr, w, h, target) in zip(arr, images):
            r.pixels, r.width, r.height = ptr, w, h
            r.row_stride, r.channels, r.butteraugli_target = 3 * w, 3, target
        return arr

    def set_schedule(self, lanes: int, largest_first: bool):
        _check(_lib.load().gjxl_b200_batch_set_schedule(self.handle, lanes, int(largest_first)),
               "gjxl_b200_batch_set_schedule")

    def analyze(self, requests: ctypes.Array, host_input: bool = False):
        """Returns (per-image dicts, batch milliseconds)."""
        results = (Result * len(requests))()
        ms = c_double()
        _check(_lib.load().gjxl_b200_batch_analyze(self.handle, requests, len(requests),
                                                   int(host_input), results, ctypes.byref(ms)),
               "gjxl_b200_batch_analyze")
        out = [{"status": r.status, "session": r.session, "lane": r.lane,
                "queue_ms": r.queue_ms, "service_ms": r.service_ms, "ready_ms": r.ready_ms}
               for r in results]
        return out, ms.value

    def autotune(self, requests: ctypes.Array, lane_counts=(1, 2, 4, 8)) -> tuple[int, bool]:
        counts = (c_int * len(lane_counts))(*lane_counts)
        lanes, order = c_int(), c_int()
        _check(_lib.load().gjxl_b200_batch_autotune(self.handle, requests, len(requests), counts,
                                                    len(lane_counts), ctypes.byref(lanes),
                                                    ctypes.byref(order)),
               "gjxl_b200_batch_autotune")
        return lanes.value, bool(order.value)

    def device_bytes(self) -> int:
        return int(_lib.load().gjxl_b200_batch_device_bytes(self.handle))

    @staticmethod
    def session(result: dict, width: int, height: int) -> AnalysisSession:
        """Non-owning view of the session that analysed one image."""
        return AnalysisSession.borrow(result["session"], width, height)
