"""Python wrapper of the analysis session (gjxl_b200_session_* in the C ABI).

The session owns its device buffers; analyses run on the current torch CUDA
stream (or an explicit stream handle).
"""

from __future__ import annotations

import ctypes
from ctypes import POINTER, Structure, c_float, c_int, c_size_t, c_uint8, c_void_p

import numpy as np

from . import _lib


class Options(Structure):
    _fields_ = [("struct_size", c_size_t), ("butteraugli_target", c_float), ("effort", c_int),
                ("intensity_target", c_float), ("profile_stages", c_int), ("tokenize", c_int),
                ("order_mode", c_int), ("precision", c_int), ("proposal_weights", c_void_p),
                ("learned_iterations", c_int), ("proposal_confidence", c_float)]


class Outputs(Structure):
    _fields_ = [(n, c_size_t) for n in ("padded_width", "padded_height", "blocks_x", "blocks_y",
                                        "tiles_x", "tiles_y", "iterations")] + [
        ("linear", c_void_p), ("linear_stride", c_size_t), ("linear_plane_pitch", c_size_t),
        ("opsin", c_void_p), ("preprocessed_opsin", c_void_p), ("opsin_stride", c_size_t),
        ("opsin_plane_pitch", c_size_t)] + [(n, c_void_p) for n in (
            "initial_quant_field", "strategy_mask", "pixel_mask", "initial_y_to_x",
            "initial_y_to_b", "strategy_cells", "matrix_scale_stats", "matrix_scales",
            "quant_field", "adjusted_quant_field", "proposals", "proposal_mass",
            "proposal_log_scale", "tile_family_masks",
            "raw_quant_field", "y_to_x", "y_to_b", "quantized_ac", "quantized_dc",
            "dc", "block_distance", "reconstructed_linear", "distance_map", "score_history",
            "quantizer_params", "device_error", "host_strategy_cells",
            "host_initial_quant_field", "host_y_to_x", "host_y_to_b", "host_matrix_scale_stats",
            "host_device_error", "host_quant_field", "host_raw_quant_field", "host_quantized_dc",
            "host_score_history", "host_quantizer_params", "host_quantized_ac")] + [
        ("groups", c_size_t)] + [(n, c_void_p) for n in (
            "token_values", "token_contexts", "group_offsets", "token_histogram", "scans",
            "order_masks", "host_token_values", "host_token_contexts", "host_group_offsets")] + [
        ("host_token_count", c_size_t), ("device_bytes", c_size_t),
        ("input_pixels", c_void_p), ("input_capacity", c_size_t), ("graph_replay", c_int),
        ("pnorm_history", c_void_p), ("host_pnorm_history", c_void_p),
        ("dc_groups", c_size_t), ("dc_tokens", c_void_p), ("meta_tokens", c_void_p),
        ("dc_group_info", c_void_p), ("dc_histogram", c_void_p), ("host_dc_tokens", c_void_p),
        ("host_meta_tokens", c_void_p), ("host_dc_group_info", c_void_p),
        ("host_dc_histogram", c_void_p), ("host_meta_token_count", c_size_t)]


_BOUND = False


def _bind():
    global _BOUND
    if _BOUND:
        return
    lib = _lib.load()
    lib.gjxl_b200_default_options.argtypes = [POINTER(Options)]
    lib.gjxl_b200_default_options.restype = None
    lib.gjxl_b200_session_create.argtypes = [c_size_t, c_size_t, POINTER(Options),
                                             POINTER(c_void_p)]
    lib.gjxl_b200_session_create.restype = c_int
    lib.gjxl_b200_session_destroy.argtypes = [c_void_p]
    lib.gjxl_b200_session_destroy.restype = None
    lib.gjxl_b200_session_set_butteraugli_target.argtypes = [c_void_p, c_float]
    lib.gjxl_b200_session_set_butteraugli_target.restype = c_int
    lib.gjxl_b200_session_analyze.argtypes = [c_void_p, c_void_p, c_size_t, c_int, c_void_p]
    lib.gjxl_b200_session_analyze.restype = c_int
    lib.gjxl_b200_session_analyze_host.argtypes = [c_void_p, c_void_p, c_size_t, c_int, c_void_p]
    lib.gjxl_b200_session_analyze_host.restype = c_int
    lib.gjxl_b200_session_outputs.argtypes = [c_void_p, POINTER(Outputs)]
    lib.gjxl_b200_session_outputs.restype = c_int
    lib.gjxl_b200_session_stage_times.argtypes = [c_void_p, POINTER(c_float), c_int]
    lib.gjxl_b200_session_stage_times.restype = c_int
    lib.gjxl_b200_stage_name.argtypes = [c_int]
    lib.gjxl_b200_stage_name.restype = ctypes.c_char_p
    lib.gjxl_b200_session_kernel_count.argtypes = [c_void_p, c_void_p, c_size_t, c_int,
                                                   POINTER(c_size_t)]
    lib.gjxl_b200_session_kernel_count.restype = c_int
    _BOUND = True


def _check(code: int, name: str) -> int:
    if code < 0 or code > 0 and name != "gjxl_b200_session_stage_times":
        raise _lib.GjxlB200Error(code, name, _lib.load().gjxl_b200_last_error().decode())
    return code


class AnalysisSession:
    """Runs the B200 analysis path for images of one extent."""

    def __init__(self, width: int, height: int, butteraugli_target: float = 1.0,
                 effort: int = 7, intensity_target: float = 255.0, profile_stages: bool = False,
                 tokenize: bool = True, order_mode: int = -1, precision: int = 0,
                 proposal_weights: int = 0, learned_iterations: int = 1,
                 proposal_confidence: float = 0.6):
        _bind()
        lib = _lib.load()
        opts = Options()
        lib.gjxl_b200_default_options(ctypes.byref(opts))
        opts.butteraugli_target = butteraugli_target
        opts.effort = effort
        opts.intensity_target = intensity_target
        opts.profile_stages = int(profile_stages)
        opts.tokenize = int(tokenize)
        opts.order_mode = order_mode
        opts.precision = precision
        opts.proposal_weights = proposal_weights or None
        opts.learned_iterations = learned_iterations
        opts.proposal_confidence = proposal_confidence
        handle = c_void_p()
        _check(lib.gjxl_b200_session_create(width, height, ctypes.byref(opts),
                                            ctypes.byref(handle)), "gjxl_b200_session_create")
        self.handle = handle
        self.width, self.height = width, height
        self.outputs = Outputs()
        _check(lib.gjxl_b200_session_outputs(handle, ctypes.byref(self.outputs)),
               "gjxl_b200_session_outputs")

    @classmethod
    def borrow(cls, handle: int, width: int, height: int) -> "AnalysisSession":
        """A non-owning view of a session that another object owns (a batch's
        pooled sessions); close() leaves it alone."""
        _bind()
        self = cls.__new__(cls)
        self.handle = None
        self._borrowed = c_void_p(handle)
        self.width, self.height = width, height
        self.outputs = Outputs()
        _check(_lib.load().gjxl_b200_session_outputs(self._borrowed, ctypes.byref(self.outputs)),
               "gjxl_b200_session_outputs")
        return self

    def set_butteraugli_target(self, target: float):
        """Retargets later analyses; every buffer is kept."""
        _check(_lib.load().gjxl_b200_session_set_butteraugli_target(self.handle, target),
               "gjxl_b200_session_set_butteraugli_target")

    def close(self):
        if self.handle:
            _lib.load().gjxl_b200_session_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def analyze(self, device_pixels_ptr: int, row_stride: int, channels: int, stream: int = 0):
        lib = _lib.load()
        _check(lib.gjxl_b200_session_analyze(self.handle, device_pixels_ptr, row_stride,
                                             channels, stream),
               "gjxl_b200_session_analyze")
        _check(lib.gjxl_b200_session_outputs(self.handle, ctypes.byref(self.outputs)),
               "gjxl_b200_session_outputs")

    def kernel_count(self, device_pixels_ptr: int, row_stride: int, channels: int) -> int:
        """Kernels one analyze() call on these arguments launches (counted
        from a captured graph; nothing executes)."""
        count = c_size_t()
        _check(_lib.load().gjxl_b200_session_kernel_count(self.handle, device_pixels_ptr,
                                                          row_stride, channels,
                                                          ctypes.byref(count)),
               "gjxl_b200_session_kernel_count")
        return int(count.value)

    def analyze_host(self, host_pixels: np.ndarray, stream: int = 0):
        assert host_pixels.dtype == np.uint8 and host_pixels.flags["C_CONTIGUOUS"]
        h, w, ch = host_pixels.shape
        lib = _lib.load()
        _check(lib.gjxl_b200_session_analyze_host(self.handle, host_pixels.ctypes.data,
                                                  w * ch, ch, stream),
               "gjxl_b200_session_analyze_host")
        _check(lib.gjxl_b200_session_outputs(self.handle, ctypes.byref(self.outputs)),
               "gjxl_b200_session_outputs")

    def stage_times(self) -> dict[str, float]:
        lib = _lib.load()
        buf = (c_float * 32)()
        n = lib.gjxl_b200_session_stage_times(self.handle, buf, 32)
        if n < 0 or n > 32:
            raise _lib.GjxlB200Error(n, "stage_times", lib.gjxl_b200_last_error().decode())
        if n == 0:
            return {}
        return {lib.gjxl_b200_stage_name(i).decode(): float(buf[i]) for i in range(n)}

    # Host views of the results of analyze_host (valid after the stream completes).
    def host_strategy_cells(self) -> np.ndarray:
        o = self.outputs
        return np.ctypeslib.as_array(ctypes.cast(o.host_strategy_cells, POINTER(c_uint8)),
                                     shape=(o.blocks_y, o.blocks_x)).copy()

    def _host(self, name: str, ctype, shape) -> np.ndarray:
        ptr = ctypes.cast(getattr(self.outputs, name), POINTER(ctype))
        return np.ctypeslib.as_array(ptr, shape=shape).copy()

    def host_error(self) -> int:
        """Analysis error word OR'ed with the Butteraugli error word."""
        words = self._host("host_device_error", ctypes.c_uint32, (3,))
        return int(words[0]) | int(words[1]) | int(words[2])

    def host_results(self) -> dict[str, np.ndarray]:
        """Host copies of the final frame's results (after analyze_host)."""
        o = self.outputs
        blocks = (o.blocks_y, o.blocks_x)
        tiles = (o.tiles_y, o.tiles_x)
        return {
            "cells": self.host_strategy_cells(),
            "initial_quant": self._host("host_initial_quant_field", c_float, blocks),
            "y_to_x": self._host("host_y_to_x", ctypes.c_int8, tiles),
            "y_to_b": self._host("host_y_to_b", ctypes.c_int8, tiles),
            "final_quant": self._host("host_quant_field", c_float, blocks),
            "raw_quant": self._host("host_raw_quant_field", ctypes.c_int32, blocks),
            "quantized_dc": self._host("host_quantized_dc", ctypes.c_int32, (3,) + blocks),
            "score_history": self._host("host_score_history", ctypes.c_double,
                                        (o.iterations + 1,)),
            "pnorm_history": self._host("host_pnorm_history", ctypes.c_double,
                                        (o.iterations + 1,)),
            "quantizer_params": self._host("host_quantizer_params", ctypes.c_uint32, (2,)),
        } | self.host_tokens() | ({} if o.host_token_values else {
            "quantized_ac": self._host("host_quantized_ac", ctypes.c_int32,
                                       (3, o.padded_height, o.padded_width))})

    def host_tokens(self) -> dict[str, np.ndarray]:
        """AC tokens of the last analyze_host (empty without tokenization)."""
        o = self.outputs
        if not o.host_token_values:
            return {}
        n = o.host_token_count
        blocks = o.blocks_x * o.blocks_y
        return {
            "token_values": self._host("host_token_values", ctypes.c_uint32, (n,)),
            "token_contexts": self._host("host_token_contexts", ctypes.c_uint16, (n,)),
            "group_offsets": self._host("host_group_offsets", ctypes.c_uint32, (o.groups + 1,)),
            # DC-group streams: (context, value) pairs and the group table.
            "dc_tokens": self._host("host_dc_tokens", ctypes.c_uint32, (3 * blocks, 2)),
            "meta_tokens": self._host("host_meta_tokens", ctypes.c_uint32,
                                      (o.host_meta_token_count, 2)),
            "dc_group_info": self._host("host_dc_group_info", ctypes.c_uint32, (o.dc_groups, 5)),
            "dc_histogram": self._host("host_dc_histogram", ctypes.c_uint32, (45, 128)),
        }
