"""numpy-facing wrapper of oracle/_ref/libgjxl_ref.so (the reference's own CPU
analysis code built from its sources by oracle/Makefile, see ref_shim.cpp).

Test infrastructure only (the checker and the timed CPU baseline).
"""

from __future__ import annotations

import ctypes
from ctypes import c_double, c_float, c_int, c_size_t, c_void_p
from pathlib import Path

import numpy as np

LIBRARY_PATH = Path(__file__).resolve().parent / "_ref" / "libgjxl_ref.so"

_P, _Z, _F, _I = c_void_p, c_size_t, c_float, c_int
_SIGNATURES = {
    "gjxl_ref_entropy_build": [_I, _P, _P, _P, _Z, ctypes.c_uint32, ctypes.c_uint32, _P],
    "gjxl_ref_entropy_free": [_P],
    "gjxl_ref_entropy_info": [_P, _P, _P, _P],
    "gjxl_ref_entropy_tables": [_P] * 9,
    "gjxl_ref_entropy_write": [_P, _P, _P, _P, _Z, _P, _Z, _P, _P],
    "gjxl_ref_entropy_count": [_P, _P, _P, _P, _Z, _P],
    "gjxl_ref_srgb8_to_linear": [_P, _Z, _Z, _Z, _I, _P],
    "gjxl_ref_linear_to_padded_opsin": [_P, _Z, _Z, _P, _Z, _Z, _F],
    "gjxl_ref_opsin_to_linear": [_P, _Z, _Z, _F, _P],
    "gjxl_ref_initial_quant_field": [_P, _Z, _Z, _F, _F, _I, _P, _P, _P],
    "gjxl_ref_gaborish_inverse": [_P, _Z, _Z, _P, _P],
    "gjxl_ref_gaborish": [_P, _Z, _Z, _P],
    "gjxl_ref_initial_cfl": [_P, _Z, _Z, _I, _P, _P],
    "gjxl_ref_ac_strategy_cost": [_P, _Z, _Z, _P, _P, _I, _Z, _Z, _F, _F, _P, _P],
    "gjxl_ref_ac_strategy_search": [_P, _Z, _Z, _P, _P, _P, _P, _F, _I, _P],
    "gjxl_ref_butteraugli": [_P, _P, _Z, _Z, _F, _P, _P],
    "gjxl_ref_quant_matrix": [_I, _I, _P, _P, _Z],
    "gjxl_ref_ac_strategy_cost_table": [_P, _Z, _Z, _P, _P, _P, _P, _F, _I, _P],
    "gjxl_ref_matrix_scale_stats": [_P, _Z, _Z, _Z, _Z, _P],
    "gjxl_ref_select_matrix_scales": [_P, _F, _P],
    "gjxl_ref_encode_cpu": [_P, _Z, _Z, _F, _I, _P, _Z, _P, _P],
    "gjxl_ref_encode_cpu_target_size": [_P, _Z, _Z, _Z, c_double, _Z, _I, _P, _Z, _P, _P,
                                        _P, _P],
    "gjxl_ref_dc_group_tokens": [_P, _P, _P, _P, _P, _P, _Z, _Z, _I, _P, _Z, _P, _Z, _P],
    "gjxl_ref_hybrid_uint": [_P, _Z, _I, _I, _I, _P],
}

_lib = None


def available() -> bool:
    return LIBRARY_PATH.exists()


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIBRARY_PATH.exists():
            raise FileNotFoundError(
                f"{LIBRARY_PATH} is missing; build it with `make -C oracle`")
        handle = ctypes.CDLL(str(LIBRARY_PATH))
        handle.gjxl_ref_last_error.restype = ctypes.c_char_p
        for name, args in _SIGNATURES.items():
            fn = getattr(handle, name, None)
            if fn is None:
                continue
            fn.argtypes = args
            fn.restype = c_int
        _lib = handle
    return _lib


def _ptr(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def _check(code: int, name: str) -> None:
    if code != 0:
        raise RuntimeError(f"{name}: status {code}: {lib().gjxl_ref_last_error().decode()}")


def set_threads(threads: int) -> None:
    """CPU thread budget of the pipeline entry points (0: the caller's)."""
    fn = lib().gjxl_ref_set_threads
    fn.argtypes = [_Z]
    fn.restype = c_int
    fn(threads)


def padded_extent(width: int, height: int) -> tuple[int, int]:
    return (width + 7) // 8 * 8, (height + 7) // 8 * 8


def srgb8_to_linear(pixels: np.ndarray) -> np.ndarray:
    """(H, W, 3|4) uint8 -> (3, H, W) float32 linear RGB."""
    pixels = np.ascontiguousarray(pixels)
    h, w, ch = pixels.shape
    out = np.empty((3, h, w), np.float32)
    _check(lib().gjxl_ref_srgb8_to_linear(_ptr(pixels), w, h, w * ch, ch, _ptr(out)),
           "srgb8_to_linear")
    return out


def linear_to_padded_opsin(linear: np.ndarray, intensity_target: float = 255.0) -> np.ndarray:
    linear = np.ascontiguousarray(linear, np.float32)
    _, h, w = linear.shape
    pw, ph = padded_extent(w, h)
    out = np.empty((3, ph, pw), np.float32)
    _check(lib().gjxl_ref_linear_to_padded_opsin(_ptr(linear), w, h, _ptr(out), pw, ph,
                                                 intensity_target), "linear_to_padded_opsin")
    return out


def opsin_to_linear(opsin: np.ndarray, intensity_target: float = 255.0) -> np.ndarray:
    opsin = np.ascontiguousarray(opsin, np.float32)
    _, h, w = opsin.shape
    out = np.empty_like(opsin)
    _check(lib().gjxl_ref_opsin_to_linear(_ptr(opsin), w, h, intensity_target, _ptr(out)),
           "opsin_to_linear")
    return out


def matrix_scale_stats(opsin: np.ndarray, width: int, height: int) -> np.ndarray:
    """ComputeQuantizationMatrixScaleStatsFromFiniteOpsin
    (src/codestream/workflow.cpp:1318) over the unpadded region:
    [x_edge, b_edge, exposed_blue]."""
    opsin = np.ascontiguousarray(opsin, np.float32)
    _, ph, pw = opsin.shape
    out = np.empty(3, np.float32)
    _check(lib().gjxl_ref_matrix_scale_stats(_ptr(opsin), pw, ph, width, height, _ptr(out)),
           "matrix_scale_stats")
    return out


def select_matrix_scales(stats: np.ndarray, target: float) -> tuple[int, int]:
    """SelectQuantizationMatrixScales (src/codestream/workflow.cpp:1435) for a
    Butteraugli-target encode: (x_qm_scale, b_qm_scale)."""
    stats = np.ascontiguousarray(stats, np.float32)
    out = np.zeros(2, np.int32)
    _check(lib().gjxl_ref_select_matrix_scales(_ptr(stats), target, _ptr(out)),
           "select_matrix_scales")
    return int(out[0]), int(out[1])


def encode_cpu(linear: np.ndarray, target: float = 1.0, effort: int = 7) -> tuple[bytes, float]:
    """The reference's whole CPU encode (EncodeLinearRgbVarDctCodestream,
    src/codestream/workflow.h:281): (codestream bytes, final Butteraugli
    score)."""
    linear = np.ascontiguousarray(linear, np.float32)
    _, h, w = linear.shape
    capacity = max(1 << 16, 4 * w * h)
    out = np.empty(capacity, np.uint8)
    size = c_size_t(0)
    score = c_double(0.0)
    _check(lib().gjxl_ref_encode_cpu(_ptr(linear), w, h, target, effort, _ptr(out), capacity,
                                     ctypes.byref(size), ctypes.byref(score)), "encode_cpu")
    return out[:size.value].tobytes(), score.value


def encode_cpu_target_size(linear: np.ndarray, target_bytes: int, tolerance: float = 0.005,
                           maximum_attempts: int = 12, effort: int = 7) -> dict:
    """The reference's whole CPU encode under target-size rate control
    (kTargetBytes, its bounded search over complete encodes)."""
    linear = np.ascontiguousarray(linear, np.float32)
    _, h, w = linear.shape
    capacity = max(1 << 16, 4 * w * h)
    out = np.empty(capacity, np.uint8)
    size, target = c_size_t(0), c_float(0.0)
    attempts, met = c_size_t(0), c_int(0)
    _check(lib().gjxl_ref_encode_cpu_target_size(
        _ptr(linear), w, h, target_bytes, tolerance, maximum_attempts, effort, _ptr(out),
        capacity, ctypes.byref(size), ctypes.byref(target), ctypes.byref(attempts),
        ctypes.byref(met)), "encode_cpu_target_size")
    return {"codestream": out[:size.value].tobytes(), "target": target.value,
            "attempts": attempts.value, "met": bool(met.value)}


def initial_quant_field(opsin: np.ndarray, target: float = 1.0, rescale: float = 1.0,
                        uniform: bool = False):
    opsin = np.ascontiguousarray(opsin, np.float32)
    _, ph, pw = opsin.shape
    quant = np.empty((ph // 8, pw // 8), np.float32)
    mask = np.empty_like(quant)
    pixel_mask = np.empty((ph, pw), np.float32)
    _check(lib().gjxl_ref_initial_quant_field(_ptr(opsin), pw, ph, target, rescale,
                                              int(uniform), _ptr(quant), _ptr(mask),
                                              _ptr(pixel_mask)), "initial_quant_field")
    return quant, mask, pixel_mask


def gaborish_inverse(opsin: np.ndarray, multipliers=(1.0, 1.0, 1.0)) -> np.ndarray:
    opsin = np.ascontiguousarray(opsin, np.float32)
    _, h, w = opsin.shape
    m = np.asarray(multipliers, np.float32)
    out = np.empty_like(opsin)
    _check(lib().gjxl_ref_gaborish_inverse(_ptr(opsin), w, h, _ptr(m), _ptr(out)),
           "gaborish_inverse")
    return out


def gaborish(opsin: np.ndarray) -> np.ndarray:
    opsin = np.ascontiguousarray(opsin, np.float32)
    _, h, w = opsin.shape
    out = np.empty_like(opsin)
    _check(lib().gjxl_ref_gaborish(_ptr(opsin), w, h, _ptr(out)), "gaborish")
    return out


def initial_cfl(opsin: np.ndarray, fast: bool = False):
    opsin = np.ascontiguousarray(opsin, np.float32)
    _, ph, pw = opsin.shape
    tiles = ((ph + 63) // 64, (pw + 63) // 64)
    ytox = np.empty(tiles, np.int8)
    ytob = np.empty(tiles, np.int8)
    _check(lib().gjxl_ref_initial_cfl(_ptr(opsin), pw, ph, int(fast), _ptr(ytox), _ptr(ytob)),
           "initial_cfl")
    return ytox, ytob


def ac_strategy_cost(opsin, quant, pixel_mask, strategy: int, bx: int, by: int,
                     target: float, entropy_multiplier: float, cfl_factors) -> float:
    opsin = np.ascontiguousarray(opsin, np.float32)
    quant = np.ascontiguousarray(quant, np.float32)
    pixel_mask = np.ascontiguousarray(pixel_mask, np.float32)
    _, ph, pw = opsin.shape
    f = np.asarray(cfl_factors, np.float32)
    cost = np.zeros(1, np.float32)
    _check(lib().gjxl_ref_ac_strategy_cost(_ptr(opsin), pw, ph, _ptr(quant), _ptr(pixel_mask),
                                           strategy, bx, by, target, entropy_multiplier,
                                           _ptr(f), _ptr(cost)), "ac_strategy_cost")
    return float(cost[0])


def ac_strategy_search(opsin, quant, pixel_mask, ytox, ytob, target: float = 1.0,
                       dense: bool = False) -> np.ndarray:
    opsin = np.ascontiguousarray(opsin, np.float32)
    quant = np.ascontiguousarray(quant, np.float32)
    pixel_mask = np.ascontiguousarray(pixel_mask, np.float32)
    ytox = np.ascontiguousarray(ytox, np.int8)
    ytob = np.ascontiguousarray(ytob, np.int8)
    _, ph, pw = opsin.shape
    cells = np.empty((ph // 8, pw // 8), np.uint8)
    _check(lib().gjxl_ref_ac_strategy_search(_ptr(opsin), pw, ph, _ptr(quant), _ptr(pixel_mask),
                                             _ptr(ytox), _ptr(ytob), target, int(dense),
                                             _ptr(cells)), "ac_strategy_search")
    return cells


def butteraugli(reference: np.ndarray, distorted: np.ndarray, intensity_target: float = 80.0):
    reference = np.ascontiguousarray(reference, np.float32)
    distorted = np.ascontiguousarray(distorted, np.float32)
    _, h, w = reference.shape
    dmap = np.empty((h, w), np.float32)
    score = np.zeros(1, np.float64)
    _check(lib().gjxl_ref_butteraugli(_ptr(reference), _ptr(distorted), w, h, intensity_target,
                                      _ptr(dmap), _ptr(score)), "butteraugli")
    return dmap, float(score[0])


def quant_matrix(strategy: int, channel: int):
    dq = np.zeros(1024, np.float32)
    inv = np.zeros(1024, np.float32)
    n = lib().gjxl_ref_quant_matrix(strategy, channel, _ptr(dq), _ptr(inv), 1024)
    if n <= 0:
        raise RuntimeError(f"quant_matrix({strategy}, {channel}) failed")
    return dq[:n], inv[:n]


def ac_strategy_cost_table(opsin, quant, pixel_mask, ytox, ytob, target: float = 1.0,
                           dense: bool = False) -> np.ndarray:
    """(7, blocks_y, blocks_x) costs; NaN where no candidate is anchored."""
    opsin = np.ascontiguousarray(opsin, np.float32)
    quant = np.ascontiguousarray(quant, np.float32)
    pixel_mask = np.ascontiguousarray(pixel_mask, np.float32)
    ytox = np.ascontiguousarray(ytox, np.int8)
    ytob = np.ascontiguousarray(ytob, np.int8)
    _, ph, pw = opsin.shape
    costs = np.full((7, ph // 8, pw // 8), np.nan, np.float32)
    _check(lib().gjxl_ref_ac_strategy_cost_table(_ptr(opsin), pw, ph, _ptr(quant),
                                                 _ptr(pixel_mask), _ptr(ytox), _ptr(ytob),
                                                 target, int(dense), _ptr(costs)),
           "ac_strategy_cost_table")
    return costs


class _PipelineOutputs(ctypes.Structure):
    _fields_ = [(name, c_void_p) for name in (
        "initial_quant", "strategy_mask", "pixel_mask", "final_quant", "block_distance",
        "reconstructed", "cells", "raw_quant", "quantizer_params", "y_to_x", "y_to_b",
        "quantized_dc", "dc", "ac", "group_used", "score_history")]


def quantization_pipeline(linear: np.ndarray, opsin: np.ndarray, target: float = 1.0,
                          effort: int = 7, x_qm_scale: int = 3, b_qm_scale: int = 2) -> dict:
    """The reference's whole CPU analysis half (RunCpuQuantizationPipeline)
    with the workflow's settings for an ordinary Butteraugli-target encode."""
    linear = np.ascontiguousarray(linear, np.float32)
    opsin = np.ascontiguousarray(opsin, np.float32)
    _, h, w = linear.shape
    _, ph, pw = opsin.shape
    by, bx = ph // 8, pw // 8
    ty, tx = (ph + 63) // 64, (pw + 63) // 64
    gy, gx = (by + 31) // 32, (bx + 31) // 32
    iterations = 0 if effort <= 5 else {6: 1, 7: 2, 8: 3}.get(effort, 4)
    res = {
        "initial_quant": np.zeros((by, bx), np.float32),
        "strategy_mask": np.zeros((by, bx), np.float32),
        "pixel_mask": np.zeros((ph, pw), np.float32),
        "final_quant": np.zeros((by, bx), np.float32),
        "block_distance": np.zeros((by, bx), np.float32),
        "reconstructed": np.zeros((3, h, w), np.float32),
        "cells": np.zeros((by, bx), np.uint8),
        "raw_quant": np.zeros((by, bx), np.int32),
        "quantizer_params": np.zeros(2, np.uint32),
        "y_to_x": np.zeros((ty, tx), np.int8),
        "y_to_b": np.zeros((ty, tx), np.int8),
        "quantized_dc": np.zeros((3, by, bx), np.int32),
        "dc": np.zeros((3, by, bx), np.float32),
        "ac": np.zeros(3 * ph * pw, np.int32),
        "group_used": np.zeros(gy * gx, np.uint64),
        "score_history": np.zeros(iterations + 1, np.float64),
    }
    outs = _PipelineOutputs(**{k: v.ctypes.data for k, v in res.items()})
    fn = lib().gjxl_ref_quantization_pipeline
    fn.argtypes = [_P, _Z, _Z, _P, _Z, _Z, _F, _I, _I, _I, ctypes.POINTER(_PipelineOutputs)]
    fn.restype = c_int
    _check(fn(_ptr(linear), w, h, _ptr(opsin), pw, ph, target, effort, x_qm_scale, b_qm_scale,
              ctypes.byref(outs)), "quantization_pipeline")
    return res


# Block-context maps of the reference (src/codestream/simple_ac_context.h:27-31,
# src/codestream/block_context_map.cpp:35-39): (qf thresholds, 3x13 map rows
# per threshold segment, number of contexts).
SIMPLE_BLOCK_CONTEXT_MAP = ((), bytes([0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 1,
                                      2, 2, 2, 2, 3, 3, 3, 3, 3, 3, 3, 3, 3,
                                      2, 2, 2, 2, 3, 3, 3, 3, 3, 3, 3, 3, 3]), 4)
JXL_DEFAULT_BLOCK_CONTEXT_MAP = ((), bytes([0, 1, 2, 2, 3, 3, 4, 5, 6, 6, 6, 6, 6,
                                           7, 8, 9, 9, 10, 11, 12, 13, 14, 14, 14, 14, 14,
                                           7, 8, 9, 9, 10, 11, 12, 13, 14, 14, 14, 14, 14]), 15)


class _TokenRequest(ctypes.Structure):
    _fields_ = [("qf_thresholds", c_void_p), ("threshold_count", c_size_t),
                ("context_map", c_void_p), ("num_contexts", ctypes.c_uint32),
                ("order_mode", c_int), ("orders", c_void_p), ("used_order_mask", c_void_p),
                ("group_tokens", c_void_p), ("values", c_void_p), ("contexts", c_void_p),
                ("capacity", c_size_t), ("histogram", c_void_p), ("fixed_dct8", c_int)]


def pipeline_tokens(linear: np.ndarray, opsin: np.ndarray, target: float = 1.0, effort: int = 7,
                    x_qm_scale: int = 3, b_qm_scale: int = 2,
                    block_context_map=SIMPLE_BLOCK_CONTEXT_MAP, order_mode: int = 0,
                    fixed_dct8: bool = False) -> dict:
    """quantization_pipeline, then the reference's coefficient orders
    (order_mode 0 natural, 1 full counts, 2 effort-7 sampled DCT8) and AC
    tokens of every group with the given block-context map
    (TokenizeSimpleAcGroupForEncoder, populations collected)."""
    linear = np.ascontiguousarray(linear, np.float32)
    opsin = np.ascontiguousarray(opsin, np.float32)
    _, h, w = linear.shape
    _, ph, pw = opsin.shape
    by, bx = ph // 8, pw // 8
    ty, tx = (ph + 63) // 64, (pw + 63) // 64
    gy, gx = (by + 31) // 32, (bx + 31) // 32
    iterations = 0 if effort <= 5 else {6: 1, 7: 2, 8: 3}.get(effort, 4)
    res = {
        "initial_quant": np.zeros((by, bx), np.float32),
        "strategy_mask": np.zeros((by, bx), np.float32),
        "pixel_mask": np.zeros((ph, pw), np.float32),
        "final_quant": np.zeros((by, bx), np.float32),
        "block_distance": np.zeros((by, bx), np.float32),
        "reconstructed": np.zeros((3, h, w), np.float32),
        "cells": np.zeros((by, bx), np.uint8),
        "raw_quant": np.zeros((by, bx), np.int32),
        "quantizer_params": np.zeros(2, np.uint32),
        "y_to_x": np.zeros((ty, tx), np.int8),
        "y_to_b": np.zeros((ty, tx), np.int8),
        "quantized_dc": np.zeros((3, by, bx), np.int32),
        "dc": np.zeros((3, by, bx), np.float32),
        "ac": np.zeros(3 * ph * pw, np.int32),
        "group_used": np.zeros(gy * gx, np.uint64),
        "score_history": np.zeros(iterations + 1, np.float64),
    }
    outs = _PipelineOutputs(**{k: v.ctypes.data for k, v in res.items()})
    thresholds, cmap, num_contexts = block_context_map
    thresholds = np.ascontiguousarray(np.array(thresholds, np.uint32))
    cmap = np.frombuffer(bytes(cmap), np.uint8).copy()
    assert cmap.size == 39 * (thresholds.size + 1)
    capacity = 3 * ph * pw + 3 * by * bx
    tok = {
        "orders": np.zeros((13, 3, 1024), np.uint32),
        "used_order_mask": np.zeros(1, np.uint32),
        "group_tokens": np.zeros(gy * gx, np.uint64),
        "values": np.zeros(capacity, np.uint32),
        "contexts": np.zeros(capacity, np.uint16),
        "histogram": np.zeros((num_contexts * 495, 128), np.uint32),
    }
    req = _TokenRequest(thresholds.ctypes.data if thresholds.size else None, thresholds.size,
                        cmap.ctypes.data, num_contexts, order_mode, tok["orders"].ctypes.data,
                        tok["used_order_mask"].ctypes.data, tok["group_tokens"].ctypes.data,
                        tok["values"].ctypes.data, tok["contexts"].ctypes.data, capacity,
                        tok["histogram"].ctypes.data, int(fixed_dct8))
    fn = lib().gjxl_ref_pipeline_tokens
    fn.argtypes = [_P, _Z, _Z, _P, _Z, _Z, _F, _I, _I, _I, ctypes.POINTER(_PipelineOutputs),
                   ctypes.POINTER(_TokenRequest)]
    fn.restype = c_int
    _check(fn(_ptr(linear), w, h, _ptr(opsin), pw, ph, target, effort, x_qm_scale, b_qm_scale,
              ctypes.byref(outs), ctypes.byref(req)), "pipeline_tokens")
    total = int(tok["group_tokens"].sum())
    tok["values"] = tok["values"][:total]
    tok["contexts"] = tok["contexts"][:total]
    tok["used_order_mask"] = int(tok["used_order_mask"][0])
    res.update(tok)
    return res


# ---------------------------------------------------------------------------
# The reference's own CUDA path (oracle/_ref/libgjxl_ref_cuda.so, built by
# `make -C oracle cuda`): the reference GPU baseline.

CUDA_LIBRARY_PATH = Path(__file__).resolve().parent / "_ref" / "libgjxl_ref_cuda.so"
_cuda_lib = None


def dc_group_tokens(quantized_dc: np.ndarray, cells: np.ndarray, raw_quant: np.ndarray,
                    sharpness: np.ndarray, ytox: np.ndarray, ytob: np.ndarray,
                    prediction: int = 1) -> dict:
    """The encoder's DC-group token streams (dc_group.cpp:469-546): quantized
    DC (3, by, bx) int32 in X, Y, B planes, cells (by, bx) uint8, raw quant
    (by, bx) int32, EPF sharpness (by, bx) uint8, CfL maps per 64x64 tile.
    Returns {"dc": (N, 2), "meta": (M, 2)} (context, value) uint32 pairs in
    group order, and "info": per group (dc_offset, dc_count, meta_offset,
    meta_count, anchors)."""
    _, by, bx = quantized_dc.shape
    groups = ((bx + 255) // 256) * ((by + 255) // 256)
    tiles = ((bx + 7) // 8) * ((by + 7) // 8)
    dc = np.zeros((3 * bx * by, 2), np.uint32)
    meta = np.zeros((2 * tiles + 3 * bx * by, 2), np.uint32)
    info = np.zeros((groups, 5), np.uint32)
    args = [np.ascontiguousarray(quantized_dc, np.int32), np.ascontiguousarray(cells, np.uint8),
            np.ascontiguousarray(raw_quant, np.int32), np.ascontiguousarray(sharpness, np.uint8),
            np.ascontiguousarray(ytox, np.int8), np.ascontiguousarray(ytob, np.int8)]
    _check(lib().gjxl_ref_dc_group_tokens(*[_ptr(a) for a in args], bx, by, int(prediction),
                                          _ptr(dc), dc.shape[0], _ptr(meta), meta.shape[0],
                                          _ptr(info)), "dc_group_tokens")
    meta_used = int(info[-1, 2] + info[-1, 3])
    return {"dc": dc, "meta": meta[:meta_used], "info": info}


def hybrid_uint(values: np.ndarray, split_exponent: int = 4, msb_in_token: int = 2,
                lsb_in_token: int = 0) -> np.ndarray:
    """EncodeHybridUint of each value: (N, 3) uint32 (symbol, extra bit count,
    extra bits)."""
    values = np.ascontiguousarray(values, np.uint32)
    out = np.zeros((values.size, 3), np.uint32)
    _check(lib().gjxl_ref_hybrid_uint(_ptr(values), values.size, split_exponent, msb_in_token,
                                      lsb_in_token, _ptr(out)), "hybrid_uint")
    return out


def cuda_available() -> bool:
    return CUDA_LIBRARY_PATH.exists()


def cuda_lib() -> ctypes.CDLL:
    global _cuda_lib
    if _cuda_lib is None:
        if not CUDA_LIBRARY_PATH.exists():
            raise FileNotFoundError(
                f"{CUDA_LIBRARY_PATH} is missing; build it with `make -C oracle cuda`")
        handle = ctypes.CDLL(str(CUDA_LIBRARY_PATH))
        handle.gjxl_ref_cuda_last_error.restype = ctypes.c_char_p
        handle.gjxl_ref_cuda_init.restype = c_int
        handle.gjxl_ref_cuda_encode.argtypes = [_P, _Z, _Z, _F, _I, _P, _Z, _P, _P, _P, _P]
        handle.gjxl_ref_cuda_encode.restype = c_int
        _cuda_lib = handle
    return _cuda_lib


def cuda_encode(linear: np.ndarray, target: float = 1.0, effort: int = 7) -> dict:
    """The reference's whole encode on its CUDA backend, fully-resident AQ
    (as its cuda_encoding_benchmark runs it): codestream bytes, final
    Butteraugli score, and the workflow's analysis (quantization pipeline)
    and total wall times in milliseconds."""
    lib = cuda_lib()
    code = lib.gjxl_ref_cuda_init()
    if code != 0:
        raise RuntimeError(f"gjxl_ref_cuda_init: status {code}: "
                           f"{lib.gjxl_ref_cuda_last_error().decode()}")
    linear = np.ascontiguousarray(linear, np.float32)
    _, h, w = linear.shape
    capacity = max(1 << 16, 4 * w * h)
    out = np.empty(capacity, np.uint8)
    size, score = c_size_t(0), c_double(0.0)
    analysis, total = ctypes.c_uint64(0), ctypes.c_uint64(0)
    code = lib.gjxl_ref_cuda_encode(_ptr(linear), w, h, target, effort, _ptr(out), capacity,
                                    ctypes.byref(size), ctypes.byref(score),
                                    ctypes.byref(analysis), ctypes.byref(total))
    if code != 0:
        raise RuntimeError(f"gjxl_ref_cuda_encode: status {code}: "
                           f"{lib.gjxl_ref_cuda_last_error().decode()}")
    return {"codestream": out[:size.value].tobytes(), "score": score.value,
            "analysis_ms": analysis.value / 1e6, "total_ms": total.value / 1e6}


# ---- Entropy-coded sections: the reference's model builders, writers and
# bit counters (ref_shim.cpp, gjxl_ref_entropy_*).

ENTROPY_KINDS = {"prefix": 0, "ans": 1, "ans_high_density": 2, "ans_rate": 3}


def _split(values: np.ndarray, contexts: np.ndarray, offsets: np.ndarray):
    return (np.ascontiguousarray(values, np.uint32), np.ascontiguousarray(contexts, np.uint16),
            np.ascontiguousarray(offsets, np.uint32))


class RefEntropyCode:
    """An EntropyCode built by the reference over split token sections
    (values uint32, contexts uint16, offsets uint32 [count + 1])."""

    def __init__(self, kind: str, values, contexts, offsets, context_count: int,
                 max_clusters: int = 32):
        v, c, o = _split(values, contexts, offsets)
        handle = ctypes.c_void_p()
        _check(lib().gjxl_ref_entropy_build(ENTROPY_KINDS[kind], _ptr(v), _ptr(c), _ptr(o),
                                            o.size - 1, context_count, max_clusters,
                                            ctypes.addressof(handle)), "entropy_build")
        self.handle = handle

    def close(self):
        if self.handle and _lib is not None:
            _lib.gjxl_ref_entropy_free(self.handle)
        self.handle = None

    def __del__(self):
        self.close()

    def tables(self) -> dict:
        mode, ctx, clusters = c_int(), ctypes.c_uint32(), ctypes.c_uint32()
        _check(lib().gjxl_ref_entropy_info(self.handle, ctypes.addressof(mode),
                                           ctypes.addressof(ctx), ctypes.addressof(clusters)),
               "entropy_info")
        n, k = ctx.value, clusters.value
        t = {"mode": mode.value, "context_count": n, "cluster_count": k,
             "context_map": np.zeros(n, np.uint8), "configs": np.zeros((k, 3), np.uint8),
             "depths": np.zeros((k, 128), np.uint8), "bits": np.zeros((k, 128), np.uint16),
             "degenerate": np.zeros(k, np.uint16),
             "frequencies": np.zeros((k, 256), np.uint16),
             "reverse_offsets": np.zeros((k, 256), np.uint16),
             "reverse_map": np.zeros((k, 4096), np.uint16)}
        _check(lib().gjxl_ref_entropy_tables(
            self.handle, *[_ptr(t[name]) for name in (
                "context_map", "configs", "depths", "bits", "degenerate", "frequencies",
                "reverse_offsets", "reverse_map")]), "entropy_tables")
        return t

    def write(self, values, contexts, offsets) -> dict:
        """Each section via WriteValidatedTokenStream: bit_counts, the padded
        section bytes concatenated, byte_offsets [count + 1]."""
        v, c, o = _split(values, contexts, offsets)
        count = o.size - 1
        out = np.zeros(8 * (47 * v.size // 64 + 2 * count + 2), np.uint8)
        bits = np.zeros(count, np.uint64)
        byte_offsets = np.zeros(count + 1, np.uint64)
        _check(lib().gjxl_ref_entropy_write(self.handle, _ptr(v), _ptr(c), _ptr(o), count,
                                            _ptr(out), out.size, _ptr(bits),
                                            _ptr(byte_offsets)), "entropy_write")
        return {"bit_counts": bits, "bytes": out[:int(byte_offsets[-1])],
                "byte_offsets": byte_offsets}

    def count(self, values, contexts, offsets) -> np.ndarray:
        """CountAnsTokenStreamBits / CountTokenStreamBits per section."""
        v, c, o = _split(values, contexts, offsets)
        bits = np.zeros(o.size - 1, np.uint64)
        _check(lib().gjxl_ref_entropy_count(self.handle, _ptr(v), _ptr(c), _ptr(o), o.size - 1,
                                            _ptr(bits)), "entropy_count")
        return bits
