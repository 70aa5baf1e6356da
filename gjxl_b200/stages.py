"""Stage-level Python binding over the C ABI, taking torch CUDA tensors.

Torch provides device memory and the current stream only; all computation is
in libgjxl_b200.so. Images are (3, rows, stride) float32 tensors whose last
dimension is the row stride (a multiple of 4).
"""

from __future__ import annotations

import ctypes

import torch

from . import _lib


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def padded_extent(width: int, height: int) -> tuple[int, int]:
    return (width + 7) // 8 * 8, (height + 7) // 8 * 8


def _check_planes(t: torch.Tensor, rows: int, cols: int) -> None:
    if t.dtype != torch.float32 or not t.is_cuda or t.dim() != 3 or t.shape[0] != 3:
        raise ValueError("expected a (3, rows, stride) float32 CUDA tensor")
    if t.shape[1] < rows or t.shape[2] < cols or not t.is_contiguous():
        raise ValueError("plane tensor is too small or not contiguous")


def prepare_input(pixels: torch.Tensor, width: int, height: int, row_stride: int,
                  channels: int, linear: torch.Tensor, opsin: torch.Tensor,
                  intensity_target: float = 255.0, device_error: torch.Tensor | None = None):
    pw, ph = padded_extent(width, height)
    _check_planes(linear, height, width)
    _check_planes(opsin, ph, pw)
    _lib.call("gjxl_b200_prepare_input", pixels.data_ptr(), width, height, row_stride,
              channels, intensity_target, linear.data_ptr(), linear.shape[2],
              linear.shape[1] * linear.shape[2], opsin.data_ptr(), opsin.shape[2],
              opsin.shape[1] * opsin.shape[2], pw, ph,
              None if device_error is None else device_error.data_ptr(), _stream())


def matrix_scale_stats(opsin: torch.Tensor, width: int, height: int, stats: torch.Tensor):
    _lib.call("gjxl_b200_matrix_scale_stats", opsin.data_ptr(), opsin.shape[2],
              opsin.shape[1] * opsin.shape[2], width, height, stats.data_ptr(), _stream())


def initial_quant_field(opsin: torch.Tensor, padded_width: int, padded_height: int,
                        target: float, rescale: float, quant_field: torch.Tensor,
                        strategy_mask: torch.Tensor, pixel_mask: torch.Tensor,
                        scratch: torch.Tensor, device_error: torch.Tensor | None = None):
    _lib.call("gjxl_b200_initial_quant_field", opsin.data_ptr(), opsin.shape[2],
              opsin.shape[1] * opsin.shape[2], padded_width, padded_height, target, rescale,
              quant_field.data_ptr(), strategy_mask.data_ptr(), pixel_mask.data_ptr(),
              pixel_mask.shape[-1], scratch.data_ptr(), scratch.numel() * scratch.element_size(),
              None if device_error is None else device_error.data_ptr(), _stream())


def initial_quant_scratch_bytes(padded_width: int, padded_height: int) -> int:
    return _lib.load().gjxl_b200_initial_quant_scratch_bytes(padded_width, padded_height)


def gaborish_inverse(src: torch.Tensor, dst: torch.Tensor, width: int, height: int,
                     multipliers=(1.0, 1.0, 1.0), device_error: torch.Tensor | None = None):
    import ctypes
    m = (ctypes.c_float * 3)(*multipliers)
    _lib.call("gjxl_b200_gaborish_inverse", src.data_ptr(), src.shape[2],
              src.shape[1] * src.shape[2], dst.data_ptr(), dst.shape[2],
              dst.shape[1] * dst.shape[2], width, height, ctypes.addressof(m),
              None if device_error is None else device_error.data_ptr(), _stream())


def ac_strategy_cost_bytes(padded_width: int, padded_height: int) -> int:
    return _lib.load().gjxl_b200_ac_strategy_cost_bytes(padded_width, padded_height)


def _search_args(opsin, quant_field, pixel_mask, y_to_x, y_to_b, target, dense):
    return (opsin.data_ptr(), opsin.shape[2], opsin.shape[1] * opsin.shape[2], opsin.shape[2],
            opsin.shape[1], quant_field.data_ptr(), pixel_mask.data_ptr(), pixel_mask.shape[-1],
            y_to_x.data_ptr(), y_to_b.data_ptr(), target, int(dense))


PRECISION_EXACT, PRECISION_FAST = 0, 1


def ac_strategy_costs(opsin, quant_field, pixel_mask, y_to_x, y_to_b, costs, target=1.0,
                      dense=False, device_error=None, precision=PRECISION_EXACT):
    """opsin: (3, PH, PW) Gaborish-inverted XYB; costs: float tensor of
    ac_strategy_cost_bytes() bytes."""
    _lib.call("gjxl_b200_ac_strategy_costs",
              *_search_args(opsin, quant_field, pixel_mask, y_to_x, y_to_b, target, dense),
              precision, costs.data_ptr(),
              None if device_error is None else device_error.data_ptr(), _stream())


def ac_strategy_search(opsin, quant_field, pixel_mask, y_to_x, y_to_b, costs, cells,
                       target=1.0, dense=False, device_error=None, precision=PRECISION_EXACT):
    _lib.call("gjxl_b200_ac_strategy_search",
              *_search_args(opsin, quant_field, pixel_mask, y_to_x, y_to_b, target, dense),
              precision, costs.data_ptr(), cells.data_ptr(),
              None if device_error is None else device_error.data_ptr(), _stream())


def initial_cfl(opsin: torch.Tensor, y_to_x: torch.Tensor, y_to_b: torch.Tensor):
    """opsin: (3, PH, PW) Gaborish-inverted XYB; outputs int8 per 64x64 tile."""
    pw, ph = opsin.shape[2], opsin.shape[1]
    _lib.call("gjxl_b200_initial_cfl", opsin.data_ptr(), pw, ph * pw, pw, ph,
              y_to_x.data_ptr(), y_to_b.data_ptr(), _stream())


def dc_tokenize(quantized_dc: torch.Tensor, cells: torch.Tensor, raw_quant: torch.Tensor,
                y_to_x: torch.Tensor, y_to_b: torch.Tensor, prediction: int = 1,
                sharpness: torch.Tensor | None = None, histogram: bool = True) -> dict:
    """DC-group token streams of a frame (gjxl_b200_dc_tokenize): quantized DC
    (3, by, bx) int32, cells (by, bx) uint8, raw quant (by, bx) int32, CfL maps
    per tile. Returns device tensors: dc (N, 2) and meta (M, 2) (context,
    value) uint32 pairs, info (groups, 5), histogram (45, 128), and the
    device error word."""
    _, by, bx = quantized_dc.shape
    sizes = [ctypes.c_size_t(0) for _ in range(4)]
    _lib.call("gjxl_b200_dc_token_sizes", bx, by, *[ctypes.addressof(v) for v in sizes])
    n_dc, n_meta, groups, scratch_bytes = (v.value for v in sizes)
    dev = quantized_dc.device
    dc = torch.zeros((n_dc, 2), dtype=torch.int32, device=dev)
    meta = torch.zeros((n_meta, 2), dtype=torch.int32, device=dev)
    info = torch.zeros((groups, 5), dtype=torch.int32, device=dev)
    hist = torch.zeros((45, 128), dtype=torch.int32, device=dev)
    scratch = torch.empty(scratch_bytes // 4, dtype=torch.int32, device=dev)
    error = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.call("gjxl_b200_dc_tokenize", quantized_dc.data_ptr(), bx * by, cells.data_ptr(),
              raw_quant.data_ptr(), 0 if sharpness is None else sharpness.data_ptr(),
              y_to_x.data_ptr(), y_to_b.data_ptr(), bx, by, prediction, dc.data_ptr(),
              meta.data_ptr(), info.data_ptr(), hist.data_ptr() if histogram else 0,
              scratch.data_ptr(), scratch_bytes, error.data_ptr(), _stream())
    return {"dc": dc, "meta": meta, "info": info, "histogram": hist, "error": error}


class Butteraugli:
    """Prepared-reference Butteraugli on the device (gjxl_b200_butteraugli_*)."""

    def __init__(self, width: int, height: int, intensity_target: float = 80.0):
        import ctypes
        lib = _lib.load()
        lib.gjxl_b200_butteraugli_destroy.argtypes = [ctypes.c_void_p]
        lib.gjxl_b200_butteraugli_destroy.restype = None
        handle = ctypes.c_void_p()
        _lib.call("gjxl_b200_butteraugli_create", width, height, intensity_target,
                  ctypes.addressof(handle))
        self.handle = handle.value
        self.width, self.height = width, height

    def prepare(self, reference: torch.Tensor):
        _lib.call("gjxl_b200_butteraugli_prepare", self.handle, reference.data_ptr(),
                  reference.shape[2], reference.shape[1] * reference.shape[2], _stream())

    def compare(self, distorted: torch.Tensor, distance_map: torch.Tensor,
                score: torch.Tensor | None = None, device_error: torch.Tensor | None = None):
        _lib.call("gjxl_b200_butteraugli_compare", self.handle, distorted.data_ptr(),
                  distorted.shape[2], distorted.shape[1] * distorted.shape[2],
                  distance_map.data_ptr(), distance_map.shape[-1],
                  None if score is None else score.data_ptr(),
                  None if device_error is None else device_error.data_ptr(), _stream())

    def close(self):
        if self.handle:
            _lib.load().gjxl_b200_butteraugli_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BlockContextMap(ctypes.Structure):
    """gjxl_b200_block_context_map."""
    _fields_ = [("threshold_count", ctypes.c_uint32), ("qf_thresholds", ctypes.c_uint32 * 15),
                ("num_contexts", ctypes.c_uint32), ("context_map", ctypes.c_uint8 * (3 * 13 * 16))]

    @classmethod
    def make(cls, thresholds, context_map: bytes, num_contexts: int) -> "BlockContextMap":
        m = cls()
        m.threshold_count = len(thresholds)
        for i, t in enumerate(thresholds):
            m.qf_thresholds[i] = t
        m.num_contexts = num_contexts
        for i, v in enumerate(context_map):
            m.context_map[i] = v
        return m


class AcTokenOutputs(ctypes.Structure):
    """gjxl_b200_ac_token_outputs."""
    _fields_ = [("token_values", ctypes.c_void_p), ("token_contexts", ctypes.c_void_p),
                ("token_capacity", ctypes.c_size_t), ("group_offsets", ctypes.c_void_p),
                ("histogram", ctypes.c_void_p), ("packed_ac", ctypes.c_void_p),
                ("group_coef_offsets", ctypes.c_void_p), ("order_population", ctypes.c_void_p),
                ("present_mask", ctypes.c_void_p), ("used_order_mask", ctypes.c_void_p),
                ("orders", ctypes.c_void_p), ("device_error", ctypes.c_void_p)]


class AcTokens:
    """AC group packing, coefficient-order populations and AC tokenization
    for one block extent (gjxl_b200_ac_tokens_*)."""

    def __init__(self, blocks_x: int, blocks_y: int):
        self.bx, self.by = blocks_x, blocks_y
        handle = ctypes.c_void_p()
        _lib.call("gjxl_b200_ac_tokens_create", blocks_x, blocks_y, ctypes.byref(handle))
        self.handle = handle
        self.capacity = _lib.load().gjxl_b200_ac_token_capacity(blocks_x, blocks_y)
        self.groups = ((blocks_x + 31) // 32) * ((blocks_y + 31) // 32)

    def close(self):
        if self.handle:
            _lib.load().gjxl_b200_ac_tokens_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tokenize(self, cells: torch.Tensor, raw_quant: torch.Tensor, quantized_ac: torch.Tensor,
                 block_context_map: BlockContextMap, order_mode: int = 0,
                 histogram: bool = True, packed: bool = True) -> dict:
        """Returns device tensors: values, contexts, group_offsets, histogram,
        packed_ac, group_coef_offsets, order_population, masks (present, used),
        orders and the error word. `quantized_ac` is (3, padded_h, padded_w)
        int32 in footprint layout."""
        dev = quantized_ac.device
        u32 = torch.int32
        res = {
            "values": torch.empty(self.capacity, dtype=u32, device=dev),
            "contexts": torch.empty(self.capacity, dtype=torch.int16, device=dev),
            "group_offsets": torch.zeros(self.groups + 1, dtype=u32, device=dev),
            "group_coef_offsets": torch.zeros(self.groups + 1, dtype=u32, device=dev),
            "order_population": torch.zeros(6144, dtype=u32, device=dev),
            "masks": torch.zeros(2, dtype=u32, device=dev),
            "orders": torch.zeros((13, 3, 1024), dtype=u32, device=dev),
            "error": torch.zeros(1, dtype=u32, device=dev),
        }
        if histogram:
            res["histogram"] = torch.zeros((block_context_map.num_contexts * 495, 128), dtype=u32,
                                           device=dev)
        if packed:
            res["packed_ac"] = torch.zeros(3 * 64 * self.bx * self.by, dtype=u32, device=dev)
        out = AcTokenOutputs(
            res["values"].data_ptr(), res["contexts"].data_ptr(), self.capacity,
            res["group_offsets"].data_ptr(),
            res["histogram"].data_ptr() if histogram else None,
            res["packed_ac"].data_ptr() if packed else None,
            res["group_coef_offsets"].data_ptr(), res["order_population"].data_ptr(),
            res["masks"].data_ptr(), res["masks"].data_ptr() + 4, res["orders"].data_ptr(),
            res["error"].data_ptr())
        _, ph, pw = quantized_ac.shape
        _lib.call("gjxl_b200_ac_tokenize", self.handle, cells.data_ptr(), raw_quant.data_ptr(),
                  quantized_ac.data_ptr(), pw, ph * pw, ctypes.byref(block_context_map),
                  order_mode, ctypes.byref(out), _stream())
        return res
