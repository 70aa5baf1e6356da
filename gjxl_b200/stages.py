"""Stage-level Python binding over the C ABI, taking torch CUDA tensors.

Torch provides device memory and the current stream only; all computation is
in libgjxl_b200.so. Images are (3, rows, stride) float32 tensors whose last
dimension is the row stride (a multiple of 4).
"""

from __future__ import annotations

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


def ac_strategy_costs(opsin, quant_field, pixel_mask, y_to_x, y_to_b, costs, target=1.0,
                      dense=False, device_error=None):
    """opsin: (3, PH, PW) Gaborish-inverted XYB; costs: float tensor of
    ac_strategy_cost_bytes() bytes."""
    _lib.call("gjxl_b200_ac_strategy_costs",
              *_search_args(opsin, quant_field, pixel_mask, y_to_x, y_to_b, target, dense),
              costs.data_ptr(), None if device_error is None else device_error.data_ptr(),
              _stream())


def ac_strategy_search(opsin, quant_field, pixel_mask, y_to_x, y_to_b, costs, cells,
                       target=1.0, dense=False, device_error=None):
    _lib.call("gjxl_b200_ac_strategy_search",
              *_search_args(opsin, quant_field, pixel_mask, y_to_x, y_to_b, target, dense),
              costs.data_ptr(), cells.data_ptr(),
              None if device_error is None else device_error.data_ptr(), _stream())


def initial_cfl(opsin: torch.Tensor, y_to_x: torch.Tensor, y_to_b: torch.Tensor):
    """opsin: (3, PH, PW) Gaborish-inverted XYB; outputs int8 per 64x64 tile."""
    _lib.call("gjxl_b200_initial_cfl", opsin.data_ptr(), opsin.shape[2],
              opsin.shape[1] * opsin.shape[2], opsin.shape[2], opsin.shape[1],
              y_to_x.data_ptr(), y_to_b.data_ptr(), _stream())


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
