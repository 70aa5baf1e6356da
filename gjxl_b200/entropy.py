"""Entropy-coded sections on the device (gjxl_b200_entropy_*): token streams
written with a prebuilt ANS or prefix code bit for bit as the reference's
WriteValidatedTokenStream (src/codestream/entropy.cpp:29) writes them, and
their exact token-bit counts (CountAnsTokenStreamBits, ans.cpp:1774).

An EntropyCode holds the flattened tables of one code on the device; the
caller builds the code (clustering, normalisation) as the reference does."""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from gjxl_b200 import _lib

PREFIX, ANS = 0, 1


class EntropyCodeStruct(ctypes.Structure):
    """gjxl_b200_entropy_code."""
    _fields_ = [("mode", ctypes.c_int), ("context_count", ctypes.c_uint32),
                ("cluster_count", ctypes.c_uint32), ("context_map", ctypes.c_void_p),
                ("uint_configs", ctypes.c_void_p), ("prefix_depths", ctypes.c_void_p),
                ("prefix_bits", ctypes.c_void_p), ("prefix_degenerate", ctypes.c_void_p),
                ("ans_frequencies", ctypes.c_void_p), ("ans_reverse_offsets", ctypes.c_void_p),
                ("ans_reverse_map", ctypes.c_void_p)]


class TokenSectionsStruct(ctypes.Structure):
    """gjxl_b200_token_sections."""
    _fields_ = [("pairs", ctypes.c_void_p), ("values", ctypes.c_void_p),
                ("contexts", ctypes.c_void_p), ("offsets", ctypes.c_void_p),
                ("count", ctypes.c_uint32), ("capacity", ctypes.c_uint32)]


def _device(a: np.ndarray, dtype: np.dtype, device) -> torch.Tensor:
    a = np.ascontiguousarray(a, dtype)
    if a.dtype == np.uint16:
        return torch.from_numpy(a.view(np.int16)).to(device)
    if a.dtype == np.uint32:
        return torch.from_numpy(a.view(np.int32)).to(device)
    return torch.from_numpy(a).to(device)


class EntropyCode:
    """Device tables of one entropy code: `tables` as the reference's
    EntropyCode flattens (context_map, configs [clusters, 3], and either
    prefix depths/bits [clusters, 128] + degenerate [clusters] or ANS
    frequencies/reverse_offsets [clusters, 256] + reverse_map [clusters,
    4096])."""

    def __init__(self, tables: dict, device="cuda"):
        self.mode = int(tables["mode"])
        self.context_count = int(tables["context_count"])
        self.cluster_count = int(tables["cluster_count"])
        self._keep = {
            "context_map": _device(tables["context_map"], np.uint8, device),
            "configs": _device(tables["configs"], np.uint8, device),
        }
        if self.mode == PREFIX:
            self._keep["depths"] = _device(tables["depths"], np.uint8, device)
            self._keep["bits"] = _device(tables["bits"], np.uint16, device)
            self._keep["degenerate"] = _device(tables["degenerate"], np.uint16, device)
        else:
            self._keep["frequencies"] = _device(tables["frequencies"], np.uint16, device)
            self._keep["reverse_offsets"] = _device(tables["reverse_offsets"], np.uint16, device)
            self._keep["reverse_map"] = _device(tables["reverse_map"], np.uint16, device)

    def struct(self) -> EntropyCodeStruct:
        k = self._keep
        c = EntropyCodeStruct()
        c.mode = self.mode
        c.context_count = self.context_count
        c.cluster_count = self.cluster_count
        c.context_map = k["context_map"].data_ptr()
        c.uint_configs = k["configs"].data_ptr()
        if self.mode == PREFIX:
            c.prefix_depths = k["depths"].data_ptr()
            c.prefix_bits = k["bits"].data_ptr()
            c.prefix_degenerate = k["degenerate"].data_ptr()
        else:
            c.ans_frequencies = k["frequencies"].data_ptr()
            c.ans_reverse_offsets = k["reverse_offsets"].data_ptr()
            c.ans_reverse_map = k["reverse_map"].data_ptr()
        return c


def _sections(offsets: torch.Tensor, values=None, contexts=None, pairs=None):
    t = TokenSectionsStruct()
    t.offsets = offsets.data_ptr()
    t.count = offsets.numel() - 1
    if pairs is not None:
        t.pairs = pairs.data_ptr()
        t.capacity = pairs.shape[0]
    else:
        t.values = values.data_ptr()
        t.contexts = contexts.data_ptr()
        t.capacity = min(values.numel(), contexts.numel())
    return t


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def write_sections(code: EntropyCode, offsets: torch.Tensor, values=None, contexts=None,
                   pairs=None, packed: bool = True, tokens: int | None = None) -> dict:
    """Writes every section (gjxl_b200_entropy_write_sections). offsets:
    device int32 [count + 1]; tokens split (values int32, contexts int16) or
    interleaved (pairs int32 [N, 2], context first). Returns device tensors:
    slots, bit_counts, and with `packed` the byte-aligned concatenation and
    byte_offsets [count + 1]; plus the device error word."""
    count = offsets.numel() - 1
    total = int(offsets[-1]) if tokens is None else tokens
    lib = _lib.load()
    words = lib.gjxl_b200_entropy_slot_words(code.mode, total, count)
    dev = offsets.device
    slots = torch.empty(max(words, 1), dtype=torch.int64, device=dev)
    bit_counts = torch.zeros(count, dtype=torch.int64, device=dev)
    out = {"slots": slots, "bit_counts": bit_counts,
           "error": torch.zeros(1, dtype=torch.int32, device=dev)}
    if packed:
        out["packed"] = torch.zeros(8 * slots.numel(), dtype=torch.uint8, device=dev)
        out["byte_offsets"] = torch.zeros(count + 1, dtype=torch.int64, device=dev)
    c = code.struct()
    t = _sections(offsets, values, contexts, pairs)
    _lib.call("gjxl_b200_entropy_write_sections", ctypes.addressof(c), ctypes.addressof(t),
              slots.data_ptr(), slots.numel(), bit_counts.data_ptr(),
              out["packed"].data_ptr() if packed else None,
              out["packed"].numel() if packed else 0,
              out["byte_offsets"].data_ptr() if packed else None, out["error"].data_ptr(),
              _stream())
    return out


def count_sections(codes: list[EntropyCode], offsets: torch.Tensor, values=None,
                   contexts=None, pairs=None) -> dict:
    """Exact token bits of every section under each code
    (gjxl_b200_entropy_count_sections): bit_counts [count, len(codes)]."""
    count = offsets.numel() - 1
    structs = (EntropyCodeStruct * len(codes))(*[c.struct() for c in codes])
    bit_counts = torch.zeros((count, len(codes)), dtype=torch.int64, device=offsets.device)
    error = torch.zeros(1, dtype=torch.int32, device=offsets.device)
    t = _sections(offsets, values, contexts, pairs)
    _lib.call("gjxl_b200_entropy_count_sections", ctypes.addressof(structs), len(codes),
              ctypes.addressof(t), bit_counts.data_ptr(), error.data_ptr(), _stream())
    return {"bit_counts": bit_counts, "error": error}
