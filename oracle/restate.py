"""numpy-facing wrapper of the C restatement (oracle/restate.c, built into
oracle/_build/librestate.so). Test infrastructure only."""

from __future__ import annotations

import ctypes
from ctypes import c_float, c_int, c_size_t, c_void_p
from pathlib import Path

import numpy as np

LIBRARY_PATH = Path(__file__).resolve().parent / "_build" / "librestate.so"
_P, _Z, _F, _I = c_void_p, c_size_t, c_float, c_int
_SIGNATURES = {
    "restate_srgb_table": [_P],
    "restate_prepare_input": [_P, _Z, _Z, _Z, _I, _F, _P, _P, _Z, _Z],
    "restate_matrix_scale_stats": [_P, _Z, _Z, _Z, _Z, _P],
    "restate_select_matrix_scales": [_P, _F, _P],
}
_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        handle = ctypes.CDLL(str(LIBRARY_PATH))
        for name, args in _SIGNATURES.items():
            fn = getattr(handle, name, None)
            if fn is not None:
                fn.argtypes = args
                fn.restype = None
        _lib = handle
    return _lib


def _ptr(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def padded_extent(width: int, height: int) -> tuple[int, int]:
    return (width + 7) // 8 * 8, (height + 7) // 8 * 8


def srgb_table() -> np.ndarray:
    t = np.empty(256, np.float32)
    lib().restate_srgb_table(_ptr(t))
    return t


def prepare_input(pixels: np.ndarray, intensity_target: float = 255.0):
    """(H, W, 3|4) uint8 -> (linear (3,H,W), padded opsin (3,PH,PW))."""
    pixels = np.ascontiguousarray(pixels)
    h, w, ch = pixels.shape
    pw, ph = padded_extent(w, h)
    linear = np.empty((3, h, w), np.float32)
    opsin = np.empty((3, ph, pw), np.float32)
    lib().restate_prepare_input(_ptr(pixels), w, h, w * ch, ch, intensity_target,
                                _ptr(linear), _ptr(opsin), pw, ph)
    return linear, opsin


def matrix_scale_stats(opsin: np.ndarray, width: int, height: int) -> np.ndarray:
    opsin = np.ascontiguousarray(opsin, np.float32)
    _, ph, pw = opsin.shape
    out = np.empty(3, np.float32)
    lib().restate_matrix_scale_stats(_ptr(opsin), pw, ph, width, height, _ptr(out))
    return out


def select_matrix_scales(stats: np.ndarray, target: float) -> tuple[int, int]:
    stats = np.ascontiguousarray(stats, np.float32)
    out = np.zeros(2, np.int32)
    lib().restate_select_matrix_scales(_ptr(stats), target, _ptr(out))
    return int(out[0]), int(out[1])


def butteraugli_pnorm(distance_map: np.ndarray, p: float = 3.0) -> float:
    """Global p-norm of a distance map in double precision, restated from
    libjxl's published p-norm summary (the mean of the p-, 2p- and 4p-norms,
    ((S_p/n)^(1/p) + (S_2p/n)^(1/2p) + (S_4p/n)^(1/4p)) / 3, S_q = sum d^q
    with d^p of each pixel in double, squared for 2p and again for 4p). The
    reference itself has no p-norm (its score is the maximum). Sums in
    numpy's pairwise order: the device's fixed tree order differs, within
    1e-12 relative."""
    d = np.asarray(distance_map, np.float32).astype(np.float64).ravel()
    dp = d * d * d if p == 3.0 else np.power(d, p)
    d2p = dp * dp
    n = float(d.size)
    sums = (dp.sum(), d2p.sum(), (d2p * d2p).sum())
    return float(sum((s / n) ** (1.0 / (p * (1 << i))) for i, s in enumerate(sums)) / 3.0)
