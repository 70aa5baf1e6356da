"""Small helpers shared by the GPU parity tests: device buffers through torch
(plumbing only) and raw pointers for the C ABI."""

import numpy as np
import torch


def stream_ptr() -> int:
    return torch.cuda.current_stream().cuda_stream


def to_device(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def empty(shape, dtype=torch.float32) -> torch.Tensor:
    return torch.empty(shape, dtype=dtype, device="cuda")


def zeros(shape, dtype=torch.float32) -> torch.Tensor:
    return torch.zeros(shape, dtype=dtype, device="cuda")


def host(t: torch.Tensor) -> np.ndarray:
    torch.cuda.synchronize()
    return t.cpu().numpy()


def assert_bitexact(actual: np.ndarray, expected: np.ndarray, what: str = "") -> None:
    assert actual.shape == expected.shape, (what, actual.shape, expected.shape)
    a = np.ascontiguousarray(actual).view(np.uint8)
    e = np.ascontiguousarray(expected).view(np.uint8)
    if not np.array_equal(a, e):
        diff = np.argwhere(actual != expected)
        first = tuple(diff[0]) if len(diff) else None
        raise AssertionError(
            f"{what}: {len(diff)} of {actual.size} elements differ; first at {first}: "
            f"{actual[first] if first else ''} vs {expected[first] if first else ''}")


def device_to_host(ptr: int, shape, dtype) -> np.ndarray:
    """Copies a device view published by the C ABI (a raw pointer) to the host."""
    import ctypes
    out = np.empty(shape, dtype)
    torch.cuda.synchronize()
    cudart = ctypes.CDLL("libcudart.so.12")
    cudart.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    cudart.cudaMemcpy.restype = ctypes.c_int
    rc = cudart.cudaMemcpy(out.ctypes.data, ptr, out.nbytes, 2)  # device to host
    assert rc == 0, f"cudaMemcpy failed: {rc}"
    return out


# Covered blocks (width, height) per strategy id of the mixed-transform search.
STRATEGY_COVERED = {0: (1, 1), 4: (2, 2), 5: (4, 4), 6: (1, 2), 7: (2, 1), 10: (2, 4), 11: (4, 2)}


def footprint_to_group_order(qac: np.ndarray, cells: np.ndarray) -> np.ndarray:
    """Reorders quantized AC from footprint layout (coefficient i of the
    transform anchored at block (bx, by) at pixel (bx*8 + i % W, by*8 + i / W))
    into the reference's AC group order: per 256x256 group, per channel, the
    anchors in raster order, each adding its coefficients 0..N-1."""
    by, bx = cells.shape
    gy, gx = (by + 31) // 32, (bx + 31) // 32
    out = []
    for g in range(gy * gx):
        y0, x0 = (g // gx) * 32, (g % gx) * 32
        anchors = []
        for y in range(y0, min(y0 + 32, by)):
            for x in range(x0, min(x0 + 32, bx)):
                if cells[y, x] & 1:
                    cw, ch = STRATEGY_COVERED[int(cells[y, x]) >> 1]
                    anchors.append((x, y, cw * 8, ch * 8))
        for c in range(3):
            for x, y, w, h in anchors:
                out.append(qac[c, y * 8:y * 8 + h, x * 8:x * 8 + w].reshape(-1))
    return np.concatenate(out) if out else np.zeros(0, np.int32)


def group_order_to_footprint(ac: np.ndarray, cells: np.ndarray) -> np.ndarray:
    """Inverse of footprint_to_group_order: the reference's AC group order
    back to 3 padded planes in footprint layout."""
    by, bx = cells.shape
    out = np.zeros((3, by * 8, bx * 8), np.int32)
    gy, gx = (by + 31) // 32, (bx + 31) // 32
    offset = 0
    for g in range(gy * gx):
        y0, x0 = (g // gx) * 32, (g % gx) * 32
        anchors = []
        for y in range(y0, min(y0 + 32, by)):
            for x in range(x0, min(x0 + 32, bx)):
                if cells[y, x] & 1:
                    cw, ch = STRATEGY_COVERED[int(cells[y, x]) >> 1]
                    anchors.append((x, y, cw * 8, ch * 8))
        for c in range(3):
            for x, y, w, h in anchors:
                out[c, y * 8:y * 8 + h, x * 8:x * 8 + w] = ac[offset:offset + w * h].reshape(h, w)
                offset += w * h
    return out


def differing_blocks(a: np.ndarray, b: np.ndarray, pixels: bool = False) -> np.ndarray:
    """Boolean (blocks_y, blocks_x) map of the blocks where two arrays differ
    in any element. Arrays are (..., blocks_y, blocks_x), or with `pixels`
    (..., blocks_y*8, blocks_x*8)."""
    d = np.asarray(a != b)
    while d.ndim > 2:
        d = d.any(axis=0)
    if pixels:
        h, w = d.shape
        d = d.reshape(h // 8, 8, w // 8, 8).any(axis=(1, 3))
    return d


class _CudaArray:
    """__cuda_array_interface__ over a raw device pointer (no copy)."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 3,
                                         "strides": None}


def device_view(ptr: int, shape, dtype=np.uint8) -> torch.Tensor:
    """A torch view of device memory the library owns (read it before the
    owner reuses it)."""
    return torch.as_tensor(_CudaArray(ptr, shape, np.dtype(dtype).str), device="cuda")
