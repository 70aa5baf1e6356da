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
