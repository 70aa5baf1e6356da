"""gjxl_b200_initial_quant_field_noalloc (library-owned static scratch, no
device allocation) against gjxl_b200_initial_quant_field (caller scratch),
called through the C ABI. Two calls in a row on different images and extents
must each match the caller-scratch results bit for bit, so scratch left over
from the first call cannot leak into the second; a call takes no device
memory (free device memory is the same before and after it); sizes beyond
the static scratch are rejected."""

import numpy as np
import pytest
import torch

from gjxl_b200 import _lib
from gjxl_b200.synthetic import generate_srgb8
from oracle import ref
from tests.gpu_util import assert_bitexact, host, stream_ptr, to_device, zeros

pytestmark = pytest.mark.gpu

# 16 MiB of static scratch at 4.25 bytes per padded pixel.
MAX_PADDED_PIXELS = 3_947_580


def padded_opsin(w: int, h: int, seed: int) -> np.ndarray:
    return ref.linear_to_padded_opsin(ref.srgb8_to_linear(generate_srgb8(w, h, seed)))


def outputs(pw: int, ph: int):
    return (zeros((ph // 8, pw // 8)), zeros((ph // 8, pw // 8)), zeros((ph, pw)),
            zeros((1,), torch.int32))


def run(opsin_np: np.ndarray, target: float, noalloc: bool):
    _, ph, pw = opsin_np.shape
    opsin = to_device(opsin_np)
    q, m, pm, err = outputs(pw, ph)
    common = (opsin.data_ptr(), pw, ph * pw, pw, ph, target, 1.0, q.data_ptr(), m.data_ptr(),
              pm.data_ptr(), pw)
    if noalloc:
        _lib.call("gjxl_b200_initial_quant_field_noalloc", *common, err.data_ptr(), stream_ptr())
    else:
        nbytes = _lib.load().gjxl_b200_initial_quant_scratch_bytes(pw, ph)
        scratch = zeros((nbytes // 4,))
        _lib.call("gjxl_b200_initial_quant_field", *common, scratch.data_ptr(), nbytes,
                  err.data_ptr(), stream_ptr())
    torch.cuda.synchronize()
    return host(q), host(m), host(pm), int(host(err)[0])


def test_noalloc_matches_caller_scratch_on_consecutive_calls(cuda):
    cases = [(1000, 700, 71, 1.0), (509, 261, 72, 0.5)]
    for w, h, seed, target in cases:
        opsin = padded_opsin(w, h, seed)
        got = run(opsin, target, noalloc=True)
        want = run(opsin, target, noalloc=False)
        assert got[3] == 0 and want[3] == 0
        for name, a, b in zip(("quant_field", "strategy_mask", "pixel_mask"), got, want):
            assert_bitexact(a, b, f"{name} {w}x{h}")


def test_noalloc_largest_extent(cuda):
    w, h = 2048, 1920  # 3,932,160 padded pixels
    assert w * h <= MAX_PADDED_PIXELS
    opsin = padded_opsin(w, h, 73)
    got = run(opsin, 1.0, noalloc=True)
    want = run(opsin, 1.0, noalloc=False)
    for name, a, b in zip(("quant_field", "strategy_mask", "pixel_mask"), got, want):
        assert_bitexact(a, b, name)


def test_noalloc_rejects_extent_beyond_static_scratch(cuda):
    pw, ph = 2048, 1928  # 3,948,544 padded pixels: just over the limit
    assert pw * ph > MAX_PADDED_PIXELS
    opsin = zeros((3, ph, pw))
    q, m, pm, err = outputs(pw, ph)
    with pytest.raises(_lib.GjxlB200Error) as info:
        _lib.call("gjxl_b200_initial_quant_field_noalloc", opsin.data_ptr(), pw, ph * pw, pw, ph,
                  1.0, 1.0, q.data_ptr(), m.data_ptr(), pm.data_ptr(), pw, err.data_ptr(),
                  stream_ptr())
    assert info.value.code == 1 and "16 MiB" in str(info.value)


def test_noalloc_call_takes_no_device_memory(cuda):
    """After a warm-up call (which loads the library's module and with it the
    static scratch), a call on another extent leaves the device's free memory
    exactly where it was: the entry point allocates nothing."""
    warm = padded_opsin(128, 96, 74)
    run(warm, 1.0, noalloc=True)
    w, h = 700, 500
    opsin_np = padded_opsin(w, h, 75)
    _, ph, pw = opsin_np.shape
    opsin = to_device(opsin_np)
    q, m, pm, err = outputs(pw, ph)
    torch.cuda.synchronize()
    before = torch.cuda.mem_get_info()[0]
    _lib.call("gjxl_b200_initial_quant_field_noalloc", opsin.data_ptr(), pw, ph * pw, pw, ph,
              1.0, 1.0, q.data_ptr(), m.data_ptr(), pm.data_ptr(), pw, err.data_ptr(),
              stream_ptr())
    torch.cuda.synchronize()
    after = torch.cuda.mem_get_info()[0]
    assert after == before, f"free device memory changed by {before - after} bytes"
    want = run(opsin_np, 1.0, noalloc=False)
    assert_bitexact(host(q), want[0], "quant_field")
    assert int(host(err)[0]) == 0
