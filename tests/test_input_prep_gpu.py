"""Row a1/a2 parity: packed sRGB -> linear RGB + padded XYB, and the
quantization-matrix statistics, against the reference (oracle/_ref) and the C
restatement. Bit-exact."""

import numpy as np
import pytest
import torch

from gjxl_b200 import stages
from gjxl_b200.synthetic import generate_srgb8
from oracle import ref, restate
from tests.gpu_util import assert_bitexact, host, to_device, zeros

pytestmark = pytest.mark.gpu

SIZES = [(1, 1), (7, 9), (8, 8), (33, 17), (509, 261), (512, 512), (1023, 77)]


def run_gpu(pixels: np.ndarray, channels: int):
    h, w = pixels.shape[:2]
    pw, ph = stages.padded_extent(w, h)
    d_pixels = to_device(pixels.reshape(h, -1))
    lin_stride = (w + 3) // 4 * 4
    linear = zeros((3, h, lin_stride))
    opsin = zeros((3, ph, pw))
    err = zeros((1,), torch.int32)
    stages.prepare_input(d_pixels, w, h, w * channels, channels, linear, opsin,
                         device_error=err)
    stats = zeros((3,))
    stages.matrix_scale_stats(opsin, w, h, stats)
    return host(linear)[:, :, :w], host(opsin), host(stats), int(host(err)[0])


@pytest.mark.parametrize("w,h", SIZES)
@pytest.mark.parametrize("channels", [3, 4])
def test_prepare_input_matches_reference(cuda, w, h, channels):
    img = generate_srgb8(max(w, 2), max(h, 2), 1000 + w * 7 + h)[:h, :w]
    if channels == 4:
        img = np.concatenate([img, np.full(img.shape[:2] + (1,), 255, np.uint8)], axis=2)
    lin, ops, stats, err = run_gpu(img, channels)
    assert err == 0
    ref_lin = ref.srgb8_to_linear(img)
    ref_ops = ref.linear_to_padded_opsin(ref_lin)
    assert_bitexact(lin, ref_lin, "linear")
    assert_bitexact(ops, ref_ops, "opsin")
    assert_bitexact(stats, restate.matrix_scale_stats(ref_ops, w, h), "stats")


def test_prepare_input_full_size_properties(cuda):
    """4032x3024 with sensor noise: bit-exact against the C restatement."""
    img = generate_srgb8(4032, 3024, 2_000_000, sensor_noise=True)
    lin, ops, stats, err = run_gpu(img, 3)
    assert err == 0
    r_lin, r_ops = restate.prepare_input(img)
    assert_bitexact(lin, r_lin, "linear")
    assert_bitexact(ops, r_ops, "opsin")
    assert_bitexact(stats, restate.matrix_scale_stats(r_ops, 4032, 3024), "stats")


def test_prepare_input_rejects_bad_geometry(cuda):
    from gjxl_b200._lib import GjxlB200Error
    img = to_device(np.zeros((8, 24), np.uint8))
    linear = zeros((3, 8, 8))
    opsin = zeros((3, 8, 8))
    with pytest.raises(GjxlB200Error):
        stages.prepare_input(img, 8, 8, 24, 5, linear, opsin)
