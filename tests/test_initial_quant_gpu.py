"""Rows a3/a4 parity: initial quant field, strategy mask, blurred pixel mask
and inverse Gaborish against the reference's CPU code (oracle/_ref).
Bit-exact."""

import numpy as np
import pytest
import torch

from gjxl_b200 import stages
from gjxl_b200.synthetic import generate_srgb8
from oracle import ref
from tests.gpu_util import assert_bitexact, host, to_device, zeros

pytestmark = pytest.mark.gpu

SIZES = [(8, 8), (16, 24), (33, 17), (509, 261), (512, 512), (1000, 72)]


def reference_opsin(w, h, seed, noise=False):
    img = generate_srgb8(max(w, 2), max(h, 2), seed, sensor_noise=noise)[:h, :w]
    return ref.linear_to_padded_opsin(ref.srgb8_to_linear(img))


def gpu_initial_quant(opsin_np, target=1.0, rescale=1.0):
    _, ph, pw = opsin_np.shape
    opsin = to_device(opsin_np)
    q = zeros((ph // 8, pw // 8))
    m = zeros((ph // 8, pw // 8))
    pm = zeros((ph, pw))
    scratch = zeros((stages.initial_quant_scratch_bytes(pw, ph) // 4,))
    err = zeros((1,), torch.int32)
    stages.initial_quant_field(opsin, pw, ph, target, rescale, q, m, pm, scratch, err)
    return host(q), host(m), host(pm), int(host(err)[0])


@pytest.mark.parametrize("w,h", SIZES)
@pytest.mark.parametrize("target", [0.5, 1.0, 3.0])
def test_initial_quant_field_matches_reference(cuda, w, h, target):
    opsin = reference_opsin(w, h, 300 + w + h, noise=(w == 509))
    q, m, pm, err = gpu_initial_quant(opsin, target)
    rq, rm, rpm = ref.initial_quant_field(opsin, target)
    assert err == 0
    assert_bitexact(q, rq, "quant_field")
    assert_bitexact(m, rm, "strategy_mask")
    assert_bitexact(pm, rpm, "pixel_mask")


@pytest.mark.parametrize("w,h", [(1, 1), (3, 5), (8, 8), (33, 17), (509, 261)])
def test_gaborish_inverse_matches_reference(cuda, w, h):
    rng = np.random.default_rng(w * 31 + h)
    img = rng.uniform(-0.5, 1.0, (3, h, w)).astype(np.float32)
    mult = (1.0, 0.75, 1.25)
    src = to_device(img)
    dst = zeros((3, h, w))
    stages.gaborish_inverse(src, dst, w, h, mult)
    assert_bitexact(host(dst), ref.gaborish_inverse(img, mult), "gaborish_inverse")


def test_initial_quant_full_size(cuda):
    opsin = reference_opsin(4032, 3024, 2_000_000, noise=True)
    q, m, pm, err = gpu_initial_quant(opsin, 1.0)
    rq, rm, rpm = ref.initial_quant_field(opsin, 1.0)
    assert err == 0
    assert_bitexact(q, rq, "quant_field")
    assert_bitexact(m, rm, "strategy_mask")
    assert_bitexact(pm, rpm, "pixel_mask")
