"""Row a5 parity: initial chroma-from-luma maps against the reference's CPU
ComputeInitialColorCorrelationMap (oracle/_ref). Bit-exact."""

import numpy as np
import pytest
import torch

from gjxl_b200 import stages
from gjxl_b200.synthetic import generate_srgb8
from oracle import ref
from tests.gpu_util import assert_bitexact, host, to_device, zeros

pytestmark = pytest.mark.gpu


def preprocessed(w, h, seed, noise=False, saturation_boost=False):
    img = generate_srgb8(max(w, 2), max(h, 2), seed, sensor_noise=noise)[:h, :w]
    if saturation_boost:  # strongly coloured content so the maps are nonzero
        img = np.clip((img.astype(np.int32) - 128) * 2 + 128, 0, 255).astype(np.uint8)
        img[..., 2] = 255 - img[..., 0]
    opsin = ref.linear_to_padded_opsin(ref.srgb8_to_linear(img))
    return ref.gaborish_inverse(opsin)


@pytest.mark.parametrize("w,h", [(8, 8), (40, 24), (200, 136), (509, 261), (640, 512)])
@pytest.mark.parametrize("boost", [False, True])
def test_initial_cfl_matches_reference(cuda, w, h, boost):
    pre = preprocessed(w, h, 700 + w + h, noise=(w == 509), saturation_boost=boost)
    _, ph, pw = pre.shape
    tiles = ((ph + 63) // 64, (pw + 63) // 64)
    ytox = zeros(tiles, torch.int8)
    ytob = zeros(tiles, torch.int8)
    stages.initial_cfl(to_device(pre), ytox, ytob)
    rx, rb = ref.initial_cfl(pre)
    assert_bitexact(host(ytox), rx, "y_to_x")
    assert_bitexact(host(ytob), rb, "y_to_b")
