"""Boundary: the candidate-batch form of the AC-strategy costs
(gjxl_b200_ac_strategy_candidate_costs, the reference's
GpuAcStrategyEvaluation seam, src/gpu/ops/ac_strategy.h:72-170). Batches of
AcStrategyCandidate descriptors give exactly the costs the tile enumeration
writes for the same anchors (both precisions), from the device's own quant
norm and CfL factors (resident form) or from the descriptors'; against the
reference's CPU cost of single candidates (oracle/_ref) within its 1-ulp
powf tolerance; a descriptor outside the image gets NaN."""

import numpy as np
import pytest
import torch

from gjxl_b200 import _lib, stages
from tests.gpu_util import host, to_device, zeros
from tests.test_ac_strategy_gpu import search_inputs, ulp_distance
from oracle import ref

pytestmark = pytest.mark.gpu

# family: (strategy code, covered blocks w, h, entropy multiplier)
FAMILIES = [(0, 1, 1, 1.0), (6, 1, 2, 1.21), (7, 2, 1, 1.21), (4, 2, 2, 1.34), (10, 2, 4, 1.49),
            (11, 4, 2, 1.49), (5, 4, 4, 1.48)]
DESC = np.dtype([("block_x", "<u4"), ("block_y", "<u4"), ("quant_norm", "<f4"),
                 ("entropy_multiplier", "<f4"), ("cfl_x", "<f4"), ("cfl_b", "<f4")])


def plane_costs(inputs, precision):
    pre, quant, mask, ytox, ytob = inputs
    _, ph, pw = pre.shape
    costs = zeros((stages.ac_strategy_cost_bytes(pw, ph) // 4,))
    stages.ac_strategy_costs(to_device(pre), to_device(quant), to_device(mask), to_device(ytox),
                             to_device(ytob), costs, 1.0, False, None, precision)
    return host(costs).reshape(7, ph // 8, pw // 8)


def batch_costs(inputs, strategy, desc, precision, resident):
    pre, quant, mask, ytox, ytob = inputs
    _, ph, pw = pre.shape
    d_pre, d_mask = to_device(pre), to_device(mask)
    d_desc = torch.from_numpy(desc.view(np.uint8).copy()).cuda()
    out = zeros((len(desc),))
    args = (to_device(quant), to_device(ytox), to_device(ytob)) if resident else (None,) * 3
    _lib.call("gjxl_b200_ac_strategy_candidate_costs", strategy, d_pre.data_ptr(), pw, ph * pw,
              d_mask.data_ptr(), pw, pw, ph, d_desc.data_ptr(), len(desc), None,
              *[a.data_ptr() if a is not None else None for a in args], 1.0, precision,
              out.data_ptr(), None, torch.cuda.current_stream().cuda_stream)
    return host(out)


def descriptors(plane, quant, ytox, ytob, cw, ch, entropy):
    ys, xs = np.nonzero(~np.isnan(plane))
    desc = np.zeros(len(xs), DESC)
    desc["block_x"], desc["block_y"] = xs, ys
    desc["entropy_multiplier"] = entropy
    if cw * ch == 1:
        desc["quant_norm"] = quant[ys, xs]
    elif cw * ch == 2:
        desc["quant_norm"] = np.maximum(quant[ys, xs], quant[ys + ch - 1, xs + cw - 1])
    desc["cfl_x"] = ytox[ys // 8, xs // 8].astype(np.float32) / np.float32(84)
    desc["cfl_b"] = np.float32(1) + ytob[ys // 8, xs // 8].astype(np.float32) / np.float32(84)
    return desc


@pytest.mark.parametrize("precision", [0, 1])
def test_resident_batches_match_the_tile_enumeration(cuda, precision):
    inputs = search_inputs(330, 204, 61)
    planes = plane_costs(inputs, precision)
    _, quant, _, ytox, ytob = inputs
    for f, (strategy, cw, ch, entropy) in enumerate(FAMILIES):
        desc = descriptors(planes[f], quant, ytox, ytob, cw, ch, entropy)
        rng = np.random.default_rng(f)
        desc = desc[rng.permutation(len(desc))]  # any order
        got = batch_costs(inputs, strategy, desc, precision, resident=True)
        want = planes[f][desc["block_y"], desc["block_x"]]
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), strategy


@pytest.mark.parametrize("precision", [0, 1])
def test_descriptor_batches_match_the_tile_enumeration(cuda, precision):
    """Quant norms and CfL factors from the descriptors (families of one and
    two blocks, whose quant norm is a plain value or maximum)."""
    inputs = search_inputs(200, 136, 62)
    planes = plane_costs(inputs, precision)
    _, quant, _, ytox, ytob = inputs
    for f, (strategy, cw, ch, entropy) in enumerate(FAMILIES[:3]):
        desc = descriptors(planes[f], quant, ytox, ytob, cw, ch, entropy)
        got = batch_costs(inputs, strategy, desc, precision, resident=False)
        want = planes[f][desc["block_y"], desc["block_x"]]
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), strategy


def test_batch_costs_match_reference_cpu_costs(cuda):
    inputs = search_inputs(256, 192, 63)
    pre, quant, mask, ytox, ytob = inputs
    for strategy, cw, ch, entropy in FAMILIES:
        desc = np.zeros(4, DESC)
        desc["block_x"] = [0, 8, 16, 24 - cw]
        desc["block_y"] = [0, 4, 8, 16]
        desc["entropy_multiplier"] = entropy
        got = batch_costs(inputs, strategy, desc, 0, resident=True)
        for d, g in zip(desc, got):
            tx, ty = int(d["block_x"]) // 8, int(d["block_y"]) // 8
            cf = [np.float32(ytox[ty, tx]) / np.float32(84), np.float32(0),
                  np.float32(1) + np.float32(ytob[ty, tx]) / np.float32(84)]
            want = ref.ac_strategy_cost(pre, quant, mask, strategy, int(d["block_x"]),
                                        int(d["block_y"]), 1.0, entropy, cf)
            assert ulp_distance(np.float32([g]), np.float32([want]))[0] <= 1, (strategy, g, want)


def test_descriptor_outside_the_image_costs_nan(cuda):
    inputs = search_inputs(64, 64, 64)
    _, quant, _, ytox, ytob = inputs
    desc = np.zeros(3, DESC)
    desc["block_x"] = [0, 7, 6]
    desc["block_y"] = [0, 0, 6]
    desc["quant_norm"] = 1.0
    desc["entropy_multiplier"] = 1.34
    desc["cfl_b"] = 1.0
    got = batch_costs(inputs, 4, desc, 0, resident=False)  # DCT16x16 covers 2x2 blocks
    assert np.isfinite(got[0]) and np.isnan(got[1]) and np.isfinite(got[2])
