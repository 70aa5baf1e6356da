"""Rows a17/a18 parity: AC group packing, coefficient-order populations and
scans, and AC tokens against the reference's CPU path (oracle/_ref) on the
reference's own frame. The frame's strategy grid, raw quant field and
quantized AC (converted to footprint layout) go to the device; the device
tokens (values and contexts, group by group), histograms, scans in use and
packed AC must equal the reference's bit for bit.

Reference entry points: ComputeSimpleCoefficientOrdersForEncoder
(src/codestream/coefficient_order.cpp:568-830), TokenizeSimpleAcGroupForEncoder
(src/codestream/ac_group.cpp:1245, direct path with populations)."""

import numpy as np
import pytest
import torch

from gjxl_b200 import stages
from gjxl_b200.synthetic import generate_srgb8
from oracle import ref
from tests.gpu_util import (STRATEGY_COVERED, assert_bitexact, group_order_to_footprint, host,
                            to_device)

pytestmark = pytest.mark.gpu

# A map with raw-quant thresholds and 8 contexts (valid: entries < num_contexts).
_RNG = np.random.default_rng(11)
THRESHOLD_MAP = ((3, 7, 15), bytes(_RNG.integers(0, 8, 3 * 13 * 4, dtype=np.uint8)), 8)
MAPS = {"simple": ref.SIMPLE_BLOCK_CONTEXT_MAP, "jxl_default": ref.JXL_DEFAULT_BLOCK_CONTEXT_MAP,
        "thresholds": THRESHOLD_MAP}

FAMILY_OF_STRATEGY = {0: 0, 4: 2, 5: 3, 6: 4, 7: 4, 10: 6, 11: 6}
POPULATION_OFFSET = {0: 0, 2: 64, 3: 320, 4: 1344, 6: 1472}


def reference_population(cells: np.ndarray, qac: np.ndarray) -> tuple[np.ndarray, int]:
    """CountGroupZeros full counts in the CoefficientOrderPopulation layout:
    zeros per family, channel and physical index over all anchors."""
    pop = np.zeros(6144, np.uint32)
    present = 0
    ys, xs = np.nonzero(cells & 1)
    for y, x in zip(ys, xs):
        strategy = int(cells[y, x]) >> 1
        family = FAMILY_OF_STRATEGY[strategy]
        present |= 1 << family
        cw, ch = STRATEGY_COVERED[strategy]
        for c in range(3):
            block = qac[c, y * 8:y * 8 + ch * 8, x * 8:x * 8 + cw * 8].reshape(-1)
            pop[c * 1984 + POPULATION_OFFSET[family] + np.arange(block.size)] += block == 0
    return pop, present


def run_case(img, effort, map_name, order_mode, fixed_dct8=False):
    lin = ref.srgb8_to_linear(img)
    ops = ref.linear_to_padded_opsin(lin)
    want = ref.pipeline_tokens(lin, ops, 1.0, effort, 3, 2, MAPS[map_name], order_mode,
                               fixed_dct8=fixed_dct8)
    cells = want["cells"]
    by, bx = cells.shape
    qac = group_order_to_footprint(want["ac"], cells)
    tok = stages.AcTokens(bx, by)
    thresholds, cmap, nctx = MAPS[map_name]
    got = tok.tokenize(to_device(cells), to_device(want["raw_quant"]), to_device(qac),
                       stages.BlockContextMap.make(thresholds, cmap, nctx), order_mode)
    torch.cuda.synchronize()
    return want, got, qac


@pytest.mark.parametrize("w,h,seed,effort", [(509, 261, 4509, 5), (256, 256, 77, 7),
                                             (1000, 700, 5000, 7)])
@pytest.mark.parametrize("map_name", ["simple", "jxl_default", "thresholds"])
@pytest.mark.parametrize("order_mode", [0, 1, 2])
def test_tokens_match_reference(cuda, w, h, seed, effort, map_name, order_mode):
    img = generate_srgb8(w, h, seed)
    want, got, qac = run_case(img, effort, map_name, order_mode)
    offsets = host(got["group_offsets"]).astype(np.int64)
    total = int(offsets[-1])
    assert int(host(got["error"])[0]) == 0
    assert_bitexact(np.diff(offsets), want["group_tokens"].astype(np.int64), "group token counts")
    assert_bitexact(host(got["values"])[:total].view(np.uint32), want["values"], "token values")
    assert_bitexact(host(got["contexts"])[:total].view(np.uint16), want["contexts"],
                    "token contexts")
    assert_bitexact(host(got["histogram"]).view(np.uint32), want["histogram"], "histogram")
    masks = host(got["masks"]).view(np.uint32)
    assert int(masks[1]) == want["used_order_mask"]
    orders = host(got["orders"]).view(np.uint32)
    for family, n in ((0, 64), (2, 256), (3, 1024), (4, 128), (6, 512)):
        assert_bitexact(orders[family, :, :n], want["orders"][family, :, :n], f"scan {family}")
    used = int(host(got["group_coef_offsets"])[-1])
    assert_bitexact(host(got["packed_ac"])[:used], want["ac"][:used], "packed AC")
    if order_mode != 0:
        pop, present = reference_population(want["cells"], qac)
        assert int(masks[0]) == present
        got_pop = host(got["order_population"]).view(np.uint32)
        assert_bitexact(got_pop[:5952], pop[:5952], "order population")


def test_pure_dct8_sampled_orders(cuda):
    """A DCT8-only frame: effort-7 custom DCT8 scans come from the sampled
    population (xorshift128+ draws per block, groups first)."""
    img = generate_srgb8(509, 261, 99)
    want, got, _ = run_case(img, 5, "simple", 2, fixed_dct8=True)
    assert np.all(want["cells"] == 1)
    masks = host(got["masks"]).view(np.uint32)
    assert int(masks[0]) == 1 and int(masks[1]) == want["used_order_mask"]
    orders = host(got["orders"]).view(np.uint32)
    assert_bitexact(orders[0, :, :64], want["orders"][0, :, :64], "sampled DCT8 scans")
    total = int(host(got["group_offsets"])[-1])
    assert_bitexact(host(got["values"])[:total].view(np.uint32), want["values"], "token values")
    assert_bitexact(host(got["contexts"])[:total].view(np.uint16), want["contexts"],
                    "token contexts")
