"""The fast precision mode of the AC-strategy search (rows a6-a8): the
families with 16/32-pixel sides on tcgen05 tensor cores (three-piece
split-bf16 operands, f32 accumulation in tensor memory), the 8-pixel families
with FP32 fused multiply-adds. The reference for every cost is the
reference's own CPU evaluator (FP64 transforms, oracle/_ref); its CUDA path
also evaluates in FP32 and differs from the CPU path in the same way
(src/gpu/cuda/cuda_kernels.cu:653).

Tolerances (FP32-class arithmetic): the median candidate cost within 1e-6
relative and 99% of candidates within 1e-4 (the rest are candidates where one
quantized coefficient sits within rounding of a .5 boundary and rounds the
other way, which moves the cost by up to a few percent); the strategy grid
within 0.1% of blocks on the benchmarked 4032x3024 image, and within 1% on
small images, where a single 32x32 transform is 16 blocks of a few thousand."""

import numpy as np
import pytest
import torch

from gjxl_b200 import stages
from gjxl_b200.synthetic import workload_seed
from oracle import ref
from tests.gpu_util import host, to_device, zeros
from tests.test_ac_strategy_gpu import search_inputs

pytestmark = pytest.mark.gpu


def fast_search(pre, quant, pmask, ytox, ytob, target=1.0, dense=False):
    _, ph, pw = pre.shape
    costs = zeros((stages.ac_strategy_cost_bytes(pw, ph) // 4,))
    cells = zeros((ph // 8, pw // 8), torch.uint8)
    err = zeros((1,), torch.int32)
    stages.ac_strategy_search(to_device(pre), to_device(quant), to_device(pmask),
                              to_device(ytox), to_device(ytob), costs, cells, target, dense,
                              err, precision=stages.PRECISION_FAST)
    return host(costs).reshape(7, ph // 8, pw // 8), host(cells), int(host(err)[0])


def check_fast_costs(costs, ref_costs):
    assert np.array_equal(np.isnan(costs), np.isnan(ref_costs)), "anchor sets differ"
    for f in range(7):
        valid = ~np.isnan(ref_costs[f])
        if not valid.any():
            continue
        want = ref_costs[f][valid].astype(np.float64)
        rel = np.abs(costs[f][valid] - want) / np.abs(want)
        assert np.isfinite(costs[f][valid]).all()
        assert np.median(rel) <= 1e-6, (f, np.median(rel))
        assert np.quantile(rel, 0.99) <= 1e-4, (f, np.quantile(rel, 0.99))
        assert rel.max() <= 0.05, (f, rel.max())


@pytest.mark.parametrize("w,h,seed,noise,target", [(512, 512, workload_seed(1, 0), False, 1.0),
                                                   (509, 261, 4509, True, 1.0),
                                                   (1000, 700, 5000, False, 1.0),
                                                   (200, 136, 91, False, 2.5),
                                                   (24, 40, 623, False, 1.0)])
def test_fast_costs_and_grid(cuda, w, h, seed, noise, target):
    pre, quant, pmask, ytox, ytob = search_inputs(w, h, seed, noise=noise, target=target)
    costs, cells, err = fast_search(pre, quant, pmask, ytox, ytob, target)
    assert err == 0
    check_fast_costs(costs, ref.ac_strategy_cost_table(pre, quant, pmask, ytox, ytob, target))
    ref_cells = ref.ac_strategy_search(pre, quant, pmask, ytox, ytob, target)
    assert (cells != ref_cells).sum() <= 0.01 * cells.size


def test_fast_grid_full_size(cuda):
    """The benchmarked 4032x3024 image: grid within 0.1% of blocks of the
    reference search."""
    pre, quant, pmask, ytox, ytob = search_inputs(4032, 3024, workload_seed(2, 0), noise=True)
    costs, cells, err = fast_search(pre, quant, pmask, ytox, ytob)
    assert err == 0
    ref_cells = ref.ac_strategy_search(pre, quant, pmask, ytox, ytob)
    assert (cells != ref_cells).sum() <= 0.001 * cells.size


def test_fast_dense_dct32(cuda):
    pre, quant, pmask, ytox, ytob = search_inputs(200, 136, 91)
    costs, cells, err = fast_search(pre, quant, pmask, ytox, ytob, 1.0, dense=True)
    assert err == 0
    ref_cells = ref.ac_strategy_search(pre, quant, pmask, ytox, ytob, 1.0, dense=True)
    assert (cells != ref_cells).sum() <= 0.01 * cells.size


def test_fast_mode_rejects_unknown_precision(cuda):
    from gjxl_b200 import _lib
    pre, quant, pmask, ytox, ytob = search_inputs(64, 64, 3)
    _, ph, pw = pre.shape
    costs = zeros((stages.ac_strategy_cost_bytes(pw, ph) // 4,))
    with pytest.raises(_lib.GjxlB200Error) as info:
        stages.ac_strategy_costs(to_device(pre), to_device(quant), to_device(pmask),
                                 to_device(ytox), to_device(ytob), costs, precision=2)
    assert info.value.code == 1
