"""The precision form's configuration (6000x4000 from the configurations'
generator, effort 9, d1.0) with the transforms the reference codes: the fast
precision (DCT16+ families as split-BF16x3 tcgen05 products with FP32
accumulation, 8-pixel families in FP32) against the exact FP64 restatement
of the reference's CPU evaluator, which is the FP64 oracle here (the exact
costs equal the reference CPU's within 1 ulp, tests/test_ac_strategy_gpu.py).

Per-result error: every candidate cost of the image, median within 1e-6 and
99% within 1e-4 relative. Decisions: the strategy grid within 0.1% of
blocks; the final quant field, after four field updates that spread each
grid difference over its Butteraugli neighbourhood, identical farther than
24 blocks from a differing cell (and within 1% of blocks); the score within
0.2%. File size: the two
precisions' codestreams through the reference's unchanged serializer within
0.2% of each other, Butteraugli distance within 0.2%."""

import time

import numpy as np
import pytest
import torch
from scipy import ndimage

from gjxl_b200.session import AnalysisSession
from gjxl_b200.synthetic import generate_srgb8, workload_seed
from tests.test_ac_strategy_fast_gpu import fast_search
from tests.test_ac_strategy_gpu import gpu_search, search_inputs
from tests.test_codestream_gpu import b200_encode

pytestmark = pytest.mark.gpu

W, H = 6000, 4000
SEED = workload_seed(3, 0)


def test_precision_form_costs_against_fp64(cuda):
    pre, quant, pmask, ytox, ytob = search_inputs(W, H, SEED)
    exact, exact_cells, err = gpu_search(pre, quant, pmask, ytox, ytob)[:3]
    assert err == 0
    fast, fast_cells, err = fast_search(pre, quant, pmask, ytox, ytob)
    assert err == 0
    exact = exact.reshape(fast.shape)
    assert np.array_equal(np.isnan(fast), np.isnan(exact))
    for f in range(7):
        valid = ~np.isnan(exact[f])
        want = exact[f][valid].astype(np.float64)
        rel = np.abs(fast[f][valid] - want) / np.abs(want)
        print(f"family {f}: {valid.sum()} costs, median {np.median(rel):.2e}, "
              f"p99 {np.quantile(rel, 0.99):.2e}, max {rel.max():.2e}")
        assert np.median(rel) <= 1e-6 and np.quantile(rel, 0.99) <= 1e-4, f
    differ = int((fast_cells != exact_cells).sum())
    print(f"grid: {differ} of {exact_cells.size} blocks differ")
    assert differ <= 0.001 * exact_cells.size


def analyse(img, precision):
    s = AnalysisSession(W, H, butteraugli_target=1.0, effort=9, precision=precision)
    stream = torch.cuda.current_stream().cuda_stream
    s.analyze_host(img, stream)  # first call: graph capture
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.analyze_host(img, stream)
    torch.cuda.synchronize()
    seconds = time.perf_counter() - t0
    assert s.host_error() == 0
    return s, s.host_results(), seconds


def test_precision_form_session_and_file_size(cuda):
    img = generate_srgb8(W, H, SEED)
    exact_s, exact, exact_t = analyse(img, 0)
    fast_s, fast, fast_t = analyse(img, 1)
    print(f"6000x4000 e9 analysis: exact {W * H / 1e6 / exact_t:.1f} MP/s, "
          f"fast {W * H / 1e6 / fast_t:.1f} MP/s, iterations {exact_s.outputs.iterations}")
    assert exact_s.outputs.iterations == 4  # AdaptiveQuantizationIterations at effort 9
    blocks = exact["cells"].size
    cells_differ = exact["cells"] != fast["cells"]
    print(f"cells: {int(cells_differ.sum())} of {blocks} blocks differ")
    assert cells_differ.sum() <= 0.001 * blocks
    # Four field updates, each from Butteraugli distances blurred over a few
    # blocks, spread every strategy difference over its neighbourhood (the
    # radius grows with each update); the field elsewhere must be identical.
    quant_differ = exact["final_quant"] != fast["final_quant"]
    near = ndimage.binary_dilation(cells_differ, iterations=24)
    print(f"final_quant: {int(quant_differ.sum())} of {blocks} blocks differ, "
          f"{int((quant_differ & ~near).sum())} farther than 24 blocks from a differing cell")
    assert quant_differ.sum() <= 0.01 * blocks
    assert not (quant_differ & ~near).any()
    a, b = exact["score_history"][-1], fast["score_history"][-1]
    assert abs(a - b) <= 2e-3 * a, (a, b)
    exact_s.close()
    fast_s.close()
    exact_bytes, exact_score = b200_encode(img, 1.0, 9, device_tokens=True, precision=0)
    fast_bytes, fast_score = b200_encode(img, 1.0, 9, device_tokens=True, precision=1)
    size_rel = abs(len(fast_bytes) - len(exact_bytes)) / len(exact_bytes)
    print(f"codestream: exact {len(exact_bytes)} B, fast {len(fast_bytes)} B "
          f"({size_rel:.4%}); distance {exact_score:.5f} vs {fast_score:.5f}")
    assert size_rel <= 2e-3
    assert abs(fast_score - exact_score) <= 2e-3 * exact_score
