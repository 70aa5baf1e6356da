"""The library's quantization matrices (built from the JPEG XL default
parameters) equal the reference's tables bit for bit."""

import ctypes

import numpy as np
import pytest

from gjxl_b200 import _lib
from oracle import ref


@pytest.mark.parametrize("strategy", [0, 4, 5, 6, 7, 10, 11])
@pytest.mark.parametrize("channel", [0, 1, 2])
def test_quant_matrix_matches_reference(strategy, channel):
    dq = np.zeros(1024, np.float32)
    inv = np.zeros(1024, np.float32)
    _lib.call("gjxl_b200_quant_matrix", strategy, channel, dq.ctypes.data, inv.ctypes.data, 1024)
    rdq, rinv = ref.quant_matrix(strategy, channel)
    n = len(rdq)
    assert np.array_equal(dq[:n].view(np.uint32), rdq.view(np.uint32))
    assert np.array_equal(inv[:n].view(np.uint32), rinv.view(np.uint32))


def test_quant_matrix_rejects_unsearched_strategy():
    dq = np.zeros(1024, np.float32)
    with pytest.raises(_lib.GjxlB200Error):
        _lib.call("gjxl_b200_quant_matrix", 18, 0, dq.ctypes.data, dq.ctypes.data, 1024)
