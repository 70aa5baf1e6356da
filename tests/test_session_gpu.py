"""The analysis session (the C-ABI entry point a caller uses) against the
reference, through the host-input path: strategy grid, initial quant field
and CfL maps of a whole image."""

import ctypes

import numpy as np
import pytest
import torch

from gjxl_b200.session import AnalysisSession
from gjxl_b200.synthetic import generate_srgb8
from oracle import ref, restate

pytestmark = pytest.mark.gpu


def host_array(ptr, shape, ctype, dtype):
    return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctype)), shape=shape).copy()


@pytest.mark.parametrize("w,h", [(509, 261), (1000, 700)])
def test_session_matches_reference(cuda, w, h):
    img = generate_srgb8(w, h, 4000 + w)
    s = AnalysisSession(w, h)
    s.analyze_host(img, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    o = s.outputs
    assert s.host_error() == 0
    cells = s.host_strategy_cells()
    quant = host_array(o.host_initial_quant_field, (o.blocks_y, o.blocks_x), ctypes.c_float,
                       np.float32)
    ytox = host_array(o.host_y_to_x, (o.tiles_y, o.tiles_x), ctypes.c_int8, np.int8)
    ytob = host_array(o.host_y_to_b, (o.tiles_y, o.tiles_x), ctypes.c_int8, np.int8)
    stats = host_array(o.host_matrix_scale_stats, (3,), ctypes.c_float, np.float32)

    opsin = ref.linear_to_padded_opsin(ref.srgb8_to_linear(img))
    rq, _, rpm = ref.initial_quant_field(opsin, 1.0)
    pre = ref.gaborish_inverse(opsin)
    rx, rb = ref.initial_cfl(pre)
    rcells = ref.ac_strategy_search(pre, rq, rpm, rx, rb, 1.0)
    assert np.array_equal(quant.view(np.uint32), rq.view(np.uint32))
    assert np.array_equal(ytox, rx) and np.array_equal(ytob, rb)
    assert np.array_equal(stats.view(np.uint32),
                          restate.matrix_scale_stats(opsin, w, h).view(np.uint32))
    assert (cells != rcells).sum() <= 0.001 * cells.size
    s.close()


def test_session_rejects_unsupported_effort(cuda):
    from gjxl_b200._lib import GjxlB200Error
    with pytest.raises(GjxlB200Error):
        AnalysisSession(64, 64, effort=3)
