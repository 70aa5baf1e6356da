"""Pins the C restatement against the compiled reference (oracle/_ref)."""

import numpy as np
import pytest

from gjxl_b200.synthetic import generate_srgb8
from oracle import ref, restate


@pytest.mark.parametrize("w,h", [(1, 1), (7, 9), (509, 261), (256, 256)])
@pytest.mark.parametrize("channels", [3, 4])
def test_restated_input_preparation_matches_reference(w, h, channels):
    img = generate_srgb8(max(w, 2), max(h, 2), 77 + w + h)[:h, :w]
    if channels == 4:
        img = np.concatenate([img, np.full(img.shape[:2] + (1,), 255, np.uint8)], axis=2)
    lin, ops = restate.prepare_input(img)
    r_lin = ref.srgb8_to_linear(img)
    r_ops = ref.linear_to_padded_opsin(r_lin)
    assert np.array_equal(lin.view(np.uint32), r_lin.view(np.uint32))
    assert np.array_equal(ops.view(np.uint32), r_ops.view(np.uint32))


def test_restated_srgb_table_is_monotone_and_anchored():
    t = restate.srgb_table()
    assert t[0] == 0.0 and t[255] == 1.0 and np.all(np.diff(t) > 0)


def test_matrix_scale_selection_thresholds():
    assert restate.select_matrix_scales(np.array([0, 0, 0], np.float32), 1.0) == (3, 2)
    assert restate.select_matrix_scales(np.array([0.03, 0.4, 0.2], np.float32), 1.0) == (5, 5)
    assert restate.select_matrix_scales(np.array([0.016, 0.3, 0.0], np.float32), 3.0) == (4, 2)
