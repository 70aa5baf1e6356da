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


@pytest.mark.parametrize("w,h,seed,noise", [(2, 2, 5, False), (1, 9, 6, False), (9, 1, 7, False),
                                            (509, 261, 4509, False), (256, 256, 77, True),
                                            (333, 200, 91, True)])
def test_restated_matrix_scale_stats_match_reference(w, h, seed, noise):
    """The restated statistics (the CUDA path's OpsinMatrixScaleStatsKernel
    semantics) equal the reference's own
    ComputeQuantizationMatrixScaleStatsFromFiniteOpsin
    (src/codestream/workflow.cpp:1318) bit for bit, over the unpadded region
    of the padded opsin image (including 1-pixel-wide images, which have no
    statistics)."""
    img = generate_srgb8(max(w, 2), max(h, 2), seed, sensor_noise=noise)[:h, :w]
    opsin = ref.linear_to_padded_opsin(ref.srgb8_to_linear(img))
    want = ref.matrix_scale_stats(opsin, w, h)
    got = restate.matrix_scale_stats(opsin, w, h)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (got, want)


def test_restated_matrix_scale_selection_matches_reference():
    """SelectQuantizationMatrixScales (src/codestream/workflow.cpp:1435) over
    a grid that crosses every threshold (x_edge 0.015/0.022/0.026, b_edge
    0.28/0.33/0.38, exposed blue 0.13, target 2.5/5.5/9.5), each threshold
    probed at the float just below, at, and just above it."""
    def around(values):
        out = [0.0]
        for v in values:
            f = np.float32(v)
            out += [np.nextafter(f, np.float32(0)), f, np.nextafter(f, np.float32(1))]
        return out
    xs = around([0.015, 0.022, 0.026])
    bs = around([0.28, 0.33, 0.38])
    es = around([0.13])
    targets = [0.5, 1.0, 2.5, 2.6, 5.5, 6.0, 9.5, 12.0]
    checked = 0
    for x in xs:
        for b in bs:
            for e in es:
                stats = np.array([x, b, e], np.float32)
                for t in targets:
                    assert restate.select_matrix_scales(stats, t) == \
                        ref.select_matrix_scales(stats, t), (stats, t)
                    checked += 1
    assert checked == len(xs) * len(bs) * len(es) * len(targets)


def test_pnorm_restatement_properties():
    """The FP64 p-norm restatement: a constant map is its own norm, the norm
    is positively homogeneous, and it lies between the mean and the maximum
    of the map for p >= 1."""
    const = np.full((31, 17), 1.75, np.float32)
    assert abs(restate.butteraugli_pnorm(const, 3.0) - 1.75) <= 1e-14
    m = np.abs(np.random.default_rng(7).standard_normal((64, 48))).astype(np.float32)
    a = restate.butteraugli_pnorm(m, 3.0)
    b = restate.butteraugli_pnorm((2 * m).astype(np.float32), 3.0)
    assert abs(b - 2 * a) <= 1e-13 * b
    assert m.astype(np.float64).mean() <= a <= float(m.max())
