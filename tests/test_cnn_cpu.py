"""Row N4 oracle: the numpy restatement of the proposal network
(oracle/cnn_ref.py) is pinned by finite differences of its own loss in
float64, and its parameter layout matches the library's."""

import ctypes

import numpy as np
import pytest

from oracle import cnn_ref


def test_param_count_matches_library():
    from gjxl_b200 import _lib
    assert _lib.load().gjxl_b200_cnn_param_count() == cnn_ref.PARAMS == 29852


def batch(seed: int, n: int = 2):
    rng = np.random.default_rng(seed)
    x0 = rng.normal(0, 1, (n, 80, 80, 4))
    labels = rng.integers(0, 27, (n, 64)).astype(np.uint8)
    targets = rng.normal(0, 0.3, (n, 64))
    weights = (rng.random((n, 64)) > 0.1).astype(np.float64)
    return x0, labels, targets, weights


def loss_of(flat, x0, labels, targets, weights):
    fwd = cnn_ref.forward(flat, x0, bf16=False)
    loss, _ = cnn_ref.loss_and_grad(fwd["head"], labels, targets, weights, 0.5)
    return loss


@pytest.mark.parametrize("seed", [1, 2])
def test_backward_matches_finite_differences(seed):
    x0, labels, targets, weights = batch(seed)
    flat = cnn_ref.init_params(seed).astype(np.float64)
    flat += np.random.default_rng(seed).normal(0, 0.01, flat.size)  # nonzero biases
    fwd = cnn_ref.forward(flat, x0, bf16=False)
    _, dhead = cnn_ref.loss_and_grad(fwd["head"], labels, targets, weights, 0.5)
    grad = cnn_ref.backward(flat, fwd, dhead, bf16=False)
    rng = np.random.default_rng(100 + seed)
    picks = []
    for name, offset, shape in cnn_ref.param_layout():
        picks += list(offset + rng.integers(0, int(np.prod(shape)), 4))
    eps = 1e-6
    for i in picks:
        up, down = flat.copy(), flat.copy()
        up[i] += eps
        down[i] -= eps
        numeric = (loss_of(up, x0, labels, targets, weights) -
                   loss_of(down, x0, labels, targets, weights)) / (2 * eps)
        assert abs(numeric - grad[i]) <= 1e-6 + 1e-4 * abs(numeric), (i, numeric, grad[i])


def test_round_bf16_ties_to_even():
    vals = np.array([1.0, 1.00390625, 1.01171875, -3.0e-3, 65504.0], np.float32)
    got = cnn_ref.round_bf16(vals)
    assert got[0] == 1.0
    assert got[1] == 1.0          # halfway between 1 and 1 + 2^-7: even mantissa
    assert got[2] == 1.015625     # halfway, rounds up to the even neighbour
    assert abs(got[3] - vals[3]) <= 2 ** -8 * abs(vals[3])  # half of a 7-bit ulp
