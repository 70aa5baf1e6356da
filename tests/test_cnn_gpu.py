"""Row N4: the proposal network's device kernels against the numpy oracle
(oracle/cnn_ref.py) — forward pass, loss and parameter gradients of one
training step, AdamW, the input gather — and the learned analysis mode:
with an uninformative network (every tile falls back to the full search, no
field correction, the effort's iterations) it reproduces the plain analysis
bit for bit, and training on plain-search examples lowers the loss."""

import numpy as np
import pytest
import torch

from gjxl_b200 import _lib
from gjxl_b200.learned import (ProposalNetwork, build_examples, device_array, metrics,
                               tile_targets, train)
from gjxl_b200.session import AnalysisSession
from gjxl_b200.synthetic import generate_srgb8
from oracle import cnn_ref
from tests.gpu_util import host

pytestmark = pytest.mark.gpu


def random_batch(n: int, seed: int):
    rng = np.random.default_rng(seed)
    x0 = cnn_ref.round_bf16(rng.normal(0, 1, (n, 80, 80, 4)).astype(np.float32))
    labels = rng.integers(0, 27, (n, 64)).astype(np.uint8)
    targets = rng.normal(0, 0.3, (n, 64)).astype(np.float32)
    weights = (rng.random((n, 64)) > 0.1).astype(np.float32)
    return x0, labels, targets, weights


def bf16_bits(a: np.ndarray) -> torch.Tensor:
    bits = (np.ascontiguousarray(a, np.float32).view(np.uint32) >> 16).astype(np.uint16)
    return torch.from_numpy(bits.view(np.int16)).cuda()


def load_batch(net: ProposalNetwork, x0: np.ndarray):
    n = x0.shape[0]
    net.ensure(n)
    net.inputs(n).copy_(bf16_bits(x0))


def params(seed: int) -> np.ndarray:
    flat = cnn_ref.init_params(seed)
    flat += np.random.default_rng(seed).normal(0, 0.02, flat.size).astype(np.float32)
    return flat


@pytest.mark.parametrize("tensor_cores", [False, True])
def test_forward_matches_oracle(cuda, tensor_cores):
    """SIMT and tcgen05 convolutions against the oracle (the tensor-core form
    over 70 tiles, several M tiles of every layer)."""
    n = 70 if tensor_cores else 6
    x0, *_ = random_batch(n, 1)
    flat = params(1)
    net = ProposalNetwork(flat)
    load_batch(net, x0)
    got = host(net.forward(n, tensor_cores=tensor_cores))
    want = cnn_ref.forward(flat, x0)["head"]
    # FP32 sums in different orders can move a BF16-rounded activation by one
    # BF16 step; the head agrees to a small fraction of its scale.
    scale = np.abs(want).max()
    assert np.abs(got - want).max() <= 2e-2 * scale
    assert np.mean(np.abs(got - want) <= 2e-3 * scale) >= 0.99


def test_train_step_gradients_match_oracle(cuda):
    """Loss and every parameter block's gradient of one training step."""
    x0, labels, targets, weights = random_batch(4, 2)
    flat = params(2)
    net = ProposalNetwork(flat)
    load_batch(net, x0)
    net.train_step(4, torch.from_numpy(labels).cuda(), torch.from_numpy(targets).cuda(),
                   torch.from_numpy(weights).cuda(), lr=0.0, weight_decay=0.0)
    got = host(net.grads)
    fwd = cnn_ref.forward(flat, x0)
    loss, dhead = cnn_ref.loss_and_grad(fwd["head"], labels, targets, weights, 4.0)
    want = cnn_ref.backward(flat, fwd, dhead)
    assert abs(float(host(net.loss)[0]) - loss) <= 1e-3 * abs(loss)
    for name, offset, shape in cnn_ref.param_layout():
        g = got[offset:offset + int(np.prod(shape))].astype(np.float64)
        w = want[offset:offset + int(np.prod(shape))]
        cos = g @ w / (np.linalg.norm(g) * np.linalg.norm(w) + 1e-30)
        assert cos >= 0.999, (name, cos)
        assert np.linalg.norm(g - w) <= 2e-2 * np.linalg.norm(w) + 1e-9, name


def test_adamw_matches_oracle(cuda):
    rng = np.random.default_rng(3)
    n = cnn_ref.PARAMS
    p0 = rng.normal(0, 1, n).astype(np.float32)
    g = rng.normal(0, 1, n).astype(np.float32)
    m0 = rng.normal(0, 0.1, n).astype(np.float32)
    v0 = rng.random(n).astype(np.float32)
    net = ProposalNetwork(p0)
    net.grads.copy_(torch.from_numpy(g))
    net.m.copy_(torch.from_numpy(m0))
    net.v.copy_(torch.from_numpy(v0))
    _lib.call("gjxl_b200_cnn_adamw", net.params.data_ptr(), net.grads.data_ptr(),
              net.m.data_ptr(), net.v.data_ptr(), 7, 1e-3, 0.9, 0.999, 1e-8, 1e-2,
              torch.cuda.current_stream().cuda_stream)
    want, m, v = cnn_ref.adamw(p0, g, m0, v0, 7, 1e-3, weight_decay=1e-2)
    # FP32 on both sides; the constants (1 - beta) round differently in
    # numpy (double, then FP32) and on the device (FP32), a few ulp at most.
    np.testing.assert_allclose(host(net.params), want, rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(host(net.m), m, rtol=1e-6, atol=2e-7)
    np.testing.assert_allclose(host(net.v), v, rtol=1e-6, atol=2e-7)


def test_gather_matches_restatement(cuda):
    """Input tiles: edge-clamped 80x80 windows of the Gaborish-inverted XYB,
    scaled per channel and rounded to BF16, and log2 of the distance."""
    img = generate_srgb8(200, 136, 5)
    s = AnalysisSession(200, 136, tokenize=False)
    s.analyze_host(img, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    o = s.outputs
    pre = host(device_array(o.preprocessed_opsin, (3, o.padded_height, o.padded_width),
                            np.float32))
    net = ProposalNetwork()
    tiles = o.tiles_x * o.tiles_y
    net.gather(o.preprocessed_opsin, o.opsin_stride, o.opsin_plane_pitch, o.padded_width,
               o.padded_height, tiles, 2.0)
    got = host(net.inputs(tiles)).astype(np.int16)
    for t in range(tiles):
        tx, ty = t % o.tiles_x, t // o.tiles_x
        ys = np.clip(np.arange(ty * 64 - 8, ty * 64 + 72), 0, o.padded_height - 1)
        xs = np.clip(np.arange(tx * 64 - 8, tx * 64 + 72), 0, o.padded_width - 1)
        win = pre[:, ys][:, :, xs].astype(np.float32)
        want = np.stack([win[0] * np.float32(24), win[1] * np.float32(2) - np.float32(1),
                         (win[2] - win[1]) * np.float32(4),
                         np.full(win[0].shape, 1.0, np.float32)], -1)
        want_bits = (cnn_ref.round_bf16(want).view(np.uint32) >> 16).astype(np.uint16)
        assert np.array_equal(got[t].view(np.uint16), want_bits), t
    s.close()


def plain_and_learned(img, flat, learned_iterations, confidence):
    h, w, _ = img.shape
    plain = AnalysisSession(w, h, effort=7)
    plain.analyze_host(img, torch.cuda.current_stream().cuda_stream)
    weights = torch.from_numpy(flat).cuda()
    learned = AnalysisSession(w, h, effort=7, proposal_weights=weights.data_ptr(),
                              learned_iterations=learned_iterations,
                              proposal_confidence=confidence)
    learned.analyze_host(img, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return plain, learned, weights


def test_uninformative_network_reproduces_plain_analysis(cuda):
    """All-zero parameters: uniform logits (top-3 mass 3/27 < 0.6, every
    tile falls back to the full search) and no field correction; with the
    effort's two field updates the learned mode is the plain analysis."""
    img = generate_srgb8(300, 260, 12)
    plain, learned, _ = plain_and_learned(img, np.zeros(cnn_ref.PARAMS, np.float32), 2, 0.6)
    a, b = plain.host_results(), learned.host_results()
    for key in ("cells", "raw_quant", "quantized_dc", "final_quant", "score_history",
                "token_values", "dc_tokens", "meta_tokens"):
        assert np.array_equal(a[key], b[key]), key
    o = learned.outputs
    masks = host(device_array(o.tile_family_masks, (o.tiles_y, o.tiles_x), np.uint8))
    assert (masks == 0x7F).all()
    plain.close()
    learned.close()


def test_confident_network_restricts_the_search(cuda):
    """A network whose head always prefers DCT8, 16x16 and 32x32 with full
    confidence: every tile searches exactly those families, and the chosen
    strategies lie among them; zero iterations leave one evaluation."""
    flat = np.zeros(cnn_ref.PARAMS, np.float32)
    layout = {name: (offset, shape) for name, offset, shape in cnn_ref.param_layout()}
    bh = layout["bh"][0]
    flat[bh + 0] = flat[bh + 4] = flat[bh + 5] = 20.0  # DCT8, DCT16x16, DCT32x32
    img = generate_srgb8(256, 192, 13)
    plain, learned, _ = plain_and_learned(img, flat, 0, 0.6)
    o = learned.outputs
    masks = host(device_array(o.tile_family_masks, (o.tiles_y, o.tiles_x), np.uint8))
    assert (masks == (1 | 8 | 64)).all()
    cells = learned.host_results()["cells"] >> 1
    assert set(np.unique(cells)) <= {0, 4, 5}
    assert o.iterations == 0 and learned.host_results()["score_history"].size == 1
    plain.close()
    learned.close()


def test_training_lowers_the_loss(cuda):
    """A few plain analyses' examples: the training loss falls and the
    held-out top-3 strategy accuracy rises."""
    net = ProposalNetwork(seed=4)
    train_imgs = [generate_srgb8(256, 256, 700 + i) for i in range(6)]
    held = [generate_srgb8(256, 256, 800 + i) for i in range(2)]
    ex = build_examples(train_imgs, net, distances=(1.0, 2.0))
    held_ex = build_examples(held, net, distances=(1.0, 2.0))
    before = metrics(net, held_ex)
    losses = train(net, ex, epochs=30, batch=16, lr=3e-3)
    after = metrics(net, held_ex)
    assert losses[-1] < 0.7 * losses[0], losses
    assert after["top3"] > before["top3"], (before, after)


def test_tile_targets_layout():
    cells = np.arange(10 * 12, dtype=np.uint8).reshape(10, 12) * 2 + 1
    final = np.full((10, 12), 2.0, np.float32)
    adjusted = np.ones((10, 12), np.float32)
    labels, targets, weights = tile_targets(cells, final, adjusted, 2, 2)
    assert labels.shape == (4, 64)
    assert labels[1, 0] == (cells[0, 8] >> 1) and weights[1, 4] == 0.0
    assert weights[3].sum() == 2 * 4 and np.allclose(targets[0], np.log(2.0))
