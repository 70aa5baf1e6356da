"""Row f1 parity: the DC-group token streams (DC residuals with the weighted
or gradient predictor, AC metadata) and their (context, hybrid-uint symbol)
histogram, against the reference's own CPU tokenizers (oracle/_ref:
TokenizeWeightedDcGroup, TokenizeSimpleDcGroup, TokenizeSimpleAcMetadata over
the encoder's group slices). Bit-exact, token by token."""

import numpy as np
import pytest
import torch

from gjxl_b200 import stages
from gjxl_b200.session import AnalysisSession
from gjxl_b200.synthetic import generate_srgb8, workload_seed
from oracle import ref
from tests.gpu_util import assert_bitexact, host, to_device

pytestmark = pytest.mark.gpu


def reference_histogram(tokens: np.ndarray) -> np.ndarray:
    """[45][128] counts of (context, EncodeHybridUint {4,2,0} symbol)."""
    symbols = ref.hybrid_uint(tokens[:, 1])[:, 0]
    hist = np.zeros((45, 128), np.int64)
    np.add.at(hist, (tokens[:, 0].astype(np.int64), symbols.astype(np.int64)), 1)
    return hist


def random_frame(bx: int, by: int, seed: int, wide: bool):
    """All-DCT8 frame with random DC (some samples past the 32-bit fast path
    of the weighted predictor when `wide`), quant fields, sharpness and CfL
    maps."""
    rng = np.random.default_rng(seed)
    # Smooth DC plus noise, as real DC is; `wide` adds rare large spikes.
    yy, xx = np.mgrid[0:by, 0:bx]
    base = (np.sin(xx / 17.0) * 300 + np.cos(yy / 23.0) * 200).astype(np.int64)
    dc = np.stack([base // (c + 1) + rng.integers(-40, 40, (by, bx)) for c in range(3)])
    if wide:
        spikes = rng.random((3, by, bx)) < 0.002
        dc[spikes] = rng.integers(-(1 << 24), 1 << 24, spikes.sum())
    cells = np.ones((by, bx), np.uint8)  # DCT8 anchors
    raw = rng.integers(1, 257, (by, bx)).astype(np.int32)
    sharp = rng.integers(0, 8, (by, bx)).astype(np.uint8)
    tiles = ((by + 7) // 8, (bx + 7) // 8)
    ytox = rng.integers(-20, 20, tiles).astype(np.int8)
    ytob = rng.integers(-20, 20, tiles).astype(np.int8)
    return dc.astype(np.int32), cells, raw, sharp, ytox, ytob


def check(got: dict, want: dict, what: str):
    info = host(got["info"]).astype(np.uint32)
    assert_bitexact(info, want["info"], f"{what}: group table")
    assert_bitexact(host(got["dc"]).astype(np.uint32), want["dc"], f"{what}: DC tokens")
    n_meta = want["meta"].shape[0]
    assert_bitexact(host(got["meta"])[:n_meta].astype(np.uint32), want["meta"],
                    f"{what}: metadata tokens")
    hist = reference_histogram(np.concatenate([want["dc"], want["meta"]]))
    assert_bitexact(host(got["histogram"]).astype(np.int64), hist, f"{what}: histogram")
    assert int(host(got["error"])[0]) == 0


@pytest.mark.parametrize("bx,by", [(1, 1), (37, 21), (256, 256), (300, 520), (513, 40)])
@pytest.mark.parametrize("prediction", [0, 1])
def test_dc_tokens_match_reference(cuda, bx, by, prediction):
    dc, cells, raw, sharp, ytox, ytob = random_frame(bx, by, 1000 + bx + by, wide=bx >= 256)
    got = stages.dc_tokenize(to_device(dc), to_device(cells), to_device(raw), to_device(ytox),
                             to_device(ytob), prediction=prediction, sharpness=to_device(sharp))
    want = ref.dc_group_tokens(dc, cells, raw, sharp, ytox, ytob, prediction)
    check(got, want, f"{bx}x{by} prediction {prediction}")


def test_dc_tokens_default_sharpness(cuda):
    """No sharpness plane: the default 4 everywhere (FillDefaultEpfSharpness)."""
    dc, cells, raw, _, ytox, ytob = random_frame(90, 70, 5, wide=False)
    got = stages.dc_tokenize(to_device(dc), to_device(cells), to_device(raw), to_device(ytox),
                             to_device(ytob), prediction=1)
    want = ref.dc_group_tokens(dc, cells, raw, np.full(raw.shape, 4, np.uint8), ytox, ytob, 1)
    check(got, want, "default sharpness")


def test_dc_tokens_reject_invalid_quant(cuda):
    """A raw quant value outside [1, 256] (the reference's InvalidArgument)
    sets the device error word."""
    dc, cells, raw, sharp, ytox, ytob = random_frame(40, 30, 6, wide=False)
    raw[3, 5] = 300
    got = stages.dc_tokenize(to_device(dc), to_device(cells), to_device(raw), to_device(ytox),
                             to_device(ytob), prediction=1, sharpness=to_device(sharp))
    assert int(host(got["error"])[0]) & 4


@pytest.mark.parametrize("w,h,seed", [(512, 512, workload_seed(1, 0)), (2100, 700, 77)])
def test_session_dc_tokens_match_reference(cuda, w, h, seed):
    """The analysis session's own DC-group streams (DC tokens fused into its
    last DC quantization, metadata from the final strategy, quant field and
    CfL maps) against the reference tokenizers run on the session's final
    frame. 2100 px wide spans two DC groups."""
    img = generate_srgb8(w, h, seed)
    s = AnalysisSession(w, h, butteraugli_target=1.0, effort=7)
    s.analyze_host(img, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert s.host_error() == 0
    r = s.host_results()
    want = ref.dc_group_tokens(r["quantized_dc"], r["cells"], r["raw_quant"],
                               np.full(r["raw_quant"].shape, 4, np.uint8), r["y_to_x"],
                               r["y_to_b"], 1)
    assert_bitexact(r["dc_group_info"], want["info"], "group table")
    assert_bitexact(r["dc_tokens"], want["dc"], "DC tokens")
    assert_bitexact(r["meta_tokens"], want["meta"], "metadata tokens")
    hist = reference_histogram(np.concatenate([want["dc"], want["meta"]]))
    assert_bitexact(r["dc_histogram"].astype(np.int64), hist, "histogram")
    s.close()
