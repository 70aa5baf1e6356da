"""Row N3: the batched analysis (gjxl_b200_batch_*). Every image of a batch of
uneven sizes and targets gives exactly the results of its own standalone
session (the lanes share device memory and run concurrently, which must not
change a result); repeated calls reuse the pooled sessions; the per-image
timings are consistent; the autotuner picks one of the offered lane counts."""

import numpy as np
import pytest
import torch

from gjxl_b200.batch import BatchAnalyzer
from gjxl_b200.session import AnalysisSession
from gjxl_b200.synthetic import generate_srgb8
from tests.gpu_util import device_view, host

pytestmark = pytest.mark.gpu

# (width, height, target): uneven sizes, a repeated extent, two DC groups.
IMAGES = [(256, 192, 1.0), (700, 300, 0.5), (1000, 1000, 2.0), (130, 517, 3.0),
          (256, 192, 1.5), (2100, 300, 1.0), (64, 64, 1.0)]

KEYS = ["cells", "raw_quant", "quantized_dc", "y_to_x", "y_to_b", "score_history",
        "token_values", "token_contexts", "dc_tokens", "meta_tokens"]


def standalone(img, target):
    h, w, _ = img.shape
    s = AnalysisSession(w, h, butteraugli_target=target, effort=7)
    s.analyze_host(img, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    r = s.host_results()
    s.close()
    return r


def images():
    return [generate_srgb8(w, h, 900 + i) for i, (w, h, _) in enumerate(IMAGES)]


def check_same(got: dict, want: dict, what: str):
    for k in KEYS:
        assert np.array_equal(got[k], want[k]), f"{what}: {k} differs"


def test_host_input_batch_matches_standalone_sessions(cuda):
    imgs = images()
    wants = [standalone(img, t) for img, (_, _, t) in zip(imgs, IMAGES)]
    b = BatchAnalyzer(max_in_flight=3)
    reqs = b.requests([(img.ctypes.data, w, h, t) for img, (w, h, t) in zip(imgs, IMAGES)])
    for call in range(2):  # the second call reuses every pooled session
        results, ms = b.analyze(reqs, host_input=True)
        assert ms > 0
        for i, (r, (w, h, _)) in enumerate(zip(results, IMAGES)):
            assert r["status"] == 0
            assert 0 <= r["lane"] < 3
            assert r["ready_ms"] <= ms + 1e-3
            assert abs(r["queue_ms"] + r["service_ms"] - r["ready_ms"]) < 0.05
            got = BatchAnalyzer.session(r, w, h).host_results()
            check_same(got, wants[i], f"call {call} image {i} ({w}x{h})")
        if call == 0:
            first_sessions = [r["session"] for r in results]
    assert [r["session"] for r in results] == first_sessions
    b.close()


def test_device_input_batch_matches_standalone_sessions(cuda):
    """Device-resident input, one lane per image (device views of every
    image stay valid), then fewer lanes than images: the lanes' sessions
    share memory, so each lane's last image keeps its device results, and
    every image's error words are checked as it completes."""
    imgs = images()
    dev = [torch.from_numpy(img.reshape(img.shape[0], -1)).cuda() for img in imgs]
    wants = [standalone(img, t) for img, (_, _, t) in zip(imgs, IMAGES)]
    b = BatchAnalyzer(max_in_flight=len(IMAGES))
    reqs = b.requests([(d.data_ptr(), w, h, t) for d, (w, h, t) in zip(dev, IMAGES)])
    results, _ = b.analyze(reqs)
    torch.cuda.synchronize()
    assert len({r["lane"] for r in results}) == len(IMAGES)
    for i, (r, (w, h, _)) in enumerate(zip(results, IMAGES)):
        assert r["status"] == 0
        o = BatchAnalyzer.session(r, w, h).outputs
        for name, key, dtype, shape in [
                ("strategy_cells", "cells", np.uint8, (o.blocks_y, o.blocks_x)),
                ("raw_quant_field", "raw_quant", np.int32, (o.blocks_y, o.blocks_x)),
                ("quantized_dc", "quantized_dc", np.int32, (3, o.blocks_y, o.blocks_x)),
                ("y_to_x", "y_to_x", np.int8, (o.tiles_y, o.tiles_x))]:
            got = host(device_view(getattr(o, name), shape, dtype))
            assert np.array_equal(got, wants[i][key]), f"image {i}: {key} differs"
    b.set_schedule(2, True)
    results, _ = b.analyze(reqs)
    assert all(r["status"] == 0 for r in results)
    assert {r["lane"] for r in results} == {0, 1}
    for lane in (0, 1):
        i = max((k for k, r in enumerate(results) if r["lane"] == lane),
                key=lambda k: results[k]["ready_ms"])
        w, h, _ = IMAGES[i]
        o = BatchAnalyzer.session(results[i], w, h).outputs
        got = host(device_view(o.strategy_cells, (o.blocks_y, o.blocks_x), np.uint8))
        assert np.array_equal(got, wants[i]["cells"]), f"lane {lane} image {i}"
    b.close()


def test_autotune_picks_an_offered_lane_count(cuda):
    imgs = images()
    dev = [torch.from_numpy(img.reshape(img.shape[0], -1)).cuda() for img in imgs]
    b = BatchAnalyzer()
    reqs = b.requests([(d.data_ptr(), w, h, t) for d, (w, h, t) in zip(dev, IMAGES)])
    lanes, _ = b.autotune(reqs, lane_counts=(1, 2, 4))
    assert lanes in (1, 2, 4)
    results, ms = b.analyze(reqs)
    assert all(r["status"] == 0 for r in results) and ms > 0
    assert b.device_bytes() > 0
    b.close()
