"""Error paths of the C ABI, made on the host: nothing here faults, traps or
hangs the device.

* A device error word maps to StatusCode 7 (DEVICE_ERROR), as the
  reference's ReadAndCheckDeviceError does
  (src/gpu/cuda/cuda_aq_resident.cpp:3451): a non-finite distorted plane sets
  the Butteraugli word.
* Deterministic failure injection (gjxl_b200_test_arm_failure), the
  counterpart of the reference's CudaBackendOptions::test_fail_submission /
  ArmNextCudaSubmissionFailureForTest (src/gpu/cuda/cuda_backend.h:19-21,60):
  every allocation check point of session creation fails cleanly with
  OUT_OF_MEMORY and releases what it had taken; a failed graph instantiation
  falls back to direct launches with identical results; a failed submission
  returns SUBMISSION_FAILED and leaves every output unchanged."""

import numpy as np
import pytest
import torch

from gjxl_b200 import _lib
from gjxl_b200.session import AnalysisSession
from gjxl_b200.stages import Butteraugli
from gjxl_b200.synthetic import generate_srgb8
from oracle import ref
from tests.gpu_util import assert_bitexact, device_to_host, stream_ptr, to_device, zeros

pytestmark = pytest.mark.gpu

ALLOCATION, GRAPH, SUBMISSION = 1, 2, 3


def arm(kind: int, check_point: int) -> None:
    _lib.call("gjxl_b200_test_arm_failure", kind, check_point)


def free_bytes() -> int:
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def test_device_error_word_maps_to_device_error(cuda):
    w, h = 64, 48
    lin = ref.srgb8_to_linear(generate_srgb8(w, h, 5))
    distorted = lin.copy()
    distorted[1, 10, 17] = np.nan
    b = Butteraugli(w, h, 80.0)
    b.prepare(to_device(lin))
    dmap, score = zeros((h, w)), zeros((1,), torch.float64)
    err = zeros((1,), torch.int32)
    b.compare(to_device(lin), dmap, score, err)
    _lib.call("gjxl_b200_check_device_error", err.data_ptr(), 1, stream_ptr())
    b.compare(to_device(distorted), dmap, score, err)
    with pytest.raises(_lib.GjxlB200Error) as info:
        _lib.call("gjxl_b200_check_device_error", err.data_ptr(), 1, stream_ptr())
    assert info.value.code == 7
    assert int(err.cpu()[0]) & 1  # non-finite input
    b.close()


def test_every_allocation_failure_is_clean(cuda):
    """Session creation has several allocation check points (the arena, the
    Butteraugli planes, the AC tokenizer's tables). Failing each one in turn
    returns OUT_OF_MEMORY and leaves device memory where it was; past the
    last one, creation succeeds."""
    # One-time per-device set-up (shared tables, module loading) first.
    AnalysisSession(64, 64).close()
    before = free_bytes()
    failures = 0
    for check_point in range(1, 32):
        arm(ALLOCATION, check_point)
        try:
            s = AnalysisSession(200, 120)
        except _lib.GjxlB200Error as e:
            assert e.code == 4, str(e)
            assert "out of memory" in str(e).lower() or "alloc" in str(e).lower()
            assert free_bytes() == before, f"check point {check_point} leaked device memory"
            failures += 1
            continue
        arm(ALLOCATION, 0)
        s.close()
        break
    else:
        pytest.fail("session creation never succeeded")
    assert failures >= 3
    assert free_bytes() == before


def test_host_mirror_allocation_failure_is_clean(cuda):
    """The pinned host mirrors come with the first host-input analysis: a
    failed allocation there returns OUT_OF_MEMORY, and the next call, with
    nothing armed, allocates them and succeeds."""
    img = generate_srgb8(120, 96, 17)
    s = AnalysisSession(120, 96)
    arm(ALLOCATION, 1)
    with pytest.raises(_lib.GjxlB200Error) as info:
        s.analyze_host(img, stream_ptr())
    arm(ALLOCATION, 0)
    assert info.value.code == 4
    s.analyze_host(img, stream_ptr())
    torch.cuda.synchronize()
    assert s.host_error() == 0
    assert s.host_results()["cells"].shape == (12, 15)
    s.close()


def test_graph_failure_falls_back_to_direct_launches(cuda):
    img = generate_srgb8(300, 200, 41)
    stream = stream_ptr()
    d_img = torch.from_numpy(img.reshape(200, -1)).cuda()
    plain = AnalysisSession(300, 200)
    plain.analyze(d_img.data_ptr(), 900, 3, stream)
    fallback = AnalysisSession(300, 200)
    arm(GRAPH, 1)
    fallback.analyze(d_img.data_ptr(), 900, 3, stream)
    fallback.analyze(d_img.data_ptr(), 900, 3, stream)
    torch.cuda.synchronize()
    assert plain.outputs.graph_replay == 1
    assert fallback.outputs.graph_replay == 0
    a, b = plain.outputs, fallback.outputs
    blocks = a.blocks_x * a.blocks_y
    for name, count, dtype in (("strategy_cells", blocks, np.uint8),
                               ("quant_field", blocks, np.float32),
                               ("raw_quant_field", blocks, np.int32),
                               ("quantized_dc", 3 * blocks, np.int32),
                               ("score_history", a.iterations + 1, np.float64),
                               ("group_offsets", a.groups + 1, np.uint32)):
        assert_bitexact(device_to_host(getattr(b, name), count, dtype),
                        device_to_host(getattr(a, name), count, dtype), name)
    plain.close()
    fallback.close()


def test_submission_failure_leaves_outputs_unchanged(cuda):
    s = AnalysisSession(256, 192)
    first = generate_srgb8(256, 192, 51)
    s.analyze_host(first, stream_ptr())
    before = s.host_results()
    arm(SUBMISSION, 1)
    with pytest.raises(_lib.GjxlB200Error) as info:
        s.analyze_host(generate_srgb8(256, 192, 52), stream_ptr())
    assert info.value.code == 6
    after = s.host_results()
    for key, value in before.items():
        assert_bitexact(after[key], value, key)
    # The session still works after the failure.
    s.analyze_host(first, stream_ptr())
    again = s.host_results()
    for key, value in before.items():
        assert_bitexact(again[key], value, key)
    s.close()


def test_new_input_pointer_replays_without_recapture(cuda):
    """A device-resident caller passing a different buffer per image gets the
    results of a fresh session on that image, from the same graph."""
    a_img = generate_srgb8(320, 240, 61)
    b_img = generate_srgb8(320, 240, 62)
    stream = stream_ptr()
    d_a = torch.from_numpy(a_img.reshape(240, -1)).cuda()
    d_b = torch.from_numpy(b_img.reshape(240, -1)).cuda()
    s = AnalysisSession(320, 240)
    s.analyze(d_a.data_ptr(), 960, 3, stream)
    s.analyze(d_b.data_ptr(), 960, 3, stream)
    fresh = AnalysisSession(320, 240)
    fresh.analyze(d_b.data_ptr(), 960, 3, stream)
    torch.cuda.synchronize()
    assert s.outputs.graph_replay == 1
    o, f = s.outputs, fresh.outputs
    blocks = o.blocks_x * o.blocks_y
    for name, count, dtype in (("strategy_cells", blocks, np.uint8),
                               ("raw_quant_field", blocks, np.int32),
                               ("quantized_dc", 3 * blocks, np.int32),
                               ("group_offsets", o.groups + 1, np.uint32)):
        assert_bitexact(device_to_host(getattr(o, name), count, dtype),
                        device_to_host(getattr(f, name), count, dtype), name)
    s.close()
    fresh.close()
