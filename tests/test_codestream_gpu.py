"""Codestreams from B200 analysis through the reference's unchanged CPU back
half (integration/b200_encoder.cpp): the session's results are assembled into
the reference's VarDctEncoderFrame, validated by its
ValidateSimpleCodestreamFrame (src/codec/codestream.h:87) and serialized by
its EncodeVarDctCodestreamToBuffer (src/codestream/encoder_internal.h:168),
with the CPU AC tokenizer or the device one installed as the
AcTokenizationProvider (src/codestream/ac_tokenization_provider_internal.h).

Checks, against the reference's whole CPU encode of the same image
(EncodeLinearRgbVarDctCodestream, src/codestream/workflow.h:281):
* the device tokenizer gives the same codestream bytes as the CPU one;
* where the analysis is bit-exact (one evaluation, effort 5) the codestream
  is byte-identical to the reference's;
* with field updates (effort 7) the codestream is byte-identical or its size
  and final Butteraugli distance are within 0.2% of the reference's.
No decoder is available here; the reference's frame validation and byte
identity with its own CPU codestream stand in for decoding."""

import ctypes
from ctypes import c_double, c_float, c_int, c_size_t, c_void_p
from pathlib import Path

import numpy as np
import pytest

from gjxl_b200.synthetic import generate_srgb8, workload_seed
from oracle import ref

pytestmark = pytest.mark.gpu

LIBRARY = Path(__file__).resolve().parent.parent / "integration" / "_build" / \
    "libgjxl_b200_encoder.so"


def encoder() -> ctypes.CDLL:
    if not LIBRARY.exists():
        pytest.fail(f"{LIBRARY} is missing: build it with `make -C integration`")
    lib = ctypes.CDLL(str(LIBRARY))
    lib.gjxl_b200_encode_image.argtypes = [c_void_p, c_size_t, c_size_t, c_size_t, c_int,
                                           c_float, c_int, c_int, c_int, c_void_p, c_size_t,
                                           ctypes.POINTER(c_size_t), ctypes.POINTER(c_double)]
    lib.gjxl_b200_encode_image.restype = c_int
    lib.gjxl_b200_integration_last_error.restype = ctypes.c_char_p
    return lib


def b200_encode(img: np.ndarray, target: float, effort: int, device_tokens: bool,
                precision: int = 0):
    import torch  # noqa: F401  (initializes the CUDA context on cuda:0)
    lib = encoder()
    img = np.ascontiguousarray(img)
    h, w, ch = img.shape
    capacity = max(1 << 16, 4 * w * h)
    out = np.empty(capacity, np.uint8)
    size, score = c_size_t(0), c_double(0.0)
    rc = lib.gjxl_b200_encode_image(img.ctypes.data, w, h, w * ch, ch, target, effort,
                                    precision, int(device_tokens), out.ctypes.data, capacity,
                                    ctypes.byref(size), ctypes.byref(score))
    assert rc == 0, lib.gjxl_b200_integration_last_error().decode()
    return out[:size.value].tobytes(), score.value


def check_against_reference(img, target, effort, exact_required, precision=0,
                            distance_tolerance=2e-3):
    ours, score = b200_encode(img, target, effort, device_tokens=False, precision=precision)
    ours_device, score_device = b200_encode(img, target, effort, device_tokens=True,
                                            precision=precision)
    assert ours_device == ours, "device AC tokens changed the codestream"
    assert score_device == score
    want, want_score = ref.encode_cpu(ref.srgb8_to_linear(img), target, effort)
    assert ours[:2] == b"\xff\x0a"  # JPEG XL codestream signature
    if ours == want:
        return "identical"
    assert not exact_required, (f"codestream differs from the reference: {len(ours)} vs "
                                f"{len(want)} bytes")
    size_rel = abs(len(ours) - len(want)) / len(want)
    assert size_rel <= 2e-3, f"size {len(ours)} vs {len(want)} bytes ({size_rel:.3%})"
    assert abs(score - want_score) <= distance_tolerance * want_score, (score, want_score)
    return f"size within {size_rel:.3%}"


@pytest.mark.parametrize("w,h,seed", [(256, 256, 77), (509, 261, 4509), (64, 40, 9)])
def test_single_evaluation_codestream_is_byte_identical(cuda, w, h, seed):
    check_against_reference(generate_srgb8(w, h, seed), 1.0, 5, exact_required=True)


@pytest.mark.parametrize("w,h,seed", [(512, 512, workload_seed(1, 0)), (1000, 700, 5000),
                                      (300, 200, 23)])
def test_effort7_codestream_matches_reference(cuda, w, h, seed):
    check_against_reference(generate_srgb8(w, h, seed), 1.0, 7, exact_required=False)


@pytest.mark.parametrize("target,effort", [(0.5, 6), (3.0, 7), (2.0, 8)])
def test_other_distances_and_efforts(cuda, target, effort):
    check_against_reference(generate_srgb8(384, 256, 100 + effort), target, effort,
                            exact_required=False)


@pytest.mark.parametrize("w,h,seed", [(512, 512, workload_seed(1, 0)), (1000, 700, 5000)])
def test_fast_precision_codestream_within_tolerance(cuda, w, h, seed):
    """Fast (tensor-core) candidate costs: the codestream's size within 0.2%
    of the reference CPU encode. The final Butteraugli score is the maximum
    over all pixels, which moves with any local strategy decision that the
    FP32-class costs take differently (up to 62 blocks of 11,000 here), so
    it is held to 2%."""
    check_against_reference(generate_srgb8(w, h, seed), 1.0, 7, exact_required=False,
                            precision=1, distance_tolerance=2e-2)


@pytest.mark.parametrize("w,h,seed", [(512, 512, workload_seed(1, 0)), (1000, 700, 5000)])
def test_against_reference_cuda_path(cuda, w, h, seed):
    """The reference's own CUDA path (its gjxl_cuda sources built for
    sm_100a, fully-resident AQ) on the same image: our codestream (both
    precisions) within 0.2% of its size. Its fully-resident path itself
    departs from the reference CPU path (different FP32 operation order and
    AQ schedule), so the maximum Butteraugli score, which moves with any local
    decision, is held to 3% of it; against the CPU path it is within 0.2%
    (the tests above)."""
    if not ref.cuda_available():
        pytest.fail("oracle/_ref/libgjxl_ref_cuda.so is missing: `make -C oracle cuda`")
    img = generate_srgb8(w, h, seed)
    theirs = ref.cuda_encode(ref.srgb8_to_linear(img), 1.0, 7)
    for precision in (0, 1):
        ours, score = b200_encode(img, 1.0, 7, device_tokens=False, precision=precision)
        size_rel = abs(len(ours) - len(theirs["codestream"])) / len(theirs["codestream"])
        assert size_rel <= 2e-3, (precision, len(ours), len(theirs["codestream"]))
        assert abs(score - theirs["score"]) <= 3e-2 * theirs["score"], (score, theirs["score"])


def b200_encode_target_size(img, target_bytes, tolerance=0.005, attempts=12, precision=0):
    import torch  # noqa: F401
    lib = encoder()
    fn = lib.gjxl_b200_encode_target_size
    fn.argtypes = [c_void_p, c_size_t, c_size_t, c_size_t, c_int, c_int, c_int, c_size_t,
                   c_double, c_size_t, c_void_p, c_size_t, ctypes.POINTER(c_size_t),
                   ctypes.POINTER(c_float), ctypes.POINTER(c_size_t), ctypes.POINTER(c_int)]
    fn.restype = c_int
    img = np.ascontiguousarray(img)
    h, w, ch = img.shape
    capacity = max(1 << 16, 4 * w * h)
    out = np.empty(capacity, np.uint8)
    size, target, n, met = c_size_t(0), c_float(0.0), c_size_t(0), c_int(0)
    rc = fn(img.ctypes.data, w, h, w * ch, ch, 7, precision, target_bytes, tolerance, attempts,
            out.ctypes.data, capacity, ctypes.byref(size), ctypes.byref(target), ctypes.byref(n),
            ctypes.byref(met))
    assert rc == 0, lib.gjxl_b200_integration_last_error().decode()
    return {"codestream": out[:size.value].tobytes(), "target": target.value,
            "attempts": n.value, "met": bool(met.value)}


@pytest.mark.parametrize("fraction", [0.7, 1.3])
def test_target_size_rate_control_matches_reference(cuda, fraction):
    """Target-size rate control (row f4): the reference's own bounded search
    (codestream_internal::SearchTargetSize, src/codestream/rate_control.cpp)
    driving one prepared B200 session retargeted per attempt, against the
    reference's CPU target-size encode of the same image. Every attempt's
    analysis matches the CPU path (within 0.1% of blocks), so the searches take
    the same steps: the same selected Butteraugli target and attempt count,
    or, if one attempt's size lands on the other side of the tolerance edge,
    selected sizes within 1% of each other."""
    img = generate_srgb8(256, 192, 31)
    lin = ref.srgb8_to_linear(img)
    base, _ = ref.encode_cpu(lin, 1.0, 7)
    target_bytes = int(len(base) * fraction)
    want = ref.encode_cpu_target_size(lin, target_bytes)
    got = b200_encode_target_size(img, target_bytes)
    assert got["codestream"][:2] == b"\xff\x0a"
    assert 1 <= got["attempts"] <= 12
    if got["target"] == want["target"]:
        assert got["attempts"] == want["attempts"]
        assert got["met"] == want["met"]
        assert abs(len(got["codestream"]) - len(want["codestream"])) <= \
            2e-3 * len(want["codestream"])
    else:
        assert abs(len(got["codestream"]) - len(want["codestream"])) <= \
            1e-2 * len(want["codestream"])
    if got["met"]:
        assert target_bytes - len(got["codestream"]) <= int(np.ceil(target_bytes * 0.005))
        assert len(got["codestream"]) <= target_bytes


@pytest.mark.parametrize("w,h,prefix", [(1000, 700, 0), (1000, 700, 1), (4032, 3024, 0)])
def test_device_ac_sections_match_reference_writer(cuda, w, h, prefix):
    """The binding's WriteAcSectionsOnDevice (device tables of the code the
    serializer builds from the device populations, the sections written by
    gjxl_b200_entropy_write_sections) against the reference's
    WriteValidatedTokenStream on every AC group: identical bytes and bit
    counts, including the 4032x3024 benchmark image."""
    import torch  # noqa: F401  (initializes the CUDA context on cuda:0)
    lib = encoder()
    fn = lib.gjxl_b200_compare_ac_sections
    fn.argtypes = [c_void_p, c_size_t, c_size_t, c_size_t, c_int, c_float, c_int, c_int,
                   ctypes.POINTER(c_size_t), ctypes.POINTER(c_size_t), ctypes.POINTER(c_int),
                   ctypes.POINTER(c_double), ctypes.POINTER(c_double)]
    fn.restype = c_int
    img = (generate_srgb8(w, h, 31) if w < 4000
           else generate_srgb8(w, h, workload_seed(2, 0), sensor_noise=True))
    img = np.ascontiguousarray(img)
    sections, nbytes, same = c_size_t(0), c_size_t(0), c_int(0)
    device_ms, host_ms = c_double(0.0), c_double(0.0)
    rc = fn(img.ctypes.data, w, h, w * 3, 3, 1.0, 7, prefix, ctypes.byref(sections),
            ctypes.byref(nbytes), ctypes.byref(same), ctypes.byref(device_ms),
            ctypes.byref(host_ms))
    assert rc == 0, lib.gjxl_b200_integration_last_error().decode()
    print(f"\n{w}x{h} {'prefix' if prefix else 'ANS'}: {sections.value} sections, "
          f"{nbytes.value} bytes, device {device_ms.value:.3f} ms, "
          f"reference writer {host_ms.value:.1f} ms (one thread)")
    assert sections.value == ((w + 255) // 256) * ((h + 255) // 256)
    assert same.value == 1
