"""Entropy-coded sections on the device against the reference's own section
writers: for codes the reference builds (fast prefix, direct ANS in its
balanced, high-density and rate-optimized modes), every section written by
gjxl_b200_entropy_write_sections must equal WriteValidatedTokenStream's
bytes and bit count, the packed concatenation must equal the sections in
order, and gjxl_b200_entropy_count_sections must equal
CountAnsTokenStreamBits / CountTokenStreamBits. Tokens: seeded synthetic
streams (split and interleaved layouts, empty and one-token sections,
values with 29 extra bits) and the AC tokens of real analyses, among them
the 4032x3024 benchmark image."""

import numpy as np
import pytest
import torch

from gjxl_b200 import _lib
from gjxl_b200.entropy import EntropyCode, count_sections, write_sections
from gjxl_b200.learned import device_array
from gjxl_b200.session import AnalysisSession
from gjxl_b200.synthetic import generate_srgb8, workload_seed
from oracle import ref
from tests.gpu_util import host

pytestmark = pytest.mark.gpu

KINDS = ["prefix", "ans", "ans_high_density", "ans_rate"]


def sample_tokens(seed: int, n: int, contexts: int):
    rng = np.random.default_rng(seed)
    ctx = rng.integers(0, contexts, n).astype(np.uint16)
    p = 0.05 + 0.9 * (ctx.astype(np.float64) / max(1, contexts - 1))
    values = (rng.geometric(p) - 1).astype(np.uint32)
    big = rng.random(n) < 0.01
    values[big] = rng.integers(0, 2**32, int(big.sum()), dtype=np.uint64).astype(np.uint32)
    return values, ctx


def device_split(values, contexts, offsets):
    return (torch.from_numpy(values.view(np.int32)).cuda(),
            torch.from_numpy(contexts.view(np.int16)).cuda(),
            torch.from_numpy(offsets.astype(np.uint32).view(np.int32)).cuda())


def check_sections(code_ref, values, contexts, offsets, pairs=False):
    want = code_ref.write(values, contexts, offsets)
    code = EntropyCode(code_ref.tables())
    v, c, o = device_split(values, contexts, offsets)
    if pairs:
        inter = np.stack([contexts.astype(np.uint32), values], 1)
        got = write_sections(code, o, pairs=torch.from_numpy(inter.view(np.int32)).cuda())
    else:
        got = write_sections(code, o, values=v, contexts=c)
    bits = host(got["bit_counts"]).astype(np.uint64)
    assert int(host(got["error"])[0]) == 0
    assert np.array_equal(bits, want["bit_counts"])
    byte_offsets = host(got["byte_offsets"]).astype(np.uint64)
    assert np.array_equal(byte_offsets, want["byte_offsets"])
    packed = host(got["packed"])[:int(byte_offsets[-1])]
    if not np.array_equal(packed, want["bytes"]):
        for s in range(offsets.size - 1):
            lo, hi = int(want["byte_offsets"][s]), int(want["byte_offsets"][s + 1])
            assert np.array_equal(packed[lo:hi], want["bytes"][lo:hi]), f"section {s} differs"
    # Every section also sits from bit 0 of its slot.
    slots = host(got["slots"]).view(np.uint8)
    words = _lib.load().gjxl_b200_entropy_slot_words
    for s in range(offsets.size - 1):
        start = 8 * words(code.mode, int(offsets[s]), s)
        n = (int(bits[s]) + 7) // 8
        lo = int(want["byte_offsets"][s])
        assert np.array_equal(slots[start:start + n], want["bytes"][lo:lo + n]), s
    return code


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("pairs", [False, True])
def test_synthetic_sections_match_reference(cuda, kind, pairs):
    values, contexts = sample_tokens(11, 30000, 48)
    offsets = np.array([0, 0, 1, 1, 517, 9000, 9001, 20000, 30000], np.uint32)
    code_ref = ref.RefEntropyCode(kind, values, contexts, offsets, 48)
    check_sections(code_ref, values, contexts, offsets, pairs)


def test_counts_match_reference_for_several_codes(cuda):
    values, contexts = sample_tokens(12, 40000, 40)
    offsets = np.linspace(0, 40000, 17).astype(np.uint32)
    offsets[3] = offsets[2]  # an empty section
    refs = [ref.RefEntropyCode(k, values, contexts, offsets, 40) for k in KINDS]
    codes = [EntropyCode(r.tables()) for r in refs]
    v, c, o = device_split(values, contexts, offsets)
    got = count_sections(codes, o, values=v, contexts=c)
    counts = host(got["bit_counts"]).astype(np.uint64)
    assert int(host(got["error"])[0]) == 0
    for i, r in enumerate(refs):
        assert np.array_equal(counts[:, i], r.count(values, contexts, offsets)), KINDS[i]


def test_invalid_tokens_raise_the_error_word(cuda):
    """A context beyond the code and a symbol the code lacks set bit 2 of
    the error word (the reference's InvalidArgument), without a fault."""
    values, contexts = sample_tokens(13, 2000, 8)
    offsets = np.array([0, 1000, 2000], np.uint32)
    values[values > 200] = 0
    for kind in ("prefix", "ans"):
        code = EntropyCode(ref.RefEntropyCode(kind, values, contexts, offsets, 8).tables())
        for bad_values, bad_contexts in (
                (values, np.where(np.arange(2000) == 1500, 9, contexts).astype(np.uint16)),
                (np.where(np.arange(2000) == 10, 1 << 30, values).astype(np.uint32), contexts)):
            v, c, o = device_split(bad_values, bad_contexts, offsets)
            got = write_sections(code, o, values=v, contexts=c)
            assert int(host(got["error"])[0]) & 4, kind
            counted = count_sections([code], o, values=v, contexts=c)
            assert int(host(counted["error"])[0]) & 4, kind
            torch.cuda.synchronize()


def test_sections_past_the_token_arrays_are_refused(cuda):
    """Offsets reaching past the arrays' capacity set bit 2 of the error
    word; the section is not read (no fault), the others are written."""
    values, contexts = sample_tokens(14, 3000, 8)
    offsets = np.array([0, 1000, 3000], np.uint32)
    code_ref = ref.RefEntropyCode("ans", values, contexts, offsets, 8)
    want = code_ref.write(values, contexts, offsets)
    v, c, o = device_split(values, contexts, offsets)
    got = write_sections(EntropyCode(code_ref.tables()), o, values=v[:2500],
                         contexts=c[:2500], tokens=3000)
    assert int(host(got["error"])[0]) & 4
    bits = host(got["bit_counts"]).astype(np.uint64)
    assert bits[0] == want["bit_counts"][0] and bits[1] == 0


def session_tokens(img):
    h, w, _ = img.shape
    s = AnalysisSession(w, h, effort=7)
    s.analyze_host(img, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    t = s.host_tokens()
    values = t["token_values"].copy()
    contexts = t["token_contexts"].copy()
    offsets = t["group_offsets"].copy()
    o = s.outputs
    n = int(offsets[-1])
    # The device streams themselves, as the session left them.
    dev = (device_array(o.token_values, (n,), np.int32),
           device_array(o.token_contexts, (n,), np.int16),
           device_array(o.group_offsets, (offsets.size,), np.int32))
    return s, values, contexts, offsets, dev


@pytest.mark.parametrize("size", [(1000, 700), (4032, 3024)])
def test_session_ac_sections_match_reference(cuda, size):
    w, h = size
    img = (generate_srgb8(w, h, 21) if w < 4000
           else generate_srgb8(w, h, workload_seed(2, 0), sensor_noise=True))
    s, values, contexts, offsets, (dv, dc, do) = session_tokens(img)
    context_count = int(contexts.max()) + 1
    clusters = 64 if w * h >= 3840 * 2160 else 32
    for kind in ("ans", "prefix"):
        code_ref = ref.RefEntropyCode(kind, values, contexts, offsets, context_count, clusters)
        want = code_ref.write(values, contexts, offsets)
        code = EntropyCode(code_ref.tables())
        got = write_sections(code, do, values=dv, contexts=dc, tokens=int(offsets[-1]))
        assert int(host(got["error"])[0]) == 0
        byte_offsets = host(got["byte_offsets"]).astype(np.uint64)
        assert np.array_equal(host(got["bit_counts"]).astype(np.uint64), want["bit_counts"])
        assert np.array_equal(byte_offsets, want["byte_offsets"])
        assert np.array_equal(host(got["packed"])[:int(byte_offsets[-1])], want["bytes"]), kind
    s.close()
