"""Entropy-coded sections, CPU side: the reference's model builders, writers
and counters reached through the oracle shim, and a Python model of the
device writer's scheme (records, the top-down reverse writer and the final
shift for ANS; scanned lengths for prefix codes) checked byte for byte
against the reference's own section bytes."""

import numpy as np
import pytest

from oracle import ref

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle library not built")


def hybrid(value: int, split: int, msb: int, lsb: int):
    if value < (1 << split):
        return value, 0, 0
    e = value.bit_length() - 1
    m = value - (1 << e)
    symbol = ((1 << split) + ((e - split) << (msb + lsb)) + ((m >> (e - msb)) << lsb)
              + (m & ((1 << lsb) - 1)))
    count = e - msb - lsb
    return symbol, count, (value >> lsb) & ((1 << count) - 1)


def model_ans(tables, values, contexts):
    """The device scheme: chunks stored top-down into a bit string, the
    final state pushed last, the stream read from its lowest bit."""
    chunks = []
    state = 0x13 << 16
    for value, context in zip(values[::-1], contexts[::-1]):
        cluster = int(tables["context_map"][context])
        split, msb, lsb = (int(x) for x in tables["configs"][cluster])
        symbol, count, extra = hybrid(int(value), split, msb, lsb)
        f = int(tables["frequencies"][cluster, symbol])
        off = int(tables["reverse_offsets"][cluster, symbol])
        assert f != 0
        if count:
            chunks.append((extra, count))
        if (state >> 20) >= f:
            chunks.append((state & 0xFFFF, 16))
            state >>= 16
        recip = ((1 << 44) + f - 1) // f
        q = (state * recip) >> 44
        assert q == state // f
        state = (q << 12) + int(tables["reverse_map"][cluster, off + state - q * f])
    chunks.append((state, 32))
    # Top-down: the first chunk pushed occupies the highest bits.
    total = sum(n for _, n in chunks)
    stream = 0
    top = total
    for v, n in chunks:
        top -= n
        stream |= v << top
    return stream, total


def model_prefix(tables, values, contexts):
    stream, at = 0, 0
    for value, context in zip(values, contexts):
        cluster = int(tables["context_map"][context])
        split, msb, lsb = (int(x) for x in tables["configs"][cluster])
        symbol, count, extra = hybrid(int(value), split, msb, lsb)
        depth = int(tables["depths"][cluster, symbol])
        assert depth != 0
        if int(tables["degenerate"][cluster]) == symbol:
            depth = 0
        stream |= (int(tables["bits"][cluster, symbol]) | (extra << depth)) << at
        at += depth + count
    return stream, at


def to_bytes(stream: int, bits: int) -> bytes:
    return stream.to_bytes((bits + 7) // 8, "little")


def sample_tokens(seed: int, n: int, contexts: int):
    rng = np.random.default_rng(seed)
    ctx = rng.integers(0, contexts, n).astype(np.uint16)
    values = (rng.geometric(0.25 + 0.5 * (ctx % 3 == 0), n) - 1).astype(np.uint32)
    big = rng.random(n) < 0.01
    values[big] = rng.integers(0, 2**32, int(big.sum()), dtype=np.uint64).astype(np.uint32)
    return values, ctx


@pytest.mark.parametrize("kind", ["prefix", "ans", "ans_high_density", "ans_rate"])
def test_model_matches_reference_writer(kind):
    values, contexts = sample_tokens(3, 4000, 24)
    offsets = np.array([0, 1, 1, 700, 2500, 4000], np.uint32)
    code = ref.RefEntropyCode(kind, values, contexts, offsets, 24)
    tables = code.tables()
    want = code.write(values, contexts, offsets)
    counts = code.count(values, contexts, offsets)
    assert np.array_equal(counts, want["bit_counts"])
    model = model_prefix if tables["mode"] == 0 else model_ans
    for s in range(offsets.size - 1):
        a, b = offsets[s], offsets[s + 1]
        stream, bits = model(tables, values[a:b], contexts[a:b])
        assert bits == want["bit_counts"][s], s
        lo, hi = want["byte_offsets"][s], want["byte_offsets"][s + 1]
        assert to_bytes(stream, bits) == want["bytes"][lo:hi].tobytes(), s


def test_reference_counts_match_writers_on_skewed_clusters():
    """Contexts with very different statistics give several clusters."""
    rng = np.random.default_rng(7)
    n = 20000
    contexts = rng.integers(0, 64, n).astype(np.uint16)
    p = 0.05 + 0.9 * (contexts.astype(np.float64) / 63.0)
    values = (rng.geometric(p) - 1).astype(np.uint32)
    offsets = np.linspace(0, n, 9).astype(np.uint32)
    for kind in ("prefix", "ans"):
        code = ref.RefEntropyCode(kind, values, contexts, offsets, 64)
        t = code.tables()
        assert t["cluster_count"] > 1
        w = code.write(values, contexts, offsets)
        assert np.array_equal(code.count(values, contexts, offsets), w["bit_counts"])


def test_slot_sizes_and_argument_checks_without_gpu():
    """Slot layout of gjxl_b200_entropy_write_sections (host arithmetic, no
    GPU): section s starts at ceil(B * offset / 64) + 2 s words and every
    slot holds the section's largest stream (32 + 47 bits per ANS token, 46
    per prefix token); invalid arguments are rejected before any launch."""
    from gjxl_b200 import _lib
    lib = _lib.load()
    words = lib.gjxl_b200_entropy_slot_words
    assert words(1, 1000, 4) == (47 * 1000 + 63) // 64 + 8
    assert words(0, 1000, 4) == (46 * 1000 + 63) // 64 + 8
    assert words(7, 10, 1) == 0
    rng = np.random.default_rng(9)
    offsets = np.concatenate([[0], np.cumsum(rng.integers(0, 5000, 300))])
    for mode, bits in ((1, 47), (0, 46)):
        start = [words(mode, int(o), s) for s, o in enumerate(offsets)]
        for s in range(offsets.size - 1):
            n = int(offsets[s + 1] - offsets[s])
            need = (32 + bits * n + 63) // 64 if mode == 1 else (bits * n + 63) // 64
            assert start[s + 1] - start[s] >= max(need, 1), (mode, s)
    assert lib.gjxl_b200_entropy_write_sections(None, None, None, 0, None, None, 0, None, None,
                                                None) == 1
    assert lib.gjxl_b200_entropy_count_sections(None, 1, None, None, None, None) == 1
