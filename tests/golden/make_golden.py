#!/usr/bin/env python3
"""Regenerates the committed golden fixtures from the reference.

Run in a checkout where oracle/_ref/libgjxl_ref.so has been built from the
reference sources (`make -C oracle`). Writes tests/golden/butteraugli.npz:

* the reference test suite's four scalar-libjxl full-map goldens
  (flat, texture, contrast, chromatic fixtures at 32x24), with the fixture
  images they were computed on (the reference's own MakeFixture), and the
  reference CPU implementation's map and score on the same inputs;
* the reference's synthetic differential corpus (impulses at 1x1..8x8,
  gradient, texture, contrast, chromatic, random, option variants) with the
  reference CPU implementation's maps and scores.
"""

from __future__ import annotations

import ctypes
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import ref  # noqa: E402

# FixtureKind numbering of the reference's tests/butteraugli_fixtures.h.
KIND = {"flat": 0, "texture": 1, "contrast": 2, "chromatic": 3, "gradient": 4,
        "intermediate": 5, "identity_texture": 6, "impulse": 7, "random_low": 8,
        "random_normal": 9, "random_wide": 10}

# The reference's BuildSyntheticDifferentialCorpus (tests/butteraugli_fixtures.cpp).
CORPUS = ([("identity_texture", 32, 24, 0x12345678, 0, (1.0, 1.0, 80.0))]
          + [("impulse", w, h, 0x12345678, c, (1.0, 1.0, 80.0))
             for (w, h) in ((1, 1), (3, 7), (7, 3), (8, 8)) for c in range(3)]
          + [("gradient", 9, 13, 0x12345678, 0, (1.0, 1.0, 80.0)),
             ("texture", 32, 24, 0x12345678, 0, (1.0, 1.0, 80.0)),
             ("contrast", 33, 17, 0x12345678, 0, (1.0, 1.0, 80.0)),
             ("chromatic", 17, 29, 0x12345678, 0, (1.0, 1.0, 80.0)),
             ("random_low", 31, 23, 0x9E3779B9, 0, (1.0, 1.0, 80.0)),
             ("random_normal", 13, 9, 0x243F6A88, 0, (1.0, 1.0, 80.0)),
             ("random_wide", 23, 15, 0xB7E15162, 0, (1.0, 1.0, 80.0)),
             ("texture", 32, 24, 0x12345678, 0, (1.6, 1.0, 80.0)),
             ("texture", 32, 24, 0x12345678, 0, (1.0, 0.75, 80.0)),
             ("texture", 32, 24, 0x12345678, 0, (1.0, 1.0, 255.0))])


def fixture(kind, w, h, seed, channel, options):
    lib = ref.lib()
    fn = lib.gjxl_ref_butteraugli_fixture
    fn.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_uint32,
                   ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    r = np.zeros((3, h, w), np.float32)
    d = np.zeros((3, h, w), np.float32)
    o = np.asarray(options, np.float32)
    assert fn(KIND[kind], w, h, seed, channel, r.ctypes.data, d.ctypes.data, o.ctypes.data) == 0
    return r, d


def reference_map(r, d, options):
    lib = ref.lib()
    fn = lib.gjxl_ref_butteraugli_options
    fn.argtypes = [ctypes.c_void_p] * 2 + [ctypes.c_size_t] * 2 + [ctypes.c_void_p] * 3
    _, h, w = r.shape
    m = np.zeros((h, w), np.float32)
    s = np.zeros(1, np.float64)
    o = np.asarray(options, np.float32)
    assert fn(r.ctypes.data, d.ctypes.data, w, h, o.ctypes.data, m.ctypes.data, s.ctypes.data) == 0
    return m, float(s[0])


def main():
    out = {}
    lib = ref.lib()
    fn = lib.gjxl_ref_butteraugli_golden_full_map
    fn.argtypes = [ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p]
    for index, name in enumerate(["flat", "texture", "contrast", "chromatic"]):
        r, d = fixture(name, 32, 24, 0x12345678, 0, (1.0, 1.0, 80.0))
        bits = np.zeros(32 * 24, np.uint32)
        score_bits = np.zeros(1, np.uint64)
        assert fn(index, bits.ctypes.data, score_bits.ctypes.data) == 32 * 24
        out[f"golden{index}_reference"] = r
        out[f"golden{index}_distorted"] = d
        out[f"golden{index}_libjxl_map"] = bits.view(np.float32).reshape(24, 32)
        out[f"golden{index}_libjxl_score"] = score_bits.view(np.float64)
        m, s = reference_map(r, d, (1.0, 1.0, 80.0))
        out[f"golden{index}_ref_map"] = m
        out[f"golden{index}_ref_score"] = np.array([s])
    for i, (kind, w, h, seed, channel, options) in enumerate(CORPUS):
        r, d = fixture(kind, w, h, seed, channel, options)
        m, s = reference_map(r, d, options)
        out[f"corpus{i}_reference"] = r
        out[f"corpus{i}_distorted"] = d
        out[f"corpus{i}_options"] = np.asarray(options, np.float32)
        out[f"corpus{i}_ref_map"] = m
        out[f"corpus{i}_ref_score"] = np.array([s])
    out["corpus_count"] = np.array([len(CORPUS)])
    np.savez_compressed(Path(__file__).with_name("butteraugli.npz"), **out)


if __name__ == "__main__":
    main()
