"""Pins the Butteraugli oracle: the reference's CPU implementation reproduces
the reference test suite's scalar-libjxl golden maps (committed in
tests/golden/butteraugli.npz) within the reference's own tolerance, and the
committed corpus maps are what the oracle computes now."""

from pathlib import Path

import numpy as np
import pytest

from oracle import ref

GOLDEN = np.load(Path(__file__).parent / "golden" / "butteraugli.npz")


@pytest.mark.parametrize("index", range(4))
def test_oracle_matches_libjxl_goldens(index):
    r = GOLDEN[f"golden{index}_reference"]
    d = GOLDEN[f"golden{index}_distorted"]
    m, s = ref.butteraugli(r, d)
    expected = GOLDEN[f"golden{index}_libjxl_map"]
    # The reference's tolerance between its native and libjxl's scalar
    # Butteraugli (kScalarDispatchTolerance in tests/butteraugli_test_tolerances.h:
    # 3e-4 for full maps, 1e-4 for scores).
    assert np.abs(m - expected).max() <= 3e-4
    assert abs(s - float(GOLDEN[f"golden{index}_libjxl_score"][0])) <= 1e-4


def test_corpus_fixtures_are_current():
    for i in range(int(GOLDEN["corpus_count"][0])):
        r = GOLDEN[f"corpus{i}_reference"]
        d = GOLDEN[f"corpus{i}_distorted"]
        opts = GOLDEN[f"corpus{i}_options"]
        if opts[0] != 1.0 or opts[1] != 1.0:
            continue
        m, s = ref.butteraugli(r, d, float(opts[2]))
        assert np.array_equal(m.view(np.uint32), GOLDEN[f"corpus{i}_ref_map"].view(np.uint32))
        assert s == float(GOLDEN[f"corpus{i}_ref_score"][0])
