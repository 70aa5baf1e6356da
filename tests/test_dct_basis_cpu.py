"""The DCT bases compiled into the transform kernels (csrc/dct_basis.inc) are
the reference's double-precision bases (src/codec/dct.cpp:21-41): the
committed literals equal what the generator computes with the C library's
cos, and each 1-D forward basis inverts the inverse basis to FP64 accuracy."""

import importlib.util
import re
from pathlib import Path

import numpy as np

CSRC = Path(__file__).resolve().parent.parent / "gjxl_b200" / "csrc"


def load_generator():
    spec = importlib.util.spec_from_file_location("gen_dct_basis", CSRC / "gen_dct_basis.py")
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def committed_tables():
    text = (CSRC / "dct_basis.inc").read_text()
    tables = {}
    for name, body in re.findall(r"kDct(\w+)\[\d+\] = \{(.*?)\};", text, re.S):
        values = re.findall(r"(-?0x[0-9a-f.]+p[+-]?\d+)f?", body)
        tables[name] = np.array([float.fromhex(v) for v in values])
    return tables


def test_committed_basis_matches_generator():
    gen = load_generator()
    assert (CSRC / "dct_basis.inc").read_text() == gen.render()


def test_bases_are_inverse_pairs():
    tables = committed_tables()
    for n in (8, 16, 32):
        forward = tables[f"Forward{n}"].reshape(n, n)
        inverse = tables[f"Inverse{n}"].reshape(n, n)
        # X[f] = sum_s x[s] forward[f][s] and x[s] = sum_f X[f] inverse[f][s].
        product = inverse.T @ forward
        assert np.abs(product - np.eye(n)).max() < 1e-14


def test_transposed_forward_tables():
    tables = committed_tables()
    for n in (8, 16, 32):
        forward = tables[f"Forward{n}"].reshape(n, n)
        assert np.array_equal(tables[f"ForwardT{n}"].reshape(n, n), forward.T)


def test_staged_tables_equal_constant_tables():
    tables = committed_tables()
    assert np.array_equal(tables["StagedForwardT32"], tables["ForwardT32"])
    assert np.array_equal(tables["StagedInverse32"], tables["Inverse32"])


def test_single_precision_tables_are_rounded_double_tables():
    """The FP32 tables of the fast cost mode are the double bases rounded to
    nearest float."""
    tables = committed_tables()
    for direction in ("Forward", "Inverse"):
        for n in (8, 16):
            double = tables[f"{direction}{n}"]
            single = tables[f"{direction}{n}F"]
            assert np.array_equal(single, double.astype(np.float32).astype(np.float64))
