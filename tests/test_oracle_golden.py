"""Pin the oracle: its scan / sort / hash-set restatements must reproduce the
reference tests' own known answers (tests/golden/primitives.json, made by
tests/golden/make_golden.py from the reference tests' generators)."""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle

GOLDEN = json.loads((Path(__file__).parent / "golden" / "primitives.json").read_text())


@pytest.mark.parametrize("name", [k for k in GOLDEN if k.startswith("scan_")])
def test_oracle_scan_matches_golden(name):
    case = GOLDEN[name]
    x = np.array(case["input"], np.uint32)
    assert oracle.exclusive_sum(x).tolist() == case["exclusive"]
    assert oracle.inclusive_sum(x).tolist() == case["inclusive"]


@pytest.mark.parametrize("name", [k for k in GOLDEN if k.startswith("sort_")])
def test_oracle_sort_matches_golden(name):
    case = GOLDEN[name]
    dt = np.uint64 if case["key_bytes"] == 8 else np.uint32
    keys = np.array(case["keys"], dt)
    vals = np.array(case["values"], np.uint32) if "values" in case else None
    k, v = oracle.stable_sort_pairs(keys, vals, case["key_bits"])
    assert k.tolist() == case["sorted_keys"]
    if vals is not None:
        assert v.tolist() == case["sorted_values"]


def test_oracle_scan_wraps_u32():
    x = np.full(5, 0xFFFFFFFF, np.uint32)
    assert oracle.exclusive_sum(x).tolist() == [0, 0xFFFFFFFF, 0xFFFFFFFE,
                                                0xFFFFFFFD, 0xFFFFFFFC]


def test_oracle_hash_set_statuses():
    ins = np.array([5, 7, 5, 2**64 - 1, 2**64 - 2, 9], np.uint64)
    st, found = oracle.hash_set(ins, np.array([5, 6, 7, 9, 2**64 - 1], np.uint64))
    # Inserted, Inserted, AlreadyPresent, InvalidKey, InvalidKey, Inserted
    assert st.tolist() == [1, 1, 7, 5, 5, 1]
    assert found.tolist() == [1, 0, 1, 1, 0]


def test_oracle_mt_baselines_match_single_thread():
    rng = np.random.default_rng(11)
    x = rng.integers(0, 256, 100_003, dtype=np.uint32)
    out = np.empty_like(x)
    oracle.lib().orc_exclusive_scan_u32_mt(x.ctypes.data, out.ctypes.data, x.size, 4)
    assert np.array_equal(out, oracle.exclusive_sum(x))
    keys = rng.integers(0, 2**60, 50_001, dtype=np.uint64)
    vals = np.arange(keys.size, dtype=np.uint32)
    k1, v1 = oracle.stable_sort_pairs(keys, vals, 60)
    k2, v2 = keys.copy(), vals.copy()
    oracle.lib().orc_radix_sort_pairs_u64_mt(k2.ctypes.data, v2.ctypes.data,
                                             k2.size, 60, 3)
    assert np.array_equal(k1, k2) and np.array_equal(v1, v2)
