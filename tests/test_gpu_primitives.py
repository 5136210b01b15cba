"""GPU parity of scan and radix sort against the oracle and the reference
tests' golden vectors, through the C ABI.  Bit-exact (integer work)."""
import json
from pathlib import Path

import numpy as np
import pytest
import torch

import oracle
import voxel_b200 as vx

pytestmark = pytest.mark.gpu
GOLDEN = json.loads((Path(__file__).parent / "golden" / "primitives.json").read_text())


def to_dev(a: np.ndarray, device):
    if a.dtype == np.uint64:
        return torch.from_numpy(a.view(np.int64)).to(device)
    return torch.from_numpy(a.view(np.int32)).to(device)


def to_np(t: torch.Tensor, dtype):
    return t.cpu().numpy().view(dtype)


@pytest.mark.parametrize("name", [k for k in GOLDEN if k.startswith("scan_")])
def test_scan_golden(cuda, name):
    case = GOLDEN[name]
    x = np.array(case["input"], np.uint32)
    d = to_dev(x, cuda)
    vx.exclusive_sum(d)
    assert to_np(d, np.uint32).tolist() == case["exclusive"]
    d = to_dev(x, cuda)
    vx.inclusive_sum(d)
    assert to_np(d, np.uint32).tolist() == case["inclusive"]


@pytest.mark.parametrize("n", [0, 1, 2, 31, 32, 33, 4095, 4096, 4097, 8191,
                               8192, 8193, 65536 * 3 + 7, 1 << 22, 5_000_011])
def test_scan_sizes_match_oracle(cuda, n):
    rng = np.random.default_rng(n)
    x = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    d = to_dev(x, cuda)
    ws = torch.empty(max(vx.lib().vx_scan_workspace_size(n), 1), dtype=torch.uint8, device=cuda)
    vx.exclusive_sum(d, ws)
    assert np.array_equal(to_np(d, np.uint32), oracle.exclusive_sum(x))
    if n:
        assert vx.workspace_status(ws) == 0


def test_scan_unaligned_pointer(cuda):
    x = np.arange(100_003, dtype=np.uint32) * 7
    d = to_dev(x, cuda)
    sub = d[1:]  # 4-byte offset: not 16-byte aligned
    vx.exclusive_sum(sub)
    assert np.array_equal(to_np(sub, np.uint32), oracle.exclusive_sum(x[1:]))


@pytest.mark.parametrize("n", [3, 257, 100_000, 1 << 20, 3_000_017])
def test_scan_u64_and_workspace_reuse(cuda, n):
    rng = np.random.default_rng(n + 1)
    x = rng.integers(0, 2**63, n, dtype=np.uint64)
    ws = torch.empty(vx.lib().vx_scan_workspace_size(n), dtype=torch.uint8, device=cuda)
    for _ in range(2):  # workspace reuse (test_cuda_scan.cu:818)
        d = to_dev(x, cuda)
        vx.exclusive_sum(d, ws)
        assert np.array_equal(to_np(d, np.uint64), oracle.exclusive_sum(x))


def test_scan_rejects_bad_arguments(cuda):
    lib = vx.lib()
    d = torch.zeros(1025, dtype=torch.int32, device=cuda)
    ws = torch.empty(4, dtype=torch.uint8, device=cuda)
    s = vx.stream_handle()
    assert lib.vx_scan_exclusive_sum_u32(d.data_ptr(), 1025, ws.data_ptr(), 4, s) == vx.VX_ERR_INVALID_VALUE
    assert lib.vx_scan_exclusive_sum_u32(None, 5, ws.data_ptr(), 4, s) == vx.VX_ERR_INVALID_VALUE
    assert lib.vx_scan_exclusive_sum_u32(None, 0, None, 0, s) == vx.VX_OK


@pytest.mark.parametrize("name", [k for k in GOLDEN if k.startswith("sort_")])
def test_sort_golden(cuda, name):
    case = GOLDEN[name]
    dt = np.uint64 if case["key_bytes"] == 8 else np.uint32
    keys = to_dev(np.array(case["keys"], dt), cuda)
    vals = to_dev(np.array(case["values"], np.uint32), cuda) if "values" in case else None
    vx.sort_pairs(keys, vals, case["key_bits"])
    assert to_np(keys, dt).tolist() == case["sorted_keys"]
    if vals is not None:
        assert to_np(vals, np.uint32).tolist() == case["sorted_values"]


@pytest.mark.parametrize("key_bytes,key_bits,n", [
    (4, 32, 2), (4, 32, 3071), (4, 32, 3072), (4, 32, 4097), (4, 32, 1 << 20),
    (4, 12, 1 << 20), (4, 17, 2_000_003), (8, 64, 50_001), (8, 60, 1 << 21),
    (8, 33, 777_777), (8, 8, 100_000)])
def test_sort_matches_oracle(cuda, key_bytes, key_bits, n):
    rng = np.random.default_rng(key_bits * 7 + n)
    dt = np.uint64 if key_bytes == 8 else np.uint32
    keys = rng.integers(0, 2**63, n, dtype=np.uint64).astype(dt)
    keys[::7] = keys[0]  # plenty of duplicate keys: stability matters
    vals = np.arange(n, dtype=np.uint32)
    dk, dv = to_dev(keys, cuda), to_dev(vals, cuda)
    vx.sort_pairs(dk, dv, key_bits)
    ek, ev = oracle.stable_sort_pairs(keys, vals, key_bits)
    assert np.array_equal(to_np(dk, dt), ek)
    assert np.array_equal(to_np(dv, np.uint32), ev)


def test_sort_morton_clustered(cuda):
    """Clustered u64 Morton keys (64 Gaussian blobs), the skewed-digit case."""
    rng = np.random.default_rng(4)
    n = 1 << 20
    centers = rng.integers(0, 1 << 20, (64, 3))
    pts = centers[rng.integers(0, 64, n)] + rng.normal(0, 2**14, (n, 3)).astype(np.int64)
    pts = np.clip(pts, 0, (1 << 20) - 1).astype(np.uint64)
    key = np.zeros(n, np.uint64)
    for b in range(20):
        for a in range(3):
            key |= ((pts[:, a] >> np.uint64(b)) & np.uint64(1)) << np.uint64(3 * b + a)
    vals = np.arange(n, dtype=np.uint32)
    dk, dv = to_dev(key, cuda), to_dev(vals, cuda)
    vx.sort_pairs(dk, dv, 60)
    ek, ev = oracle.stable_sort_pairs(key, vals, 60)
    assert np.array_equal(to_np(dk, np.uint64), ek)
    assert np.array_equal(to_np(dv, np.uint32), ev)


def test_sort_keys_only_and_rejections(cuda):
    rng = np.random.default_rng(9)
    keys = rng.integers(0, 2**32, 12345, dtype=np.uint64).astype(np.uint32)
    dk = to_dev(keys, cuda)
    vx.sort_pairs(dk, None, 32)
    assert np.array_equal(to_np(dk, np.uint32), np.sort(keys, kind="stable"))
    lib = vx.lib()
    s = vx.stream_handle()
    ws = torch.empty(8, dtype=torch.uint8, device=cuda)
    assert lib.vx_sort_pairs_u32(dk.data_ptr(), None, 12345, 32, ws.data_ptr(), 8, s) == vx.VX_ERR_INVALID_VALUE
    assert lib.vx_sort_pairs_u32(dk.data_ptr(), None, 12345, 0, None, 0, s) == vx.VX_ERR_INVALID_VALUE
    assert lib.vx_sort_pairs_u32(dk.data_ptr(), None, 1, 32, None, 0, s) == vx.VX_OK
