"""GPU slab hash set and cuckoo map (u64 keys) against the oracle's set
semantics and the reference's status codes (slab_hash/common.cuh:18-25)."""
import numpy as np
import pytest
import torch

import oracle
import voxel_b200 as vx

pytestmark = pytest.mark.gpu


def dev64(a, device):
    return torch.from_numpy(np.ascontiguousarray(a, np.uint64).view(np.int64)).to(device)


def u32(t):
    return t.cpu().numpy().view(np.uint32)


def unique_keys(rng, n):
    k = np.unique(rng.integers(0, 2**64 - 2, int(n * 1.1) + 16, dtype=np.uint64))
    rng.shuffle(k)
    return k[:n]


@pytest.mark.parametrize("n,buckets", [(1, 1), (31, 1), (32, 4), (33, 4),
                                       (255, 16), (256, 16), (257, 16),
                                       (100_000, 8_000), (1_000_000, 83_334)])
def test_slab_set_insert_contains_matches_oracle(cuda, n, buckets):
    rng = np.random.default_rng(n)
    keys = unique_keys(rng, n)
    queries = np.concatenate([keys[: n // 2], unique_keys(rng, n)])
    rng.shuffle(queries)
    t = vx.SlabHashSet(buckets, max(64, n // 4))
    st = torch.empty(n, dtype=torch.int32, device=cuda)
    t.insert(dev64(keys, cuda), st)
    found = t.contains(dev64(queries, cuda))
    est, efound = oracle.hash_set(keys, queries)
    assert np.array_equal(u32(st), est)
    assert np.array_equal(u32(found), efound)


def test_slab_set_duplicates_reserved_keys_and_erase(cuda):
    keys = np.array([5, 7, 5, 2**64 - 1, 2**64 - 2, 9, 7, 7], np.uint64)
    t = vx.SlabHashSet(2, 16)
    st = torch.empty(keys.size, dtype=torch.int32, device=cuda)
    t.insert(dev64(keys, cuda), st)
    s = u32(st)
    assert s[3] == vx.HASH_INVALID_KEY and s[4] == vx.HASH_INVALID_KEY
    for k in (5, 7, 9):  # exactly one insert per distinct key wins
        idx = np.where(keys == k)[0]
        assert (s[idx] == vx.HASH_INSERTED).sum() == 1
        assert set(s[idx]) <= {vx.HASH_INSERTED, vx.HASH_ALREADY_PRESENT}
    es = torch.empty(3, dtype=torch.int32, device=cuda)
    t.erase(dev64(np.array([7, 8, 7], np.uint64), cuda), es)
    assert u32(es).tolist() == [vx.HASH_ERASED, vx.HASH_NOT_FOUND, vx.HASH_NOT_FOUND]
    f = t.contains(dev64(np.array([5, 7, 9], np.uint64), cuda))
    assert u32(f).tolist() == [1, 0, 1]
    # an erased slot is reused by a later insert
    t.insert(dev64(np.array([7], np.uint64), cuda), st[:1])
    assert u32(st[:1]).tolist() == [vx.HASH_INSERTED]


def test_slab_set_pool_overflow_reports_overflow(cuda):
    rng = np.random.default_rng(3)
    keys = unique_keys(rng, 200)
    t = vx.SlabHashSet(1, 2)  # 1 bucket + 2 pool slabs = 45 keys at most
    st = torch.empty(200, dtype=torch.int32, device=cuda)
    t.insert(dev64(keys, cuda), st)
    s = u32(st)
    # racing chain growth may leave a pool slab unused, so at most 45 fit
    assert 15 <= (s == vx.HASH_INSERTED).sum() <= 45
    assert (s == vx.HASH_INSERTED).sum() + (s == vx.HASH_OVERFLOW).sum() == 200
    f = u32(t.contains(dev64(keys, cuda)))
    assert np.array_equal(f, (s == vx.HASH_INSERTED).astype(np.uint32))


@pytest.mark.parametrize("n,load", [(1, 0.5), (1000, 0.5), (1_000_000, 0.8),
                                    (3_000_000, 0.8)])
def test_cuckoo_insert_find(cuda, n, load):
    rng = np.random.default_rng(n + 17)
    keys = unique_keys(rng, n)
    vals = rng.integers(0, 2**32 - 1, n, dtype=np.uint64).astype(np.uint32)
    m = vx.CuckooMap(int(n / load) + 1, 1000)
    st = torch.empty(n, dtype=torch.int32, device=cuda)
    m.insert(dev64(keys, cuda), torch.from_numpy(vals.view(np.int32)).to(cuda), st)
    assert (u32(st) == vx.HASH_INSERTED).all()
    assert m.dropped() == 0
    misses = unique_keys(rng, n)
    q = np.concatenate([keys, misses])
    out = u32(m.find(dev64(q, cuda)))
    inserted = set(keys.tolist())
    expect_miss = np.array([k not in inserted for k in misses.tolist()])
    assert np.array_equal(out[:n], vals)
    assert (out[n:][expect_miss] == vx.HASH_NOT_FOUND_VALUE).all()


def test_cuckoo_replace_and_overflow(cuda):
    m = vx.CuckooMap(64, 8)
    k = dev64(np.array([11, 12], np.uint64), cuda)
    m.insert(k, torch.tensor([1, 2], dtype=torch.int32, device=cuda))
    st = torch.empty(1, dtype=torch.int32, device=cuda)
    m.insert(k[:1], torch.tensor([99], dtype=torch.int32, device=cuda), st)
    assert u32(st).tolist() == [vx.HASH_REPLACED]
    assert u32(m.find(k)).tolist() == [99, 2]
    # over-full table: chains run out, every drop is reported and counted
    rng = np.random.default_rng(5)
    keys = unique_keys(rng, 200)
    t = vx.CuckooMap(64, 16)
    st = torch.empty(200, dtype=torch.int32, device=cuda)
    t.insert(dev64(keys, cuda), None, st)
    s = u32(st)
    assert set(s.tolist()) <= {vx.HASH_INSERTED, vx.HASH_OVERFLOW}
    assert (s == vx.HASH_OVERFLOW).sum() == t.dropped() > 0
    found = u32(t.find(dev64(keys, cuda))) != vx.HASH_NOT_FOUND_VALUE
    assert found.sum() <= 64


def _mix64(x: int) -> int:
    m = (1 << 64) - 1
    x ^= x >> 30
    x = (x * 0xbf58476d1ce4e5b9) & m
    x ^= x >> 27
    x = (x * 0x94d049bb133111eb) & m
    x ^= x >> 31
    return x


_CUCKOO_SALTS = (0x9e3779b97f4a7c15, 0xc2b2ae3d27d4eb4f)


def _cuckoo_bucket(key: int, choice: int, buckets: int) -> int:
    return (_mix64(key ^ _CUCKOO_SALTS[choice]) * buckets) >> 64


def _raw_slots(m) -> np.ndarray:
    """The table's 16-byte slots {key, value | choice << 32}, copied to the host."""
    import ctypes
    v = m.device_view()
    out = np.empty((v.slot_count, 2), np.uint64)
    rt = ctypes.CDLL("libcudart.so.12")
    torch.cuda.synchronize()
    assert rt.cudaMemcpy(ctypes.c_void_p(out.ctypes.data), ctypes.c_void_p(v.slots),
                         ctypes.c_size_t(out.nbytes), 2) == 0
    return out


def test_cuckoo_replace_keeps_hash_id_through_later_evictions(cuda):
    """A replaced entry keeps the choice bits that placed it, so the evictions
    that later move it go to its other bucket: every stored entry sits in the
    bucket (two slots) its recorded choice names, and nothing is dropped."""
    n_slots = 4096
    rng = np.random.default_rng(77)
    keys = unique_keys(rng, 3200)               # final load 0.78
    vals = np.arange(keys.size, dtype=np.uint32)
    m = vx.CuckooMap(n_slots, 1000)
    half = keys.size // 2
    m.insert(dev64(keys[:half], cuda), torch.from_numpy(vals[:half].view(np.int32)).to(cuda))
    # replace every entry of the first half (values + 10^6)
    st = torch.empty(half, dtype=torch.int32, device=cuda)
    new = vals[:half] + 1_000_000
    m.insert(dev64(keys[:half], cuda), torch.from_numpy(new.view(np.int32)).to(cuda), st)
    assert (u32(st) == vx.HASH_REPLACED).all()
    # the second half evicts many of the replaced entries
    m.insert(dev64(keys[half:], cuda), torch.from_numpy(vals[half:].view(np.int32)).to(cuda))
    assert m.dropped() == 0
    expect = np.concatenate([new, vals[half:]])
    assert np.array_equal(u32(m.find(dev64(keys, cuda))), expect)
    raw = _raw_slots(m)
    empty = np.uint64(0xFFFFFFFFFFFFFFFF)
    for pos in np.nonzero(raw[:, 0] != empty)[0]:
        key, word = int(raw[pos, 0]), int(raw[pos, 1])
        assert _cuckoo_bucket(key, word >> 32, n_slots // 2) == pos // 2
