"""Content-addressed item store (AccelerationHashSet32) against the
reference's own tests (test/cuda/test_cuda_acceleration_hash.cu: empty table,
insert and find of large items, full-payload comparison, reading through the
returned pointer, overflow) and, for find_or_insert, dict semantics with
duplicates inside and across batches."""
import numpy as np
import pytest
import torch

import voxel_b200 as vx

pytestmark = pytest.mark.gpu


def fill_items(count, width, seed=0):
    """The reference tests' item generator."""
    i = np.arange(count, dtype=np.uint64)[:, None]
    w = np.arange(width, dtype=np.uint64)[None, :]
    return (0x10000 + seed * 97 + i * 131 + w * 17).astype(np.uint32)


def dev(a, cuda):
    return torch.from_numpy(np.ascontiguousarray(a, np.uint32).view(np.int32)).to(cuda)


def test_reference_cases(cuda):
    # EmptyTableFindsNothing
    s = vx.ItemSet(2, 64)
    p, st = s.find(dev(fill_items(4, 2), cuda))
    assert (st.cpu() == vx.VX_HASH_NOT_FOUND).all() and (p.cpu() == 0).all()
    # InsertAndFindLargeItems / ReadsPayloadFromReturnedPointer
    s = vx.ItemSet(6, 64)
    items = fill_items(16, 6)
    p, st = s.insert_unique_unchecked(dev(items, cuda))
    assert (st.cpu() == vx.VX_HASH_INSERTED).all() and (p.cpu() != 0).all()
    q, st = s.find(dev(items, cuda))
    assert (st.cpu() == vx.VX_HASH_FOUND).all() and torch.equal(q, p)
    out, st = s.read(p)
    assert (st.cpu() == vx.VX_HASH_FOUND).all()
    assert np.array_equal(out.cpu().numpy().view(np.uint32).reshape(-1, 6), items)
    # FindComparesFullPayload
    s = vx.ItemSet(2, 64)
    s.insert_unique_unchecked(dev([[1, 2]], cuda))
    p, st = s.find(dev([[1, 3]], cuda))
    assert st.cpu()[0] == vx.VX_HASH_NOT_FOUND and p.cpu()[0] == 0
    # ReportsOverflowWhenNoSlabCanGrow: capacity for 31 items, 32 inserted
    s = vx.ItemSet(2, 31)
    p, st = s.insert_unique_unchecked(dev(fill_items(32, 2), cuda))
    st = st.cpu().numpy()
    assert (st == vx.VX_HASH_INSERTED).sum() == 31 and (st == vx.VX_HASH_OVERFLOW).sum() == 1
    assert s.count() == 31
    # reads of null / unknown pointers
    out, st = s.read(torch.tensor([0, 10_000], dtype=torch.int32, device=cuda))
    assert (st.cpu() == vx.VX_HASH_NOT_FOUND).all() and (out.cpu() == 0).all()


@pytest.mark.parametrize("width", [1, 3, 9])
def test_find_or_insert_dedups(cuda, width):
    rng = np.random.default_rng(width)
    universe = rng.integers(0, 2**32, (50_000, width), dtype=np.uint64).astype(np.uint32)
    s = vx.ItemSet(width, 60_000)
    seen: dict[bytes, int] = {}
    for _ in range(4):
        pick = universe[rng.integers(0, len(universe), 40_000)]  # duplicates inside too
        p, st = s.find_or_insert(dev(pick, cuda))
        p, st = p.cpu().numpy(), st.cpu().numpy()
        assert (p != 0).all()
        assert np.isin(st, [vx.VX_HASH_INSERTED, vx.VX_HASH_FOUND]).all()
        for row, ptr_ in zip(pick, p):
            key = row.tobytes()
            assert seen.setdefault(key, int(ptr_)) == int(ptr_)  # one pointer per content
        new_keys = {r.tobytes() for r, x in zip(pick, st) if x == vx.VX_HASH_INSERTED}
        assert len(new_keys) == (st == vx.VX_HASH_INSERTED).sum()  # each inserted once
    assert s.count() == len(seen)
    ptrs = torch.tensor(list(seen.values()), dtype=torch.int32, device=cuda)
    out, st = s.read(ptrs)
    got = out.cpu().numpy().view(np.uint32).reshape(-1, width)
    assert [r.tobytes() for r in got] == list(seen.keys())
