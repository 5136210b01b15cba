"""u32 -> u32 slab hash map against the reference's own map tests
(test/cuda/test_cuda_slab_hash.cu: insert-or-replace, first available or
matching slot, duplicates in one batch, erase-all, overflow) and against
dict semantics on random batches."""
import numpy as np
import pytest
import torch

import voxel_b200 as vx

pytestmark = pytest.mark.gpu
SLOTS = 15  # kSlabHashMapSlotsPerSlab


def u32(a, device):
    return torch.from_numpy(np.asarray(a, np.uint32).view(np.int32)).to(device)


def ops(m, cuda):
    def ins(keys, vals):
        st = torch.zeros(len(keys), dtype=torch.int32, device=cuda)
        m.insert_or_replace(u32(keys, cuda), u32(vals, cuda), st)
        return st.cpu().numpy()

    def find(keys):
        st = torch.zeros(len(keys), dtype=torch.int32, device=cuda)
        v = m.find(u32(keys, cuda), statuses=st)
        return v.cpu().numpy().view(np.uint32), st.cpu().numpy()

    def erase(keys):
        st = torch.zeros(len(keys), dtype=torch.int32, device=cuda)
        m.erase_all(u32(keys, cuda), st)
        return st.cpu().numpy()
    return ins, find, erase


def test_reference_known_answers(cuda):
    # InsertOrReplaceUpdatesExistingValue
    ins, find, erase = ops(vx.SlabHashMap(4, 2), cuda)
    assert ins([5], [100])[0] == vx.VX_HASH_INSERTED
    assert ins([5], [200])[0] == vx.VX_HASH_REPLACED
    v, st = find([5])
    assert st[0] == vx.VX_HASH_FOUND and v[0] == 200
    # InsertOrReplaceUsesFirstAvailableOrMatchingSlot (1 bucket, 2 pool slabs)
    ins, find, erase = ops(vx.SlabHashMap(1, 2), cuda)
    n = SLOTS + 1
    assert (ins(np.arange(1, n + 1), 100 + np.arange(n)) == vx.VX_HASH_INSERTED).all()
    assert erase([1])[0] == vx.VX_HASH_ERASED
    assert ins([n], [999])[0] == vx.VX_HASH_INSERTED  # the freed first slot
    v, st = find([n])
    assert st[0] == vx.VX_HASH_FOUND and v[0] == 999
    assert erase([n])[0] == vx.VX_HASH_ERASED
    v, st = find([n])
    assert st[0] == vx.VX_HASH_NOT_FOUND and v[0] == vx.VX_HASH_NOT_FOUND_VALUE
    # DuplicateKeysInSameBatchReplaceOneSlot
    ins, find, erase = ops(vx.SlabHashMap(4, 2), cuda)
    st = ins([99] * 8, 1000 + np.arange(8))
    assert (st == vx.VX_HASH_INSERTED).sum() == 1 and (st == vx.VX_HASH_REPLACED).sum() == 7
    v, st = find([99])
    assert st[0] == vx.VX_HASH_FOUND and v[0] == 1007
    # EraseAllMarksKeyDeleted
    ins, find, erase = ops(vx.SlabHashMap(4, 2), cuda)
    ins([7, 11], [70, 110])
    assert erase([7])[0] == vx.VX_HASH_ERASED
    v, st = find([7, 11])
    assert list(st) == [vx.VX_HASH_NOT_FOUND, vx.VX_HASH_FOUND]
    assert v[0] == vx.VX_HASH_NOT_FOUND_VALUE and v[1] == 110
    # ReportsOverflowWhenSlabPoolIsFull (1 bucket, no pool)
    ins, find, erase = ops(vx.SlabHashMap(1, 0), cuda)
    st = ins(np.arange(1, SLOTS + 2), 100 + np.arange(SLOTS + 1))
    assert (st == vx.VX_HASH_INSERTED).sum() == SLOTS and (st == vx.VX_HASH_OVERFLOW).sum() == 1
    # MissingKeysReturnNotFound, reserved keys
    ins, find, erase = ops(vx.SlabHashMap(8, 4), cuda)
    v, st = find([1, 2, 3])
    assert (st == vx.VX_HASH_NOT_FOUND).all() and (v == vx.VX_HASH_NOT_FOUND_VALUE).all()
    st = ins([vx.VX_MAP_EMPTY_KEY, vx.VX_MAP_DELETED_KEY], [1, 2])
    assert (st == vx.VX_HASH_INVALID_KEY).all()


def test_random_batches_follow_dict_semantics(cuda):
    rng = np.random.default_rng(51)
    m = vx.SlabHashMap(1 << 12, 1 << 16)
    ins, find, erase = ops(m, cuda)
    model: dict[int, int] = {}
    universe = rng.choice(2**32 - 2, 400_000, replace=False).astype(np.uint32)
    for step in range(6):
        keys = rng.choice(universe, 100_000, replace=False)  # distinct within a batch
        vals = rng.integers(0, 2**32, keys.size, dtype=np.uint64).astype(np.uint32)
        st = ins(keys, vals)
        present = np.array([int(k) in model for k in keys])
        if step == 0:  # nothing erased yet: statuses are exactly dict semantics
            assert np.array_equal(st, np.where(present, vx.VX_HASH_REPLACED,
                                               vx.VX_HASH_INSERTED))
        else:
            # After erases a deleted slot can come before a present key in its
            # chain: the reference inserts a new copy there (status INSERTED,
            # found first from then on; erase_all removes every copy).
            assert np.isin(st, [vx.VX_HASH_INSERTED, vx.VX_HASH_REPLACED]).all()
            assert present[st == vx.VX_HASH_REPLACED].all()
            assert (st[~present] == vx.VX_HASH_INSERTED).all()
        model.update(zip(keys.tolist(), vals.tolist()))
        gone = rng.choice(universe, 20_000, replace=False)
        st = erase(gone)
        exp = np.array([vx.VX_HASH_ERASED if int(k) in model else vx.VX_HASH_NOT_FOUND
                        for k in gone])
        assert np.array_equal(st, exp)
        for k in gone.tolist():
            model.pop(k, None)
        q = rng.choice(universe, 50_000, replace=False)
        v, st = find(q)
        hit = np.array([int(k) in model for k in q])
        assert np.array_equal(st == vx.VX_HASH_FOUND, hit)
        assert np.array_equal(v[hit], np.array([model[int(k)] for k in q[hit]], np.uint32))
        assert (v[~hit] == vx.VX_HASH_NOT_FOUND_VALUE).all()
