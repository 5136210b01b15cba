"""The allocation-free exclusive sum (for callers that cannot allocate device
memory where they scan) must give the same result as the regular entry point
with a caller workspace, call after call: its scratch lives in the library
and keeps the previous call's contents, so the second call checks that the
part it uses is cleared.  Collected last (file name) so that a run that stops
at the first failure has run every other test first."""
import numpy as np
import pytest
import torch

import voxel_b200 as vx

pytestmark = pytest.mark.gpu


def regular(x: np.ndarray, dev) -> np.ndarray:
    d = torch.from_numpy(x.view(np.int32)).to(dev)
    lib = vx.lib()
    ws = torch.empty(max(lib.vx_scan_workspace_size(x.size), 1), dtype=torch.uint8, device=dev)
    assert lib.vx_scan_exclusive_sum_u32(d.data_ptr(), x.size, ws.data_ptr(), ws.numel(),
                                         vx.stream_handle()) == 0
    return d.cpu().numpy().view(np.uint32)


def no_alloc(x: np.ndarray, dev) -> np.ndarray:
    d = torch.from_numpy(x.view(np.int32)).to(dev)
    assert vx.lib().vx_scan_exclusive_sum_u32_noalloc(d.data_ptr(), x.size,
                                                      vx.stream_handle()) == 0
    return d.cpu().numpy().view(np.uint32)


def test_no_alloc_scan_matches_regular_on_consecutive_calls():
    assert torch.cuda.is_available()
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(2024)
    # two calls in a row, the second smaller than the first and then larger
    for n in (3_000_017, 1_000_003, 5_000_000):
        x = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
        assert np.array_equal(no_alloc(x, dev), regular(x, dev))
    x = np.full(70_000, 0xFFFFFFFF, np.uint32)  # wrapping sums
    assert np.array_equal(no_alloc(x, dev), regular(x, dev))
    # the look-back status of the last call is readable without a workspace
    assert vx.lib().vx_scan_noalloc_status(vx.stream_handle()) == vx.VX_OK


def test_no_alloc_scan_rejects_counts_beyond_its_scratch():
    assert torch.cuda.is_available()
    d = torch.arange(8, dtype=torch.int32, device="cuda:0")
    lib = vx.lib()
    st = lib.vx_scan_exclusive_sum_u32_noalloc(d.data_ptr(), (1 << 28) + 1, vx.stream_handle())
    assert st == vx.VX_ERR_CAPACITY
    assert d.cpu().tolist() == list(range(8))  # nothing touched
    assert lib.vx_scan_exclusive_sum_u32_noalloc(None, 0, vx.stream_handle()) == vx.VX_OK
