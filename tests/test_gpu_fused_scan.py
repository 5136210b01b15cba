"""Fused transform -> scan -> post-op (voxel_b200_fused_scan.cuh) from a
user's kernels (tests/user_fused_scan.cu, built here with nvcc): stream
compaction with an exclusive sum, a running signed maximum, u64 popcount
offsets and double sums, against numpy, from one element to many tiles;
and the workspace rejection of the reference (null / short workspace)."""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent
SIZES = [1, 7, 2048, 2049, 100_003, 3_000_017]


@pytest.fixture(scope="module")
def fused(tmp_path_factory):
    if shutil.which("nvcc") is None:
        pytest.skip("nvcc is needed to build the user kernels")
    out = tmp_path_factory.mktemp("fused") / "libfused.so"
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2",
           "-shared", "-Xcompiler", "-fPIC", str(ROOT / "tests" / "user_fused_scan.cu"),
           "-I", str(ROOT / "include"), "-o", str(out)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    lib = C.CDLL(str(out))
    for n in ("compact", "running_max", "popc_offsets", "real_sums"):
        getattr(lib, n).argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_size_t]
        getattr(lib, n).restype = C.c_int
    for n in ("compact_ws", "max_ws", "popc_ws", "real_ws"):
        getattr(lib, n).argtypes = [C.c_uint32]
        getattr(lib, n).restype = C.c_size_t
    return lib


def ws(lib, name, n, cuda):
    size = getattr(lib, name)(n)
    buf = torch.empty(max(size, 1), dtype=torch.uint8, device=cuda)
    return buf, size


@pytest.mark.parametrize("n", SIZES)
def test_stream_compaction(cuda, fused, n):
    rng = np.random.default_rng(n)
    x = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    dx = torch.from_numpy(x.view(np.int32)).to(cuda)
    out = torch.full((n,), -1, dtype=torch.int32, device=cuda)
    buf, size = ws(fused, "compact_ws", n, cuda)
    assert fused.compact(dx.data_ptr(), out.data_ptr(), n, buf.data_ptr(), size) == 0
    kept = x[x % 3 == 0]
    got = out.cpu().numpy().view(np.uint32)
    assert np.array_equal(got[: kept.size], kept)


@pytest.mark.parametrize("n", SIZES)
def test_running_max_and_popcount_offsets(cuda, fused, n):
    rng = np.random.default_rng(n + 1)
    x = rng.integers(-2**31, 2**31, n, dtype=np.int64).astype(np.int32)
    dx = torch.from_numpy(x).to(cuda)
    out = torch.empty(n, dtype=torch.int32, device=cuda)
    buf, size = ws(fused, "max_ws", n, cuda)
    assert fused.running_max(dx.data_ptr(), out.data_ptr(), n, buf.data_ptr(), size) == 0
    assert np.array_equal(out.cpu().numpy(), np.maximum.accumulate(x))
    w = rng.integers(0, 2**63, n, dtype=np.uint64) * 2 + 1
    dw = torch.from_numpy(w.view(np.int64)).to(cuda)
    out = torch.empty(n, dtype=torch.int64, device=cuda)
    buf, size = ws(fused, "popc_ws", n, cuda)
    assert fused.popc_offsets(dw.data_ptr(), out.data_ptr(), n, buf.data_ptr(), size) == 0
    pc = np.array([bin(int(v)).count("1") for v in w[: min(n, 200_000)]], np.uint64)
    expect = np.concatenate([[0], np.cumsum(pc)[:-1]]).astype(np.uint64)
    assert np.array_equal(out.cpu().numpy().view(np.uint64)[: pc.size], expect)


@pytest.mark.parametrize("n", [2049, 1_000_003])
def test_double_sums_within_tolerance(cuda, fused, n):
    """Floating point: the tile order differs from a serial sum; the
    tolerance is 1e-9 relative to the running sum of magnitudes."""
    rng = np.random.default_rng(7)
    x = rng.normal(0.0, 1.0, n)
    dx = torch.from_numpy(x).to(cuda)
    out = torch.empty(n, dtype=torch.float64, device=cuda)
    buf, size = ws(fused, "real_ws", n, cuda)
    assert fused.real_sums(dx.data_ptr(), out.data_ptr(), n, buf.data_ptr(), size) == 0
    ref = np.cumsum(x)
    scale = np.cumsum(np.abs(x))
    assert (np.abs(out.cpu().numpy() - ref) <= 1e-9 * scale + 1e-12).all()


def test_workspace_rules(cuda, fused):
    n = 100_000
    dx = torch.zeros(n, dtype=torch.int32, device=cuda)
    out = torch.zeros(n, dtype=torch.int32, device=cuda)
    size = fused.compact_ws(n)
    assert size > 0 and fused.compact_ws(2048) == 0  # one tile needs none
    assert fused.compact(dx.data_ptr(), out.data_ptr(), n, None, 0) == 1  # cudaErrorInvalidValue
    buf = torch.empty(size, dtype=torch.uint8, device=cuda)
    assert fused.compact(dx.data_ptr(), out.data_ptr(), n, buf.data_ptr(), size - 1) == 1
    assert fused.compact(dx.data_ptr(), out.data_ptr(), 0, None, 0) == 0
