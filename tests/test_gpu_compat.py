"""A C++ program written against the reference's API (algo::cuda::sort /
scan, algo::svt::hash_dag_gpu, algo::svt::cuda via
include/voxel_b200_compat.hpp) is built with nvcc and run: its sorts must
order keys exactly as the reference's KeyBits contract says (the default
config orders u64 keys by their low 32 bits, stably), carry any number of
value arrays, sort UIntKey<W> keys, scan with operators, report the
reference's error codes, and its edits must land in the structures."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle

ROOT = Path(__file__).resolve().parent.parent
N = 200_003
NV = 5_000
INVALID = 1  # cudaErrorInvalidValue


def build(tmp_path: Path) -> Path:
    exe = tmp_path / "compat_program"
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2",
           str(ROOT / "tests" / "compat_program.cu"), "-I", str(ROOT / "include"),
           "-L", str(ROOT / "voxel_b200"), "-lvoxel_b200",
           f"-Xlinker=-rpath,{ROOT / 'voxel_b200'}", "-o", str(exe)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return exe


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="no nvcc")
def test_compat_program_builds(tmp_path):
    build(tmp_path)


class Reader:
    def __init__(self, raw: bytes):
        self.raw, self.o = raw, 0

    def take(self, dtype, n):
        a = np.frombuffer(self.raw, dtype, n, self.o)
        self.o += a.nbytes
        return a

    def status(self):
        return int(self.take(np.int32, 1)[0])


@pytest.mark.gpu
def test_compat_program_matches_reference_semantics(cuda, tmp_path):
    rng = np.random.default_rng(77)
    # u64 keys whose high words differ while many low words collide
    k64 = (rng.integers(0, 2**31, N, dtype=np.uint64) << np.uint64(32)) | \
        rng.integers(0, 5000, N, dtype=np.uint64)
    k32 = rng.integers(0, 2**32, N, dtype=np.uint64).astype(np.uint32)
    k32[::7] = 12345  # duplicates
    k96 = rng.integers(0, 2**32, 3 * N, dtype=np.uint64).astype(np.uint32)
    k96[0::3][::5] = 9  # low words collide, so higher words decide
    i32 = rng.integers(-2**31, 2**31, N, dtype=np.int64).astype(np.int32)
    vox = rng.integers(0, 1024, (NV, 3)).astype(np.uint32)
    with open(tmp_path / "in.bin", "wb") as f:
        f.write(np.array([N, NV], np.uint32).tobytes())
        for a in (k64, k32, k96, i32, vox):
            f.write(np.ascontiguousarray(a).tobytes())
    exe = build(tmp_path)
    res = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr
    r = Reader((tmp_path / "out.bin").read_bytes())
    idx = np.arange(N, dtype=np.uint32)

    # (1) default config: low 32 bits, stable (oracle = the reference's semantics)
    assert r.status() == 0
    ek, ev = oracle.stable_sort_pairs(k64, idx, 32)
    assert np.array_equal(r.take(np.uint64, N), ek)
    assert np.array_equal(r.take(np.uint32, N), ev)
    # (2) KeyBits 64
    assert r.status() == 0
    ek, ev = oracle.stable_sort_pairs(k64, idx, 64)
    assert np.array_equal(r.take(np.uint64, N), ek)
    assert np.array_equal(r.take(np.uint32, N), ev)
    # (3) three value arrays follow the keys
    assert r.status() == 0
    order = np.argsort(k32, kind="stable")
    assert np.array_equal(r.take(np.uint32, N), k32[order])
    assert np.array_equal(r.take(np.uint32, N), order)
    rec = r.take(np.uint32, 3 * N).reshape(N, 3)
    assert np.array_equal(rec[:, 0], order) and np.array_equal(rec[:, 1], ~order.astype(np.uint32))
    assert np.array_equal(rec[:, 2], (order * 7).astype(np.uint32))
    assert np.array_equal(r.take(np.uint8, N), (order * 13).astype(np.uint8))
    # (4) UIntKey<3>: 96 and 40 key bits
    w = k96.reshape(N, 3)
    for order in (np.lexsort((w[:, 0], w[:, 1], w[:, 2])),
                  np.lexsort((w[:, 0], w[:, 1] & 0xFF))):
        assert r.status() == 0
        assert np.array_equal(r.take(np.uint32, 3 * N).reshape(N, 3), w[order])
        pay = (order.astype(np.uint64) << np.uint64(32)) | np.uint64(0xABC)
        assert np.array_equal(r.take(np.uint64, N), pay)
    # (5) sort_keys
    assert r.status() == 0
    assert np.array_equal(r.take(np.uint32, N), np.sort(k32))
    # (6) errors as the reference reports them
    assert [r.status() for _ in range(4)] == [INVALID, INVALID, INVALID, 0]
    # (7) scans
    a = k32 & np.uint32(0xFF)
    assert r.status() == 0
    assert np.array_equal(r.take(np.uint32, N), oracle.exclusive_sum(a))
    assert r.status() == 0
    assert np.array_equal(r.take(np.uint32, N), oracle.inclusive_sum(a))
    assert r.status() == 0
    assert np.array_equal(r.take(np.uint64, N), oracle.exclusive_sum(k64))
    assert r.status() == 0
    incl = np.maximum.accumulate(i32)
    assert np.array_equal(r.take(np.int32, N), incl)
    assert r.status() == 0
    excl = np.concatenate([[np.iinfo(np.int32).min], incl[:-1]]).astype(np.int32)
    assert np.array_equal(r.take(np.int32, N), excl)
    assert r.status() == 0
    fl = (k32 & np.uint32(3)).astype(np.float32)
    assert np.array_equal(r.take(np.float32, N), np.cumsum(fl, dtype=np.float64).astype(np.float32))
    assert r.status() == INVALID
    # (8) Hash DAG: placed voxels, every third destroyed; a short workspace rejected
    assert [r.status() for _ in range(3)] == [0, 0, 0]
    assert r.status() == INVALID
    gone = {tuple(v) for v in vox[::3].tolist()}
    want = np.array([0 if tuple(v) in gone else 1 for v in vox.tolist()], np.uint8)
    assert np.array_equal(r.take(np.uint8, NV), want)
    # (9) GPU SVO: placed voxels minus the destroyed cell [512,1024) x [0,512) x [512,1024)
    assert [r.status() for _ in range(3)] == [0, 0, 0]
    inside = (vox[:, 0] >= 512) & (vox[:, 1] < 512) & (vox[:, 2] >= 512)
    assert np.array_equal(r.take(np.uint8, NV), (~inside).astype(np.uint8))
    assert r.o == len(r.raw)
