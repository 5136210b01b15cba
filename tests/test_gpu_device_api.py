"""The device-side reads of voxel_b200_device.cuh, called from a user's own
kernels (tests/user_kernels.cu, built here with nvcc for sm_100a): DAG and
SVO point lookups, the warp-cooperative slab-set membership and the cuckoo
find give the same answers as the library's batch calls."""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest
import torch

import oracle
import voxel_b200 as vx

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def user_lib(tmp_path_factory):
    if shutil.which("nvcc") is None:
        pytest.skip("nvcc is needed to build the user kernels")
    out = tmp_path_factory.mktemp("user") / "libuser.so"
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2",
           "-shared", "-Xcompiler", "-fPIC", str(ROOT / "tests" / "user_kernels.cu"),
           "-I", str(ROOT / "include"), "-o", str(out)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    lib = C.CDLL(str(out))
    for name in ("user_dag_points", "user_svo_points", "user_slab_contains",
                 "user_cuckoo_values"):
        getattr(lib, name).argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
        getattr(lib, name).restype = C.c_int
    return lib


def points(rng, n, world):
    p = rng.integers(0, world + 8, (n, 3)).astype(np.uint32)  # some outside
    return vx.voxels_to_device(p, "cuda"), n


def test_dag_and_svo_point_lookups(cuda, user_lib):
    depth = 6
    world = 4 << depth
    rng = np.random.default_rng(41)
    dag = vx.HashDag(depth, 1 << 18, 64 << 20)
    dag.build_terrain(9, 1, True)
    svo = vx.Svo(depth, 1 << 18, 1 << 18, materials=True, arena_bytes=64 << 20)
    svo.build_terrain(9, 1, True)
    assert dag.status() == 0 and svo.status() == 0
    pts, n = points(rng, 200_000, world)
    out = torch.zeros(n, dtype=torch.uint8, device=cuda)
    v = dag.device_view()
    assert user_lib.user_dag_points(C.addressof(v), pts.data_ptr(), n, out.data_ptr()) == 0
    assert torch.equal(out, dag.query(pts))
    v = svo.device_view()
    assert user_lib.user_svo_points(C.addressof(v), pts.data_ptr(), n, out.data_ptr()) == 0
    assert torch.equal(out, svo.query(pts))
    assert int(out.count_nonzero()) > 0


def test_hash_lookups(cuda, user_lib):
    rng = np.random.default_rng(42)
    n = 300_000
    keys = rng.integers(1, 2**62, n, dtype=np.uint64)
    probe = np.concatenate([keys[: n // 2], rng.integers(1, 2**62, n // 2, dtype=np.uint64)])
    dk = torch.from_numpy(keys.view(np.int64)).to(cuda)
    dq = torch.from_numpy(probe.view(np.int64)).to(cuda)
    s = vx.SlabHashSet(1 << 14, 1 << 16)
    s.insert(dk)
    expect = s.contains(dq)
    got = torch.zeros(n, dtype=torch.int32, device=cuda)
    v = s.device_view()
    assert user_lib.user_slab_contains(C.addressof(v), dq.data_ptr(), n, got.data_ptr()) == 0
    assert torch.equal(got.to(expect.dtype), expect)
    assert int(got.sum()) >= n // 2
    m = vx.CuckooMap(1 << 19)
    vals = torch.arange(n, dtype=torch.int32, device=cuda)
    m.insert(dk, vals)
    expect = m.find(dq)
    v = m.device_view()
    assert user_lib.user_cuckoo_values(C.addressof(v), dq.data_ptr(), n, got.data_ptr()) == 0
    assert torch.equal(got.to(expect.dtype), expect)
