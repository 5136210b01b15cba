"""The C++ compatibility header (the reference's call shapes over the C ABI)
compiles and links against the library; nothing runs on a device."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
SRC = r'''
#include "voxel_b200_compat.hpp"
int main() {
  namespace hdg = algo::svt::hash_dag_gpu;
  std::uint32_t *d = nullptr; std::uint64_t *k = nullptr;
  (void)algo::cuda::scan::required_workspace_size<std::uint32_t>(10);
  (void)algo::cuda::scan::exclusive_sum(d, 0, nullptr, 0);
  (void)algo::cuda::sort::sort_by_key(k, algo::cuda::sort::value_arrays(d), 0, nullptr, 0);
  (void)hdg::apply_voxel_edits_workspace_size(4);
  hdg::VoxelEdit e{1, 2, 3};
  (void)e;
  namespace svt = algo::svt::cuda;
  using Cfg = svt::DefaultTerminalEditConfig;
  (void)svt::detail::apply_terminal_edits_workspace_size<Cfg::allocation, Cfg::release>(1, 1, 16);
  svt::TerminalNodeInput node{0u, 0u, 0, 0, 0};
  svt::TerminalLeafInput leaf{};
  static_assert(sizeof(node) == 20 && sizeof(leaf) == 32, "reference layouts");
  if (false) {  // link-time check only: needs a device to run
    svt::GpuSvo<256, 64> svo;
    (void)svt::reset_svo(svo.view());
    (void)svt::place_terminal_edits(svo.view(), &node, 1, &leaf, 1, nullptr, 0);
    (void)svt::destroy_terminal_edits(svo.view(), &node, 1, &leaf, 1, nullptr, 0);
    (void)svt::place_voxel_edits(svo.view(), nullptr, 0, nullptr, 0);
    (void)svt::apply_voxel_edits_workspace_size(4);
  }
  return 0;
}
'''


@pytest.mark.skipif(shutil.which("g++") is None, reason="no g++")
def test_compat_header_compiles_and_links(tmp_path):
    src = tmp_path / "use.cpp"
    src.write_text(SRC)
    exe = tmp_path / "use"
    cmd = ["g++", "-std=c++17", str(src), "-I", str(ROOT / "include"),
           "-I", "/usr/local/cuda/include", "-L", str(ROOT / "voxel_b200"),
           "-lvoxel_b200", "-L", "/usr/local/cuda/lib64", "-lcudart", "-o", str(exe)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="no nvcc")
def test_device_header_compiles_for_sm100a(tmp_path):
    """A user kernel built against voxel_b200_device.cuh (cross-compiled for
    sm_100a here; run by tests/test_gpu_device_api.py on a GPU)."""
    obj = tmp_path / "user.o"
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-c",
           str(ROOT / "tests" / "user_kernels.cu"), "-I", str(ROOT / "include"), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="no nvcc")
def test_fused_scan_header_compiles_for_sm100a(tmp_path):
    """User fused scans against voxel_b200_fused_scan.cuh (cross-compiled for
    sm_100a; run by tests/test_gpu_fused_scan.py on a GPU)."""
    obj = tmp_path / "fused.o"
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-c",
           str(ROOT / "tests" / "user_fused_scan.cu"), "-I", str(ROOT / "include"), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
