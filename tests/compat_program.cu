// A caller of the reference's C++ API, built against include/voxel_b200_compat.hpp
// with nvcc and run by tests/test_gpu_compat.py: it reads inputs written by
// the test, makes the reference's sort / scan / Hash DAG / SVO calls and writes
// every result back for the test to check against the oracle.
//
// usage: compat_program <dir>   (reads <dir>/in.bin, writes <dir>/out.bin)
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "voxel_b200_compat.hpp"

namespace sort = algo::cuda::sort;
namespace scan = algo::cuda::scan;
namespace hdg = algo::svt::hash_dag_gpu;
namespace svt = algo::svt::cuda;

struct Rec12 {
  std::uint32_t a, b, c;
};

static std::vector<char> g_out;
template <class T> static void put(const std::vector<T> &v) {
  const char *p = reinterpret_cast<const char *>(v.data());
  g_out.insert(g_out.end(), p, p + v.size() * sizeof(T));
}
static void put_status(cudaError_t e) { put(std::vector<std::int32_t>{static_cast<std::int32_t>(e)}); }

#define CHECK(x)                                                                                   \
  do {                                                                                             \
    cudaError_t e_ = (x);                                                                          \
    if (e_ != cudaSuccess) {                                                                       \
      std::fprintf(stderr, "%s:%d %s -> %d\n", __FILE__, __LINE__, #x, int(e_));                   \
      std::exit(1);                                                                                \
    }                                                                                              \
  } while (0)

template <class T> static T *dev(const std::vector<T> &h) {
  T *d = nullptr;
  CHECK(cudaMalloc(&d, h.size() * sizeof(T) + 16));
  CHECK(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  return d;
}
template <class T> static std::vector<T> host(const T *d, std::size_t n) {
  std::vector<T> h(n);
  CHECK(cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost));
  return h;
}
static void *workspace(std::size_t n) {
  void *p = nullptr;
  CHECK(cudaMalloc(&p, n ? n : 1));
  return p;
}

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  const std::string dir = argv[1];
  FILE *f = std::fopen((dir + "/in.bin").c_str(), "rb");
  if (!f) return 3;
  std::uint32_t n = 0, nv = 0;
  if (std::fread(&n, 4, 1, f) != 1 || std::fread(&nv, 4, 1, f) != 1) return 4;
  std::vector<std::uint64_t> k64(n);
  std::vector<std::uint32_t> k32(n), k96(3 * size_t(n)), vox(3 * size_t(nv));
  std::vector<std::int32_t> i32(n);
  if (std::fread(k64.data(), 8, n, f) != n || std::fread(k32.data(), 4, n, f) != n ||
      std::fread(k96.data(), 4, 3 * size_t(n), f) != 3 * size_t(n) ||
      std::fread(i32.data(), 4, n, f) != n || std::fread(vox.data(), 4, 3 * size_t(nv), f) != 3 * size_t(nv))
    return 5;
  std::fclose(f);
  std::vector<std::uint32_t> idx(n);
  for (std::uint32_t i = 0; i < n; ++i) idx[i] = i;

  // (1) u64 keys, default config: ordered by the low 32 bits, stable
  {
    std::uint64_t *k = dev(k64);
    std::uint32_t *v = dev(idx);
    const auto need = sort::required_sort_by_key_workspace_size<std::uint64_t>(n, sort::value_arrays(v));
    void *ws = workspace(need);
    put_status(sort::sort_by_key(k, sort::value_arrays(v), n, ws, need));
    put(host(k, n));
    put(host(v, n));
    cudaFree(k), cudaFree(v), cudaFree(ws);
  }
  // (2) u64 keys, RadixSort<OneSweepPass<...>, 512, 8, 64>: all 64 bits
  {
    using Cfg = sort::RadixSort<sort::OneSweepPass<sort::WarpBallotBlockHistogram,
                                                   sort::WarpLevelMultiSplitWarpRank,
                                                   sort::SharedAtomicGlobalOffsetsBlockHistogram, 4>,
                                512, 8, 64>;
    std::uint64_t *k = dev(k64);
    std::uint32_t *v = dev(idx);
    const auto need = sort::required_sort_by_key_workspace_size<Cfg, std::uint64_t, std::uint32_t>(n);
    void *ws = workspace(need);
    put_status(sort::sort_by_key<Cfg>(k, sort::value_arrays(v), n, ws, need));
    put(host(k, n));
    put(host(v, n));
    cudaFree(k), cudaFree(v), cudaFree(ws);
  }
  // (3) u32 keys with three value arrays of 4, 12 and 1 bytes
  {
    std::vector<Rec12> r(n);
    std::vector<std::uint8_t> b(n);
    for (std::uint32_t i = 0; i < n; ++i) {
      r[i] = Rec12{i, ~i, i * 7u};
      b[i] = static_cast<std::uint8_t>(i * 13u);
    }
    std::uint32_t *k = dev(k32), *v = dev(idx);
    Rec12 *dr = dev(r);
    std::uint8_t *db = dev(b);
    const auto va = sort::value_arrays(v, dr, db);
    const auto need = sort::required_sort_by_key_workspace_size<std::uint32_t>(n, va);
    void *ws = workspace(need);
    put_status(sort::sort_by_key(k, va, n, ws, need));
    put(host(k, n));
    put(host(v, n));
    put(host(dr, n));
    put(host(db, n));
    cudaFree(k), cudaFree(v), cudaFree(dr), cudaFree(db), cudaFree(ws);
  }
  // (4) UIntKey<3> keys, KeyBits 96 and 40, with a u64 payload
  for (int kb = 0; kb < 2; ++kb) {
    using K = sort::UIntKey<3>;
    std::vector<K> keys(n);
    std::memcpy(keys.data(), k96.data(), 12 * size_t(n));
    std::vector<std::uint64_t> pay(n);
    for (std::uint32_t i = 0; i < n; ++i) pay[i] = (std::uint64_t(i) << 32) | 0xabcu;
    K *dk = dev(keys);
    std::uint64_t *dp = dev(pay);
    cudaError_t st;
    std::size_t need;
    void *ws;
    if (kb == 0) {
      using Cfg = sort::RadixSort<sort::HistogramPass<sort::SharedAtomicHistogram,
                                                      sort::WarpLevelMultiSplitWarpRank, 4>,
                                  256, 8, 96>;
      need = sort::required_sort_by_key_workspace_size<Cfg, K, std::uint64_t>(n);
      ws = workspace(need);
      st = sort::sort_by_key<Cfg>(dk, sort::value_arrays(dp), n, ws, need);
    } else {
      using Cfg = sort::RadixSort<sort::FlagPrefixSumPass<>, 256, 8, 40>;
      need = sort::required_sort_by_key_workspace_size<Cfg, K, std::uint64_t>(n);
      ws = workspace(need);
      st = sort::sort_by_key<Cfg>(dk, sort::value_arrays(dp), n, ws, need);
    }
    put_status(st);
    std::vector<K> out = host(dk, n);
    std::vector<std::uint32_t> flat(3 * size_t(n));
    std::memcpy(flat.data(), out.data(), 12 * size_t(n));
    put(flat);
    put(host(dp, n));
    cudaFree(dk), cudaFree(dp), cudaFree(ws);
  }
  // (5) sort_keys u32 (default config)
  {
    std::uint32_t *k = dev(k32);
    const auto need = sort::required_workspace_size<std::uint32_t>(n);
    void *ws = workspace(need);
    put_status(sort::sort_keys(k, n, ws, need));
    put(host(k, n));
    cudaFree(k), cudaFree(ws);
  }
  // (6) errors: null keys, null value array, short workspace
  {
    std::uint32_t *v = dev(idx);
    std::uint64_t *k = dev(k64);
    const auto need = sort::required_sort_by_key_workspace_size<std::uint64_t>(n, sort::value_arrays(v));
    void *ws = workspace(need);
    put_status(sort::sort_by_key(static_cast<std::uint64_t *>(nullptr), sort::value_arrays(v), n, ws, need));
    put_status(sort::sort_by_key(k, sort::value_arrays(static_cast<std::uint32_t *>(nullptr)), n, ws, need));
    put_status(sort::sort_by_key(k, sort::value_arrays(v), n, ws, need - 1));
    put_status(sort::sort_by_key(k, sort::value_arrays(v), 0, nullptr, 0));
    cudaFree(k), cudaFree(v), cudaFree(ws);
  }
  // (7) scans: exclusive / inclusive sums (u32, u64), Max over int32, Plus over float
  {
    std::vector<std::uint32_t> a(n);
    std::vector<std::uint64_t> a64(n);
    std::vector<float> fl(n);
    for (std::uint32_t i = 0; i < n; ++i) {
      a[i] = k32[i] & 0xff;
      a64[i] = k64[i];
      fl[i] = static_cast<float>(k32[i] & 3u);
    }
    const auto need = scan::required_workspace_size<scan::detail::DefaultConfig, scan::Max<std::int32_t>,
                                                    std::uint64_t>(n);
    void *ws = workspace(need);
    std::uint32_t *d = dev(a);
    put_status(scan::exclusive_sum(d, n, ws, need));
    put(host(d, n));
    cudaFree(d);
    d = dev(a);
    put_status(scan::inclusive_sum(d, n, ws, need));
    put(host(d, n));
    cudaFree(d);
    std::uint64_t *d64 = dev(a64);
    put_status(scan::exclusive_sum(d64, n, ws, need));
    put(host(d64, n));
    cudaFree(d64);
    std::int32_t *di = dev(i32);
    put_status(scan::inclusive_scan<scan::Max<std::int32_t>>(di, n, ws, need));
    put(host(di, n));
    cudaFree(di);
    di = dev(i32);
    put_status(scan::exclusive_scan<scan::detail::DefaultConfig, scan::Max<std::int32_t>>(di, n, ws, need));
    put(host(di, n));
    cudaFree(di);
    float *df = dev(fl);
    put_status(scan::inclusive_sum(df, n, ws, need));
    put(host(df, n));
    cudaFree(df);
    put_status(scan::exclusive_sum(static_cast<std::uint32_t *>(nullptr), n, ws, need));
    cudaFree(ws);
  }
  // (8) Hash DAG: place, then destroy every third voxel; query all of them
  {
    hdg::HashDagGpu<1024, 1024> dag(8, 1u << 20);
    put_status(dag.status());
    std::vector<hdg::VoxelEdit> e(nv), gone;
    std::memcpy(e.data(), vox.data(), 12 * size_t(nv));
    for (std::uint32_t i = 0; i < nv; i += 3) gone.push_back(e[i]);
    hdg::VoxelEdit *de = dev(e), *dg = dev(gone);
    const auto need = hdg::apply_voxel_edits_workspace_size(nv);
    void *ws = workspace(need);
    put_status(hdg::place_voxel_edits(dag.view(), de, nv, ws, need));
    put_status(hdg::destroy_voxel_edits(dag.view(), dg, std::uint32_t(gone.size()), ws, need));
    put_status(hdg::place_voxel_edits(dag.view(), de, nv, ws, need - 1));
    std::uint8_t *q = nullptr;
    CHECK(cudaMalloc(&q, nv));
    CHECK(cudaDeviceSynchronize());
    if (vx_dag_query(dag.view().dag, reinterpret_cast<const vx_voxel *>(de), nv, q, nullptr) != VX_OK)
      return 6;
    put(host(q, nv));
    cudaFree(de), cudaFree(dg), cudaFree(ws), cudaFree(q);
  }
  // (9) GPU SVO: voxel edits, then a terminal cell write
  {
    svt::GpuSvo<1u << 16, 1u << 18> svo;
    put_status(svo.status());
    std::vector<svt::VoxelEdit> e(nv);
    std::memcpy(e.data(), vox.data(), 12 * size_t(nv));
    svt::VoxelEdit *de = dev(e);
    const auto need = svt::apply_voxel_edits_workspace_size(nv);
    void *ws = workspace(need);
    put_status(svt::place_voxel_edits(svo.view(), de, nv, ws, need));
    svt::TerminalNodeInput cell{3u, 5u, 0, 0, 0}; // depth-3 cell, prefix 5
    const auto need_t = svt::detail::apply_terminal_edits_workspace_size<
        svt::DefaultTerminalEditConfig::allocation, svt::DefaultTerminalEditConfig::release>(1, 0, 64);
    void *wst = workspace(need_t);
    svt::TerminalNodeInput *dc = dev(std::vector<svt::TerminalNodeInput>{cell});
    put_status(svt::destroy_terminal_edits(svo.view(), dc, 1, nullptr, 0, wst, need_t));
    std::uint8_t *q = nullptr;
    CHECK(cudaMalloc(&q, nv));
    CHECK(cudaDeviceSynchronize());
    if (vx_svo_query(svo.view().svo, reinterpret_cast<const vx_voxel *>(de), nv, q, nullptr) != VX_OK)
      return 7;
    put(host(q, nv));
    cudaFree(de), cudaFree(ws), cudaFree(wst), cudaFree(dc), cudaFree(q);
  }
  FILE *o = std::fopen((dir + "/out.bin").c_str(), "wb");
  if (!o || std::fwrite(g_out.data(), 1, g_out.size(), o) != g_out.size()) return 8;
  std::fclose(o);
  return 0;
}
