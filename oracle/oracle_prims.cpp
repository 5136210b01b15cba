// ORACLE - test infrastructure only.  CPU restatement of the reference's
// scan / radix sort / hash-table semantics, used by tests/ as the checker and
// by bench.py as the CPU baseline.  Never linked into or called by the
// product library.
//
//   scan:  algo::cuda::scan::{inclusive,exclusive}_sum (cuda/scan/scan.cuh:
//          107-151) - sequential prefix sums with wrapping unsigned
//          arithmetic, as the reference tests' cpu_inclusive_sum /
//          cpu_exclusive_sum compute them (test/cuda/test_cuda_scan.cu).
//   sort:  algo::cuda::sort::sort_by_key with KeyBits (docs/cuda/sort.md,
//          "UIntKey" and KeyBits sections) - std::stable_sort by the low
//          key_bits bits, as test/cuda/test_cuda_sort.cu:188-260 does.
//   hash:  slab hash set statuses (cuda/hash_table/slab_hash/common.cuh:18-25)
//          restated over std::unordered_set.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <thread>
#include <unordered_set>
#include <vector>

using u32 = std::uint32_t;
using u64 = std::uint64_t;

namespace {

template <class T>
void prefix(const T *in, T *out, u64 n, bool inclusive) {
  T run = 0;
  for (u64 i = 0; i < n; ++i) {
    const T x = in[i];
    if (inclusive) {
      run += x;
      out[i] = run;
    } else {
      out[i] = run;
      run += x;
    }
  }
}

template <class K>
void stable_sort_pairs(K *keys, u32 *vals, u64 n, u32 key_bits) {
  const K mask = key_bits >= sizeof(K) * 8 ? ~K(0) : ((K(1) << key_bits) - 1);
  std::vector<u64> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](u64 a, u64 b) {
    return (keys[a] & mask) < (keys[b] & mask);
  });
  std::vector<K> k2(n);
  std::vector<u32> v2(vals ? n : 0);
  for (u64 i = 0; i < n; ++i) {
    k2[i] = keys[order[i]];
    if (vals) v2[i] = vals[order[i]];
  }
  std::memcpy(keys, k2.data(), n * sizeof(K));
  if (vals) std::memcpy(vals, v2.data(), n * sizeof(u32));
}

// Multi-threaded LSD radix sort (8-bit digits), the CPU baseline for the
// primitives sweep: per-thread histograms, a serial offset scan per pass,
// then a stable per-thread scatter.
template <class K>
void radix_sort_pairs_mt(K *keys, u32 *vals, u64 n, u32 key_bits, int threads) {
  if (n <= 1) return;
  threads = std::max(1, threads);
  std::vector<K> tk(n);
  std::vector<u32> tv(vals ? n : 0);
  K *sk = keys, *dk = tk.data();
  u32 *sv = vals, *dv = vals ? tv.data() : nullptr;
  const u32 passes = (key_bits + 7) / 8;
  std::vector<u64> hist(static_cast<size_t>(threads) * 256);
  for (u32 p = 0; p < passes; ++p) {
    const u32 shift = p * 8;
    std::fill(hist.begin(), hist.end(), 0);
    auto range = [&](int t, u64 &b, u64 &e) {
      b = n * t / threads;
      e = n * (t + 1) / threads;
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
      pool.emplace_back([&, t] {
        u64 b, e;
        range(t, b, e);
        u64 *h = &hist[t * 256];
        for (u64 i = b; i < e; ++i) ++h[(sk[i] >> shift) & 0xff];
      });
    for (auto &th : pool) th.join();
    pool.clear();
    u64 run = 0;
    for (u32 d = 0; d < 256; ++d)
      for (int t = 0; t < threads; ++t) {
        const u64 c = hist[t * 256 + d];
        hist[t * 256 + d] = run;
        run += c;
      }
    for (int t = 0; t < threads; ++t)
      pool.emplace_back([&, t] {
        u64 b, e;
        range(t, b, e);
        u64 *h = &hist[t * 256];
        for (u64 i = b; i < e; ++i) {
          const u64 dst = h[(sk[i] >> shift) & 0xff]++;
          dk[dst] = sk[i];
          if (sv) dv[dst] = sv[i];
        }
      });
    for (auto &th : pool) th.join();
    std::swap(sk, dk);
    std::swap(sv, dv);
  }
  if (sk != keys) {
    std::memcpy(keys, sk, n * sizeof(K));
    if (vals) std::memcpy(vals, sv, n * sizeof(u32));
  }
}

} // namespace

extern "C" {

void orc_scan_u32(const u32 *in, u32 *out, u64 n, int inclusive) {
  prefix<u32>(in, out, n, inclusive != 0);
}

void orc_scan_u64(const u64 *in, u64 *out, u64 n, int inclusive) {
  prefix<u64>(in, out, n, inclusive != 0);
}

// Two-pass parallel exclusive scan (CPU baseline on all host threads).
void orc_exclusive_scan_u32_mt(const u32 *in, u32 *out, u64 n, int threads) {
  threads = std::max(1, threads);
  std::vector<u32> sums(threads + 1, 0);
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&, t] {
      const u64 b = n * t / threads, e = n * (t + 1) / threads;
      u32 s = 0;
      for (u64 i = b; i < e; ++i) s += in[i];
      sums[t + 1] = s;
    });
  for (auto &th : pool) th.join();
  pool.clear();
  for (int t = 0; t < threads; ++t) sums[t + 1] += sums[t];
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&, t] {
      const u64 b = n * t / threads, e = n * (t + 1) / threads;
      u32 run = sums[t];
      for (u64 i = b; i < e; ++i) {
        const u32 x = in[i];
        out[i] = run;
        run += x;
      }
    });
  for (auto &th : pool) th.join();
}

void orc_stable_sort_pairs_u32(u32 *keys, u32 *vals, u64 n, u32 key_bits) {
  stable_sort_pairs<u32>(keys, vals, n, key_bits);
}

void orc_stable_sort_pairs_u64(u64 *keys, u32 *vals, u64 n, u32 key_bits) {
  stable_sort_pairs<u64>(keys, vals, n, key_bits);
}

void orc_radix_sort_pairs_u32_mt(u32 *keys, u32 *vals, u64 n, u32 key_bits,
                                 int threads) {
  radix_sort_pairs_mt<u32>(keys, vals, n, key_bits, threads);
}

void orc_radix_sort_pairs_u64_mt(u64 *keys, u32 *vals, u64 n, u32 key_bits,
                                 int threads) {
  radix_sort_pairs_mt<u64>(keys, vals, n, key_bits, threads);
}

// Hash-set semantics of BasicSlabHashSetU32, widened to u64 keys: insert
// statuses (Inserted / AlreadyPresent / InvalidKey) in input order, then
// contains flags for the queries.  Returns the number of hits.
u64 orc_hash_set_u64(const u64 *ins, u64 n_ins, u32 *ins_status,
                     const u64 *queries, u64 n_q, u32 *found) {
  constexpr u64 kEmpty = ~0ull, kDeleted = ~0ull - 1;
  std::unordered_set<u64> set;
  set.reserve(n_ins);
  for (u64 i = 0; i < n_ins; ++i) {
    const u64 k = ins[i];
    u32 st;
    if (k == kEmpty || k == kDeleted) st = 5;          // InvalidKey
    else st = set.insert(k).second ? 1u : 7u;          // Inserted / AlreadyPresent
    if (ins_status) ins_status[i] = st;
  }
  u64 hits = 0;
  for (u64 i = 0; i < n_q; ++i) {
    const u32 f = set.count(queries[i]) ? 1u : 0u;
    hits += f;
    if (found) found[i] = f;
  }
  return hits;
}

} // extern "C"
