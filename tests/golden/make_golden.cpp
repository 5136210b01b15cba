// Generates tests/golden/primitives.json: the inputs of the reference's own
// scan and sort tests, reproduced with the same generators (std::mt19937 and
// libstdc++'s std::uniform_int_distribution), and the expected outputs
// computed the way those tests compute them (std::stable_sort by the low
// key bits, sequential prefix sums).  Built and run by make_golden.py.
//
// Sources of each case (algorithm/test/cuda/...):
//   test_cuda_scan.cu:252-330   fixed input {3,1,4,1,5,9,2,6,5}
//   test_cuda_scan.cu:339-343   mt19937(123), U{0..9}, n = 257
//   test_cuda_scan.cu:417-420   mt19937(456), U{0..9}, n = 4097
//   test_cuda_scan.cu:605-612   mt19937(789), U{0..9}, n = 4097, x -> 2x + 1
//   test_cuda_scan.cu:664-667   mt19937(987), U{0..9}, n = 4097
//   test_cuda_sort.cu:485-493   fixed keys {3,1,4,1,5,9,2,6,5}
//   test_cuda_sort.cu:495-503   fixed keys {9,7,5,3,1,8,6,4,2,0}
//   test_cuda_sort.cu:505-520   mt19937(123), U{0..4095}, n = 257
//   test_cuda_sort.cu:522-530   low 4 bits of {0x30,0x21,0x12,0x03,...}
//   test_cuda_sort.cu:800-811   u64 keys incl. 0xffff'ffffffffffff
//   test_cuda_sort.cu:947-956   keys + values {30,10,40,11,...}
//   test_cuda_sort.cu:958-968   duplicate keys, values = index
//   test_cuda_sort.cu:970-988   mt19937(123), U{0..4095}, n = 257, values
//   test_cuda_sort.cu:990-998   low 4 bits with values
//   test_cuda_sort.cu:1184-1198 4097 equal keys, values = index
//   test_cuda_sort.cu:1200-1217 mt19937(987), full-range u32, n = 8197
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <numeric>
#include <random>
#include <string>
#include <vector>

using u32 = std::uint32_t;
using u64 = std::uint64_t;

static std::string join(const std::vector<u64> &v) {
  std::string s = "[";
  for (size_t i = 0; i < v.size(); ++i) {
    if (i) s += ",";
    s += std::to_string(v[i]);
  }
  return s + "]";
}

template <class T> static std::vector<u64> widen(const std::vector<T> &v) {
  return std::vector<u64>(v.begin(), v.end());
}

static bool first = true;
static void emit(const char *name, const std::string &body) {
  std::printf("%s\n  \"%s\": {%s}", first ? "" : ",", name, body.c_str());
  first = false;
}

static void scan_case(const char *name, const std::vector<u32> &in) {
  std::vector<u32> inc(in.size()), exc(in.size());
  u32 run = 0;
  for (size_t i = 0; i < in.size(); ++i) {
    exc[i] = run;
    run += in[i];
    inc[i] = run;
  }
  emit(name, "\"input\": " + join(widen(in)) + ", \"inclusive\": " +
                 join(widen(inc)) + ", \"exclusive\": " + join(widen(exc)));
}

template <class K>
static void sort_case(const char *name, const std::vector<K> &keys,
                      const std::vector<u32> *values, u32 key_bits) {
  std::vector<size_t> order(keys.size());
  std::iota(order.begin(), order.end(), 0);
  const K mask = key_bits >= sizeof(K) * 8 ? ~K(0) : ((K(1) << key_bits) - 1);
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
    return (keys[a] & mask) < (keys[b] & mask);
  });
  std::vector<u64> ok, ov;
  for (size_t i : order) {
    ok.push_back(keys[i]);
    if (values) ov.push_back((*values)[i]);
  }
  std::string body = "\"key_bytes\": " + std::to_string(sizeof(K)) +
                     ", \"key_bits\": " + std::to_string(key_bits) +
                     ", \"keys\": " + join(widen(keys)) +
                     ", \"sorted_keys\": " + join(ok);
  if (values)
    body += ", \"values\": " + join(widen(*values)) +
            ", \"sorted_values\": " + join(ov);
  emit(name, body);
}

static std::vector<u32> iota_u32(size_t n) {
  std::vector<u32> v(n);
  std::iota(v.begin(), v.end(), 0u);
  return v;
}

int main() {
  std::printf("{");
  scan_case("scan_fixed", {3, 1, 4, 1, 5, 9, 2, 6, 5});
  {
    std::mt19937 rng(123);
    std::uniform_int_distribution<u32> dist(0, 9);
    std::vector<u32> in(257);
    for (auto &v : in) v = dist(rng);
    scan_case("scan_random_257_seed123", in);
  }
  {
    std::mt19937 rng(456);
    std::uniform_int_distribution<u32> dist(0, 9);
    std::vector<u32> in(4097);
    for (auto &v : in) v = dist(rng);
    scan_case("scan_random_4097_seed456", in);
  }
  {
    std::mt19937 rng(789);
    std::uniform_int_distribution<u32> dist(0, 9);
    std::vector<u32> in(4097);
    for (auto &v : in) v = dist(rng) * 2u + 1u;
    scan_case("scan_transformed_4097_seed789", in);
  }
  {
    std::mt19937 rng(987);
    std::uniform_int_distribution<u32> dist(0, 9);
    std::vector<u32> in(4097);
    for (auto &v : in) v = dist(rng);
    scan_case("scan_random_4097_seed987", in);
  }

  sort_case<u32>("sort_fixed", {3, 1, 4, 1, 5, 9, 2, 6, 5}, nullptr, 32);
  sort_case<u32>("sort_fixed_descending", {9, 7, 5, 3, 1, 8, 6, 4, 2, 0},
                 nullptr, 32);
  {
    std::mt19937 rng(123);
    std::uniform_int_distribution<u32> dist(0, 4095);
    std::vector<u32> in(257);
    for (auto &v : in) v = dist(rng);
    sort_case<u32>("sort_random_257_seed123", in, nullptr, 32);
    const auto vals = iota_u32(in.size());
    sort_case<u32>("sort_pairs_random_257_seed123", in, &vals, 32);
  }
  sort_case<u32>("sort_lower4_keys",
                 {0x30u, 0x21u, 0x12u, 0x03u, 0x34u, 0x25u, 0x16u, 0x07u},
                 nullptr, 4);
  sort_case<u64>("sort_u64_keys",
                 {0x100000000ull, 3ull, 0xffffffffffffffffull, 0ull,
                  0x8000000000000000ull, 0x0000000100000001ull},
                 nullptr, 64);
  {
    const std::vector<u32> vals{30, 10, 40, 11, 50, 90, 20, 60, 51};
    sort_case<u32>("sort_pairs_fixed", {3, 1, 4, 1, 5, 9, 2, 6, 5}, &vals, 32);
  }
  {
    const auto vals = iota_u32(12);
    sort_case<u32>("sort_pairs_duplicates",
                   {0, 42, 0, 42, 7, 7, 7, 1, 0, 999, 42, 3}, &vals, 32);
  }
  {
    const auto vals = iota_u32(6);
    sort_case<u32>("sort_pairs_lower4",
                   {0x11u, 0x21u, 0x01u, 0x12u, 0x02u, 0x33u}, &vals, 4);
  }
  {
    const std::vector<u32> keys(4097, 7u);
    const auto vals = iota_u32(keys.size());
    sort_case<u32>("sort_pairs_equal_4097", keys, &vals, 32);
  }
  {
    std::mt19937 rng(987);
    std::uniform_int_distribution<u32> dist;
    std::vector<u32> keys(8197);
    for (auto &v : keys) v = dist(rng);
    const auto vals = iota_u32(keys.size());
    sort_case<u32>("sort_pairs_random_8197_seed987", keys, &vals, 32);
  }
  std::printf("\n}\n");
  return 0;
}
