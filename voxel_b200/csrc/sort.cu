// Stable LSD radix sort, onesweep form (Adinets & Merrill 2022, "Onesweep: A
// Faster Least Significant Digit Radix Sort for GPUs"), for u32 / u64 keys
// with an optional u32 payload, on sm_100a:
//
//   1. one read of the keys builds every pass's 256-bin digit histogram
//      (shared-memory counters per block, then one global atomicAdd per bin);
//   2. one partition kernel per 8-bit digit:
//        - dynamic tile id, so a tile only waits on tiles already running;
//        - the tile's keys and payloads arrive in shared memory by bulk copies
//          (TMA); each warp takes 32 x kItems of them and ranks them by digit
//          with __match_any_sync (stable: rank follows the original order
//          inside the warp);
//        - warp counts are combined per digit, the tile publishes its digit
//          counts and looks back over predecessor tiles per digit, eight
//          tiles per round trip (bounded by the GPU timer);
//        - keys and payloads are first sorted inside the tile in shared
//          memory, then written out in that order so consecutive threads write
//          consecutive addresses of each digit's run.
//
// Replaces algo::cuda::sort::sort_by_key with OneSweepPass
// (cuda/sort/radix/onesweep/host.cuh:135-204, partition.cuh:117-200,
// lookback.cuh:7-79, global_offsets.cuh:52-146), whose scatter is direct and
// uncoalesced and whose look-back spin is unbounded.
#include "common.cuh"
#include "profile.cuh"
#include "tuning.cuh"

#include <type_traits>

namespace vx::sort {

constexpr uint32_t kRadixBits = 8;    // the widest digit (256 counters per table)
constexpr uint32_t kMinRadixBits = 6; // the narrowest the "sort.radix_bits" knob offers
constexpr uint32_t kBins = 1u << kRadixBits;
constexpr uint32_t kBlock = 256;
constexpr uint32_t kWarps = kBlock / kWarp;
constexpr uint32_t kMaxPasses = 8;
constexpr uint32_t kMaxCount = (1u << 30) - 1u;

// Look-back record: state in bits 30-31, count in bits 0-29.
constexpr uint32_t kRecAgg = 1u << 30, kRecInc = 2u << 30;
constexpr uint32_t kRecValue = (1u << 30) - 1u;

// Items per thread of the partition kernel (the tile is 256 x items keys):
// the small setting fits four blocks per SM (64 registers, ~35 KB of shared
// memory each), the large one three with more keys per tile (on B200 the
// large one is faster: 2.72 vs 3.13 ms for 2^26 u32 pairs).  The tuning
// knobs "sort.items_u32" / "sort.items_u64" pick one per device.
template <class K> struct Shape;
template <> struct Shape<uint32_t> {
  static constexpr uint32_t kSmall = 12, kLarge = 16;
};
template <> struct Shape<uint64_t> {
  static constexpr uint32_t kSmall = 8, kLarge = 10;
};
template <uint32_t Items, class K> constexpr uint32_t min_blocks() {
  return Items == Shape<K>::kSmall ? 4u : 3u;
}
// Tiles of the small setting: the most tiles, so the workspace covers both.
template <class K> inline uint32_t max_tiles(uint32_t count) {
  return ceil_div(count, kBlock * Shape<K>::kSmall);
}

inline uint32_t pass_count(uint32_t key_bits, uint32_t radix_bits = kRadixBits) {
  return (key_bits + radix_bits - 1) / radix_bits;
}

// The digit width of a sort: the "sort.radix_bits" knob (6 to 8 bits; the
// tables of 256 digit counters hold any of them), or 8 when the narrower
// digit would take more than kMaxPasses passes (64-bit keys).  Digits wider
// than 8 bits are not offered: the decoupled look-back keeps a record per
// digit and tile, 2^width per tile, and 2048-digit tables leave no shared
// memory for per-warp ranking.
inline uint32_t radix_bits_for(uint32_t key_bits) {
  const uint32_t r = static_cast<uint32_t>(tune::get(tune::kSortRadixBits));
  return r >= kMinRadixBits && r <= kRadixBits && pass_count(key_bits, r) <= kMaxPasses
             ? r
             : kRadixBits;
}

template <class K>
__device__ __forceinline__ uint32_t digit_of(K key, uint32_t shift,
                                             uint32_t mask) {
  return static_cast<uint32_t>(key >> shift) & mask;
}

struct PassInfo {
  uint32_t shift[kMaxPasses];
  uint32_t mask[kMaxPasses];
};

struct Layout {
  uint32_t *counters;  // [1] device status, [2 + p] tile counter of pass p
  uint32_t *hist;      // passes x 256 digit counts
  uint32_t *records;   // passes x tiles x 256
  void *tmp_keys;
  uint32_t *tmp_vals;
  size_t clear_bytes;
};

template <class K> Layout carve(void *ws, uint32_t count, uint32_t passes) {
  const uint32_t tiles = max_tiles<K>(count);
  Carver c(ws);
  Layout l;
  l.counters = c.take<uint32_t>(kMaxPasses + 2);
  l.hist = c.take<uint32_t>(kMaxPasses * kBins);
  l.records = c.take<uint32_t>(static_cast<size_t>(passes) * tiles * kBins);
  l.clear_bytes = c.offset;
  l.tmp_keys = c.take<K>(count);
  l.tmp_vals = c.take<uint32_t>(count);
  return l;
}

template <class K> size_t workspace_bytes(uint32_t count, uint32_t passes) {
  const uint32_t tiles = max_tiles<K>(count);
  Sizer s;
  s.take<uint32_t>(kMaxPasses + 2);
  s.take<uint32_t>(kMaxPasses * kBins);
  s.take<uint32_t>(static_cast<size_t>(passes) * tiles * kBins);
  s.take<K>(count);
  s.take<uint32_t>(count);
  return s.offset;
}

// ------------------------------------------------------------ histogram --

template <class K>
__global__ void __launch_bounds__(kBlock)
    histogram_kernel(const K *__restrict__ keys, uint32_t count,
                     uint32_t passes, PassInfo info, uint32_t *hist) {
  // Two copies of the per-pass counters (even / odd warps) halve contention
  // on skewed digits.
  __shared__ uint32_t s_hist[2][kMaxPasses][kBins];
  for (uint32_t i = threadIdx.x; i < 2 * kMaxPasses * kBins; i += kBlock)
    (&s_hist[0][0][0])[i] = 0;
  __syncthreads();
  const uint32_t copy = (threadIdx.x / kWarp) & 1u;
  constexpr uint32_t kPerVec = 16 / sizeof(K);
  const uint32_t vecs = count / kPerVec;
  const uint4 *vkeys = reinterpret_cast<const uint4 *>(keys);
  const bool aligned = (reinterpret_cast<uintptr_t>(keys) & 15u) == 0;
  const uint32_t stride = gridDim.x * kBlock;
  if (aligned) {
    for (uint32_t v = blockIdx.x * kBlock + threadIdx.x; v < vecs; v += stride) {
      const uint4 q = ld_stream_u4(vkeys + v);
      const K *kq = reinterpret_cast<const K *>(&q);
#pragma unroll
      for (uint32_t e = 0; e < kPerVec; ++e)
        for (uint32_t p = 0; p < passes; ++p)
          atomicAdd(&s_hist[copy][p][digit_of(kq[e], info.shift[p], info.mask[p])], 1u);
    }
  }
  const uint32_t tail_begin = aligned ? vecs * kPerVec : 0;
  for (uint32_t i = tail_begin + blockIdx.x * kBlock + threadIdx.x; i < count;
       i += stride) {
    const K k = keys[i];
    for (uint32_t p = 0; p < passes; ++p)
      atomicAdd(&s_hist[copy][p][digit_of(k, info.shift[p], info.mask[p])], 1u);
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < passes * kBins; i += kBlock) {
    const uint32_t c = (&s_hist[0][0][0])[i] + (&s_hist[1][0][0])[i];
    if (c != 0) atomicAdd(hist + i, c);
  }
}

// ------------------------------------------------------------ partition --

// Exclusive scan of one value per thread across the 256-thread block.
__device__ __forceinline__ uint32_t block_exclusive_256(uint32_t v,
                                                        uint32_t *s_tmp) {
  const uint32_t lane = lane_id(), warp = threadIdx.x / kWarp;
  const uint32_t inc = warp_inclusive_sum<uint32_t>(v);
  if (lane == kWarp - 1) s_tmp[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const uint32_t w = lane < kWarps ? s_tmp[lane] : 0u;
    const uint32_t wi = warp_inclusive_sum<uint32_t>(w);
    if (lane < kWarps) s_tmp[lane] = wi - w;
  }
  __syncthreads();
  const uint32_t r = s_tmp[warp] + inc - v;
  __syncthreads();
  return r;
}

// Per-digit decoupled look-back over predecessor tiles, once this tile's
// count is published: thread t (digit t) reads the records of kWindow
// predecessors at once (independent loads, one round trip to L2), sums back
// to the nearest inclusive record and retries the window while a tile before
// that one has not published its count (bounded by the GPU timer); then it
// publishes this tile's inclusive count.  Returns the digit's count over all
// earlier tiles.
__device__ __forceinline__ uint32_t digit_lookback(uint32_t *records, uint32_t tile, uint32_t t,
                                                   uint32_t tile_count, uint32_t *status) {
  if (tile == 0) return 0;
  constexpr uint32_t kWindow = 8;
  uint32_t exclusive = 0;
  const uint64_t t0 = global_ns();
  int64_t pred = static_cast<int64_t>(tile) - 1;
  for (;;) {
    uint32_t r[kWindow];
#pragma unroll
    for (uint32_t j = 0; j < kWindow; ++j)
      r[j] = pred - static_cast<int64_t>(j) >= 0
                 ? ld_relaxed_u32(records + static_cast<size_t>(pred - j) * kBins + t)
                 : kRecInc;
    uint32_t sum = 0;
    bool found = false, wait = false;
#pragma unroll
    for (uint32_t j = 0; j < kWindow; ++j) {
      if (found || wait) continue;
      const uint32_t state = r[j] & ~kRecValue;
      if (state == 0) {
        wait = true;
      } else {
        sum += r[j] & kRecValue;
        found = state == kRecInc;
      }
    }
    if (wait) {
      if (global_ns() - t0 > kWaitLimitNs) {
        set_status(status, kDevTimeout);
        break;
      }
      __nanosleep(20);
      continue;
    }
    exclusive += sum;
    if (found) break;
    pred -= kWindow;
  }
  st_relaxed_u32(records + static_cast<size_t>(tile) * kBins + t,
                 kRecInc | (exclusive + tile_count));
  return exclusive;
}

// Early = publish the tile's digit counts (from a shared-atomic histogram)
// before ranking, so later tiles' look-backs wait less; otherwise they are
// published after ranking, from the per-warp counts.
// Ballots = find a key's peers (the lanes of its warp with the same digit)
// with one ballot per digit bit (warp-level multi-split, Adinets & Merrill);
// otherwise every lane ORs its bit into a per-warp, per-digit word in shared
// memory and reads the word back (three shared-memory operations per key in
// place of eight ballots and their selects).
//
// The pass is bound by instruction issue, so the per-key work is kept short:
// a full tile (every tile but the last) runs without validity tests, 32-bit
// indices throughout, two ranks share a register, and one table gives each
// (warp, digit) its tile-local base.
template <class K, bool HasValues, uint32_t kItems, bool Early, bool Ballots>
__global__ void __launch_bounds__(kBlock, (min_blocks<kItems, K>()))
    partition_kernel(const K *__restrict__ in_keys,
                     const uint32_t *__restrict__ in_vals,
                     K *__restrict__ out_keys, uint32_t *__restrict__ out_vals,
                     uint32_t count, uint32_t shift, uint32_t mask,
                     const uint32_t *__restrict__ pass_hist,
                     uint32_t *records, uint32_t *tile_counter,
                     uint32_t *status, bool aligned) {
  constexpr uint32_t kTile = kBlock * kItems;
  constexpr uint32_t kKeyBytes = kTile * sizeof(K);
  constexpr uint32_t kValBytes = HasValues ? kTile * 4u : 0u;
  static_assert(kTile <= 0xffffu, "ranks are 16-bit");
  __shared__ uint64_t s_bar;
  __shared__ uint32_t s_tile;
  // per (warp, digit): the warp's count, then its tile-local base
  __shared__ uint16_t s_warp_base[kWarps][kBins];
  __shared__ uint32_t s_match[Ballots ? 1 : kWarps][Ballots ? 1 : kBins];
  __shared__ uint32_t s_count[Early ? kBins : 1];
  __shared__ uint32_t s_global[kBins];
  __shared__ uint32_t s_tmp[kWarps];
  // The tile arrives here (input order), and later holds it sorted by digit.
  __shared__ __align__(128) K s_keys[kTile];
  __shared__ __align__(128) uint32_t s_vals[HasValues ? kTile : 1];

  const uint32_t t = threadIdx.x, lane = lane_id(), warp = t / kWarp;
  if (t == 0) {
    const uint32_t tile = atomicAdd(tile_counter, 1u);
    s_tile = tile;
    if (aligned && static_cast<uint64_t>(tile + 1) * kTile <= count) {
      const uint64_t b = static_cast<uint64_t>(tile) * kTile;
      mbar_init(&s_bar, 1);
      mbar_arrive_expect_tx(&s_bar, kKeyBytes + kValBytes);
      bulk_load(s_keys, in_keys + b, kKeyBytes, &s_bar);
      if (HasValues) bulk_load(s_vals, in_vals + b, kValBytes, &s_bar);
    }
  }
  // Where each digit's run of this pass starts (independent of the tile).
  const uint32_t hist_t = pass_hist[t];
#pragma unroll
  for (uint32_t w = 0; w < kWarps; ++w) s_warp_base[w][t] = 0;
  if (!Ballots) {
#pragma unroll
    for (uint32_t w = 0; w < kWarps; ++w) s_match[w][t] = 0;
  }
  if (Early) s_count[t] = 0;
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint32_t tile_base = tile * kTile; // count < 2^30
  const uint32_t valid_in_tile = count - tile_base < kTile ? count - tile_base : kTile;
  const bool full = valid_in_tile == kTile;
  if (aligned && full) {
    if (!mbar_wait(&s_bar, 0)) {
      // Never expected: report, let the copies land, give up on this tile.
      if (t == 0) set_status(status, kDevTimeout);
      mbar_wait(&s_bar, 0);
      return;
    }
  } else {
    for (uint32_t j = t; j < valid_in_tile; j += kBlock) {
      s_keys[j] = in_keys[tile_base + j];
      if (HasValues) s_vals[j] = in_vals[tile_base + j];
    }
    __syncthreads();
  }
  const uint32_t warp_first = warp * kWarp * kItems; // tile-local index of item 0
  // Item i of this lane is tile-local key warp_first + i * 32 + lane; a lane
  // past the end of a partial tile holds no key (digit kBins).
  auto valid = [&](uint32_t i) { return full || warp_first + i * kWarp + lane < valid_in_tile; };

  K key[kItems];
  uint32_t val[kItems];
  uint32_t rank2[(kItems + 1) / 2]; // ranks within the warp's keys of a digit, 16 bits each
#pragma unroll
  for (uint32_t i = 0; i < kItems; ++i) {
    const uint32_t j = warp_first + i * kWarp + lane;
    key[i] = valid(i) ? s_keys[j] : K(0);
    val[i] = HasValues && valid(i) ? s_vals[j] : 0u;
  }

  uint32_t *rec = records + static_cast<size_t>(tile) * kBins + t;
  if (Early) {
#pragma unroll
    for (uint32_t i = 0; i < kItems; ++i)
      if (valid(i)) atomicAdd(&s_count[digit_of(key[i], shift, mask)], 1u);
    __syncthreads();
    st_relaxed_u32(rec, (tile == 0 ? kRecInc : kRecAgg) | s_count[t]);
  }

  // Rank each key among the warp's earlier keys of its digit (stable: the
  // order of items, then of lanes).
#pragma unroll
  for (uint32_t i = 0; i < kItems; ++i) {
    const bool v = valid(i);
    const uint32_t d = v ? digit_of(key[i], shift, mask) : kBins;
    uint32_t peers;
    if (Ballots) {
      peers = kFullMask;
      if (!full) { // lanes without a key form their own group
        const uint32_t vb = __ballot_sync(kFullMask, v);
        peers = v ? vb : ~vb;
      }
#pragma unroll
      for (uint32_t b = 0; b < kRadixBits; ++b) {
        const bool bit = (d >> b) & 1u;
        const uint32_t bb = __ballot_sync(kFullMask, bit);
        peers &= bit ? bb : ~bb;
      }
    } else {
      if (v) atomicOr(&s_match[warp][d], 1u << lane);
      __syncwarp();
      peers = v ? s_match[warp][d] : 0u;
    }
    uint32_t pre = 0;
    if (v) pre = s_warp_base[warp][d];
    __syncwarp();
    if (v && lane == 31u - __clz(peers)) { // the digit's last lane
      s_warp_base[warp][d] = static_cast<uint16_t>(pre + __popc(peers));
      if (!Ballots) s_match[warp][d] = 0u;
    }
    __syncwarp();
    const uint32_t rk = pre + __popc(peers & lanemask_lt());
    if (i & 1u) rank2[i / 2] |= rk << 16;
    else rank2[i / 2] = rk;
  }
  __syncthreads();

  // Thread t owns digit t: the warps' counts become tile-local bases.
  uint32_t wc[kWarps], tile_count = 0;
#pragma unroll
  for (uint32_t w = 0; w < kWarps; ++w) {
    wc[w] = s_warp_base[w][t];
    tile_count += wc[w];
  }
  if (!Early) st_relaxed_u32(rec, (tile == 0 ? kRecInc : kRecAgg) | tile_count);
  const uint32_t digit_off = block_exclusive_256(tile_count, s_tmp);
  {
    uint32_t run = digit_off;
#pragma unroll
    for (uint32_t w = 0; w < kWarps; ++w) {
      s_warp_base[w][t] = static_cast<uint16_t>(run);
      run += wc[w];
    }
  }
  const uint32_t global_start = block_exclusive_256(hist_t, s_tmp);
  const uint32_t exclusive = digit_lookback(records, tile, t, tile_count, status);
  s_global[t] = global_start + exclusive - digit_off;
  __syncthreads();

  // Sort the tile in shared memory (its input copy is in registers now).
#pragma unroll
  for (uint32_t i = 0; i < kItems; ++i) {
    if (!valid(i)) continue;
    const uint32_t d = digit_of(key[i], shift, mask);
    const uint32_t rk = (i & 1u) ? (rank2[i / 2] >> 16) : (rank2[i / 2] & 0xffffu);
    const uint32_t pos = s_warp_base[warp][d] + rk;
    s_keys[pos] = key[i];
    if (HasValues) s_vals[pos] = val[i];
  }
  __syncthreads();

  // Write the tile's runs out in order: consecutive threads, consecutive
  // addresses of each run.  dst stays below count even after a look-back
  // timeout (a partial prefix is a lower bound of the true one).
#pragma unroll
  for (uint32_t r = 0; r < kItems; ++r) {
    const uint32_t j = r * kBlock + t;
    if (!full && j >= valid_in_tile) break;
    const K k = s_keys[j];
    const uint32_t dst = s_global[digit_of(k, shift, mask)] + j;
    out_keys[dst] = k;
    if (HasValues) out_vals[dst] = s_vals[j];
  }
}

template <class K>
vx_status sort_pairs(K *keys, uint32_t *values, uint32_t count,
                     uint32_t key_bits, void *workspace, size_t ws_bytes,
                     cudaStream_t stream) {
  constexpr uint32_t kMaxBits = sizeof(K) * 8;
  if (key_bits == 0 || key_bits > kMaxBits) return VX_ERR_INVALID_VALUE;
  if (keys == nullptr && count != 0) return VX_ERR_INVALID_VALUE;
  if (count > kMaxCount) return VX_ERR_INVALID_VALUE;
  if (count <= 1) return VX_OK;
  const uint32_t radix = radix_bits_for(key_bits);
  const uint32_t passes = pass_count(key_bits, radix);
  if (workspace == nullptr || ws_bytes < workspace_bytes<K>(count, passes))
    return VX_ERR_INVALID_VALUE;
  const Layout l = carve<K>(workspace, count, passes);
  VX_TRY_CUDA(cudaMemsetAsync(workspace, 0, l.clear_bytes, stream));

  PassInfo info{};
  for (uint32_t p = 0; p < passes; ++p) {
    info.shift[p] = p * radix;
    const uint32_t bits = key_bits - p * radix < radix ? key_bits - p * radix : radix;
    info.mask[p] = (1u << bits) - 1u;
  }
  const uint32_t hist_blocks =
      std::min<uint32_t>(ceil_div(count, kBlock * 16), sm_count() * 4);
  {
    prof::Scope scope(sizeof(K) == 4 ? "sort_histogram_u32" : "sort_histogram_u64", stream);
    histogram_kernel<K><<<hist_blocks, kBlock, 0, stream>>>(keys, count, passes,
                                                            info, l.hist);
  }
  VX_TRY_CUDA(cudaGetLastError());

  const bool large = tune::get(sizeof(K) == 4 ? tune::kSortItemsU32 : tune::kSortItemsU64) ==
                     static_cast<int64_t>(Shape<K>::kLarge);
  const bool early = tune::get(tune::kSortEarlyCounts) != 0;
  const bool ballots = tune::get(tune::kSortRankBallots) != 0;
  const uint32_t items = large ? Shape<K>::kLarge : Shape<K>::kSmall;
  const uint32_t tiles = ceil_div(count, kBlock * items);
  K *src_k = keys, *dst_k = static_cast<K *>(l.tmp_keys);
  uint32_t *src_v = values, *dst_v = l.tmp_vals;
  auto aligned16 = [](const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
  for (uint32_t p = 0; p < passes; ++p) {
    uint32_t *rec = l.records + static_cast<size_t>(p) * tiles * kBins;
    prof::Scope scope(sizeof(K) == 4 ? "sort_partition_u32" : "sort_partition_u64", stream);
    const bool aligned = aligned16(src_k) && (values == nullptr || aligned16(src_v));
    auto launch = [&](auto kernel) {
      kernel<<<tiles, kBlock, 0, stream>>>(src_k, src_v, dst_k, dst_v, count, info.shift[p],
                                           info.mask[p], l.hist + p * kBins, rec,
                                           l.counters + 2 + p, l.counters + 1, aligned);
    };
    // (values, items, early, ballots) -> one of 16 instantiations
    auto by_ballots = [&](auto hv, auto it, auto ea) {
      constexpr bool HV = decltype(hv)::value, E = decltype(ea)::value;
      constexpr uint32_t I = decltype(it)::value;
      if (ballots) launch(partition_kernel<K, HV, I, E, true>);
      else launch(partition_kernel<K, HV, I, E, false>);
    };
    auto by_early = [&](auto hv, auto it) {
      if (early) by_ballots(hv, it, std::true_type{});
      else by_ballots(hv, it, std::false_type{});
    };
    auto by_items = [&](auto hv) {
      if (large) by_early(hv, std::integral_constant<uint32_t, Shape<K>::kLarge>{});
      else by_early(hv, std::integral_constant<uint32_t, Shape<K>::kSmall>{});
    };
    if (values != nullptr) by_items(std::true_type{});
    else by_items(std::false_type{});
    VX_TRY_CUDA(cudaGetLastError());
    std::swap(src_k, dst_k);
    std::swap(src_v, dst_v);
  }
  if (src_k != keys) {
    VX_TRY_CUDA(cudaMemcpyAsync(keys, src_k, sizeof(K) * count,
                                cudaMemcpyDeviceToDevice, stream));
    if (values != nullptr)
      VX_TRY_CUDA(cudaMemcpyAsync(values, src_v, sizeof(uint32_t) * count,
                                  cudaMemcpyDeviceToDevice, stream));
  }
  return VX_OK;
}

// ------------------------------------------------ multi-word keys --
//
// Keys of `words` 32-bit words (word 0 least significant, the reference's
// UIntKey<W>, cuda/sort/uint_key.cuh:15-66) are sorted least significant
// chunk first: each chunk of up to 64 key bits (words 2c, 2c + 1) is
// gathered through the permutation built so far and sorted stably together
// with it by this file's onesweep sort, so the permutation ends up ordering
// the keys by their low key_bits bits, stably; the keys are then gathered
// once through it.

__global__ void iota_kernel(uint32_t *p, uint32_t n) {
  const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (i < n) p[i] = static_cast<uint32_t>(i);
}

template <class C>
__global__ void chunk_kernel(const uint32_t *__restrict__ keys, uint32_t words,
                             const uint32_t *__restrict__ perm, uint32_t first_word,
                             uint32_t n, C *__restrict__ out) {
  const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const uint32_t *k = keys + static_cast<size_t>(perm[i]) * words + first_word;
  C v = k[0];
  if constexpr (sizeof(C) == 8)
    if (first_word + 1 < words) v |= static_cast<uint64_t>(k[1]) << 32;
  out[i] = v;
}

// dst[i] = src[index[i]] for elements of W-byte words x n_words.
template <class W>
__global__ void gather_kernel(W *__restrict__ dst, const W *__restrict__ src,
                              const uint32_t *__restrict__ index, uint32_t count,
                              uint32_t n_words) {
  const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (i >= count) return;
  const W *s = src + static_cast<size_t>(index[i]) * n_words;
  W *d = dst + i * n_words;
  for (uint32_t w = 0; w < n_words; ++w) d[w] = s[w];
}

namespace {

constexpr size_t kWordsAlign = 256;
inline size_t align_up(size_t v) { return (v + kWordsAlign - 1) & ~(kWordsAlign - 1); }

struct WordsLayout {
  size_t sort_ws, perm, chunk, keys, total;
};
inline WordsLayout words_layout(uint32_t count, uint32_t words) {
  WordsLayout l{};
  l.sort_ws = 0;
  const size_t sort_bytes = workspace_bytes<uint64_t>(count, kMaxPasses);
  l.perm = align_up(sort_bytes);
  l.chunk = l.perm + align_up(sizeof(uint32_t) * size_t(count));
  l.keys = l.chunk + align_up(sizeof(uint64_t) * size_t(count));
  l.total = l.keys + align_up(sizeof(uint32_t) * size_t(words) * count);
  return l;
}

} // namespace

vx_status gather(void *dst, const void *src, const uint32_t *index, uint32_t count,
                 uint32_t elem_bytes, cudaStream_t stream) {
  if (count == 0) return VX_OK;
  if (dst == nullptr || src == nullptr || index == nullptr || elem_bytes == 0)
    return VX_ERR_INVALID_VALUE;
  const uintptr_t a = reinterpret_cast<uintptr_t>(dst) | reinterpret_cast<uintptr_t>(src);
  const uint32_t grid = ceil_div(count, kBlock);
  prof::Scope scope("sort_gather", stream);
  if (elem_bytes % 16 == 0 && (a & 15u) == 0)
    gather_kernel<uint4><<<grid, kBlock, 0, stream>>>(static_cast<uint4 *>(dst),
                                                      static_cast<const uint4 *>(src), index,
                                                      count, elem_bytes / 16);
  else if (elem_bytes % 8 == 0 && (a & 7u) == 0)
    gather_kernel<uint64_t><<<grid, kBlock, 0, stream>>>(static_cast<uint64_t *>(dst),
                                                         static_cast<const uint64_t *>(src),
                                                         index, count, elem_bytes / 8);
  else if (elem_bytes % 4 == 0 && (a & 3u) == 0)
    gather_kernel<uint32_t><<<grid, kBlock, 0, stream>>>(static_cast<uint32_t *>(dst),
                                                         static_cast<const uint32_t *>(src),
                                                         index, count, elem_bytes / 4);
  else if (elem_bytes % 2 == 0 && (a & 1u) == 0)
    gather_kernel<uint16_t><<<grid, kBlock, 0, stream>>>(static_cast<uint16_t *>(dst),
                                                         static_cast<const uint16_t *>(src),
                                                         index, count, elem_bytes / 2);
  else
    gather_kernel<uint8_t><<<grid, kBlock, 0, stream>>>(static_cast<uint8_t *>(dst),
                                                        static_cast<const uint8_t *>(src),
                                                        index, count, elem_bytes);
  return from_cuda(cudaGetLastError());
}

vx_status sort_words(uint32_t *keys, uint32_t words, uint32_t count, uint32_t key_bits,
                     uint32_t *perm_out, void *workspace, size_t ws_bytes,
                     cudaStream_t stream) {
  if (words == 0 || words > 64 || key_bits == 0 || key_bits > 32u * words)
    return VX_ERR_INVALID_VALUE;
  if (keys == nullptr && count != 0) return VX_ERR_INVALID_VALUE;
  if (count > kMaxCount) return VX_ERR_INVALID_VALUE;
  if (count == 0) return VX_OK;
  const WordsLayout l = words_layout(count, words);
  if (workspace == nullptr || ws_bytes < l.total) return VX_ERR_INVALID_VALUE;
  char *base = static_cast<char *>(workspace);
  uint32_t *perm = reinterpret_cast<uint32_t *>(base + l.perm);
  void *chunk = base + l.chunk;
  const uint32_t grid = ceil_div(count, kBlock);
  iota_kernel<<<grid, kBlock, 0, stream>>>(perm, count);
  VX_TRY_CUDA(cudaGetLastError());
  const size_t sort_bytes = workspace_bytes<uint64_t>(count, kMaxPasses);
  for (uint32_t lo = 0; lo < key_bits; lo += 64) {
    const uint32_t bits = key_bits - lo < 64 ? key_bits - lo : 64;
    const uint32_t first = lo / 32;
    if (bits <= 32) {
      auto *c = static_cast<uint32_t *>(chunk);
      chunk_kernel<uint32_t><<<grid, kBlock, 0, stream>>>(keys, words, perm, first, count, c);
      VX_TRY_CUDA(cudaGetLastError());
      VX_TRY(sort_pairs<uint32_t>(c, perm, count, bits, workspace, sort_bytes, stream));
    } else {
      auto *c = static_cast<uint64_t *>(chunk);
      chunk_kernel<uint64_t><<<grid, kBlock, 0, stream>>>(keys, words, perm, first, count, c);
      VX_TRY_CUDA(cudaGetLastError());
      VX_TRY(sort_pairs<uint64_t>(c, perm, count, bits, workspace, sort_bytes, stream));
    }
  }
  uint32_t *tmp = reinterpret_cast<uint32_t *>(base + l.keys);
  VX_TRY(gather(tmp, keys, perm, count, 4u * words, stream));
  VX_TRY_CUDA(cudaMemcpyAsync(keys, tmp, sizeof(uint32_t) * size_t(words) * count,
                              cudaMemcpyDeviceToDevice, stream));
  if (perm_out != nullptr)
    VX_TRY_CUDA(cudaMemcpyAsync(perm_out, perm, sizeof(uint32_t) * size_t(count),
                                cudaMemcpyDeviceToDevice, stream));
  return VX_OK;
}

} // namespace vx::sort

extern "C" {

size_t vx_sort_words_workspace_size(uint32_t count, uint32_t words) {
  if (count == 0 || words == 0) return 0;
  return vx::sort::words_layout(count, words).total;
}

vx_status vx_sort_words(uint32_t *keys, uint32_t words, uint32_t count, uint32_t key_bits,
                        uint32_t *perm, void *workspace, size_t workspace_bytes,
                        vx_stream stream) {
  return vx::sort::sort_words(keys, words, count, key_bits, perm, workspace, workspace_bytes,
                              static_cast<cudaStream_t>(stream));
}

vx_status vx_gather(void *dst, const void *src, const uint32_t *index, uint32_t count,
                    uint32_t elem_bytes, vx_stream stream) {
  return vx::sort::gather(dst, src, index, count, elem_bytes, static_cast<cudaStream_t>(stream));
}

size_t vx_sort_workspace_size(uint32_t count, uint32_t key_bytes) {
  if (count <= 1) return 0;
  if (key_bytes == 8)
    return vx::sort::workspace_bytes<uint64_t>(count, vx::sort::kMaxPasses);
  // passes of 32-bit keys at the narrowest digit
  return vx::sort::workspace_bytes<uint32_t>(count,
                                             vx::sort::pass_count(32, vx::sort::kMinRadixBits));
}

vx_status vx_sort_pairs_u32(uint32_t *keys, uint32_t *values, uint32_t count,
                            uint32_t key_bits, void *workspace,
                            size_t workspace_bytes, vx_stream stream) {
  return vx::sort::sort_pairs<uint32_t>(keys, values, count, key_bits,
                                        workspace, workspace_bytes,
                                        static_cast<cudaStream_t>(stream));
}

vx_status vx_sort_pairs_u64(uint64_t *keys, uint32_t *values, uint32_t count,
                            uint32_t key_bits, void *workspace,
                            size_t workspace_bytes, vx_stream stream) {
  return vx::sort::sort_pairs<uint64_t>(keys, values, count, key_bits,
                                        workspace, workspace_bytes,
                                        static_cast<cudaStream_t>(stream));
}

} // extern "C"
