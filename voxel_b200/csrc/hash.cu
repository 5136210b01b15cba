// u64-keyed hash tables for sm_100a.
//
// Slab hash set: the u64 widening of the reference's BasicSlabHashSetU32
// (cuda/hash_table/slab_hash/set/host.cuh:13-121, device.cuh:31-315).  A slab
// is one 128-byte line: 15 u64 key slots and a u64 link to the next slab of
// the bucket's chain.  Where the reference's warp serves one key at a time,
// here every thread walks its own key: a slab is read one 32-byte sector at a
// time starting at the key's home sector, and the walk ends at the first
// empty slot (inserts take the first free slot in that order), so most
// lookups read one sector and a warp has 32 keys in flight.  Inserts CAS an
// empty or deleted slot; full chains grow from a pool of overflow slabs taken
// with a bump counter.  Statuses are the reference's kSlabHashStatus*
// values.  Every retry loop is bounded (the reference's
// kSlabHashMaxContentionRetries).
//
// Slab map: u32 -> u32, the reference's SlabHashMapU32 (below).
//
// Cuckoo map: the u64-keyed widening of cuckoo_insert / cuckoo_find
// (cuda/cuckoo_hash.cuh:54-120), bucketed: two hash functions each name a
// bucket of two 16-byte slots {key, value | choice << 32} (one 32-byte
// sector), so a lookup is two independent sector loads; an eviction moves a
// whole slot with one 128-bit atomic exchange (atom.exch.b128, sm_90+), so
// key and value never separate.  Eviction chains are bounded by
// max_evictions (the reference's insertion_attempts); a chain that runs out
// drops the key in hand, reports VX_HASH_OVERFLOW and counts it.
#include "common.cuh"
#include "profile.cuh"
#include "voxel_b200_device.cuh"

#include <algorithm>
#include <new>

namespace vx::hash {

constexpr uint64_t kEmpty = VX_HASH_EMPTY_KEY;
constexpr uint64_t kDeleted = VX_HASH_DELETED_KEY;
constexpr uint64_t kNullLink = ~0ull;
constexpr uint32_t kSlotsPerSlab = 15;
constexpr uint32_t kMaxContentionRetries = 65536;
constexpr uint32_t kBlock = 256;

// The hashes are voxel_b200_device.cuh's, which user kernels share.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) { return vx_mix64(x); }
__device__ __forceinline__ uint32_t reduce(uint64_t h, uint32_t n) {
  return vx_reduce_hash(h, n);
}

struct Slab {
  uint64_t w[16]; // w[0..14] keys, w[15] link
};
static_assert(sizeof(Slab) == 128, "slab must be one 128-byte line");

} // namespace vx::hash

struct vx_slab_set {
  vx::hash::Slab *slabs = nullptr; // buckets, then the overflow pool
  uint32_t *alloc = nullptr;       // overflow slabs handed out
  uint32_t bucket_count = 0;
  uint32_t capacity = 0;
};

struct vx_slab_map {
  vx::hash::Slab *slabs = nullptr; // buckets, then the overflow pool
  uint32_t *alloc = nullptr;
  uint32_t bucket_count = 0;
  uint32_t capacity = 0;
};

struct vx_cuckoo {
  ulonglong2 *slots = nullptr;
  unsigned long long *dropped = nullptr;
  uint32_t slot_count = 0;
  uint32_t max_evictions = 0;
};

namespace vx::hash {

struct SetView {
  Slab *slabs;
  uint32_t *alloc;
  uint32_t bucket_count;
  uint32_t capacity;
};

__global__ void slab_init_kernel(SetView t, uint64_t words) {
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
       i < words; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    reinterpret_cast<uint64_t *>(t.slabs)[i] = (i & 15u) == 15u ? kNullLink : kEmpty;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *t.alloc = 0;
}

enum class SetOp { Insert, Contains, Erase };

// Probe order of a key inside every slab of its chain: its home sector (32
// bytes: 4 key slots; the last sector has 3 and the link) first, then the
// next ones cyclically.  An insert takes the first free slot (empty or
// deleted) in that order, so a key present in the chain always lies before
// the first empty slot of its order: a lookup reads one sector at a time and
// stops at the first empty slot, which for most keys is in the home sector.
__device__ __forceinline__ uint32_t home_sector(uint64_t h) { return static_cast<uint32_t>(h) & 3u; }

__device__ __forceinline__ ulonglong2 ld_relaxed_u64x2(const uint64_t *p) {
  ulonglong2 v;
  asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];"
               : "=l"(v.x), "=l"(v.y)
               : "l"(p)
               : "memory");
  return v;
}

// Sector j of a slab: words 4j .. 4j + 3 (two 16-byte relaxed loads, one
// 32-byte sector).
__device__ __forceinline__ void ld_sector(const Slab *slab, uint32_t j, uint64_t w[4]) {
  const ulonglong2 a = ld_relaxed_u64x2(&slab->w[4 * j]);
  const ulonglong2 b = ld_relaxed_u64x2(&slab->w[4 * j + 2]);
  w[0] = a.x;
  w[1] = a.y;
  w[2] = b.x;
  w[3] = b.y;
}

// One key per thread: every lane walks its own key's chain (no warp
// cooperation), so a warp has 32 keys in flight.
template <SetOp Op>
__global__ void __launch_bounds__(kBlock)
    slab_set_kernel(SetView t, const uint64_t *__restrict__ keys,
                    uint32_t count, uint32_t *contains, uint32_t *statuses) {
  for (uint64_t idx = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; idx < count;
       idx += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint64_t k = keys[idx];
    uint32_t result;
    if (k == kEmpty || k == kDeleted) {
      result = VX_HASH_INVALID_KEY;
    } else {
      const uint64_t h = mix64(k);
      const uint32_t home = home_sector(h);
      Slab *const first = &t.slabs[reduce(h, t.bucket_count)];
      result = VX_HASH_OVERFLOW;
      // a chain is at most the pool long; a lost CAS restarts the walk
      const uint64_t max_steps = (t.capacity + 1ull) * 4ull;
      uint32_t restarts = 0;
      bool restart = true;
      while (restart && restarts++ < kMaxContentionRetries) {
        restart = false;
        Slab *slab = first;
        uint64_t *free_slot = nullptr; // first free slot of the walk (insert)
        uint64_t free_old = 0;
        bool done = false;
        for (uint64_t step = 0; step < max_steps && !done;) {
          uint64_t link = kNullLink;
          bool ended = false; // met an empty slot: the key is not further on
          for (uint32_t q = 0; q < 4 && !done && !ended; ++q, ++step) {
            const uint32_t j = (home + q) & 3u;
            uint64_t w[4];
            ld_sector(slab, j, w);
            const uint32_t slots = j == 3 ? 3u : 4u;
            if (j == 3) link = w[3];
            for (uint32_t i = 0; i < slots; ++i) {
              if (w[i] == k) {
                if (Op == SetOp::Erase) {
                  const unsigned long long old = atomicCAS(
                      reinterpret_cast<unsigned long long *>(&slab->w[4 * j + i]), k, kDeleted);
                  if (old == k) result = VX_HASH_ERASED;
                  else restart = true; // changed meanwhile: walk again
                } else {
                  result = Op == SetOp::Insert ? VX_HASH_ALREADY_PRESENT : VX_HASH_FOUND;
                }
                done = true;
                break;
              }
              if (Op == SetOp::Insert && free_slot == nullptr && (w[i] == kEmpty || w[i] == kDeleted)) {
                free_slot = &slab->w[4 * j + i];
                free_old = w[i];
              }
              if (w[i] == kEmpty) {
                ended = true;
                break;
              }
            }
          }
          if (done) break;
          if (ended || link == kNullLink) {
            if (Op != SetOp::Insert) {
              result = VX_HASH_NOT_FOUND;
              done = true;
              break;
            }
            if (free_slot != nullptr) {
              const unsigned long long old = atomicCAS(
                  reinterpret_cast<unsigned long long *>(free_slot), free_old, k);
              if (old == free_old) result = VX_HASH_INSERTED;
              else restart = true;
              done = true;
              break;
            }
            // Full chain: take a pool slab, initialise it, link it with CAS.
            const uint32_t ord = atomicAdd(t.alloc, 1u);
            if (ord >= t.capacity) {
              // pool exhausted; another thread may have linked a slab since
              const uint64_t again = ld_relaxed_u64(&slab->w[15]);
              if (again != kNullLink) {
                slab = &t.slabs[again];
                continue;
              }
              result = VX_HASH_OVERFLOW;
              done = true;
              break;
            }
            Slab *fresh = &t.slabs[t.bucket_count + ord];
            for (uint32_t i = 0; i < 15; ++i) fresh->w[i] = kEmpty;
            fresh->w[15] = kNullLink;
            __threadfence();
            const unsigned long long observed = atomicCAS(
                reinterpret_cast<unsigned long long *>(&slab->w[15]), kNullLink,
                t.bucket_count + ord);
            // either our slab was linked or another thread's was: follow it
            // (a pool slab that lost the race stays unused)
            slab = &t.slabs[observed == kNullLink ? t.bucket_count + ord : observed];
            continue;
          }
          slab = &t.slabs[link];
        }
      }
    }
    if (statuses) statuses[idx] = result;
    if (Op == SetOp::Contains && contains) contains[idx] = result == VX_HASH_FOUND ? 1u : 0u;
  }
}

// ---------------------------------------------------------- slab map --
//
// u32 -> u32 map (the reference's SlabHashMapU32, cuda/hash_table/slab_hash/
// map/device.cuh:49-372): a 128-byte slab holds 15 slots packed as
// key | value << 32 and a link, so a slot changes with one 64-bit CAS.  As in
// the reference a warp serves its keys one at a time in lane order (later
// duplicates of a key in a batch replace earlier ones), an insert takes the
// first slot of the chain that holds the key, is empty or is deleted, a find
// returns the first match, and erase_all deletes every match.

constexpr uint32_t kMapEmpty = VX_MAP_EMPTY_KEY, kMapDeleted = VX_MAP_DELETED_KEY;

__device__ __forceinline__ uint64_t map_pack(uint32_t k, uint32_t v) {
  return static_cast<uint64_t>(k) | (static_cast<uint64_t>(v) << 32);
}

__global__ void map_init_kernel(SetView t, uint64_t words) {
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
       i < words; i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    reinterpret_cast<uint64_t *>(t.slabs)[i] = (i & 15u) == 15u ? kNullLink : map_pack(kMapEmpty, 0);
  if (blockIdx.x == 0 && threadIdx.x == 0) *t.alloc = 0;
}

enum class MapOp { InsertOrReplace, Find, EraseAll };

template <MapOp Op>
__global__ void __launch_bounds__(kBlock)
    slab_map_kernel(SetView t, const uint32_t *__restrict__ keys,
                    const uint32_t *__restrict__ values, uint32_t count,
                    uint32_t *out_values, uint32_t *statuses) {
  const uint32_t lane = lane_id();
  const uint32_t sub = lane & 15u;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  const uint64_t warp_first = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) - lane;
  for (uint64_t base = warp_first; base < count; base += stride) {
    const uint64_t idx = base + lane;
    bool active = idx < count;
    const uint32_t key = active ? keys[idx] : 0u;
    const uint32_t val = (active && Op == MapOp::InsertOrReplace) ? values[idx] : 0u;
    uint32_t status = VX_HASH_NOT_FOUND, out = VX_HASH_NOT_FOUND_VALUE;
    if (active && (key == kMapEmpty || key == kMapDeleted)) {
      status = VX_HASH_INVALID_KEY;
      active = false;
    }
    uint32_t queue = __ballot_sync(kFullMask, active);
    while (queue) {
      const uint32_t src = __ffs(queue) - 1u;
      const uint32_t k = __shfl_sync(kFullMask, key, src);
      const uint32_t v = __shfl_sync(kFullMask, val, src);
      Slab *slab = &t.slabs[reduce(mix64(k), t.bucket_count)];
      uint32_t result = VX_HASH_OVERFLOW, found_value = VX_HASH_NOT_FOUND_VALUE;
      bool erased_any = false;
      const uint64_t max_steps =
          Op == MapOp::Find ? t.capacity + 1ull
                            : (t.capacity + 1ull) * static_cast<uint64_t>(kMaxContentionRetries);
      for (uint64_t step = 0; step < max_steps; ++step) {
        // lanes 0..15 read the slab (16 words); lanes 16..31 mirror them
        const uint64_t w = ld_relaxed_u64(&slab->w[sub]);
        const bool slot = lane < kSlotsPerSlab;
        const uint32_t wk = static_cast<uint32_t>(w);
        if (Op == MapOp::Find) {
          const uint32_t hit = __ballot_sync(kFullMask, slot && wk == k);
          if (hit) {
            const uint64_t hw = __shfl_sync(kFullMask, w, __ffs(hit) - 1u);
            found_value = static_cast<uint32_t>(hw >> 32);
            result = VX_HASH_FOUND;
            break;
          }
        } else if (Op == MapOp::EraseAll) {
          const uint32_t hit = __ballot_sync(kFullMask, slot && wk == k);
          if (hit) {
            const uint32_t dst = __ffs(hit) - 1u;
            const uint64_t expect = __shfl_sync(kFullMask, w, dst);
            unsigned long long old = 0;
            if (lane == dst)
              old = atomicCAS(reinterpret_cast<unsigned long long *>(&slab->w[sub]), expect,
                              map_pack(kMapDeleted, static_cast<uint32_t>(expect >> 32)));
            old = __shfl_sync(kFullMask, old, dst);
            if (old == expect) erased_any = true;
            continue; // re-read this slab for further matches
          }
        } else {
          const uint32_t cand = __ballot_sync(
              kFullMask, slot && (wk == k || wk == kMapEmpty || wk == kMapDeleted));
          if (cand) {
            const uint32_t dst = __ffs(cand) - 1u;
            const uint64_t expect = __shfl_sync(kFullMask, w, dst);
            unsigned long long old = 0;
            if (lane == dst)
              old = atomicCAS(reinterpret_cast<unsigned long long *>(&slab->w[sub]), expect,
                              map_pack(k, v));
            old = __shfl_sync(kFullMask, old, dst);
            if (old == expect) {
              result = static_cast<uint32_t>(expect) == k ? VX_HASH_REPLACED : VX_HASH_INSERTED;
              break;
            }
            continue; // slot changed meanwhile: re-read this slab
          }
        }
        const uint64_t link = __shfl_sync(kFullMask, w, 15u);
        if (link != kNullLink) {
          slab = &t.slabs[link];
          continue;
        }
        if (Op == MapOp::Find) {
          result = VX_HASH_NOT_FOUND;
          break;
        }
        if (Op == MapOp::EraseAll) {
          result = erased_any ? VX_HASH_ERASED : VX_HASH_NOT_FOUND;
          break;
        }
        // Grow the chain: take a pool slab, initialise it, link it with CAS.
        uint32_t ord = 0;
        if (lane == 0) ord = atomicAdd(t.alloc, 1u);
        ord = __shfl_sync(kFullMask, ord, 0);
        if (ord >= t.capacity) {
          uint64_t again = 0;
          if (lane == 15u) again = ld_relaxed_u64(&slab->w[15]);
          again = __shfl_sync(kFullMask, again, 15u);
          if (again != kNullLink) {
            slab = &t.slabs[again];
            continue;
          }
          result = VX_HASH_OVERFLOW;
          break;
        }
        Slab *fresh = &t.slabs[t.bucket_count + ord];
        if (lane < 16u) fresh->w[sub] = sub == 15u ? kNullLink : map_pack(kMapEmpty, 0);
        __threadfence();
        __syncwarp();
        unsigned long long observed = 0;
        if (lane == 15u)
          observed = atomicCAS(reinterpret_cast<unsigned long long *>(&slab->w[15]),
                               kNullLink, t.bucket_count + ord);
        observed = __shfl_sync(kFullMask, observed, 15u);
        slab = &t.slabs[observed == kNullLink ? t.bucket_count + ord : observed];
      }
      if (lane == src) {
        status = result;
        out = found_value;
        active = false;
      }
      queue = __ballot_sync(kFullMask, active);
    }
    if (idx < count) {
      if (statuses) statuses[idx] = status;
      if (Op == MapOp::Find && out_values) out_values[idx] = out;
    }
  }
}

// ------------------------------------------------------------ cuckoo --
//
// Two-choice bucketed cuckoo: a bucket is one 32-byte sector holding two
// 16-byte slots {key, value | choice << 32}, and a key lives in one of its
// two buckets (vx_cuckoo_bucket).  A lookup loads both sectors at once (one
// round trip, two sectors).  An insert first replaces the value of a present
// key (128-bit CAS, keeping its choice), else claims a free slot of either
// bucket (128-bit CAS from empty), else evicts a slot of one of the buckets
// with a 128-bit exchange and carries the evicted entry to its other bucket,
// for at most max_evictions moves.

__device__ __forceinline__ ulonglong2 exch128(ulonglong2 *p, ulonglong2 v) {
  ulonglong2 old;
  asm volatile(
      "{\n\t.reg .b128 d, b;\n\t"
      "mov.b128 b, {%2, %3};\n\t"
      "atom.global.exch.b128 d, [%4], b;\n\t"
      "mov.b128 {%0, %1}, d;\n\t}"
      : "=l"(old.x), "=l"(old.y)
      : "l"(v.x), "l"(v.y), "l"(p)
      : "memory");
  return old;
}

// 128-bit compare-and-swap of one slot; returns the slot's previous contents.
__device__ __forceinline__ ulonglong2 cas128(ulonglong2 *p, ulonglong2 expected,
                                             ulonglong2 desired) {
  ulonglong2 old;
  asm volatile(
      "{\n\t.reg .b128 d, c, b;\n\t"
      "mov.b128 c, {%2, %3};\n\t"
      "mov.b128 b, {%4, %5};\n\t"
      "atom.global.cas.b128 d, [%6], c, b;\n\t"
      "mov.b128 {%0, %1}, d;\n\t}"
      : "=l"(old.x), "=l"(old.y)
      : "l"(expected.x), "l"(expected.y), "l"(desired.x), "l"(desired.y), "l"(p)
      : "memory");
  return old;
}

__device__ __forceinline__ ulonglong2 ld_slot(const ulonglong2 *p) {
  ulonglong2 v;
  asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];"
               : "=l"(v.x), "=l"(v.y)
               : "l"(p)
               : "memory");
  return v;
}

__global__ void cuckoo_init_kernel(ulonglong2 *slots, uint32_t n,
                                   unsigned long long *dropped) {
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
       i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    slots[i] = make_ulonglong2(kEmpty, 0);
  if (blockIdx.x == 0 && threadIdx.x == 0) *dropped = 0;
}

__device__ __forceinline__ uint64_t with_choice(uint64_t key_value_word, uint32_t choice) {
  return (key_value_word & 0xffffffffull) | (static_cast<uint64_t>(choice) << 32);
}

// Replace the value stored for key, keeping the slot's choice bits (the
// bucket the next eviction of this entry moves it from).  The swap is a
// 128-bit CAS on {key, old word}, so an entry that a concurrent eviction
// moved is looked up again rather than overwritten in its new occupant's
// slot.  Returns false when the key is not in the table (duplicate keys
// inside one insert batch are not supported, as in the reference).
__device__ __forceinline__ bool cuckoo_replace(ulonglong2 *slots, uint32_t nb, uint64_t key,
                                               uint32_t value) {
  for (uint32_t attempt = 0; attempt < 64; ++attempt) {
    ulonglong2 *b0 = slots + 2ull * vx_cuckoo_bucket(key, 0, nb);
    ulonglong2 *b1 = slots + 2ull * vx_cuckoo_bucket(key, 1, nb);
    ulonglong2 *where = nullptr;
    ulonglong2 cur{};
    ulonglong2 *cand[4] = {b0, b0 + 1, b1, b1 + 1};
    ulonglong2 v[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = ld_slot(cand[i]);
#pragma unroll
    for (int i = 0; i < 4; ++i)
      if (where == nullptr && v[i].x == key) {
        where = cand[i];
        cur = v[i];
      }
    if (where == nullptr) return false;
    const ulonglong2 want = make_ulonglong2(key, (cur.y & 0xffffffff00000000ull) | value);
    const ulonglong2 seen = cas128(where, cur, want);
    if (seen.x == cur.x && seen.y == cur.y) return true;
  }
  return false;
}

// Claim a free slot of bucket b for entry e (choice c); true on success.
__device__ __forceinline__ bool cuckoo_claim(ulonglong2 *bucket, ulonglong2 e, uint32_t c) {
  const ulonglong2 want = make_ulonglong2(e.x, with_choice(e.y, c));
  for (int i = 0; i < 2; ++i) {
    if (ld_slot(bucket + i).x != kEmpty) continue;
    const ulonglong2 seen = cas128(bucket + i, make_ulonglong2(kEmpty, 0ull), want);
    if (seen.x == kEmpty && seen.y == 0ull) return true;
  }
  return false;
}

__global__ void __launch_bounds__(kBlock)
    cuckoo_insert_kernel(ulonglong2 *slots, uint32_t n, uint32_t max_evictions,
                         unsigned long long *dropped,
                         const uint64_t *__restrict__ keys,
                         const uint32_t *__restrict__ values, uint32_t count,
                         uint32_t *statuses) {
  const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (i >= count) return;
  const uint32_t nb = n / 2u;
  const uint64_t key = keys[i];
  const uint32_t value = values ? values[i] : static_cast<uint32_t>(i);
  uint32_t status;
  if (key == kEmpty || key == kDeleted) {
    status = VX_HASH_INVALID_KEY;
  } else if (cuckoo_replace(slots, nb, key, value)) {
    status = VX_HASH_REPLACED;
  } else {
    ulonglong2 cur = make_ulonglong2(key, value);
    status = VX_HASH_OVERFLOW;
    // a new key may go to either bucket; an evicted one to its other bucket
    int from = -1;
    uint64_t rnd = mix64(key ^ 0x5851f42d4c957f2dull);
    for (uint32_t a = 0; a <= max_evictions; ++a) {
      bool placed = false;
      uint32_t target;
      if (from < 0) {
        const uint32_t first = static_cast<uint32_t>(rnd >> 63);
        placed = cuckoo_claim(slots + 2ull * vx_cuckoo_bucket(cur.x, first, nb), cur, first) ||
                 cuckoo_claim(slots + 2ull * vx_cuckoo_bucket(cur.x, 1u - first, nb), cur,
                              1u - first);
        target = first;
      } else {
        target = 1u - static_cast<uint32_t>(from);
        placed = cuckoo_claim(slots + 2ull * vx_cuckoo_bucket(cur.x, target, nb), cur, target);
      }
      if (placed) {
        status = VX_HASH_INSERTED;
        break;
      }
      // evict one of the target bucket's two slots
      rnd = mix64(rnd + a);
      ulonglong2 *victim = slots + 2ull * vx_cuckoo_bucket(cur.x, target, nb) + (rnd & 1u);
      const ulonglong2 prev =
          exch128(victim, make_ulonglong2(cur.x, with_choice(cur.y, target)));
      if (prev.x == kEmpty || prev.x == cur.x) { // a free slot, or the same key
        status = VX_HASH_INSERTED;
        break;
      }
      cur = prev;
      from = static_cast<int>(prev.y >> 32) & 1;
    }
    if (status == VX_HASH_OVERFLOW) atomicAdd(dropped, 1ull);
  }
  if (statuses) statuses[i] = status;
}

__global__ void __launch_bounds__(kBlock)
    cuckoo_find_kernel(const ulonglong2 *slots, uint32_t n,
                       const uint64_t *__restrict__ keys, uint32_t count,
                       uint32_t *values) {
  const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (i >= count) return;
  uint32_t v = VX_HASH_NOT_FOUND_VALUE;
  vx_cuckoo_find(vx_cuckoo_view{slots, n, 0}, keys[i], &v);
  values[i] = v;
}

inline uint32_t grid_for(uint64_t items, uint32_t per_block = kBlock) {
  const uint64_t g = (items + per_block - 1) / per_block;
  const uint64_t cap = static_cast<uint64_t>(sm_count()) * 16u;
  return static_cast<uint32_t>(g < 1 ? 1 : (g > cap ? cap : g));
}

} // namespace vx::hash

using namespace vx::hash;

static SetView view_of(const vx_slab_set *s) {
  return SetView{s->slabs, s->alloc, s->bucket_count, s->capacity};
}

template <SetOp Op>
static vx_status slab_launch(const vx_slab_set *s, const uint64_t *keys,
                             uint32_t count, uint32_t *contains,
                             uint32_t *statuses, vx_stream stream,
                             const char *name) {
  if (s == nullptr || (keys == nullptr && count != 0)) return VX_ERR_INVALID_VALUE;
  if (Op == SetOp::Contains && contains == nullptr && count != 0)
    return VX_ERR_INVALID_VALUE;
  if (count == 0) return VX_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  vx::prof::Scope scope(name, st);
  slab_set_kernel<Op><<<grid_for(count), kBlock, 0, st>>>(view_of(s), keys, count,
                                                          contains, statuses);
  return vx::from_cuda(cudaGetLastError());
}


template <MapOp Op>
static vx_status map_launch(const vx_slab_map *m, const uint32_t *keys, const uint32_t *values,
                            uint32_t count, uint32_t *out_values, uint32_t *statuses,
                            vx_stream stream, const char *name) {
  if (m == nullptr || (keys == nullptr && count != 0)) return VX_ERR_INVALID_VALUE;
  if (Op == MapOp::InsertOrReplace && values == nullptr && count != 0)
    return VX_ERR_INVALID_VALUE;
  if (Op == MapOp::Find && out_values == nullptr && count != 0) return VX_ERR_INVALID_VALUE;
  if (count == 0) return VX_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  vx::prof::Scope scope(name, st);
  slab_map_kernel<Op><<<grid_for(count), kBlock, 0, st>>>(
      SetView{m->slabs, m->alloc, m->bucket_count, m->capacity}, keys, values, count,
      out_values, statuses);
  return vx::from_cuda(cudaGetLastError());
}


extern "C" {

vx_status vx_slab_set_clear(vx_slab_set *s, vx_stream stream) {
  if (s == nullptr) return VX_ERR_INVALID_VALUE;
  const uint64_t words = (static_cast<uint64_t>(s->bucket_count) + s->capacity) * 16u;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  vx::prof::Scope scope("slab_init", st);
  slab_init_kernel<<<grid_for(words), kBlock, 0, st>>>(view_of(s), words);
  return vx::from_cuda(cudaGetLastError());
}



vx_status vx_slab_set_create(uint32_t bucket_count, uint32_t slab_capacity,
                             vx_slab_set **out) {
  if (out == nullptr || bucket_count == 0) return VX_ERR_INVALID_VALUE;
  auto *s = new (std::nothrow) vx_slab_set;
  if (s == nullptr) return VX_ERR_MEMORY_ALLOCATION;
  s->bucket_count = bucket_count;
  s->capacity = slab_capacity;
  const size_t slabs = static_cast<size_t>(bucket_count) + slab_capacity;
  cudaError_t e = cudaMalloc(&s->slabs, slabs * sizeof(Slab));
  if (e == cudaSuccess) e = cudaMalloc(&s->alloc, sizeof(uint32_t));
  if (e != cudaSuccess) {
    vx_slab_set_destroy(s);
    return vx::from_cuda(e);
  }
  const vx_status st = vx_slab_set_clear(s, nullptr);
  if (st != VX_OK) {
    vx_slab_set_destroy(s);
    return st;
  }
  VX_TRY_CUDA(cudaStreamSynchronize(nullptr));
  *out = s;
  return VX_OK;
}

vx_status vx_slab_set_destroy(vx_slab_set *s) {
  if (s == nullptr) return VX_ERR_INVALID_VALUE;
  cudaFree(s->slabs);
  cudaFree(s->alloc);
  delete s;
  return VX_OK;
}

vx_status vx_slab_set_insert(vx_slab_set *s, const uint64_t *keys,
                             uint32_t count, uint32_t *statuses,
                             vx_stream stream) {
  return slab_launch<SetOp::Insert>(s, keys, count, nullptr, statuses, stream,
                                    "slab_insert");
}

vx_status vx_slab_set_contains(const vx_slab_set *s, const uint64_t *keys,
                               uint32_t count, uint32_t *contains,
                               uint32_t *statuses, vx_stream stream) {
  return slab_launch<SetOp::Contains>(s, keys, count, contains, statuses,
                                      stream, "slab_contains");
}

vx_status vx_slab_set_erase(vx_slab_set *s, const uint64_t *keys,
                            uint32_t count, uint32_t *statuses,
                            vx_stream stream) {
  return slab_launch<SetOp::Erase>(s, keys, count, nullptr, statuses, stream,
                                   "slab_erase");
}

vx_status vx_slab_map_create(uint32_t bucket_count, uint32_t slab_capacity,
                             vx_slab_map **out) {
  if (out == nullptr || bucket_count == 0) return VX_ERR_INVALID_VALUE;
  auto *m = new (std::nothrow) vx_slab_map;
  if (m == nullptr) return VX_ERR_MEMORY_ALLOCATION;
  m->bucket_count = bucket_count;
  m->capacity = slab_capacity;
  const size_t slabs = static_cast<size_t>(bucket_count) + slab_capacity;
  cudaError_t e = cudaMalloc(&m->slabs, slabs * sizeof(Slab));
  if (e == cudaSuccess) e = cudaMalloc(&m->alloc, sizeof(uint32_t));
  if (e != cudaSuccess) {
    vx_slab_map_destroy(m);
    return vx::from_cuda(e);
  }
  const vx_status st = vx_slab_map_clear(m, nullptr);
  if (st != VX_OK) {
    vx_slab_map_destroy(m);
    return st;
  }
  VX_TRY_CUDA(cudaStreamSynchronize(nullptr));
  *out = m;
  return VX_OK;
}

vx_status vx_slab_map_destroy(vx_slab_map *m) {
  if (m == nullptr) return VX_ERR_INVALID_VALUE;
  cudaFree(m->slabs);
  cudaFree(m->alloc);
  delete m;
  return VX_OK;
}

vx_status vx_slab_map_clear(vx_slab_map *m, vx_stream stream) {
  if (m == nullptr) return VX_ERR_INVALID_VALUE;
  const uint64_t words = (static_cast<uint64_t>(m->bucket_count) + m->capacity) * 16u;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  vx::prof::Scope scope("slab_map_init", st);
  map_init_kernel<<<grid_for(words), kBlock, 0, st>>>(
      SetView{m->slabs, m->alloc, m->bucket_count, m->capacity}, words);
  return vx::from_cuda(cudaGetLastError());
}

vx_status vx_slab_map_insert_or_replace(vx_slab_map *m, const uint32_t *keys,
                                        const uint32_t *values, uint32_t count,
                                        uint32_t *statuses, vx_stream stream) {
  return map_launch<MapOp::InsertOrReplace>(m, keys, values, count, nullptr, statuses, stream,
                                            "slab_map_insert");
}

vx_status vx_slab_map_find(const vx_slab_map *m, const uint32_t *keys, uint32_t count,
                           uint32_t *values, uint32_t *statuses, vx_stream stream) {
  return map_launch<MapOp::Find>(m, keys, nullptr, count, values, statuses, stream,
                                 "slab_map_find");
}

vx_status vx_slab_map_erase_all(vx_slab_map *m, const uint32_t *keys, uint32_t count,
                                uint32_t *statuses, vx_stream stream) {
  return map_launch<MapOp::EraseAll>(m, keys, nullptr, count, nullptr, statuses, stream,
                                     "slab_map_erase");
}

size_t vx_slab_map_bytes(const vx_slab_map *m) {
  return m ? (static_cast<size_t>(m->bucket_count) + m->capacity) * sizeof(Slab) : 0;
}

vx_status vx_slab_set_device_view(const vx_slab_set *s, vx_slab_set_view *out) {
  if (s == nullptr || out == nullptr) return VX_ERR_INVALID_VALUE;
  *out = vx_slab_set_view{s->slabs, s->bucket_count, s->capacity};
  return VX_OK;
}

vx_status vx_cuckoo_device_view(const vx_cuckoo *c, vx_cuckoo_view *out) {
  if (c == nullptr || out == nullptr) return VX_ERR_INVALID_VALUE;
  *out = vx_cuckoo_view{c->slots, c->slot_count, 0};
  return VX_OK;
}

size_t vx_slab_set_bytes(const vx_slab_set *s) {
  if (s == nullptr) return 0;
  return (static_cast<size_t>(s->bucket_count) + s->capacity) * sizeof(Slab);
}

vx_status vx_cuckoo_create(uint32_t slot_count, uint32_t max_evictions,
                           vx_cuckoo **out) {
  if (out == nullptr || slot_count == 0 || slot_count > 0xfffffffeu) return VX_ERR_INVALID_VALUE;
  auto *c = new (std::nothrow) vx_cuckoo;
  if (c == nullptr) return VX_ERR_MEMORY_ALLOCATION;
  c->slot_count = std::max<uint32_t>(2u, (slot_count + 1u) & ~1u); // whole two-slot buckets
  c->max_evictions = max_evictions;
  cudaError_t e = cudaMalloc(&c->slots, sizeof(ulonglong2) * slot_count);
  if (e == cudaSuccess) e = cudaMalloc(&c->dropped, sizeof(unsigned long long));
  if (e != cudaSuccess) {
    vx_cuckoo_destroy(c);
    return vx::from_cuda(e);
  }
  const vx_status st = vx_cuckoo_clear(c, nullptr);
  if (st != VX_OK) {
    vx_cuckoo_destroy(c);
    return st;
  }
  VX_TRY_CUDA(cudaStreamSynchronize(nullptr));
  *out = c;
  return VX_OK;
}

vx_status vx_cuckoo_destroy(vx_cuckoo *c) {
  if (c == nullptr) return VX_ERR_INVALID_VALUE;
  cudaFree(c->slots);
  cudaFree(c->dropped);
  delete c;
  return VX_OK;
}

vx_status vx_cuckoo_clear(vx_cuckoo *c, vx_stream stream) {
  if (c == nullptr) return VX_ERR_INVALID_VALUE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  vx::prof::Scope scope("cuckoo_init", st);
  cuckoo_init_kernel<<<grid_for(c->slot_count), kBlock, 0, st>>>(
      c->slots, c->slot_count, c->dropped);
  return vx::from_cuda(cudaGetLastError());
}

vx_status vx_cuckoo_insert(vx_cuckoo *c, const uint64_t *keys,
                           const uint32_t *values, uint32_t count,
                           uint32_t *statuses, vx_stream stream) {
  if (c == nullptr || (keys == nullptr && count != 0)) return VX_ERR_INVALID_VALUE;
  if (count == 0) return VX_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  vx::prof::Scope scope("cuckoo_insert", st);
  cuckoo_insert_kernel<<<vx::ceil_div(count, kBlock), kBlock, 0, st>>>(
      c->slots, c->slot_count, c->max_evictions, c->dropped, keys, values,
      count, statuses);
  return vx::from_cuda(cudaGetLastError());
}

vx_status vx_cuckoo_find(const vx_cuckoo *c, const uint64_t *keys,
                         uint32_t count, uint32_t *values, vx_stream stream) {
  if (c == nullptr || ((keys == nullptr || values == nullptr) && count != 0))
    return VX_ERR_INVALID_VALUE;
  if (count == 0) return VX_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  vx::prof::Scope scope("cuckoo_find", st);
  cuckoo_find_kernel<<<vx::ceil_div(count, kBlock), kBlock, 0, st>>>(
      c->slots, c->slot_count, keys, count, values);
  return vx::from_cuda(cudaGetLastError());
}

size_t vx_cuckoo_bytes(const vx_cuckoo *c) {
  return c == nullptr ? 0 : sizeof(ulonglong2) * static_cast<size_t>(c->slot_count);
}

vx_status vx_cuckoo_dropped(const vx_cuckoo *c, uint64_t *host_count,
                            vx_stream stream) {
  if (c == nullptr || host_count == nullptr) return VX_ERR_INVALID_VALUE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned long long v = 0;
  VX_TRY_CUDA(cudaMemcpyAsync(&v, c->dropped, sizeof(v), cudaMemcpyDeviceToHost, st));
  VX_TRY_CUDA(cudaStreamSynchronize(st));
  *host_count = v;
  return VX_OK;
}

} // extern "C"
