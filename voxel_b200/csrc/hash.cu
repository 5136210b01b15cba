// u64-keyed hash tables for sm_100a.
//
// Slab hash set: the u64 widening of the reference's BasicSlabHashSetU32
// (cuda/hash_table/slab_hash/set/host.cuh:13-121, device.cuh:31-315).  A slab
// is one 128-byte line: 15 u64 key slots and a u64 link to the next slab of
// the bucket's chain.  Sixteen lanes read a slab with one coalesced request,
// so each warp works on two keys at once (one per half-warp), where the
// reference's u32 slab needs the whole warp per key.  Inserts CAS an empty or
// deleted slot; full chains grow from a pool of overflow slabs taken with a
// bump counter.  Statuses are the reference's kSlabHashStatus* values.  Every
// retry loop is bounded (the reference's kSlabHashMaxContentionRetries).
//
// Slab map: u32 -> u32, the reference's SlabHashMapU32 (below).
//
// Cuckoo map: the u64-keyed widening of cuckoo_insert / cuckoo_find
// (cuda/cuckoo_hash.cuh:54-120).  Four hash functions address one array of
// 16-byte slots {key, value | hash id << 32}; an eviction moves a whole slot
// with one 128-bit atomic exchange (atom.exch.b128, sm_90+), so key and value
// never separate.  Eviction chains are bounded by max_evictions (the
// reference's insertion_attempts); a chain that runs out drops the key in
// hand, reports VX_HASH_OVERFLOW and counts it.
#include "common.cuh"
#include "profile.cuh"
#include "voxel_b200_device.cuh"

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

// One key per half-warp at a time.  All 32 lanes call this; each half-warp
// drains its own queue of active lanes.
template <SetOp Op>
__global__ void __launch_bounds__(kBlock)
    slab_set_kernel(SetView t, const uint64_t *__restrict__ keys,
                    uint32_t count, uint32_t *contains, uint32_t *statuses) {
  const uint32_t lane = lane_id();
  const uint32_t sub = lane & 15u;
  const uint32_t half = lane >> 4;
  const uint32_t hmask = half ? 0xffff0000u : 0x0000ffffu;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  // Every lane of a warp iterates the same number of rounds.
  const uint64_t warp_first = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) - lane;
  for (uint64_t base = warp_first; base < count; base += stride) {
    const uint64_t idx = base + lane;
    bool active = idx < count;
    uint64_t key = active ? keys[idx] : 0;
    uint32_t status = VX_HASH_NOT_FOUND, found = 0;
    if (active && (key == kEmpty || key == kDeleted)) {
      status = VX_HASH_INVALID_KEY;
      active = false;
    }
    uint32_t queue = __ballot_sync(hmask, active) & hmask;
    while (queue) {
      const uint32_t src = __ffs(queue) - 1u;
      const uint64_t k = __shfl_sync(hmask, key, src);
      Slab *slab = &t.slabs[reduce(mix64(k), t.bucket_count)];
      uint32_t result = VX_HASH_OVERFLOW;
      const uint64_t max_steps =
          Op == SetOp::Contains
              ? t.capacity + 1ull
              : (t.capacity + 1ull) * static_cast<uint64_t>(kMaxContentionRetries);
      for (uint64_t step = 0; step < max_steps; ++step) {
        const uint64_t w = ld_relaxed_u64(&slab->w[sub]);
        const bool key_slot = sub < kSlotsPerSlab;
        const uint32_t hit = __ballot_sync(hmask, key_slot && w == k) & hmask;
        if (hit) {
          if (Op == SetOp::Erase) {
            const uint32_t dst = __ffs(hit) - 1u;
            unsigned long long old = 0;
            if (lane == dst)
              old = atomicCAS(reinterpret_cast<unsigned long long *>(&slab->w[sub]),
                              k, kDeleted);
            old = __shfl_sync(hmask, old, dst);
            if (old != k) continue; // lost a race: re-read this slab
            result = VX_HASH_ERASED;
          } else {
            result = Op == SetOp::Insert ? VX_HASH_ALREADY_PRESENT : VX_HASH_FOUND;
          }
          break;
        }
        if (Op == SetOp::Insert) {
          const uint32_t free_mask =
              __ballot_sync(hmask, key_slot && (w == kEmpty || w == kDeleted)) & hmask;
          if (free_mask) {
            const uint32_t dst = __ffs(free_mask) - 1u;
            const uint64_t expect = __shfl_sync(hmask, w, dst);
            unsigned long long old = 0;
            if (lane == dst)
              old = atomicCAS(reinterpret_cast<unsigned long long *>(&slab->w[sub]),
                              expect, k);
            old = __shfl_sync(hmask, old, dst);
            if (old == expect) {
              result = VX_HASH_INSERTED;
              break;
            }
            continue; // slot taken meanwhile: re-read this slab
          }
        }
        const uint64_t link = __shfl_sync(hmask, w, (half << 4) + 15u);
        if (link != kNullLink) {
          slab = &t.slabs[link];
          continue;
        }
        if (Op != SetOp::Insert) {
          result = VX_HASH_NOT_FOUND;
          break;
        }
        // Grow the chain: take a pool slab, initialise it, link it with CAS.
        uint32_t ord = 0;
        if (sub == 0) ord = atomicAdd(t.alloc, 1u);
        ord = __shfl_sync(hmask, ord, half << 4);
        if (ord >= t.capacity) {
          // Pool exhausted; another half-warp may have linked a slab since.
          uint64_t again = 0;
          if (sub == 15u) again = ld_relaxed_u64(&slab->w[15]);
          again = __shfl_sync(hmask, again, (half << 4) + 15u);
          if (again != kNullLink) {
            slab = &t.slabs[again];
            continue;
          }
          result = VX_HASH_OVERFLOW;
          break;
        }
        Slab *fresh = &t.slabs[t.bucket_count + ord];
        fresh->w[sub] = sub == 15u ? kNullLink : kEmpty;
        __threadfence();
        __syncwarp(hmask);
        unsigned long long observed = 0;
        if (sub == 15u)
          observed = atomicCAS(reinterpret_cast<unsigned long long *>(&slab->w[15]),
                               kNullLink, t.bucket_count + ord);
        observed = __shfl_sync(hmask, observed, (half << 4) + 15u);
        // Either our slab was linked or another warp's was; follow the link.
        // (A pool slab that lost the race stays unused.)
        slab = &t.slabs[observed == kNullLink ? t.bucket_count + ord : observed];
      }
      if (lane == src) {
        status = result;
        found = (result == VX_HASH_FOUND) ? 1u : 0u;
        active = false;
      }
      queue = __ballot_sync(hmask, active) & hmask;
    }
    if (idx < count) {
      if (statuses) statuses[idx] = status;
      if (Op == SetOp::Contains && contains) contains[idx] = found;
    }
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

constexpr uint32_t kCuckooHashes = 4;

__device__ __forceinline__ uint32_t cuckoo_slot(uint64_t key, uint32_t hid,
                                                uint32_t n) {
  return vx_cuckoo_slot(key, hid, n);
}

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

__device__ __forceinline__ bool cuckoo_lookup(const ulonglong2 *slots,
                                              uint32_t n, uint64_t key,
                                              uint32_t &value, uint32_t &where) {
#pragma unroll
  for (uint32_t h = 0; h < kCuckooHashes; ++h) {
    const uint32_t s = cuckoo_slot(key, h, n);
    const ulonglong2 v = ld_slot(slots + s);
    if (v.x == key) {
      value = static_cast<uint32_t>(v.y);
      where = s;
      return true;
    }
  }
  return false;
}

// Replace the value stored for key, keeping the slot's hash id (bits 32..63
// of .y, which the next eviction of this entry continues from).  The swap is
// a 128-bit CAS on {key, old word}, so an entry that a concurrent eviction
// moved is looked up again rather than overwritten in its new occupant's
// slot.  Returns false when the key is not in the table (duplicate keys
// inside one insert batch are not supported, as in the reference, so a key
// held in flight by another thread's eviction chain is not expected).
__device__ __forceinline__ bool cuckoo_replace(ulonglong2 *slots, uint32_t n,
                                               uint64_t key, uint32_t value) {
  uint32_t old_value, where;
  for (uint32_t attempt = 0; attempt < 64; ++attempt) {
    if (!cuckoo_lookup(slots, n, key, old_value, where)) return false;
    const ulonglong2 cur = ld_slot(slots + where);
    if (cur.x != key) continue;
    const ulonglong2 want =
        make_ulonglong2(key, (cur.y & 0xffffffff00000000ull) | value);
    const ulonglong2 seen = cas128(slots + where, cur, want);
    if (seen.x == cur.x && seen.y == cur.y) return true;
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
  const uint64_t key = keys[i];
  const uint32_t value = values ? values[i] : static_cast<uint32_t>(i);
  uint32_t status;
  if (key == kEmpty || key == kDeleted) {
    status = VX_HASH_INVALID_KEY;
  } else if (cuckoo_replace(slots, n, key, value)) {
    status = VX_HASH_REPLACED;
  } else {
    ulonglong2 cur = make_ulonglong2(key, value);
    uint32_t hid = 0;
    status = VX_HASH_OVERFLOW;
    for (uint32_t a = 0; a <= max_evictions; ++a) {
      cur.y = (cur.y & 0xffffffffull) | (static_cast<uint64_t>(hid) << 32);
      const ulonglong2 prev = exch128(slots + cuckoo_slot(cur.x, hid, n), cur);
      if (prev.x == kEmpty) {
        status = VX_HASH_INSERTED;
        break;
      }
      if (prev.x == cur.x) { // same key displaced: keep the newer value
        status = VX_HASH_INSERTED;
        break;
      }
      cur = prev;
      hid = (static_cast<uint32_t>(prev.y >> 32) + 1u) % kCuckooHashes;
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
  if (out == nullptr || slot_count == 0) return VX_ERR_INVALID_VALUE;
  auto *c = new (std::nothrow) vx_cuckoo;
  if (c == nullptr) return VX_ERR_MEMORY_ALLOCATION;
  c->slot_count = slot_count;
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
