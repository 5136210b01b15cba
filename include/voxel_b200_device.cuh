/* voxel_b200_device.cuh - device-side lookups for user kernels (nvcc only).
 *
 * The reference's read paths are __device__ functions that user kernels call
 * directly: svt::hash_dag_gpu::get_voxel (svt/hash_dag_gpu/query.cuh:12-39),
 * svt::cuda::get_voxel (svt/cuda/query.cuh:11-35), the warp-cooperative
 * DeviceSlabHashSetU32::contains (cuda/hash_table/slab_hash/set/
 * device.cuh:148-234) and cuckoo_find (cuda/cuckoo_hash.cuh:101-120).  This
 * header gives the same reads over this library's structures: get a view on
 * the host (vx_dag_device_view, vx_svo_device_view, vx_slab_set_device_view,
 * vx_cuckoo_device_view in voxel_b200.h), pass it to a kernel by value and
 * call the functions below.  The library's own query kernels use these same
 * functions.  A view stays valid while its structure lives; concurrent edits
 * of the structure race with reads, as in the reference.
 */
#ifndef VOXEL_B200_DEVICE_CUH
#define VOXEL_B200_DEVICE_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "voxel_b200.h"

#define VX_SVO_CHILD_BIT (1u << 30)  /* child_data: a child node / leaf exists */
#define VX_SVO_FILLED_BIT (1u << 31) /* child_data: uniform region is filled */
#define VX_SVO_INDEX_MASK ((1u << 30) - 1u)

/* ---------------------------------------------------------------- hashing */

/* splitmix64 finaliser (Steele, Lea & Flood 2014): the tables' hash. */
__host__ __device__ __forceinline__ uint64_t vx_mix64(uint64_t x) {
  x ^= x >> 30;
  x *= 0xbf58476d1ce4e5b9ull;
  x ^= x >> 27;
  x *= 0x94d049bb133111ebull;
  x ^= x >> 31;
  return x;
}

/* A 64-bit hash mapped onto [0, n) by a multiply-high. */
__device__ __forceinline__ uint32_t vx_reduce_hash(uint64_t h, uint32_t n) {
  return (uint32_t)__umul64hi(h, (uint64_t)n);
}

/* Bucket of key under choice c (0 or 1) in a cuckoo table of `buckets`
 * buckets of two 16-byte slots (one 32-byte sector each). */
__device__ __forceinline__ uint32_t vx_cuckoo_bucket(uint64_t key, uint32_t c, uint32_t buckets) {
  const uint64_t salt = c == 0 ? 0x9e3779b97f4a7c15ull : 0xc2b2ae3d27d4eb4full;
  return vx_reduce_hash(vx_mix64(key ^ salt), buckets);
}

__device__ __forceinline__ uint64_t vx_ld_relaxed_u64(const uint64_t *p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

/* ------------------------------------------------------------- Hash DAG -- */

/* Child c (x | y << 1 | z << 2) of the inner item at `item`:
 * [child_mask | fill_mask << 8, child refs of child_mask in order].
 * Returns a ref (0 empty, 1 full, else item / leaf slot + 2). */
__device__ __forceinline__ uint32_t vx_dag_item_child(const uint32_t *item, uint32_t c) {
  const uint32_t header = item[0];
  const uint32_t cm = header & 0xffu, fm = (header >> 8) & 0xffu;
  const uint32_t bit = 1u << c;
  if (cm & bit) return item[1 + __popc(cm & (bit - 1u))];
  return (fm & bit) ? 1u : 0u;
}

/* 1 if voxel (x, y, z) is filled, 0 if empty or outside the world. */
__device__ __forceinline__ uint8_t vx_dag_get_voxel(const vx_dag_view &v, uint32_t x,
                                                    uint32_t y, uint32_t z) {
  const uint32_t side_exp = v.depth + 2;
  if ((x >> side_exp) | (y >> side_exp) | (z >> side_exp)) return 0;
  uint32_t ref = *v.root;
  for (uint32_t l = 0; l < v.depth && ref >= 2u; ++l) {
    const uint32_t s = side_exp - 1 - l;
    const uint32_t c = ((x >> s) & 1u) | (((y >> s) & 1u) << 1) | (((z >> s) & 1u) << 2);
    ref = vx_dag_item_child(v.pool[l] + (ref - 2u), c);
  }
  if (ref <= 1u) return (uint8_t)ref;
  const uint32_t bit = (x & 3u) + 4u * (y & 3u) + 16u * (z & 3u);
  return (uint8_t)((v.leaves[ref - 2u] >> bit) & 1ull);
}

/* Occupancy mask of the 4^3 leaf at leaf coordinates (lx, ly, lz) (voxel
 * coordinates / 4; bit = x + 4y + 16z); 0 outside the world. */
__device__ __forceinline__ uint64_t vx_dag_get_leaf(const vx_dag_view &v, uint32_t lx,
                                                    uint32_t ly, uint32_t lz) {
  if ((lx >> v.depth) | (ly >> v.depth) | (lz >> v.depth)) return 0;
  uint32_t ref = *v.root;
  for (uint32_t l = 0; l < v.depth && ref >= 2u; ++l) {
    const uint32_t s = v.depth - 1 - l;
    const uint32_t c = ((lx >> s) & 1u) | (((ly >> s) & 1u) << 1) | (((lz >> s) & 1u) << 2);
    ref = vx_dag_item_child(v.pool[l] + (ref - 2u), c);
  }
  if (ref <= 1u) return ref ? ~0ull : 0ull;
  return v.leaves[ref - 2u];
}

/* First solid voxel along a ray (vx_dag_raycast in voxel_b200.h).  The ray is
 * clipped to the world box; from the voxel it enters, each step walks the DAG
 * to the largest uniform cell (or leaf voxel) holding the current voxel: a
 * full cell or a set leaf bit is the hit, otherwise the ray leaves the cell
 * through the side with the smallest exit parameter (ties: x, then y, then
 * z), the next voxel across that side is the next position, and the other
 * coordinates are floor(origin + t dir) kept inside the cell and never moving
 * against the ray.  Each step advances one coordinate, so at most
 * 3 * world steps run. */
__device__ inline vx_ray_hit vx_dag_raycast(const vx_dag_view &v, const vx_ray &ray) {
  vx_ray_hit miss;
  miss.voxel[0] = miss.voxel[1] = miss.voxel[2] = ~0u;
  miss.face = VX_FACE_NO_HIT;
  miss.t = -1.0f;
  const uint32_t D = v.depth;
  const int32_t W = 4 << D;
  const float Wf = (float)W;
  const float o[3] = {ray.origin[0], ray.origin[1], ray.origin[2]};
  const float d[3] = {ray.dir[0], ray.dir[1], ray.dir[2]};
  float t0 = 0.0f, t1 = __int_as_float(0x7f800000);
  int entry = -1;
  for (int a = 0; a < 3; ++a) {
    if (d[a] == 0.0f) {
      if (!(o[a] >= 0.0f && o[a] < Wf)) return miss;
      continue;
    }
    const float ta = __fdiv_rn(__fsub_rn(0.0f, o[a]), d[a]);
    const float tb = __fdiv_rn(__fsub_rn(Wf, o[a]), d[a]);
    const float tn = ta < tb ? ta : tb, tf = ta < tb ? tb : ta;
    if (tn > t0) {
      t0 = tn;
      entry = a;
    }
    if (tf < t1) t1 = tf;
  }
  if (!(t0 < t1) || !(t0 <= ray.t_max)) return miss;
  int32_t vox[3];
  for (int a = 0; a < 3; ++a) {
    if (a == entry) {
      vox[a] = d[a] > 0.0f ? 0 : W - 1;
    } else {
      float f = floorf(__fadd_rn(o[a], __fmul_rn(t0, d[a])));
      f = f < 0.0f ? 0.0f : (f > Wf - 1.0f ? Wf - 1.0f : f);
      vox[a] = (int32_t)f;
    }
  }
  uint32_t face = entry < 0 ? 0u : (d[entry] > 0.0f ? 2u * entry + 1u : 2u * entry);
  float t = t0;
  /* path[k] = ref of the level-k cell holding the current voxel, valid for
   * k <= l; a step keeps the cells that still hold the next voxel, so the
   * walk resumes below the deepest common cell instead of at the root. */
  uint32_t path[15]; /* depth <= 14 */
  path[0] = *v.root;
  uint32_t l = 0;
  const uint32_t limit = 3u * (uint32_t)W + 8u;
  for (uint32_t step = 0; step < limit; ++step) {
    uint32_t ref = path[l];
    for (; l < D && ref >= 2u; ++l) {
      const uint32_t sh = D + 1 - l;
      const uint32_t c = (((uint32_t)vox[0] >> sh) & 1u) | ((((uint32_t)vox[1] >> sh) & 1u) << 1) |
                         ((((uint32_t)vox[2] >> sh) & 1u) << 2);
      ref = vx_dag_item_child(v.pool[l] + (ref - 2u), c);
      path[l + 1] = ref;
    }
    int32_t side;
    if (ref == 1u) {
      side = 0;
    } else if (ref >= 2u) {
      const uint32_t bit = (vox[0] & 3) + 4u * (vox[1] & 3) + 16u * (vox[2] & 3);
      side = ((v.leaves[ref - 2u] >> bit) & 1ull) ? 0 : 1;
    } else {
      side = 4 << (D - l);
    }
    if (side == 0) {
      vx_ray_hit h;
      h.voxel[0] = (uint32_t)vox[0];
      h.voxel[1] = (uint32_t)vox[1];
      h.voxel[2] = (uint32_t)vox[2];
      h.face = face;
      h.t = t;
      return h;
    }
    int32_t cmin[3];
    for (int a = 0; a < 3; ++a) cmin[a] = vox[a] & ~(side - 1);
    float tx = 0.0f;
    int ax = -1;
    for (int a = 0; a < 3; ++a) {
      if (d[a] == 0.0f) continue;
      const float b = (float)(d[a] > 0.0f ? cmin[a] + side : cmin[a]);
      const float ta = __fdiv_rn(__fsub_rn(b, o[a]), d[a]);
      if (ax < 0 || ta < tx) {
        tx = ta;
        ax = a;
      }
    }
    if (ax < 0 || !(tx <= ray.t_max)) return miss;
    const int32_t nv = d[ax] > 0.0f ? cmin[ax] + side : cmin[ax] - 1;
    if (nv < 0 || nv >= W) return miss;
    uint32_t moved = (uint32_t)(vox[ax] ^ nv);
    for (int b = 0; b < 3; ++b) {
      if (b == ax || d[b] == 0.0f) continue;
      const float lo = (float)(d[b] > 0.0f ? vox[b] : cmin[b]);
      const float hi = (float)(d[b] > 0.0f ? cmin[b] + side - 1 : vox[b]);
      float f = floorf(__fadd_rn(o[b], __fmul_rn(tx, d[b])));
      f = f < lo ? lo : (f > hi ? hi : f);
      moved |= (uint32_t)(vox[b] ^ (int32_t)f);
      vox[b] = (int32_t)f;
    }
    vox[ax] = nv;
    /* The level-k cell (side 2^(D+2-k)) still holds the voxel iff no
     * coordinate bit at or above D + 2 - k changed. */
    const uint32_t keep = D + 1u - (31u - (uint32_t)__clz((int)moved));
    if (keep < l) l = keep;
    t = tx;
    face = d[ax] > 0.0f ? 2u * ax + 1u : 2u * ax;
  }
  return miss;
}

/* ------------------------------------------------------------------ SVO -- */

/* Value of a child word without a child: material (or 1 without materials)
 * when filled, 0 when empty. */
__device__ __forceinline__ uint32_t vx_svo_word_value(uint32_t w, bool materials) {
  return (w & VX_SVO_FILLED_BIT) ? (materials ? (w & 0xffu) : 1u) : 0u;
}

/* Material of voxel (x, y, z) (1 for filled without materials), 0 if empty
 * or outside the world. */
__device__ __forceinline__ uint8_t vx_svo_get_voxel(const vx_svo_view &v, uint32_t x,
                                                    uint32_t y, uint32_t z) {
  const uint32_t side_exp = v.depth + 2;
  const bool mats = v.materials != 0;
  if ((x >> side_exp) | (y >> side_exp) | (z >> side_exp)) return 0;
  uint32_t w = VX_SVO_CHILD_BIT; /* root node 0 */
  for (uint32_t l = 0; l < v.depth && (w & VX_SVO_CHILD_BIT); ++l) {
    const uint32_t s = side_exp - 1 - l;
    const uint32_t c = ((x >> s) & 1u) | (((y >> s) & 1u) << 1) | (((z >> s) & 1u) << 2);
    w = v.nodes[(size_t)(w & VX_SVO_INDEX_MASK) * 8u + c];
  }
  if (!(w & VX_SVO_CHILD_BIT)) return (uint8_t)vx_svo_word_value(w, mats);
  const uint32_t li = w & VX_SVO_INDEX_MASK;
  const uint32_t bit = (x & 3u) + 4u * (y & 3u) + 16u * (z & 3u);
  if (mats) return v.materials_data[(size_t)li * 64u + bit];
  return (uint8_t)((v.leaves[li] >> bit) & 1ull);
}

/* ---------------------------------------------------------- hash tables -- */

/* Cuckoo find: true and *value if key is present.  Both candidate buckets
 * (two 32-byte sectors) are loaded at once. */
__device__ __forceinline__ bool vx_cuckoo_find(const vx_cuckoo_view &v, uint64_t key,
                                               uint32_t *value) {
  if (key == VX_HASH_EMPTY_KEY || key == VX_HASH_DELETED_KEY) return false;
  const ulonglong2 *slots = (const ulonglong2 *)v.slots;
  const uint32_t nb = v.slot_count / 2u;
  const ulonglong2 *b[2] = {slots + 2ull * vx_cuckoo_bucket(key, 0, nb),
                            slots + 2ull * vx_cuckoo_bucket(key, 1, nb)};
  ulonglong2 e[4];
#pragma unroll
  for (uint32_t i = 0; i < 4; ++i)
    asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];"
                 : "=l"(e[i].x), "=l"(e[i].y)
                 : "l"(b[i >> 1] + (i & 1u))
                 : "memory");
#pragma unroll
  for (uint32_t i = 0; i < 4; ++i)
    if (e[i].x == key) {
      *value = (uint32_t)e[i].y;
      return true;
    }
  return false;
}

/* Slab set membership, warp-cooperative: all 32 lanes of a warp call it
 * together (the reference's contract), each with its key and whether it is
 * active; each half-warp walks one key's chain at a time, a 128-byte slab
 * (15 keys + link) per coalesced read.  Returns true for an active lane whose
 * key is present. */
__device__ __forceinline__ bool vx_slab_set_contains_warp(const vx_slab_set_view &v,
                                                          uint64_t key, bool active) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t sub = lane & 15u;
  const uint32_t half = lane >> 4;
  const uint32_t hmask = half ? 0xffff0000u : 0x0000ffffu;
  const uint64_t *slabs = (const uint64_t *)v.slabs;
  if (key == VX_HASH_EMPTY_KEY || key == VX_HASH_DELETED_KEY) active = false;
  bool found = false;
  uint32_t queue = __ballot_sync(0xffffffffu, active) & hmask;
  while (queue) {
    const uint32_t src = __ffs(queue) - 1u;
    const uint64_t k = __shfl_sync(hmask, key, src);
    uint64_t slab = vx_reduce_hash(vx_mix64(k), v.bucket_count);
    bool hit = false;
    /* a chain is at most the pool long: the loop ends even on a damaged table */
    for (uint64_t step = 0; step <= (uint64_t)v.capacity; ++step) {
      const uint64_t w = vx_ld_relaxed_u64(slabs + slab * 16u + sub);
      hit = (__ballot_sync(hmask, sub < 15u && w == k) & hmask) != 0;
      if (hit) break;
      const uint64_t link = __shfl_sync(hmask, w, (half << 4) + 15u);
      if (link == ~0ull) break;
      slab = link;
    }
    if (lane == src) {
      found = hit;
      active = false;
    }
    queue = __ballot_sync(hmask, active) & hmask;
  }
  return found;
}

#endif /* VOXEL_B200_DEVICE_CUH */
