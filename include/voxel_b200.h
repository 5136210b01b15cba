/*
 * voxel_b200.h - C ABI of the B200-native voxel-editing library.
 *
 * The reference (yamaatsu1112/voxel, algorithm/lib/include/algo) is a
 * header-only C++/CUDA template library whose entry points all have the shape
 *
 *     cudaError_t f(View, const T* in, uint32_t count,
 *                   void* workspace, size_t workspace_size, cudaStream_t)
 *     size_t      f_workspace_size(uint32_t count)
 *
 * This header exposes the same contract as plain C: device pointers, counts,
 * a caller-owned workspace whose size depends only on the count, a stream, and
 * a status code.  Status values 0..999 are cudaError_t values (0 = success,
 * 1 = cudaErrorInvalidValue, 2 = cudaErrorMemoryAllocation, ...); values from
 * 1000 up are this library's own.  No C++ exception crosses this boundary.
 * Every pointer is a device pointer unless its name starts with host_.
 * Every call is stream-ordered and asynchronous unless documented otherwise.
 *
 * Each declaration names the reference interface it replaces (file:line,
 * relative to algorithm/lib/include/algo/).
 */
#ifndef VOXEL_B200_H
#define VOXEL_B200_H

#include <stddef.h>
#include <stdint.h>

#include "vx_workload.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t vx_status;
typedef void *vx_stream; /* a cudaStream_t; NULL = legacy default stream */

#define VX_OK 0
#define VX_ERR_INVALID_VALUE 1      /* == cudaErrorInvalidValue */
#define VX_ERR_MEMORY_ALLOCATION 2  /* == cudaErrorMemoryAllocation */
#define VX_ERR_TIMEOUT 1001         /* a bounded device wait gave up */
#define VX_ERR_CAPACITY 1002        /* a node pool / table / arena is full */
#define VX_ERR_NO_DEVICE 1003       /* no CUDA device is visible */
#define VX_ERR_IO 1004         /* a file could not be read or written */

/* Library version and a human-readable name for a status code. */
uint32_t vx_version(void);
const char *vx_status_string(vx_status status);

/* Scan and sort calls are fully asynchronous; a bounded device wait that gave
 * up is recorded in their workspace.  This synchronises the stream and returns
 * VX_OK or VX_ERR_TIMEOUT for the last call that used the workspace. */
vx_status vx_workspace_status(const void *workspace, vx_stream stream);

/* Built-in per-kernel timing (off by default): when enabled, every kernel
 * launch of the library is bracketed by a CUDA event pair on its stream;
 * vx_profile_query sums the elapsed milliseconds and launches per kernel name
 * since the last reset (it synchronises on those events). */
void vx_profile_enable(uint32_t on);
void vx_profile_reset(void);
/* Number of kernels the library has launched in this process. */
uint64_t vx_profile_launches(void);
vx_status vx_profile_query(const char *name, double *host_total_ms,
                           uint64_t *host_launches);

/* Seeded edit primitives of a benchmark mix, into host memory (the generator
 * defined in vx_workload.h: PCG32 stream `stream` seeded with `seed`). */
vx_status vx_generate_primitives(const vx_edit_mix *mix, uint64_t seed,
                                 uint64_t stream, uint64_t count,
                                 vx_primitive *host_out);

/* ---------------------------------------------------------------- tuning --
 * Launch-shape knobs (partition items per thread and count publishing of the
 * radix sort, the long-list threshold and grid of the edit pipelines).  Every
 * allowed value gives the same results; they only trade speed, and
 * voxel_b200/autotune.py picks them per device by timing.  Settings are
 * process-wide and apply to launches made after the call.  The reference
 * fixes these as template policies (cuda/sort/radix/onesweep/host.cuh,
 * svt/hash_dag_gpu/config.cuh); there is no runtime counterpart. */
uint32_t vx_tuning_count(void);
const char *vx_tuning_name(uint32_t index);  /* NULL past the last knob */
vx_status vx_tuning_options(const char *name, int64_t *host_values,
                            uint32_t capacity, uint32_t *host_count);
vx_status vx_tuning_get(const char *name, int64_t *host_value);
/* VX_ERR_INVALID_VALUE for an unknown knob or a value it does not allow. */
vx_status vx_tuning_set(const char *name, int64_t value);
vx_status vx_tuning_reset(void);             /* back to the defaults */

/* ------------------------------------------------------------------ scan --
 * In-place prefix sums over uint32 / uint64 with modular (wrapping)
 * arithmetic.  Replaces algo::cuda::scan::{exclusive,inclusive}_sum<T> and
 * required_workspace_size<T> (cuda/scan/scan.cuh:107-161, defaults at
 * cuda/scan/scan.cuh:18-19) with a single-pass decoupled look-back scan.
 * count == 0 is a no-op; data == NULL with count > 0, or a NULL/short
 * workspace, returns VX_ERR_INVALID_VALUE (docs/cuda/scan.md).
 * A look-back wait that exceeds its iteration bound returns VX_ERR_TIMEOUT. */
size_t vx_scan_workspace_size(uint32_t count);
vx_status vx_scan_exclusive_sum_u32(uint32_t *data, uint32_t count,
                                    void *workspace, size_t workspace_bytes,
                                    vx_stream stream);
vx_status vx_scan_inclusive_sum_u32(uint32_t *data, uint32_t count,
                                    void *workspace, size_t workspace_bytes,
                                    vx_stream stream);
vx_status vx_scan_exclusive_sum_u64(uint64_t *data, uint32_t count,
                                    void *workspace, size_t workspace_bytes,
                                    vx_stream stream);
/* In-place exclusive sum of u32 that allocates nothing and takes no
 * workspace, for callers that cannot allocate device memory where they need
 * the scan (a fixed device-memory budget, or code that must not call
 * cudaMalloc / cudaFree because they synchronise the device).  No counterpart
 * in the reference: its scans always take a caller workspace.  The scratch is
 * a 256 KiB array inside this library on each device, so count must be at
 * most 2^28 (larger counts return VX_ERR_CAPACITY and touch nothing); calls
 * that can overlap on the GPU share that array and race; the first call in a
 * CUDA context (again after a device reset) looks up the array's address and
 * should precede any stream capture.  The call is asynchronous: a look-back
 * wait that gives up cannot be reported by its return value, so read
 * vx_scan_noalloc_status afterwards where that matters. */
vx_status vx_scan_exclusive_sum_u32_noalloc(uint32_t *data, uint32_t count,
                                            vx_stream stream);
/* Synchronises the stream and returns the device status that the most recent
 * vx_scan_exclusive_sum_u32_noalloc on the current device left in the shared
 * scratch: VX_OK, or VX_ERR_TIMEOUT when a bounded look-back wait gave up and
 * that call's sums are invalid.  Allocates nothing.  No counterpart in the
 * reference (its scans report through a caller workspace).  With overlapping
 * calls the word belongs to whichever call wrote it last. */
vx_status vx_scan_noalloc_status(vx_stream stream);

/* ------------------------------------------------------------------ sort --
 * Stable LSD radix sort ("onesweep": one all-pass digit histogram, then one
 * partition kernel per digit with decoupled look-back), in place.  The digit
 * is 8 bits wide unless the "sort.radix_bits" tuning knob narrows it (6 or
 * 7 bits; keys that would then take more than 8 passes keep 8-bit digits).
 * Only the low key_bits bits of each key order the output (key_bits in
 * [1, 32] for u32 keys, [1, 64] for u64 keys), matching the KeyBits contract
 * of algo::cuda::sort::RadixSort (docs/cuda/sort.md "Configuration").
 * Replaces sort::sort_keys / sort::sort_by_key with one value array and
 * required_sort_by_key_workspace_size (cuda/sort/sort.cuh:100-167,
 * cuda/sort/radix/onesweep/host.cuh:135-204).  values may be NULL for a
 * key-only sort.  count <= 1 needs no workspace; count must be < 2^30
 * (the reference's onesweep bound, cuda/sort/radix/onesweep/host.cuh:85-86). */
size_t vx_sort_workspace_size(uint32_t count, uint32_t key_bytes);
vx_status vx_sort_pairs_u32(uint32_t *keys, uint32_t *values, uint32_t count,
                            uint32_t key_bits, void *workspace,
                            size_t workspace_bytes, vx_stream stream);
vx_status vx_sort_pairs_u64(uint64_t *keys, uint32_t *values, uint32_t count,
                            uint32_t key_bits, void *workspace,
                            size_t workspace_bytes, vx_stream stream);

/* Stable LSD radix sort of multi-word unsigned keys, in place: each key is
 * `words` 32-bit words (word 0 least significant; the reference's
 * UIntKey<W>, cuda/sort/uint_key.cuh:15-66, also u32 = 1 word and u64 = 2),
 * ordered by its low key_bits bits (1 <= key_bits <= 32 * words; the KeyBits
 * contract of RadixSort, cuda/sort/radix.cuh:55-67).  perm (optional, count
 * entries) receives, for every output position, the input position of its
 * key, which orders any number of value arrays of any element size through
 * vx_gather (the reference's value_arrays, cuda/sort/value_arrays.cuh).
 * words <= 64; count < 2^30. */
size_t vx_sort_words_workspace_size(uint32_t count, uint32_t words);
vx_status vx_sort_words(uint32_t *keys, uint32_t words, uint32_t count, uint32_t key_bits,
                        uint32_t *perm, void *workspace, size_t workspace_bytes,
                        vx_stream stream);

/* dst[i] = src[index[i]] for count elements of elem_bytes bytes each (device
 * memory, dst and src distinct). */
vx_status vx_gather(void *dst, const void *src, const uint32_t *index, uint32_t count,
                    uint32_t elem_bytes, vx_stream stream);

/* ----------------------------------------------------------- hash tables --
 * Per-key status codes, identical in value to the reference's
 * kSlabHashStatus* (cuda/hash_table/slab_hash/common.cuh:18-25). */
#define VX_HASH_NOT_FOUND 0u
#define VX_HASH_INSERTED 1u
#define VX_HASH_REPLACED 2u
#define VX_HASH_ERASED 3u
#define VX_HASH_OVERFLOW 4u
#define VX_HASH_INVALID_KEY 5u
#define VX_HASH_FOUND 6u
#define VX_HASH_ALREADY_PRESENT 7u

/* Reserved u64 keys (the u64 widening of kSlabHashEmptyKey / DeletedKey). */
#define VX_HASH_EMPTY_KEY 0xFFFFFFFFFFFFFFFFull
#define VX_HASH_DELETED_KEY 0xFFFFFFFFFFFFFFFEull
#define VX_HASH_NOT_FOUND_VALUE 0xFFFFFFFFu

/* Slab hash set of u64 keys: buckets of 128-byte slabs (15 keys + link),
 * chained through a pool of slab_capacity overflow slabs.  The u64 widening
 * of BasicSlabHashSetU32 (cuda/hash_table/slab_hash/set/host.cuh:13-121,
 * device ops cuda/hash_table/slab_hash/set/device.cuh:31-315).  statuses may
 * be NULL.  A full slab pool reports VX_HASH_OVERFLOW for that key. */
typedef struct vx_slab_set vx_slab_set;
vx_status vx_slab_set_create(uint32_t bucket_count, uint32_t slab_capacity,
                             vx_slab_set **out);
vx_status vx_slab_set_destroy(vx_slab_set *set);
vx_status vx_slab_set_clear(vx_slab_set *set, vx_stream stream);
vx_status vx_slab_set_insert(vx_slab_set *set, const uint64_t *keys,
                             uint32_t count, uint32_t *statuses,
                             vx_stream stream);
vx_status vx_slab_set_contains(const vx_slab_set *set, const uint64_t *keys,
                               uint32_t count, uint32_t *contains,
                               uint32_t *statuses, vx_stream stream);
vx_status vx_slab_set_erase(vx_slab_set *set, const uint64_t *keys,
                            uint32_t count, uint32_t *statuses,
                            vx_stream stream);
/* Bytes of device memory the table holds (buckets + overflow pool). */
size_t vx_slab_set_bytes(const vx_slab_set *set);

/* Slab hash map u32 -> u32 (SlabHashMapU32, cuda/hash_table/slab_hash/map/
 * host.cuh, common.cuh:40-94, device.cuh:49-372): 128-byte slabs of 15
 * packed key/value slots and a link.  Keys VX_MAP_EMPTY_KEY /
 * VX_MAP_DELETED_KEY are reserved (VX_HASH_INVALID_KEY).  insert_or_replace
 * takes the first slot of the chain that holds the key, is empty or deleted
 * (VX_HASH_INSERTED / VX_HASH_REPLACED / VX_HASH_OVERFLOW); duplicates of a
 * key in one batch apply in array order within a warp.  find writes the value
 * of the first match or VX_HASH_NOT_FOUND_VALUE (VX_HASH_FOUND /
 * VX_HASH_NOT_FOUND); erase_all deletes every match (VX_HASH_ERASED /
 * VX_HASH_NOT_FOUND).  statuses may be NULL. */
#define VX_MAP_EMPTY_KEY 0xFFFFFFFFu
#define VX_MAP_DELETED_KEY 0xFFFFFFFEu
typedef struct vx_slab_map vx_slab_map;
vx_status vx_slab_map_create(uint32_t bucket_count, uint32_t slab_capacity,
                             vx_slab_map **out);
vx_status vx_slab_map_destroy(vx_slab_map *map);
vx_status vx_slab_map_clear(vx_slab_map *map, vx_stream stream);
vx_status vx_slab_map_insert_or_replace(vx_slab_map *map, const uint32_t *keys,
                                        const uint32_t *values, uint32_t count,
                                        uint32_t *statuses, vx_stream stream);
vx_status vx_slab_map_find(const vx_slab_map *map, const uint32_t *keys,
                           uint32_t count, uint32_t *values, uint32_t *statuses,
                           vx_stream stream);
vx_status vx_slab_map_erase_all(vx_slab_map *map, const uint32_t *keys,
                                uint32_t count, uint32_t *statuses, vx_stream stream);
size_t vx_slab_map_bytes(const vx_slab_map *map);

/* Content-addressed store of fixed-width items (1..9 u32 words): the
 * reference's AccelerationHashSet32<ItemWords> (cuda/hash_table/
 * acceleration_hash/set/host.cuh:15-117, device.cuh:29-321), built on one
 * hash-consing table of the Hash DAG's kind (open-addressing index of
 * {tag, ref} over a word pool).  Items are count x width words; pointers
 * are item index + 1, 0 = null (kAccelerationHashNullPtr).  find: FOUND /
 * NOT_FOUND; insert_unique_unchecked (the caller guarantees no equal item is
 * present or concurrently inserted): INSERTED / OVERFLOW; find_or_insert
 * (hash-consing, safe under concurrent equal inserts): FOUND / INSERTED /
 * OVERFLOW; read copies the words of each pointer (NOT_FOUND and zeros for
 * null or unknown pointers).  statuses may be NULL. */
typedef struct vx_itemset vx_itemset;
vx_status vx_itemset_create(uint32_t width, uint32_t max_items, vx_itemset **out);
vx_status vx_itemset_destroy(vx_itemset *set);
vx_status vx_itemset_clear(vx_itemset *set, vx_stream stream);
vx_status vx_itemset_find(const vx_itemset *set, const uint32_t *items, uint32_t count,
                          uint32_t *ptrs, uint32_t *statuses, vx_stream stream);
vx_status vx_itemset_find_or_insert(vx_itemset *set, const uint32_t *items, uint32_t count,
                                    uint32_t *ptrs, uint32_t *statuses, vx_stream stream);
vx_status vx_itemset_insert_unique_unchecked(vx_itemset *set, const uint32_t *items,
                                             uint32_t count, uint32_t *ptrs,
                                             uint32_t *statuses, vx_stream stream);
vx_status vx_itemset_read(const vx_itemset *set, const uint32_t *ptrs, uint32_t count,
                          uint32_t *items, uint32_t *statuses, vx_stream stream);
/* Items stored (host read, synchronises). */
vx_status vx_itemset_count(const vx_itemset *set, uint64_t *host_count, vx_stream stream);

/* Cuckoo hash map u64 -> u32 with 4 hash functions over one slot array and a
 * bounded eviction chain (max_evictions).  The u64-keyed, inline-key
 * widening of cuckoo_insert / cuckoo_find / initialize_cuckoo_table
 * (cuda/cuckoo_hash.cuh:54-120), which store an index into triple-u32 key
 * arrays instead.  insert reports VX_HASH_INSERTED, VX_HASH_REPLACED (key
 * already present: value overwritten) or VX_HASH_OVERFLOW (eviction chain
 * exhausted: the key that was in hand at the end is dropped and reported).
 * find writes the value or VX_HASH_NOT_FOUND_VALUE. */
typedef struct vx_cuckoo vx_cuckoo;
vx_status vx_cuckoo_create(uint32_t slot_count, uint32_t max_evictions,
                           vx_cuckoo **out);
vx_status vx_cuckoo_destroy(vx_cuckoo *table);
vx_status vx_cuckoo_clear(vx_cuckoo *table, vx_stream stream);
vx_status vx_cuckoo_insert(vx_cuckoo *table, const uint64_t *keys,
                           const uint32_t *values, uint32_t count,
                           uint32_t *statuses, vx_stream stream);
vx_status vx_cuckoo_find(const vx_cuckoo *table, const uint64_t *keys,
                         uint32_t count, uint32_t *values, vx_stream stream);
size_t vx_cuckoo_bytes(const vx_cuckoo *table);
/* Keys lost to exhausted eviction chains since the last clear (host read,
 * synchronises the stream). */
vx_status vx_cuckoo_dropped(const vx_cuckoo *table, uint64_t *host_count,
                            vx_stream stream);

/* ------------------------------------------------------- common records -- */

/* Voxel coordinate; coordinates outside the world are ignored by edits and
 * read as empty by queries (hash_dag_gpu/types.cuh:11-15,
 * svt/cuda/voxel/types.cuh:11-15). */
typedef struct vx_voxel {
    uint32_t x, y, z;
} vx_voxel;

#define VX_EDIT_DESTROY 0u /* EditOp::Destroy (hash_dag_gpu/types.cuh:30-33) */
#define VX_EDIT_PLACE 1u   /* EditOp::Place */

/* ------------------------------------------------------------- Hash DAG --
 * A hash-consed sparse voxel DAG resident on one GPU.  World side is
 * 4 << depth voxels (depth = inner levels above the 4^3 leaves, the
 * reference's HashDAG(depth), svt/hash_dag.hpp:32-36); the reference GPU DAG
 * is fixed at depth 8 (hash_dag_gpu/config.cuh:14-24), this one takes
 * 1 <= depth <= 14.  Refs are 32-bit: 0 = empty subtree, 1 = full subtree,
 * otherwise a node of that level's pool.  One content-addressed table per
 * level; inner items are [child_mask | fill_mask << 8, child refs...]
 * (hash_dag_gpu/detail/node.cuh:266-289); leaves are 64-bit occupancy masks,
 * bit = x + 4y + 16z.  Replaces HashDagGpu / DeviceHashDagGpu
 * (hash_dag_gpu/storage.cuh:16-105). */
typedef struct vx_dag vx_dag;

typedef struct vx_dag_config {
    uint32_t depth;            /* inner levels, 1..14 */
    uint32_t reserved0;
    uint64_t max_nodes;        /* capacity per level (inner and leaf) */
    uint64_t arena_bytes;      /* scratch for batched / terrain builds (0 = default) */
} vx_dag_config;

vx_status vx_dag_create(const vx_dag_config *config, vx_dag **out);
vx_status vx_dag_destroy(vx_dag *dag);
/* Clear every table and publish the empty root (HashDagGpu::reset,
 * hash_dag_gpu/storage.cuh:57-69). */
vx_status vx_dag_reset(vx_dag *dag, vx_stream stream);
uint32_t vx_dag_depth(const vx_dag *dag);

/* Plain per-call path: one op applied to a list of voxels.  Replaces
 * hash_dag_gpu::{place,destroy,apply}_voxel_edits and
 * apply_voxel_edits_workspace_size (hash_dag_gpu/edit.cuh:16-61).
 * Errors: VX_ERR_INVALID_VALUE for NULL edits with count > 0 or a NULL/short
 * workspace; VX_ERR_CAPACITY (reported as cudaErrorMemoryAllocation's
 * meaning: a node table is full) leaves the previous root published
 * (hash_dag_gpu/detail/edit/root.cuh:13-48).  Synchronises the stream once to
 * read the status, as the reference does. */
size_t vx_dag_voxel_workspace_size(uint32_t count);
vx_status vx_dag_apply_voxels(vx_dag *dag, const vx_voxel *edits,
                              uint32_t count, uint32_t op, void *workspace,
                              size_t workspace_bytes, vx_stream stream);

/* Batched path: a list of sphere / box primitives of mixed add/remove,
 * applied as if sequentially in array order, in one stream-ordered
 * submission with no host synchronisation (capturable in a CUDA graph).
 * Uses the DAG's own arena; the status is left on the device and read with
 * vx_dag_status.  No counterpart in the reference API (which applies one op
 * per call to voxel lists); its result equals applying each primitive's voxel
 * list with apply_voxel_edits in order. */
vx_status vx_dag_apply_primitives(vx_dag *dag, const vx_primitive *prims,
                                  uint32_t count, vx_stream stream);
/* Read and clear the device status of the last submissions (synchronises). */
vx_status vx_dag_status(vx_dag *dag, vx_stream stream);

/* Build the terrain of the given generator into an empty DAG (replaces the
 * DAG with the terrain; stream-ordered, status via vx_dag_status). */
vx_status vx_dag_build_terrain(vx_dag *dag, const vx_terrain *terrain,
                               vx_stream stream);

/* Point queries: out[i] = 1 if voxel pts[i] is solid (hash_dag_gpu::get_voxel,
 * hash_dag_gpu/query.cuh:12-39). */
vx_status vx_dag_query(const vx_dag *dag, const vx_voxel *pts, uint32_t count,
                       uint8_t *out, vx_stream stream);

/* A ray in the DAG's voxel coordinates (the world is [0, 4 << depth)^3, voxel
 * (x, y, z) the unit cube at x, y, z): points origin + t * dir for
 * 0 <= t <= t_max; dir need not be normalised.  32 bytes. */
typedef struct vx_ray {
    float origin[3];
    float dir[3];
    float t_max;
    uint32_t reserved;
} vx_ray;

/* First solid voxel a ray meets: the voxel engine's raycast result words
 * (voxel-engine/engine/voxel/src/voxel/raycast_data.rs:31-47: voxel x, y, z,
 * face, distance), 20 bytes.  face is the hit voxel's side the ray entered
 * through, in the engine's Face order (shaders/svo/face.slang: 0 X+, 1 X-,
 * 2 Y+, 3 Y-, 4 Z+, 5 Z-), 0 when the ray starts inside the world, and 6 =
 * VX_FACE_NO_HIT (voxel ~0, t = -1) when nothing solid lies on [0, t_max]
 * inside the world; t is the ray parameter where it enters the voxel. */
typedef struct vx_ray_hit {
    uint32_t voxel[3];
    uint32_t face;
    float t;
} vx_ray_hit;
#define VX_FACE_NO_HIT 6u

/* Cast rays through the resident DAG: hits[i] for rays[i] (device memory).
 * A DDA over voxel boundaries that steps over whole empty cells of the DAG
 * (one root-to-cell walk per step); every floating-point operation is a
 * correctly rounded single-precision add, multiply, divide or floor, so the
 * result is reproducible bit for bit (voxel_b200_device.cuh vx_dag_raycast).
 * The GPU counterpart of the engine's raycast compute pass
 * (voxel-engine/engine/voxel/src/shaders/svo/raycast_compute_algorithm.slang),
 * over the Hash DAG and for any number of rays. */
vx_status vx_dag_raycast(const vx_dag *dag, const vx_ray *rays, uint32_t count,
                         vx_ray_hit *hits, vx_stream stream);

/* The voxel engine's leaf edit record (voxel-engine/engine/voxel/src/voxel/
 * command.rs:8-16, #[repr(C)], 20 bytes): a leaf at leaf coordinates (voxel
 * coordinates / 4) and a 64-bit voxel mask (bit = x + 4y + 16z) split into
 * low and high words. */
typedef struct vx_leaf_command {
    uint32_t leaf_x, leaf_y, leaf_z;
    uint32_t voxel_data_low, voxel_data_high;
} vx_leaf_command;

/* Apply leaf edit commands in one batched edit: the masks of commands that
 * name the same leaf are OR-merged (LeafEditCommand::merge_commands,
 * command.rs:30-52), then every named leaf is OR-ed with its mask
 * (VX_EDIT_PLACE, the engine's OrPolicy) or cleared by it (VX_EDIT_DESTROY,
 * AndNotPolicy; voxel-engine/engine/voxel/src/shaders/svo/leaf_edit_policy.
 * slang).  Leaves outside the world are ignored; count 0 is a no-op; the
 * workspace contract and statuses are those of vx_dag_apply_voxels.  The SVO
 * form writes `material` (1 when 0) into placed voxels of a material SVO. */
size_t vx_leaf_command_workspace_size(uint32_t count);
vx_status vx_dag_apply_leaf_commands(vx_dag *dag, const vx_leaf_command *cmds, uint32_t count,
                                     uint32_t op, void *workspace, size_t workspace_bytes,
                                     vx_stream stream);

/* Dense read of a box of leaves: out[(z * ny + y) * nx + x] (device memory)
 * = occupancy mask of the leaf at leaf coordinates (lx0 + x, ly0 + y,
 * lz0 + z) (voxel coordinates / 4, bit = x + 4y + 16z; 0 outside the world).
 * The region counterpart of hash_dag_gpu::get_voxel (query.cuh:12-39): one
 * root-to-leaf walk per leaf instead of per voxel, e.g. to mesh or check a
 * region.  nx * ny * nz must be below 2^32. */
vx_status vx_dag_read_leaves(const vx_dag *dag, uint32_t lx0, uint32_t ly0, uint32_t lz0,
                             uint32_t nx, uint32_t ny, uint32_t nz, uint64_t *out,
                             vx_stream stream);

/* Canonical dump (host memory, synchronises): DFS from the root, children
 * 0..7, first visit numbers the nodes of each level.  Each inner node is
 * written as 10 words [child_mask, fill_mask, child ids x 8] (id 0 = empty,
 * 1 = full, k + 2 = k-th node of the next level); each leaf as its u64 mask.
 * host_counts[depth + 1] receives the number of nodes per level.  Call with
 * NULL arrays to query the sizes first.  The root is reported in *host_root
 * (0 empty, 1 full, 2 = node 0 of level 0). */
vx_status vx_dag_export_canonical(const vx_dag *dag, uint32_t *host_root,
                                  uint64_t *host_counts, uint32_t *host_nodes,
                                  uint64_t nodes_capacity_words,
                                  uint64_t *host_leaves,
                                  uint64_t leaves_capacity, vx_stream stream);

/* Rebuild the DAG from a canonical dump in host memory (the format of
 * vx_dag_export_canonical: root 0 / 1 / 2, per-level counts, 10-word node
 * records of levels 0..depth-1 in order, leaf masks).  The tables are reset
 * first; VX_ERR_CAPACITY if a level does not fit, VX_ERR_INVALID_VALUE for a
 * malformed dump.  Synchronises. */
vx_status vx_dag_import_canonical(vx_dag *dag, uint32_t root, const uint64_t *host_counts,
                                  const uint32_t *host_nodes, const uint64_t *host_leaves,
                                  vx_stream stream);
/* Checkpoint / resume of a resident DAG: the canonical dump as a file
 * ("VXDAGCN1", version, depth, root, counts, node records, leaf masks;
 * little-endian) and its import into a DAG of the same depth (any capacity
 * that holds it).  The on-disk counterpart of the reference CPU DAG's
 * compaction (svt/hash_dag.hpp:133-191); the reference has no file format.
 * VX_ERR_IO when the file cannot be read or written. */
vx_status vx_dag_save(const vx_dag *dag, const char *path, vx_stream stream);
vx_status vx_dag_load(vx_dag *dag, const char *path, vx_stream stream);

/* Copy the complete table state of src into dst (same configuration): a
 * device-side snapshot / restore of a resident DAG.  No counterpart in the
 * reference (its GPU DAG is not copyable, hash_dag_gpu/storage.cuh:40-43). */
vx_status vx_dag_copy(vx_dag *dst, const vx_dag *src, vx_stream stream);

/* Compaction: keep only the nodes reachable from the root (edits are
 * copy-on-write, so superseded items accumulate), re-hash-consing them into
 * cleared tables; the canonical content is unchanged.  The GPU counterpart of
 * the reference CPU DAG's collect_garbage (svt/hash_dag.hpp:133-191); the
 * reference GPU DAG has none (append-only, hash_dag_gpu/storage.cuh:14-15).
 * Synchronises; its temporaries live in the DAG's edit arena (returns
 * VX_ERR_CAPACITY, changing nothing, when the arena is too small). */
vx_status vx_dag_compact(vx_dag *dag, vx_stream stream);

/* The same dump for an earlier root ref (e.g. one a served batch published):
 * valid while the tables still hold it, i.e. until the next reset or
 * compaction.  root = 0xffffffff means the current root. */
vx_status vx_dag_export_canonical_at(const vx_dag *dag, uint32_t root,
                                     uint32_t *host_root, uint64_t *host_counts,
                                     uint32_t *host_nodes,
                                     uint64_t nodes_capacity_words,
                                     uint64_t *host_leaves,
                                     uint64_t leaves_capacity, vx_stream stream);

typedef struct vx_dag_stats {
    uint64_t nodes_per_level[16]; /* items stored (live and superseded) */
    uint64_t words_per_level[16];
    uint32_t items_per_level[16]; /* work items of the last edit submission */
    uint32_t pairs_per_level[16]; /* (cell, primitive) pairs of the last submission */
    uint64_t bytes_reserved;
    uint32_t root;
    uint32_t status;
} vx_dag_stats;
vx_status vx_dag_get_stats(const vx_dag *dag, vx_dag_stats *host_stats,
                           vx_stream stream);

/* ------------------------------------------------------------------ SVO --
 * Pointer-based sparse voxel octree with free lists.  World side 4 << depth,
 * 1 <= depth <= 12 (the reference GPU SVO is fixed at depth 10,
 * svt/cuda/config.cuh:17-31).  Node = 8 x u32 child_data: bits 0-29 child
 * index, bit 30 child present, bit 31 filled-when-absent (svt/cuda/config.cuh:
 * 36-42).  Leaves are u64 masks, bit = x + 4y + 16z.  With materials enabled
 * each leaf also holds 64 material bytes, a uniform filled child stores its
 * material in bits 0-7, and a region collapses only when occupancy and
 * material are both uniform; with materials disabled the structure is exactly
 * the reference's (svt/svo.hpp, svt/cuda/voxel/detail/collapse).
 * Replaces GpuSvo / DeviceGpuSvo / reset_svo (svt/cuda/storage.cuh:12-122,
 * svt/cuda/device_view.cuh:11-44, svt/cuda/svo.cuh:17-22). */
typedef struct vx_svo vx_svo;

typedef struct vx_svo_config {
    uint32_t depth;           /* inner levels, 1..12 */
    uint32_t materials;       /* 0 = occupancy only, 1 = uint8 material per voxel */
    uint32_t max_nodes;
    uint32_t max_leaves;
    uint64_t arena_bytes;     /* scratch for batched / terrain builds (0 = default) */
} vx_svo_config;

vx_status vx_svo_create(const vx_svo_config *config, vx_svo **out);
vx_status vx_svo_destroy(vx_svo *svo);
vx_status vx_svo_reset(vx_svo *svo, vx_stream stream);
uint32_t vx_svo_depth(const vx_svo *svo);

/* Plain per-call path: place (with a material) or destroy a voxel list.
 * Replaces svt::cuda::{place,destroy}_voxel_edits and
 * apply_voxel_edits_workspace_size (svt/cuda/voxel/edit.cuh:14-92). */
size_t vx_svo_voxel_workspace_size(uint32_t count);
vx_status vx_svo_apply_voxels(vx_svo *svo, const vx_voxel *edits,
                              uint32_t count, uint32_t op, uint32_t material,
                              void *workspace, size_t workspace_bytes,
                              vx_stream stream);
/* Batched primitives, sequential semantics in array order (see the DAG). */
vx_status vx_svo_apply_primitives(vx_svo *svo, const vx_primitive *prims,
                                  uint32_t count, vx_stream stream);
vx_status vx_svo_status(vx_svo *svo, vx_stream stream);
vx_status vx_svo_build_terrain(vx_svo *svo, const vx_terrain *terrain,
                               vx_stream stream);
/* out[i] = material of voxel pts[i] (0 = empty; 1 for solid without
 * materials) (svt::cuda::get_voxel, svt/cuda/query.cuh:11-35). */
vx_status vx_svo_query(const vx_svo *svo, const vx_voxel *pts, uint32_t count,
                       uint8_t *out, vx_stream stream);
/* Leaf edit commands on the SVO (see vx_dag_apply_leaf_commands). */
vx_status vx_svo_apply_leaf_commands(vx_svo *svo, const vx_leaf_command *cmds, uint32_t count,
                                     uint32_t op, uint32_t material, void *workspace,
                                     size_t workspace_bytes, vx_stream stream);
/* Canonical dump (host, synchronises): DFS first-visit renumbering of nodes
 * and leaves; host_nodes gets 8 words per node with child indices replaced by
 * canonical ones and bits 30/31 (and materials) kept; host_leaves gets the u64
 * masks; host_materials (may be NULL) 64 bytes per leaf.  NULL arrays query
 * the counts. */
vx_status vx_svo_export_canonical(const vx_svo *svo, uint32_t *host_node_count,
                                  uint32_t *host_leaf_count,
                                  uint32_t *host_nodes, uint32_t nodes_capacity,
                                  uint64_t *host_leaves,
                                  uint8_t *host_materials,
                                  uint32_t leaves_capacity, vx_stream stream);

/* Garbage collection.  A subtree that an edit overwrites with a uniform
 * region becomes unreachable; its nodes and leaves go back to the free lists
 * when a collection runs (mark from the root, then rebuild the free lists).
 * Edits collect lazily: only when one would not fit in the room left (free
 * lists plus the never-used tail) does the collection run, inside that edit
 * and before it allocates anything; the edit fails with VX_ERR_CAPACITY only
 * if it still does not fit.  vx_svo_collect runs a collection now (stream
 * ordered; nothing runs when no subtree was detached since the last one), so
 * that the counters below count only reachable storage.  The reference frees
 * a collapsed node's storage as part of each edit (svt/cuda/voxel/detail/
 * collapse/pipeline.cuh:55-110). */
vx_status vx_svo_collect(vx_svo *svo, vx_stream stream);

/* Counters (GpuSvoCounters, svt/cuda/device_view.cuh:24-29). */
typedef struct vx_svo_counters {
    uint32_t node_count;
    uint32_t leaf_count;
    uint32_t free_node_count;
    uint32_t free_leaf_count;
} vx_svo_counters;
vx_status vx_svo_get_counters(const vx_svo *svo, vx_svo_counters *host_counters,
                              vx_stream stream);

/* ------------------------------------------------------- device views --
 * Trivially copyable views for user kernels that read the structures with
 * the __device__ functions of voxel_b200_device.cuh (vx_dag_get_voxel,
 * vx_svo_get_voxel, vx_slab_set_contains_warp, vx_cuckoo_find), the
 * counterparts of the reference's view() / device_view() and its device read
 * functions (svt/hash_dag_gpu/device_view.cuh:14-31, svt/cuda/device_view.cuh:
 * 11-44, cuda/hash_table/slab_hash/set/device.cuh).  All pointers are device
 * pointers, valid while the structure lives; the DAG view reads the current
 * root at each lookup. */
typedef struct vx_dag_view {
    uint32_t depth;
    uint32_t reserved;
    const uint32_t *root;      /* the published root ref */
    const uint32_t *pool[14];  /* inner items of levels 0..depth-1 */
    const uint64_t *leaves;    /* leaf masks (ref - 2 = slot) */
} vx_dag_view;

typedef struct vx_svo_view {
    uint32_t depth;
    uint32_t materials;
    const uint32_t *nodes;          /* 8 child words per node, root = node 0 */
    const uint64_t *leaves;         /* leaf masks */
    const uint8_t *materials_data;  /* 64 bytes per leaf (materials only) */
} vx_svo_view;

typedef struct vx_slab_set_view {
    const void *slabs;       /* buckets then overflow slabs, 128 bytes each */
    uint32_t bucket_count;
    uint32_t capacity;       /* overflow slabs */
} vx_slab_set_view;

typedef struct vx_cuckoo_view {
    const void *slots;       /* buckets of two 16-byte slots {key, value | choice << 32} */
    uint32_t slot_count;
    uint32_t reserved;
} vx_cuckoo_view;

vx_status vx_dag_device_view(const vx_dag *dag, vx_dag_view *out);
vx_status vx_svo_device_view(const vx_svo *svo, vx_svo_view *out);
vx_status vx_slab_set_device_view(const vx_slab_set *set, vx_slab_set_view *out);
vx_status vx_cuckoo_device_view(const vx_cuckoo *map, vx_cuckoo_view *out);

/* --------------------------------------------------------------- graphs --
 * A batched edit as a CUDA graph: the capture records every kernel, memset
 * and copy of one edit; each vx_graph_launch replays them with one launch.
 * The graph reads its input from the given device addresses when it runs
 * (rewrite the buffers between launches; same addresses), keeps the
 * structure's table addresses (valid while it lives, through resets,
 * copies into it and compactions) and the tuning knobs of capture time.
 * vx_*_graph_primitives: the list at `prims` of *device_count primitives
 * (read on the device at each launch; at most `capacity`, else the edit is
 * rejected with VX_ERR_INVALID_VALUE), or of `capacity` primitives when
 * device_count is NULL.  vx_dag_graph_voxels: the plain path (sort, merge into
 * leaf masks, rebuild) for `count` voxels at `edits` with op and workspace.
 * Check results with vx_*_status after a launch.  The reference runs its
 * pipelines as separate launches with host synchronisations (svt/hash_dag_gpu/
 * detail/edit_pipeline.cuh:31-97); there is no counterpart. */
typedef struct vx_graph vx_graph;
vx_status vx_dag_graph_primitives(vx_dag *dag, const vx_primitive *prims,
                                  const uint32_t *device_count, uint32_t capacity,
                                  vx_graph **out);
vx_status vx_dag_graph_voxels(vx_dag *dag, const vx_voxel *edits, uint32_t count,
                              uint32_t op, void *workspace, size_t workspace_bytes,
                              vx_graph **out);
vx_status vx_svo_graph_primitives(vx_svo *svo, const vx_primitive *prims,
                                  const uint32_t *device_count, uint32_t capacity,
                                  vx_graph **out);
vx_status vx_graph_launch(vx_graph *graph, vx_stream stream);
/* Kernel launches one replay performs. */
vx_status vx_graph_kernels(const vx_graph *graph, uint64_t *host_kernels);
vx_status vx_graph_destroy(vx_graph *graph);

/* ------------------------------------------------------- terminal edits --
 * Place or destroy whole octree cells and 4^3 bricks (svt/cuda/terminal/
 * types.cuh:15-31, detail/pipeline.cuh:27-222).  A node input is the cell at
 * `depth` (0 = the whole world, `depth` of the structure = one leaf) whose
 * path from the root is `prefix` (3 bits per level, the root's child in the
 * highest triple, child = x | y << 1 | z << 2), moved by a voxel offset; a leaf
 * input is a 4^3 brick (bit x + 4y + 16z of mask64) at the full-depth path
 * `leaf_prefix`, moved by a voxel offset.  Every voxel of the union of the
 * moved inputs that lies inside the world becomes filled (place) or empty
 * (destroy); inputs with depth > structure depth or prefix bits above
 * 3 * depth are ignored, as in the reference.  Structures of depth <= 10
 * (prefixes are 32-bit).  Layouts match TerminalNodeInput (20 B) and
 * TerminalLeafInput (32 B). */
typedef struct vx_terminal_node {
    uint32_t depth;
    uint32_t prefix;
    int32_t offset[3];
} vx_terminal_node;

typedef struct vx_terminal_leaf {
    uint32_t leaf_prefix;
    uint32_t pad0;
    uint64_t mask64;
    int32_t offset[3];
    uint32_t pad1;
} vx_terminal_leaf;

/* Workspace for one call (> 0 even for empty inputs: a NULL workspace is
 * rejected as in the reference, detail/pipeline.cuh:41-46). */
size_t vx_terminal_workspace_size(uint32_t node_count, uint32_t leaf_count);
/* Synchronise and return the edit's status (as the reference does).
 * Replaces place_terminal_edits / destroy_terminal_edits
 * (svt/cuda/terminal/detail/pipeline.cuh:200-222); `material` is used when
 * the SVO has materials (0 = 1). */
vx_status vx_svo_apply_terminal(vx_svo *svo, const vx_terminal_node *nodes,
                                uint32_t node_count, const vx_terminal_leaf *leaves,
                                uint32_t leaf_count, uint32_t op, uint32_t material,
                                void *workspace, size_t workspace_bytes,
                                vx_stream stream);
/* The same edit on a Hash DAG (depth <= 10). */
vx_status vx_dag_apply_terminal(vx_dag *dag, const vx_terminal_node *nodes,
                                uint32_t node_count, const vx_terminal_leaf *leaves,
                                uint32_t leaf_count, uint32_t op, void *workspace,
                                size_t workspace_bytes, vx_stream stream);

/* -------------------------------------------------------------- serving --
 * A request loop over a resident Hash DAG with continuous batching: submitted
 * requests (lists of primitives) are applied in submission order; queued
 * requests are coalesced into one batched edit per launch, up to two launches
 * are in flight.  Admission is by the memory a request needs: each request's
 * new nodes per level are estimated from its primitives' surfaces, and a
 * request joins a batch only while the tables' use plus the estimates of the
 * batches in flight and of the batch stay within compact_at_fill of every
 * table's room; when not even the next request fits, the DAG is compacted
 * first.  Completions report the
 * commit time (host clock of vx_serve_now_ns, when the batch's completion was
 * observed) and the root the batch published.  The server owns the DAG's
 * stream while it runs.  Creation compacts the DAG once (synchronously), which
 * also loads the compaction kernels before the first request.  No
 * counterpart in the reference (no serving path). */
typedef struct vx_server vx_server;

typedef struct vx_serve_config {
    uint32_t max_batch_prims;    /* primitives per launch (0 = 65536) */
    uint32_t max_batch_requests; /* requests per launch (0 = unlimited, 1 = one each) */
    double compact_at_fill;      /* fill limit of admission (0 = 0.9; above 1 never compacts
                                    before a batch overflows) */
    uint32_t max_inflight;       /* launches in flight, 1 or 2 (0 = 2) */
    uint32_t launch_mode;        /* 0 = one CUDA graph launch per batch,
                                    1 = the pipeline's kernels one by one */
} vx_serve_config;

typedef struct vx_serve_completion {
    uint64_t request_id;
    uint64_t arrival_ns;
    uint64_t commit_ns;
    uint32_t status;             /* 0 = committed */
    uint32_t root;               /* root ref published by the request's batch */
} vx_serve_completion;

typedef struct vx_serve_stats {
    uint64_t batches;
    uint64_t requests;
    uint64_t prims;
    uint64_t compactions;
    uint64_t recoveries;
    double compact_ms;
} vx_serve_stats;

uint64_t vx_serve_now_ns(void);
vx_status vx_serve_create(vx_dag *dag, const vx_serve_config *config, vx_server **out);
/* Copies the host primitives; thread-safe. */
vx_status vx_serve_submit(vx_server *server, uint64_t request_id,
                          const vx_primitive *host_prims, uint32_t count,
                          uint64_t arrival_ns);
/* Moves up to `capacity` completions into host_out. */
vx_status vx_serve_poll(vx_server *server, vx_serve_completion *host_out,
                        uint32_t capacity, uint32_t *host_count);
/* Blocks until every submitted request has completed. */
vx_status vx_serve_drain(vx_server *server);
vx_status vx_serve_get_stats(vx_server *server, vx_serve_stats *host_stats);
/* Drains, stops the threads and frees the server (not the DAG). */
vx_status vx_serve_destroy(vx_server *server);

/* Seeded served-request stream (vx_workload.h): Poisson arrivals at `rate`
 * per second for `seconds`, Zipf(zipf_s) sizes over [1, max_size], primitives
 * from `mix`.  NULL arrays return only the counts. */
vx_status vx_generate_requests(const vx_edit_mix *mix, uint64_t seed, double rate,
                               double seconds, double zipf_s, uint32_t max_size,
                               uint64_t max_requests, uint64_t *host_arrival_ns,
                               uint32_t *host_sizes, uint64_t max_prims,
                               vx_primitive *host_prims, uint64_t *host_requests,
                               uint64_t *host_total_prims);

/* ---------------------------------------------------------- rasterising --
 * Expand primitives into voxel lists (the plain path's input shape).
 * out_offsets[i] = first voxel of primitive i (exclusive scan of counts);
 * voxels are clipped to [0, world)^3.  Returns VX_ERR_CAPACITY if the total
 * exceeds capacity (out_total still receives it). */
vx_status vx_rasterize_count(const vx_primitive *prims, uint32_t count,
                             uint32_t world_exp, uint64_t *out_counts,
                             vx_stream stream);
vx_status vx_rasterize(const vx_primitive *prims, uint32_t count,
                       uint32_t world_exp, const uint64_t *offsets,
                       vx_voxel *out, vx_stream stream);

#ifdef __cplusplus
}
#endif

#endif /* VOXEL_B200_H */
