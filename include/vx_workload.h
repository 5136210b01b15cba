/*
 * vx_workload.h - seeded synthetic workloads for the voxel-editing path.
 *
 * The reference ships no dataset: its benches synthesise voxel spheres
 * (algorithm/bench/bench_cuda_svt.cu:37-80) and random/dense edit lists
 * (algorithm/bench/bench_cuda_hash_dag_gpu.cu:60-75).  This header defines the
 * workloads this library is measured on, in integer arithmetic only, so that the
 * CUDA kernels, the C++ host code and the CPU oracle evaluate bit-identical
 * occupancy for the same seed:
 *
 *   - PCG32 (O'Neill 2014, "PCG: A Family of Simple Fast Space-Efficient
 *     Statistically Good Algorithms for Random Number Generation"), restated;
 *   - value noise whose lattice values are PCG32 outputs keyed by the lattice
 *     point, interpolated bilinearly (2-D height) or trilinearly (3-D caves) in
 *     exact 64-bit fixed point;
 *   - a heightfield terrain  z < base + amp * v(x, y)  with 3 octaves
 *     (spacings 64/32/16 * scale, amplitudes 1/.5/.25), optional caves where the
 *     3-D noise (spacing 8 * scale) exceeds 0.55, and a uint8 material per
 *     height band;
 *   - sphere and axis-aligned box edit primitives.  A voxel p is inside a
 *     sphere iff |p - c|^2 <= r^2 (the reference's voxel_inside_sphere,
 *     algorithm/bench/bench_cuda_svt.cu:37-44) and inside a box iff
 *     |p_i - c_i| <= h_i on every axis.
 *
 * Everything here is header-only and usable from C, C++ and CUDA device code.
 */
#ifndef VX_WORKLOAD_H
#define VX_WORKLOAD_H

#include <stdint.h>

#ifdef __CUDACC__
#define VX_HD __host__ __device__ __forceinline__
#else
#define VX_HD static inline
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- PCG32 -- */

typedef struct vx_pcg32 {
    uint64_t state;
    uint64_t inc;
} vx_pcg32;

VX_HD uint32_t vx_pcg32_next(vx_pcg32 *rng) {
    const uint64_t old = rng->state;
    rng->state = old * 6364136223846793005ULL + rng->inc;
    const uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = (uint32_t)(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((0u - rot) & 31u));
}

VX_HD void vx_pcg32_seed(vx_pcg32 *rng, uint64_t initstate, uint64_t initseq) {
    rng->state = 0u;
    rng->inc = (initseq << 1u) | 1u;
    (void)vx_pcg32_next(rng);
    rng->state += initstate;
    (void)vx_pcg32_next(rng);
}

/* Uniform integer in [0, bound) without modulo bias (rejection of the low
 * remainder, as in the PCG paper's pcg32_boundedrand). */
VX_HD uint32_t vx_pcg32_bounded(vx_pcg32 *rng, uint32_t bound) {
    const uint32_t threshold = (0u - bound) % bound;
    for (;;) {
        const uint32_t r = vx_pcg32_next(rng);
        if (r >= threshold) return r % bound;
    }
}

/* ---------------------------------------------------------- value noise -- */

/* Lattice values are signed integers in [-32768, 32767], i.e. [-1, 1) with a
 * fixed-point scale of 32768. */
#define VX_NOISE_ONE 32768

VX_HD int32_t vx_lattice_value(uint32_t seed, uint32_t stream, int64_t i,
                               int64_t j, int64_t k) {
    vx_pcg32 rng;
    const uint64_t key = ((uint64_t)(uint32_t)i * 0x9E3779B97F4A7C15ULL) ^
                         ((uint64_t)(uint32_t)j * 0xC2B2AE3D27D4EB4FULL) ^
                         ((uint64_t)(uint32_t)k * 0x165667B19E3779F9ULL) ^
                         ((uint64_t)seed << 32);
    vx_pcg32_seed(&rng, key, stream);
    return (int32_t)(vx_pcg32_next(&rng) >> 16) - 32768;
}

/* Bilinear value noise numerator at (x, y) for lattice spacing s:
 * v = result / (s * s * VX_NOISE_ONE). */
VX_HD int64_t vx_noise2_num(uint32_t seed, uint32_t stream, uint32_t s,
                            uint32_t x, uint32_t y) {
    const int64_t i = x / s, j = y / s;
    const int64_t fx = x % s, fy = y % s;
    const int64_t gx = (int64_t)s - fx, gy = (int64_t)s - fy;
    const int64_t v00 = vx_lattice_value(seed, stream, i, j, 0);
    const int64_t v10 = vx_lattice_value(seed, stream, i + 1, j, 0);
    const int64_t v01 = vx_lattice_value(seed, stream, i, j + 1, 0);
    const int64_t v11 = vx_lattice_value(seed, stream, i + 1, j + 1, 0);
    return gx * gy * v00 + fx * gy * v10 + gx * fy * v01 + fx * fy * v11;
}

/* Trilinear value noise numerator: v = result / (s^3 * VX_NOISE_ONE). */
VX_HD int64_t vx_noise3_num(uint32_t seed, uint32_t stream, uint32_t s,
                            uint32_t x, uint32_t y, uint32_t z) {
    const int64_t i = x / s, j = y / s, k = z / s;
    const int64_t f[3] = {(int64_t)(x % s), (int64_t)(y % s), (int64_t)(z % s)};
    int64_t acc = 0;
    for (uint32_t c = 0; c < 8u; ++c) {
        const int64_t wx = (c & 1u) ? f[0] : (int64_t)s - f[0];
        const int64_t wy = (c & 2u) ? f[1] : (int64_t)s - f[1];
        const int64_t wz = (c & 4u) ? f[2] : (int64_t)s - f[2];
        acc += wx * wy * wz *
               vx_lattice_value(seed, stream, i + (c & 1u), j + ((c >> 1) & 1u),
                                k + ((c >> 2) & 1u));
    }
    return acc;
}

/* -------------------------------------------------------------- terrain -- */

typedef struct vx_terrain {
    uint32_t seed;
    uint32_t scale;       /* 1 for 256^3, 16 for 4096^3, 32 / 64 for 8192^3 / 16384^3 */
    uint32_t caves;       /* 0 = heightfield only, 1 = carve 3-D noise caves */
    uint32_t world_exp;   /* log2(world side) */
} vx_terrain;

/* Height noise at column (x, y), scaled so that
 *   v(x, y) = vx_terrain_hnum(...) / (s0^2 * VX_NOISE_ONE),  s0 = 64 * scale.
 * Octaves 64/32/16 * scale with amplitudes 1/.5/.25 share the denominator
 * s0^2 because .5 / (s0/2)^2 = 2 / s0^2 and .25 / (s0/4)^2 = 4 / s0^2. */
VX_HD int64_t vx_terrain_hnum(const vx_terrain *t, uint32_t x, uint32_t y) {
    const uint32_t s0 = 64u * t->scale;
    return vx_noise2_num(t->seed, 1u, s0, x, y) +
           2 * vx_noise2_num(t->seed, 2u, s0 / 2u, x, y) +
           4 * vx_noise2_num(t->seed, 3u, s0 / 4u, x, y);
}

/* Denominator of the height noise, s0^2 * VX_NOISE_ONE. */
VX_HD int64_t vx_terrain_hden(const vx_terrain *t) {
    const int64_t s0 = 64 * (int64_t)t->scale;
    return s0 * s0 * VX_NOISE_ONE;
}

/* True iff voxel height z lies below the surface: z < 128s + 40s * v. */
VX_HD int vx_terrain_below(const vx_terrain *t, int64_t hnum, uint32_t z) {
    const int64_t den = vx_terrain_hden(t);
    const int64_t s = t->scale;
    return (int64_t)z * den < 128 * s * den + 40 * s * hnum;
}

/* Cave noise numerator; the voxel is carved iff 100 * num > 55 * c^3 * ONE. */
VX_HD int vx_terrain_carved(const vx_terrain *t, uint32_t x, uint32_t y,
                            uint32_t z) {
    const int64_t c = 8 * (int64_t)t->scale;
    return 100 * vx_noise3_num(t->seed, 4u, (uint32_t)c, x, y, z) >
           55 * c * c * c * VX_NOISE_ONE;
}

VX_HD int vx_terrain_solid(const vx_terrain *t, uint32_t x, uint32_t y,
                           uint32_t z) {
    if (!vx_terrain_below(t, vx_terrain_hnum(t, x, y), z)) return 0;
    return !(t->caves && vx_terrain_carved(t, x, y, z));
}

/* Height-band material: eight bands of 8 * scale voxels, cycling, in [1, 8]. */
VX_HD uint32_t vx_terrain_material(const vx_terrain *t, uint32_t z) {
    return 1u + (z / (8u * t->scale)) % 8u;
}

/* Cell classification results shared by terrain and primitive tests. */
#define VX_CELL_EMPTY 0u   /* no voxel of the cell is affected / solid */
#define VX_CELL_FULL 1u    /* every voxel of the cell is affected / solid */
#define VX_CELL_MIXED 2u   /* unknown or mixed: subdivide */

/* Conservative bounds of lattice values over lattice points [i0..i1]x[j0..j1]x
 * [k0..k1].  Ranges of more than 64 points use the full value range. */
VX_HD void vx_lattice_bounds(uint32_t seed, uint32_t stream, int64_t i0,
                             int64_t i1, int64_t j0, int64_t j1, int64_t k0,
                             int64_t k1, int64_t *lo, int64_t *hi) {
    if ((i1 - i0 + 1) * (j1 - j0 + 1) * (k1 - k0 + 1) > 64) {
        *lo = -32768;
        *hi = 32767;
        return;
    }
    int64_t mn = 32767, mx = -32768;
    for (int64_t k = k0; k <= k1; ++k)
        for (int64_t j = j0; j <= j1; ++j)
            for (int64_t i = i0; i <= i1; ++i) {
                const int64_t v = vx_lattice_value(seed, stream, i, j, k);
                mn = v < mn ? v : mn;
                mx = v > mx ? v : mx;
            }
    *lo = mn;
    *hi = mx;
}

/* Bounds of one height octave (spacing sp, stream) over the footprint
 * [x0, x1] x [y0, y1] of integer columns, in numerator units (sp^2 * value).
 * Inside one lattice cell the bilinear interpolant is multilinear, so its
 * extrema are at the footprint's corner columns (exact bound); larger
 * footprints use the range of the lattice values they span. */
VX_HD void vx_octave_bounds(uint32_t seed, uint32_t stream, int64_t sp,
                            uint32_t x0, uint32_t x1, uint32_t y0, uint32_t y1,
                            int64_t *lo, int64_t *hi) {
    if (x0 / sp == x1 / sp && y0 / sp == y1 / sp) {
        const uint32_t xs[2] = {x0, x1}, ys[2] = {y0, y1};
        int64_t mn = 0, mx = 0;
        for (int k = 0; k < 4; ++k) {
            const int64_t v = vx_noise2_num(seed, stream, (uint32_t)sp, xs[k & 1], ys[k >> 1]);
            mn = (k == 0 || v < mn) ? v : mn;
            mx = (k == 0 || v > mx) ? v : mx;
        }
        *lo = mn;
        *hi = mx;
        return;
    }
    int64_t l, h;
    vx_lattice_bounds(seed, stream, x0 / sp, x1 / sp + 1, y0 / sp, y1 / sp + 1, 0, 0,
                      &l, &h);
    *lo = l * sp * sp;
    *hi = h * sp * sp;
}

/* Classify the terrain occupancy of the cube [x0, x0+n)x[y0, y0+n)x[z0, z0+n).
 * The bounds never exclude a value the noise takes inside the cube, so FULL /
 * EMPTY answers are exact; MIXED means "subdivide". */
VX_HD uint32_t vx_terrain_classify(const vx_terrain *t, uint32_t x0,
                                   uint32_t y0, uint32_t z0, uint32_t n) {
    const int64_t s = t->scale;
    const int64_t den = vx_terrain_hden(t);
    const uint32_t x1 = x0 + n - 1, y1 = y0 + n - 1, z1 = z0 + n - 1;
    int64_t hlo = 0, hhi = 0;
    for (uint32_t o = 0; o < 3u; ++o) {
        const int64_t sp = (64 * s) >> o;
        int64_t lo, hi;
        vx_octave_bounds(t->seed, 1u + o, sp, x0, x1, y0, y1, &lo, &hi);
        const int64_t w = (int64_t)1 << o; /* octave weight 1, 2, 4 */
        hlo += w * lo;
        hhi += w * hi;
    }
    /* all voxels below: z1 * den < 128 s den + 40 s hlo */
    const int all_below = (int64_t)z1 * den < 128 * s * den + 40 * s * hlo;
    /* no voxel below: z0 * den >= 128 s den + 40 s hhi */
    const int none_below = (int64_t)z0 * den >= 128 * s * den + 40 * s * hhi;
    if (none_below) return VX_CELL_EMPTY;
    if (!t->caves) return all_below ? VX_CELL_FULL : VX_CELL_MIXED;
    const int64_t c = 8 * s;
    const int64_t c3 = c * c * c;
    int64_t clo, chi;
    if (x0 / c == x1 / c && y0 / c == y1 / c && z0 / c == z1 / c) {
        /* one lattice cell: the trilinear extrema are at the 8 cube corners */
        const uint32_t xs[2] = {x0, x1}, ys[2] = {y0, y1}, zs[2] = {z0, z1};
        for (int k = 0; k < 8; ++k) {
            const int64_t v = vx_noise3_num(t->seed, 4u, (uint32_t)c, xs[k & 1],
                                            ys[(k >> 1) & 1], zs[k >> 2]);
            clo = (k == 0 || v < clo) ? v : clo;
            chi = (k == 0 || v > chi) ? v : chi;
        }
    } else {
        int64_t l, h;
        vx_lattice_bounds(t->seed, 4u, x0 / c, x1 / c + 1, y0 / c, y1 / c + 1,
                          z0 / c, z1 / c + 1, &l, &h);
        clo = l * c3;
        chi = h * c3;
    }
    const int64_t thr = 55 * c3 * VX_NOISE_ONE;
    if (100 * clo > thr) return VX_CELL_EMPTY;          /* all carved */
    const int none_carved = 100 * chi <= thr;
    return (all_below && none_carved) ? VX_CELL_FULL : VX_CELL_MIXED;
}

/* ----------------------------------------------------------- primitives -- */

#define VX_SHAPE_SPHERE 0u
#define VX_SHAPE_BOX 1u
#define VX_SHAPE_AABB 4u /* half-open box [c, c + r) per axis */
#define VX_OP_REMOVE 0u
#define VX_OP_ADD 1u

/* One edit primitive (32 bytes).  Spheres use r[0] as the radius; boxes use
 * r[0..2] as inclusive half-extents around c; axis-aligned boxes (AABB) cover
 * [c, c + r) per axis, so they can have even sides (aligned octree cells).
 * flags = shape | op << 8 | material << 16.  Within a batch, primitives
 * apply in array order (later ones win). */
typedef struct vx_primitive {
    int32_t c[3];
    uint32_t r[3];
    uint32_t flags;
    uint32_t reserved;
} vx_primitive;

VX_HD uint32_t vx_prim_shape(const vx_primitive *p) { return p->flags & 0xffu; }
VX_HD uint32_t vx_prim_op(const vx_primitive *p) { return (p->flags >> 8) & 0xffu; }
VX_HD uint32_t vx_prim_material(const vx_primitive *p) {
    return (p->flags >> 16) & 0xffu;
}
VX_HD uint32_t vx_make_flags(uint32_t shape, uint32_t op, uint32_t material) {
    return shape | (op << 8) | (material << 16);
}

/* Inclusive voxel range [lo, hi] of a box or AABB primitive along axis a
 * (empty when hi < lo). */
VX_HD void vx_prim_axis_range(const vx_primitive *p, int a, int64_t *lo, int64_t *hi) {
    if (vx_prim_shape(p) == VX_SHAPE_AABB) {
        *lo = (int64_t)p->c[a];
        *hi = (int64_t)p->c[a] + (int64_t)p->r[a] - 1;
    } else {
        *lo = (int64_t)p->c[a] - (int64_t)p->r[a];
        *hi = (int64_t)p->c[a] + (int64_t)p->r[a];
    }
}

VX_HD int vx_prim_contains_voxel(const vx_primitive *p, int64_t x, int64_t y,
                                 int64_t z) {
    if (vx_prim_shape(p) == VX_SHAPE_AABB) {
        const int64_t v[3] = {x, y, z};
        for (int a = 0; a < 3; ++a) {
            int64_t lo, hi;
            vx_prim_axis_range(p, a, &lo, &hi);
            if (v[a] < lo || v[a] > hi) return 0;
        }
        return 1;
    }
    const int64_t dx = x - p->c[0], dy = y - p->c[1], dz = z - p->c[2];
    if (vx_prim_shape(p) == VX_SHAPE_SPHERE) {
        const int64_t r = p->r[0];
        return dx * dx + dy * dy + dz * dz <= r * r;
    }
    return (dx < 0 ? -dx : dx) <= (int64_t)p->r[0] &&
           (dy < 0 ? -dy : dy) <= (int64_t)p->r[1] &&
           (dz < 0 ? -dz : dz) <= (int64_t)p->r[2];
}

/* Classify a primitive against the voxel cube [x0, x0+n)^3 (exact for both
 * shapes: the nearest and farthest voxels of the cube decide). */
VX_HD uint32_t vx_prim_classify(const vx_primitive *p, int64_t x0, int64_t y0,
                                int64_t z0, int64_t n) {
    const int64_t lo[3] = {x0, y0, z0};
    if (vx_prim_shape(p) == VX_SHAPE_SPHERE) {
        int64_t near2 = 0, far2 = 0;
        for (int a = 0; a < 3; ++a) {
            const int64_t c = p->c[a];
            const int64_t a0 = lo[a], a1 = lo[a] + n - 1;
            const int64_t d = c < a0 ? a0 - c : (c > a1 ? c - a1 : 0);
            near2 += d * d;
            const int64_t f0 = c - a0 > 0 ? c - a0 : a0 - c;
            const int64_t f1 = c - a1 > 0 ? c - a1 : a1 - c;
            const int64_t f = f0 > f1 ? f0 : f1;
            far2 += f * f;
        }
        const int64_t r2 = (int64_t)p->r[0] * (int64_t)p->r[0];
        if (near2 > r2) return VX_CELL_EMPTY;
        return far2 <= r2 ? VX_CELL_FULL : VX_CELL_MIXED;
    }
    int inside = 1;
    for (int a = 0; a < 3; ++a) {
        int64_t b0, b1;
        vx_prim_axis_range(p, a, &b0, &b1);
        if (b1 < lo[a] || b0 > lo[a] + n - 1) return VX_CELL_EMPTY;
        if (!(b0 <= lo[a] && b1 >= lo[a] + n - 1)) inside = 0;
    }
    return inside ? VX_CELL_FULL : VX_CELL_MIXED;
}

/* 64-bit mask of the voxels of the 4^3 leaf at (x0, y0, z0) that the primitive
 * covers; bit index = x + 4y + 16z (algorithm/lib/include/algo/svt/hash_dag.hpp
 * get_leaf_offset). */
VX_HD uint64_t vx_prim_leaf_mask(const vx_primitive *p, int64_t x0, int64_t y0,
                                 int64_t z0) {
    uint64_t m = 0;
    if (vx_prim_shape(p) != VX_SHAPE_SPHERE) {
        uint32_t ax[3];
        const int64_t lo[3] = {x0, y0, z0};
        for (int a = 0; a < 3; ++a) {
            int64_t b0, b1;
            vx_prim_axis_range(p, a, &b0, &b1);
            uint32_t bits = 0;
            for (int i = 0; i < 4; ++i) {
                const int64_t v = lo[a] + i;
                if (v >= b0 && v <= b1) bits |= 1u << i;
            }
            ax[a] = bits;
        }
        for (uint32_t z = 0; z < 4; ++z)
            for (uint32_t y = 0; y < 4; ++y)
                if (((ax[1] >> y) & (ax[2] >> z) & 1u) != 0u)
                    m |= (uint64_t)ax[0] << (4u * y + 16u * z);
        return m;
    }
    const int64_t r2 = (int64_t)p->r[0] * (int64_t)p->r[0];
    for (uint32_t z = 0; z < 4; ++z) {
        const int64_t dz = z0 + z - p->c[2];
        for (uint32_t y = 0; y < 4; ++y) {
            const int64_t dy = y0 + y - p->c[1];
            const int64_t rem = r2 - dz * dz - dy * dy;
            if (rem < 0) continue;
            for (uint32_t x = 0; x < 4; ++x) {
                const int64_t dx = x0 + x - p->c[0];
                if (dx * dx <= rem) m |= 1ull << (x + 4u * y + 16u * z);
            }
        }
    }
    return m;
}

/* Terrain occupancy of one 4^3 leaf as a 64-bit mask. */
VX_HD uint64_t vx_terrain_leaf_mask(const vx_terrain *t, uint32_t x0,
                                    uint32_t y0, uint32_t z0) {
    uint64_t m = 0;
    for (uint32_t y = 0; y < 4; ++y)
        for (uint32_t x = 0; x < 4; ++x) {
            const int64_t h = vx_terrain_hnum(t, x0 + x, y0 + y);
            for (uint32_t z = 0; z < 4; ++z) {
                if (!vx_terrain_below(t, h, z0 + z)) continue;
                if (t->caves && vx_terrain_carved(t, x0 + x, y0 + y, z0 + z))
                    continue;
                m |= 1ull << (x + 4u * y + 16u * z);
            }
        }
    return m;
}

/* ------------------------------------------------- edit-stream generator --
 * Host-only: seeded primitive lists for the benchmark configurations.  Per
 * primitive, in this order: centre x, y, z uniform in [0, world); shape
 * (sphere with probability sphere_permille / 1000, else box); op (add with
 * probability add_permille / 1000); radius (spheres) or three half-extents
 * (boxes), each uniform in [r_min, r_max] or, with log_uniform, floor of
 * exp(u * ln(r_max + 1)) clamped to [r_min, r_max]; material uniform in
 * [material_min, material_max] for adds, 0 for removes. */
typedef struct vx_edit_mix {
    uint32_t world_exp;
    uint32_t sphere_permille;
    uint32_t add_permille;
    uint32_t r_min;
    uint32_t r_max;
    uint32_t log_uniform;
    uint32_t material_min;
    uint32_t material_max;
} vx_edit_mix;

#include <math.h>
#include <stdlib.h>

static inline double vx_pcg32_unit(vx_pcg32 *rng) {
    return (double)vx_pcg32_next(rng) * (1.0 / 4294967296.0);
}

static inline uint32_t vx_draw_radius(vx_pcg32 *rng, const vx_edit_mix *m) {
    if (!m->log_uniform)
        return m->r_min + vx_pcg32_bounded(rng, m->r_max - m->r_min + 1u);
    double r = floor(exp(vx_pcg32_unit(rng) * log((double)m->r_max + 1.0)));
    if (r < (double)m->r_min) r = (double)m->r_min;
    if (r > (double)m->r_max) r = (double)m->r_max;
    return (uint32_t)r;
}

static inline void vx_generate_primitives_host(const vx_edit_mix *m, uint64_t seed,
                                               uint64_t stream, uint64_t count,
                                               vx_primitive *out) {
    vx_pcg32 rng;
    vx_pcg32_seed(&rng, seed, stream);
    const uint32_t world = 4u << (m->world_exp - 2u);
    for (uint64_t i = 0; i < count; ++i) {
        vx_primitive p;
        p.c[0] = (int32_t)vx_pcg32_bounded(&rng, world);
        p.c[1] = (int32_t)vx_pcg32_bounded(&rng, world);
        p.c[2] = (int32_t)vx_pcg32_bounded(&rng, world);
        const uint32_t shape =
            vx_pcg32_bounded(&rng, 1000u) < m->sphere_permille ? VX_SHAPE_SPHERE : VX_SHAPE_BOX;
        const uint32_t op = vx_pcg32_bounded(&rng, 1000u) < m->add_permille ? VX_OP_ADD : VX_OP_REMOVE;
        p.r[0] = vx_draw_radius(&rng, m);
        if (shape == VX_SHAPE_BOX) {
            p.r[1] = vx_draw_radius(&rng, m);
            p.r[2] = vx_draw_radius(&rng, m);
        } else {
            p.r[1] = p.r[2] = 0u;
        }
        uint32_t mat = m->material_min +
                       vx_pcg32_bounded(&rng, m->material_max - m->material_min + 1u);
        if (op == VX_OP_REMOVE) mat = 0u;
        p.flags = vx_make_flags(shape, op, mat);
        p.reserved = 0u;
        out[i] = p;
    }
}

/* ------------------------------------------------------- request stream --
 * Host-only: a served edit stream.  Arrivals are a Poisson process of `rate`
 * requests per second (exponential gaps, u = (next + 0.5) / 2^32), request
 * sizes follow Zipf(s) over [1, max_size] (inverse CDF over the exact
 * normalised weights k^-s), and each request's primitives come from `mix`
 * (same per-primitive draw order as vx_generate_primitives_host).  One PCG32
 * stream serves arrivals and sizes; primitives use a second stream. */
static inline uint64_t vx_generate_requests_host(
    const vx_edit_mix *mix, uint64_t seed, double rate, double seconds,
    double zipf_s, uint32_t max_size, uint64_t max_requests,
    uint64_t *arrival_ns, uint32_t *sizes, uint64_t max_prims, vx_primitive *prims,
    uint64_t *total_prims) {
    vx_pcg32 rng;
    vx_pcg32_seed(&rng, seed, 11u);
    double *cdf = (double *)malloc(sizeof(double) * (max_size ? max_size : 1u));
    if (cdf == NULL) return 0;
    double norm = 0.0;
    for (uint32_t k = 1; k <= max_size; ++k) {
        norm += pow((double)k, -zipf_s);
        cdf[k - 1] = norm;
    }
    double t = 0.0;
    uint64_t n = 0, np = 0;
    while (n < max_requests) {
        const double u = ((double)vx_pcg32_next(&rng) + 0.5) * (1.0 / 4294967296.0);
        t += -log(u) / rate;
        if (t >= seconds) break;
        const double v = ((double)vx_pcg32_next(&rng) + 0.5) * (1.0 / 4294967296.0) * norm;
        uint32_t lo = 0, hi = max_size - 1u; /* first k with cdf[k - 1] >= v */
        while (lo < hi) {
            const uint32_t mid = (lo + hi) / 2u;
            if (cdf[mid] >= v) hi = mid;
            else lo = mid + 1u;
        }
        const uint32_t k = lo + 1u;
        if (arrival_ns) arrival_ns[n] = (uint64_t)(t * 1e9);
        if (sizes) sizes[n] = k;
        np += k;
        ++n;
    }
    free(cdf);
    if (total_prims) *total_prims = np;
    if (prims && np <= max_prims) vx_generate_primitives_host(mix, seed, 12u, np, prims);
    return n;
}

#ifdef __cplusplus
}
#endif

#undef VX_HD
#endif /* VX_WORKLOAD_H */
