/*
 * rq_layouts.h — byte layouts shared by the ray-query engine, its callers and
 * its oracle.  Every struct here is a byte-for-byte stand-in for a layout that
 * the reference's BVH path writes or reads, so buffers can be handed across
 * unchanged.  Each struct cites the reference definition it must match.
 *
 * Plain C11/C++ header: no CUDA, no torch.
 */
#ifndef RQ_LAYOUTS_H
#define RQ_LAYOUTS_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__cplusplus)
#define RQ_ALIGN16 alignas(16)
#else
#define RQ_ALIGN16 _Alignas(16)
#endif

/* Binary BVH node, 32 B.  Same bytes as GpuBvhNode (common/software_bvh.hpp:11-16).
 * Inner node: left_child >= 0 is the left child index, right_child the right
 * child index.  Leaf: left_child = ~first_prim (bitwise NOT, so < 0) and
 * right_child = primitive count.  The root is node 0. */
typedef struct rq_bvh2_node {
    RQ_ALIGN16 float aabb_min[3];
    int32_t left_child;
    float aabb_max[3];
    int32_t right_child;
} rq_bvh2_node;

/* Leaf-ordered triangle, 48 B.  Same bytes as GpuTriangle
 * (common/software_bvh.hpp:18-22); the w lanes are written as 0.0f. */
typedef struct rq_triangle {
    RQ_ALIGN16 float v0[4];
    float v1[4];
    float v2[4];
} rq_triangle;

/* Four-wide BVH node in SoA form, 128 B.  Same bytes as GpuBvh4Node
 * (common/software_bvh.hpp:178-187).  child_count[k]: 0 = empty slot,
 * -1 = inner node (child_index[k] = node index), >0 = leaf with that many
 * primitives starting at ~child_index[k]. */
typedef struct rq_bvh4_node {
    RQ_ALIGN16 float min_x[4];
    float max_x[4];
    float min_y[4];
    float max_y[4];
    float min_z[4];
    float max_z[4];
    int32_t child_index[4];
    int32_t child_count[4];
} rq_bvh4_node;

/* ---- RADV acceleration-structure image (include/radv_bvh.hpp:22-215) ---- */

#define RQ_RADV_NODE_TRIANGLE 0u
#define RQ_RADV_NODE_BOX16 4u
#define RQ_RADV_NODE_BOX32 5u
#define RQ_RADV_NODE_INSTANCE 6u
#define RQ_RADV_NODE_AABB 7u
#define RQ_RADV_INVALID_NODE 0xffffffffu
#define RQ_RADV_GEOMETRY_OPAQUE 0x80000000u
#define RQ_RADV_BARYCENTRICS_CONTROL_DEFAULT 9u
#define RQ_RADV_BVH_OFFSET 192u /* root Box32 node sits at byte 0xC0 */

/* 136-B header at byte 0 of the image (radv_bvh.hpp:80-103). */
#pragma pack(push, 4)
typedef struct rq_radv_header {
    uint32_t bvh_offset;
    uint32_t root_flags;
    float aabb_min[3];
    float aabb_max[3];
    uint32_t update_dispatch_size[3];
    uint32_t padding0;
    uint64_t compacted_size;
    uint64_t serialization_size;
    uint32_t copy_dispatch_size[3];
    uint32_t padding1;
    uint64_t size;
    uint32_t geometry_type;
    uint32_t geometry_count;
    uint64_t leaf_nodes_offset;
    uint64_t primitive_count;
    uint64_t instance_count;
    uint32_t leaf_node_offsets_offset;
    uint32_t build_flags;
    uint32_t type;
    uint32_t padding2;
} rq_radv_header;

/* 128-B Box32 node (radv_bvh.hpp:128-133): children[k] = (offset from the
 * root node >> 3) | type, or RQ_RADV_INVALID_NODE with a quiet-NaN box. */
typedef struct rq_radv_box32 {
    uint32_t children[4];
    float coords[4][6]; /* per child: min xyz, max xyz */
    uint32_t flags;
    uint32_t reserved[3];
} rq_radv_box32;

/* 64-B triangle node (radv_bvh.hpp:143-150). */
typedef struct rq_radv_tri {
    float coords[3][3];
    uint32_t reserved[3];
    uint32_t triangle_id;
    uint32_t geometry_id_and_flags;
    uint32_t reserved2;
    uint32_t id;
} rq_radv_tri;
#pragma pack(pop)

/* Level plan of the implicit 4-ary tree (radv_bvh.hpp:158-215). */
typedef struct rq_radv_layout {
    uint32_t num_triangles;
    uint32_t total_boxes;
    uint32_t num_levels; /* <= 16 */
    uint32_t total_as_size_lo; /* low 32 bits, as the reference's uint32 field */
    uint64_t total_as_size; /* full size in bytes */
    uint32_t level_offsets[16]; /* root level first */
    uint32_t level_counts[16];
} rq_radv_layout;

/* ---- Rays and hits ---- */

/* 32-B ray: same bytes as RayInput (benchmarks/exp0_probe/shaders/software_bvh.comp:5-8):
 * origin.xyz, tmin, direction.xyz, tmax. */
typedef struct rq_ray {
    RQ_ALIGN16 float org[3];
    float tmin;
    float dir[3];
    float tmax;
} rq_ray;

/* 16-B hit: same bytes as HitResult (software_bvh.comp:10-15,
 * probe_triangle.comp:8-13).  A miss is {0, -1.0f, 0xffffffff, 0xffffffff}. */
typedef struct rq_hit {
    RQ_ALIGN16 uint32_t hit;
    float t;
    uint32_t instance_id;
    uint32_t primitive_id;
} rq_hit;

/* 16-B per-ray statistics: same bytes as RayStats
 * (software_bvh_bvh4.comp:30-35). */
typedef struct rq_ray_stats {
    uint32_t hit;
    uint32_t box_tests;
    uint32_t tri_tests;
    uint32_t pad;
} rq_ray_stats;

#ifdef __cplusplus
} /* extern "C" */
static_assert(sizeof(rq_bvh2_node) == 32, "rq_bvh2_node must be 32 bytes");
static_assert(sizeof(rq_triangle) == 48, "rq_triangle must be 48 bytes");
static_assert(sizeof(rq_bvh4_node) == 128, "rq_bvh4_node must be 128 bytes");
static_assert(sizeof(rq_radv_header) == 136, "rq_radv_header must be 136 bytes");
static_assert(offsetof(rq_radv_header, compacted_size) == 0x30, "header layout");
static_assert(offsetof(rq_radv_header, size) == 0x50, "header layout");
static_assert(offsetof(rq_radv_header, leaf_nodes_offset) == 0x60, "header layout");
static_assert(offsetof(rq_radv_header, build_flags) == 0x7C, "header layout");
static_assert(offsetof(rq_radv_header, type) == 0x80, "header layout");
static_assert(sizeof(rq_radv_box32) == 128, "rq_radv_box32 must be 128 bytes");
static_assert(sizeof(rq_radv_tri) == 64, "rq_radv_tri must be 64 bytes");
static_assert(sizeof(rq_ray) == 32, "rq_ray must be 32 bytes");
static_assert(sizeof(rq_hit) == 16, "rq_hit must be 16 bytes");
static_assert(sizeof(rq_ray_stats) == 16, "rq_ray_stats must be 16 bytes");
#endif

#endif /* RQ_LAYOUTS_H */
