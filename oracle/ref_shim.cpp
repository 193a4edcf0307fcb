// ref_shim.cpp — TEST INFRASTRUCTURE, not product code.
//
// Compiles the reference's own CPU BVH code (common/software_bvh.hpp,
// common/mesh_gen.hpp, include/radv_bvh.hpp — included by path from the
// reference tree, never copied) into oracle/_ref/libref.so and gives it a
// C ABI so the tests and the CPU baseline can call it through ctypes.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU legs load it.

#include "software_bvh.hpp"
#include "radv_bvh.hpp"

#include <cstring>
#include <sstream>
#include <string>
#include <new>

extern "C" {

struct ref_bvh {
    SoftwareBVH bvh2;
    SoftwareBVH4 bvh4;
};

// SoftwareBVH::build (common/software_bvh.hpp:35-87) over an indexed mesh,
// then SoftwareBVH4::fromBVH2 (:193-199).  pos: 3 floats per vertex.
ref_bvh* ref_build(const float* pos, uint32_t num_vertices, const uint32_t* idx,
                   uint32_t num_triangles, uint32_t max_leaf, int collapse4) {
    SceneMesh mesh;
    mesh.vertices.resize(num_vertices);
    for (uint32_t v = 0; v < num_vertices; ++v) {
        for (int c = 0; c < 3; ++c) {
            mesh.vertices[v].pos[c] = pos[3 * v + c];
            mesh.vertices[v].normal[c] = c == 1 ? 1.0f : 0.0f;
        }
    }
    mesh.indices.assign(idx, idx + 3ull * num_triangles);
    ref_bvh* out = new (std::nothrow) ref_bvh();
    if (!out) return nullptr;
    out->bvh2 = SoftwareBVH::build(mesh, max_leaf);
    if (collapse4) out->bvh4 = SoftwareBVH4::fromBVH2(out->bvh2);
    return out;
}

// SoftwareBVH4::fromBVH2 on a caller-provided binary BVH.
ref_bvh* ref_collapse(const void* nodes2, uint32_t num_nodes2, const void* tris, uint32_t num_tris) {
    ref_bvh* out = new (std::nothrow) ref_bvh();
    if (!out) return nullptr;
    out->bvh2.nodes.resize(num_nodes2);
    std::memcpy(out->bvh2.nodes.data(), nodes2, sizeof(GpuBvhNode) * num_nodes2);
    out->bvh2.triangles.resize(num_tris);
    std::memcpy(out->bvh2.triangles.data(), tris, sizeof(GpuTriangle) * num_tris);
    out->bvh4 = SoftwareBVH4::fromBVH2(out->bvh2);
    return out;
}

void ref_counts(const ref_bvh* b, uint32_t* n2, uint32_t* ntri, uint32_t* n4) {
    *n2 = static_cast<uint32_t>(b->bvh2.nodes.size());
    *ntri = static_cast<uint32_t>(b->bvh2.triangles.size());
    *n4 = static_cast<uint32_t>(b->bvh4.nodes.size());
}

void ref_copy(const ref_bvh* b, void* nodes2, void* tris, void* nodes4) {
    if (nodes2) std::memcpy(nodes2, b->bvh2.nodes.data(), sizeof(GpuBvhNode) * b->bvh2.nodes.size());
    if (tris) std::memcpy(tris, b->bvh2.triangles.data(), sizeof(GpuTriangle) * b->bvh2.triangles.size());
    if (nodes4) std::memcpy(nodes4, b->bvh4.nodes.data(), sizeof(GpuBvh4Node) * b->bvh4.nodes.size());
}

void ref_free(ref_bvh* b) { delete b; }

// MeshGenerator::createTessellatedTerrain (common/mesh_gen.hpp:29-83).
// Call once with pos == nullptr to get the counts.
void ref_terrain(uint32_t target, float size, float* pos, uint32_t* idx, uint32_t* nv, uint32_t* ni) {
    SceneMesh m = MeshGenerator::createTessellatedTerrain(target, size);
    *nv = static_cast<uint32_t>(m.vertices.size());
    *ni = static_cast<uint32_t>(m.indices.size());
    if (pos) {
        for (size_t v = 0; v < m.vertices.size(); ++v)
            for (int c = 0; c < 3; ++c) pos[3 * v + c] = m.vertices[v].pos[c];
    }
    if (idx) std::memcpy(idx, m.indices.data(), sizeof(uint32_t) * m.indices.size());
}

// rdna2::compute_tree_layout (include/radv_bvh.hpp:193-215).
// counts/offsets must hold 32 entries.
void ref_tree_layout(uint32_t n, uint32_t* total_boxes, uint32_t* num_levels, uint32_t* total_size,
                     uint32_t* counts, uint32_t* offsets) {
    rdna2::FastBvhTreeLayout l = rdna2::compute_tree_layout(n);
    *total_boxes = l.totalBoxes;
    *num_levels = l.numLevels;
    *total_size = l.totalAsSize;
    for (uint32_t i = 0; i < l.numLevels && i < 32; ++i) {
        counts[i] = l.levelCounts[i];
        offsets[i] = l.levelOffsets[i];
    }
}

// rdna2::generate_dynamic_grid_mesh (include/radv_bvh.hpp:224-283):
// 9 floats per triangle plus the analytic centroids (3 floats each).
void ref_dynamic_grid(uint32_t n, float time_val, float extent, float* tri9, float* centroids) {
    rdna2::DynamicMesh m = rdna2::generate_dynamic_grid_mesh(n, time_val, extent);
    std::memcpy(tri9, m.vertices.data(), sizeof(float) * m.vertices.size());
    for (uint32_t i = 0; i < m.triangleCount; ++i) {
        centroids[3 * i + 0] = m.centroids[i].x;
        centroids[3 * i + 1] = m.centroids[i].y;
        centroids[3 * i + 2] = m.centroids[i].z;
    }
}

// rdna2::dump_bvh_structure (include/radv_bvh.hpp:311-390) into `out`
// (at most cap bytes, NUL-terminated); returns the full text length.
size_t ref_dump_bvh_structure(const void* image, size_t bytes, char* out, size_t cap) {
    std::ostringstream s;
    rdna2::dump_bvh_structure(image, bytes, s);
    const std::string t = s.str();
    if (cap) {
        const size_t n = t.size() < cap ? t.size() : cap - 1;
        std::memcpy(out, t.data(), n);
        out[n] = '\0';
    }
    return t.size();
}

} // extern "C"
