// rq_software_bvh.hpp — C++ host wrapper over librq's C ABI that keeps the
// call shape of the reference's CPU builder:
//
//   SoftwareBVH  bvh  = SoftwareBVH::build(mesh, maxPrimsPerLeaf);   // common/software_bvh.hpp:35
//   SoftwareBVH4 bvh4 = SoftwareBVH4::fromBVH2(bvh);                // common/software_bvh.hpp:193
//
// compiles unchanged against this header with `rq::` in front (or a
// `using namespace rq;`): those two calls run on the calling thread's default
// engine, created on the current CUDA device at its first use.  A caller that
// wants to choose the device or hold the context passes an engine:
//
//   rq::Engine eng;                                   // one context per device / thread
//   rq::SoftwareBVH  bvh  = rq::SoftwareBVH::build(eng, mesh, maxPrimsPerLeaf);
//   rq::SoftwareBVH4 bvh4 = rq::SoftwareBVH4::fromBVH2(eng, bvh);
//
// The mesh type is any type with `vertices[i].pos[3]` floats and a
// `std::vector<uint32_t> indices` (the reference's SceneMesh qualifies).
// nodes / triangles come back in the byte layouts of GpuBvhNode, GpuTriangle
// and GpuBvh4Node (rq_layouts.h), so they upload unchanged to the reference's
// traversal shaders.  Unlike the reference, `perm` keeps the leaf-order ->
// original triangle id map.  Errors throw rq::Error (C++ side only; the C ABI
// itself never throws).
//
// The default tree is an LBVH (Morton order).  Split::Median builds the
// reference's own median-split topology (RQ_BUILD_MEDIAN): where no centroid
// value repeats on an axis its nodes equal SoftwareBVH::build's byte for byte.
#pragma once

#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "rq.h"

namespace rq {

struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& what) : std::runtime_error(what), status(s) {}
};

inline void check(int status, rq_ctx* ctx, const char* what) {
    if (status != RQ_OK)
        throw Error(status, std::string(what) + ": " + rq_status_string(status) + " " +
                                (ctx ? rq_ctx_last_error(ctx) : ""));
}

// Owns an rq_ctx on one device.
class Engine {
   public:
    explicit Engine(int device = 0) { check(rq_ctx_create(device, &ctx_), nullptr, "rq_ctx_create"); }
    ~Engine() {
        if (ctx_) rq_ctx_destroy(ctx_);
    }
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;
    rq_ctx* get() const { return ctx_; }

   private:
    rq_ctx* ctx_ = nullptr;
};

// The engine of the reference-shaped calls (no Engine argument): one per
// thread, on the CUDA device current at its first use.  It lives until the
// process exits (it is not destroyed at thread exit, when the CUDA runtime
// may already be shutting down); its device memory goes with the process.
inline Engine& default_engine() {
    thread_local Engine* eng = nullptr;
    if (!eng) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
        eng = new Engine(dev);
    }
    return *eng;
}

enum class Split { Morton, Median };

struct SoftwareBVH {
    std::vector<rq_bvh2_node> nodes;
    std::vector<rq_triangle> triangles;
    std::vector<uint32_t> perm;  // leaf order -> original triangle id

    // SoftwareBVH::build(mesh, maxPrimsPerLeaf) (common/software_bvh.hpp:35),
    // on the calling thread's default engine.
    template <class Mesh>
    static SoftwareBVH build(const Mesh& mesh, uint32_t maxPrimsPerLeaf = 4) {
        return build(default_engine(), mesh, maxPrimsPerLeaf, Split::Morton);
    }

    template <class Mesh>
    static SoftwareBVH build(Engine& eng, const Mesh& mesh, uint32_t maxPrimsPerLeaf = 4,
                             Split split = Split::Morton) {
        const size_t nv = mesh.vertices.size();
        const uint32_t nt = uint32_t(mesh.indices.size() / 3);
        if (nt == 0) {
            // what the reference returns for an empty mesh: one leaf of no
            // triangles over an empty box (common/software_bvh.hpp:101-124)
            SoftwareBVH out;
            rq_bvh2_node leaf{};
            for (int c = 0; c < 3; ++c) {
                leaf.aabb_min[c] = FLT_MAX;
                leaf.aabb_max[c] = -FLT_MAX;
            }
            leaf.left_child = ~0;
            leaf.right_child = 0;
            out.nodes.push_back(leaf);
            return out;
        }
        std::vector<float> pos(3 * nv);
        for (size_t v = 0; v < nv; ++v)
            for (int c = 0; c < 3; ++c) pos[3 * v + c] = mesh.vertices[v].pos[c];
        float* d_pos = nullptr;
        uint32_t* d_idx = nullptr;
        auto fail = [&](cudaError_t e) {
            if (e != cudaSuccess) {
                cudaFree(d_pos);
                cudaFree(d_idx);
                throw Error(RQ_ERR_CUDA, cudaGetErrorString(e));
            }
        };
        fail(cudaMalloc(&d_pos, pos.size() * sizeof(float)));
        fail(cudaMalloc(&d_idx, mesh.indices.size() * sizeof(uint32_t)));
        fail(cudaMemcpy(d_pos, pos.data(), pos.size() * sizeof(float), cudaMemcpyHostToDevice));
        fail(cudaMemcpy(d_idx, mesh.indices.data(), mesh.indices.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
        rq_bvh* h = nullptr;
        const uint32_t flags = split == Split::Median ? RQ_BUILD_MEDIAN : 0u;
        int st = rq_build(eng.get(), d_pos, 12, uint32_t(nv), d_idx, nt, maxPrimsPerLeaf, flags, &h, nullptr);
        cudaFree(d_pos);
        cudaFree(d_idx);
        check(st, eng.get(), "rq_build");
        SoftwareBVH out;
        rq_bvh_info info;
        st = rq_bvh_info_get(h, &info);
        if (st == RQ_OK) {
            out.nodes.resize(info.num_nodes2);
            out.triangles.resize(nt);
            out.perm.resize(nt);
            st = rq_bvh_download(h, 1, out.nodes.data(), info.num_nodes2, out.triangles.data(), nt, nullptr, 0,
                                 out.perm.data(), nt);
        }
        rq_bvh_destroy(h);
        check(st, eng.get(), "rq_bvh_download");
        return out;
    }
};

struct SoftwareBVH4 {
    std::vector<rq_bvh4_node> nodes;
    std::vector<rq_triangle> triangles;

    // SoftwareBVH4::fromBVH2(bvh) (common/software_bvh.hpp:193), on the
    // calling thread's default engine.
    static SoftwareBVH4 fromBVH2(const SoftwareBVH& b2) { return fromBVH2(default_engine(), b2); }

    static SoftwareBVH4 fromBVH2(Engine& eng, const SoftwareBVH& b2) {
        SoftwareBVH4 out;
        out.triangles = b2.triangles;
        if (b2.nodes.empty()) return out;
        if (b2.triangles.empty()) {
            // a single leaf of no triangles: slot 0 carries its box and
            // encoded child as written (common/software_bvh.hpp:204-218)
            const rq_bvh2_node& leaf = b2.nodes[0];
            rq_bvh4_node n4{};
            n4.min_x[0] = leaf.aabb_min[0];
            n4.max_x[0] = leaf.aabb_max[0];
            n4.min_y[0] = leaf.aabb_min[1];
            n4.max_y[0] = leaf.aabb_max[1];
            n4.min_z[0] = leaf.aabb_min[2];
            n4.max_z[0] = leaf.aabb_max[2];
            n4.child_index[0] = leaf.left_child;
            n4.child_count[0] = leaf.right_child;
            out.nodes.push_back(n4);
            return out;
        }
        rq_bvh2_node* d_n = nullptr;
        rq_triangle* d_t = nullptr;
        cudaError_t e = cudaMalloc(&d_n, b2.nodes.size() * sizeof(rq_bvh2_node));
        if (e == cudaSuccess) e = cudaMalloc(&d_t, b2.triangles.size() * sizeof(rq_triangle));
        if (e == cudaSuccess)
            e = cudaMemcpy(d_n, b2.nodes.data(), b2.nodes.size() * sizeof(rq_bvh2_node), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(d_t, b2.triangles.data(), b2.triangles.size() * sizeof(rq_triangle),
                           cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(d_n);
            cudaFree(d_t);
            throw Error(RQ_ERR_CUDA, cudaGetErrorString(e));
        }
        rq_bvh* h = nullptr;
        int st = rq_bvh_import2(eng.get(), d_n, uint32_t(b2.nodes.size()), d_t, nullptr,
                                uint32_t(b2.triangles.size()), &h, nullptr);
        cudaFree(d_n);
        cudaFree(d_t);
        check(st, eng.get(), "rq_bvh_import2");
        st = rq_collapse4(eng.get(), h, nullptr);
        rq_bvh_info info;
        if (st == RQ_OK) st = rq_bvh_info_get(h, &info);
        if (st == RQ_OK) {
            out.nodes.resize(info.num_nodes4);
            st = rq_bvh_download(h, 1, nullptr, 0, nullptr, 0, out.nodes.data(), info.num_nodes4, nullptr, 0);
        }
        rq_bvh_destroy(h);
        check(st, eng.get(), "rq_collapse4");
        return out;
    }
};

}  // namespace rq
