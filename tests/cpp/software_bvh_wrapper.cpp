// Test driver for include/rq_software_bvh.hpp, the C++ wrapper that keeps the
// call shape of the reference's SoftwareBVH::build / SoftwareBVH4::fromBVH2
// (common/software_bvh.hpp:35, 193).  It reads an indexed mesh, builds through
// the wrapper exactly as a reference call site would, and writes the bytes the
// reference would upload:
//
//   software_bvh_wrapper MESH OUT_PREFIX MAX_LEAF SPLIT(0 morton, 1 median,
//                                                    2 the reference's call shape)
//
// SPLIT 2 calls rq::SoftwareBVH::build(mesh, maxPrimsPerLeaf) and
// rq::SoftwareBVH4::fromBVH2(bvh) with no engine argument, as
// benchmarks/exp0_probe/microbench_main.cpp:175,185 call the reference.
//
// MESH: uint32 nv, uint32 ni, nv x 3 float32 positions, ni uint32 indices.
// Writes OUT_PREFIX.nodes2 / .tris / .nodes4 / .perm; exit status 0 on
// success, 1 on a wrapper error (the message on stderr).
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "rq_software_bvh.hpp"

namespace {

// The shape of the reference's SceneMesh (common/mesh_gen.hpp:12-19).
struct SceneMesh {
    struct Vertex {
        float pos[3];
        float normal[3];
    };
    std::vector<Vertex> vertices;
    std::vector<uint32_t> indices;
};

bool read_mesh(const char* path, SceneMesh& m) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    uint32_t hdr[2];
    bool ok = std::fread(hdr, sizeof(uint32_t), 2, f) == 2;
    if (ok) {
        m.vertices.resize(hdr[0]);
        m.indices.resize(hdr[1]);
        for (auto& v : m.vertices) {
            ok = ok && std::fread(v.pos, sizeof(float), 3, f) == 3;
            v.normal[0] = v.normal[1] = 0.0f;
            v.normal[2] = 1.0f;
        }
        ok = ok && std::fread(m.indices.data(), sizeof(uint32_t), hdr[1], f) == hdr[1];
    }
    std::fclose(f);
    return ok;
}

template <class T>
bool write_vec(const std::string& path, const std::vector<T>& v) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const bool ok = v.empty() || std::fwrite(v.data(), sizeof(T), v.size(), f) == v.size();
    return std::fclose(f) == 0 && ok;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 5) {
        std::fprintf(stderr, "usage: %s MESH OUT_PREFIX MAX_LEAF SPLIT\n", argv[0]);
        return 2;
    }
    SceneMesh mesh;
    if (!read_mesh(argv[1], mesh)) {
        std::fprintf(stderr, "cannot read %s\n", argv[1]);
        return 2;
    }
    const std::string out = argv[2];
    const uint32_t max_leaf = uint32_t(std::strtoul(argv[3], nullptr, 10));
    const int mode = std::atoi(argv[4]);
    const rq::Split split = mode == 1 ? rq::Split::Median : rq::Split::Morton;
    try {
        rq::SoftwareBVH b2;
        rq::SoftwareBVH4 b4;
        if (mode == 2) {
            b2 = rq::SoftwareBVH::build(mesh, max_leaf);
            b4 = rq::SoftwareBVH4::fromBVH2(b2);
        } else {
            rq::Engine eng(0);
            b2 = rq::SoftwareBVH::build(eng, mesh, max_leaf, split);
            b4 = rq::SoftwareBVH4::fromBVH2(eng, b2);
        }
        const bool ok = write_vec(out + ".nodes2", b2.nodes) && write_vec(out + ".tris", b2.triangles) &&
                        write_vec(out + ".nodes4", b4.nodes) && write_vec(out + ".perm", b2.perm);
        if (!ok) {
            std::fprintf(stderr, "cannot write %s.*\n", out.c_str());
            return 2;
        }
    } catch (const rq::Error& e) {
        std::fprintf(stderr, "rq::Error %d: %s\n", e.status, e.what());
        return 1;
    }
    return 0;
}
