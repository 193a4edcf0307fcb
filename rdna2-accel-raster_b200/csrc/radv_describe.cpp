// radv_describe.cpp — text description of a RADV acceleration-structure image
// (rq_radv_describe): the header fields, the root Box32 node's four children
// and, when child 0 is a triangle, that triangle node.  The text is the one
// the reference's decoder prints (dump_bvh_structure,
// include/radv_bvh.hpp:311-390), line for line, so images can be compared
// with the reference's own tool; numbers are formatted as an ostream does by
// default (floats %g with 6 significant digits, hex without leading zeros).
#include <cinttypes>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/rq.h"

namespace {

struct Text {
    std::string s;
    void put(const char* fmt, ...) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        const int n = vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        if (n > 0) s.append(buf, size_t(n) < sizeof(buf) ? size_t(n) : sizeof(buf) - 1);
    }
};

const char* type_name(uint32_t t) {
    switch (t) {
        case RQ_RADV_NODE_TRIANGLE: return "Triangle (0)";
        case RQ_RADV_NODE_BOX16: return "Box16 (4)";
        case RQ_RADV_NODE_BOX32: return "Box32 (5)";
        case RQ_RADV_NODE_INSTANCE: return "Instance (6)";
        case RQ_RADV_NODE_AABB: return "AABB (7)";
        default: return "Unknown";
    }
}

const char* kRule = "================================================================================\n";

void describe(const uint8_t* raw, uint64_t bytes, Text& o) {
    if (bytes < sizeof(rq_radv_header)) {
        o.put("[ERROR] Buffer too small for RADV AS header\n");
        return;
    }
    rq_radv_header h;
    std::memcpy(&h, raw, sizeof(h));
    o.put("%s", kRule);
    o.put("           RDNA2 RADV ACCELERATION STRUCTURE LAYOUT DECODER                    \n");
    o.put("%s", kRule);
    o.put("Header Breakdown:\n");
    o.put("  [+0x00] bvh_offset:                0x%x (%u bytes)\n", h.bvh_offset, h.bvh_offset);
    o.put("  [+0x04] root_flags:                0x%x\n", h.root_flags);
    o.put("  [+0x08] AABB Min:                  (%g, %g, %g)\n", h.aabb_min[0], h.aabb_min[1], h.aabb_min[2]);
    o.put("  [+0x14] AABB Max:                  (%g, %g, %g)\n", h.aabb_max[0], h.aabb_max[1], h.aabb_max[2]);
    o.put("  [+0x20] update_dispatch_size:      [%u, %u, %u]\n", h.update_dispatch_size[0],
          h.update_dispatch_size[1], h.update_dispatch_size[2]);
    o.put("  [+0x30] compacted_size:            %" PRIu64 " bytes\n", h.compacted_size);
    o.put("  [+0x38] serialization_size:        %" PRIu64 " bytes\n", h.serialization_size);
    o.put("  [+0x40] copy_dispatch_size:        [%u, %u, %u]\n", h.copy_dispatch_size[0], h.copy_dispatch_size[1],
          h.copy_dispatch_size[2]);
    o.put("  [+0x50] base size:                 %" PRIu64 " bytes\n", h.size);
    o.put("  [+0x58] geometry_type:             %u (0 = Triangles)\n", h.geometry_type);
    o.put("  [+0x5C] geometry_count:            %u\n", h.geometry_count);
    o.put("  [+0x60] leaf_nodes_offset:         0x%" PRIx64 " (%" PRIu64 " bytes)\n", h.leaf_nodes_offset,
          h.leaf_nodes_offset);
    o.put("  [+0x68] primitive_count:           %" PRIu64 "\n", h.primitive_count);
    o.put("  [+0x70] instance_count:            %" PRIu64 "\n", h.instance_count);
    o.put("  [+0x78] leaf_node_offsets_offset:  0x%x\n", h.leaf_node_offsets_offset);
    o.put("  [+0x7C] build_flags:               0x%x\n", h.build_flags);
    o.put("  [+0x80] type:                      %u (0 = BLAS, 1 = TLAS)\n", h.type);

    const uint32_t root = h.bvh_offset;
    if (uint64_t(root) + sizeof(rq_radv_box32) > bytes) {
        o.put("[ERROR] BVH offset 0x%x exceeds buffer size\n", root);
        return;
    }
    rq_radv_box32 box;
    std::memcpy(&box, raw + root, sizeof(box));
    o.put("\nRoot Box4 Node Breakdown (Offset: 0x%x):\n", root);
    for (int i = 0; i < 4; ++i) {
        const uint32_t c = box.children[i];
        o.put("  Child [%d]: raw = 0x%x", i, c);
        if (c == RQ_RADV_INVALID_NODE) {
            o.put(" [INVALID / EMPTY]\n");
            continue;
        }
        const uint32_t rel = (c & ~7u) << 3, type = c & 7u, abs_off = root + rel;
        o.put(" -> RelOffset = 0x%x (Abs = 0x%x), Type = %s\n", rel, abs_off, type_name(type));
        o.put("           AABB Min: (%g, %g, %g)\n", box.coords[i][0], box.coords[i][1], box.coords[i][2]);
        o.put("           AABB Max: (%g, %g, %g)\n", box.coords[i][3], box.coords[i][4], box.coords[i][5]);
    }
    o.put("  Flags:                             0x%x\n", box.flags);
    const uint32_t c0 = box.children[0];
    if (c0 != RQ_RADV_INVALID_NODE && (c0 & 7u) == RQ_RADV_NODE_TRIANGLE) {
        const uint32_t at = root + ((c0 & ~7u) << 3);
        if (uint64_t(at) + sizeof(rq_radv_tri) <= bytes) {
            rq_radv_tri t;
            std::memcpy(&t, raw + at, sizeof(t));
            o.put("\nTriangle Node Breakdown (Offset: 0x%x):\n", at);
            for (int v = 0; v < 3; ++v)
                o.put("  Vertex V%d:                         (%g, %g, %g)\n", v, t.coords[v][0], t.coords[v][1],
                      t.coords[v][2]);
            o.put("  Primitive Index (triangle_id):     %u\n", t.triangle_id);
            o.put("  Geometry Flags:                    0x%x (Opaque: %s)\n", t.geometry_id_and_flags,
                  (t.geometry_id_and_flags & RQ_RADV_GEOMETRY_OPAQUE) ? "YES" : "NO");
            o.put("  Barycentrics Control (id):         0x%x (%u)\n", t.id, t.id);
        }
    }
    o.put("%s", kRule);
}

}  // namespace

extern "C" int rq_radv_describe(const void* image, uint64_t bytes, char* text, uint64_t capacity, uint64_t* length) {
    if (!image || !length || (capacity && !text)) return RQ_ERR_INVALID_ARG;
    Text o;
    describe(static_cast<const uint8_t*>(image), bytes, o);
    *length = o.s.size();
    if (!capacity) return RQ_OK;
    const uint64_t n = o.s.size() < capacity ? o.s.size() : capacity - 1;
    std::memcpy(text, o.s.data(), n);
    text[n] = '\0';
    return o.s.size() < capacity ? RQ_OK : RQ_ERR_SIZE;
}
