// scene.cpp — host-side generation of the height-field grid meshes that feed
// the BVH path (the input role of MeshGenerator::createTessellatedTerrain,
// common/mesh_gen.hpp:29-83, and rdna2::generate_dynamic_grid_mesh,
// include/radv_bvh.hpp:224-283).
//
// Vertices sit on a (qx+1) x (qy+1) lattice over [x0,x1] x [y0,y1] with
// z = amp*sin(freq*x)*cos(freq*y) + N(0, sigma).  The normal jitter comes
// from SplitMix64 (seeded) through Box-Muller, all in double precision and
// rounded to float once per coordinate.  Each quad (i, j) contributes the two
// triangles (v00, v10, v01) and (v10, v11, v01), quads in row-major order.
#include <cmath>
#include <cstdint>

#include "../../include/rq.h"

namespace {

struct SplitMix64 {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    // uniform in (0, 1]
    double uniform() { return double((next() >> 11) + 1) * (1.0 / 9007199254740992.0); }
};

}  // namespace

extern "C" int rq_scene_grid(uint32_t qx, uint32_t qy, float x0, float x1, float y0, float y1, float amp, float freq,
                             float sigma, uint64_t seed, float* pos, uint32_t* idx) {
    if (qx == 0 || qy == 0 || (!pos && !idx)) return RQ_ERR_INVALID_ARG;
    if (uint64_t(qx + 1) * uint64_t(qy + 1) >= (1ull << 32)) return RQ_ERR_UNSUPPORTED;
    const uint32_t nvx = qx + 1, nvy = qy + 1;
    if (pos) {
        SplitMix64 rng{seed};
        const double two_pi = 6.283185307179586476925286766559;
        double spare = 0.0;
        bool have_spare = false;
        for (uint32_t j = 0; j < nvy; ++j) {
            const double y = double(y0) + (double(y1) - double(y0)) * double(j) / double(qy);
            for (uint32_t i = 0; i < nvx; ++i) {
                const double x = double(x0) + (double(x1) - double(x0)) * double(i) / double(qx);
                double g;
                if (have_spare) {
                    g = spare;
                    have_spare = false;
                } else {
                    double u1 = rng.uniform(), u2 = rng.uniform();
                    double r = std::sqrt(-2.0 * std::log(u1));
                    g = r * std::cos(two_pi * u2);
                    spare = r * std::sin(two_pi * u2);
                    have_spare = true;
                }
                const double z = double(amp) * std::sin(double(freq) * x) * std::cos(double(freq) * y) +
                                  double(sigma) * g;
                float* p = pos + 3ull * (size_t(j) * nvx + i);
                p[0] = float(x);
                p[1] = float(y);
                p[2] = float(z);
            }
        }
    }
    if (idx) {
        uint32_t* o = idx;
        for (uint32_t j = 0; j < qy; ++j)
            for (uint32_t i = 0; i < qx; ++i) {
                const uint32_t v00 = j * nvx + i, v10 = v00 + 1, v01 = v00 + nvx, v11 = v01 + 1;
                o[0] = v00;
                o[1] = v10;
                o[2] = v01;
                o[3] = v10;
                o[4] = v11;
                o[5] = v01;
                o += 6;
            }
    }
    return RQ_OK;
}

extern "C" int rq_scene_rays_down(uint32_t n, float x0, float x1, float y0, float y1, float z, float spread,
                                  float tmin, float tmax, uint64_t seed, rq_ray* rays) {
    if (!rays && n) return RQ_ERR_INVALID_ARG;
    SplitMix64 rng{seed};
    for (uint32_t i = 0; i < n; ++i) {
        double ox = double(x0) + (double(x1) - double(x0)) * rng.uniform();
        double oy = double(y0) + (double(y1) - double(y0)) * rng.uniform();
        double dx = double(spread) * (2.0 * rng.uniform() - 1.0);
        double dy = double(spread) * (2.0 * rng.uniform() - 1.0);
        double dz = -1.0;
        double len = std::sqrt(dx * dx + dy * dy + dz * dz);
        rq_ray& r = rays[i];
        r.org[0] = float(ox);
        r.org[1] = float(oy);
        r.org[2] = z;
        r.tmin = tmin;
        r.dir[0] = float(dx / len);
        r.dir[1] = float(dy / len);
        r.dir[2] = float(dz / len);
        r.tmax = tmax;
    }
    return RQ_OK;
}
