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
#include <algorithm>
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

// Right-handed look-at view and a Vulkan-style perspective (depth 0..1, y
// flipped), combined and inverted in double precision, stored column-major.
extern "C" int rq_camera_look_at(const float eye[3], const float target[3], const float up[3], float fovy_deg,
                                 uint32_t width, uint32_t height, rq_camera* out) {
    if (!eye || !target || !up || !out || width == 0 || height == 0 || !(fovy_deg > 0.0f && fovy_deg < 180.0f))
        return RQ_ERR_INVALID_ARG;
    double e[3] = {eye[0], eye[1], eye[2]}, t[3] = {target[0], target[1], target[2]}, u0[3] = {up[0], up[1], up[2]};
    auto norm = [](double* v) {
        double l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        v[0] /= l;
        v[1] /= l;
        v[2] /= l;
    };
    auto cross = [](const double* a, const double* b, double* o) {
        o[0] = a[1] * b[2] - a[2] * b[1];
        o[1] = a[2] * b[0] - a[0] * b[2];
        o[2] = a[0] * b[1] - a[1] * b[0];
    };
    double f[3] = {t[0] - e[0], t[1] - e[1], t[2] - e[2]};
    norm(f);
    double sx[3], ux[3];
    cross(f, u0, sx);
    norm(sx);
    cross(sx, f, ux);
    // view (column-major M[col][row])
    double V[4][4] = {{sx[0], ux[0], -f[0], 0}, {sx[1], ux[1], -f[1], 0}, {sx[2], ux[2], -f[2], 0},
                      {-(sx[0] * e[0] + sx[1] * e[1] + sx[2] * e[2]), -(ux[0] * e[0] + ux[1] * e[1] + ux[2] * e[2]),
                       f[0] * e[0] + f[1] * e[1] + f[2] * e[2], 1}};
    const double aspect = double(width) / double(height);
    const double th = std::tan(double(fovy_deg) * 3.14159265358979323846 / 360.0);
    const double zn = 0.1, zf = 100.0;
    double Pm[4][4] = {{1.0 / (aspect * th), 0, 0, 0},
                       {0, -1.0 / th, 0, 0},
                       {0, 0, zf / (zn - zf), -1},
                       {0, 0, -(zf * zn) / (zf - zn), 0}};
    // VP = P * V  (column-major: VP[c][r] = sum_k P[k][r] * V[c][k])
    double A[4][8];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            double acc = 0;
            for (int k = 0; k < 4; ++k) acc += Pm[k][r] * V[c][k];
            A[r][c] = acc;  // row-major copy for the inversion
            A[r][4 + c] = r == c ? 1.0 : 0.0;
        }
    for (int col = 0; col < 4; ++col) {
        int piv = col;
        for (int r = col + 1; r < 4; ++r)
            if (std::fabs(A[r][col]) > std::fabs(A[piv][col])) piv = r;
        if (std::fabs(A[piv][col]) < 1e-300) return RQ_ERR_INVALID_ARG;
        if (piv != col)
            for (int k = 0; k < 8; ++k) std::swap(A[piv][k], A[col][k]);
        const double d = A[col][col];
        for (int k = 0; k < 8; ++k) A[col][k] /= d;
        for (int r = 0; r < 4; ++r)
            if (r != col) {
                const double m = A[r][col];
                for (int k = 0; k < 8; ++k) A[r][k] -= m * A[col][k];
            }
    }
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) out->inv_view_proj[4 * c + r] = float(A[r][4 + c]);
    out->cam_pos[0] = eye[0];
    out->cam_pos[1] = eye[1];
    out->cam_pos[2] = eye[2];
    out->width = width;
    out->height = height;
    out->jitter = 0;
    out->seed = 0;
    out->tmin = 0.01f;
    out->tmax = 10000.0f;
    out->flags = 0;
    return RQ_OK;
}
