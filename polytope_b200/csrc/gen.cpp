// gen.cpp -- deterministic synthetic workloads (the reference ships only a UV-sphere tessellator,
// src/cpu/shapes/tesselators.cpp:10-84; the workloads here need an icosphere, value noise and
// seeded ray sets, defined once in this file and fed identically to the oracle and the GPU).
//
// All arithmetic is double precision with correctly rounded operations (+ - * / sqrt), rounded to
// float at the end, so the outputs are the same on every IEEE-754 host.

#include <cmath>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "pt_internal.h"

namespace {

inline uint64_t mix64(uint64_t z) {  // splitmix64 finalizer (Steele, Lea, Flood 2014)
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline double unit(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }  // [0, 1)

// Lattice value in [-1, 1] at integer point (i, j, k).
inline double lattice(int64_t i, int64_t j, int64_t k, uint64_t seed) {
    const uint64_t h = mix64(seed ^ ((uint64_t)i * 0x8CB92BA72F3D8DD7ull) ^ ((uint64_t)j * 0x9E3779B97F4A7C15ull) ^
                             ((uint64_t)k * 0xC2B2AE3D27D4EB4Full));
    return 2.0 * unit(h) - 1.0;
}
inline double smooth(double t) { return t * t * (3.0 - 2.0 * t); }

// Value noise: smoothstep-weighted trilinear interpolation of lattice values.
double value_noise(double x, double y, double z, uint64_t seed) {
    const double fx = std::floor(x), fy = std::floor(y), fz = std::floor(z);
    const int64_t ix = (int64_t)fx, iy = (int64_t)fy, iz = (int64_t)fz;
    const double tx = smooth(x - fx), ty = smooth(y - fy), tz = smooth(z - fz);
    double c[2][2][2];
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
            for (int d = 0; d < 2; ++d) c[a][b][d] = lattice(ix + a, iy + b, iz + d, seed);
    const double x00 = c[0][0][0] + (c[1][0][0] - c[0][0][0]) * tx;
    const double x10 = c[0][1][0] + (c[1][1][0] - c[0][1][0]) * tx;
    const double x01 = c[0][0][1] + (c[1][0][1] - c[0][0][1]) * tx;
    const double x11 = c[0][1][1] + (c[1][1][1] - c[0][1][1]) * tx;
    const double y0 = x00 + (x10 - x00) * ty;
    const double y1 = x01 + (x11 - x01) * ty;
    return y0 + (y1 - y0) * tz;
}

// Three octaves (frequency 2, 4, 8; weights 1, 1/2, 1/4), normalized to [-1, 1].
double fractal_noise(double x, double y, double z, uint64_t seed) {
    double sum = 0.0, amp = 1.0, freq = 2.0, norm = 0.0;
    for (int o = 0; o < 3; ++o) {
        sum += amp * value_noise(x * freq, y * freq, z * freq, seed + 0x632BE59BD9B4E019ull * (uint64_t)o);
        norm += amp;
        amp *= 0.5;
        freq *= 2.0;
    }
    return sum / norm;
}

}  // namespace

extern "C" int pt_gen_icosphere(uint32_t level, float radius, float noise_amp, uint64_t noise_seed, float* x, float* y,
                                float* z, uint32_t* num_vertices, uint32_t* fv0, uint32_t* fv1, uint32_t* fv2,
                                uint32_t* num_faces) {
    if (level > 10) return pt::fail(PT_EINVAL, "icosphere level above 10");
    const uint64_t nf = 20ull << (2 * level);
    const uint64_t nv = 10ull * (1ull << (2 * level)) + 2;
    if (!x || !y || !z || !fv0 || !fv1 || !fv2) {
        if (num_vertices) *num_vertices = (uint32_t)nv;
        if (num_faces) *num_faces = (uint32_t)nf;
        return PT_OK;
    }
    if (num_vertices && *num_vertices < nv) return pt::fail(PT_EINVAL, "vertex buffer too small");
    if (num_faces && *num_faces < nf) return pt::fail(PT_EINVAL, "face buffer too small");
    // icosahedron: 12 vertices (0, +-1, +-phi) cyclic, 20 outward-wound faces
    const double phi = (1.0 + std::sqrt(5.0)) / 2.0;
    std::vector<double> v = {-1, phi, 0, 1, phi, 0, -1, -phi, 0, 1, -phi, 0, 0, -1, phi, 0, 1, phi,
                             0, -1, -phi, 0, 1, -phi, phi, 0, -1, phi, 0, 1, -phi, 0, -1, -phi, 0, 1};
    for (size_t i = 0; i < v.size(); i += 3) {
        const double n = std::sqrt(v[i] * v[i] + v[i + 1] * v[i + 1] + v[i + 2] * v[i + 2]);
        v[i] /= n; v[i + 1] /= n; v[i + 2] /= n;
    }
    std::vector<uint32_t> f = {0, 11, 5, 0, 5, 1, 0, 1, 7, 0, 7, 10, 0, 10, 11, 1, 5, 9, 5, 11, 4,
                               11, 10, 2, 10, 7, 6, 7, 1, 8, 3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6, 8,
                               3, 8, 9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7, 9, 8, 1};
    v.reserve(3 * nv);
    for (uint32_t l = 0; l < level; ++l) {
        std::unordered_map<uint64_t, uint32_t> mid;
        mid.reserve(f.size());
        auto midpoint = [&](uint32_t a, uint32_t b) -> uint32_t {
            const uint64_t key = a < b ? ((uint64_t)a << 32 | b) : ((uint64_t)b << 32 | a);
            auto it = mid.find(key);
            if (it != mid.end()) return it->second;
            double m[3] = {(v[3 * a] + v[3 * b]) * 0.5, (v[3 * a + 1] + v[3 * b + 1]) * 0.5, (v[3 * a + 2] + v[3 * b + 2]) * 0.5};
            const double n = std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
            const uint32_t id = (uint32_t)(v.size() / 3);
            v.push_back(m[0] / n); v.push_back(m[1] / n); v.push_back(m[2] / n);
            mid.emplace(key, id);
            return id;
        };
        std::vector<uint32_t> g;
        g.reserve(f.size() * 4);
        for (size_t i = 0; i < f.size(); i += 3) {
            const uint32_t a = f[i], b = f[i + 1], c = f[i + 2];
            const uint32_t ab = midpoint(a, b), bc = midpoint(b, c), ca = midpoint(c, a);
            const uint32_t q[12] = {a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca};
            g.insert(g.end(), q, q + 12);
        }
        f.swap(g);
    }
    for (uint64_t i = 0; i < nv; ++i) {
        const double px = v[3 * i], py = v[3 * i + 1], pz = v[3 * i + 2];
        const double r = (double)radius * (1.0 + (double)noise_amp * fractal_noise(px, py, pz, noise_seed));
        x[i] = (float)(px * r);
        y[i] = (float)(py * r);
        z[i] = (float)(pz * r);
    }
    for (uint64_t i = 0; i < nf; ++i) {
        fv0[i] = f[3 * i];
        fv1[i] = f[3 * i + 1];
        fv2[i] = f[3 * i + 2];
    }
    if (num_vertices) *num_vertices = (uint32_t)nv;
    if (num_faces) *num_faces = (uint32_t)nf;
    return PT_OK;
}

extern "C" int pt_gen_rays(uint64_t n, float origin_radius, uint64_t seed, pt_ray* rays) {
    if (!rays && n) return pt::fail(PT_EINVAL, "rays is NULL");
    const double two_pi = 6.283185307179586476925;
    for (uint64_t i = 0; i < n; ++i) {
        const uint64_t base = mix64(seed ^ mix64(i));
        const double u1 = unit(mix64(base + 1)), u2 = unit(mix64(base + 2));
        const double u3 = unit(mix64(base + 3)), u4 = unit(mix64(base + 4)), u5 = unit(mix64(base + 5));
        // origin: uniform on the sphere of radius origin_radius
        const double oz = 1.0 - 2.0 * u1, orr = std::sqrt(std::fmax(0.0, 1.0 - oz * oz));
        const double ox = orr * std::cos(two_pi * u2), oy = orr * std::sin(two_pi * u2);
        const double O[3] = {origin_radius * ox, origin_radius * oy, origin_radius * oz};
        // target: uniform in the unit ball (radius cbrt(u3), uniform direction)
        const double tz = 1.0 - 2.0 * u4, trr = std::sqrt(std::fmax(0.0, 1.0 - tz * tz));
        const double rr = std::cbrt(u3);
        const double T[3] = {rr * trr * std::cos(two_pi * u5), rr * trr * std::sin(two_pi * u5), rr * tz};
        const double d[3] = {T[0] - O[0], T[1] - O[1], T[2] - O[2]};
        const double len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        pt_ray& r = rays[i];
        for (int k = 0; k < 3; ++k) {
            r.org[k] = (float)O[k];
            r.dir[k] = (float)(d[k] / len);
        }
        if (i & 1) {
            r.tmax = (float)len;
            r.flags = PT_RAY_ANY_HIT;
        } else {
            r.tmax = INFINITY;
            r.flags = 0;
        }
    }
    return PT_OK;
}
