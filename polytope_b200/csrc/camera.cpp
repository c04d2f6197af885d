// camera.cpp -- host-side pinhole camera setup, as the reference builds it from a PBRT scene.
//
//   pbrt_parser.cpp:1099-1119  LookAt directive -> Transform::LookAt(eye, lookAt, up, false),
//                              applied with `current_transform *= t` on an identity Transform
//   Transform.cpp:322-365      Transform::LookAt
//   Matrix4x4.cpp:244-303      Matrix4x4::operator*= (row . column, summed left to right)
//   PerspectiveCamera.cpp:17-25 OneOverWidth, OneOverHeight, AspectRatio, TanFOVOver2
//   Transform.cpp:93-111       Apply(Point) of the camera-space origin (0, 0, 0)
// Compiled with -ffp-contract=off so each expression is the reference's float sequence.

#include <cmath>

#include "render.h"

namespace pt {

namespace {
struct V { float x, y, z; };
V vsub(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V vcross(V s, V r) { return {s.y * r.z - s.z * r.y, s.z * r.x - s.x * r.z, s.x * r.y - s.y * r.x}; }
float vlen(V v) { return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
V vnorm(V v) {
    const float d = 1.0f / vlen(v);
    return {v.x * d, v.y * d, v.z * d};
}
}  // namespace

CameraConst make_camera(const pt_camera& c, uint32_t width, uint32_t height) {
    float m[16];
    m[3] = c.eye[0]; m[7] = c.eye[1]; m[11] = c.eye[2]; m[15] = 1;
    const V dir = vnorm(vsub({c.look_at[0], c.look_at[1], c.look_at[2]}, {c.eye[0], c.eye[1], c.eye[2]}));
    const V up = vnorm({c.up[0], c.up[1], c.up[2]});
    V left = vcross(up, dir);
    if (vlen(left) == 0) {  // degenerate LookAt: the reference falls back to the identity
        for (int i = 0; i < 16; ++i) m[i] = (i % 5 == 0) ? 1.f : 0.f;
    } else {
        left = vnorm(left);
        const V nup = vcross(dir, left);
        m[0] = left.x; m[4] = left.y; m[8] = left.z; m[12] = 0;
        m[1] = nup.x; m[5] = nup.y; m[9] = nup.z; m[13] = 0;
        m[2] = dir.x; m[6] = dir.y; m[10] = dir.z; m[14] = 0;  // right_handed = false
    }
    CameraConst cc{};
    float id[16];
    for (int i = 0; i < 16; ++i) id[i] = (i % 5 == 0) ? 1.f : 0.f;
    for (int r = 0; r < 4; ++r)
        for (int k = 0; k < 4; ++k)
            cc.m[r * 4 + k] = id[r * 4 + 0] * m[0 * 4 + k] + id[r * 4 + 1] * m[1 * 4 + k] + id[r * 4 + 2] * m[2 * 4 + k] +
                              id[r * 4 + 3] * m[3 * 4 + k];
    cc.one_over_w = 1.0f / (float)width;
    cc.one_over_h = 1.0f / (float)height;
    cc.aspect = (float)width * cc.one_over_h;
    constexpr float pi_over_180 = 3.14159265358979323846 / 180.0f;
    cc.tan_half = (float)std::tan(c.fov_deg * pi_over_180 * .5f);
    // world-space origin: Apply(Point(0, 0, 0)) (constant for every pixel)
    const float* q = cc.m;
    float ox = 0.f * q[0] + 0.f * q[1] + 0.f * q[2] + q[3];
    float oy = 0.f * q[4] + 0.f * q[5] + 0.f * q[6] + q[7];
    float oz = 0.f * q[8] + 0.f * q[9] + 0.f * q[10] + q[11];
    const float ow = 0.f * q[12] + 0.f * q[13] + 0.f * q[14] + q[15];
    if (ow != 1) {
        const float div = 1.f / ow;
        ox = ox * div; oy = oy * div; oz = oz * div;
    }
    cc.org[0] = ox; cc.org[1] = oy; cc.org[2] = oz;
    return cc;
}

}  // namespace pt
