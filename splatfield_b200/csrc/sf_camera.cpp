// Host camera math: Camera::look_at / Camera::focal (src/camera.rs:38-63) and
// CameraViewLaunch::for_camera (src/project.rs:76-96), which the reference
// builds on glam 0.33.6. Restated glam algorithms, f32, no contraction (this
// file is compiled with -ffp-contract=off):
//   Quat::from_rotation_arc: q = normalize(from x to, 1 + from.to), identity
//     near 0 degrees, a half turn about any_orthonormal_vector(from) near 180;
//   Vec4::normalize: v * (1/sqrt((x*x + z*z) + (y*y + w*w))) (SSE2 lane order);
//   Mat3::from_quat with doubled products; Mat3::inverse as adjugate rows
//   (y x z, z x x, x x y) scaled by 1/det; Affine3A::inverse translation
//   -(M^-1 t).
#include <cmath>
#include "sf_internal.h"

namespace sfk {

namespace {
struct V3 { float x, y, z; };
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
inline V3 mul(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
}  // namespace

void camera_look_at(const float position[3], const float target[3], sf_camera* out) {
    V3 d = sub(V3{target[0], target[1], target[2]}, V3{position[0], position[1], position[2]});
    d = mul(d, 1.0f / std::sqrt(dot(d, d)));
    const V3 from{0.0f, 0.0f, 1.0f};
    const float dp = dot(from, d);
    const float limit = 1.0f - 2.0f * 1.1920929e-07f;
    float q[4];
    if (dp > limit) {
        q[0] = 0.0f; q[1] = 0.0f; q[2] = 0.0f; q[3] = 1.0f;
    } else if (dp < -limit) {
        const float half = 3.14159274f * 0.5f;
        q[0] = 0.0f; q[1] = std::sin(half); q[2] = -0.0f * std::sin(half); q[3] = std::cos(half);
    } else {
        const V3 c = cross(from, d);
        q[0] = c.x; q[1] = c.y; q[2] = c.z; q[3] = 1.0f + dp;
        const float len2 = (q[0] * q[0] + q[2] * q[2]) + (q[1] * q[1] + q[3] * q[3]);
        const float r = 1.0f / std::sqrt(len2);
        for (float& v : q) v = v * r;
    }
    out->fov[0] = 0.8f;
    out->fov[1] = 0.8f;
    for (int k = 0; k < 3; ++k) out->position[k] = position[k];
    for (int k = 0; k < 4; ++k) out->rotation[k] = q[k];
}

void view_for_camera(const sf_camera& cam, uint32_t w, uint32_t h, sf_view* out) {
    const float qx = cam.rotation[0], qy = cam.rotation[1], qz = cam.rotation[2], qw = cam.rotation[3];
    const float x2 = qx + qx, y2 = qy + qy, z2 = qz + qz;
    const float xx = qx * x2, xy = qx * y2, xz = qx * z2;
    const float yy = qy * y2, yz = qy * z2, zz = qz * z2;
    const float wx = qw * x2, wy = qw * y2, wz = qw * z2;
    const V3 ax{1.0f - (yy + zz), xy + wz, xz - wy};
    const V3 ay{xy - wz, 1.0f - (xx + zz), yz + wx};
    const V3 az{xz + wy, yz - wx, 1.0f - (xx + yy)};
    const V3 t0 = cross(ay, az), t1 = cross(az, ax), t2 = cross(ax, ay);
    const float inv_det = 1.0f / dot(az, t2);
    const V3 r0 = mul(t0, inv_det), r1 = mul(t1, inv_det), r2 = mul(t2, inv_det);
    const V3 p{cam.position[0], cam.position[1], cam.position[2]};
    const V3 rows[3] = {r0, r1, r2};
    float* dst[3] = {out->rot0, out->rot1, out->rot2};
    for (int k = 0; k < 3; ++k) {
        dst[k][0] = rows[k].x;
        dst[k][1] = rows[k].y;
        dst[k][2] = rows[k].z;
        out->trans[k] = -dot(rows[k], p);
    }
    const float fw = (float)w, fh = (float)h;
    out->focal[0] = (fw * 0.5f) / std::tan(cam.fov[0] * 0.5f);
    out->focal[1] = (fh * 0.5f) / std::tan(cam.fov[1] * 0.5f);
    for (int k = 0; k < 3; ++k) out->world_pos[k] = cam.position[k];
    out->img[0] = fw;
    out->img[1] = fh;
    out->tile_bounds[0] = (float)((w + 15u) / 16u);
    out->tile_bounds[1] = (float)((h + 15u) / 16u);
}

}  // namespace sfk

#include <atomic>

namespace sfk {
namespace {
std::atomic<uint64_t> g_launches{0};
}
void note_launches(uint32_t k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
void forget_launches(uint64_t k) { g_launches.fetch_sub(k, std::memory_order_relaxed); }
uint64_t launches() { return g_launches.load(std::memory_order_relaxed); }
}  // namespace sfk
