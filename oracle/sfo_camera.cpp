// Oracle camera math (TEST INFRASTRUCTURE ONLY).
//
// Restates src/camera.rs:38-63 and src/project.rs:76-96 of the reference,
// which lean on glam 0.33.6 (a crates.io dependency, not vendored in the
// reference tree). The glam algorithms restated here are its published ones:
//   Quat::from_rotation_arc  half-way quaternion (c = from x to, w = 1 + dot),
//                            180-degree branch through any_orthonormal_vector
//                            (Duff et al., "Building an Orthonormal Basis,
//                            Revisited", JCGT 2017);
//   Mat3::from_quat          doubled-product rotation matrix;
//   Mat3::inverse            adjugate rows (y x z, z x x, x x y) over det;
//   Affine3A::inverse        translation = -(M^-1 * t).
// f32 throughout, products then sums left to right, no contraction.
#include <cmath>
#include "sfo.h"
#include "sfo_math.h"

namespace {

struct V3 { float x, y, z; };

inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
inline V3 scale(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }

// glam Vec4::normalize: v * (1/sqrt(dot)), SSE2 dot order (x2+z2)+(y2+w2).
void quat_normalize(float q[4]) {
    const float d = (q[0] * q[0] + q[2] * q[2]) + (q[1] * q[1] + q[3] * q[3]);
    const float r = 1.0f / std::sqrt(d);
    for (int k = 0; k < 4; ++k) q[k] = q[k] * r;
}

}  // namespace

extern "C" void sfo_camera_look_at(const float position[3], const float target[3],
                                   sfo_camera* out) {
    V3 d = sub(V3{target[0], target[1], target[2]}, V3{position[0], position[1], position[2]});
    d = scale(d, 1.0f / std::sqrt(dot(d, d)));
    const V3 from{0.0f, 0.0f, 1.0f};
    const float dp = dot(from, d);
    const float one_minus_eps = 1.0f - 2.0f * 1.1920929e-07f;
    float q[4];
    if (dp > one_minus_eps) {
        q[0] = 0.0f; q[1] = 0.0f; q[2] = 0.0f; q[3] = 1.0f;
    } else if (dp < -one_minus_eps) {
        // any_orthonormal_vector(+Z) = (0, 1, -0); half-turn about it.
        const float half = 3.14159274f * 0.5f;
        q[0] = 0.0f; q[1] = std::sin(half); q[2] = -0.0f * std::sin(half); q[3] = std::cos(half);
    } else {
        const V3 c = cross(from, d);
        q[0] = c.x; q[1] = c.y; q[2] = c.z; q[3] = 1.0f + dp;
        quat_normalize(q);
    }
    out->fov[0] = 0.8f;
    out->fov[1] = 0.8f;
    for (int k = 0; k < 3; ++k) out->position[k] = position[k];
    for (int k = 0; k < 4; ++k) out->rotation[k] = q[k];
}

extern "C" void sfo_view_for_camera(const sfo_camera* cam, uint32_t w, uint32_t h,
                                    sfo_view* out) {
    const float qx = cam->rotation[0], qy = cam->rotation[1], qz = cam->rotation[2],
                qw = cam->rotation[3];
    const float x2 = qx + qx, y2 = qy + qy, z2 = qz + qz;
    const float xx = qx * x2, xy = qx * y2, xz = qx * z2;
    const float yy = qy * y2, yz = qy * z2, zz = qz * z2;
    const float wx = qw * x2, wy = qw * y2, wz = qw * z2;
    // Columns of the camera-to-world rotation.
    const V3 cx{1.0f - (yy + zz), xy + wz, xz - wy};
    const V3 cy{xy - wz, 1.0f - (xx + zz), yz + wx};
    const V3 cz{xz + wy, yz - wx, 1.0f - (xx + yy)};
    const V3 t0 = cross(cy, cz), t1 = cross(cz, cx), t2 = cross(cx, cy);
    const float det = dot(cz, t2);
    const float inv_det = 1.0f / det;
    // Rows of the inverse = adjugate rows over det.
    const V3 r0 = scale(t0, inv_det), r1 = scale(t1, inv_det), r2 = scale(t2, inv_det);
    const V3 p{cam->position[0], cam->position[1], cam->position[2]};
    out->rot0[0] = r0.x; out->rot0[1] = r0.y; out->rot0[2] = r0.z;
    out->rot1[0] = r1.x; out->rot1[1] = r1.y; out->rot1[2] = r1.z;
    out->rot2[0] = r2.x; out->rot2[1] = r2.y; out->rot2[2] = r2.z;
    out->trans[0] = -dot(r0, p);
    out->trans[1] = -dot(r1, p);
    out->trans[2] = -dot(r2, p);
    const float img_x = (float)w, img_y = (float)h;
    out->focal[0] = (img_x * 0.5f) / std::tan(cam->fov[0] * 0.5f);
    out->focal[1] = (img_y * 0.5f) / std::tan(cam->fov[1] * 0.5f);
    for (int k = 0; k < 3; ++k) out->world_pos[k] = cam->position[k];
    out->img[0] = img_x;
    out->img[1] = img_y;
    out->tile_bounds[0] = (float)((w + 15u) / 16u);
    out->tile_bounds[1] = (float)((h + 15u) / 16u);
}
