// Render kernels for sm_100a: projection, intersection emission, tile ranges
// and the tile rasterizer in its RGB / total-responsibility / evidence modes.
//
// Reference: src/project.rs:235-327 (project_splats), src/raster.rs:13-48
// (map_isects), :53-65 (lower_bound), :88-230 (rasterize_kernel). The
// arithmetic is the reference's in a fixed f32 operation order (sf_math.cuh)
// so that counts, keys, bboxes, images and fixed-point words match the CPU
// oracle bit for bit. Everything here is FP32/integer work: no step is a dense
// contraction, so the tensor cores have no part in it.
#include <cstdint>
#include "sf_internal.h"
#include "sf_math.cuh"

namespace sfk {

namespace {

using namespace sfm;

constexpr float kAlphaCutoff = 10.0f / 255.0f;
constexpr float kSHC0 = 0.2820948f, kSHC1 = 0.48860252f;
constexpr float kSHC2_0 = 0.9461747f, kSHC2_1 = 0.31539157f, kSHC2_2 = -1.0925485f,
                kSHC2_3 = 0.54627424f;
// power above which alpha = op*exp(-power) < 1/255 for sure: ln(255*op) plus
// a 1% relative margin in alpha, far above the exp/log rounding (<1e-6).
constexpr float kPowerMargin = 0.01f;

struct V3 { float x, y, z; };
__device__ __forceinline__ float dot3(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

// sh_to_rgb (src/project.rs:344-388) over coefficients already in registers,
// c[k*3 + channel].
template <int K>
__device__ __forceinline__ void sh_to_rgb(V3 d, const float (&c)[3 * K], float& r, float& g, float& b) {
    auto sh = [&](int k) { return c[k]; };
    r = kSHC0 * sh(0);
    g = kSHC0 * sh(1);
    b = kSHC0 * sh(2);
    if (K >= 4) {
        r += kSHC1 * ((-d.y * sh(3) + d.z * sh(6)) - d.x * sh(9));
        g += kSHC1 * ((-d.y * sh(4) + d.z * sh(7)) - d.x * sh(10));
        b += kSHC1 * ((-d.y * sh(5) + d.z * sh(8)) - d.x * sh(11));
    }
    if (K >= 9) {
        const float b4 = (kSHC2_2 * d.z) * d.x;
        const float b5 = (kSHC2_2 * d.z) * d.y;
        const float b6 = (kSHC2_0 * d.z) * d.z - kSHC2_1;
        const float b7 = ((kSHC2_3 * 2.0f) * d.x) * d.y;
        const float b8 = kSHC2_3 * (d.x * d.x - d.y * d.y);
        r += (((b6 * sh(18) + b7 * sh(12)) + b5 * sh(15)) + b4 * sh(21)) + b8 * sh(24);
        g += (((b6 * sh(19) + b7 * sh(13)) + b5 * sh(16)) + b4 * sh(22)) + b8 * sh(25);
        b += (((b6 * sh(20) + b7 * sh(14)) + b5 * sh(17)) + b4 * sh(23)) + b8 * sh(26);
    }
    if (K >= 16) {
        const float c1x = d.x * d.x - d.y * d.y;
        const float c1y = (2.0f * d.x) * d.y;
        const float tmp0c = (-2.285229f * d.z) * d.z + 0.4570458f;
        const float tmp1b = 1.4453057f * d.z;
        const float b9 = (-0.5900436f * d.x) * c1y + d.y * c1x;
        const float b10 = (-0.5900436f * d.x) * c1x - d.y * c1y;
        const float b11 = tmp0c * d.y;
        const float b12 = tmp0c * d.x;
        const float b13 = d.z * ((1.8658817f * d.z) * d.z - 1.119529f);
        const float b14 = tmp1b * c1y;
        const float b15 = tmp1b * c1x;
        r += (((((b9 * sh(27) + b10 * sh(30)) + b11 * sh(33)) + b12 * sh(36)) + b13 * sh(39)) +
              b14 * sh(42)) + b15 * sh(45);
        g += (((((b9 * sh(28) + b10 * sh(31)) + b11 * sh(34)) + b12 * sh(37)) + b13 * sh(40)) +
              b14 * sh(43)) + b15 * sh(46);
        b += (((((b9 * sh(29) + b10 * sh(32)) + b11 * sh(35)) + b12 * sh(38)) + b13 * sh(41)) +
              b14 * sh(44)) + b15 * sh(47);
    }
}

// The camera-independent terms of project_splats (src/project.rs:235-327),
// once per splat when the splats are created, in the f32 operations the
// projection would spend on them every frame: M = R(q) diag(exp(log_scale))
// (rows m0, m1, m2), opacity = sigmoid(logit), the extent cutoff
// log(opacity / (10/255)) and power_max = log(255 opacity) + margin.
// geom planes [kGeomPlanes][n]: m0.xyz, m1.xyz, m2.xyz, opacity, cutoff,
// power_max.
__global__ void splat_geom_kernel(const float* __restrict__ attr, uint32_t n, float* __restrict__ geom) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t N = n;
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = attr[(3 + k) * N + i];
    const float qw = a[0], qx = a[1], qy = a[2], qz = a[3];
    const V3 s{exp_(a[4]), exp_(a[5]), exp_(a[6])};
    const float opacity = sigmoid_(a[7]);
    const float x2 = qx * qx, y2 = qy * qy, z2 = qz * qz;
    const float xy = qx * qy, xz = qx * qz, yz = qy * qz;
    const float wx = qw * qx, wy = qw * qy, wz = qw * qz;
    const V3 r0{1.0f - 2.0f * (y2 + z2), 2.0f * (xy - wz), 2.0f * (xz + wy)};
    const V3 r1{2.0f * (xy + wz), 1.0f - 2.0f * (x2 + z2), 2.0f * (yz - wx)};
    const V3 r2{2.0f * (xz - wy), 2.0f * (yz + wx), 1.0f - 2.0f * (x2 + y2)};
    const float g[kGeomPlanes] = {r0.x * s.x, r0.y * s.y, r0.z * s.z, r1.x * s.x, r1.y * s.y, r1.z * s.z,
                                  r2.x * s.x, r2.y * s.y, r2.z * s.z, opacity, log_(opacity / kAlphaCutoff),
                                  log_(255.0f * opacity) + kPowerMargin};
#pragma unroll
    for (int k = 0; k < kGeomPlanes; ++k) geom[k * N + i] = g[k];
}

// project_splats (src/project.rs:235-327) for splat i, with the
// camera-independent terms read from geom (splat_geom_kernel). Field-major
// planes make every plane load a coalesced 128-byte warp access. Returns
// whether the splat is visible (not culled).
template <int K>
__device__ __forceinline__ bool project_one(const sf_view& v, const float* __restrict__ attr,
                                            const float* __restrict__ geom, const float* __restrict__ shs,
                                            uint32_t n, const ProjOut& o, uint32_t i) {
    const size_t N = n;
    // Every load is issued before any use (all planes in flight at once);
    // culled splats (a few percent) read their colour planes for nothing.
    float a[3], gm[kGeomPlanes];
#pragma unroll
    for (int k = 0; k < 3; ++k) a[k] = __ldg(attr + k * N + i);
#pragma unroll
    for (int k = 0; k < kGeomPlanes; ++k) gm[k] = __ldg(geom + k * N + i);
    float c[3 * K];
    const bool want_color = o.color != nullptr;
    if (want_color) {
#pragma unroll
        for (int k = 0; k < 3 * K; ++k) c[k] = __ldg(shs + k * N + i);
    }
    const float opacity = gm[9];
    const V3 mean{a[0], a[1], a[2]};
    const V3 rot0{v.rot0[0], v.rot0[1], v.rot0[2]};
    const V3 rot1{v.rot1[0], v.rot1[1], v.rot1[2]};
    const V3 rot2{v.rot2[0], v.rot2[1], v.rot2[2]};
    const float cam_z = dot3(rot2, mean) + v.trans[2];
    if (!(opacity >= kAlphaCutoff) || !(cam_z > 0.1f)) {
        o.depth_keys[i] = 0xffffffffu;
        o.tile_counts[i] = 0u;
        o.bbox[i] = make_uint2(0u, 0u);
        return false;
    }
    const float cam_x = dot3(rot0, mean) + v.trans[0];
    const float cam_y = dot3(rot1, mean) + v.trans[1];
    const float inv_z = 1.0f / cam_z;
    const V3 m0{gm[0], gm[1], gm[2]};
    const V3 m1{gm[3], gm[4], gm[5]};
    const V3 m2{gm[6], gm[7], gm[8]};
    const float lim_x = (1.3f * v.img[0]) / (2.0f * v.focal[0]);
    const float lim_y = (1.3f * v.img[1]) / (2.0f * v.focal[1]);
    const float u = clamp_(cam_x * inv_z, -lim_x, lim_x);
    const float vv = clamp_(cam_y * inv_z, -lim_y, lim_y);
    const float fx_iz = v.focal[0] * inv_z;
    const float fu_iz = fx_iz * u;
    const V3 t0{fx_iz * rot0.x - fu_iz * rot2.x, fx_iz * rot0.y - fu_iz * rot2.y,
                fx_iz * rot0.z - fu_iz * rot2.z};
    const float fy_iz = v.focal[1] * inv_z;
    const float fv_iz = fy_iz * vv;
    const V3 t1{fy_iz * rot1.x - fv_iz * rot2.x, fy_iz * rot1.y - fv_iz * rot2.y,
                fy_iz * rot1.z - fv_iz * rot2.z};
    const V3 j0{(t0.x * m0.x + t0.y * m1.x) + t0.z * m2.x, (t0.x * m0.y + t0.y * m1.y) + t0.z * m2.y,
                (t0.x * m0.z + t0.y * m1.z) + t0.z * m2.z};
    const V3 j1{(t1.x * m0.x + t1.y * m1.x) + t1.z * m2.x, (t1.x * m0.y + t1.y * m1.y) + t1.z * m2.y,
                (t1.x * m0.z + t1.y * m1.z) + t1.z * m2.z};
    const float ca = dot3(j0, j0) + 0.3f;
    const float cb = dot3(j0, j1);
    const float cc = dot3(j1, j1) + 0.3f;
    const float det = max_(ca * cc - cb * cb, 1e-6f);
    const float inv_det = 1.0f / det;
    const float cx = cc * inv_det, cy = -cb * inv_det, cz = ca * inv_det;

    const float mx = (v.focal[0] * cam_x) * inv_z + v.img[0] * 0.5f;
    const float my = (v.focal[1] * cam_y) * inv_z + v.img[1] * 0.5f;

    if (o.color) {
        V3 dir{mean.x - v.world_pos[0], mean.y - v.world_pos[1], mean.z - v.world_pos[2]};
        const float inv = 1.0f / sqrtf(dot3(dir, dir));
        dir = V3{dir.x * inv, dir.y * inv, dir.z * inv};
        float r, g, b;
        sh_to_rgb<K>(dir, c, r, g, b);
        o.color[i] = make_float4(r + 0.5f, g + 0.5f, b + 0.5f, 0.0f);
    }
    const float cutoff = gm[10];
    const float ext_x = sqrtf((2.0f * cutoff) * ca);
    const float ext_y = sqrtf((2.0f * cutoff) * cc);
    const float inv_tile = 1.0f / 16.0f;
    const uint32_t min_x = sat_u32(clamp_((mx - ext_x) * inv_tile, 0.0f, v.tile_bounds[0]));
    const uint32_t min_y = sat_u32(clamp_((my - ext_y) * inv_tile, 0.0f, v.tile_bounds[1]));
    const uint32_t max_x = sat_u32(clamp_((mx + ext_x) * inv_tile + 1.0f, 0.0f, v.tile_bounds[0]));
    const uint32_t max_y = sat_u32(clamp_((my + ext_y) * inv_tile + 1.0f, 0.0f, v.tile_bounds[1]));
    const float power_max = gm[11];

    o.depth_keys[i] = f2u(cam_z);
    o.tile_counts[i] = (max_x - min_x) * (max_y - min_y);
    o.bbox[i] = make_uint2(min_x | (min_y << 16), max_x | (max_y << 16));
    o.geo0[i] = make_float4(mx, my, 0.5f * cx, cy);
    o.geo1[i] = make_float4(0.5f * cz, opacity, power_max, 0.0f);
    if (o.ext) {
        // Half extents of the box around {power <= P}, P = power_max with a
        // 1e-4 margin for rounding: for q = hx dx^2 + hz dy^2 + cy dx dy the
        // level set's x extent is sqrt(P * hz / det), det = hx hz - cy^2/4.
        // Outside the box the computed power exceeds power_max, so the
        // rasterizer may skip the pair. A degenerate form gets no box.
        const float hx = 0.5f * cx, hz = 0.5f * cz;
        const float dq = hx * hz - 0.25f * (cy * cy);
        const float P = power_max * 1.0001f + 1e-4f;
        float ex = INFINITY, ey = INFINITY;
        if (dq > 0.0f && P > 0.0f) {
            ex = sqrtf(P * hz / dq) * 1.0001f + 1e-3f;
            ey = sqrtf(P * hx / dq) * 1.0001f + 1e-3f;
        }
        o.ext[i] = make_float2(ex, ey);
    }
    return true;
}

// One thread per splat. The visible count goes to one counter: the
// colour-free form (K = 1, a short kernel) sums it per block, since one
// atomic per warp on a single address serialises in L2 and bounded that
// kernel; the colour forms add it per warp (a block-wide count costs them
// registers).
template <int K>
__global__ __launch_bounds__(256, 3) void project_kernel(sf_view v_arg, const sf_view* __restrict__ v_dev,
                                                      const float* __restrict__ attr,
                                                      const float* __restrict__ geom,
                                                      const float* __restrict__ shs, uint32_t n,
                                                      ProjOut o) {
    pdl_trigger();  // the kernel after it may be scheduled in its last wave
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    // The view comes by value, or (for captured graphs re-run with new
    // cameras) from device memory.
    if (K == 1 && o.visible) {
        bool vis = false;
        if (i < n) vis = project_one<K>(v_dev ? *v_dev : v_arg, attr, geom, shs, n, o, i);
        const int c = __syncthreads_count(vis);
        if (threadIdx.x == 0 && c) atomicAdd(o.visible, (uint32_t)c);
        return;
    }
    if (i >= n) return;
    const sf_view v = v_dev ? *v_dev : v_arg;
    if (project_one<K>(v, attr, geom, shs, n, o, i) && o.visible) {
        const uint32_t active = __activemask();
        if ((threadIdx.x & 31u) == (uint32_t)(__ffs(active) - 1)) atomicAdd(o.visible, __popc(active));
    }
}

// map_isects (src/raster.rs:13-48): rank r writes its bbox tiles row-major at
// its scan offset. The 32 ranks of a warp own one contiguous output run
// (their offsets are consecutive), so the warp writes that run cooperatively:
// lane l emits outputs l, l+32, ... and finds the owning rank by a 5-step
// shuffle search over the lanes' inclusive ends. Every store is coalesced.
// Past capacity the write is dropped and flagged.
__global__ __launch_bounds__(256) void emit_kernel(const uint32_t* __restrict__ order,
                                                   const uint2* __restrict__ bbox,
                                                   const uint32_t* __restrict__ offsets, uint32_t n,
                                                   uint32_t tiles_per_row, uint32_t capacity,
                                                   uint32_t* __restrict__ tile_ids,
                                                   uint32_t* __restrict__ gaussian_ids,
                                                   uint32_t* err) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t r0 = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u;
    if (r0 >= n) return;
    const uint32_t r = r0 + lane;
    const bool valid = r < n;
    uint32_t vis = 0, min_x = 0, min_y = 0, width = 1, cnt = 0, off = 0;
    if (valid) {
        vis = order[r];
        const uint2 bb = bbox[vis];
        min_x = bb.x & 0xffffu;
        min_y = bb.x >> 16;
        const uint32_t max_x = bb.y & 0xffffu, max_y = bb.y >> 16;
        width = max(max_x - min_x, 1u);
        cnt = (max_x - min_x) * (max_y - min_y);
        off = offsets[r];
    }
    const uint32_t base = __shfl_sync(0xffffffffu, off, 0);
    uint32_t incl = valid ? off - base + cnt : 0u;
    const uint32_t total = __reduce_max_sync(0xffffffffu, incl);
    if (!valid) incl = total;
    bool over = false;
    // `total` is warp-uniform: every lane runs every iteration (the owner lane
    // of a shuffle must be active), only the stores are predicated.
    for (uint32_t p0 = 0; p0 < total; p0 += 32) {
        const uint32_t p = p0 + lane;
        // Owner: the first lane whose inclusive end exceeds p.
        uint32_t o = 0;
#pragma unroll
        for (uint32_t step = 16; step > 0; step >>= 1) {
            const uint32_t v = __shfl_sync(0xffffffffu, incl, o + step - 1);
            if (v <= p) o += step;
        }
        const uint32_t oend = __shfl_sync(0xffffffffu, incl, o);
        const uint32_t ocnt = __shfl_sync(0xffffffffu, cnt, o);
        const uint32_t ow = __shfl_sync(0xffffffffu, width, o);
        const uint32_t ox = __shfl_sync(0xffffffffu, min_x, o);
        const uint32_t oy = __shfl_sync(0xffffffffu, min_y, o);
        const uint32_t ovis = __shfl_sync(0xffffffffu, vis, o);
        if (p < total) {
            const uint32_t k = p - (oend - ocnt);
            const uint32_t slot = base + p;
            if (slot < capacity) {
                tile_ids[slot] = (ox + k % ow) + (oy + k / ow) * tiles_per_row;
                gaussian_ids[slot] = ovis;
            } else {
                over = true;
            }
        }
    }
    if (over) atomicOr(err, SF_DEV_ERR_CAPACITY);
}

// tile_start[t] = lower_bound(ids, t) for t in [0, num_tiles]: each thread
// scans 8 consecutive sorted ids and writes the starts of the tiles whose
// first entry (or an empty tile's insertion point) falls in its range.
constexpr uint32_t kStartItems = 8;
__global__ __launch_bounds__(256) void tile_start_kernel(const uint32_t* __restrict__ ids,
                                                         uint32_t n_static, const uint32_t* n_dev,
                                                         uint32_t num_tiles,
                                                         uint32_t* __restrict__ start) {
    const uint32_t n = n_dev ? *n_dev : n_static;
    const uint32_t i0 = (blockIdx.x * blockDim.x + threadIdx.x) * kStartItems;
    if (i0 > n) return;
    uint32_t prev = (i0 == 0) ? 0u : ids[i0 - 1] + 1u;
    for (uint32_t k = 0; k < kStartItems; ++k) {
        const uint32_t i = i0 + k;
        if (i > n) break;
        const uint32_t hi = (i == n) ? num_tiles : min(ids[i], num_tiles);
        for (uint32_t t = prev; t <= hi; ++t) start[t] = i;
        if (i == n) break;
        prev = max(prev, hi + 1u);
    }
}

__global__ void export_rows_kernel(const float4* __restrict__ geo0, const float4* __restrict__ geo1,
                                   const float4* __restrict__ color,
                                   const uint32_t* __restrict__ keys, uint32_t n,
                                   float* __restrict__ rows) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float* r = rows + (size_t)i * 9;
    if (keys[i] == 0xffffffffu) {
        for (int k = 0; k < 9; ++k) r[k] = 0.0f;
        return;
    }
    const float4 g0 = geo0[i], g1 = geo1[i];
    const float4 c = color ? color[i] : make_float4(0, 0, 0, 0);
    r[0] = g0.x; r[1] = g0.y; r[2] = 2.0f * g0.z; r[3] = g0.w; r[4] = 2.0f * g1.x;
    r[5] = c.x; r[6] = c.y; r[7] = c.z; r[8] = g1.y;
}

}  // namespace

cudaError_t launch_splat_geom(const float* attr, uint32_t n, float* geom, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    splat_geom_kernel<<<(n + 255) / 256, 256, 0, stream>>>(attr, n, geom);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_project(const sf_view& view, const float* attr, const float* geom, const float* sh, uint32_t n,
                           uint32_t sh_per_ch, const ProjOut& out, cudaStream_t stream,
                           const sf_view* view_dev) {
    if (n == 0) return cudaSuccess;
    const uint32_t grid = (n + 255) / 256;
    // Without colour no SH plane is read: the 1-coefficient form has the
    // fewest registers (more warps in flight for the attribute loads).
    sh_per_ch = out.color ? sh_degree_coeffs(sh_per_ch) : 1u;
    switch (sh_per_ch) {
        case 1: project_kernel<1><<<grid, 256, 0, stream>>>(view, view_dev, attr, geom, sh, n, out); break;
        case 4: project_kernel<4><<<grid, 256, 0, stream>>>(view, view_dev, attr, geom, sh, n, out); break;
        case 9: project_kernel<9><<<grid, 256, 0, stream>>>(view, view_dev, attr, geom, sh, n, out); break;
        case 16: project_kernel<16><<<grid, 256, 0, stream>>>(view, view_dev, attr, geom, sh, n, out); break;
        default: return cudaErrorInvalidValue;
    }
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_emit(const uint32_t* order, const uint2* bbox, const uint32_t* offsets,
                        uint32_t n, uint32_t tiles_per_row, uint32_t capacity, uint32_t* tile_ids,
                        uint32_t* gaussian_ids, uint32_t* err, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    emit_kernel<<<(n + 255) / 256, 256, 0, stream>>>(order, bbox, offsets, n, tiles_per_row,
                                                      capacity, tile_ids, gaussian_ids, err);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_tile_starts(const uint32_t* sorted_tile_ids, uint32_t num_isects,
                               const uint32_t* num_isects_dev, uint32_t max_isects,
                               uint32_t num_tiles, uint32_t* tile_start, cudaStream_t stream) {
    const uint32_t grid_n = ((num_isects_dev ? max_isects : num_isects) + 1 + kStartItems - 1) / kStartItems;
    tile_start_kernel<<<(grid_n + 255) / 256, 256, 0, stream>>>(sorted_tile_ids, num_isects,
                                                                num_isects_dev, num_tiles, tile_start);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_export_rows(const float4* geo0, const float4* geo1, const float4* color,
                               const uint32_t* depth_keys, uint32_t n, float* rows,
                               cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    export_rows_kernel<<<(n + 255) / 256, 256, 0, stream>>>(geo0, geo1, color, depth_keys, n, rows);
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace sfk
