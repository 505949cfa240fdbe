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

// Bit w set: the box around the splat's {power <= power_max} (half extents
// `e`, computed with margin by the projection) overlaps the pixel centres of
// warp w's 8x4 block of tile (tx, ty). A pair outside the box has computed
// power above power_max, which the per-pixel path skips as well, so dropping
// it changes nothing.
__device__ __forceinline__ uint32_t warp_mask(float mx, float my, float2 e, uint32_t tx, uint32_t ty) {
    const float bx = (float)(tx * 16) + 0.5f, by = (float)(ty * 16) + 0.5f;
    const float lx = mx - e.x - bx, hxr = mx + e.x - bx;  // box relative to the tile's first centre
    const float ly = my - e.y - by, hyr = my + e.y - by;
    // columns [0,7] and [8,15]; rows [0,3], [4,7], [8,11], [12,15]
    const uint32_t cx = (uint32_t)(lx <= 7.0f && hxr >= 0.0f) | ((uint32_t)(lx <= 15.0f && hxr >= 8.0f) << 1);
    uint32_t m = 0;
#pragma unroll
    for (uint32_t r = 0; r < 4; ++r) {
        const float y0 = (float)(r * 4);
        if (ly <= y0 + 3.0f && hyr >= y0) m |= cx << (2 * r);
    }
    return m;
}

// rasterize_kernel (src/raster.rs:88-230). One 256-thread block per 16x16
// tile; each warp owns an 8x4 pixel block. Chunks of 256 splat records are
// staged in shared memory. Pairs whose power exceeds the splat's power_max
// (alpha < 1/255 there, the reference's skip) bypass the exponential. The
// tile stops once every pixel is saturated (T < 1/255).
// CULL: each staged splat also gets an 8-bit mask of the warp blocks its
// power_max box reaches (warp_mask) and a warp walks only its splats (and
// stops once its own pixels are saturated) — fewer steps, more registers;
// which form is faster depends on the scene, so both are kept.
// DETAIL: per-pair diagnostic counters (evaluated / contributing / walked
// pairs); off in the timed kernels.
// Responsibility/evidence words are reduced per warp (redux.sync), then per
// tile in shared memory, then added to global memory once per (tile, splat):
// integer sums, so the words equal the reference's per-pixel atomics exactly.
//
// LAZY: the tile's list comes unsorted — the binned build's placed (depth
// key, splat id) pairs — and is put in order here, slab by slab, only as far
// as the tile needs: a 256-bin histogram over the 64-bit (key, id) values
// left picks the longest run of bins holding at most kSlab entries (narrowing
// the key interval while even the first bin holds more), those entries are
// gathered and bitonic-sorted in shared memory and composited, and the next
// slab starts after the last bin taken. (key, id) values are distinct and
// slabs end on bin boundaries, so the composite order is exactly the sorted
// list's; most tiles saturate inside their first slab, so most of the list is
// never sorted. The stored per-pixel last-contributor index counts positions
// in that order.

constexpr uint32_t kSlab = 2048;
constexpr uint32_t kFirstSlab = 256;

struct RasterSmem {
    float4* g0;
    float4* g1;
    float4* col;
    uint32_t* gid;
    uint32_t* acc0;
    uint32_t* acc1;
    uint8_t* mask;
};

struct PixelState {
    float T, pr, pg, pb;
    uint32_t last;
    bool done;
    uint32_t n_eval, n_hit, n_proc;
};

// Composites list entries [0, count) in order; id(i) gives entry i's splat
// id, list_off the entry's offset in the tile's whole sorted list. Returns
// true once every pixel of the tile is saturated (uniform).
template <int MODE, bool CULL, bool DETAIL, typename IdOf>
__device__ bool composite_list(const RasterArgs& a, const RasterSmem& sm, IdOf id, uint32_t count,
                               uint32_t list_off, uint32_t tx, uint32_t ty, float fx, float fy, uint32_t inside,
                               PixelState& ps) {
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const float inv255 = 1.0f / 255.0f;
    for (uint32_t chunk = 0; chunk < count; chunk += 256) {
        __syncthreads();
        const uint32_t idx = chunk + tid;
        if (idx < count) {
            const uint32_t g = id(idx);
            const float4 g0 = a.geo0[g], g1 = a.geo1[g];
            sm.g0[tid] = g0;
            sm.g1[tid] = g1;
            if (CULL) sm.mask[tid] = (uint8_t)warp_mask(g0.x, g0.y, a.ext[g], tx, ty);
            if (MODE == 0) {
                sm.col[tid] = a.color[g];
            } else {
                sm.gid[tid] = g;
                sm.acc0[tid] = 0u;
                if (MODE == 2) sm.acc1[tid] = 0u;
            }
        }
        if (__syncthreads_count(ps.done) == 256) return true;
        const uint32_t cnt = min(256u, count - chunk);
        // One (warp, entry) step: every lane of the warp runs it together.
        auto step = [&](uint32_t j) {
            if (DETAIL) ++ps.n_proc;
            uint32_t q = 0;
            // CULL: a warp whose pixels are all done has left the chunk, so
            // the power is formed unconditionally and one branch tests both.
            // Otherwise a done warp skips the loads and arithmetic.
            if (CULL || !ps.done) {
                const float4 g0 = sm.g0[j];
                const float4 g1 = sm.g1[j];
                const float dx = g0.x - fx, dy = g0.y - fy;
                const float power = fma_(g0.z * dx, dx, fma_(g1.x * dy, dy, (g0.w * dx) * dy));
                if ((!CULL || !ps.done) && !(power > g1.z)) {
                    if (DETAIL) ++ps.n_eval;
                    const float alpha = fminf(g1.y * exp_neg_(-power), 0.999f);
                    if (alpha >= inv255) {
                        if (DETAIL) ++ps.n_hit;
                        const float vis = alpha * ps.T;
                        if (MODE == 0) {
                            const float4 c = sm.col[j];
                            ps.pr = fma_(c.x, vis, ps.pr);
                            ps.pg = fma_(c.y, vis, ps.pg);
                            ps.pb = fma_(c.z, vis, ps.pb);
                        } else {
                            q = sat_u32(vis * a.scale);
                        }
                        ps.T = ps.T * (1.0f - alpha);
                        ps.last = list_off + chunk + j + 1;
                        if (ps.T < inv255) ps.done = true;
                    }
                }
            }
            if (MODE == 1) {
                const uint32_t s = __reduce_add_sync(0xffffffffu, q);
                if (lane == 0 && s) atomicAdd(&sm.acc0[j], s);
            } else if (MODE == 2) {
                const uint32_t qf = inside ? q : 0u;
                const uint32_t sf = __reduce_add_sync(0xffffffffu, qf);
                const uint32_t sb = __reduce_add_sync(0xffffffffu, q - qf);
                if (lane == 0) {
                    if (sf) atomicAdd(&sm.acc0[j], sf);
                    if (sb) atomicAdd(&sm.acc1[j], sb);
                }
            }
        };
        if (CULL) {
            // This warp's entries of the chunk, 32 candidates per ballot;
            // only entries with the warp's bit are walked, in list order.
            for (uint32_t g32 = 0; g32 < cnt; g32 += 32) {
                if (__all_sync(0xffffffffu, ps.done)) break;
                uint32_t word = __ballot_sync(0xffffffffu,
                                              g32 + lane < cnt && ((sm.mask[g32 + lane] >> warp) & 1u));
                while (word) {
                    const uint32_t j = g32 + (uint32_t)(__ffs(word) - 1);
                    word &= word - 1u;
                    step(j);
                }
            }
        } else {
            for (uint32_t j = 0; j < cnt; ++j) step(j);
        }
        if (MODE != 0) {
            __syncthreads();
            if (tid < cnt) {
                const uint32_t g = sm.gid[tid];
                if (MODE == 1) {
                    if (sm.acc0[tid]) atomicAdd(a.resp + g, sm.acc0[tid]);
                } else {
                    if (sm.acc0[tid]) atomicAdd(a.fg + g, sm.acc0[tid]);
                    if (sm.acc1[tid]) atomicAdd(a.bg + g, sm.acc1[tid]);
                }
            }
        }
    }
    return false;
}

__device__ __forceinline__ unsigned long long pair_value(uint2 p) {
    return ((unsigned long long)p.x << 32) | p.y;
}

// Block min / max of 64-bit values (uniform); s64 holds 2 * 8 words.
__device__ void block_minmax64(unsigned long long lo, unsigned long long hi, unsigned long long* s64,
                               unsigned long long& mn, unsigned long long& mx) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
#pragma unroll
    for (uint32_t d = 16; d > 0; d >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, d));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, d));
    }
    __syncthreads();
    if (lane == 0) {
        s64[warp] = lo;
        s64[8 + warp] = hi;
    }
    __syncthreads();
    mn = s64[0];
    mx = s64[8];
    for (uint32_t w = 1; w < 8; ++w) {
        mn = min(mn, s64[w]);
        mx = max(mx, s64[8 + w]);
    }
    __syncthreads();
}

// Bitonic sort of v[0, m) ascending in shared memory (m <= kSlab), padded to
// a power of two with the largest value.
__device__ void bitonic_sort64(unsigned long long* v, uint32_t m) {
    uint32_t p = 1;
    while (p < m) p <<= 1;
    for (uint32_t i = m + threadIdx.x; i < p; i += 256) v[i] = ~0ull;
    __syncthreads();
    for (uint32_t k = 2; k <= p; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < p; i += 256) {
                const uint32_t ixj = i ^ j;
                if (ixj > i) {
                    const unsigned long long x = v[i], y = v[ixj];
                    const bool up = (i & k) == 0;
                    if ((x > y) == up) {
                        v[i] = y;
                        v[ixj] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// One tile (block-uniform); the shared arrays are the kernel's.
template <int MODE, bool CULL, bool DETAIL, bool LAZY>
__device__ __forceinline__ void raster_tile(const RasterArgs& a, const uint32_t tile) {
    __shared__ float4 s_g0[256];
    __shared__ float4 s_g1[256];
    __shared__ float4 s_col[MODE == 0 ? 256 : 1];
    __shared__ uint32_t s_gid[MODE == 0 ? 1 : 256];
    __shared__ uint32_t s_acc0[MODE == 0 ? 1 : 256];
    __shared__ uint32_t s_acc1[MODE == 2 ? 256 : 1];
    __shared__ uint8_t s_mask[256];
    __shared__ unsigned long long s_slab[LAZY ? kSlab : 1];
    __shared__ uint32_t s_hist[LAZY ? 256 : 1];
    __shared__ unsigned long long s_64[16];
    __shared__ uint32_t s_ctl[4];

    const uint32_t tx = tile % a.tiles_x, ty = tile / a.tiles_x;
    const uint32_t tid = threadIdx.x, lane = tid & 31u;
    const uint32_t warp = tid >> 5;
    const uint32_t px = tx * 16 + (warp & 1u) * 8 + (lane & 7u);
    const uint32_t py = ty * 16 + (warp >> 1) * 4 + (lane >> 3);
    const bool in_bounds = px < a.w && py < a.h;
    const float fx = (float)px + 0.5f, fy = (float)py + 0.5f;
    uint32_t inside = 0;
    if (MODE == 2 && in_bounds) inside = (a.mask[px / 32 + py * a.mask_wpr] >> (px % 32)) & 1u;
    const uint32_t start = a.tile_start[tile], end = a.tile_start[tile + 1];
    const RasterSmem sm{s_g0, s_g1, s_col, s_gid, s_acc0, s_acc1, s_mask};
    PixelState ps{1.0f, 0.0f, 0.0f, 0.0f, 0u, !in_bounds, 0u, 0u, 0u};

    if (!LAZY || end - start <= a.lazy_min) {
        const uint32_t* ids = a.gaussian_ids + start;
        composite_list<MODE, CULL, DETAIL>(
            a, sm, [&](uint32_t i) { return ids[i]; }, end - start, 0, tx, ty, fx, fy, inside, ps);
    } else if (end > start) {
        const uint2* pairs = a.pairs + start;
        const uint32_t n = end - start;
        unsigned long long lo = ~0ull, hi = 0;
        for (uint32_t i = tid; i < n; i += 256) {
            const unsigned long long v = pair_value(pairs[i]);
            lo = min(lo, v);
            hi = max(hi, v);
        }
        unsigned long long vmin, vmax;
        block_minmax64(lo, hi, s_64, vmin, vmax);
        auto slab_id = [&](uint32_t i) { return (uint32_t)s_slab[i]; };
        if (n <= kFirstSlab) {
            for (uint32_t i = tid; i < n; i += 256) s_slab[i] = pair_value(pairs[i]);
            __syncthreads();
            bitonic_sort64(s_slab, n);
            composite_list<MODE, CULL, DETAIL>(a, sm, slab_id, n, 0, tx, ty, fx, fy, inside, ps);
        } else {
            unsigned long long cur = vmin;
            uint32_t pos = 0;
            // The first slab aims at kFirstSlab entries (most tiles saturate
            // well inside it), later ones at the full kSlab.
            uint32_t target = kFirstSlab;
            for (;;) {
                // Pick [cur, sel] holding at most `target` of the values left
                // (one whole bin of up to kSlab when the first bin alone is
                // past the target).
                unsigned long long top = vmax, sel = vmax;
                for (;;) {
                    const unsigned long long width = top - cur;
                    const uint32_t wbits = width == 0 ? 0u : 64u - (uint32_t)__clzll(width);
                    const uint32_t shift = wbits > 8 ? wbits - 8 : 0u;
                    s_hist[tid] = 0;
                    __syncthreads();
                    for (uint32_t i = tid; i < n; i += 256) {
                        const unsigned long long v = pair_value(pairs[i]);
                        if (v >= cur && v <= top) atomicAdd(&s_hist[(uint32_t)((v - cur) >> shift)], 1u);
                    }
                    __syncthreads();
                    if (tid < 32) {
                        // Warp 0: prefix over the 256 bins (8 per lane), the
                        // last bin whose running total stays within target.
                        const uint32_t nb = (uint32_t)(width >> shift) + 1u;
                        uint32_t c[8], run = 0;
#pragma unroll
                        for (uint32_t q = 0; q < 8; ++q) {
                            const uint32_t b = lane * 8 + q;
                            c[q] = b < nb ? s_hist[b] : 0u;
                            run += c[q];
                        }
                        uint32_t incl = run;
#pragma unroll
                        for (uint32_t d = 1; d < 32; d <<= 1) {
                            const uint32_t x = __shfl_up_sync(0xffffffffu, incl, d);
                            if (lane >= d) incl += x;
                        }
                        uint32_t acc = incl - run, best = 0u;
                        bool any = false;
#pragma unroll
                        for (uint32_t q = 0; q < 8; ++q) {
                            acc += c[q];
                            const uint32_t b = lane * 8 + q;
                            if (b < nb && acc <= target) {
                                best = b;
                                any = true;
                            }
                        }
                        const uint32_t e = __reduce_max_sync(0xffffffffu, any ? best + 1u : 0u);
                        if (lane == 0) {
                            const uint32_t h0 = s_hist[0];
                            // e == 0: even bin 0 is past the target.
                            s_ctl[0] = e > 0 ? 1u : (h0 <= kSlab ? 1u : 0u);
                            s_ctl[1] = e > 0 ? e - 1u : 0u;
                            s_ctl[2] = nb;
                        }
                    }
                    __syncthreads();
                    const uint32_t e = s_ctl[1], bins = s_ctl[2];
                    if (!s_ctl[0]) {
                        // The first bin holds more than kSlab: narrow to it.
                        top = cur + ((1ull << shift) - 1ull);
                        continue;
                    }
                    sel = (e + 1 >= bins) ? top : cur + (((unsigned long long)(e + 1)) << shift) - 1ull;
                    break;
                }
                if (tid == 0) s_ctl[3] = 0;
                __syncthreads();
                for (uint32_t i = tid; i < n; i += 256) {
                    const unsigned long long v = pair_value(pairs[i]);
                    if (v >= cur && v <= sel) s_slab[atomicAdd(&s_ctl[3], 1u)] = v;
                }
                __syncthreads();
                const uint32_t m = s_ctl[3];
                bitonic_sort64(s_slab, m);
                if (composite_list<MODE, CULL, DETAIL>(a, sm, slab_id, m, pos, tx, ty, fx, fy, inside, ps))
                    break;
                pos += m;
                if (sel == vmax) break;
                cur = sel + 1;
                target = kSlab;
                __syncthreads();
            }
        }
    }
    if (a.stats) {
        if (DETAIL) {
            const uint32_t e = __reduce_add_sync(0xffffffffu, ps.n_eval);
            const uint32_t c = __reduce_add_sync(0xffffffffu, ps.n_hit);
            const uint32_t pr_ = __reduce_add_sync(0xffffffffu, ps.n_proc);
            if (lane == 0) {
                atomicAdd(a.stats + 1, (unsigned long long)e);
                atomicAdd(a.stats + 2, (unsigned long long)c);
                atomicAdd(a.stats + 3, (unsigned long long)pr_);
            }
        }
        // Algorithmic pairs: 256 per entry of the sorted list that a walk
        // in 256-entry chunks covers until every pixel is saturated — the
        // entry that saturates the tile's last pixel, rounded up to a chunk
        // (the whole list if a pixel never saturates). The same count for
        // either list order.
        const uint32_t n_list = end - start;
        uint32_t e = ps.done ? ps.last : n_list;
        e = __reduce_max_sync(0xffffffffu, e);
        __syncthreads();
        if (tid == 0) s_ctl[0] = 0;
        __syncthreads();
        if (lane == 0) atomicMax(&s_ctl[0], e);
        __syncthreads();
        if (tid == 0) {
            const uint32_t emax = s_ctl[0];
            const uint64_t chunks = ((uint64_t)emax + 255u) / 256u * 256u;
            const uint64_t walked = chunks < n_list ? chunks : (uint64_t)n_list;
            atomicAdd(a.stats, 256ull * walked);
        }
    }
    if (!in_bounds) return;
    const size_t pix = (size_t)py * a.w + px;
    if (MODE == 0) {
        if (a.bitmap) {
            const uint32_t r = sat_u32(clamp_(ps.pr * 255.0f, 0.0f, 255.0f));
            const uint32_t g = sat_u32(clamp_(ps.pg * 255.0f, 0.0f, 255.0f));
            const uint32_t b = sat_u32(clamp_(ps.pb * 255.0f, 0.0f, 255.0f));
            const uint32_t al = sat_u32(clamp_((1.0f - ps.T) * 255.0f, 0.0f, 255.0f));
            a.bitmap[(size_t)py * a.row_stride + px] = r | (g << 8) | (b << 16) | (al << 24);
        }
        if (a.rgba) a.rgba[pix] = make_float4(ps.pr, ps.pg, ps.pb, 1.0f - ps.T);
    }
    if (a.final_t) a.final_t[pix] = ps.T;
    if (a.n_contrib) a.n_contrib[pix] = ps.last;
}

// One block per tile: block i takes tile i, or with class lists the i-th
// tile in longest-list-first order.
template <int MODE, bool CULL, bool DETAIL, bool LAZY>
__global__ __launch_bounds__(256) void raster_kernel(RasterArgs a) {
    uint32_t tile = blockIdx.x;
    if (a.class_lists) {
        const uint32_t tiles = a.tiles_x * a.tiles_y;
        uint32_t j = blockIdx.x;
        int k = kSortClasses - 1;
        for (; k >= 0; --k) {
            const uint32_t c = a.class_n[k];
            if (j < c) break;
            j -= c;
        }
        // k < 0: the empty tiles (the counts sum to the tile count).
        tile = a.class_lists[(size_t)(k < 0 ? kSortClasses : k) * tiles + j];
    }
    raster_tile<MODE, CULL, DETAIL, LAZY>(a, tile);
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

template <int MODE, bool LAZY>
void raster_dispatch2(const RasterArgs& a, uint32_t tiles, cudaStream_t stream) {
    if (a.cull) {
        if (a.detail) raster_kernel<MODE, true, true, LAZY><<<tiles, 256, 0, stream>>>(a);
        else raster_kernel<MODE, true, false, LAZY><<<tiles, 256, 0, stream>>>(a);
    } else {
        if (a.detail) raster_kernel<MODE, false, true, LAZY><<<tiles, 256, 0, stream>>>(a);
        else raster_kernel<MODE, false, false, LAZY><<<tiles, 256, 0, stream>>>(a);
    }
}

template <int MODE>
void raster_dispatch(const RasterArgs& a, uint32_t tiles, cudaStream_t stream) {
    if (a.pairs) raster_dispatch2<MODE, true>(a, tiles, stream);
    else raster_dispatch2<MODE, false>(a, tiles, stream);
}

cudaError_t launch_raster(int mode, const RasterArgs& a, cudaStream_t stream) {
    const uint32_t tiles = a.tiles_x * a.tiles_y;
    if (tiles == 0) return cudaSuccess;
    switch (mode) {
        case 0: raster_dispatch<0>(a, tiles, stream); break;
        case 1: raster_dispatch<1>(a, tiles, stream); break;
        case 2: raster_dispatch<2>(a, tiles, stream); break;
        default: return cudaErrorInvalidValue;
    }
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
