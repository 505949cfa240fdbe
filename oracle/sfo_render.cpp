// Oracle FP32 render pipeline (TEST INFRASTRUCTURE ONLY; also the timed
// multi-core CPU baseline). Restates the reference's kernels in the canonical
// f32 operation order that the CUDA path must reproduce bit for bit:
//   project_splats            src/project.rs:235-327 (+ :98-232, SH :329-388)
//   depth sort                src/render.rs:310-316 (ties by splat id)
//   exclusive_scan_gather     crates/sort/src/scan.rs:219-255
//   map_isects                src/raster.rs:13-48
//   stable tile sort          src/render.rs:345-352, crates/sort/src/sort.rs:311-380
//   lower_bound ranges        src/raster.rs:53-65
//   rasterize_kernel          src/raster.rs:88-230
// Canonical choices where the reference leaves rounding to the GPU driver:
//   * exp/log/sqrt/divide per sfo_math.h;
//   * raster power = fma(hx*dx, dx, fma(hz*dy, dy, (cy*dx)*dy)), hx = 0.5*cx,
//     hz = 0.5*cz (algebraically the reference's 0.5*(cx dx^2 + cz dy^2) +
//     cy dx dy, src/raster.rs:68-70);
//   * colour accumulation pix += c*vis is fma(c, vis, pix);
//   * a splat whose opacity or camera z is NaN is culled (the reference's
//     `<`/`<=` culls let NaN through into garbage keys).
#include <algorithm>
#include <cstring>
#include <vector>
#include <omp.h>
#include "sfo.h"
#include "sfo_math.h"

using namespace sfo;

namespace {

constexpr float kAlphaCutoff = 10.0f / 255.0f;   // project.rs:13
constexpr float kSHC0 = 0.2820948f;              // project.rs:329
constexpr float kSHC1 = 0.48860252f;             // project.rs:336
constexpr float kSHC2_0 = 0.9461747f;            // project.rs:337-340
constexpr float kSHC2_1 = 0.31539157f;
constexpr float kSHC2_2 = -1.0925485f;
constexpr float kSHC2_3 = 0.54627424f;

struct V3 { float x, y, z; };
inline float dot3(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

// sh_to_rgb (project.rs:344-388): per-channel sums in source order.
void sh_to_rgb(uint32_t chs, V3 d, uint32_t s, uint32_t n, const float* shs, float rgb[3]) {
    const size_t st = n;
    auto sh = [&](int k) { return shs[(size_t)k * st + s]; };
    float r = kSHC0 * sh(0);
    float g = kSHC0 * sh(1);
    float b = kSHC0 * sh(2);
    if (chs >= 4) {
        r += kSHC1 * ((-d.y * sh(3) + d.z * sh(6)) - d.x * sh(9));
        g += kSHC1 * ((-d.y * sh(4) + d.z * sh(7)) - d.x * sh(10));
        b += kSHC1 * ((-d.y * sh(5) + d.z * sh(8)) - d.x * sh(11));
    }
    if (chs >= 9) {
        const float b4 = (kSHC2_2 * d.z) * d.x;
        const float b5 = (kSHC2_2 * d.z) * d.y;
        const float b6 = (kSHC2_0 * d.z) * d.z - kSHC2_1;
        const float b7 = ((kSHC2_3 * 2.0f) * d.x) * d.y;
        const float b8 = kSHC2_3 * (d.x * d.x - d.y * d.y);
        r += (((b6 * sh(18) + b7 * sh(12)) + b5 * sh(15)) + b4 * sh(21)) + b8 * sh(24);
        g += (((b6 * sh(19) + b7 * sh(13)) + b5 * sh(16)) + b4 * sh(22)) + b8 * sh(25);
        b += (((b6 * sh(20) + b7 * sh(14)) + b5 * sh(17)) + b4 * sh(23)) + b8 * sh(26);
    }
    if (chs >= 16) {
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
    rgb[0] = r; rgb[1] = g; rgb[2] = b;
}

// One splat through project_splats. Returns false when culled.
bool project_one(const sfo_view& v, const float* attr, const float* shs, uint32_t n,
                 uint32_t sh_per_ch, uint32_t i, uint32_t* key, uint32_t* count,
                 uint32_t bb[2], float row[9]) {
    const size_t N = n;
    const V3 mean{attr[0 * N + i], attr[1 * N + i], attr[2 * N + i]};
    const float qw = attr[3 * N + i], qx = attr[4 * N + i], qy = attr[5 * N + i],
                qz = attr[6 * N + i];
    const V3 s{expf_c(attr[7 * N + i]), expf_c(attr[8 * N + i]), expf_c(attr[9 * N + i])};
    const float opacity = sigmoid(attr[10 * N + i]);
    if (!(opacity >= kAlphaCutoff)) return false;
    const V3 rot0{v.rot0[0], v.rot0[1], v.rot0[2]};
    const V3 rot1{v.rot1[0], v.rot1[1], v.rot1[2]};
    const V3 rot2{v.rot2[0], v.rot2[1], v.rot2[2]};
    const V3 cam{dot3(rot0, mean) + v.trans[0], dot3(rot1, mean) + v.trans[1],
                 dot3(rot2, mean) + v.trans[2]};
    if (!(cam.z > 0.1f)) return false;
    const float inv_z = 1.0f / cam.z;

    // compute_cov2d (project.rs:176-221)
    const float x2 = qx * qx, y2 = qy * qy, z2 = qz * qz;
    const float xy = qx * qy, xz = qx * qz, yz = qy * qz;
    const float wx = qw * qx, wy = qw * qy, wz = qw * qz;
    const V3 r0{1.0f - 2.0f * (y2 + z2), 2.0f * (xy - wz), 2.0f * (xz + wy)};
    const V3 r1{2.0f * (xy + wz), 1.0f - 2.0f * (x2 + z2), 2.0f * (yz - wx)};
    const V3 r2{2.0f * (xz - wy), 2.0f * (yz + wx), 1.0f - 2.0f * (x2 + y2)};
    const V3 m0{r0.x * s.x, r0.y * s.y, r0.z * s.z};
    const V3 m1{r1.x * s.x, r1.y * s.y, r1.z * s.z};
    const V3 m2{r2.x * s.x, r2.y * s.y, r2.z * s.z};
    const float lim_x = (1.3f * v.img[0]) / (2.0f * v.focal[0]);
    const float lim_y = (1.3f * v.img[1]) / (2.0f * v.focal[1]);
    const float u = clampf(cam.x * inv_z, -lim_x, lim_x);
    const float vv = clampf(cam.y * inv_z, -lim_y, lim_y);
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
    // compute_conic (project.rs:224-232)
    const float det = maxf(ca * cc - cb * cb, 1e-6f);
    const float inv_det = 1.0f / det;
    const float cx = cc * inv_det, cy = -cb * inv_det, cz = ca * inv_det;

    // SH colour along the normalised view direction (project.rs:285-296)
    V3 dir{mean.x - v.world_pos[0], mean.y - v.world_pos[1], mean.z - v.world_pos[2]};
    const float inv = 1.0f / std::sqrt(dot3(dir, dir));
    dir = V3{dir.x * inv, dir.y * inv, dir.z * inv};
    float rgb[3];
    sh_to_rgb(sh_per_ch, dir, i, n, shs, rgb);

    const float mx = (v.focal[0] * cam.x) * inv_z + v.img[0] * 0.5f;
    const float my = (v.focal[1] * cam.y) * inv_z + v.img[1] * 0.5f;
    row[0] = mx; row[1] = my; row[2] = cx; row[3] = cy; row[4] = cz;
    row[5] = rgb[0] + 0.5f; row[6] = rgb[1] + 0.5f; row[7] = rgb[2] + 0.5f;
    row[8] = opacity;

    // Tile bbox (project.rs:37-46, 313-326)
    const float cutoff = logf_c(opacity / kAlphaCutoff);
    const float ext_x = std::sqrt((2.0f * cutoff) * ca);
    const float ext_y = std::sqrt((2.0f * cutoff) * cc);
    const float inv_tile = 1.0f / 16.0f;
    const uint32_t min_x = sat_u32(clampf((mx - ext_x) * inv_tile, 0.0f, v.tile_bounds[0]));
    const uint32_t min_y = sat_u32(clampf((my - ext_y) * inv_tile, 0.0f, v.tile_bounds[1]));
    const uint32_t max_x = sat_u32(clampf((mx + ext_x) * inv_tile + 1.0f, 0.0f, v.tile_bounds[0]));
    const uint32_t max_y = sat_u32(clampf((my + ext_y) * inv_tile + 1.0f, 0.0f, v.tile_bounds[1]));
    *count = (max_x - min_x) * (max_y - min_y);
    bb[0] = min_x | (min_y << 16);
    bb[1] = max_x | (max_y << 16);
    *key = f2u(cam.z);
    return true;
}

// Stable LSD radix sort of (key, value) pairs, 8-bit digits over `bits`.
void radix_pairs(std::vector<uint32_t>& k, std::vector<uint32_t>& v, uint32_t bits) {
    const size_t n = k.size();
    std::vector<uint32_t> k2(n), v2(n);
    for (uint32_t shift = 0; shift < bits; shift += 8) {
        size_t cnt[257] = {0};
        for (size_t i = 0; i < n; ++i) cnt[((k[i] >> shift) & 0xffu) + 1]++;
        for (int d = 0; d < 256; ++d) cnt[d + 1] += cnt[d];
        for (size_t i = 0; i < n; ++i) {
            const size_t p = cnt[(k[i] >> shift) & 0xffu]++;
            k2[p] = k[i];
            v2[p] = v[i];
        }
        k.swap(k2);
        v.swap(v2);
    }
}

}  // namespace

extern "C" int sfo_num_threads(void) { return omp_get_max_threads(); }
extern "C" void sfo_set_num_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }

extern "C" uint32_t sfo_project(const sfo_view* view, const float* attributes, const float* sh,
                                uint32_t n, uint32_t sh_per_ch, uint32_t* depth_keys,
                                uint32_t* tile_counts, uint32_t* bbox, float* projected,
                                uint64_t* total_isects) {
    uint64_t total = 0;
    uint32_t visible = 0;
#pragma omp parallel for schedule(static) reduction(+ : total, visible)
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        const uint32_t i = (uint32_t)ii;
        uint32_t key = 0xffffffffu, count = 0, bb[2] = {0, 0};
        float row[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (project_one(*view, attributes, sh, n, sh_per_ch, i, &key, &count, bb, row)) {
            visible += 1;
            total += count;
        }
        if (depth_keys) depth_keys[i] = key;
        if (tile_counts) tile_counts[i] = count;
        if (bbox) { bbox[2 * (size_t)i] = bb[0]; bbox[2 * (size_t)i + 1] = bb[1]; }
        if (projected) std::memcpy(projected + 9 * (size_t)i, row, sizeof(row));
    }
    if (total_isects) *total_isects = total;
    return visible;
}

extern "C" uint32_t sfo_depth_order(const uint32_t* depth_keys, uint32_t n, uint32_t* order) {
    std::vector<uint32_t> k, v;
    k.reserve(n);
    v.reserve(n);
    for (uint32_t i = 0; i < n; ++i) {
        if (depth_keys[i] != 0xffffffffu) { k.push_back(depth_keys[i]); v.push_back(i); }
    }
    radix_pairs(k, v, 32);
    std::memcpy(order, v.data(), v.size() * 4);
    return (uint32_t)v.size();
}

extern "C" uint64_t sfo_scan_gather(const uint32_t* gids, const uint32_t* counts, uint32_t n,
                                    uint32_t* offsets) {
    uint64_t running = 0;
    for (uint32_t r = 0; r < n; ++r) {
        offsets[r] = (uint32_t)running;
        running += counts[gids[r]];
    }
    return running;
}

extern "C" void sfo_emit(const uint32_t* order, const uint32_t* bbox, const uint32_t* offsets,
                         uint32_t num_visible, uint32_t tiles_per_row, uint32_t* tile_ids,
                         uint32_t* gaussian_ids) {
#pragma omp parallel for schedule(static)
    for (int64_t rr = 0; rr < (int64_t)num_visible; ++rr) {
        const uint32_t vis = order[rr];
        const uint32_t lo = bbox[2 * (size_t)vis], hi = bbox[2 * (size_t)vis + 1];
        size_t slot = offsets[rr];
        for (uint32_t ty = lo >> 16; ty < (hi >> 16); ++ty)
            for (uint32_t tx = lo & 0xffffu; tx < (hi & 0xffffu); ++tx) {
                tile_ids[slot] = tx + ty * tiles_per_row;
                gaussian_ids[slot] = vis;
                ++slot;
            }
    }
}

extern "C" void sfo_sort_pairs(const uint32_t* keys, const uint32_t* vals, uint32_t n,
                               uint32_t bits, uint32_t* keys_out, uint32_t* vals_out) {
    if (bits == 0 || n <= 1) {
        std::memmove(keys_out, keys, (size_t)n * 4);
        std::memmove(vals_out, vals, (size_t)n * 4);
        return;
    }
    const uint32_t mask = bits >= 32 ? 0xffffffffu : ((1u << bits) - 1u);
    // Stable sort on the masked key; the output carries the full key word.
    std::vector<uint32_t> idx(n);
    for (uint32_t i = 0; i < n; ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(),
                     [&](uint32_t a, uint32_t b) { return (keys[a] & mask) < (keys[b] & mask); });
    std::vector<uint32_t> ko(n), vo(n);
    for (uint32_t i = 0; i < n; ++i) { ko[i] = keys[idx[i]]; vo[i] = vals[idx[i]]; }
    std::memcpy(keys_out, ko.data(), (size_t)n * 4);
    std::memcpy(vals_out, vo.data(), (size_t)n * 4);
}

// Parallel stable counting sort by tile id (keys < num_tiles): each thread
// histograms a contiguous chunk, offsets run tile-major then chunk-major, so
// equal tiles keep input order.
static void tile_sort(const uint32_t* keys, const uint32_t* vals, size_t n, uint32_t num_tiles,
                      uint32_t* keys_out, uint32_t* vals_out) {
    const int max_nt = omp_get_max_threads();
    std::vector<size_t> hist((size_t)max_nt * num_tiles, 0);
#pragma omp parallel num_threads(max_nt)
    {
        const int nt = omp_get_num_threads();
        const int t = omp_get_thread_num();
        const size_t lo = n * t / nt, hi = n * (t + 1) / nt;
        size_t* hp = hist.data() + (size_t)t * num_tiles;
        for (size_t i = lo; i < hi; ++i) hp[keys[i]]++;
#pragma omp barrier
#pragma omp single
        {
            size_t running = 0;
            for (uint32_t k = 0; k < num_tiles; ++k)
                for (int tt = 0; tt < nt; ++tt) {
                    size_t& c = hist[(size_t)tt * num_tiles + k];
                    const size_t cc = c;
                    c = running;
                    running += cc;
                }
        }
        for (size_t i = lo; i < hi; ++i) {
            const size_t p = hp[keys[i]]++;
            keys_out[p] = keys[i];
            vals_out[p] = vals[i];
        }
    }
}

extern "C" void sfo_tile_ranges(const uint32_t* ids, uint32_t num_isects, uint32_t num_tiles,
                                uint32_t* ranges) {
    for (uint32_t t = 0; t < num_tiles; ++t) {
        ranges[2 * t] = (uint32_t)(std::lower_bound(ids, ids + num_isects, t) - ids);
        ranges[2 * t + 1] = (uint32_t)(std::lower_bound(ids, ids + num_isects, t + 1) - ids);
    }
}

extern "C" void sfo_rasterize(int mode, uint32_t w, uint32_t h, uint32_t row_stride,
                              const uint32_t* ranges, const uint32_t* gaussian_ids,
                              const float* projected, float scale, const uint32_t* mask,
                              uint32_t mask_words_per_row, uint32_t* bitmap, float* rgba_f32,
                              uint32_t* resp, uint32_t* fg, uint32_t* bg, float* final_t,
                              uint32_t* n_contrib) {
    const uint32_t tx_n = (w + 15) / 16, ty_n = (h + 15) / 16;
    const int64_t num_tiles = (int64_t)tx_n * ty_n;
    const float inv255 = 1.0f / 255.0f;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t tile = 0; tile < num_tiles; ++tile) {
        const uint32_t tx = (uint32_t)(tile % tx_n), ty = (uint32_t)(tile / tx_n);
        const uint32_t start = ranges[2 * tile], end = ranges[2 * tile + 1];
        for (uint32_t ly = 0; ly < 16; ++ly)
            for (uint32_t lx = 0; lx < 16; ++lx) {
                const uint32_t px = tx * 16 + lx, py = ty * 16 + ly;
                if (px >= w || py >= h) continue;
                const float pixel_x = (float)px + 0.5f, pixel_y = (float)py + 0.5f;
                uint32_t inside = 0;
                if (mode == 2) inside = (mask[px / 32 + py * mask_words_per_row] >> (px % 32)) & 1u;
                float T = 1.0f, pr = 0.0f, pg = 0.0f, pb = 0.0f;
                uint32_t last = 0;
                for (uint32_t j = start; j < end; ++j) {
                    const uint32_t gid = gaussian_ids[j];
                    const float* row = projected + 9 * (size_t)gid;
                    const float dx = row[0] - pixel_x, dy = row[1] - pixel_y;
                    const float hx = 0.5f * row[2], hz = 0.5f * row[4];
                    const float power = std::fma(hx * dx, dx, std::fma(hz * dy, dy, (row[3] * dx) * dy));
                    const float alpha = minf(row[8] * expf_c(-power), 0.999f);
                    if (!(alpha >= inv255)) continue;
                    const float vis = alpha * T;
                    if (mode == 0) {
                        pr = std::fma(row[5], vis, pr);
                        pg = std::fma(row[6], vis, pg);
                        pb = std::fma(row[7], vis, pb);
                    } else {
                        const uint32_t q = sat_u32(vis * scale);
                        if (mode == 2) {
                            if (inside) {
#pragma omp atomic
                                fg[gid] += q;
                            } else {
#pragma omp atomic
                                bg[gid] += q;
                            }
                        } else {
#pragma omp atomic
                            resp[gid] += q;
                        }
                    }
                    T = T * (1.0f - alpha);
                    last = j - start + 1;
                    if (T < inv255) break;
                }
                const size_t pix = (size_t)py * w + px;
                if (mode == 0) {
                    if (bitmap) {
                        const uint32_t r = sat_u32(clampf(pr * 255.0f, 0.0f, 255.0f));
                        const uint32_t g = sat_u32(clampf(pg * 255.0f, 0.0f, 255.0f));
                        const uint32_t b = sat_u32(clampf(pb * 255.0f, 0.0f, 255.0f));
                        const uint32_t a = sat_u32(clampf((1.0f - T) * 255.0f, 0.0f, 255.0f));
                        bitmap[(size_t)py * row_stride + px] = r | (g << 8) | (b << 16) | (a << 24);
                    }
                    if (rgba_f32) {
                        rgba_f32[4 * pix + 0] = pr;
                        rgba_f32[4 * pix + 1] = pg;
                        rgba_f32[4 * pix + 2] = pb;
                        rgba_f32[4 * pix + 3] = 1.0f - T;
                    }
                }
                if (final_t) final_t[pix] = T;
                if (n_contrib) n_contrib[pix] = last;
            }
    }
}

extern "C" int sfo_prepare(const sfo_camera* cam, uint32_t w, uint32_t h, const float* attributes,
                           const float* sh, uint32_t n, uint32_t sh_per_ch, uint32_t* depth_keys,
                           uint32_t* tile_counts, uint32_t* bbox, float* projected,
                           uint32_t* order, uint32_t* offsets, uint32_t* tile_ids,
                           uint32_t* gaussian_ids, uint64_t isect_capacity, uint32_t* ranges,
                           sfo_frame_info* out) {
    sfo_view view;
    sfo_view_for_camera(cam, w, h, &view);
    const uint32_t tx = (w + 15) / 16, ty = (h + 15) / 16;
    uint64_t total = 0;
    sfo_project(&view, attributes, sh, n, sh_per_ch, depth_keys, tile_counts, bbox, projected,
                &total);
    const uint32_t V = sfo_depth_order(depth_keys, n, order);
    const uint64_t I = sfo_scan_gather(order, tile_counts, V, offsets);
    out->num_visible = V;
    out->num_isects = I;
    out->tiles_x = tx;
    out->tiles_y = ty;
    out->row_stride = ((4 * w + 255) / 256 * 256) / 4;
    if (I > isect_capacity) return -1;
    std::vector<uint32_t> t_ids(I), g_ids(I);
    sfo_emit(order, bbox, offsets, V, tx, t_ids.data(), g_ids.data());
    tile_sort(t_ids.data(), g_ids.data(), I, tx * ty, tile_ids, gaussian_ids);
    sfo_tile_ranges(tile_ids, (uint32_t)I, tx * ty, ranges);
    return 0;
}
