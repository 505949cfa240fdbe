/* Oracle C interface (TEST INFRASTRUCTURE ONLY: the CPU checker for the CUDA
 * splat path, also timed as the CPU baseline; never part of the product).
 *
 * Every function restates one piece of the reference suous/splatfield v0.2.0
 * (Rust/cubecl); the comment beside each names the reference file:line it
 * follows. Layouts are the reference's:
 *   attributes  field-major, plane k of splat i at k*n+i, planes
 *               [x,y,z,qw,qx,qy,qz,sx,sy,sz,opacity]      (src/layout.rs:44-58)
 *   sh          field-major, coefficient k channel c of splat i at (k*3+c)*n+i
 *               (src/project.rs:344-388)
 *   projected   9 floats per splat [mean.xy, conic.xyz, rgb+0.5, opacity]
 *               (src/layout.rs:60-61)
 *   bbox        2 words per splat, min_x|min_y<<16, max_x|max_y<<16
 *               (src/project.rs:324-326)
 */
#ifndef SFO_H
#define SFO_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Camera{fov, position, rotation} (src/camera.rs:5-9); rotation is a glam
 * quaternion stored x, y, z, w. */
typedef struct {
    float fov[2];
    float position[3];
    float rotation[4];
} sfo_camera;

/* CameraView kernel scalars (src/project.rs:63-96). */
typedef struct {
    float rot0[3], rot1[3], rot2[3];
    float trans[3];
    float focal[2];
    float world_pos[3];
    float img[2];
    float tile_bounds[2];
} sfo_view;

/* ---- camera math (src/camera.rs:38-63; glam 0.33.6 restated) ---- */
void sfo_camera_look_at(const float position[3], const float target[3], sfo_camera* out);
void sfo_view_for_camera(const sfo_camera* cam, uint32_t w, uint32_t h, sfo_view* out);

/* ---- FP32 pipeline pieces ---- */
/* project_splats (src/project.rs:235-327). Writes, per splat i: depth_keys[i]
 * (f32 bits of camera z, 0xFFFFFFFF if culled), tile_counts[i] (0 if culled),
 * bbox[2i..2i+1] (0 if culled), projected[9i..9i+8] (0 if culled). Returns the
 * visible count; *total_isects gets the sum of tile counts. Any output may be
 * NULL. */
uint32_t sfo_project(const sfo_view* view, const float* attributes, const float* sh,
                     uint32_t n, uint32_t sh_per_ch, uint32_t* depth_keys,
                     uint32_t* tile_counts, uint32_t* bbox, float* projected,
                     uint64_t* total_isects);

/* Stable depth order of the visible splats: ascending (depth key, splat id)
 * (src/render.rs:310-316; ties ordered by splat id). Returns V. */
uint32_t sfo_depth_order(const uint32_t* depth_keys, uint32_t n, uint32_t* order);

/* exclusive_scan_gather (crates/sort/src/scan.rs:219-255):
 * offsets[r] = sum_{r'<r} counts[gids[r']] (u32 wrap). Returns the 64-bit total. */
uint64_t sfo_scan_gather(const uint32_t* gids, const uint32_t* counts, uint32_t n,
                         uint32_t* offsets);

/* map_isects (src/raster.rs:13-48) without truncation. */
void sfo_emit(const uint32_t* order, const uint32_t* bbox, const uint32_t* offsets,
              uint32_t num_visible, uint32_t tiles_per_row, uint32_t* tile_ids,
              uint32_t* gaussian_ids);

/* Stable argsort by key (crates/sort/src/sort.rs:311-380) of n (key, value)
 * pairs using the low `bits` key bits. */
void sfo_sort_pairs(const uint32_t* keys, const uint32_t* vals, uint32_t n,
                    uint32_t bits, uint32_t* keys_out, uint32_t* vals_out);

/* Per-tile [start, end) over sorted tile ids: lower_bound pairs
 * (src/raster.rs:53-65, 114-115). ranges holds 2 words per tile. */
void sfo_tile_ranges(const uint32_t* sorted_tile_ids, uint32_t num_isects,
                     uint32_t num_tiles, uint32_t* ranges);

/* rasterize_kernel (src/raster.rs:88-230). mode 0 = RGB (bitmap packed RGBA8
 * with row_stride words per row, optional float RGBA plane rgba_f32 [h*w*4]),
 * 1 = total responsibility into resp, 2 = evidence split into fg/bg by mask.
 * final_t / n_contrib (optional, h*w) record each pixel's final
 * transmittance and the 1-based position of its last contributor in its
 * tile's range. Accumulators are added to (the caller clears them). */
void sfo_rasterize(int mode, uint32_t w, uint32_t h, uint32_t row_stride,
                   const uint32_t* ranges, const uint32_t* gaussian_ids,
                   const float* projected, float scale, const uint32_t* mask,
                   uint32_t mask_words_per_row, uint32_t* bitmap, float* rgba_f32,
                   uint32_t* resp, uint32_t* fg, uint32_t* bg, float* final_t,
                   uint32_t* n_contrib);

/* Whole frame, every intermediate exposed (src/render.rs:274-460). Buffers:
 * depth_keys, tile_counts [n]; bbox [2n]; projected [9n]; order, offsets [n];
 * tile_ids/gaussian_ids (sorted) [isect_capacity]; ranges [2*tiles]. Returns
 * 0, or -1 if the intersections exceed isect_capacity (out->num_isects still
 * reports the count). */
typedef struct {
    uint32_t num_visible;
    uint64_t num_isects;
    uint32_t tiles_x, tiles_y;
    uint32_t row_stride;
} sfo_frame_info;

int sfo_prepare(const sfo_camera* cam, uint32_t w, uint32_t h, const float* attributes,
                const float* sh, uint32_t n, uint32_t sh_per_ch, uint32_t* depth_keys,
                uint32_t* tile_counts, uint32_t* bbox, float* projected, uint32_t* order,
                uint32_t* offsets, uint32_t* tile_ids, uint32_t* gaussian_ids,
                uint64_t isect_capacity, uint32_t* ranges, sfo_frame_info* out);

/* ---- segmentation math (src/seg/mod.rs, src/seg/beta.rs) ---- */
uint32_t sfo_fractional_bits(uint32_t w, uint32_t h);          /* seg/mod.rs:31-34 */
float sfo_scale_for(uint32_t w, uint32_t h);                    /* seg/mod.rs:178 */
uint32_t sfo_mask_pack(const uint8_t* bytes, uint32_t w, uint32_t h, uint32_t* bits); /* seg/mod.rs:118-143; returns fg pixels */
double sfo_lgamma(double x);                                    /* beta.rs:55-73 */
double sfo_digamma(double x);                                   /* beta.rs:77-86 */
double sfo_beta_entropy(double a, double b);                    /* beta.rs:92-96 */
void sfo_entropy_table(float* table);                           /* beta.rs:100-112, 445*445 */
float sfo_table_entropy(float a, float b, const float* table);  /* beta.rs:128-144 */
/* Per-splat f32 LUT delta (entropy_delta_kernel body, beta.rs:166-189). */
float sfo_delta_lut(float a, float b, uint32_t resp_bits, float scale, const float* table);
/* The same delta in f64 from the f64 formulas (no LUT). */
double sfo_delta_f64(float a, float b, uint32_t resp_bits, float scale);
/* EIG = sum of deltas, summed in f64. mode 0 = f32 LUT deltas, 1 = f64. */
double sfo_eig(int mode, const float* a, const float* b, const uint32_t* resp, uint32_t n,
               float scale, const float* table);
/* beta_update_kernel (beta.rs:206-212), in place. */
void sfo_beta_update(float scale, const uint32_t* fg, const uint32_t* bg, float* a, float* b,
                     uint32_t n);

/* ---- FP64 twin and adjoint (no reference counterpart) ---- */
/* Same pipeline in double with libm exp/log: float RGBA [h*w*4]. */
int sfo64_render(const sfo_camera* cam, uint32_t w, uint32_t h, const double* attributes,
                 const double* sh, uint32_t n, uint32_t sh_per_ch, double* rgba);
/* L = sum(dl_drgba * rgba) over pixels of the FP64 render (alpha = 1 - T);
 * writes dL/d(attributes) [11n] and dL/d(sh) [3*K*n]. */
int sfo64_render_backward(const sfo_camera* cam, uint32_t w, uint32_t h,
                          const double* attributes, const double* sh, uint32_t n,
                          uint32_t sh_per_ch, const double* dl_drgba, double* d_attr,
                          double* d_sh);
/* FP64 L2 loss over a tile region with one parameter of one splat replaced
 * (central differences on large scenes; sfo_grad.cpp). */
void* sfo64_probe_open(const sfo_camera* cam, uint32_t w, uint32_t h, const double* attributes,
                       const double* sh, uint32_t n, uint32_t K, const double* target_rgba);
void sfo64_probe_close(void* handle);
int sfo64_probe_bbox(void* handle, uint32_t i, uint32_t out[2]);
double sfo64_probe_loss(void* handle, uint32_t i, uint32_t param, double value, uint32_t tx0, uint32_t ty0,
                        uint32_t tx1, uint32_t ty1);

/* threads the OpenMP regions use */
int sfo_num_threads(void);
void sfo_set_num_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
