/* splatfield_cuda.h — C ABI of the B200 (sm_100a) splat render +
 * segmentation-evidence path.
 *
 * Drop-in for the GPU path of suous/splatfield v0.2.0 (Rust crate API; the
 * reference has no FFI, so each entry point below names the Rust item it
 * replaces, as path:line in that project). A Rust caller binds these through a
 * thin `extern "C"` crate; the Python package `splatfield_b200` binds them
 * with ctypes.
 *
 * Conventions
 *  - Every call returns an int status: SF_OK (0) or an SF_ERR_* code; the
 *    message of the last failure on the calling thread is sf_last_error().
 *    No exception crosses the ABI.
 *  - `sf_stream` is a cudaStream_t (NULL = the legacy default stream). Work is
 *    ordered on that stream; a call returns after enqueuing unless noted
 *    ("syncs") — the reference likewise blocks once per frame on its counters
 *    readback (src/render.rs:308).
 *  - Handles are not thread-safe: serialise each handle on one stream, as the
 *    reference serialises everything on one ordered stream (src/lib.rs:20-27).
 *  - Device pointers returned by a handle alias that handle's storage and stay
 *    valid until the handle's next call of the same kind or its destruction
 *    (the reference's returned tensors alias scratch the same way,
 *    src/render.rs:366-368, crates/sort/src/sort.rs:278-281).
 *  - Layouts are the reference's: attributes field-major, plane k of splat i
 *    at k*n+i, planes [x,y,z,qw,qx,qy,qz,sx,sy,sz,opacity] (src/layout.rs:44-58);
 *    SH coefficient k, channel c of splat i at (k*3+c)*n+i (src/project.rs:344-388);
 *    RGBA8 pixels r|g<<8|b<<16|a<<24 with row_stride words per row
 *    (src/raster.rs:223-229, src/render.rs:150); masks bit-packed LSB-first,
 *    ceil(w/32) words per row (src/seg/mod.rs:105-143).
 */
#ifndef SPLATFIELD_CUDA_H
#define SPLATFIELD_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SF_ABI_VERSION 1

enum {
    SF_OK = 0,
    SF_ERR_ARG = 1,       /* null handle/pointer, bad enum */
    SF_ERR_SHAPE = 2,     /* sizes inconsistent (e.g. zero splats, n > capacity) */
    SF_ERR_CAPACITY = 3,  /* intersections exceed a fixed capacity (graph rounds) */
    SF_ERR_TIMEOUT = 4,   /* a bounded device spin-wait gave up */
    SF_ERR_CUDA = 5,      /* CUDA runtime error */
    SF_ERR_NOMEM = 6      /* device allocation failed */
};

typedef void* sf_stream; /* cudaStream_t */
typedef struct sf_ctx_t* sf_ctx;
typedef struct sf_splats_t* sf_splats;
typedef struct sf_scratch_t* sf_scratch;
typedef struct sf_accum_t* sf_accum;
typedef struct sf_mask_t* sf_mask;
typedef struct sf_beta_t* sf_beta;
typedef struct sf_radix_t* sf_radix;
typedef struct sf_scan_t* sf_scan;

/* Camera{fov, position, rotation} (src/camera.rs:5-9); rotation is a unit
 * quaternion stored x, y, z, w (glam order). */
typedef struct {
    float fov[2];
    float position[3];
    float rotation[4];
} sf_camera;

/* CameraView kernel scalars (src/project.rs:63-74), built by
 * CameraViewLaunch::for_camera (src/project.rs:76-96). */
typedef struct {
    float rot0[3], rot1[3], rot2[3];
    float trans[3];
    float focal[2];
    float world_pos[3];
    float img[2];
    float tile_bounds[2];
} sf_view;

/* TileIsects (src/render.rs:463-471), device pointers into the scratch. */
typedef struct {
    const uint32_t* tile_ids;     /* sorted tile id per intersection [num_isects] */
    const uint32_t* gaussian_ids; /* splat id per intersection, tile-major depth-minor */
    const uint32_t* tile_start;   /* [tiles+1]: tile t's run is [start[t], start[t+1]) */
    uint32_t num_isects;
    uint32_t num_visible;
    uint32_t tile_bounds[2];
    uint32_t row_stride;
} sf_isects;

/* ---------------------------------------------------------------- runtime */
const char* sf_last_error(void);
int sf_abi_version(void);
/* Number of kernels this library has launched in this process (all
 * devices, all handles); a diagnostic for launch accounting. */
uint64_t sf_kernel_launches(void);
/* Context on one CUDA device; holds the entropy LUT and device properties. */
int sf_ctx_create(int device, sf_ctx* out);
int sf_ctx_destroy(sf_ctx ctx);
/* Plain device buffers for callers without CUDA bindings of their own. */
int sf_buffer_alloc(sf_ctx ctx, size_t bytes, void** dptr);
int sf_buffer_free(sf_ctx ctx, void* dptr);
int sf_memcpy_htod(void* dst_dev, const void* src_host, size_t bytes, sf_stream stream);
int sf_memcpy_dtoh(void* dst_host, const void* src_dev, size_t bytes, sf_stream stream);
int sf_memset(void* dst_dev, int value, size_t bytes, sf_stream stream);
int sf_stream_sync(sf_stream stream);
/* Page-locked host memory, for overlapped copies. */
int sf_host_alloc(size_t bytes, void** hptr);
int sf_host_free(void* hptr);

/* ----------------------------------------------------------- camera math */
/* Camera::look_at (src/camera.rs:57-63): minimal arc from +Z, fov 0.8 rad. */
int sf_camera_look_at(const float position[3], const float target[3], sf_camera* out);
/* Camera::focal (src/camera.rs:38-40). */
int sf_camera_focal(const sf_camera* cam, uint32_t w, uint32_t h, float out[2]);
/* CameraViewLaunch::for_camera (src/project.rs:76-96). */
int sf_view_for_camera(const sf_camera* cam, uint32_t w, uint32_t h, sf_view* out);

/* ---------------------------------------------------------------- splats */
/* Splats::new / CpuSplats::upload (src/render.rs:31-33, 242-269): uploads
 * field-major attributes [11*n] and SH [3*sh_per_ch*n] from host memory;
 * n must be > 0 (the reference asserts it) and sh_per_ch >= 1; colour reads
 * the largest whole SH degree the coefficients hold (1, 4, 9 or 16 per
 * channel, src/project.rs:343-388), like the reference. */
int sf_splats_create(sf_ctx ctx, const float* attributes, const float* sh, uint32_t n,
                     uint32_t sh_per_ch, sf_splats* out);
int sf_splats_destroy(sf_splats s);
/* Splat count, SH coefficients per channel, bounds (min xyz, max xyz) and the
 * device planes. */
int sf_splats_info(sf_splats s, uint32_t* n, uint32_t* sh_per_ch, float bounds[6],
                   const float** attributes_dev, const float** sh_dev);

/* --------------------------------------------------------------- scratch */
/* RenderScratch::new (src/render.rs:144-167): per-frame buffers for `total`
 * splats at w x h, reused across frames; rebuilt in place when a frame's shape
 * differs (src/render.rs:171-197). Intersection capacity grows to the exact
 * scan total before emission, so nothing is truncated. */
int sf_scratch_create(sf_ctx ctx, uint32_t total, uint32_t w, uint32_t h, sf_scratch* out);
int sf_scratch_destroy(sf_scratch s);
/* Current intersection capacity (entries). */
int sf_scratch_capacity(sf_scratch s, uint64_t* capacity);
/* Grows the intersection capacity ahead of time to at least `isects`
 * entries (the next power of two), so frames up to that size never
 * reallocate; the capacity never shrinks. */
int sf_scratch_reserve(sf_scratch s, uint64_t isects);

/* Kernel forms a scratch launches; all forms give identical results (the
 * autotuner picks by measured time). */
typedef struct {
    uint32_t raster_cull; /* 0: every warp walks every staged entry;
                             1: per-warp culling by each splat's power_max box,
                             then by the minimum of its quadratic form over
                             the warp's 8x4 pixel block */
    /* Intersection build, same lists either way:
     *   SF_ISECTS_BINNED (default, frames up to 49152 tiles): per-tile
     *     counts in shared memory, place, then a sort of each tile's list by
     *     (depth, id) (in shared memory up to 12288 entries);
     *   SF_ISECTS_DEPTH_SORTED: the reference's order of steps
     *     (src/render.rs:318-352): depth argsort, gather scan, emit, stable
     *     tile sort; keeps the depth order and offsets for sf_scratch_read. */
    uint32_t isect_build;
    /* 1: the rasterizer also counts out[1..3] of sf_scratch_stats (a slower
     * diagnostic form); 0 (default): only out[0]. */
    uint32_t raster_detail;
    /* Tile-list order for the render calls that hand no lists back
     * (sf_render_with / _float / _to_host / _posterior /
     * sf_render_responsibility, the round), binned build only:
     *   SF_ORDER_SORTED (default): every tile list is sorted first;
     *   SF_ORDER_IN_RASTER: the rasterizer orders each tile's placed pairs
     *     slab by slab, only as far as the tile saturates;
     *   SF_ORDER_HYBRID: lists of up to 12288 entries are sorted, longer
     *     ones are ordered in the rasterizer.
     * Same results either way. sf_prepare_isects and sf_render_forward always
     * sort (their lists are handed out or replayed). */
    uint32_t raster_order;
    /* Block schedule of the rasterizer for binned RGB frames
     * (sf_render_with / _to_host, sf_render_frames / _frames_to_host):
     *   SF_SCHEDULE_LONGEST (default): blocks take the tiles by list size
     *     class, longest first, so the longest walks do not trail the grid;
     *   SF_SCHEDULE_TILES: block i takes tile i. */
    uint32_t raster_schedule;
    /* Rasterizer CTAs per 16x16 tile: 0 or 1 (default), one CTA of 8 warps;
     * 2 or 4: CTAs of 4 or 2 warps, each walking the tile's whole list for
     * its part of the pixels (a long unsaturated list is then walked on
     * several SMs at once). The intersection tiles stay 16x16, so results
     * are unchanged. */
    uint32_t raster_split;
    /* Digit width of the depth-sorted build's onesweep sorts, 4..8 bits per
     * pass (0: 8). Same order either way; narrower digits take more passes
     * with fewer bins each. */
    uint32_t radix_bits;
    /* Frame pipes of the camera-path calls (sf_render_frames / _to_host):
     * 0 or 2 (default): frames alternate between the scratch and a second,
     * internal copy of its frame buffers, each with its own frame graph and
     * stream, so one frame's projection and build run while the other's
     * raster finishes (the copy is allocated on the first path of two or
     * more frames and holds the scratch's capacity; when the device has no
     * room for it, the path runs on one pipe); 1: one pipe. Same images
     * either way. */
    uint32_t frame_pipes;
} sf_tuning;
#define SF_ISECTS_BINNED 0u
#define SF_ISECTS_DEPTH_SORTED 1u
#define SF_ORDER_SORTED 0u
#define SF_ORDER_IN_RASTER 1u
#define SF_ORDER_HYBRID 2u
#define SF_SCHEDULE_LONGEST 0u
#define SF_SCHEDULE_TILES 1u
int sf_scratch_set_tuning(sf_scratch s, const sf_tuning* t);
int sf_scratch_get_tuning(sf_scratch s, sf_tuning* t);
/* Frame autotuner (no counterpart in the reference): times sf_render_frames
 * over cams[count] at w x h for each raster form in a coordinate search (two
 * sweeps over raster_cull {0,1}, raster_split {1,2,4}, raster_order {sorted,
 * hybrid, in-raster}, raster_schedule {longest, tiles} and frame_pipes
 * {2, 1}; best of three
 * paths after a warm-up path), keeps the fastest on the scratch and returns
 * it with its time per frame. Images are the same in every form. */
int sf_scratch_autotune(sf_splats s, sf_scratch scratch, const sf_camera* cams, uint32_t count, uint32_t w,
                        uint32_t h, sf_stream stream, sf_tuning* best, double* best_ms);

/* ---------------------------------------------------------------- render */
/* Splats::render_with (src/render.rs:371-380): one RGBA8 frame. Syncs once
 * (intersection total). *bitmap receives a device pointer [h][row_stride]
 * aliasing the scratch, valid until the next render on it. */
int sf_render_with(sf_splats s, sf_scratch scratch, const sf_camera* cam, uint32_t w, uint32_t h,
                   sf_stream stream, const uint32_t** bitmap, uint32_t* row_stride);
/* Splats::render_posterior (src/seg/paint.rs:22-47): the frame with every
 * splat painted grey by its posterior mean a / (a + b) (no +0.5 offset). A
 * posterior of another size renders the plain colours, as the reference. */
int sf_render_posterior(sf_splats s, sf_scratch scratch, sf_beta beta, const sf_camera* cam,
                        uint32_t w, uint32_t h, sf_stream stream, const uint32_t** bitmap,
                        uint32_t* row_stride);
/* Splats::tint (src/seg/paint.rs:49-66): DC colour (r, g, b) for every
 * foreground splat (a > b), in place. */
int sf_splats_tint(sf_splats s, sf_beta beta, float r, float g, float b, sf_stream stream);
/* Splats::save_colors / restore_colors (src/seg/paint.rs:68-95): the three
 * DC planes (3 n floats) to / from a device buffer, on the copy engine. */
int sf_splats_save_colors(sf_splats s, float* dst, sf_stream stream);
int sf_splats_restore_colors(sf_splats s, const float* src, sf_stream stream);
/* The same frame with a float RGBA plane [h][w][4] (r, g, b, 1-T before
 * quantisation) in addition to the RGBA8 bitmap. */
int sf_render_float(sf_splats s, sf_scratch scratch, const sf_camera* cam, uint32_t w, uint32_t h,
                    sf_stream stream, const float** rgba);
/* render_with plus the read-back: packed RGBA8 rows [h][w] (stride removed)
 * written to host memory `out`; syncs. */
int sf_render_to_host(sf_splats s, sf_scratch scratch, const sf_camera* cam, uint32_t w,
                      uint32_t h, sf_stream stream, uint32_t* out);
/* `count` frames, camera cams[i] to out + i * w * h (packed RGBA8 rows
 * [h][w], as sf_render_to_host writes them); syncs once at the end. Each
 * image leaves the device (from a staging copy, on a stream of its own)
 * while the next frame renders, so the read-backs overlap the rendering when
 * `out` is pinned host memory. The images equal `count` sf_render_to_host
 * calls; frames past the intersection capacity are rendered again after it
 * has grown. The scratch is left holding the last frame. A camera path over
 * the reference's per-frame render_with (src/render.rs:371-380). */
int sf_render_frames_to_host(sf_splats s, sf_scratch scratch, const sf_camera* cams, uint32_t count,
                             uint32_t w, uint32_t h, sf_stream stream, uint32_t* out);
/* `count` frames, as `count` sf_render_with calls, enqueued back to back
 * with one sync at the end (each frame's intersection total is checked
 * then; frames past the capacity are rendered again after it has grown).
 * The last frame's image is the scratch's bitmap (sf_scratch_buffers). */
int sf_render_frames(sf_splats s, sf_scratch scratch, const sf_camera* cams, uint32_t count, uint32_t w,
                     uint32_t h, sf_stream stream);
/* Adjoint (no counterpart in the reference, which renders forward only).
 * sf_render_forward: sf_render_float that also keeps, per pixel, the final
 * transmittance and the position of the last contributor, for the backward.
 * sf_render_backward: for L = sum_p <dl_drgba[p], rgba[p]> (dl_drgba: device
 * [h][w][4]) of that forward (same camera and size, nothing rendered on the
 * scratch in between), writes dL/d(attributes) [11*n] and dL/d(sh)
 * [3*sh_per_ch*n] to device memory, field-major like the inputs. d_proj
 * (device [n][9], may be NULL) receives the per-splat 2D adjoint
 * (mean2d xy, conic xyz, colour rgb, opacity); its colour entries with
 * dl_drgba = (m, 1-m, 1, 0) are the real-valued mask/background/total
 * responsibilities sum_p m_p alpha T. */
int sf_render_forward(sf_splats s, sf_scratch scratch, const sf_camera* cam, uint32_t w, uint32_t h,
                      sf_stream stream, const float** rgba);
int sf_render_backward(sf_splats s, sf_scratch scratch, const sf_camera* cam, uint32_t w, uint32_t h,
                       const float* dl_drgba, float* d_attr, float* d_sh, float* d_proj,
                       sf_stream stream);
/* Adjoint of a per-splat scalar feature (no counterpart in the reference,
 * whose evidence lift is the u32 rasterizer, src/raster.rs:194-211): for the
 * feature render F(p) = sum_i f_i alpha_i T_i(p), dL/df_i with dL/dF(p) =
 * mask(p) into fg[i] and with dL/dF(p) = 1 - mask(p) into bg[i] (device
 * [n] floats; mask NULL: all of it in fg) — the real-valued mask and
 * background responsibilities sum_p m_p alpha_i T_i(p), which the u32 lift
 * truncates per pixel to (u32)(alpha T scale). A transmittance-only forward
 * keeps each pixel's final T and last contributor; the adjoint replays the
 * sorted lists back to front from them. Float sums, added in no fixed order.
 * Syncs once (the intersection total). Overwrites an sf_render_forward's
 * state on the scratch. */
int sf_render_feature_adjoint(sf_splats s, sf_scratch scratch, const sf_camera* cam, uint32_t w, uint32_t h,
                              sf_mask mask, sf_stream stream, float* fg, float* bg);

/* Splats::prepare_isects (src/render.rs:274-364): project, depth sort, gather
 * scan, emit, stable tile sort, tile ranges. Syncs once. */
int sf_prepare_isects(sf_splats s, sf_scratch scratch, const sf_camera* cam, uint32_t w, uint32_t h,
                      sf_stream stream, sf_isects* out);
/* Splats::finalize(Finalize::Rgb) (src/render.rs:387-460) over prepared
 * intersections; optionally also the float plane. */
int sf_finalize_rgb(sf_splats s, sf_scratch scratch, const sf_isects* isects, uint32_t w,
                    uint32_t h, int want_float, sf_stream stream);

/* The scratch's frame outputs (device pointers; rgba is NULL until a float
 * render ran). */
int sf_scratch_buffers(sf_scratch s, const uint32_t** bitmap, const float** rgba,
                       uint32_t* row_stride);

/* Pair statistics of the scratch's last rasterization (syncs): out[0] =
 * (pixel, splat) pairs visited (256 per tile-list entry walked before the
 * tile's early exit); with sf_tuning.raster_detail = 1 also out[1] =
 * exponentials evaluated, out[2] = contributing pairs (alpha >= 1/255),
 * out[3] = pairs processed (32 per warp-entry step the warps ran); else
 * zero. */
int sf_scratch_stats(sf_scratch s, uint64_t out[4], sf_stream stream);

/* Intermediates of the last prepare, copied to host (syncs), for parity
 * checks and debugging. `what`: */
enum {
    SF_READ_DEPTH_KEYS = 0,  /* u32 [total]: f32 bits of camera z, 0xFFFFFFFF culled */
    SF_READ_TILE_COUNTS = 1, /* u32 [total] */
    SF_READ_BBOX = 2,        /* u32 [2*total] packed min/max */
    SF_READ_PROJECTED = 3,   /* f32 [9*total] reference row [mean.xy, conic.xyz, rgb, opacity] */
    SF_READ_ORDER = 4,       /* u32 [num_visible] depth order */
    SF_READ_OFFSETS = 5,     /* u32 [num_visible] gather-scan offsets */
    SF_READ_TILE_IDS = 6,    /* u32 [num_isects] sorted */
    SF_READ_GAUSSIAN_IDS = 7,/* u32 [num_isects] sorted */
    SF_READ_TILE_START = 8,  /* u32 [tiles+1] */
    SF_READ_BITMAP = 9,      /* u32 [h*row_stride] */
    SF_READ_RGBA = 10,       /* f32 [h*w*4] */
    SF_READ_FINAL_T = 11,    /* f32 [h*w] */
    SF_READ_N_CONTRIB = 12   /* u32 [h*w] */
};
int sf_scratch_read(sf_scratch s, int what, void* host, size_t bytes, sf_stream stream);

/* ------------------------------------------------------ responsibility / evidence */
/* Accumulators::new (src/seg/mod.rs:62-69): u32 fixed-point resp/fg/bg [total]. */
int sf_accum_create(sf_ctx ctx, uint32_t total, sf_accum* out);
int sf_accum_destroy(sf_accum a);
/* The current fixed-point scale and the device arrays. */
int sf_accum_info(sf_accum a, float* scale, const uint32_t** resp, const uint32_t** fg,
                  const uint32_t** bg);
/* Set the fixed-point scale (the render paths set it from the frame size;
 * the reference's tests build accumulators with an explicit scale,
 * src/seg/beta.rs:351-359). */
int sf_accum_set_scale(sf_accum a, float scale);
/* Mask::from_bytes (src/seg/mod.rs:118-143): one byte per pixel, nonzero =
 * foreground; packs and uploads. *fg_pixels gets the foreground count. */
int sf_mask_create(sf_ctx ctx, uint32_t w, uint32_t h, const uint8_t* bytes, sf_mask* out,
                   uint32_t* fg_pixels);
/* A mask already packed (u32 words [h*ceil(w/32)], host memory). */
int sf_mask_create_packed(sf_ctx ctx, uint32_t w, uint32_t h, const uint32_t* words, sf_mask* out);
int sf_mask_destroy(sf_mask m);
/* Splats::render_responsibility (src/seg/mod.rs:150-159): clears resp and
 * accumulates eps_i = sum_p trunc(alpha*T*scale). Syncs once. */
int sf_render_responsibility(sf_splats s, sf_scratch scratch, sf_accum acc, const sf_camera* cam,
                             uint32_t w, uint32_t h, sf_stream stream);
/* Splats::accumulate_prepared (src/seg/mod.rs:170-210): over intersections
 * already prepared for this camera and size; mask NULL = total
 * responsibility, else the fg/bg evidence split. */
int sf_accumulate_prepared(sf_splats s, sf_scratch scratch, const sf_isects* isects, uint32_t w,
                           uint32_t h, sf_accum acc, sf_mask mask, sf_stream stream);
/* fractional_bits (src/seg/mod.rs:31-34) and the scale 2^bits. */
uint32_t sf_fractional_bits(uint32_t w, uint32_t h);

/* ------------------------------------------------------------ Beta / EIG */
enum { SF_EIG_LUT_F32 = 0, SF_EIG_FP64 = 1 };
/* BetaState::new_uniform (src/seg/beta.rs:230-238): a = b = 1. */
int sf_beta_create_uniform(sf_ctx ctx, uint32_t total, sf_beta* out);
/* A posterior from host arrays (the reference's test `state`, beta.rs:302-310). */
int sf_beta_create(sf_ctx ctx, const float* a, const float* b, uint32_t n, sf_beta* out);
int sf_beta_destroy(sf_beta beta);
int sf_beta_read(sf_beta beta, float* a, float* b, sf_stream stream);
int sf_beta_info(sf_beta beta, uint32_t* n, float** a_dev, float** b_dev);
/* BetaState::eig (src/seg/beta.rs:241-268): EIG = sum_i dH_i for the accumulator's
 * responsibility: its ε words, or fg + bg when its last fill was a masked
 * sf_accumulate_prepared (the same words, src/seg/tests.rs:208-227).
 * mode SF_EIG_LUT_F32 reads the f32 445x445 log-spaced LUT
 * (beta.rs:128-201); SF_EIG_FP64 evaluates the f64 lgamma/digamma entropy on
 * the GPU. Reduced on the device in f64 (no partials read-back); syncs. */
int sf_beta_eig(sf_beta beta, sf_accum acc, int mode, sf_stream stream, double* eig);
/* Asynchronous form: the EIG lands in device memory `eig_dev` (one double). */
int sf_beta_eig_async(sf_beta beta, sf_accum acc, int mode, double* eig_dev, sf_stream stream);
/* BetaState::update (src/seg/beta.rs:273-286): a += fg/scale, b += bg/scale. */
int sf_beta_update(sf_beta beta, sf_accum acc, sf_stream stream);
/* The EIG (beta.rs:152-201) and the Beta update (beta.rs:206-212) over
 * real-valued responsibilities (sf_render_feature_adjoint,
 * sf_round_adjoint_responsibility; device [n] floats): eps = fg + bg (bg
 * may be NULL for the EIG), a += fg, b += bg. The EIG syncs. */
int sf_beta_eig_real(sf_beta beta, const float* fg, const float* bg, int mode, sf_stream stream, double* eig);
int sf_beta_update_real(sf_beta beta, const float* fg, const float* bg, sf_stream stream);
/* localize (src/seg/views.rs:24-66): weighted centre and mean distance of
 * the foreground set {a > b}, weights m = a / (a + b), positions from the
 * splats' mean planes. *found = 0 (and zeros) while no splat is foreground.
 * Reduced on the device in f64 over a fixed partition (deterministic); the
 * reference sums in f32 on the host after an a / b read-back. Syncs. */
int sf_localize(sf_splats s, sf_beta beta, sf_stream stream, int* found, float center[3],
                float* radius);
/* map_labels (src/seg/beta.rs:294-297): out[i] = a[i] > b[i]. Host arrays. */
int sf_map_labels(const float* a, const float* b, uint32_t n, uint8_t* out);
/* The f32 entropy LUT the EIG kernel reads (445*445 floats, host copy). */
int sf_entropy_table(float* out);
/* table_entropy probe (beta.rs:336-342): out[i] = H_LUT(a[i], b[i]), device arrays. */
int sf_table_entropy(sf_ctx ctx, const float* a, const float* b, uint32_t n, float* out,
                     sf_stream stream);

/* ------------------------------------------------------ batched round */
/* A round of candidate views scored together (the batched form of
 * Segmenter::select_view, src/seg/active.rs:113-129, which renders and
 * scores one view at a time with two blocking read-backs each). Every view's
 * project -> depth sort -> scan -> emit -> tile sort -> responsibility
 * raster -> EIG is captured once into a CUDA graph with device-side counts
 * and replayed each round; views may have different sizes. */
typedef struct sf_round_t* sf_round;
typedef struct {
    uint32_t lanes;       /* capture streams the views are spread over (1..64) */
    uint32_t raster_cull; /* as sf_tuning.raster_cull */
    uint32_t isect_build; /* as sf_tuning.isect_build */
    uint32_t raster_order; /* as sf_tuning.raster_order */
    uint32_t raster_split; /* as sf_tuning.raster_split */
    uint32_t radix_bits;   /* as sf_tuning.radix_bits */
    uint32_t reserved[2];
} sf_round_tuning;
int sf_round_create(sf_ctx ctx, uint32_t total, uint32_t n_views, const uint32_t* widths,
                    const uint32_t* heights, sf_round* out);
int sf_round_destroy(sf_round r);
int sf_round_set_tuning(sf_round r, const sf_round_tuning* t);
int sf_round_get_tuning(sf_round r, sf_round_tuning* t);
/* One round for cameras cams[n_views]: every view's total responsibility
 * and, when beta is non-NULL, its EIG (mode SF_EIG_LUT_F32 / SF_EIG_FP64)
 * into host eig[n_views]. Syncs once. A view whose intersections outgrow the
 * round's capacity is re-run after the capacity grows. The words equal the
 * per-view sf_render_responsibility words bit for bit. */
int sf_round_eig(sf_round r, sf_splats s, sf_beta beta, const sf_camera* cams, int mode,
                 sf_stream stream, double* eig);
/* View `view` of the last round: device responsibility words [total], the
 * fixed-point scale, the intersection count and the visible count. */
int sf_round_responsibility(sf_round r, uint32_t view, const uint32_t** resp, float* scale,
                            uint64_t* num_isects, uint32_t* num_visible);
/* Evidence round: the observe half of Segmenter::step (src/seg/active.rs:
 * 133-176, the masked finalize of src/render.rs:387-470) batched over several
 * views. masks[n_views] (each the size
 * of its view) split every view's weights into fg / bg words, as
 * sf_accumulate_prepared with a mask does; when beta is non-NULL each view's
 * EIG over eps = fg + bg goes to eig[n_views]. Syncs once. After it,
 * sf_round_responsibility returns the fg words. */
int sf_round_evidence(sf_round r, sf_splats s, sf_beta beta, const sf_camera* cams,
                      const sf_mask* masks, int mode, sf_stream stream, double* eig);
/* View `view` of the last evidence round: device fg and bg words [total]. */
int sf_round_evidence_words(sf_round r, uint32_t view, const uint32_t** fg, const uint32_t** bg);
/* Adjoint evidence round (no counterpart in the reference): every view's
 * responsibilities from the adjoint of a per-splat scalar feature
 * (sf_render_feature_adjoint: transmittance-only forward, back-to-front
 * replay) in the round's graph, real-valued fg / bg per splat (masks NULL,
 * or a NULL entry: all of the view in fg), and with beta each view's EIG
 * over fg + bg (sf_beta_eig_real). Syncs once. The lists are sorted for the
 * replay whatever the tuning's raster_order. */
int sf_round_evidence_adjoint(sf_round r, sf_splats s, sf_beta beta, const sf_camera* cams,
                              const sf_mask* masks, int mode, sf_stream stream, double* eig);
/* View `view` of the last adjoint round: device fg and bg floats [total]. */
int sf_round_adjoint_responsibility(sf_round r, uint32_t view, const float** fg, const float** bg);
/* Autotuner (the round's kernel forms picked by measured time): a
 * coordinate search, two sweeps, over lanes {1,2,4,8}, isect_build {binned,
 * depth-sorted}, raster_order {sorted, in-raster, hybrid} (binned build),
 * raster_cull {0,1}, raster_split {1,2,4} (rasterizer warps per CTA 8, 4
 * or 2 on 16x16 tiles) and radix_bits {4,6,8} (sort digit width, depth-sorted
 * build), each candidate timed as the best of three rounds
 * after a warm-up round. The winner and its time stay on the round and in
 * a process-wide cache keyed by (device, splats, view sizes, kind); a cached
 * shape is not searched again (best_ms then gives the cached time). sf_round_autotune
 * tunes the responsibility round (sf_round_eig); sf_round_autotune_kind the
 * round of `kind`: SF_ROUND_RESPONSIBILITY, SF_ROUND_EVIDENCE
 * (sf_round_evidence with `masks`) or SF_ROUND_ADJOINT
 * (sf_round_evidence_adjoint; `masks` may be NULL). */
enum { SF_ROUND_RESPONSIBILITY = 0, SF_ROUND_EVIDENCE = 1, SF_ROUND_ADJOINT = 2 };
int sf_round_autotune(sf_round r, sf_splats s, sf_beta beta, const sf_camera* cams, int mode,
                      sf_stream stream, sf_round_tuning* best, double* best_ms);
int sf_round_autotune_kind(sf_round r, sf_splats s, sf_beta beta, const sf_camera* cams,
                           const sf_mask* masks, int kind, int mode, sf_stream stream,
                           sf_round_tuning* best, double* best_ms);

/* -------------------------------------------------------- PLY scenes */
/* parse_ply's header rules (src/ply.rs:9-77) on a whole file image: the
 * vertex count and SH coefficients per channel (1 + f_rest count / 3). Host only
 * (no CUDA call). Errors: SF_ERR_ARG with the reference's messages
 * ("Unsupported PLY format: ...", "Missing property: ...", ...). */
int sf_ply_inspect(const void* bytes, size_t len, uint32_t* n, uint32_t* sh_per_ch);
/* parse_ply (src/ply.rs:9-112) + CpuSplats::upload: the vertex block goes
 * to the device as stored and one kernel writes the field-major planes
 * (rotations normalised as glam does, bounds reduced on the device). */
int sf_ply_load(sf_ctx ctx, const void* bytes, size_t len, sf_splats* out);
int sf_ply_load_file(sf_ctx ctx, const char* path, sf_splats* out);
/* CpuSplats::write_ply (src/ply.rs:115-180) from host planes: out = NULL
 * reports the byte length in *len; else writes it (cap >= *len). */
int sf_ply_write(const float* attr, const float* sh, uint32_t n, uint32_t sh_per_ch, void* out,
                 size_t cap, size_t* len);

/* --------------------------------------------------------- SOG scenes */
/* parse_sog (src/sog.rs:97-198): a SOG archive (zip: meta.json + lossless
 * WebP planes) to splats, with the reference's checks and messages
 * ("not a SOG archive", "missing meta.json", "invalid meta.json", "SOG
 * contains no splats", "missing <file>", "<file>: WxH < N pixels", codebook
 * sizes, "quats: invalid rotation tag T", "shN.bands B outside 1..=3",
 * "shN label L >= palette size P"); errors are SF_ERR_ARG. The planes are
 * decoded on the host (zip stored / deflate entries, WebP lossless) and
 * dequantised on the device into the field-major attribute and SH planes
 * (sh_per_ch 1, 4, 9 or 16 for shN bands 0..3). sf_sog_inspect reads only
 * meta.json (no CUDA call). */
int sf_sog_inspect(const void* bytes, size_t len, uint32_t* n, uint32_t* sh_per_ch);
int sf_sog_load(sf_ctx ctx, const void* bytes, size_t len, sf_splats* out);
int sf_sog_load_file(sf_ctx ctx, const char* path, sf_splats* out);
/* No counterpart in the reference (its SOG planes go through the `image`
 * crate): the lossless WebP decoder the SOG loader uses, host only. Writes
 * *w, *h and, when rgba is non-NULL and cap >= w * h * 4, the RGBA8 pixels
 * row-major. Lossy WebP is refused (SF_ERR_ARG). */
int sf_webp_decode(const void* bytes, size_t len, uint32_t* w, uint32_t* h, uint8_t* rgba, size_t cap);

/* ------------------------------------------------------- sort / scan */
/* bits_for (crates/sort/src/sort.rs:259-261). */
uint32_t sf_bits_for(uint32_t max_exclusive);
/* RadixScratch::new (crates/sort/src/sort.rs:291-300). */
int sf_radix_create(sf_ctx ctx, uint32_t max_elems, sf_radix* out);
int sf_radix_destroy(sf_radix r);
/* RadixScratch::argsort (crates/sort/src/sort.rs:311-380): stable LSD sort of
 * keys[0..n) by their low `bits` bits, carrying vals. Inputs are only read.
 * Outputs are device pointers into the scratch (or the inputs themselves when
 * n <= 1 or bits == 0, as the reference returns). write_keys = 0 leaves the
 * returned keys stale (values are always sorted). Onesweep: 8-bit digits, one
 * upfront histogram, one decoupled-look-back pass per digit. The call waits
 * for the stream and reads the sort's device error word: a look-back wait
 * that ran out returns SF_ERR_TIMEOUT (the outputs are then not valid). */
int sf_radix_argsort(sf_radix r, const uint32_t* keys, const uint32_t* vals, uint32_t n,
                     uint32_t bits, int write_keys, sf_stream stream, const uint32_t** keys_out,
                     const uint32_t** vals_out);
/* No counterpart in the reference (its sorts block on their own read-backs).
 * sf_radix_argsort without the wait: the sort is only enqueued, so a caller
 * can run several sorts (or other work) back to back on the stream; a
 * look-back wait that ran out is kept in the scratch's error word until
 * sf_radix_status, which waits for the stream and returns SF_ERR_TIMEOUT if
 * any sort on the scratch since the last status (or synchronous sort) timed
 * out, then clears the word. */
int sf_radix_argsort_async(sf_radix r, const uint32_t* keys, const uint32_t* vals, uint32_t n,
                           uint32_t bits, int write_keys, sf_stream stream, const uint32_t** keys_out,
                           const uint32_t** vals_out);
int sf_radix_status(sf_radix r, sf_stream stream);
/* Digit width of the scratch's passes, 4..8 bits (default 8; the
 * reference's RADIX_BITS is 6, crates/sort/src/sort.rs:11-17). The order is
 * the same at every width. */
int sf_radix_set_digit_bits(sf_radix r, uint32_t digit_bits);
/* ScanScratch::new (crates/sort/src/scan.rs:54-59). */
int sf_scan_create(sf_ctx ctx, uint32_t max_elems, sf_scan* out);
int sf_scan_destroy(sf_scan s);
/* exclusive_scan_gather (crates/sort/src/scan.rs:219-255):
 * offsets[i] = sum_{j<i} counts[gids[j]], single-pass decoupled look-back;
 * n = 0 writes nothing. Like sf_radix_argsort, the call waits for the stream
 * and returns SF_ERR_TIMEOUT if a look-back wait ran out. */
int sf_exclusive_scan_gather(sf_scan s, const uint32_t* gids, const uint32_t* counts,
                             uint32_t* offsets, uint32_t n, sf_stream stream);
/* No counterpart in the reference. sf_exclusive_scan_gather without the
 * wait; sf_scan_status reports and clears a timed-out wait, as
 * sf_radix_status does for sorts. */
int sf_exclusive_scan_gather_async(sf_scan s, const uint32_t* gids, const uint32_t* counts,
                                   uint32_t* offsets, uint32_t n, sf_stream stream);
int sf_scan_status(sf_scan s, sf_stream stream);
/* exclusive_scan_buf (crates/sort/src/scan.rs:185-213): in place. */
int sf_exclusive_scan(sf_scan s, uint32_t* buf, uint32_t n, sf_stream stream);
/* No counterpart in the reference. sf_exclusive_scan_gather for callers that
 * cannot call cudaMalloc (a host whose device memory belongs to another
 * allocator's pool, or a per-frame loop that may not take cudaMalloc's
 * device-wide synchronisation): same result, but the look-back scratch is a
 * fixed static device array, so the call allocates nothing. Runs on the
 * calling thread's current device; n > SF_SCAN_NOALLOC_MAX_ELEMS (2^24) is
 * rejected with SF_ERR_SHAPE before any CUDA call. Every call on a device
 * shares the one array: calls that overlap on the GPU race, so order them
 * (one stream). The first call on a device finds the array's device address
 * (cudaGetSymbolAddress) and keeps it; a cudaDeviceReset invalidates it. The
 * call waits for the stream, reads the error word into a host stack variable
 * and returns SF_ERR_TIMEOUT if a look-back wait ran out. */
#define SF_SCAN_NOALLOC_MAX_ELEMS (1u << 24)
int sf_exclusive_scan_gather_noalloc(const uint32_t* gids, const uint32_t* counts,
                                     uint32_t* offsets, uint32_t n, sf_stream stream);

/* ------------------------------------------------------- test hooks */
/* No counterpart in the reference. Knobs of the bounded look-back waits of
 * the scan and the radix sort, for tests of the timeout path: spin_limit caps
 * the polls of one wait (0 restores the default); withhold = 1 keeps the first
 * partition of every scan and digit pass from publishing its status, so the
 * waits after it run out and the calls return SF_ERR_TIMEOUT instead of
 * hanging. Process-wide host state; call (0, 0) afterwards. Only
 * sf_radix_argsort, sf_exclusive_scan_gather, sf_exclusive_scan and
 * sf_exclusive_scan_gather_noalloc pass the knobs to their kernels; the
 * frame, round and backward paths never see them. */
int sf_debug_lookback(uint32_t spin_limit, int withhold);

/* No counterpart in the reference. The binned build sorts each list longer
 * than 12288 entries by cutting it into key-contiguous segments over many
 * CTAs, for up to 4096 such lists per frame; the later ones of a frame are
 * sorted by one CTA each. Scratches and rounds created after this call cut
 * at most `lists` lists (0: none), so tests can reach the one-CTA form;
 * 4096 restores the default. Both forms give the same order. */
int sf_debug_giant_lists(uint32_t lists);

#ifdef __cplusplus
}
#endif
#endif /* SPLATFIELD_CUDA_H */
