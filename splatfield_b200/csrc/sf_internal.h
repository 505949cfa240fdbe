// Internal declarations shared by the CUDA translation units.
#pragma once
#include <cuda_runtime.h>
#include <algorithm>
#include <cstddef>
#include <cstdint>
#include "../../include/splatfield_cuda.h"

// Device error word bits (sticky, OR-ed by kernels, read by the host at sync
// points).
#define SF_DEV_ERR_TIMEOUT 1u
#define SF_DEV_ERR_CAPACITY 2u

namespace sfk {

// Process-wide count of kernels launched by this library.
void note_launches(uint32_t k);

// Programmatic dependent launch: a kernel launched by launch_pdl may be
// scheduled while the kernel before it on the stream drains (that kernel's
// blocks call pdl_trigger as they start); it calls pdl_wait before its first
// memory access, which returns once the previous kernel has completed and
// its writes are visible. Both are no-ops for a kernel launched without the
// attribute.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                       Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}
// A stream capture enqueues kernels without running them: the capture takes
// its count back (forget_launches) and each graph launch notes it again.
void forget_launches(uint64_t k);
uint64_t launches();

// Per-splat projected record, split so that the responsibility modes read 32
// bytes and the RGB mode 48:
//   geo0 = {mean.x, mean.y, 0.5*conic.x, conic.y}
//   geo1 = {0.5*conic.z, opacity, power_max, 0}  (power_max: above it alpha < 1/255)
//   color = {r+0.5, g+0.5, b+0.5, 0}
struct ProjOut {
    uint32_t* depth_keys;   // [n] f32 bits of camera z; 0xFFFFFFFF culled
    uint32_t* tile_counts;  // [n]
    uint2* bbox;            // [n] packed min / max
    float4* geo0;           // [n]
    float4* geo1;           // [n]
    float4* color;          // [n] (may be null: colour not needed)
    uint32_t* visible;      // atomic counter (may be null)
    float2* ext;            // [n] half extents of the box holding power <= power_max
};

// Coefficients per channel the SH evaluation reads for sh_per_ch stored
// ones: the largest whole degree, 1 / 4 / 9 / 16 (src/project.rs:343-388 tests
// chs >= 4, >= 9, >= 16).
inline uint32_t sh_degree_coeffs(uint32_t sh_per_ch) {
    return sh_per_ch >= 16 ? 16u : sh_per_ch >= 9 ? 9u : sh_per_ch >= 4 ? 4u : 1u;
}

// Per-splat camera-independent projection terms, [kGeomPlanes][n]: the
// rows of M = R(q) diag(exp(log_scale)) (9), opacity, extent cutoff,
// power_max. Computed once per splat set (launch_splat_geom).
constexpr int kGeomPlanes = 12;
cudaError_t launch_splat_geom(const float* attr, uint32_t n, float* geom, cudaStream_t stream);
// view_dev (optional) supplies the view from device memory instead.
cudaError_t launch_project(const sf_view& view, const float* attr, const float* geom, const float* sh, uint32_t n,
                           uint32_t sh_per_ch, const ProjOut& out, cudaStream_t stream,
                           const sf_view* view_dev = nullptr);

cudaError_t launch_emit(const uint32_t* order, const uint2* bbox, const uint32_t* offsets,
                        uint32_t n, uint32_t tiles_per_row, uint32_t capacity, uint32_t* tile_ids,
                        uint32_t* gaussian_ids, uint32_t* err, cudaStream_t stream);

// tile_start[t] = lower_bound(t) over sorted ids, t in [0, num_tiles].
cudaError_t launch_tile_starts(const uint32_t* sorted_tile_ids, uint32_t num_isects,
                               const uint32_t* num_isects_dev, uint32_t max_isects,
                               uint32_t num_tiles, uint32_t* tile_start, cudaStream_t stream);

struct RasterArgs {
    uint32_t w, h, tiles_x, tiles_y, row_stride;
    const uint32_t* tile_start;
    const uint32_t* gaussian_ids;
    // Unsorted placed (depth key, splat id) pairs of the binned build; when
    // set, the rasterizer orders itself every tile list longer than
    // lazy_min entries (the others come sorted in gaussian_ids).
    const uint2* pairs;
    uint32_t lazy_min;
    const float4* geo0;
    const float4* geo1;
    const float4* color;
    const float2* ext;
    float scale;
    const uint32_t* mask;
    uint32_t mask_wpr;
    uint32_t* bitmap;
    float4* rgba;
    uint32_t* resp;
    uint32_t* fg;
    uint32_t* bg;
    float* final_t;
    uint32_t* n_contrib;
    // Raster form: 0 walks every staged entry in every warp, 1 culls per warp
    // block with the power_max boxes (needs ext).
    uint32_t cull;
    // CTAs per 16x16 tile (0 or 1: one CTA of 8 warps; 2 or 4: CTAs of 4 or
    // 2 warps, each walking the whole list for its part of the pixels).
    uint32_t split;
    // 1: also count the per-pair diagnostics stats[1..3] (slower form).
    uint32_t detail;
    // Optional pair statistics, added to: [0] (pixel, splat) pairs visited
    // (256 per tile-list entry walked before the tile's early exit), [1]
    // exponentials evaluated, [2] contributing pairs (alpha >= 1/255).
    unsigned long long* stats;
    // Block schedule (optional, one block per tile): the binned build's
    // class lists, longest lists first (class_lists[k * tiles + i], counts
    // class_n[k], k = kSortClasses - 1 .. 0, then the empty tiles).
    const uint32_t* class_lists;
    const uint32_t* class_n;
};
// mode 0 = RGB, 1 = total responsibility, 2 = evidence, 3 = transmittance
// only (final_t and n_contrib required).
cudaError_t launch_raster(int mode, const RasterArgs& a, cudaStream_t stream);

// Adjoint (sf_backward.cu).
struct BwdArgs {
    uint32_t w, h, tiles_x, tiles_y;
    const uint32_t* tile_start;
    const uint32_t* gaussian_ids;
    const float4* geo0;
    const float4* geo1;
    const float4* color;
    const float* final_t;      // forward's final transmittance per pixel
    const uint32_t* n_contrib; // forward's 1-based last contributor per pixel
    const float4* dl;          // dL/d(r, g, b, a) per pixel
    float* d2d;                // [n][9] accumulated: mean2d xy, conic xyz, rgb, opacity
};
cudaError_t launch_raster_bwd(const BwdArgs& a, cudaStream_t stream);
// Adjoint of a per-splat scalar feature: fg[i] += sum_p mask(p) alpha_i
// T_i(p), bg[i] += sum_p (1 - mask(p)) alpha_i T_i(p) (mask null: all in
// fg), replayed from the state of the transmittance-only raster (mode 3)
// over the same sorted lists.
struct FeatureBwdArgs {
    uint32_t w, h, tiles_x, tiles_y;
    const uint32_t* tile_start;
    const uint32_t* gaussian_ids;
    const float4* geo0;
    const float4* geo1;
    const float* final_t;
    const uint32_t* n_contrib;
    const uint32_t* mask;
    uint32_t mask_wpr;
    float* fg;
    float* bg;
};
cudaError_t launch_feature_bwd(const FeatureBwdArgs& a, cudaStream_t stream);
cudaError_t launch_project_bwd(const sf_view& view, const float* attr, const float* sh, uint32_t n,
                               uint32_t sh_per_ch, const float* d2d, float* d_attr, float* d_sh,
                               cudaStream_t stream);

// Reference-layout projected rows [n][9] from the split records.
cudaError_t launch_export_rows(const float4* geo0, const float4* geo1, const float4* color,
                               const uint32_t* depth_keys, uint32_t n, float* rows,
                               cudaStream_t stream);

// ---- sort / scan (sf_sort.cu)
// Test knobs of the bounded look-back waits (sf_debug_lookback): spin_limit
// caps the polls of one wait (0: the default), withhold = 1 keeps partition 0
// from publishing so the later waits run out. Zero in every internal call;
// only the standalone sort and scan entry points pass lookback_test_knobs().
struct LookbackKnobs {
    uint32_t spin_limit;
    uint32_t withhold;
};
LookbackKnobs lookback_test_knobs();
// Passes of an LSD sort of `bits` key bits at digit_bits per pass (4..8).
uint32_t radix_passes(uint32_t bits, uint32_t digit_bits = 8);
size_t radix_temp_bytes(uint32_t max_elems, uint32_t max_passes);
// Sorts keys_in/vals_in by the low `bits` bits into the (a, b) ping-pong
// buffers; *out_in_b tells which holds the result. n_dev (optional) supplies
// the element count on the device, with max_n sizing the grid.
cudaError_t radix_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_a,
                             uint32_t* vals_a, uint32_t* keys_b, uint32_t* vals_b, uint32_t n,
                             const uint32_t* n_dev, uint32_t max_n, uint32_t bits, bool write_keys,
                             bool vals_iota, void* temp, uint32_t* err, int sm_count,
                             cudaStream_t stream, int* out_in_b, LookbackKnobs knobs = {0u, 0u},
                             uint32_t digit_bits = 8);
size_t scan_temp_bytes(uint32_t max_elems);
cudaError_t exclusive_scan(const uint32_t* gids, const uint32_t* counts, uint32_t* out, uint32_t n,
                           const uint32_t* n_dev, uint32_t max_n, void* temp,
                           unsigned long long* total_out, uint32_t* err, cudaStream_t stream,
                           LookbackKnobs knobs = {0u, 0u});

// ---- binned intersection build (sf_bin.cu)
// Tiles per frame the binned build handles (one u32 shared-memory counter
// per tile in the count and place kernels).
constexpr uint32_t kBinMaxTiles = 49152;
uint32_t bin_chunks(uint32_t n, int sm_count);
// Per-tile sort size classes: k = 0 .. kSortClasses - 2 hold lists of up to
// bin_class_limit(k) entries; the last class holds the longer lists.
constexpr int kSortClasses = 7;
uint32_t bin_class_limit(int k);
// Longest list the shared-memory classes sort; longer lists go to the global
// form (or, with the hybrid order, to the rasterizer).
constexpr uint32_t kBinSharedMax = 12288;
// hist: [chunks][tiles] counts, then (after colscan) per-chunk exclusive
// prefixes. cnt: [tiles + 1] per-tile totals (cnt[tiles] = 0). lists:
// [kSortClasses + 1][tiles] tiles of each size class, then the empty tiles.
// words: [6] max tile total, [8 + k] tiles in class k, k <= kSortClasses
// (all zero on entry).
cudaError_t launch_bin_count(const uint2* bbox, uint32_t n, uint32_t tiles_x, uint32_t tiles, uint32_t chunks,
                             uint32_t* hist, cudaStream_t st);
// Segmented sort of the longest lists (sf_bin.cu): each list past 24576
// entries (up to `lists` of them per frame) gets a key histogram of
// kGiantBins buckets, cut into segments of about kGiantSegTarget entries that
// are sorted on separate CTAs; shorter lists of the longest class, and any
// past `lists`, are sorted by one CTA each.
constexpr uint32_t kGiantBins = 2048, kGiantSegTarget = 4096, kGiantMaxLists = 4096;
constexpr uint32_t kGiantMinList = 24576;
struct GiantState {
    uint32_t* ctrl = nullptr;  // [4]: lists taken, chunks, short segments, long segments
    uint4* sel = nullptr;      // [lists]: (tile, first slot, entries, first chunk)
    uint32_t* mm = nullptr;    // [2 * lists]: key min, max of each taken list
    uint32_t* hist = nullptr;  // [lists][kGiantBins]
    uint32_t* taken = nullptr; // [tiles]: 1 where the longest class's entry i was taken
    uint4* segs = nullptr;     // [seg_cap]: (tile, first slot, entries, 0)
    uint32_t lists = 0;
    uint32_t seg_cap = 0;
};
// Whether a captured graph includes the segmented sort, from the longest
// list of the frames seen so far (`on`: the last graph had it): on past
// kGiantMinList entries, off again below half of that. Either way the lists
// come out in the same order; the choice is only about speed (the segmented
// chain's seven launches cost more than they save when no list is that long).
inline bool giant_wanted(uint32_t longest, bool on) {
    return on ? longest > kGiantMinList / 2 : longest > kGiantMinList;
}
// lists = min(tiles, kGiantMaxLists); seg_cap bounds the segments of lists
// holding up to 2^30 slots in all (each list has at most n / target + 1).
uint32_t giant_lists(uint32_t tiles);
uint32_t giant_seg_cap(uint32_t lists);
// Test hook: scratches built afterwards segment at most `lists` lists (0:
// none), so the one-CTA form takes the rest.
void set_giant_max_lists(uint32_t lists);
cudaError_t launch_bin_colscan(uint32_t* hist, uint32_t chunks, uint32_t tiles, uint32_t* cnt, uint32_t* lists,
                               uint32_t* words, cudaStream_t st);

cudaError_t launch_bin_place(const uint2* bbox, const uint32_t* depth_keys, uint32_t n, uint32_t tiles_x,
                             uint32_t tiles, uint32_t chunks, const uint32_t* hist, const uint32_t* tile_start,
                             uint32_t capacity, uint2* pairs, uint32_t* err, cudaStream_t st);
// grids[k]: CTAs launched for class k (the class count when the host knows
// it, else `tiles`; CTAs past the device count exit); grids[3] = 0 leaves
// the longest lists unsorted.
// Device-side capacity handling when the intersection total is not read
// on the host first: n32 = min(total, cap) with SF_DEV_ERR_CAPACITY set past
// it, and tile starts cut back to the capacity (every slot below it holds a
// placed pair, so the sorts and the raster stay inside the buffers).
cudaError_t launch_clamp_count(const unsigned long long* total, uint32_t cap, uint32_t* n32, uint32_t* err,
                               cudaStream_t st);
// A frame's 16 status words to slot *counter of a device ring (when it is
// below ring_frames), then ++*counter: the last node of the frame graph, so
// frames enqueued back to back keep their words on the device.
cudaError_t launch_save_words(const uint32_t* words, uint32_t* ring, uint32_t* counter, uint32_t ring_frames,
                              cudaStream_t st);
cudaError_t launch_clamp_starts(uint32_t* tile_start, uint32_t count, uint32_t cap, cudaStream_t st);

// Side streams the per-tile sort classes run on concurrently inside a
// captured graph (the tail of one class overlaps the others); null runs them
// in turn on one stream (outside a graph the extra event calls cost more
// host time than the overlap gains).
struct SortStreams {
    cudaStream_t s[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t e[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
};
cudaError_t sort_streams_create(SortStreams* ss);
void sort_streams_destroy(SortStreams* ss);

// pairs: the placed (depth key, splat id) per slot (overwritten for the
// longest lists); ids / tids_out receive the sorted splat ids / tile ids
// (tids_out may be null); keys_tmp: capacity u32 of scratch (may alias
// tids_out). grids[k]: the tile count of size class k, or an upper bound
// when the counts are on the device (0 skips the class).
// gs (may be null: every longest list on the one-CTA form): the segmented
// sort's buffers, sized for `tiles` tiles.
cudaError_t launch_tile_sorts(const uint32_t grids[kSortClasses], const uint32_t* lists, const uint32_t* words,
                              uint32_t tiles, const uint32_t* tile_start, uint32_t capacity, uint2* pairs,
                              uint32_t* ids, uint32_t* tids_out, uint32_t* keys_tmp, int sm_count,
                              cudaStream_t st, const SortStreams* side = nullptr, const GiantState* gs = nullptr);

// ---- segmentation (sf_seg.cu)
constexpr int kGridPts = 445;
constexpr float kLnStep = 0.015611423f;
void build_entropy_table(float* table);  // host, f64 formulas
double beta_entropy_host(double a, double b);
// Per-block f64 partial sums of dH; then a single-block final sum into out.
// resp2 (optional) is added word for word: eps = fg + bg of an evidence split.
// h0 (optional): H(a_i, b_i) of every splat from launch_entropy (f32 for the
// LUT mode, f64 for FP64), read instead of recomputed; the sums are the same.
cudaError_t launch_eig(int mode, const float* a, const float* b, const uint32_t* resp, uint32_t n,
                       float scale, const float* table, double* partials, uint32_t max_blocks,
                       double* out, cudaStream_t stream, const uint32_t* resp2 = nullptr,
                       const void* h0 = nullptr);
// out[i] = H(a_i, b_i) (mode SF_EIG_LUT_F32: f32 table values; SF_EIG_FP64: f64).
cudaError_t launch_entropy(int mode, const float* a, const float* b, uint32_t n, const float* table, void* out,
                           cudaStream_t stream);
uint32_t eig_blocks(uint32_t n, int sm_count);
// Posterior heatmap colours and foreground tint (src/seg/paint.rs).
cudaError_t launch_paint_posterior(const float* a, const float* b, uint32_t n, float4* color,
                                   cudaStream_t stream);
cudaError_t launch_tint(float* sh, const float* a, const float* b, uint32_t n, float r, float g, float bl,
                        cudaStream_t stream);
// Object localization: partials [blocks][4] doubles, out [8] doubles
// ([0] sum of weights, [4..6] centre, [7] radius).
cudaError_t launch_localize(const float* attr, const float* a, const float* b, uint32_t n, double* partials,
                            uint32_t blocks, double* out, cudaStream_t stream);
cudaError_t launch_beta_update(float scale, const uint32_t* fg, const uint32_t* bg, float* a,
                               float* b, uint32_t n, cudaStream_t stream);
// EIG and Beta update from real-valued responsibilities (eps = fg + bg; bg
// may be null for the EIG).
cudaError_t launch_eig_real(int mode, const float* a, const float* b, const float* fg, const float* bg,
                            uint32_t n, const float* table, double* partials, uint32_t blocks, double* out,
                            cudaStream_t stream, const void* h0 = nullptr);
cudaError_t launch_beta_update_real(const float* fg, const float* bg, float* a, float* b, uint32_t n,
                                    cudaStream_t stream);
cudaError_t launch_table_probe(const float* a, const float* b, uint32_t n, const float* table,
                               float* out, cudaStream_t stream);

// ---- camera (sf_camera.cpp)
void camera_look_at(const float position[3], const float target[3], sf_camera* out);
void view_for_camera(const sf_camera& cam, uint32_t w, uint32_t h, sf_view* out);

}  // namespace sfk
