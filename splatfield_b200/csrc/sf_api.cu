// C ABI of the splat path: handles, buffer ownership, capacity management and
// the per-frame orchestration of the kernels (see include/splatfield_cuda.h).
//
// Frame = project -> depth sort (onesweep, 32-bit keys, values = splat ids)
// -> gather scan of tile counts in depth order (decoupled look-back) ->
// [one host sync: intersection total] -> grow capacity if needed -> emit ->
// stable tile sort (onesweep over bits_for(tiles) bits) -> tile starts ->
// rasterize. This is the reference's prepare_isects/finalize sequence
// (src/render.rs:274-460) with its 3-launch-per-digit sort and hierarchical
// scan replaced, and with capacity grown before emission instead of the
// reference's silent truncation (src/raster.rs:38-46).
#include <cuda_runtime.h>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>
#include "sf_handles.h"

using namespace sfk;

namespace {
thread_local std::string g_err;
}  // namespace

namespace sfk {
int set_error(int code, const std::string& msg) {
    g_err = msg;
    return code;
}
}  // namespace sfk

namespace {

int fail(int code, const std::string& msg) { return set_error(code, msg); }

#define SF_CK(expr)                                                                        \
    do {                                                                                   \
        cudaError_t e_ = (expr);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            if (e_ == cudaErrorMemoryAllocation)                                           \
                return fail(SF_ERR_NOMEM, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
            return fail(SF_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_));  \
        }                                                                                  \
    } while (0)

#define SF_TRY(body)                                                  \
    try {                                                             \
        body                                                          \
    } catch (const std::bad_alloc&) {                                 \
        return fail(SF_ERR_NOMEM, "host allocation failed");          \
    } catch (const std::exception& ex) {                              \
        return fail(SF_ERR_ARG, ex.what());                           \
    } catch (...) {                                                   \
        return fail(SF_ERR_ARG, "unknown exception");                 \
    }

inline cudaStream_t S(sf_stream s) { return reinterpret_cast<cudaStream_t>(s); }

cudaError_t use_device(int dev) {
    int cur = -1;
    cudaError_t e = cudaGetDevice(&cur);
    if (e != cudaSuccess) return e;
    return cur == dev ? cudaSuccess : cudaSetDevice(dev);
}

template <typename T>
cudaError_t dalloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    return cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T));
}

template <typename T>
void dfree(T*& p) {
    if (p) cudaFree(reinterpret_cast<void*>(p));
    p = nullptr;
}

uint32_t bits_for_u32(uint32_t max_exclusive) {
    const uint32_t m = max_exclusive > 0 ? max_exclusive - 1 : 0;
    return m == 0 ? 0u : 32u - (uint32_t)__builtin_clz(m);
}

uint64_t next_pow2(uint64_t v) {
    uint64_t p = 1;
    while (p < v) p <<= 1;
    return p;
}

uint32_t frac_bits(uint32_t w, uint32_t h) {
    const uint64_t pixels = (uint64_t)w * h;
    uint32_t tz = 0;
    uint64_t p2 = 1;
    while (p2 < pixels) { p2 <<= 1; ++tz; }
    return tz >= 32 ? 0u : 32u - tz;
}

// Largest intersection capacity: the look-back status words carry 30-bit
// counts.
constexpr uint64_t kMaxIsects = (1ull << 30) - 1;
// First-frame capacity cap (the reference's INITIAL_ISECTS_CAP, render.rs:18).
constexpr uint64_t kInitialIsects = 1ull << 22;

}  // namespace

struct sf_scratch_t {
    sf_ctx ctx = nullptr;
    uint32_t total = 0, w = 0, h = 0, tiles_x = 0, tiles_y = 0, row_stride = 0;
    uint32_t* depth_keys = nullptr;
    uint32_t* tile_counts = nullptr;
    uint2* bbox = nullptr;
    float4* geo0 = nullptr;
    float4* geo1 = nullptr;
    float4* color = nullptr;
    float2* ext = nullptr;
    uint32_t *keys_a = nullptr, *keys_b = nullptr, *order_a = nullptr, *order_b = nullptr;
    const uint32_t* order = nullptr;
    uint32_t* offsets = nullptr;
    void* sort_tmp = nullptr;
    size_t sort_tmp_bytes = 0;
    void* scan_tmp = nullptr;
    uint64_t cap = 0;
    uint32_t *tid_e = nullptr, *gid_e = nullptr, *tid_a = nullptr, *gid_a = nullptr;
    const uint32_t* tids = nullptr;
    const uint32_t* gids = nullptr;
    uint32_t* tile_start = nullptr;
    // Binned build: [chunks][tiles] histogram / prefixes, per-tile totals,
    // per-class tile lists.
    uint32_t bin_chunks = 0;
    uint32_t* bin_hist = nullptr;
    uint32_t* bin_cnt = nullptr;
    uint32_t* bin_lists = nullptr;
    GiantState giant;  // segmented sort of the longest lists
    uint32_t longest = 0;  // longest tile list of the last binned frame
    bool binned = false;
    // The last prepare left the binned build's placed pairs unsorted: the
    // rasterizer orders each tile's list itself (no gaussian_ids).
    bool lazy = false;
    uint32_t lazy_min = 0;  // lists longer than this are ordered in the raster
    SortStreams sort_streams;  // concurrent per-tile sort classes inside the frame graph
    // Frame graph (binned RGB frames): one capture per (splats, size,
    // capacity, tuning), replayed with the camera copied in by its first node.
    struct FrameGraph {
        cudaGraphExec_t exec = nullptr;
        uint32_t kernels = 0;           // kernel nodes of exec
        cudaStream_t stream = nullptr;  // capture stream
        sf_view* view_dev = nullptr;
        sf_view* view_host = nullptr;   // pinned
        const void* splats = nullptr;
        const float* attr = nullptr;
        const float* sh = nullptr;
        uint32_t K = 0, n = 0, w = 0, h = 0;
        uint64_t cap = 0;
        sf_tuning tuning{};
        bool giant = false;  // the graph includes the segmented sort
        // Frames to host memory in a batch: each image is copied out of the
        // bitmap into one of two staging images, whose device-to-host copy
        // (copy stream) runs while the next frame renders.
        cudaStream_t copy = nullptr;
        cudaEvent_t ready[2] = {nullptr, nullptr}, copied[2] = {nullptr, nullptr};
        uint32_t* stage[2] = {nullptr, nullptr};
        size_t stage_words = 0;
        sf_view* views = nullptr;     // pinned, one per frame of the batch
        uint32_t* frame_words = nullptr;  // pinned, 16 per frame of the batch
        // Device ring the graph's last node saves each frame's words to
        // (slot = *ring_counter, which it then increments), read back once a
        // run of frames has finished.
        uint32_t* ring = nullptr;
        uint32_t* ring_counter = nullptr;
        uint32_t batch_cap = 0;
    } fg;
    uint32_t* bitmap = nullptr;
    float4* rgba = nullptr;
    float* final_t = nullptr;
    uint32_t* n_contrib = nullptr;
    // device words: [0] visible, [1] error bits, [2..3] spare, [4..5] u64
    // total, [6..14] binned-build tile statistics (sf_internal.h)
    uint32_t* words = nullptr;
    uint32_t* host_words = nullptr;  // pinned mirror
    unsigned long long* stats = nullptr;  // raster pair statistics of the last finalize
    uint32_t num_visible = 0, num_isects = 0;
    uint64_t last_isects_raw = 0;
    bool prepared = false;
    sf_tuning tuning{};
    // Adjoint state: the camera of the last forward that kept per-pixel
    // final T / last contributor, and the per-splat 2D adjoint buffer.
    bool has_forward = false;
    sf_camera fwd_cam{};
    float* d2d = nullptr;
    // Second frame pipe of the camera-path calls (tuning.frame_pipes): an
    // internal scratch with its own frame buffers, frame graph and launch
    // stream; frames alternate between it and this scratch. fork / join
    // order its stream after the caller's and the caller's after it.
    sf_scratch_t* twin = nullptr;
    cudaStream_t twin_stream = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};

struct sf_radix_t {
    sf_ctx ctx = nullptr;
    uint32_t max = 0;
    uint32_t digit_bits = 8;
    uint32_t *ka = nullptr, *va = nullptr, *kb = nullptr, *vb = nullptr;
    void* tmp = nullptr;
    uint32_t* err = nullptr;
};

struct sf_scan_t {
    sf_ctx ctx = nullptr;
    uint32_t max = 0;
    void* tmp = nullptr;
    unsigned long long* total = nullptr;
    uint32_t* err = nullptr;
};

// ---------------------------------------------------------------- helpers

namespace {

cudaError_t ensure_lut(sf_ctx ctx) {
    if (ctx->lut) return cudaSuccess;
    std::vector<float> t((size_t)kGridPts * kGridPts);
    build_entropy_table(t.data());
    cudaError_t e = dalloc(&ctx->lut, t.size());
    if (e != cudaSuccess) return e;
    return cudaMemcpy(ctx->lut, t.data(), t.size() * 4, cudaMemcpyHostToDevice);
}

void scratch_free_frame(sf_scratch s) {
    dfree(s->depth_keys); dfree(s->tile_counts); dfree(s->bbox); dfree(s->geo0); dfree(s->geo1);
    dfree(s->color); dfree(s->ext); dfree(s->keys_a); dfree(s->keys_b); dfree(s->order_a); dfree(s->order_b);
    dfree(s->offsets); dfree(s->scan_tmp); dfree(s->tile_start); dfree(s->bitmap);
    dfree(s->bin_hist); dfree(s->bin_cnt); dfree(s->bin_lists);
    dfree(s->giant.ctrl); dfree(s->giant.sel); dfree(s->giant.mm); dfree(s->giant.hist);
    dfree(s->giant.taken); dfree(s->giant.segs);
    s->giant.lists = s->giant.seg_cap = 0;
    dfree(s->rgba); dfree(s->final_t); dfree(s->n_contrib); dfree(s->d2d);
    s->order = nullptr;
    s->prepared = false;
    s->has_forward = false;
}

void scratch_free_isects(sf_scratch s) {
    dfree(s->tid_e); dfree(s->gid_e); dfree(s->tid_a);
    s->gid_a = nullptr;  // second half of the tid_a allocation
    if (s->sort_tmp) cudaFree(s->sort_tmp);
    s->sort_tmp = nullptr;
    s->sort_tmp_bytes = 0;
    s->cap = 0;
    s->tids = s->gids = nullptr;
}

cudaError_t ensure_sort_tmp(sf_scratch s, size_t bytes) {
    if (s->sort_tmp_bytes >= bytes) return cudaSuccess;
    if (s->sort_tmp) cudaFree(s->sort_tmp);
    s->sort_tmp = nullptr;
    s->sort_tmp_bytes = 0;
    cudaError_t e = cudaMalloc(&s->sort_tmp, bytes);
    if (e == cudaSuccess) s->sort_tmp_bytes = bytes;
    return e;
}

cudaError_t grow_isects(sf_scratch s, uint64_t want) {
    if (want <= s->cap && s->tid_e) return cudaSuccess;
    const uint64_t cap = std::min<uint64_t>(std::max<uint64_t>(next_pow2(want), 1024), kMaxIsects + 1);
    dfree(s->tid_e); dfree(s->gid_e); dfree(s->tid_a);
    s->gid_a = nullptr;
    s->cap = 0;
    cudaError_t e;
    if ((e = dalloc(&s->tid_e, cap)) != cudaSuccess) return e;
    if ((e = dalloc(&s->gid_e, cap)) != cudaSuccess) return e;
    // tid_a and gid_a are one allocation: the binned build places packed
    // (depth key, splat id) pairs across both.
    if ((e = dalloc(&s->tid_a, 2 * cap)) != cudaSuccess) return e;
    s->gid_a = s->tid_a + cap;
    s->cap = cap;
    return ensure_sort_tmp(s, std::max(radix_temp_bytes((uint32_t)std::min<uint64_t>(cap, kMaxIsects), 4),
                                       radix_temp_bytes(s->total, 4)));
}

cudaError_t scratch_build(sf_scratch s, uint32_t total, uint32_t w, uint32_t h) {
    scratch_free_frame(s);
    s->total = total;
    s->w = w;
    s->h = h;
    s->tiles_x = (w + 15) / 16;
    s->tiles_y = (h + 15) / 16;
    s->row_stride = ((4 * w + 255) / 256 * 256) / 4;
    cudaError_t e;
#define SF_AL(ptr, cnt) if ((e = dalloc(&(ptr), (cnt))) != cudaSuccess) return e
    SF_AL(s->depth_keys, total);
    SF_AL(s->tile_counts, total);
    SF_AL(s->bbox, total);
    SF_AL(s->geo0, total);
    SF_AL(s->geo1, total);
    SF_AL(s->color, total);
    SF_AL(s->ext, total);
    SF_AL(s->keys_a, total);
    SF_AL(s->keys_b, total);
    SF_AL(s->order_a, total);
    SF_AL(s->order_b, total);
    SF_AL(s->offsets, total);
    const size_t tiles = (size_t)s->tiles_x * s->tiles_y;
    SF_AL(s->tile_start, tiles + 1);
    if (tiles <= kBinMaxTiles) {
        s->bin_chunks = bin_chunks(total, s->ctx->sm_count);
        SF_AL(s->bin_hist, (size_t)s->bin_chunks * tiles);
        SF_AL(s->bin_cnt, tiles + 1);
        SF_AL(s->bin_lists, (size_t)(kSortClasses + 1) * tiles);
        s->giant.lists = giant_lists((uint32_t)tiles);
        s->giant.seg_cap = giant_seg_cap(s->giant.lists);
        SF_AL(s->giant.ctrl, 4);
        SF_AL(s->giant.sel, s->giant.lists);
        SF_AL(s->giant.mm, 2 * (size_t)s->giant.lists);
        SF_AL(s->giant.hist, (size_t)s->giant.lists * kGiantBins);
        SF_AL(s->giant.taken, tiles);
        SF_AL(s->giant.segs, s->giant.seg_cap);
    }
    SF_AL(s->bitmap, (size_t)h * s->row_stride);
#undef SF_AL
    // Row padding (row_stride past w) is never rendered: clear it once so
    // read-backs of whole rows are deterministic.
    if ((e = cudaMemset(s->bitmap, 0, (size_t)h * s->row_stride * 4)) != cudaSuccess) return e;
    const uint32_t scan_n = (uint32_t)std::max<size_t>(total, tiles + 1);
    if ((e = cudaMalloc(&s->scan_tmp, scan_temp_bytes(scan_n))) != cudaSuccess) return e;
    if (!s->words) {
        if ((e = dalloc(&s->stats, 4)) != cudaSuccess) return e;
        if ((e = dalloc(&s->words, 16)) != cudaSuccess) return e;
        if ((e = cudaMallocHost(reinterpret_cast<void**>(&s->host_words), 64)) != cudaSuccess) return e;
    }
    // Capacity: keep the larger of the growth hint and the reference's first
    // frame rule min(tiles*total, 2^22) (render.rs:146-147, 177-183).
    const uint64_t first = std::min<uint64_t>((uint64_t)s->tiles_x * s->tiles_y * total, kInitialIsects);
    return grow_isects(s, std::max<uint64_t>(std::max<uint64_t>(first, s->last_isects_raw), s->cap));
}

int finish_prepare(sf_scratch s, sf_isects* out);

// Binned intersection build (sf_bin.cu) after the projection: count, column
// scan, tile scan, one sync for the total, place, per-tile sorts.
// order: SF_ORDER_SORTED sorts every list; SF_ORDER_IN_RASTER none;
// SF_ORDER_HYBRID all but the longest (left to the rasterizer).
int prepare_binned(sf_scratch s, uint32_t n, uint32_t tiles, cudaStream_t st, bool want_tile_ids, uint32_t order) {
    uint32_t* words = s->words;
    unsigned long long* total_dev = reinterpret_cast<unsigned long long*>(words + 4);
    SF_CK(launch_bin_count(s->bbox, n, s->tiles_x, tiles, s->bin_chunks, s->bin_hist, st));
    SF_CK(launch_bin_colscan(s->bin_hist, s->bin_chunks, tiles, s->bin_cnt, s->bin_lists, words, st));
    SF_CK(exclusive_scan(nullptr, s->bin_cnt, s->tile_start, tiles + 1, nullptr, tiles + 1, s->scan_tmp,
                         total_dev, words + 1, st));
    SF_CK(cudaMemcpyAsync(s->host_words, words, 64, cudaMemcpyDeviceToHost, st));
    SF_CK(cudaStreamSynchronize(st));
    const uint32_t* hw = s->host_words;
    if (hw[1] & SF_DEV_ERR_TIMEOUT) return fail(SF_ERR_TIMEOUT, "device look-back wait timed out");
    uint64_t total = 0;
    std::memcpy(&total, hw + 4, 8);
    s->num_visible = hw[0];
    s->last_isects_raw = total;
    s->longest = hw[6];
    if (total > kMaxIsects) return fail(SF_ERR_CAPACITY, "intersection count exceeds 2^30-1");
    if (total > s->cap) {
        std::fprintf(stderr, "splatfield_b200: intersection capacity %llu reached (%llu needed); growing\n",
                     (unsigned long long)s->cap, (unsigned long long)total);
        SF_CK(grow_isects(s, total));
    }
    uint2* pairs = reinterpret_cast<uint2*>(s->tid_a);
    SF_CK(launch_bin_place(s->bbox, s->depth_keys, n, s->tiles_x, tiles, s->bin_chunks, s->bin_hist,
                           s->tile_start, (uint32_t)s->cap, pairs, words + 1, st));
    s->lazy = order != SF_ORDER_SORTED;
    s->lazy_min = order == SF_ORDER_HYBRID ? kBinSharedMax : 0u;
    if (order == SF_ORDER_IN_RASTER) {
        s->tids = s->gids = nullptr;
    } else {
        uint32_t grids[kSortClasses];
        for (int k = 0; k < kSortClasses; ++k) grids[k] = hw[8 + k];
        if (order == SF_ORDER_HYBRID) grids[kSortClasses - 1] = 0;
        // The longest list is known here: the segmented sort runs only when
        // some list is long enough to gain from it.
        SF_CK(launch_tile_sorts(grids, s->bin_lists, words, tiles, s->tile_start, (uint32_t)s->cap, pairs,
                                s->gid_e, want_tile_ids ? s->tid_e : nullptr, s->tid_e, s->ctx->sm_count, st,
                                nullptr, hw[6] > kGiantMinList ? &s->giant : nullptr));
        s->tids = want_tile_ids ? s->tid_e : nullptr;
        s->gids = s->gid_e;
    }
    s->num_isects = (uint32_t)total;
    s->binned = true;
    return SF_OK;
}

// prepare_isects (src/render.rs:274-364).
// lazy: the caller only rasterizes this frame (no sorted lists handed out,
// no adjoint state), so the binned build may leave each tile's order to the
// rasterizer (tuning.raster_order).
int prepare(sf_splats sp, sf_scratch s, const sf_camera* cam, uint32_t w, uint32_t h,
            cudaStream_t st, sf_isects* out, bool lazy = false) {
    if (!sp || !s || !cam) return fail(SF_ERR_ARG, "null argument");
    if (w == 0 || h == 0 || w > 65535 * 16 || h > 65535 * 16) return fail(SF_ERR_SHAPE, "bad image size");
    SF_CK(use_device(s->ctx->device));
    if (s->total != sp->n || s->w != w || s->h != h) SF_CK(scratch_build(s, sp->n, w, h));
    s->has_forward = false;
    sf_view view;
    view_for_camera(*cam, w, h, &view);
    const uint32_t n = sp->n;
    uint32_t* words = s->words;
    unsigned long long* total_dev = reinterpret_cast<unsigned long long*>(words + 4);
    SF_CK(cudaMemsetAsync(words, 0, 64, st));
    ProjOut po{s->depth_keys, s->tile_counts, s->bbox, s->geo0, s->geo1, s->color, words, s->ext};
    SF_CK(launch_project(view, sp->attr, sp->geom, sp->sh, n, sp->K, po, st));
    const uint32_t tiles = s->tiles_x * s->tiles_y;
    s->order = nullptr;
    s->tids = s->gids = nullptr;
    s->lazy = false;
    if (s->tuning.isect_build == SF_ISECTS_BINNED && s->bin_hist) {
        const int rc = prepare_binned(s, n, tiles, st, out != nullptr,
                                      (lazy && out == nullptr) ? s->tuning.raster_order : SF_ORDER_SORTED);
        if (rc != SF_OK) return rc;
        return finish_prepare(s, out);
    }
    s->binned = false;
    int in_b = 0;
    SF_CK(ensure_sort_tmp(s, radix_temp_bytes(n, 4)));
    const uint32_t digit_bits = s->tuning.radix_bits ? s->tuning.radix_bits : 8u;
    SF_CK(radix_sort_pairs(s->depth_keys, nullptr, s->keys_a, s->order_a, s->keys_b, s->order_b, n,
                           nullptr, n, 32, false, true, s->sort_tmp, words + 1, s->ctx->sm_count, st,
                           &in_b, LookbackKnobs{0u, 0u}, digit_bits));
    s->order = in_b ? s->order_b : s->order_a;
    SF_CK(exclusive_scan(s->order, s->tile_counts, s->offsets, n, nullptr, n, s->scan_tmp, total_dev,
                         words + 1, st));
    SF_CK(cudaMemcpyAsync(s->host_words, words, 64, cudaMemcpyDeviceToHost, st));
    SF_CK(cudaStreamSynchronize(st));
    if (s->host_words[1] & SF_DEV_ERR_TIMEOUT) return fail(SF_ERR_TIMEOUT, "device look-back wait timed out");
    uint64_t total = 0;
    std::memcpy(&total, s->host_words + 4, 8);
    s->num_visible = s->host_words[0];
    s->last_isects_raw = total;
    if (total > kMaxIsects) return fail(SF_ERR_CAPACITY, "intersection count exceeds 2^30-1");
    if (total > s->cap) {
        std::fprintf(stderr, "splatfield_b200: intersection capacity %llu reached (%llu emitted); growing\n",
                     (unsigned long long)s->cap, (unsigned long long)total);
        SF_CK(grow_isects(s, total));
    }
    const uint32_t I = (uint32_t)total;
    SF_CK(launch_emit(s->order, s->bbox, s->offsets, n, s->tiles_x, (uint32_t)s->cap, s->tid_e,
                      s->gid_e, words + 1, st));
    const uint32_t tbits = bits_for_u32(tiles);
    if (I <= 1 || tbits == 0) {
        s->tids = s->tid_e;
        s->gids = s->gid_e;
    } else {
        SF_CK(radix_sort_pairs(s->tid_e, s->gid_e, s->tid_a, s->gid_a, s->tid_e, s->gid_e, I, nullptr, I,
                               tbits, true, false, s->sort_tmp, words + 1, s->ctx->sm_count, st, &in_b,
                               LookbackKnobs{0u, 0u}, digit_bits));
        s->tids = in_b ? s->tid_e : s->tid_a;
        s->gids = in_b ? s->gid_e : s->gid_a;
    }
    SF_CK(launch_tile_starts(s->tids, I, nullptr, I, tiles, s->tile_start, st));
    s->num_isects = I;
    return finish_prepare(s, out);
}

int finish_prepare(sf_scratch s, sf_isects* out) {
    s->prepared = true;
    if (out) {
        out->tile_ids = s->tids;
        out->gaussian_ids = s->gids;
        out->tile_start = s->tile_start;
        out->num_isects = s->num_isects;
        out->num_visible = s->num_visible;
        out->tile_bounds[0] = s->tiles_x;
        out->tile_bounds[1] = s->tiles_y;
        out->row_stride = s->row_stride;
    }
    return SF_OK;
}

RasterArgs raster_args(sf_scratch s, const sf_isects* is) {
    RasterArgs a{};
    a.w = s->w;
    a.h = s->h;
    a.tiles_x = s->tiles_x;
    a.tiles_y = s->tiles_y;
    a.row_stride = s->row_stride;
    a.tile_start = is ? is->tile_start : s->tile_start;
    a.gaussian_ids = is ? is->gaussian_ids : s->gids;
    a.pairs = (!is && s->lazy) ? reinterpret_cast<const uint2*>(s->tid_a) : nullptr;
    a.lazy_min = s->lazy_min;
    a.geo0 = s->geo0;
    a.geo1 = s->geo1;
    a.color = s->color;
    a.ext = s->ext;
    a.cull = s->tuning.raster_cull;
    a.split = s->tuning.raster_split;
    a.detail = s->tuning.raster_detail;
    a.stats = s->stats;
    return a;
}

int finalize_rgb(sf_scratch s, const sf_isects* is, bool want_float, cudaStream_t st,
                 bool keep_state = false) {
    RasterArgs a = raster_args(s, is);
    a.bitmap = s->bitmap;
    if (want_float) {
        if (!s->rgba) SF_CK(dalloc(&s->rgba, (size_t)s->w * s->h));
        a.rgba = s->rgba;
    }
    s->has_forward = false;
    if (keep_state) {
        if (!s->final_t) SF_CK(dalloc(&s->final_t, (size_t)s->w * s->h));
        if (!s->n_contrib) SF_CK(dalloc(&s->n_contrib, (size_t)s->w * s->h));
        a.final_t = s->final_t;
        a.n_contrib = s->n_contrib;
    }
    SF_CK(cudaMemsetAsync(s->stats, 0, 32, st));
    SF_CK(launch_raster(0, a, st));
    return SF_OK;
}

int accumulate(sf_scratch s, const sf_isects* is, uint32_t w, uint32_t h, sf_accum acc, sf_mask mask,
               cudaStream_t st) {
    if (acc->total != s->total) return fail(SF_ERR_SHAPE, "accumulator size does not match the scratch");
    acc->scale = (float)((uint64_t)1 << frac_bits(w, h));
    RasterArgs a = raster_args(s, is);
    a.scale = acc->scale;
    acc->evidence = mask != nullptr;
    SF_CK(cudaMemsetAsync(s->stats, 0, 32, st));
    if (!mask) {
        SF_CK(cudaMemsetAsync(acc->resp, 0, (size_t)acc->total * 4, st));
        a.resp = acc->resp;
        SF_CK(launch_raster(1, a, st));
    } else {
        if (mask->w != w || mask->h != h) return fail(SF_ERR_SHAPE, "mask size does not match the frame");
        SF_CK(cudaMemsetAsync(acc->fg, 0, (size_t)acc->total * 4, st));
        SF_CK(cudaMemsetAsync(acc->bg, 0, (size_t)acc->total * 4, st));
        a.mask = mask->bits;
        a.mask_wpr = mask->wpr;
        a.fg = acc->fg;
        a.bg = acc->bg;
        SF_CK(launch_raster(2, a, st));
    }
    return SF_OK;
}

// ---------------------------------------------------------- frame graph
//
// A binned RGB frame with no host step in the middle: projection, counts,
// scans, placement against the current capacity (device-side guard, tile
// starts clamped), per-tile sorts as persistent kernels reading their class
// sizes on the device (the classes on side streams), raster, and the status
// words saved to a device ring — captured once and replayed with one launch
// per frame on the caller's stream. The host reads the words after the frame
// (or after a run of frames); a frame that outgrew the capacity grows it and
// runs again (the graph is captured anew).

// frame_render's answer when the frame graph does not apply (the caller
// takes the step-by-step path).
constexpr int kNoFrameGraph = -2;

bool frame_graph_usable(sf_splats sp, sf_scratch s) {
    return s->bin_hist && sp->n == s->total && s->tuning.isect_build == SF_ISECTS_BINNED &&
           !s->tuning.raster_detail;
}

constexpr uint32_t kFrameRing = 4096;  // frames whose status words the ring holds

int frame_graph_capture(sf_splats sp, sf_scratch s) {
    auto& g = s->fg;
    if (g.exec) {
        cudaGraphExecDestroy(g.exec);
        g.exec = nullptr;
    }
    if (!g.stream) SF_CK(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
    if (!g.view_dev) SF_CK(dalloc(&g.view_dev, 1));
    if (!g.ring) SF_CK(dalloc(&g.ring, 16 * (size_t)kFrameRing));
    if (!g.ring_counter) SF_CK(dalloc(&g.ring_counter, 1));
    if (!g.view_host) SF_CK(cudaMallocHost(reinterpret_cast<void**>(&g.view_host), sizeof(sf_view)));
    if (!s->sort_streams.s[0]) SF_CK(sort_streams_create(&s->sort_streams));
    const uint32_t n = sp->n;
    const uint32_t tiles = s->tiles_x * s->tiles_y;
    const uint32_t cap = (uint32_t)s->cap;
    const uint32_t order = s->tuning.raster_order;
    const bool giant = giant_wanted(s->longest, g.giant);
    uint32_t* words = s->words;
    auto* total = reinterpret_cast<unsigned long long*>(words + 4);
    cudaStream_t st = g.stream;
    // The camera's view is copied to g.view_dev before each launch (from a
    // pinned slot of the caller's choosing), outside the graph.
    const uint64_t launches0 = launches();
    SF_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaMemsetAsync(words, 0, 64, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->stats, 0, 32, st);
    ProjOut po{s->depth_keys, s->tile_counts, s->bbox, s->geo0, s->geo1, s->color, words, s->ext};
    sf_view dummy{};
    if (e == cudaSuccess) e = launch_project(dummy, sp->attr, sp->geom, sp->sh, n, sp->K, po, st, g.view_dev);
    if (e == cudaSuccess) e = launch_bin_count(s->bbox, n, s->tiles_x, tiles, s->bin_chunks, s->bin_hist, st);
    if (e == cudaSuccess)
        e = launch_bin_colscan(s->bin_hist, s->bin_chunks, tiles, s->bin_cnt, s->bin_lists, words, st);
    if (e == cudaSuccess)
        e = exclusive_scan(nullptr, s->bin_cnt, s->tile_start, tiles + 1, nullptr, tiles + 1, s->scan_tmp, total,
                           words + 1, st);
    if (e == cudaSuccess) e = launch_clamp_count(total, cap, words + 2, words + 1, st);
    uint2* pairs = reinterpret_cast<uint2*>(s->tid_a);
    if (e == cudaSuccess)
        e = launch_bin_place(s->bbox, s->depth_keys, n, s->tiles_x, tiles, s->bin_chunks, s->bin_hist,
                             s->tile_start, cap, pairs, words + 1, st);
    if (e == cudaSuccess) e = launch_clamp_starts(s->tile_start, tiles + 1, cap, st);
    if (e == cudaSuccess && order != SF_ORDER_IN_RASTER) {
        uint32_t grids[kSortClasses];
        for (int k = 0; k < kSortClasses; ++k) grids[k] = tiles;
        if (order == SF_ORDER_HYBRID) grids[kSortClasses - 1] = 0;
        e = launch_tile_sorts(grids, s->bin_lists, words, tiles, s->tile_start, cap, pairs, s->gid_e, nullptr,
                              s->tid_e, s->ctx->sm_count, st, &s->sort_streams, giant ? &s->giant : nullptr);
    }
    if (e == cudaSuccess) {
        RasterArgs a{};
        a.w = s->w;
        a.h = s->h;
        a.tiles_x = s->tiles_x;
        a.tiles_y = s->tiles_y;
        a.row_stride = s->row_stride;
        a.tile_start = s->tile_start;
        a.gaussian_ids = order == SF_ORDER_IN_RASTER ? nullptr : s->gid_e;
        a.pairs = order == SF_ORDER_SORTED ? nullptr : pairs;
        a.lazy_min = order == SF_ORDER_HYBRID ? kBinSharedMax : 0u;
        a.geo0 = s->geo0;
        a.geo1 = s->geo1;
        a.color = s->color;
        a.ext = s->ext;
        a.cull = s->tuning.raster_cull;
        a.split = s->tuning.raster_split;
        a.stats = s->stats;
        a.bitmap = s->bitmap;
        if (s->tuning.raster_schedule == SF_SCHEDULE_LONGEST && order != SF_ORDER_IN_RASTER) {
            a.class_lists = s->bin_lists;
            a.class_n = words + 8;
        }
        e = launch_raster(0, a, st);
    }
    if (e == cudaSuccess) e = launch_save_words(words, g.ring, g.ring_counter, kFrameRing, st);
    cudaGraph_t graph = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(st, &graph);
    g.kernels = (uint32_t)(launches() - launches0);
    forget_launches(g.kernels);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return fail(SF_ERR_CUDA,
                    std::string("frame graph capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    e = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        g.exec = nullptr;
        return fail(SF_ERR_CUDA, std::string("frame graph instantiate: ") + cudaGetErrorString(e));
    }
    g.splats = sp;
    g.attr = sp->attr;
    g.sh = sp->sh;
    g.K = sp->K;
    g.n = sp->n;
    g.w = s->w;
    g.h = s->h;
    g.cap = s->cap;
    g.tuning = s->tuning;
    g.giant = giant;
    return SF_OK;
}

// (Re)captures the frame graph when the splats, image size, capacity or
// tuning it was captured for changed.
int frame_graph_ready(sf_splats sp, sf_scratch s, uint32_t w, uint32_t h) {
    auto& g = s->fg;
    if (!g.exec || g.splats != sp || g.attr != sp->attr || g.sh != sp->sh || g.K != sp->K || g.n != sp->n ||
        g.w != w || g.h != h || g.cap != s->cap || std::memcmp(&g.tuning, &s->tuning, sizeof(sf_tuning)) != 0 ||
        giant_wanted(s->longest, g.giant) != g.giant)
        return frame_graph_capture(sp, s);
    return SF_OK;
}

// The scratch's prepared-frame state after a frame whose device words are
// hw (total <= capacity).
void frame_graph_settle(sf_scratch s, const uint32_t* hw, uint64_t total) {
    const uint32_t order = s->tuning.raster_order;
    s->num_visible = hw[0];
    s->last_isects_raw = total;
    s->num_isects = (uint32_t)total;
    s->longest = hw[6];
    s->binned = true;
    s->lazy = order != SF_ORDER_SORTED;
    s->lazy_min = order == SF_ORDER_HYBRID ? kBinSharedMax : 0u;
    s->order = nullptr;
    s->tids = nullptr;
    s->gids = order == SF_ORDER_IN_RASTER ? nullptr : s->gid_e;
    s->prepared = true;
    s->has_forward = false;
}

// One RGB frame through the frame graph on stream st; the image is in
// s->bitmap and, when host_out is given, copied there. Syncs once.
int frame_graph_render(sf_splats sp, sf_scratch s, const sf_camera* cam, uint32_t w, uint32_t h,
                       cudaStream_t st, uint32_t* host_out) {
    auto& g = s->fg;
    for (int attempt = 0; attempt < 4; ++attempt) {
        const int rc = frame_graph_ready(sp, s, w, h);
        if (rc != SF_OK) return rc;
        view_for_camera(*cam, w, h, g.view_host);
        SF_CK(cudaMemcpyAsync(g.view_dev, g.view_host, sizeof(sf_view), cudaMemcpyHostToDevice, st));
        SF_CK(cudaGraphLaunch(g.exec, st));
        note_launches(g.kernels);
        SF_CK(cudaMemcpyAsync(s->host_words, s->words, 64, cudaMemcpyDeviceToHost, st));
        if (host_out)
            SF_CK(cudaMemcpy2DAsync(host_out, (size_t)w * 4, s->bitmap, (size_t)s->row_stride * 4, (size_t)w * 4,
                                    h, cudaMemcpyDeviceToHost, st));
        SF_CK(cudaStreamSynchronize(st));
        const uint32_t* hw = s->host_words;
        if (hw[1] & SF_DEV_ERR_TIMEOUT) return fail(SF_ERR_TIMEOUT, "device look-back wait timed out");
        uint64_t total = 0;
        std::memcpy(&total, hw + 4, 8);
        s->num_visible = hw[0];
        s->last_isects_raw = total;
        if (total > kMaxIsects) return fail(SF_ERR_CAPACITY, "intersection count exceeds 2^30-1");
        if (total <= s->cap) {
            frame_graph_settle(s, hw, total);
            return SF_OK;
        }
        std::fprintf(stderr, "splatfield_b200: intersection capacity %llu reached (%llu needed); growing\n",
                     (unsigned long long)s->cap, (unsigned long long)total);
        SF_CK(grow_isects(s, total));
    }
    return fail(SF_ERR_CAPACITY, "frame capacity did not settle");
}

cudaError_t frames_batch_resources(sf_scratch s, uint32_t count, size_t image_words) {
    auto& g = s->fg;
    cudaError_t e;
    if (!g.copy && (e = cudaStreamCreateWithFlags(&g.copy, cudaStreamNonBlocking)) != cudaSuccess) return e;
    for (int k = 0; k < 2; ++k) {
        if (!g.ready[k] && (e = cudaEventCreateWithFlags(&g.ready[k], cudaEventDisableTiming)) != cudaSuccess)
            return e;
        if (!g.copied[k] && (e = cudaEventCreateWithFlags(&g.copied[k], cudaEventDisableTiming)) != cudaSuccess)
            return e;
    }
    if (g.stage_words < image_words) {
        for (int k = 0; k < 2; ++k) {
            dfree(g.stage[k]);
            g.stage[k] = nullptr;
        }
        g.stage_words = 0;
        for (int k = 0; k < 2; ++k)
            if ((e = dalloc(&g.stage[k], image_words)) != cudaSuccess) return e;
        g.stage_words = image_words;
    }
    if (g.batch_cap < count) {
        if (g.views) cudaFreeHost(g.views);
        if (g.frame_words) cudaFreeHost(g.frame_words);
        g.views = nullptr;
        g.frame_words = nullptr;
        g.batch_cap = 0;
        if ((e = cudaMallocHost(reinterpret_cast<void**>(&g.views), sizeof(sf_view) * count)) != cudaSuccess)
            return e;
        if ((e = cudaMallocHost(reinterpret_cast<void**>(&g.frame_words), 64 * (size_t)count)) != cudaSuccess)
            return e;

        g.batch_cap = count;
    }
    return cudaSuccess;
}

// The second frame pipe of s at w x h (allocated on first use): the twin
// scratch holds at least s's capacity and s's tuning and list statistics,
// so both pipes capture the same kernels.
int twin_ready(sf_splats sp, sf_scratch s, uint32_t w, uint32_t h) {
    if (!s->twin) {
        s->twin = new sf_scratch_t();
        s->twin->ctx = s->ctx;
    }
    sf_scratch t = s->twin;
    if (t->total != sp->n || t->w != w || t->h != h || !t->bitmap) SF_CK(scratch_build(t, sp->n, w, h));
    if (t->cap < s->cap) SF_CK(grow_isects(t, s->cap));
    t->tuning = s->tuning;
    t->longest = s->longest;
    if (!s->twin_stream) SF_CK(cudaStreamCreateWithFlags(&s->twin_stream, cudaStreamNonBlocking));
    if (!s->fork) SF_CK(cudaEventCreateWithFlags(&s->fork, cudaEventDisableTiming));
    if (!s->join) SF_CK(cudaEventCreateWithFlags(&s->join, cudaEventDisableTiming));
    return frame_graph_ready(sp, t, w, h);
}

// Copies the status words that run [first, end) of a camera path saved to
// its pipes' device rings into frame_words[16 * i] (frame i on pipe
// pipe_of(i); each pipe's ring holds its frames of the run in launch order).
template <typename PipeOf>
cudaError_t read_rings(sf_scratch const pipes[2], PipeOf pipe_of, uint32_t first, uint32_t end,
                       uint32_t* frame_words) {
    uint32_t on[2] = {0, 0};
    for (uint32_t i = first; i < end; ++i) ++on[pipe_of(i)];
    std::vector<uint32_t> ring[2];
    for (int p = 0; p < 2; ++p) {
        if (!on[p]) continue;
        ring[p].resize(16 * (size_t)on[p]);
        const cudaError_t e =
            cudaMemcpy(ring[p].data(), pipes[p]->fg.ring, 64 * (size_t)on[p], cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return e;
    }
    uint32_t k[2] = {0, 0};
    for (uint32_t i = first; i < end; ++i) {
        const int p = pipe_of(i);
        std::memcpy(frame_words + 16 * (size_t)i, ring[p].data() + 16 * (size_t)k[p]++, 64);
    }
    return cudaSuccess;
}

// `count` frames through the frame graph, frame i's image to
// host_out + i * w * h (host_out null: the images stay on the device, the
// last one in the scratch). The device-to-host copy of frame i (copy stream,
// from a staging image) overlaps the next frames. With two frame pipes the
// frames alternate between s (on st) and its twin (on the twin's stream),
// the last frame on s, so one frame's projection and intersection build
// overlap the other's raster. Frames whose intersections passed their
// pipe's capacity are rendered again, one by one, after the capacity has
// grown. Syncs at the end.
int frames_graph_render(sf_splats sp, sf_scratch s, const sf_camera* cams, uint32_t count, uint32_t w,
                        uint32_t h, cudaStream_t st, uint32_t* host_out) {
    auto& g = s->fg;
    const size_t img = (size_t)w * h;
    bool two = count >= 2 && s->tuning.frame_pipes != 1;
    int rc = frame_graph_ready(sp, s, w, h);
    if (rc != SF_OK) return rc;
    if (two && (rc = twin_ready(sp, s, w, h)) != SF_OK) {
        if (rc != SF_ERR_NOMEM) return rc;
        // No room for the second pipe: release what it took and render the
        // path on one pipe.
        cudaGetLastError();
        sf_scratch_destroy(s->twin);
        s->twin = nullptr;
        two = false;
    }
    sf_scratch const pipes[2] = {s, two ? s->twin : s};
    cudaStream_t const streams[2] = {st, two ? s->twin_stream : st};
    auto pipe_of = [&](uint32_t i) { return two ? (int)((count - 1 - i) & 1u) : 0; };
    SF_CK(frames_batch_resources(s, count, host_out ? img : 0));
    for (uint32_t i = 0; i < count; ++i) view_for_camera(cams[i], w, h, g.views + i);
    // The copy stream may still hold another batch's copies of the staging
    // images: the first two frames of this one wait for them.
    SF_CK(cudaEventRecord(g.ready[0], g.copy));
    SF_CK(cudaStreamWaitEvent(st, g.ready[0], 0));
    if (two) {
        SF_CK(cudaEventRecord(s->fork, st));
        SF_CK(cudaStreamWaitEvent(streams[1], s->fork, 0));
    }
    for (uint32_t i = 0; i < count; ++i) {
        const int slot = (int)(i & 1u);
        const int p = pipe_of(i);
        sf_scratch P = pipes[p];
        cudaStream_t ps = streams[p];
        // Each run of up to kFrameRing frames saves its words to the pipes'
        // device rings, read back once after the run has finished (a
        // read-back after every frame cost 2% of the frame rate).
        if (i % kFrameRing == 0) {
            if (i > 0) {
                SF_CK(cudaStreamSynchronize(streams[0]));
                SF_CK(cudaStreamSynchronize(streams[1]));
                SF_CK(read_rings(pipes, pipe_of, i - kFrameRing, i, g.frame_words));
            }
            SF_CK(cudaMemsetAsync(pipes[0]->fg.ring_counter, 0, 4, streams[0]));
            if (two) SF_CK(cudaMemsetAsync(pipes[1]->fg.ring_counter, 0, 4, streams[1]));
        }
        SF_CK(cudaMemcpyAsync(P->fg.view_dev, g.views + i, sizeof(sf_view), cudaMemcpyHostToDevice, ps));
        SF_CK(cudaGraphLaunch(P->fg.exec, ps));
        note_launches(P->fg.kernels);
        if (!host_out) continue;
        // Frames i and i + 2 share a staging image (and, with two pipes, a
        // pipe).
        if (i >= 2) SF_CK(cudaStreamWaitEvent(ps, g.copied[slot], 0));
        SF_CK(cudaMemcpy2DAsync(g.stage[slot], (size_t)w * 4, P->bitmap, (size_t)P->row_stride * 4,
                                (size_t)w * 4, h, cudaMemcpyDeviceToDevice, ps));
        SF_CK(cudaEventRecord(g.ready[slot], ps));
        SF_CK(cudaStreamWaitEvent(g.copy, g.ready[slot], 0));
        SF_CK(cudaMemcpyAsync(host_out + i * img, g.stage[slot], img * 4, cudaMemcpyDeviceToHost, g.copy));
        SF_CK(cudaEventRecord(g.copied[slot], g.copy));
    }
    if (two) {
        SF_CK(cudaEventRecord(s->join, streams[1]));
        SF_CK(cudaStreamWaitEvent(st, s->join, 0));
    }
    SF_CK(cudaStreamSynchronize(g.copy));
    SF_CK(cudaStreamSynchronize(st));
    SF_CK(read_rings(pipes, pipe_of, (count - 1) / kFrameRing * kFrameRing, count, g.frame_words));
    uint64_t need = 0;
    uint32_t longest = 0;
    bool over = false;
    for (uint32_t i = 0; i < count; ++i) {
        const uint32_t* hw = g.frame_words + 16 * (size_t)i;
        if (hw[1] & SF_DEV_ERR_TIMEOUT) return fail(SF_ERR_TIMEOUT, "device look-back wait timed out");
        uint64_t total = 0;
        std::memcpy(&total, hw + 4, 8);
        if (total > kMaxIsects) return fail(SF_ERR_CAPACITY, "intersection count exceeds 2^30-1");
        if (total > need) need = total;
        if (total > pipes[pipe_of(i)]->cap) over = true;
        longest = std::max(longest, hw[6]);
    }
    if (two) s->twin->longest = longest;
    if (over) {
        // Frames past their pipe's capacity (their images were drawn from
        // clamped lists) are rendered again on s after one growth.
        std::vector<uint32_t> redo;
        for (uint32_t i = 0; i < count; ++i) {
            uint64_t total = 0;
            std::memcpy(&total, g.frame_words + 16 * (size_t)i + 4, 8);
            if (total > pipes[pipe_of(i)]->cap) redo.push_back(i);
        }
        std::fprintf(stderr, "splatfield_b200: intersection capacity %llu reached (%llu needed); growing\n",
                     (unsigned long long)s->cap, (unsigned long long)need);
        SF_CK(grow_isects(s, need));
        if (two) SF_CK(grow_isects(s->twin, need));
        for (uint32_t i : redo) {
            rc = frame_graph_render(sp, s, cams + i, w, h, st, host_out ? host_out + i * img : nullptr);
            if (rc != SF_OK) return rc;
        }
        if (!redo.empty() && redo.back() == count - 1) return SF_OK;
        // The scratch's state is the last frame's (rendered again below).
        return frame_graph_render(sp, s, cams + count - 1, w, h, st, nullptr);
    }
    const uint32_t* last = g.frame_words + 16 * (size_t)(count - 1);
    uint64_t total = 0;
    std::memcpy(&total, last + 4, 8);
    frame_graph_settle(s, last, total);
    s->longest = longest;  // the batch's longest list picks the next graph's sort form
    return SF_OK;
}

int frame_render(sf_splats sp, sf_scratch s, const sf_camera* cam, uint32_t w, uint32_t h, cudaStream_t st,
                 uint32_t* host_out) {
    if (!sp || !s || !cam) return fail(SF_ERR_ARG, "null argument");
    if (w == 0 || h == 0 || w > 65535 * 16 || h > 65535 * 16) return fail(SF_ERR_SHAPE, "bad image size");
    SF_CK(use_device(s->ctx->device));
    if (s->total != sp->n || s->w != w || s->h != h) SF_CK(scratch_build(s, sp->n, w, h));
    if (!frame_graph_usable(sp, s)) return kNoFrameGraph;
    return frame_graph_render(sp, s, cam, w, h, st, host_out);
}

}  // namespace

// ================================================================ C ABI

extern "C" {

const char* sf_last_error(void) { return g_err.c_str(); }
uint64_t sf_kernel_launches(void) { return sfk::launches(); }
int sf_abi_version(void) { return SF_ABI_VERSION; }

int sf_ctx_create(int device, sf_ctx* out) {
    SF_TRY({
        if (!out) return fail(SF_ERR_ARG, "null out");
        *out = nullptr;
        int count = 0;
        SF_CK(cudaGetDeviceCount(&count));
        if (device < 0 || device >= count) return fail(SF_ERR_ARG, "no such CUDA device");
        SF_CK(cudaSetDevice(device));
        auto* c = new sf_ctx_t();
        c->device = device;
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) c->sm_count = prop.multiProcessorCount;
        *out = c;
        return SF_OK;
    })
}

int sf_ctx_destroy(sf_ctx ctx) {
    if (!ctx) return SF_OK;
    use_device(ctx->device);
    dfree(ctx->lut);
    delete ctx;
    return SF_OK;
}

int sf_buffer_alloc(sf_ctx ctx, size_t bytes, void** dptr) {
    if (!ctx || !dptr) return fail(SF_ERR_ARG, "null argument");
    SF_CK(use_device(ctx->device));
    SF_CK(cudaMalloc(dptr, bytes ? bytes : 1));
    return SF_OK;
}

int sf_buffer_free(sf_ctx ctx, void* dptr) {
    if (!ctx) return fail(SF_ERR_ARG, "null ctx");
    if (dptr) SF_CK(cudaFree(dptr));
    return SF_OK;
}

int sf_memcpy_htod(void* dst, const void* src, size_t bytes, sf_stream stream) {
    if (bytes == 0) return SF_OK;
    SF_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, S(stream)));
    return SF_OK;
}

int sf_memcpy_dtoh(void* dst, const void* src, size_t bytes, sf_stream stream) {
    if (bytes == 0) return SF_OK;
    SF_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, S(stream)));
    SF_CK(cudaStreamSynchronize(S(stream)));
    return SF_OK;
}

int sf_memset(void* dst, int value, size_t bytes, sf_stream stream) {
    if (bytes == 0) return SF_OK;
    SF_CK(cudaMemsetAsync(dst, value, bytes, S(stream)));
    return SF_OK;
}

int sf_stream_sync(sf_stream stream) {
    SF_CK(cudaStreamSynchronize(S(stream)));
    return SF_OK;
}

int sf_host_alloc(size_t bytes, void** hptr) {
    if (!hptr) return fail(SF_ERR_ARG, "null argument");
    SF_CK(cudaMallocHost(hptr, bytes ? bytes : 1));
    return SF_OK;
}

int sf_host_free(void* hptr) {
    if (hptr) SF_CK(cudaFreeHost(hptr));
    return SF_OK;
}

int sf_camera_look_at(const float position[3], const float target[3], sf_camera* out) {
    if (!position || !target || !out) return fail(SF_ERR_ARG, "null argument");
    camera_look_at(position, target, out);
    return SF_OK;
}

int sf_camera_focal(const sf_camera* cam, uint32_t w, uint32_t h, float out[2]) {
    if (!cam || !out) return fail(SF_ERR_ARG, "null argument");
    sf_view v;
    view_for_camera(*cam, w, h, &v);
    out[0] = v.focal[0];
    out[1] = v.focal[1];
    return SF_OK;
}

int sf_view_for_camera(const sf_camera* cam, uint32_t w, uint32_t h, sf_view* out) {
    if (!cam || !out) return fail(SF_ERR_ARG, "null argument");
    view_for_camera(*cam, w, h, out);
    return SF_OK;
}

int sf_splats_create(sf_ctx ctx, const float* attributes, const float* sh, uint32_t n,
                     uint32_t sh_per_ch, sf_splats* out) {
    SF_TRY({
        if (!ctx || !attributes || !sh || !out) return fail(SF_ERR_ARG, "null argument");
        *out = nullptr;
        if (n == 0) return fail(SF_ERR_SHAPE, "Splats::new: zero splats");
        if (sh_per_ch == 0) return fail(SF_ERR_SHAPE, "sh_per_ch must be at least 1");
        SF_CK(use_device(ctx->device));
        auto* s = new sf_splats_t();
        s->ctx = ctx;
        s->n = n;
        s->K = sh_per_ch;
        cudaError_t e = dalloc(&s->attr, (size_t)11 * n);
        if (e == cudaSuccess) e = dalloc(&s->sh, (size_t)3 * sh_per_ch * n);
        if (e == cudaSuccess) e = dalloc(&s->geom, (size_t)kGeomPlanes * n);
        if (e == cudaSuccess) e = cudaMemcpy(s->attr, attributes, (size_t)11 * n * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(s->sh, sh, (size_t)3 * sh_per_ch * n * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = launch_splat_geom(s->attr, n, s->geom, nullptr);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            dfree(s->attr);
            dfree(s->sh);
            dfree(s->geom);
            delete s;
            return fail(e == cudaErrorMemoryAllocation ? SF_ERR_NOMEM : SF_ERR_CUDA, cudaGetErrorString(e));
        }
        for (int k = 0; k < 3; ++k) { s->bounds[k] = 3.4028235e38f; s->bounds[3 + k] = -3.4028235e38f; }
        for (uint32_t i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) {
                const float v = attributes[(size_t)k * n + i];
                s->bounds[k] = std::min(s->bounds[k], v);
                s->bounds[3 + k] = std::max(s->bounds[3 + k], v);
            }
        *out = s;
        return SF_OK;
    })
}

int sf_splats_destroy(sf_splats s) {
    if (!s) return SF_OK;
    use_device(s->ctx->device);
    dfree(s->attr);
    dfree(s->sh);
    dfree(s->geom);
    delete s;
    return SF_OK;
}

int sf_splats_info(sf_splats s, uint32_t* n, uint32_t* sh_per_ch, float bounds[6],
                   const float** attributes_dev, const float** sh_dev) {
    if (!s) return fail(SF_ERR_ARG, "null splats");
    if (n) *n = s->n;
    if (sh_per_ch) *sh_per_ch = s->K;
    if (bounds) std::memcpy(bounds, s->bounds, sizeof(s->bounds));
    if (attributes_dev) *attributes_dev = s->attr;
    if (sh_dev) *sh_dev = s->sh;
    return SF_OK;
}

int sf_scratch_create(sf_ctx ctx, uint32_t total, uint32_t w, uint32_t h, sf_scratch* out) {
    SF_TRY({
        if (!ctx || !out) return fail(SF_ERR_ARG, "null argument");
        *out = nullptr;
        if (w == 0 || h == 0) return fail(SF_ERR_SHAPE, "zero image size");
        SF_CK(use_device(ctx->device));
        auto* s = new sf_scratch_t();
        s->ctx = ctx;
        cudaError_t e = scratch_build(s, total, w, h);
        if (e != cudaSuccess) {
            scratch_free_frame(s);
            scratch_free_isects(s);
            delete s;
            return fail(e == cudaErrorMemoryAllocation ? SF_ERR_NOMEM : SF_ERR_CUDA, cudaGetErrorString(e));
        }
        *out = s;
        return SF_OK;
    })
}

int sf_scratch_destroy(sf_scratch s) {
    if (!s) return SF_OK;
    use_device(s->ctx->device);
    if (s->twin_stream) {
        cudaStreamSynchronize(s->twin_stream);
        cudaStreamDestroy(s->twin_stream);
    }
    if (s->fork) cudaEventDestroy(s->fork);
    if (s->join) cudaEventDestroy(s->join);
    sf_scratch_destroy(s->twin);
    scratch_free_frame(s);
    scratch_free_isects(s);
    dfree(s->words);
    dfree(s->stats);
    if (s->host_words) cudaFreeHost(s->host_words);
    sort_streams_destroy(&s->sort_streams);
    if (s->fg.exec) cudaGraphExecDestroy(s->fg.exec);
    if (s->fg.stream) cudaStreamDestroy(s->fg.stream);
    dfree(s->fg.view_dev);
    if (s->fg.view_host) cudaFreeHost(s->fg.view_host);
    if (s->fg.copy) {
        cudaStreamSynchronize(s->fg.copy);
        cudaStreamDestroy(s->fg.copy);
    }
    for (int k = 0; k < 2; ++k) {
        if (s->fg.ready[k]) cudaEventDestroy(s->fg.ready[k]);
        if (s->fg.copied[k]) cudaEventDestroy(s->fg.copied[k]);
        dfree(s->fg.stage[k]);
    }
    if (s->fg.views) cudaFreeHost(s->fg.views);
    if (s->fg.frame_words) cudaFreeHost(s->fg.frame_words);
    dfree(s->fg.ring);
    dfree(s->fg.ring_counter);
    delete s;
    return SF_OK;
}

int sf_scratch_set_tuning(sf_scratch s, const sf_tuning* t) {
    if (!s || !t) return fail(SF_ERR_ARG, "null argument");
    if (t->raster_cull > 1 || t->raster_detail > 1) return fail(SF_ERR_ARG, "raster flags must be 0 or 1");
    if (t->isect_build > SF_ISECTS_DEPTH_SORTED) return fail(SF_ERR_ARG, "unknown isect_build");
    if (t->raster_order > SF_ORDER_HYBRID) return fail(SF_ERR_ARG, "unknown raster_order");
    if (t->raster_schedule > SF_SCHEDULE_TILES) return fail(SF_ERR_ARG, "unknown raster_schedule");
    if (t->raster_split != 0 && t->raster_split != 1 && t->raster_split != 2 && t->raster_split != 4)
        return fail(SF_ERR_ARG, "raster_split must be 1, 2 or 4");
    if (t->radix_bits != 0 && (t->radix_bits < 4 || t->radix_bits > 8))
        return fail(SF_ERR_ARG, "radix_bits must be 4..8 (0: 8)");
    if (t->frame_pipes > 2) return fail(SF_ERR_ARG, "frame_pipes must be 1 or 2 (0: 2)");
    s->tuning = *t;
    return SF_OK;
}

int sf_scratch_get_tuning(sf_scratch s, sf_tuning* t) {
    if (!s || !t) return fail(SF_ERR_ARG, "null argument");
    *t = s->tuning;
    return SF_OK;
}

int sf_scratch_capacity(sf_scratch s, uint64_t* capacity) {
    if (!s || !capacity) return fail(SF_ERR_ARG, "null argument");
    *capacity = s->cap;
    return SF_OK;
}

int sf_scratch_reserve(sf_scratch s, uint64_t isects) {
    SF_TRY({
        if (!s) return fail(SF_ERR_ARG, "null scratch");
        if (isects > kMaxIsects) return fail(SF_ERR_CAPACITY, "intersection count exceeds 2^30-1");
        SF_CK(use_device(s->ctx->device));
        SF_CK(grow_isects(s, isects));
        if (s->twin && s->twin->bitmap) SF_CK(grow_isects(s->twin, isects));
        return SF_OK;
    })
}

int sf_prepare_isects(sf_splats s, sf_scratch scratch, const sf_camera* cam, uint32_t w, uint32_t h,
                      sf_stream stream, sf_isects* out) {
    SF_TRY({ return prepare(s, scratch, cam, w, h, S(stream), out); })
}

int sf_finalize_rgb(sf_splats s, sf_scratch scratch, const sf_isects* isects, uint32_t w, uint32_t h,
                    int want_float, sf_stream stream) {
    SF_TRY({
        if (!s || !scratch || !isects) return fail(SF_ERR_ARG, "null argument");
        if (!scratch->prepared || scratch->w != w || scratch->h != h)
            return fail(SF_ERR_SHAPE, "finalize without a matching prepare");
        return finalize_rgb(scratch, isects, want_float != 0, S(stream));
    })
}

int sf_render_with(sf_splats s, sf_scratch scratch, const sf_camera* cam, uint32_t w, uint32_t h,
                   sf_stream stream, const uint32_t** bitmap, uint32_t* row_stride) {
    SF_TRY({
        int rc = frame_render(s, scratch, cam, w, h, S(stream), nullptr);
        if (rc != kNoFrameGraph) {
            if (rc != SF_OK) return rc;
            if (bitmap) *bitmap = scratch->bitmap;
            if (row_stride) *row_stride = scratch->row_stride;
            return SF_OK;
        }
        rc = prepare(s, scratch, cam, w, h, S(stream), nullptr, true);
        if (rc != SF_OK) return rc;
        rc = finalize_rgb(scratch, nullptr, false, S(stream));
        if (rc != SF_OK) return rc;
        if (bitmap) *bitmap = scratch->bitmap;
        if (row_stride) *row_stride = scratch->row_stride;
        return SF_OK;
    })
}

int sf_render_posterior(sf_splats s, sf_scratch scratch, sf_beta beta, const sf_camera* cam, uint32_t w,
                        uint32_t h, sf_stream stream, const uint32_t** bitmap, uint32_t* row_stride) {
    SF_TRY({
        if (!s || !scratch) return fail(SF_ERR_ARG, "null argument");
        // A posterior of another size (model swapped mid-run): the plain
        // colour render, as the reference degrades (src/seg/paint.rs:30-32).
        if (!beta || beta->n != s->n) return sf_render_with(s, scratch, cam, w, h, stream, bitmap, row_stride);
        int rc = prepare(s, scratch, cam, w, h, S(stream), nullptr, true);
        if (rc != SF_OK) return rc;
        SF_CK(launch_paint_posterior(beta->a, beta->b, s->n, scratch->color, S(stream)));
        rc = finalize_rgb(scratch, nullptr, false, S(stream));
        if (rc != SF_OK) return rc;
        if (bitmap) *bitmap = scratch->bitmap;
        if (row_stride) *row_stride = scratch->row_stride;
        return SF_OK;
    })
}

int sf_splats_tint(sf_splats s, sf_beta beta, float r, float g, float b, sf_stream stream) {
    SF_TRY({
        if (!s || !beta) return fail(SF_ERR_ARG, "null argument");
        if (beta->n != s->n) return fail(SF_ERR_SHAPE, "posterior size differs from the splat count");
        SF_CK(use_device(s->ctx->device));
        SF_CK(launch_tint(s->sh, beta->a, beta->b, s->n, r, g, b, S(stream)));
        return SF_OK;
    })
}

int sf_splats_save_colors(sf_splats s, float* dst, sf_stream stream) {
    SF_TRY({
        if (!s || !dst) return fail(SF_ERR_ARG, "null argument");
        SF_CK(use_device(s->ctx->device));
        SF_CK(cudaMemcpyAsync(dst, s->sh, (size_t)3 * s->n * 4, cudaMemcpyDeviceToDevice, S(stream)));
        return SF_OK;
    })
}

int sf_splats_restore_colors(sf_splats s, const float* src, sf_stream stream) {
    SF_TRY({
        if (!s || !src) return fail(SF_ERR_ARG, "null argument");
        SF_CK(use_device(s->ctx->device));
        SF_CK(cudaMemcpyAsync(s->sh, src, (size_t)3 * s->n * 4, cudaMemcpyDeviceToDevice, S(stream)));
        return SF_OK;
    })
}

int sf_render_float(sf_splats s, sf_scratch scratch, const sf_camera* cam, uint32_t w, uint32_t h,
                    sf_stream stream, const float** rgba) {
    SF_TRY({
        int rc = prepare(s, scratch, cam, w, h, S(stream), nullptr, true);
        if (rc != SF_OK) return rc;
        rc = finalize_rgb(scratch, nullptr, true, S(stream));
        if (rc != SF_OK) return rc;
        if (rgba) *rgba = reinterpret_cast<const float*>(scratch->rgba);
        return SF_OK;
    })
}

int sf_render_forward(sf_splats s, sf_scratch scratch, const sf_camera* cam, uint32_t w, uint32_t h,
                      sf_stream stream, const float** rgba) {
    SF_TRY({
        int rc = prepare(s, scratch, cam, w, h, S(stream), nullptr);
        if (rc != SF_OK) return rc;
        rc = finalize_rgb(scratch, nullptr, true, S(stream), true);
        if (rc != SF_OK) return rc;
        scratch->has_forward = true;
        scratch->fwd_cam = *cam;
        if (rgba) *rgba = reinterpret_cast<const float*>(scratch->rgba);
        return SF_OK;
    })
}

int sf_render_backward(sf_splats s, sf_scratch scratch, const sf_camera* cam, uint32_t w, uint32_t h,
                       const float* dl_drgba, float* d_attr, float* d_sh, float* d_proj,
                       sf_stream stream) {
    SF_TRY({
        if (!s || !scratch || !cam || !dl_drgba || !d_attr || !d_sh)
            return fail(SF_ERR_ARG, "null argument");
        if (!scratch->has_forward || scratch->w != w || scratch->h != h || scratch->total != s->n ||
            std::memcmp(&scratch->fwd_cam, cam, sizeof(sf_camera)) != 0)
            return fail(SF_ERR_SHAPE, "backward needs the scratch's last sf_render_forward of this camera and size");
        cudaStream_t st = S(stream);
        SF_CK(use_device(scratch->ctx->device));
        float* d2d = d_proj;
        if (!d2d) {
            if (!scratch->d2d) SF_CK(dalloc(&scratch->d2d, (size_t)scratch->total * 9));
            d2d = scratch->d2d;
        }
        SF_CK(cudaMemsetAsync(d2d, 0, (size_t)scratch->total * 9 * sizeof(float), st));
        BwdArgs a{};
        a.w = w;
        a.h = h;
        a.tiles_x = scratch->tiles_x;
        a.tiles_y = scratch->tiles_y;
        a.tile_start = scratch->tile_start;
        a.gaussian_ids = scratch->gids;
        a.geo0 = scratch->geo0;
        a.geo1 = scratch->geo1;
        a.color = scratch->color;
        a.final_t = scratch->final_t;
        a.n_contrib = scratch->n_contrib;
        a.dl = reinterpret_cast<const float4*>(dl_drgba);
        a.d2d = d2d;
        SF_CK(launch_raster_bwd(a, st));
        sf_view view;
        view_for_camera(*cam, w, h, &view);
        SF_CK(launch_project_bwd(view, s->attr, s->sh, s->n, s->K, d2d, d_attr, d_sh, st));
        return SF_OK;
    })
}

int sf_render_feature_adjoint(sf_splats s, sf_scratch scratch, const sf_camera* cam, uint32_t w, uint32_t h,
                              sf_mask mask, sf_stream stream, float* fg, float* bg) {
    SF_TRY({
        if (!s || !scratch || !cam || !fg || !bg) return fail(SF_ERR_ARG, "null argument");
        if (mask && (mask->w != w || mask->h != h)) return fail(SF_ERR_SHAPE, "mask size does not match the frame");
        cudaStream_t st = S(stream);
        // Sorted lists: the adjoint replays them back to front.
        int rc = prepare(s, scratch, cam, w, h, st, nullptr);
        if (rc != SF_OK) return rc;
        const size_t pixels = (size_t)w * h;
        if (!scratch->final_t) SF_CK(dalloc(&scratch->final_t, pixels));
        if (!scratch->n_contrib) SF_CK(dalloc(&scratch->n_contrib, pixels));
        scratch->has_forward = false;  // the RGB adjoint's state is overwritten
        RasterArgs a = raster_args(scratch, nullptr);
        a.final_t = scratch->final_t;
        a.n_contrib = scratch->n_contrib;
        SF_CK(cudaMemsetAsync(scratch->stats, 0, 32, st));
        SF_CK(launch_raster(3, a, st));
        SF_CK(cudaMemsetAsync(fg, 0, (size_t)s->n * 4, st));
        SF_CK(cudaMemsetAsync(bg, 0, (size_t)s->n * 4, st));
        FeatureBwdArgs f{};
        f.w = w;
        f.h = h;
        f.tiles_x = scratch->tiles_x;
        f.tiles_y = scratch->tiles_y;
        f.tile_start = scratch->tile_start;
        f.gaussian_ids = scratch->gids;
        f.geo0 = scratch->geo0;
        f.geo1 = scratch->geo1;
        f.final_t = scratch->final_t;
        f.n_contrib = scratch->n_contrib;
        f.mask = mask ? mask->bits : nullptr;
        f.mask_wpr = mask ? mask->wpr : 0u;
        f.fg = fg;
        f.bg = bg;
        SF_CK(launch_feature_bwd(f, st));
        return SF_OK;
    })
}

int sf_render_to_host(sf_splats s, sf_scratch scratch, const sf_camera* cam, uint32_t w, uint32_t h,
                      sf_stream stream, uint32_t* out) {
    SF_TRY({
        if (!out) return fail(SF_ERR_ARG, "null out");
        int rc = frame_render(s, scratch, cam, w, h, S(stream), out);
        if (rc != kNoFrameGraph) return rc;
        rc = prepare(s, scratch, cam, w, h, S(stream), nullptr, true);
        if (rc != SF_OK) return rc;
        rc = finalize_rgb(scratch, nullptr, false, S(stream));
        if (rc != SF_OK) return rc;
        SF_CK(cudaMemcpy2DAsync(out, (size_t)w * 4, scratch->bitmap, (size_t)scratch->row_stride * 4,
                                (size_t)w * 4, h, cudaMemcpyDeviceToHost, S(stream)));
        SF_CK(cudaStreamSynchronize(S(stream)));
        return SF_OK;
    })
}

int sf_render_frames(sf_splats s, sf_scratch scratch, const sf_camera* cams, uint32_t count, uint32_t w,
                     uint32_t h, sf_stream stream) {
    SF_TRY({
        if (!s || !scratch || (count && !cams)) return fail(SF_ERR_ARG, "null argument");
        if (count == 0) return SF_OK;
        if (w == 0 || h == 0 || w > 65535 * 16 || h > 65535 * 16) return fail(SF_ERR_SHAPE, "bad image size");
        cudaStream_t st = S(stream);
        SF_CK(use_device(scratch->ctx->device));
        if (scratch->total != s->n || scratch->w != w || scratch->h != h) SF_CK(scratch_build(scratch, s->n, w, h));
        if (frame_graph_usable(s, scratch)) return frames_graph_render(s, scratch, cams, count, w, h, st, nullptr);
        for (uint32_t i = 0; i < count; ++i) {
            const int rc = sf_render_with(s, scratch, cams + i, w, h, stream, nullptr, nullptr);
            if (rc != SF_OK) return rc;
        }
        return SF_OK;
    })
}

int sf_render_frames_to_host(sf_splats s, sf_scratch scratch, const sf_camera* cams, uint32_t count,
                             uint32_t w, uint32_t h, sf_stream stream, uint32_t* out) {
    SF_TRY({
        if (!s || !scratch || (count && (!cams || !out))) return fail(SF_ERR_ARG, "null argument");
        if (count == 0) return SF_OK;
        if (w == 0 || h == 0 || w > 65535 * 16 || h > 65535 * 16) return fail(SF_ERR_SHAPE, "bad image size");
        cudaStream_t st = S(stream);
        SF_CK(use_device(scratch->ctx->device));
        if (scratch->total != s->n || scratch->w != w || scratch->h != h) SF_CK(scratch_build(scratch, s->n, w, h));
        if (frame_graph_usable(s, scratch)) return frames_graph_render(s, scratch, cams, count, w, h, st, out);
        for (uint32_t i = 0; i < count; ++i) {
            const int rc = sf_render_to_host(s, scratch, cams + i, w, h, stream, out + (size_t)i * w * h);
            if (rc != SF_OK) return rc;
        }
        return SF_OK;
    })
}

static int scratch_autotune(sf_splats s, sf_scratch scratch, const sf_camera* cams, uint32_t count, uint32_t w,
                            uint32_t h, sf_stream stream, sf_tuning* best, double* best_ms) {
    {
        if (!s || !scratch || !cams || count == 0) return fail(SF_ERR_ARG, "null argument");
        SF_CK(use_device(scratch->ctx->device));
        cudaStream_t st = S(stream);
        cudaEvent_t e0, e1;
        SF_CK(cudaEventCreate(&e0));
        SF_CK(cudaEventCreate(&e1));
        // One warm-up path (captures the graph, settles the capacity), then
        // the best of three timed paths.
        auto time_of = [&](const sf_tuning& t, float* out_ms) -> int {
            int rc = sf_scratch_set_tuning(scratch, &t);
            if (rc != SF_OK) return rc;
            rc = sf_render_frames(s, scratch, cams, count, w, h, stream);
            if (rc != SF_OK) return rc;
            float ms_best = 1e30f;
            for (int rep = 0; rep < 3; ++rep) {
                SF_CK(cudaEventRecord(e0, st));
                rc = sf_render_frames(s, scratch, cams, count, w, h, stream);
                if (rc != SF_OK) return rc;
                SF_CK(cudaEventRecord(e1, st));
                SF_CK(cudaEventSynchronize(e1));
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                ms_best = std::min(ms_best, ms);
            }
            *out_ms = ms_best;
            return SF_OK;
        };
        sf_tuning winner = scratch->tuning;
        winner.raster_detail = 0;
        if (winner.raster_split == 0) winner.raster_split = 1;
        if (winner.frame_pipes == 0) winner.frame_pipes = 2;
        float winner_ms = 1e30f;
        int rc = time_of(winner, &winner_ms);
        if (rc != SF_OK) return rc;
        const uint32_t vals[5][3] = {{0, 1, 0}, {1, 2, 4}, {SF_ORDER_SORTED, SF_ORDER_HYBRID, SF_ORDER_IN_RASTER},
                                     {SF_SCHEDULE_LONGEST, SF_SCHEDULE_TILES, 0}, {2, 1, 0}};
        const int nvals[5] = {2, 3, 3, 2, 2};
        for (int sweep = 0; sweep < 2; ++sweep)
            for (int dim = 0; dim < 5; ++dim)
                for (int k = 0; k < nvals[dim]; ++k) {
                    sf_tuning t = winner;
                    uint32_t* field = dim == 0 ? &t.raster_cull : dim == 1 ? &t.raster_split
                                    : dim == 2 ? &t.raster_order : dim == 3 ? &t.raster_schedule
                                                                            : &t.frame_pipes;
                    if (*field == vals[dim][k]) continue;
                    *field = vals[dim][k];
                    float ms = 0.f;
                    rc = time_of(t, &ms);
                    if (rc != SF_OK) return rc;
                    if (ms < winner_ms) {
                        winner_ms = ms;
                        winner = t;
                    }
                }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        rc = sf_scratch_set_tuning(scratch, &winner);
        if (rc != SF_OK) return rc;
        if (best) *best = winner;
        if (best_ms) *best_ms = winner_ms / count;
        return SF_OK;
    }
}

int sf_scratch_autotune(sf_splats s, sf_scratch scratch, const sf_camera* cams, uint32_t count, uint32_t w,
                        uint32_t h, sf_stream stream, sf_tuning* best, double* best_ms) {
    SF_TRY({ return scratch_autotune(s, scratch, cams, count, w, h, stream, best, best_ms); })
}

int sf_scratch_stats(sf_scratch s, uint64_t out[4], sf_stream stream) {
    if (!s || !out) return fail(SF_ERR_ARG, "null argument");
    SF_CK(use_device(s->ctx->device));
    SF_CK(cudaMemcpyAsync(out, s->stats, 32, cudaMemcpyDeviceToHost, S(stream)));
    SF_CK(cudaStreamSynchronize(S(stream)));
    return SF_OK;
}

int sf_scratch_buffers(sf_scratch s, const uint32_t** bitmap, const float** rgba, uint32_t* row_stride) {
    if (!s) return fail(SF_ERR_ARG, "null scratch");
    if (bitmap) *bitmap = s->bitmap;
    if (rgba) *rgba = reinterpret_cast<const float*>(s->rgba);
    if (row_stride) *row_stride = s->row_stride;
    return SF_OK;
}

int sf_scratch_read(sf_scratch s, int what, void* host, size_t bytes, sf_stream stream) {
    SF_TRY({
        if (!s || !host) return fail(SF_ERR_ARG, "null argument");
        cudaStream_t st = S(stream);
        SF_CK(use_device(s->ctx->device));
        const void* src = nullptr;
        size_t avail = 0;
        float* rows = nullptr;
        switch (what) {
            case SF_READ_DEPTH_KEYS: src = s->depth_keys; avail = (size_t)s->total * 4; break;
            case SF_READ_TILE_COUNTS: src = s->tile_counts; avail = (size_t)s->total * 4; break;
            case SF_READ_BBOX: src = s->bbox; avail = (size_t)s->total * 8; break;
            case SF_READ_PROJECTED:
                SF_CK(dalloc(&rows, (size_t)s->total * 9));
                SF_CK(launch_export_rows(s->geo0, s->geo1, s->color, s->depth_keys, s->total, rows, st));
                src = rows;
                avail = (size_t)s->total * 36;
                break;
            case SF_READ_ORDER: src = s->order; avail = (size_t)s->num_visible * 4; break;
            case SF_READ_OFFSETS: src = s->offsets; avail = (size_t)s->num_visible * 4; break;
            case SF_READ_TILE_IDS: src = s->tids; avail = (size_t)s->num_isects * 4; break;
            case SF_READ_GAUSSIAN_IDS: src = s->gids; avail = (size_t)s->num_isects * 4; break;
            case SF_READ_TILE_START: src = s->tile_start; avail = ((size_t)s->tiles_x * s->tiles_y + 1) * 4; break;
            case SF_READ_BITMAP: src = s->bitmap; avail = (size_t)s->h * s->row_stride * 4; break;
            case SF_READ_RGBA: src = s->rgba; avail = s->rgba ? (size_t)s->w * s->h * 16 : 0; break;
            case SF_READ_FINAL_T: src = s->final_t; avail = s->final_t ? (size_t)s->w * s->h * 4 : 0; break;
            case SF_READ_N_CONTRIB: src = s->n_contrib; avail = s->n_contrib ? (size_t)s->w * s->h * 4 : 0; break;
            default: return fail(SF_ERR_ARG, "unknown scratch field");
        }
        if (bytes && !src) {
            dfree(rows);
            return fail(SF_ERR_ARG, "field not produced by the last prepare (the binned build keeps no depth "
                                    "order or offsets; tile ids only through sf_prepare_isects)");
        }
        if (bytes > avail) {
            dfree(rows);
            return fail(SF_ERR_SHAPE, "read exceeds the field's size");
        }
        cudaError_t e = bytes ? cudaMemcpyAsync(host, src, bytes, cudaMemcpyDeviceToHost, st) : cudaSuccess;
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        dfree(rows);
        SF_CK(e);
        return SF_OK;
    })
}

// ------------------------------------------------------------ accumulators

uint32_t sf_fractional_bits(uint32_t w, uint32_t h) { return frac_bits(w, h); }

int sf_accum_create(sf_ctx ctx, uint32_t total, sf_accum* out) {
    SF_TRY({
        if (!ctx || !out) return fail(SF_ERR_ARG, "null argument");
        *out = nullptr;
        SF_CK(use_device(ctx->device));
        auto* a = new sf_accum_t();
        a->ctx = ctx;
        a->total = total;
        cudaError_t e = dalloc(&a->resp, total);
        if (e == cudaSuccess) e = dalloc(&a->fg, total);
        if (e == cudaSuccess) e = dalloc(&a->bg, total);
        if (e == cudaSuccess) e = cudaMemset(a->resp, 0, (size_t)std::max(total, 1u) * 4);
        if (e == cudaSuccess) e = cudaMemset(a->fg, 0, (size_t)std::max(total, 1u) * 4);
        if (e == cudaSuccess) e = cudaMemset(a->bg, 0, (size_t)std::max(total, 1u) * 4);
        if (e != cudaSuccess) {
            dfree(a->resp); dfree(a->fg); dfree(a->bg);
            delete a;
            return fail(SF_ERR_NOMEM, cudaGetErrorString(e));
        }
        *out = a;
        return SF_OK;
    })
}

int sf_accum_destroy(sf_accum a) {
    if (!a) return SF_OK;
    use_device(a->ctx->device);
    dfree(a->resp); dfree(a->fg); dfree(a->bg);
    delete a;
    return SF_OK;
}

int sf_accum_info(sf_accum a, float* scale, const uint32_t** resp, const uint32_t** fg,
                  const uint32_t** bg) {
    if (!a) return fail(SF_ERR_ARG, "null accumulator");
    if (scale) *scale = a->scale;
    if (resp) *resp = a->resp;
    if (fg) *fg = a->fg;
    if (bg) *bg = a->bg;
    return SF_OK;
}

int sf_accum_set_scale(sf_accum a, float scale) {
    if (!a) return fail(SF_ERR_ARG, "null accumulator");
    if (!(scale > 0.0f)) return fail(SF_ERR_ARG, "scale must be positive");
    a->scale = scale;
    return SF_OK;
}

int sf_mask_create_packed(sf_ctx ctx, uint32_t w, uint32_t h, const uint32_t* words, sf_mask* out) {
    SF_TRY({
        if (!ctx || !words || !out) return fail(SF_ERR_ARG, "null argument");
        *out = nullptr;
        SF_CK(use_device(ctx->device));
        auto* m = new sf_mask_t();
        m->w = w;
        m->h = h;
        m->wpr = (w + 31) / 32;
        const size_t cnt = (size_t)m->wpr * h;
        cudaError_t e = dalloc(&m->bits, cnt);
        if (e == cudaSuccess && cnt) e = cudaMemcpy(m->bits, words, cnt * 4, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            dfree(m->bits);
            delete m;
            return fail(SF_ERR_CUDA, cudaGetErrorString(e));
        }
        *out = m;
        return SF_OK;
    })
}

int sf_mask_create(sf_ctx ctx, uint32_t w, uint32_t h, const uint8_t* bytes, sf_mask* out,
                   uint32_t* fg_pixels) {
    SF_TRY({
        if (!bytes) return fail(SF_ERR_ARG, "null mask bytes");
        const uint32_t wpr = (w + 31) / 32;
        std::vector<uint32_t> bits((size_t)wpr * h, 0u);
        uint32_t fg = 0;
        for (uint32_t y = 0; y < h; ++y)
            for (uint32_t x = 0; x < w; ++x)
                if (bytes[(size_t)y * w + x]) {
                    bits[(size_t)y * wpr + x / 32] |= 1u << (x % 32);
                    ++fg;
                }
        if (fg_pixels) *fg_pixels = fg;
        return sf_mask_create_packed(ctx, w, h, bits.data(), out);
    })
}

int sf_mask_destroy(sf_mask m) {
    if (!m) return SF_OK;
    dfree(m->bits);
    delete m;
    return SF_OK;
}

int sf_render_responsibility(sf_splats s, sf_scratch scratch, sf_accum acc, const sf_camera* cam,
                             uint32_t w, uint32_t h, sf_stream stream) {
    SF_TRY({
        if (!acc) return fail(SF_ERR_ARG, "null accumulator");
        int rc = prepare(s, scratch, cam, w, h, S(stream), nullptr, true);
        if (rc != SF_OK) return rc;
        return accumulate(scratch, nullptr, w, h, acc, nullptr, S(stream));
    })
}

int sf_accumulate_prepared(sf_splats s, sf_scratch scratch, const sf_isects* isects, uint32_t w,
                           uint32_t h, sf_accum acc, sf_mask mask, sf_stream stream) {
    SF_TRY({
        if (!s || !scratch || !isects || !acc) return fail(SF_ERR_ARG, "null argument");
        if (!scratch->prepared || scratch->w != w || scratch->h != h)
            return fail(SF_ERR_SHAPE, "accumulate without a matching prepare");
        SF_CK(use_device(scratch->ctx->device));
        return accumulate(scratch, isects, w, h, acc, mask, S(stream));
    })
}

// ------------------------------------------------------------------ Beta

static int beta_alloc(sf_ctx ctx, uint32_t n, sf_beta* out) {
    auto* b = new sf_beta_t();
    b->ctx = ctx;
    b->n = n;
    b->blocks = eig_blocks(n, ctx->sm_count);
    cudaError_t e = dalloc(&b->a, n);
    if (e == cudaSuccess) e = dalloc(&b->b, n);
    if (e == cudaSuccess) e = dalloc(&b->partials, b->blocks);
    if (e == cudaSuccess) e = dalloc(&b->out, 1);
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&b->host_out), 8);
    if (e == cudaSuccess) e = ensure_lut(ctx);
    if (e != cudaSuccess) {
        dfree(b->a); dfree(b->b); dfree(b->partials); dfree(b->out);
        if (b->host_out) cudaFreeHost(b->host_out);
        delete b;
        return fail(SF_ERR_NOMEM, cudaGetErrorString(e));
    }
    *out = b;
    return SF_OK;
}

int sf_beta_create_uniform(sf_ctx ctx, uint32_t total, sf_beta* out) {
    SF_TRY({
        if (!ctx || !out) return fail(SF_ERR_ARG, "null argument");
        *out = nullptr;
        SF_CK(use_device(ctx->device));
        std::vector<float> ones(std::max(total, 1u), 1.0f);
        sf_beta b = nullptr;
        int rc = beta_alloc(ctx, total, &b);
        if (rc != SF_OK) return rc;
        SF_CK(cudaMemcpy(b->a, ones.data(), (size_t)total * 4, cudaMemcpyHostToDevice));
        SF_CK(cudaMemcpy(b->b, ones.data(), (size_t)total * 4, cudaMemcpyHostToDevice));
        *out = b;
        return SF_OK;
    })
}

int sf_beta_create(sf_ctx ctx, const float* a, const float* bb, uint32_t n, sf_beta* out) {
    SF_TRY({
        if (!ctx || !a || !bb || !out) return fail(SF_ERR_ARG, "null argument");
        *out = nullptr;
        // Beta parameters are positive and finite; anything else is refused
        // here, before any CUDA call, rather than reaching the EIG kernels.
        for (uint32_t i = 0; i < n; ++i) {
            if (!(a[i] > 0.0f && a[i] < INFINITY) || !(bb[i] > 0.0f && bb[i] < INFINITY))
                return fail(SF_ERR_ARG, "Beta parameters must be positive and finite (splat " +
                                            std::to_string(i) + ")");
        }
        SF_CK(use_device(ctx->device));
        sf_beta b = nullptr;
        int rc = beta_alloc(ctx, n, &b);
        if (rc != SF_OK) return rc;
        SF_CK(cudaMemcpy(b->a, a, (size_t)n * 4, cudaMemcpyHostToDevice));
        SF_CK(cudaMemcpy(b->b, bb, (size_t)n * 4, cudaMemcpyHostToDevice));
        *out = b;
        return SF_OK;
    })
}

int sf_beta_destroy(sf_beta b) {
    if (!b) return SF_OK;
    use_device(b->ctx->device);
    dfree(b->a); dfree(b->b); dfree(b->partials); dfree(b->out);
    dfree(b->loc_partials); dfree(b->loc_out);
    if (b->host_out) cudaFreeHost(b->host_out);
    if (b->loc_host) cudaFreeHost(b->loc_host);
    delete b;
    return SF_OK;
}

int sf_beta_read(sf_beta b, float* a, float* bb, sf_stream stream) {
    if (!b) return fail(SF_ERR_ARG, "null beta");
    if (a) SF_CK(cudaMemcpyAsync(a, b->a, (size_t)b->n * 4, cudaMemcpyDeviceToHost, S(stream)));
    if (bb) SF_CK(cudaMemcpyAsync(bb, b->b, (size_t)b->n * 4, cudaMemcpyDeviceToHost, S(stream)));
    SF_CK(cudaStreamSynchronize(S(stream)));
    return SF_OK;
}

int sf_beta_info(sf_beta b, uint32_t* n, float** a_dev, float** b_dev) {
    if (!b) return fail(SF_ERR_ARG, "null beta");
    if (n) *n = b->n;
    if (a_dev) *a_dev = b->a;
    if (b_dev) *b_dev = b->b;
    return SF_OK;
}

int sf_beta_eig_async(sf_beta b, sf_accum acc, int mode, double* eig_dev, sf_stream stream) {
    SF_TRY({
        if (!b || !acc || !eig_dev) return fail(SF_ERR_ARG, "null argument");
        if (mode != SF_EIG_LUT_F32 && mode != SF_EIG_FP64) return fail(SF_ERR_ARG, "bad EIG mode");
        if (acc->total != b->n) return fail(SF_ERR_SHAPE, "accumulator and posterior sizes differ");
        SF_CK(use_device(b->ctx->device));
        // After a masked split the responsibility is fg + bg (word for word
        // the unmasked ε).
        SF_CK(launch_eig(mode, b->a, b->b, acc->evidence ? acc->fg : acc->resp, b->n, acc->scale, b->ctx->lut,
                         b->partials, b->blocks, eig_dev, S(stream), acc->evidence ? acc->bg : nullptr));
        return SF_OK;
    })
}

int sf_beta_eig(sf_beta b, sf_accum acc, int mode, sf_stream stream, double* eig) {
    SF_TRY({
        if (!eig) return fail(SF_ERR_ARG, "null out");
        int rc = sf_beta_eig_async(b, acc, mode, b ? b->out : nullptr, stream);
        if (rc != SF_OK) return rc;
        SF_CK(cudaMemcpyAsync(b->host_out, b->out, 8, cudaMemcpyDeviceToHost, S(stream)));
        SF_CK(cudaStreamSynchronize(S(stream)));
        *eig = *b->host_out;
        return SF_OK;
    })
}

int sf_beta_eig_real(sf_beta b, const float* fg, const float* bg, int mode, sf_stream stream, double* eig) {
    SF_TRY({
        if (!b || !fg || !eig) return fail(SF_ERR_ARG, "null argument");
        if (mode != SF_EIG_LUT_F32 && mode != SF_EIG_FP64) return fail(SF_ERR_ARG, "bad EIG mode");
        SF_CK(use_device(b->ctx->device));
        SF_CK(ensure_lut(b->ctx));
        cudaStream_t st = S(stream);
        SF_CK(launch_eig_real(mode, b->a, b->b, fg, bg, b->n, b->ctx->lut, b->partials, b->blocks, b->out, st));
        SF_CK(cudaMemcpyAsync(b->host_out, b->out, 8, cudaMemcpyDeviceToHost, st));
        SF_CK(cudaStreamSynchronize(st));
        *eig = *b->host_out;
        return SF_OK;
    })
}

int sf_beta_update_real(sf_beta b, const float* fg, const float* bg, sf_stream stream) {
    SF_TRY({
        if (!b || !fg || !bg) return fail(SF_ERR_ARG, "null argument");
        SF_CK(use_device(b->ctx->device));
        SF_CK(launch_beta_update_real(fg, bg, b->a, b->b, b->n, S(stream)));
        return SF_OK;
    })
}

int sf_beta_update(sf_beta b, sf_accum acc, sf_stream stream) {
    SF_TRY({
        if (!b || !acc) return fail(SF_ERR_ARG, "null argument");
        if (acc->total != b->n) return fail(SF_ERR_SHAPE, "accumulator and posterior sizes differ");
        SF_CK(use_device(b->ctx->device));
        SF_CK(launch_beta_update(acc->scale, acc->fg, acc->bg, b->a, b->b, b->n, S(stream)));
        return SF_OK;
    })
}

int sf_localize(sf_splats s, sf_beta b, sf_stream stream, int* found, float center[3], float* radius) {
    SF_TRY({
        if (!s || !b || !found || !center || !radius) return fail(SF_ERR_ARG, "null argument");
        if (s->n != b->n) return fail(SF_ERR_SHAPE, "splat count and posterior size differ");
        SF_CK(use_device(b->ctx->device));
        if (!b->loc_out) {
            SF_CK(dalloc(&b->loc_partials, 4 * (size_t)b->blocks));
            SF_CK(dalloc(&b->loc_out, 8));
            SF_CK(cudaMallocHost(reinterpret_cast<void**>(&b->loc_host), 8 * sizeof(double)));
        }
        cudaStream_t st = S(stream);
        SF_CK(launch_localize(s->attr, b->a, b->b, b->n, b->loc_partials, b->blocks, b->loc_out, st));
        SF_CK(cudaMemcpyAsync(b->loc_host, b->loc_out, 8 * sizeof(double), cudaMemcpyDeviceToHost, st));
        SF_CK(cudaStreamSynchronize(st));
        const double* o = b->loc_host;
        *found = o[0] > 0.0 ? 1 : 0;
        for (int k = 0; k < 3; ++k) center[k] = *found ? (float)o[4 + k] : 0.0f;
        *radius = *found ? (float)o[7] : 0.0f;
        return SF_OK;
    })
}

int sf_map_labels(const float* a, const float* b, uint32_t n, uint8_t* out) {
    if ((!a || !b || !out) && n) return fail(SF_ERR_ARG, "null argument");
    for (uint32_t i = 0; i < n; ++i) out[i] = a[i] > b[i] ? 1 : 0;
    return SF_OK;
}

int sf_entropy_table(float* out) {
    SF_TRY({
        if (!out) return fail(SF_ERR_ARG, "null out");
        build_entropy_table(out);
        return SF_OK;
    })
}

int sf_table_entropy(sf_ctx ctx, const float* a, const float* b, uint32_t n, float* out,
                     sf_stream stream) {
    SF_TRY({
        if (!ctx || ((!a || !b || !out) && n)) return fail(SF_ERR_ARG, "null argument");
        SF_CK(use_device(ctx->device));
        SF_CK(ensure_lut(ctx));
        SF_CK(launch_table_probe(a, b, n, ctx->lut, out, S(stream)));
        return SF_OK;
    })
}

// ------------------------------------------------------------ sort / scan

// Waits for the stream, reads a look-back error word and clears it: a wait
// that ran out returns SF_ERR_TIMEOUT (the results are then not valid).
static int read_timeout_word(uint32_t* err_dev, cudaStream_t st) {
    uint32_t word = 0;
    SF_CK(cudaMemcpyAsync(&word, err_dev, 4, cudaMemcpyDeviceToHost, st));
    SF_CK(cudaStreamSynchronize(st));
    if (word & SF_DEV_ERR_TIMEOUT) {
        SF_CK(cudaMemsetAsync(err_dev, 0, 4, st));
        SF_CK(cudaStreamSynchronize(st));
        return fail(SF_ERR_TIMEOUT, "device look-back wait timed out");
    }
    return SF_OK;
}

uint32_t sf_bits_for(uint32_t max_exclusive) { return bits_for_u32(max_exclusive); }

int sf_radix_create(sf_ctx ctx, uint32_t max_elems, sf_radix* out) {
    SF_TRY({
        if (!ctx || !out) return fail(SF_ERR_ARG, "null argument");
        *out = nullptr;
        if (max_elems > kMaxIsects) return fail(SF_ERR_SHAPE, "radix capacity exceeds 2^30-1");
        SF_CK(use_device(ctx->device));
        auto* r = new sf_radix_t();
        r->ctx = ctx;
        r->max = max_elems;
        cudaError_t e = dalloc(&r->ka, max_elems);
        if (e == cudaSuccess) e = dalloc(&r->va, max_elems);
        if (e == cudaSuccess) e = dalloc(&r->kb, max_elems);
        if (e == cudaSuccess) e = dalloc(&r->vb, max_elems);
        if (e == cudaSuccess) e = cudaMalloc(&r->tmp, radix_temp_bytes(max_elems, 4));
        if (e == cudaSuccess) e = dalloc(&r->err, 1);
        if (e == cudaSuccess) e = cudaMemset(r->err, 0, 4);
        if (e != cudaSuccess) {
            dfree(r->ka); dfree(r->va); dfree(r->kb); dfree(r->vb); dfree(r->err);
            if (r->tmp) cudaFree(r->tmp);
            delete r;
            return fail(SF_ERR_NOMEM, cudaGetErrorString(e));
        }
        *out = r;
        return SF_OK;
    })
}

int sf_radix_destroy(sf_radix r) {
    if (!r) return SF_OK;
    use_device(r->ctx->device);
    dfree(r->ka); dfree(r->va); dfree(r->kb); dfree(r->vb); dfree(r->err);
    if (r->tmp) cudaFree(r->tmp);
    delete r;
    return SF_OK;
}

// The sort of sf_radix_argsort enqueued on st; a timed-out look-back wait
// is left in r->err.
static int radix_argsort_enqueue(sf_radix r, const uint32_t* keys, const uint32_t* vals, uint32_t n,
                                 uint32_t bits, int write_keys, cudaStream_t st, const uint32_t** keys_out,
                                 const uint32_t** vals_out, bool* launched) {
    *launched = false;
    if (!r || !keys_out || !vals_out) return fail(SF_ERR_ARG, "null argument");
    if (bits > 32) return fail(SF_ERR_ARG, "bits > 32");
    if (n <= 1 || bits == 0) {
        *keys_out = keys;
        *vals_out = vals;
        return SF_OK;
    }
    if (!keys) return fail(SF_ERR_ARG, "null keys");
    if (n > r->max)
        return fail(SF_ERR_SHAPE, "radix scratch undersized: sorted " + std::to_string(n) + " elements, capacity " +
                                      std::to_string(r->max));
    SF_CK(use_device(r->ctx->device));
    int in_b = 0;
    SF_CK(radix_sort_pairs(keys, vals, r->ka, r->va, r->kb, r->vb, n, nullptr, n, bits, write_keys != 0,
                           vals == nullptr, r->tmp, r->err, r->ctx->sm_count, st, &in_b, lookback_test_knobs(),
                           r->digit_bits));
    *keys_out = in_b ? r->kb : r->ka;
    *vals_out = in_b ? r->vb : r->va;
    *launched = true;
    return SF_OK;
}

int sf_radix_argsort(sf_radix r, const uint32_t* keys, const uint32_t* vals, uint32_t n, uint32_t bits,
                     int write_keys, sf_stream stream, const uint32_t** keys_out,
                     const uint32_t** vals_out) {
    SF_TRY({
        bool launched = false;
        const int rc = radix_argsort_enqueue(r, keys, vals, n, bits, write_keys, S(stream), keys_out, vals_out,
                                             &launched);
        if (rc != SF_OK || !launched) return rc;
        return read_timeout_word(r->err, S(stream));
    })
}

int sf_radix_argsort_async(sf_radix r, const uint32_t* keys, const uint32_t* vals, uint32_t n, uint32_t bits,
                           int write_keys, sf_stream stream, const uint32_t** keys_out,
                           const uint32_t** vals_out) {
    SF_TRY({
        bool launched = false;
        return radix_argsort_enqueue(r, keys, vals, n, bits, write_keys, S(stream), keys_out, vals_out,
                                     &launched);
    })
}

int sf_radix_status(sf_radix r, sf_stream stream) {
    SF_TRY({
        if (!r) return fail(SF_ERR_ARG, "null radix scratch");
        SF_CK(use_device(r->ctx->device));
        return read_timeout_word(r->err, S(stream));
    })
}

int sf_radix_set_digit_bits(sf_radix r, uint32_t digit_bits) {
    if (!r) return fail(SF_ERR_ARG, "null radix scratch");
    if (digit_bits < 4 || digit_bits > 8) return fail(SF_ERR_ARG, "digit_bits must be 4..8");
    r->digit_bits = digit_bits;
    return SF_OK;
}

int sf_scan_create(sf_ctx ctx, uint32_t max_elems, sf_scan* out) {
    SF_TRY({
        if (!ctx || !out) return fail(SF_ERR_ARG, "null argument");
        *out = nullptr;
        SF_CK(use_device(ctx->device));
        auto* s = new sf_scan_t();
        s->ctx = ctx;
        s->max = max_elems;
        cudaError_t e = cudaMalloc(&s->tmp, scan_temp_bytes(max_elems));
        if (e == cudaSuccess) e = dalloc(&s->total, 1);
        if (e == cudaSuccess) e = dalloc(&s->err, 1);
        if (e == cudaSuccess) e = cudaMemset(s->err, 0, 4);
        if (e != cudaSuccess) {
            if (s->tmp) cudaFree(s->tmp);
            dfree(s->total); dfree(s->err);
            delete s;
            return fail(SF_ERR_NOMEM, cudaGetErrorString(e));
        }
        *out = s;
        return SF_OK;
    })
}

int sf_scan_destroy(sf_scan s) {
    if (!s) return SF_OK;
    use_device(s->ctx->device);
    if (s->tmp) cudaFree(s->tmp);
    dfree(s->total); dfree(s->err);
    delete s;
    return SF_OK;
}

// The scan of sf_exclusive_scan_gather enqueued on st; a timed-out
// look-back wait is left in s->err.
static int scan_gather_enqueue(sf_scan s, const uint32_t* gids, const uint32_t* counts, uint32_t* offsets,
                               uint32_t n, cudaStream_t st, bool* launched) {
    *launched = false;
    if (!s) return fail(SF_ERR_ARG, "null scan scratch");
    if (n == 0) return SF_OK;
    if (!counts || !offsets) return fail(SF_ERR_ARG, "null buffer");
    if (n > s->max)
        return fail(SF_ERR_SHAPE, "offsets undersized: scanned " + std::to_string(n) + " elements, capacity " +
                                      std::to_string(s->max));
    SF_CK(use_device(s->ctx->device));
    SF_CK(exclusive_scan(gids, counts, offsets, n, nullptr, n, s->tmp, s->total, s->err, st,
                         lookback_test_knobs()));
    *launched = true;
    return SF_OK;
}

int sf_exclusive_scan_gather(sf_scan s, const uint32_t* gids, const uint32_t* counts, uint32_t* offsets,
                             uint32_t n, sf_stream stream) {
    SF_TRY({
        bool launched = false;
        const int rc = scan_gather_enqueue(s, gids, counts, offsets, n, S(stream), &launched);
        if (rc != SF_OK || !launched) return rc;
        return read_timeout_word(s->err, S(stream));
    })
}

int sf_exclusive_scan_gather_async(sf_scan s, const uint32_t* gids, const uint32_t* counts, uint32_t* offsets,
                                   uint32_t n, sf_stream stream) {
    SF_TRY({
        bool launched = false;
        return scan_gather_enqueue(s, gids, counts, offsets, n, S(stream), &launched);
    })
}

int sf_scan_status(sf_scan s, sf_stream stream) {
    SF_TRY({
        if (!s) return fail(SF_ERR_ARG, "null scan scratch");
        SF_CK(use_device(s->ctx->device));
        return read_timeout_word(s->err, S(stream));
    })
}

int sf_exclusive_scan(sf_scan s, uint32_t* buf, uint32_t n, sf_stream stream) {
    return sf_exclusive_scan_gather(s, nullptr, buf, buf, n, stream);
}

}  // extern "C"
