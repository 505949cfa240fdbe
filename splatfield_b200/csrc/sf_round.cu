// Batched segmentation-evidence round: the responsibility render and EIG of
// every candidate view of a round, all in one CUDA graph.
//
// The reference scores candidates one at a time (Segmenter::select_view,
// src/seg/active.rs:113-129): per view a render_responsibility with a blocking
// counters read-back (src/render.rs:308) and an EIG with a blocking partials
// read-back (src/seg/beta.rs:265-267) — 40 host round trips for 20 views.
// Here each view's project -> depth sort -> gather scan -> emit -> tile sort
// -> tile starts -> responsibility raster -> EIG runs with its counts kept on
// the device (grids sized by capacity, kernels read the live count), views
// are spread over `lanes` capture streams so independent views overlap on the
// GPU, and the whole round is captured once into a graph and replayed; the
// cameras reach the graph through a pinned host buffer copied in by the
// graph's first node. The host syncs once per round, reads every view's EIG
// and checks the per-view intersection totals: a view that outgrew its
// capacity is re-run after the capacity grows (the graph is rebuilt then).
// The per-view words are bit-identical to the plain per-view path: same
// kernels, same inputs, integer sums.
#include <cuda_runtime.h>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>
#include "sf_handles.h"

namespace sfk {
namespace {

uint32_t bits_for(uint32_t max_exclusive) {
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

template <typename T>
cudaError_t dalloc(T** p, size_t count) {
    *p = nullptr;
    return cudaMalloc(reinterpret_cast<void**>(p), (count ? count : 1) * sizeof(T));
}
template <typename T>
void dfree(T*& p) {
    if (p) cudaFree(reinterpret_cast<void*>(p));
    p = nullptr;
}

}  // namespace

// Buffers of one capture stream: the views it runs reuse them in turn.
struct RoundLane {
    cudaStream_t stream = nullptr;
    cudaEvent_t join = nullptr;
    uint32_t *keys = nullptr, *counts = nullptr;
    uint2* bbox = nullptr;
    float4 *geo0 = nullptr, *geo1 = nullptr;
    float2* ext = nullptr;
    uint32_t *keys_a = nullptr, *keys_b = nullptr, *order_a = nullptr, *order_b = nullptr;
    uint32_t* offsets = nullptr;
    void* scan_tmp = nullptr;
    void* sort_tmp = nullptr;
    uint64_t cap = 0;
    uint32_t *tid_e = nullptr, *gid_e = nullptr, *tid_a = nullptr, *gid_a = nullptr;  // gid_a: tid_a + cap
    uint32_t* tile_start = nullptr;
    double* partials = nullptr;
    // Adjoint round: the transmittance-only forward's per-pixel state.
    float* final_t = nullptr;
    uint32_t* n_contrib = nullptr;
    // Binned build: [chunks][max_tiles] histogram, per-tile totals, class lists.
    uint32_t* hist = nullptr;
    uint32_t* cnt = nullptr;
    uint32_t* lists = nullptr;
    GiantState giant;  // segmented sort of the longest lists
    SortStreams sort_streams;
};

}  // namespace sfk

using namespace sfk;

struct sf_round_t {
    sf_ctx_t* ctx = nullptr;
    int device = 0;
    int sm_count = 148;
    uint32_t n = 0, views = 0;
    std::vector<uint32_t> w, h;
    uint32_t max_tiles = 0;
    sf_round_tuning tuning{};
    std::vector<RoundLane> lanes;
    sf_view* views_dev = nullptr;
    sf_view* views_host = nullptr;  // pinned
    uint32_t* words = nullptr;      // [views][16]: 0 visible, 1 err, 2 n32, 4..5 total u64, 6..14 binned stats
    uint32_t* words_host = nullptr; // pinned
    double* eig_dev = nullptr;
    double* eig_host = nullptr;     // pinned
    // H(a_i, b_i) of every splat, computed once per round by the graph's
    // first kernel and read by every view's EIG (f32 or f64 by mode).
    double* h0 = nullptr;
    uint32_t* resp = nullptr;       // [views][n]: total responsibility, or fg under masks
    uint32_t* bg = nullptr;         // [views][n]: bg under masks (allocated on first use)
    std::vector<const sf_mask_t*> masks;  // this round's per-view masks (empty: responsibility)
    // Adjoint round: real-valued fg / bg responsibilities [views][n]
    // (allocated on first use); masks may be null entries (all in fg).
    bool adjoint = false;
    float* afg = nullptr;
    float* abg = nullptr;
    uint64_t max_pixels = 0;
    uint32_t eig_blocks = 1;
    uint64_t want_cap = 0;
    // graph cache
    cudaStream_t main = nullptr;
    cudaEvent_t fork = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t graph_kernels = 0;  // kernel nodes of exec
    const void* g_splats = nullptr;
    const void* g_beta = nullptr;
    int g_mode = -1;
    int g_adjoint = -1;
    uint32_t g_lanes = 0, g_cull = 0, g_build = 0, g_order = 0, g_split = 0, g_radix = 0;
    // Per view: the longest tile list of the last round, and whether the
    // graph includes the segmented sort of the longest lists for the view.
    std::vector<uint32_t> longest;
    std::vector<uint8_t> g_giant;
    uint32_t chunks = 1;
    std::vector<const sf_mask_t*> g_masks;
};

namespace {

void lane_free(RoundLane& L) {
    dfree(L.keys); dfree(L.counts); dfree(L.bbox); dfree(L.geo0); dfree(L.geo1); dfree(L.ext);
    dfree(L.keys_a); dfree(L.keys_b); dfree(L.order_a); dfree(L.order_b); dfree(L.offsets);
    if (L.scan_tmp) cudaFree(L.scan_tmp);
    if (L.sort_tmp) cudaFree(L.sort_tmp);
    L.scan_tmp = L.sort_tmp = nullptr;
    dfree(L.tid_e); dfree(L.gid_e); dfree(L.tid_a);
    L.gid_a = nullptr;
    dfree(L.tile_start); dfree(L.partials); dfree(L.final_t); dfree(L.n_contrib);
    dfree(L.hist); dfree(L.cnt); dfree(L.lists);
    dfree(L.giant.ctrl); dfree(L.giant.sel); dfree(L.giant.mm); dfree(L.giant.hist);
    dfree(L.giant.taken); dfree(L.giant.segs);
    L.giant.lists = L.giant.seg_cap = 0;
    sort_streams_destroy(&L.sort_streams);
    if (L.stream) cudaStreamDestroy(L.stream);
    if (L.join) cudaEventDestroy(L.join);
    L.stream = nullptr;
    L.join = nullptr;
    L.cap = 0;
}

cudaError_t lane_alloc(sf_round_t* r, RoundLane& L, uint64_t cap) {
    const uint32_t n = r->n;
    cudaError_t e;
#define RA(ptr, cnt) if ((e = dalloc(&(ptr), (cnt))) != cudaSuccess) return e
    RA(L.keys, n); RA(L.counts, n); RA(L.bbox, n); RA(L.geo0, n); RA(L.geo1, n); RA(L.ext, n);
    RA(L.keys_a, n); RA(L.keys_b, n); RA(L.order_a, n); RA(L.order_b, n); RA(L.offsets, n);
    RA(L.tid_e, cap); RA(L.gid_e, cap); RA(L.tid_a, 2 * cap);
    L.gid_a = L.tid_a + cap;
    RA(L.tile_start, (size_t)r->max_tiles + 1);
    RA(L.partials, r->eig_blocks);
    RA(L.final_t, r->max_pixels);
    RA(L.n_contrib, r->max_pixels);
    if (r->max_tiles <= kBinMaxTiles) {
        RA(L.hist, (size_t)r->chunks * r->max_tiles);
        RA(L.cnt, (size_t)r->max_tiles + 1);
        RA(L.lists, (size_t)(kSortClasses + 1) * r->max_tiles);
        L.giant.lists = giant_lists(r->max_tiles);
        L.giant.seg_cap = giant_seg_cap(L.giant.lists);
        RA(L.giant.ctrl, 4);
        RA(L.giant.sel, L.giant.lists);
        RA(L.giant.mm, 2 * (size_t)L.giant.lists);
        RA(L.giant.hist, (size_t)L.giant.lists * kGiantBins);
        RA(L.giant.taken, r->max_tiles);
        RA(L.giant.segs, L.giant.seg_cap);
    }
#undef RA
    if ((e = cudaMalloc(&L.scan_tmp, scan_temp_bytes(std::max(n, r->max_tiles + 1)))) != cudaSuccess) return e;
    const size_t st = std::max(radix_temp_bytes(n, 4), radix_temp_bytes((uint32_t)cap, 4));
    if ((e = cudaMalloc(&L.sort_tmp, st)) != cudaSuccess) return e;
    if ((e = cudaStreamCreateWithFlags(&L.stream, cudaStreamNonBlocking)) != cudaSuccess) return e;
    if ((e = sort_streams_create(&L.sort_streams)) != cudaSuccess) return e;
    if ((e = cudaEventCreateWithFlags(&L.join, cudaEventDisableTiming)) != cudaSuccess) return e;
    L.cap = cap;
    return cudaSuccess;
}

void graph_drop(sf_round_t* r) {
    if (r->exec) cudaGraphExecDestroy(r->exec);
    r->exec = nullptr;
}

cudaError_t lanes_build(sf_round_t* r, uint32_t lanes, uint64_t cap) {
    graph_drop(r);
    for (auto& L : r->lanes) lane_free(L);
    r->lanes.assign(lanes, RoundLane());
    for (auto& L : r->lanes) {
        cudaError_t e = lane_alloc(r, L, cap);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// The reference's order of steps with device-side counts: depth argsort,
// gather scan, emit, stable tile sort, tile starts.
cudaError_t depth_sorted_isects(sf_round_t* r, RoundLane& L, uint32_t n, uint32_t tx, uint32_t tiles,
                                uint32_t* words, unsigned long long* total, cudaStream_t st,
                                const uint32_t** tids_out, const uint32_t** gids_out) {
    cudaError_t e;
    int in_b = 0;
    const uint32_t digit_bits = r->tuning.radix_bits ? r->tuning.radix_bits : 8u;
    if ((e = radix_sort_pairs(L.keys, nullptr, L.keys_a, L.order_a, L.keys_b, L.order_b, n, nullptr, n, 32,
                              false, true, L.sort_tmp, words + 1, r->sm_count, st, &in_b, LookbackKnobs{0u, 0u},
                              digit_bits)) != cudaSuccess)
        return e;
    const uint32_t* order = in_b ? L.order_b : L.order_a;
    if ((e = exclusive_scan(order, L.counts, L.offsets, n, nullptr, n, L.scan_tmp, total, words + 1, st)) !=
        cudaSuccess)
        return e;
    if ((e = launch_emit(order, L.bbox, L.offsets, n, tx, (uint32_t)L.cap, L.tid_e, L.gid_e, words + 1, st)) !=
        cudaSuccess)
        return e;
    if ((e = launch_clamp_count(total, (uint32_t)L.cap, words + 2, words + 1, st)) != cudaSuccess) return e;
    const uint32_t tbits = bits_for(tiles);
    const uint32_t *tids = L.tid_e, *gids = L.gid_e;
    if (tbits > 0) {
        if ((e = radix_sort_pairs(L.tid_e, L.gid_e, L.tid_a, L.gid_a, L.tid_e, L.gid_e, 0, words + 2,
                                  (uint32_t)L.cap, tbits, true, false, L.sort_tmp, words + 1, r->sm_count, st,
                                  &in_b, LookbackKnobs{0u, 0u}, digit_bits)) != cudaSuccess)
            return e;
        tids = in_b ? L.tid_e : L.tid_a;
        gids = in_b ? L.gid_e : L.gid_a;
    }
    if ((e = launch_tile_starts(tids, 0, words + 2, (uint32_t)L.cap, tiles, L.tile_start, st)) != cudaSuccess)
        return e;
    *tids_out = tids;
    *gids_out = gids;
    return cudaSuccess;
}

// Responsibility (or evidence) raster of view v and its EIG.
cudaError_t raster_and_eig(sf_round_t* r, RoundLane& L, uint32_t v, uint32_t tx, uint32_t ty, const uint32_t* gids,
                           const uint2* pairs, const float* beta_a, const float* beta_b, const float* lut, int mode,
                           cudaStream_t st) {
    cudaError_t e;
    const uint32_t n = r->n;
    const uint32_t w = r->w[v], h = r->h[v];
    uint32_t* resp = r->resp + (size_t)v * n;
    uint32_t* bg = r->masks.empty() ? nullptr : r->bg + (size_t)v * n;
    if ((e = cudaMemsetAsync(resp, 0, (size_t)n * 4, st)) != cudaSuccess) return e;
    if (bg && (e = cudaMemsetAsync(bg, 0, (size_t)n * 4, st)) != cudaSuccess) return e;
    RasterArgs a{};
    a.w = w;
    a.h = h;
    a.tiles_x = tx;
    a.tiles_y = ty;
    a.tile_start = L.tile_start;
    a.gaussian_ids = gids;
    a.pairs = pairs;
    a.lazy_min = r->tuning.raster_order == SF_ORDER_HYBRID ? kBinSharedMax : 0u;
    a.geo0 = L.geo0;
    a.geo1 = L.geo1;
    a.ext = L.ext;
    a.cull = r->tuning.raster_cull;
    a.split = r->tuning.raster_split;
    a.scale = (float)((uint64_t)1 << frac_bits(w, h));
    if (bg) {
        // Evidence: the mask splits each pixel's weights into fg / bg.
        a.mask = r->masks[v]->bits;
        a.mask_wpr = r->masks[v]->wpr;
        a.fg = resp;
        a.bg = bg;
        if ((e = launch_raster(2, a, st)) != cudaSuccess) return e;
    } else {
        a.resp = resp;
        if ((e = launch_raster(1, a, st)) != cudaSuccess) return e;
    }
    if (beta_a) {
        // Under masks the EIG sees eps = fg + bg, the same words mode 1 sums.
        if ((e = launch_eig(mode, beta_a, beta_b, resp, n, a.scale, lut, L.partials, r->eig_blocks,
                            r->eig_dev + v, st, bg, r->h0)) != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}

// Adjoint round, view v: the transmittance-only raster keeps each pixel's
// final T and last contributor, the feature adjoint replays them into the
// view's real-valued fg / bg responsibilities, and the EIG reads fg + bg.
cudaError_t adjoint_and_eig(sf_round_t* r, RoundLane& L, uint32_t v, uint32_t tx, uint32_t ty,
                            const uint32_t* gids, const float* beta_a, const float* beta_b, const float* lut,
                            int mode, cudaStream_t st) {
    cudaError_t e;
    const uint32_t n = r->n;
    const uint32_t w = r->w[v], h = r->h[v];
    float* fg = r->afg + (size_t)v * n;
    float* bg = r->abg + (size_t)v * n;
    const sf_mask_t* mask = r->masks.empty() ? nullptr : r->masks[v];
    RasterArgs a{};
    a.w = w;
    a.h = h;
    a.tiles_x = tx;
    a.tiles_y = ty;
    a.tile_start = L.tile_start;
    a.gaussian_ids = gids;
    a.geo0 = L.geo0;
    a.geo1 = L.geo1;
    a.ext = L.ext;
    a.cull = r->tuning.raster_cull;
    a.final_t = L.final_t;
    a.n_contrib = L.n_contrib;
    if ((e = launch_raster(3, a, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(fg, 0, (size_t)n * 4, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(bg, 0, (size_t)n * 4, st)) != cudaSuccess) return e;
    FeatureBwdArgs f{};
    f.w = w;
    f.h = h;
    f.tiles_x = tx;
    f.tiles_y = ty;
    f.tile_start = L.tile_start;
    f.gaussian_ids = gids;
    f.geo0 = L.geo0;
    f.geo1 = L.geo1;
    f.final_t = L.final_t;
    f.n_contrib = L.n_contrib;
    f.mask = mask ? mask->bits : nullptr;
    f.mask_wpr = mask ? mask->wpr : 0u;
    f.fg = fg;
    f.bg = bg;
    if ((e = launch_feature_bwd(f, st)) != cudaSuccess) return e;
    if (beta_a)
        return launch_eig_real(mode, beta_a, beta_b, fg, bg, n, lut, L.partials, r->eig_blocks, r->eig_dev + v, st,
                               r->h0);
    return cudaSuccess;
}

// One view's pipeline on lane L's stream.
cudaError_t enqueue_view(sf_round_t* r, RoundLane& L, uint32_t v, const sf_splats_t& sp,
                         const float* beta_a, const float* beta_b, const float* lut, int mode) {
    cudaStream_t st = L.stream;
    const uint32_t n = r->n;
    uint32_t* words = r->words + 16 * v;
    unsigned long long* total = reinterpret_cast<unsigned long long*>(words + 4);
    const uint32_t w = r->w[v], h = r->h[v];
    const uint32_t tx = (w + 15) / 16, ty = (h + 15) / 16;
    const uint32_t tiles = tx * ty;
    cudaError_t e;
    if ((e = cudaMemsetAsync(words, 0, 64, st)) != cudaSuccess) return e;
    ProjOut po{L.keys, L.counts, L.bbox, L.geo0, L.geo1, nullptr, words, r->tuning.raster_cull ? L.ext : nullptr};
    sf_view dummy{};
    if ((e = launch_project(dummy, sp.attr, sp.geom, sp.sh, n, sp.K, po, st, r->views_dev + v)) != cudaSuccess) return e;
    const uint32_t *tids = nullptr, *gids = nullptr;
    const uint2* lazy_pairs = nullptr;
    if (r->tuning.isect_build == SF_ISECTS_BINNED && L.hist) {
        // Binned build with device-side counts: the sorts take every tile as
        // the bound of each class and read the class sizes on the device.
        if ((e = launch_bin_count(L.bbox, n, tx, tiles, r->chunks, L.hist, st)) != cudaSuccess) return e;
        if ((e = launch_bin_colscan(L.hist, r->chunks, tiles, L.cnt, L.lists, words, st)) != cudaSuccess) return e;
        if ((e = exclusive_scan(nullptr, L.cnt, L.tile_start, tiles + 1, nullptr, tiles + 1, L.scan_tmp, total,
                                words + 1, st)) != cudaSuccess)
            return e;
        if ((e = launch_clamp_count(total, (uint32_t)L.cap, words + 2, words + 1, st)) != cudaSuccess) return e;
        uint2* pairs = reinterpret_cast<uint2*>(L.tid_a);
        if ((e = launch_bin_place(L.bbox, L.keys, n, tx, tiles, r->chunks, L.hist, L.tile_start, (uint32_t)L.cap,
                                  pairs, words + 1, st)) != cudaSuccess)
            return e;
        if ((e = launch_clamp_starts(L.tile_start, tiles + 1, (uint32_t)L.cap, st)) != cudaSuccess) return e;
        // The adjoint replays sorted lists: every class is sorted for it.
        const uint32_t order = r->adjoint ? SF_ORDER_SORTED : r->tuning.raster_order;
        if (order != SF_ORDER_SORTED) lazy_pairs = pairs;
        if (order != SF_ORDER_IN_RASTER) {
            uint32_t grids[kSortClasses];
            for (int k = 0; k < kSortClasses; ++k) grids[k] = tiles;
            if (order == SF_ORDER_HYBRID) grids[kSortClasses - 1] = 0;
            if ((e = launch_tile_sorts(grids, L.lists, words, tiles, L.tile_start, (uint32_t)L.cap, pairs, L.gid_e,
                                       nullptr, L.tid_e, r->sm_count, st, &L.sort_streams,
                                       giant_wanted(r->longest[v], r->g_giant[v]) ? &L.giant : nullptr)) !=
                cudaSuccess)
                return e;
            gids = L.gid_e;
        }
    } else {
        if ((e = depth_sorted_isects(r, L, n, tx, tiles, words, total, st, &tids, &gids)) != cudaSuccess)
            return e;
    }
    if (r->adjoint) return adjoint_and_eig(r, L, v, tx, ty, gids, beta_a, beta_b, lut, mode, st);
    return raster_and_eig(r, L, v, tx, ty, gids, lazy_pairs, beta_a, beta_b, lut, mode, st);
}

}  // namespace

namespace {

int rfail(int code, const std::string& msg) { return sfk::set_error(code, msg); }

#define RF_CK(expr)                                                                              \
    do {                                                                                         \
        cudaError_t e_ = (expr);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return rfail(e_ == cudaErrorMemoryAllocation ? SF_ERR_NOMEM : SF_ERR_CUDA,           \
                         std::string(#expr) + ": " + cudaGetErrorString(e_));                    \
    } while (0)

cudaError_t use_dev(int dev) {
    int cur = -1;
    cudaError_t e = cudaGetDevice(&cur);
    if (e != cudaSuccess) return e;
    return cur == dev ? cudaSuccess : cudaSetDevice(dev);
}

// Capture the whole round into r->exec.
int build_graph(sf_round_t* r, const sf_splats_t* sp, const sf_beta_t* beta, int mode) {
    graph_drop(r);
    const uint64_t launches0 = launches();
    RF_CK(cudaStreamBeginCapture(r->main, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaMemcpyAsync(r->views_dev, r->views_host, sizeof(sf_view) * r->views,
                                    cudaMemcpyHostToDevice, r->main);
    if (e == cudaSuccess && beta) e = launch_entropy(mode, beta->a, beta->b, r->n, beta->ctx->lut, r->h0, r->main);
    if (e == cudaSuccess) e = cudaEventRecord(r->fork, r->main);
    for (auto& L : r->lanes)
        if (e == cudaSuccess) e = cudaStreamWaitEvent(L.stream, r->fork, 0);
    for (uint32_t v = 0; v < r->views && e == cudaSuccess; ++v) {
        RoundLane& L = r->lanes[v % r->lanes.size()];
        e = enqueue_view(r, L, v, *sp, beta ? beta->a : nullptr, beta ? beta->b : nullptr,
                         beta ? beta->ctx->lut : nullptr, mode);
    }
    for (auto& L : r->lanes) {
        if (e == cudaSuccess) e = cudaEventRecord(L.join, L.stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(r->main, L.join, 0);
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(r->words_host, r->words, 64 * r->views, cudaMemcpyDeviceToHost, r->main);
    if (e == cudaSuccess && beta)
        e = cudaMemcpyAsync(r->eig_host, r->eig_dev, 8 * r->views, cudaMemcpyDeviceToHost, r->main);
    cudaGraph_t graph = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(r->main, &graph);
    r->graph_kernels = (uint32_t)(launches() - launches0);
    forget_launches(r->graph_kernels);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return rfail(SF_ERR_CUDA, std::string("round graph capture: ") +
                                      cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    e = cudaGraphInstantiate(&r->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        r->exec = nullptr;
        return rfail(SF_ERR_CUDA, std::string("round graph instantiate: ") + cudaGetErrorString(e));
    }
    r->g_splats = sp;
    r->g_beta = beta;
    r->g_mode = mode;
    r->g_adjoint = (int)r->adjoint;
    r->g_lanes = (uint32_t)r->lanes.size();
    r->g_cull = r->tuning.raster_cull;
    r->g_build = r->tuning.isect_build;
    r->g_order = r->tuning.raster_order;
    r->g_split = r->tuning.raster_split;
    r->g_radix = r->tuning.radix_bits;
    r->g_masks = r->masks;
    for (uint32_t v = 0; v < r->views; ++v) r->g_giant[v] = giant_wanted(r->longest[v], r->g_giant[v]);
    return SF_OK;
}

// Whether some view's choice of the segmented sort differs from the graph's.
bool giant_changed(const sf_round_t* r) {
    for (uint32_t v = 0; v < r->views; ++v)
        if (giant_wanted(r->longest[v], r->g_giant[v]) != (r->g_giant[v] != 0)) return true;
    return false;
}

// Launch the round (rebuilding buffers/graph when needed), wait, check.
int run_round(sf_round_t* r, const sf_splats_t* sp, const sf_beta_t* beta, const sf_camera* cams, int mode,
              cudaStream_t user) {
    for (uint32_t v = 0; v < r->views; ++v) view_for_camera(cams[v], r->w[v], r->h[v], &r->views_host[v]);
    for (int attempt = 0; attempt < 4; ++attempt) {
        const uint32_t lanes = std::max(1u, std::min(r->tuning.lanes ? r->tuning.lanes : 4u, r->views));
        if (r->lanes.size() != lanes || r->lanes[0].cap < r->want_cap) {
            RF_CK(lanes_build(r, lanes, std::max<uint64_t>(r->want_cap, r->lanes.empty() ? 1024 : r->lanes[0].cap)));
        }
        if (!r->exec || r->g_splats != sp || r->g_beta != beta || r->g_mode != mode ||
            r->g_adjoint != (int)r->adjoint ||
            r->g_cull != r->tuning.raster_cull || r->g_build != r->tuning.isect_build ||
            r->g_order != r->tuning.raster_order || r->g_split != r->tuning.raster_split ||
            r->g_radix != r->tuning.radix_bits || r->g_masks != r->masks ||
            giant_changed(r)) {
            const int rc = build_graph(r, sp, beta, mode);
            if (rc != SF_OK) return rc;
        }
        // Order after the caller's prior work on its stream.
        cudaEvent_t ev;
        RF_CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        RF_CK(cudaEventRecord(ev, user));
        RF_CK(cudaStreamWaitEvent(r->main, ev, 0));
        cudaEventDestroy(ev);
        RF_CK(cudaGraphLaunch(r->exec, r->main));
        note_launches(r->graph_kernels);
        RF_CK(cudaStreamSynchronize(r->main));
        uint64_t worst = 0;
        bool over = false;
        for (uint32_t v = 0; v < r->views; ++v) {
            const uint32_t* w = r->words_host + 16 * v;
            if (w[1] & SF_DEV_ERR_TIMEOUT) return rfail(SF_ERR_TIMEOUT, "device look-back wait timed out");
            uint64_t total;
            std::memcpy(&total, w + 4, 8);
            worst = std::max(worst, total);
            r->longest[v] = w[6];
            if (w[1] & SF_DEV_ERR_CAPACITY) over = true;
        }
        if (!over) return SF_OK;
        if (worst > (1ull << 30) - 1) return rfail(SF_ERR_CAPACITY, "intersection count exceeds 2^30-1");
        r->want_cap = next_pow2(worst);
        std::fprintf(stderr, "splatfield_b200: round capacity grown to %llu intersections per view\n",
                     (unsigned long long)r->want_cap);
    }
    return rfail(SF_ERR_CAPACITY, "round capacity did not settle");
}

// Process-wide autotuning cache: (device, splats, views, sizes) -> tuning.
std::mutex g_tune_mu;
struct TuneEntry {
    sf_round_tuning tuning;
    float ms;
};
std::map<std::string, TuneEntry> g_tune_cache;

std::string tune_key(const sf_round_t* r) {
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, r->device);
    std::string k = std::string(prop.name) + "|" + std::to_string(r->n) + "|" + std::to_string(r->views);
    for (uint32_t v = 0; v < r->views; ++v) k += "|" + std::to_string(r->w[v]) + "x" + std::to_string(r->h[v]);
    return k;
}

}  // namespace

extern "C" {

int sf_round_create(sf_ctx ctx, uint32_t total, uint32_t n_views, const uint32_t* widths,
                    const uint32_t* heights, sf_round* out) {
    if (!ctx || !widths || !heights || !out) return rfail(SF_ERR_ARG, "null argument");
    *out = nullptr;
    if (total == 0 || n_views == 0) return rfail(SF_ERR_SHAPE, "round needs splats and views");
    for (uint32_t v = 0; v < n_views; ++v)
        if (widths[v] == 0 || heights[v] == 0 || widths[v] > 65535 * 16 || heights[v] > 65535 * 16)
            return rfail(SF_ERR_SHAPE, "bad view size");
    RF_CK(use_dev(ctx->device));
    auto* r = new sf_round_t();
    r->ctx = ctx;
    r->device = ctx->device;
    r->sm_count = ctx->sm_count;
    r->n = total;
    r->views = n_views;
    r->w.assign(widths, widths + n_views);
    r->h.assign(heights, heights + n_views);
    r->longest.assign(n_views, 0u);
    r->g_giant.assign(n_views, 0u);
    for (uint32_t v = 0; v < n_views; ++v) {
        r->max_tiles = std::max(r->max_tiles, ((widths[v] + 15) / 16) * ((heights[v] + 15) / 16));
        r->max_pixels = std::max<uint64_t>(r->max_pixels, (uint64_t)widths[v] * heights[v]);
    }
    r->eig_blocks = eig_blocks(total, ctx->sm_count);
    r->chunks = bin_chunks(total, ctx->sm_count);
    r->tuning.lanes = 4;
    r->want_cap = std::min<uint64_t>((uint64_t)r->max_tiles * total, 1ull << 22);
    cudaError_t e = cudaStreamCreateWithFlags(&r->main, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = dalloc(&r->views_dev, n_views);
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&r->views_host), sizeof(sf_view) * n_views);
    if (e == cudaSuccess) e = dalloc(&r->words, 16 * (size_t)n_views);
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&r->words_host), 64 * (size_t)n_views);
    if (e == cudaSuccess) e = dalloc(&r->eig_dev, n_views);
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&r->eig_host), 8 * (size_t)n_views);
    if (e == cudaSuccess) e = dalloc(&r->resp, (size_t)n_views * total);
    if (e == cudaSuccess) e = dalloc(&r->h0, total);
    if (e != cudaSuccess) {
        sf_round_destroy(r);
        return rfail(e == cudaErrorMemoryAllocation ? SF_ERR_NOMEM : SF_ERR_CUDA, cudaGetErrorString(e));
    }
    *out = r;
    return SF_OK;
}

int sf_round_destroy(sf_round r) {
    if (!r) return SF_OK;
    use_dev(r->device);
    graph_drop(r);
    for (auto& L : r->lanes) lane_free(L);
    dfree(r->views_dev); dfree(r->words); dfree(r->eig_dev); dfree(r->resp); dfree(r->bg);
    dfree(r->afg); dfree(r->abg); dfree(r->h0);
    if (r->views_host) cudaFreeHost(r->views_host);
    if (r->words_host) cudaFreeHost(r->words_host);
    if (r->eig_host) cudaFreeHost(r->eig_host);
    if (r->fork) cudaEventDestroy(r->fork);
    if (r->main) cudaStreamDestroy(r->main);
    delete r;
    return SF_OK;
}

int sf_round_set_tuning(sf_round r, const sf_round_tuning* t) {
    if (!r || !t) return rfail(SF_ERR_ARG, "null argument");
    if (t->raster_cull > 1 || t->lanes > 64 || t->isect_build > SF_ISECTS_DEPTH_SORTED ||
        t->raster_order > SF_ORDER_HYBRID ||
        (t->raster_split != 0 && t->raster_split != 1 && t->raster_split != 2 && t->raster_split != 4) ||
        (t->radix_bits != 0 && (t->radix_bits < 4 || t->radix_bits > 8)))
        return rfail(SF_ERR_ARG, "bad tuning");
    r->tuning = *t;
    return SF_OK;
}

int sf_round_get_tuning(sf_round r, sf_round_tuning* t) {
    if (!r || !t) return rfail(SF_ERR_ARG, "null argument");
    *t = r->tuning;
    return SF_OK;
}

int sf_round_eig(sf_round r, sf_splats s, sf_beta beta, const sf_camera* cams, int mode, sf_stream stream,
                 double* eig) {
    try {
        if (!r || !s || !cams) return rfail(SF_ERR_ARG, "null argument");
        if (s->n != r->n) return rfail(SF_ERR_SHAPE, "splat count differs from the round's");
        if (beta && beta->n != r->n) return rfail(SF_ERR_SHAPE, "posterior size differs from the round's");
        if (beta && mode != SF_EIG_LUT_F32 && mode != SF_EIG_FP64) return rfail(SF_ERR_ARG, "bad EIG mode");
        if (beta && !eig) return rfail(SF_ERR_ARG, "null eig output");
        RF_CK(use_dev(r->device));
        r->masks.clear();
        r->adjoint = false;
        const int rc = run_round(r, s, beta, cams, mode, reinterpret_cast<cudaStream_t>(stream));
        if (rc != SF_OK) return rc;
        if (beta) std::memcpy(eig, r->eig_host, 8 * r->views);
        return SF_OK;
    } catch (const std::bad_alloc&) {
        return rfail(SF_ERR_NOMEM, "host allocation failed");
    }
}

int sf_round_evidence(sf_round r, sf_splats s, sf_beta beta, const sf_camera* cams, const sf_mask* masks,
                      int mode, sf_stream stream, double* eig) {
    try {
        if (!r || !s || !cams || !masks) return rfail(SF_ERR_ARG, "null argument");
        if (s->n != r->n) return rfail(SF_ERR_SHAPE, "splat count differs from the round's");
        if (beta && beta->n != r->n) return rfail(SF_ERR_SHAPE, "posterior size differs from the round's");
        if (beta && mode != SF_EIG_LUT_F32 && mode != SF_EIG_FP64) return rfail(SF_ERR_ARG, "bad EIG mode");
        if (beta && !eig) return rfail(SF_ERR_ARG, "null eig output");
        for (uint32_t v = 0; v < r->views; ++v) {
            if (!masks[v]) return rfail(SF_ERR_ARG, "null mask");
            if (masks[v]->w != r->w[v] || masks[v]->h != r->h[v])
                return rfail(SF_ERR_SHAPE, "mask size does not match its view");
        }
        RF_CK(use_dev(r->device));
        if (!r->bg) RF_CK(dalloc(&r->bg, (size_t)r->views * r->n));
        r->masks.assign(masks, masks + r->views);
        r->adjoint = false;
        const int rc = run_round(r, s, beta, cams, mode, reinterpret_cast<cudaStream_t>(stream));
        if (rc != SF_OK) return rc;
        if (beta) std::memcpy(eig, r->eig_host, 8 * r->views);
        return SF_OK;
    } catch (const std::bad_alloc&) {
        return rfail(SF_ERR_NOMEM, "host allocation failed");
    }
}

int sf_round_evidence_words(sf_round r, uint32_t view, const uint32_t** fg, const uint32_t** bg) {
    if (!r) return rfail(SF_ERR_ARG, "null round");
    if (view >= r->views) return rfail(SF_ERR_SHAPE, "no such view");
    if (r->masks.empty() || r->adjoint) return rfail(SF_ERR_ARG, "the last round was not a u32 evidence round");
    if (fg) *fg = r->resp + (size_t)view * r->n;
    if (bg) *bg = r->bg + (size_t)view * r->n;
    return SF_OK;
}

int sf_round_responsibility(sf_round r, uint32_t view, const uint32_t** resp, float* scale,
                            uint64_t* num_isects, uint32_t* num_visible) {
    if (!r) return rfail(SF_ERR_ARG, "null round");
    if (view >= r->views) return rfail(SF_ERR_SHAPE, "no such view");
    if (resp && r->adjoint) return rfail(SF_ERR_ARG, "the last round was an adjoint round (no words)");
    if (resp) *resp = r->resp + (size_t)view * r->n;
    if (scale) *scale = (float)((uint64_t)1 << frac_bits(r->w[view], r->h[view]));
    const uint32_t* w = r->words_host + 16 * view;
    if (num_isects) std::memcpy(num_isects, w + 4, 8);
    if (num_visible) *num_visible = w[0];
    return SF_OK;
}

int sf_round_evidence_adjoint(sf_round r, sf_splats s, sf_beta beta, const sf_camera* cams, const sf_mask* masks,
                              int mode, sf_stream stream, double* eig) {
    try {
        if (!r || !s || !cams) return rfail(SF_ERR_ARG, "null argument");
        if (s->n != r->n) return rfail(SF_ERR_SHAPE, "splat count differs from the round's");
        if (beta && beta->n != r->n) return rfail(SF_ERR_SHAPE, "posterior size differs from the round's");
        if (beta && mode != SF_EIG_LUT_F32 && mode != SF_EIG_FP64) return rfail(SF_ERR_ARG, "bad EIG mode");
        if (beta && !eig) return rfail(SF_ERR_ARG, "null eig output");
        if (masks)
            for (uint32_t v = 0; v < r->views; ++v)
                if (masks[v] && (masks[v]->w != r->w[v] || masks[v]->h != r->h[v]))
                    return rfail(SF_ERR_SHAPE, "mask size does not match its view");
        RF_CK(use_dev(r->device));
        if (!r->afg) RF_CK(dalloc(&r->afg, (size_t)r->views * r->n));
        if (!r->abg) RF_CK(dalloc(&r->abg, (size_t)r->views * r->n));
        if (masks) r->masks.assign(masks, masks + r->views);
        else r->masks.clear();
        r->adjoint = true;
        const int rc = run_round(r, s, beta, cams, mode, reinterpret_cast<cudaStream_t>(stream));
        if (rc != SF_OK) return rc;
        if (beta) std::memcpy(eig, r->eig_host, 8 * r->views);
        return SF_OK;
    } catch (const std::bad_alloc&) {
        return rfail(SF_ERR_NOMEM, "host allocation failed");
    }
}

int sf_round_adjoint_responsibility(sf_round r, uint32_t view, const float** fg, const float** bg) {
    if (!r) return rfail(SF_ERR_ARG, "null round");
    if (view >= r->views) return rfail(SF_ERR_SHAPE, "no such view");
    if (!r->adjoint || !r->afg) return rfail(SF_ERR_ARG, "the last round was not an adjoint round");
    if (fg) *fg = r->afg + (size_t)view * r->n;
    if (bg) *bg = r->abg + (size_t)view * r->n;
    return SF_OK;
}

}  // extern "C"

namespace {

// One round of the given kind (0 responsibility, 1 u32 evidence, 2 adjoint).
int round_of_kind(sf_round r, sf_splats s, sf_beta beta, const sf_camera* cams, const sf_mask* masks, int kind,
                  int mode, sf_stream stream, double* eig) {
    if (kind == SF_ROUND_EVIDENCE) return sf_round_evidence(r, s, beta, cams, masks, mode, stream, eig);
    if (kind == SF_ROUND_ADJOINT) return sf_round_evidence_adjoint(r, s, beta, cams, masks, mode, stream, eig);
    return sf_round_eig(r, s, beta, cams, mode, stream, eig);
}

// Coordinate search over the round's kernel forms: each dimension in turn
// (lanes, intersection build, list order, raster culling, CTAs per tile),
// each value timed as the best of three rounds after one warm-up round
// (which also captures the graph), the best kept; two sweeps.
int autotune(sf_round r, sf_splats s, sf_beta beta, const sf_camera* cams, const sf_mask* masks, int kind,
             int mode, sf_stream stream, sf_round_tuning* best, double* best_ms) {
    if (!r || !s || !cams) return rfail(SF_ERR_ARG, "null argument");
    if (kind == SF_ROUND_EVIDENCE && !masks) return rfail(SF_ERR_ARG, "an evidence round needs masks");
    RF_CK(use_dev(r->device));
    const std::string key = tune_key(r) + "|kind" + std::to_string(kind);
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            r->tuning = it->second.tuning;
            if (best) *best = it->second.tuning;
            if (best_ms) *best_ms = it->second.ms;
            return SF_OK;
        }
    }
    cudaEvent_t e0, e1;
    RF_CK(cudaEventCreate(&e0));
    RF_CK(cudaEventCreate(&e1));
    std::vector<double> eig(r->views);
    auto time_of = [&](const sf_round_tuning& t, float* out_ms) -> int {
        r->tuning = t;
        int rc = round_of_kind(r, s, beta, cams, masks, kind, mode, stream, eig.data());
        if (rc != SF_OK) return rc;
        float ms_best = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {
            RF_CK(cudaEventRecord(e0, r->main));
            rc = round_of_kind(r, s, beta, cams, masks, kind, mode, stream, eig.data());
            if (rc != SF_OK) return rc;
            RF_CK(cudaEventRecord(e1, r->main));
            RF_CK(cudaEventSynchronize(e1));
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            ms_best = std::min(ms_best, ms);
        }
        *out_ms = ms_best;
        return SF_OK;
    };
    sf_round_tuning winner = r->tuning;
    if (winner.lanes == 0) winner.lanes = 4;
    if (winner.raster_split == 0) winner.raster_split = 1;
    if (kind == SF_ROUND_ADJOINT) winner.raster_order = SF_ORDER_SORTED;
    float winner_ms = 1e30f;
    int rc = time_of(winner, &winner_ms);
    if (rc != SF_OK) return rc;
    if (winner.radix_bits == 0) winner.radix_bits = 8;
    const std::vector<uint32_t> lanes_v = {1, 2, 4, 8}, build_v = {SF_ISECTS_BINNED, SF_ISECTS_DEPTH_SORTED},
                                order_v = {SF_ORDER_SORTED, SF_ORDER_IN_RASTER, SF_ORDER_HYBRID}, cull_v = {0, 1},
                                split_v = {1, 2, 4}, radix_v = {4, 6, 8};
    for (int sweep = 0; sweep < 2; ++sweep) {
        for (int dim = 0; dim < 6; ++dim) {
            const std::vector<uint32_t>& vals = dim == 0 ? lanes_v : dim == 1 ? build_v : dim == 2 ? order_v
                                              : dim == 3 ? cull_v : dim == 4 ? split_v : radix_v;
            for (uint32_t val : vals) {
                sf_round_tuning t = winner;
                uint32_t* field = dim == 0 ? &t.lanes : dim == 1 ? &t.isect_build : dim == 2 ? &t.raster_order
                                : dim == 3 ? &t.raster_cull : dim == 4 ? &t.raster_split : &t.radix_bits;
                if (*field == val) continue;
                *field = val;
                if (dim == 0 && val > r->views) continue;
                // The orders apply to the binned build; the adjoint replays
                // sorted lists, and its transmittance pass runs one CTA per tile.
                if (dim == 2 && (t.isect_build != SF_ISECTS_BINNED || kind == SF_ROUND_ADJOINT)) continue;
                if (dim == 4 && kind == SF_ROUND_ADJOINT) continue;
                // The digit width applies to the depth-sorted build's sorts.
                if (dim == 5 && t.isect_build != SF_ISECTS_DEPTH_SORTED) continue;
                if (dim == 1 && val == SF_ISECTS_DEPTH_SORTED) t.raster_order = SF_ORDER_SORTED;
                float ms = 0.f;
                rc = time_of(t, &ms);
                if (rc != SF_OK) return rc;
                if (ms < winner_ms) {
                    winner_ms = ms;
                    winner = t;
                }
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    r->tuning = winner;
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        g_tune_cache[key] = TuneEntry{winner, winner_ms};
    }
    if (best) *best = winner;
    if (best_ms) *best_ms = winner_ms;
    return SF_OK;
}

}  // namespace

extern "C" {

int sf_round_autotune(sf_round r, sf_splats s, sf_beta beta, const sf_camera* cams, int mode,
                      sf_stream stream, sf_round_tuning* best, double* best_ms) {
    try {
        return autotune(r, s, beta, cams, nullptr, SF_ROUND_RESPONSIBILITY, mode, stream, best, best_ms);
    } catch (const std::bad_alloc&) {
        return rfail(SF_ERR_NOMEM, "host allocation failed");
    }
}

int sf_round_autotune_kind(sf_round r, sf_splats s, sf_beta beta, const sf_camera* cams, const sf_mask* masks,
                           int kind, int mode, sf_stream stream, sf_round_tuning* best, double* best_ms) {
    try {
        if (kind != SF_ROUND_RESPONSIBILITY && kind != SF_ROUND_EVIDENCE && kind != SF_ROUND_ADJOINT)
            return rfail(SF_ERR_ARG, "unknown round kind");
        return autotune(r, s, beta, cams, masks, kind, mode, stream, best, best_ms);
    } catch (const std::bad_alloc&) {
        return rfail(SF_ERR_NOMEM, "host allocation failed");
    }
}

}  // extern "C"
