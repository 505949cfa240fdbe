// Handle types shared by the C ABI translation units (sf_api.cu, sf_round.cu).
#pragma once
#include <cstdint>
#include <string>
#include "sf_internal.h"

struct sf_ctx_t {
    int device = 0;
    int sm_count = 148;
    float* lut = nullptr;  // f32 entropy LUT, built on first use
};

struct sf_splats_t {
    sf_ctx ctx = nullptr;
    uint32_t n = 0, K = 1;
    float* attr = nullptr;
    float* sh = nullptr;
    float* geom = nullptr;  // [kGeomPlanes][n] camera-independent projection terms of attr
    float bounds[6] = {0, 0, 0, 0, 0, 0};
};

struct sf_accum_t {
    sf_ctx ctx = nullptr;
    uint32_t total = 0;
    uint32_t *resp = nullptr, *fg = nullptr, *bg = nullptr;
    float scale = 1.0f;
    bool evidence = false;  // the last fill was a masked split (fg, bg), not resp
};

struct sf_mask_t {
    uint32_t w = 0, h = 0, wpr = 0;
    uint32_t* bits = nullptr;
};

struct sf_beta_t {
    sf_ctx ctx = nullptr;
    uint32_t n = 0;
    float *a = nullptr, *b = nullptr;
    double* partials = nullptr;
    uint32_t blocks = 1;
    double* out = nullptr;
    double* host_out = nullptr;
    // Localization scratch (allocated on first use): [blocks][4] partials,
    // [8] results, pinned mirror of the results.
    double* loc_partials = nullptr;
    double* loc_out = nullptr;
    double* loc_host = nullptr;
};

namespace sfk {
// Records the calling thread's last error message (sf_last_error) and
// returns `code`.
int set_error(int code, const std::string& msg);
}  // namespace sfk
