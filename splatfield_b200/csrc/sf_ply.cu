// 3DGS binary PLY scenes (parse_ply / CpuSplats::write_ply, src/ply.rs:9-180).
//
// Loading: the ASCII header is parsed on the host with the reference's rules
// (binary_little_endian only, float properties only, the 14 required
// properties reported first-missing-first in the reference's order, f_rest_*
// sorted by their number). The vertex block — n rows of `stride` floats,
// row-major as stored — is copied to the device once, and one kernel writes
// the field-major attribute and SH planes the renderer reads, normalising each
// rotation (w = rot_0) in glam's Quat::normalize operation order and reducing
// the scene bounds. No host transpose of the (often hundreds of MB) vertex
// block.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cctype>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>
#include "sf_handles.h"

namespace sfk {
namespace {

constexpr int kBaseProps = 14;
// Attribute plane of each required property (x y z scale_0..2 opacity
// rot_0..3 f_dc_0..2 in the reference's lookup order, src/ply.rs:46-53).
const char* const kRequired[kBaseProps] = {"x",       "y",       "z",     "scale_0", "scale_1",
                                           "scale_2", "opacity", "rot_0", "rot_1",   "rot_2",
                                           "rot_3",   "f_dc_0",  "f_dc_1", "f_dc_2"};
constexpr int kMaxRest = 45;

struct PlyLayout {
    uint32_t stride;        // floats per row
    uint32_t k;             // SH coefficients per channel
    int base[kBaseProps];   // column of each required property
    int rest[kMaxRest];     // columns of f_rest_* sorted by number
};

struct Header {
    PlyLayout lay{};
    uint64_t n = 0;
    size_t data_off = 0;
};

// Whitespace tokens of one header line.
std::vector<std::string> tokens(const std::string& line) {
    std::vector<std::string> t;
    size_t i = 0;
    while (i < line.size()) {
        while (i < line.size() && std::isspace((unsigned char)line[i])) ++i;
        size_t j = i;
        while (j < line.size() && !std::isspace((unsigned char)line[j])) ++j;
        if (j > i) t.emplace_back(line.substr(i, j - i));
        i = j;
    }
    return t;
}

bool parse_usize(const std::string& s, uint64_t* out) {
    if (s.empty() || s.size() > 20) return false;
    uint64_t v = 0;
    for (char c : s) {
        if (c < '0' || c > '9') return false;
        const uint64_t d = (uint64_t)(c - '0');
        if (v > (UINT64_MAX - d) / 10) return false;
        v = v * 10 + d;
    }
    *out = v;
    return true;
}

int header_fail(const std::string& msg) { return set_error(SF_ERR_ARG, msg); }

// parse_ply's header pass (src/ply.rs:9-77).
int parse_header(const uint8_t* bytes, size_t len, Header* h) {
    std::vector<std::string> props;
    size_t pos = 0;
    bool ended = false;
    while (pos < len) {
        size_t e = pos;
        while (e < len && bytes[e] != '\n') ++e;
        std::string line(reinterpret_cast<const char*>(bytes + pos), e - pos);
        if (!line.empty() && line.back() == '\r') line.pop_back();
        pos = e < len ? e + 1 : e;
        const auto t = tokens(line);
        if (!t.empty() && t[0] == "end_header") {
            ended = true;
            break;
        }
        if (t.size() >= 2 && t[0] == "format" && t[1] != "binary_little_endian")
            return header_fail("Unsupported PLY format: " + t[1]);
        if (t.size() == 3 && t[0] == "element" && t[1] == "vertex") {
            if (!parse_usize(t[2], &h->n)) return header_fail("Invalid vertex count");
        }
        if (t.size() == 3 && t[0] == "property") {
            if (t[1] != "float") return header_fail("Unsupported property type " + t[1] + ": " + t[2]);
            props.push_back(t[2]);
        }
    }
    (void)ended;
    if (h->n == 0) return header_fail("PLY contains no vertices");
    for (int k = 0; k < kBaseProps; ++k) {
        const auto it = std::find(props.begin(), props.end(), kRequired[k]);
        if (it == props.end()) return header_fail(std::string("Missing property: ") + kRequired[k]);
        h->lay.base[k] = (int)(it - props.begin());
    }
    std::vector<std::pair<uint64_t, int>> rest;
    for (size_t i = 0; i < props.size(); ++i) {
        const std::string& p = props[i];
        uint64_t num;
        if (p.rfind("f_rest_", 0) == 0 && parse_usize(p.substr(7), &num)) rest.emplace_back(num, (int)i);
    }
    std::stable_sort(rest.begin(), rest.end(),
                     [](const std::pair<uint64_t, int>& a, const std::pair<uint64_t, int>& b) {
                         return a.first < b.first;
                     });
    // n = rest / 3 coefficients per channel past the DC (src/ply.rs:66); a
    // remainder is dropped as the reference's planes leave it unfilled.
    const size_t nr = rest.size() / 3 * 3;
    if (nr > kMaxRest) return header_fail("more than 45 f_rest_* properties (SH degree above 3)");
    for (size_t j = 0; j < nr; ++j) h->lay.rest[j] = rest[j].second;
    h->lay.stride = (uint32_t)props.size();
    h->lay.k = (uint32_t)(nr / 3 + 1);
    if (h->n > (uint64_t)UINT32_MAX || h->n > UINT64_MAX / ((uint64_t)props.size() * 4))
        return header_fail("PLY vertex count overflows address space");
    h->data_off = pos;
    const uint64_t need = h->n * props.size() * 4;
    if (len - pos < need) {
        const uint64_t rows = (len - pos) / ((uint64_t)props.size() * 4);
        return header_fail("failed to read vertex " + std::to_string(rows) + " of " + std::to_string(h->n));
    }
    return SF_OK;
}

__device__ __forceinline__ uint32_t ordered(float v) {
    const uint32_t b = __float_as_uint(v);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// Rows -> planes. attr planes: x y z qw qx qy qz sx sy sz opacity; sh planes:
// dc r g b, then coefficient j channel c at plane (j + 1) * 3 + c with
// f_rest_(c * (k - 1) + j) (channel-major rest order, src/ply.rs:94-99).
// bounds_u: [6] ordered-uint min xyz / max xyz (NaN positions skipped).
__global__ void ply_planes_kernel(const float* __restrict__ rows, uint32_t n, PlyLayout lay,
                                  float* __restrict__ attr, float* __restrict__ sh, uint32_t* bounds_u) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float p[3] = {0.0f, 0.0f, 0.0f};
    bool valid = i < n;
    if (valid) {
        const float* r = rows + (size_t)i * lay.stride;
        const size_t N = n;
        p[0] = r[lay.base[0]];
        p[1] = r[lay.base[1]];
        p[2] = r[lay.base[2]];
        // glam Quat::from_xyzw(rot_1, rot_2, rot_3, rot_0).normalize(): the
        // SSE2 dot order (x2 + z2) + (y2 + w2), one reciprocal of the root.
        float qx = r[lay.base[8]], qy = r[lay.base[9]], qz = r[lay.base[10]], qw = r[lay.base[7]];
        const float d = (qx * qx + qz * qz) + (qy * qy + qw * qw);
        const float inv = 1.0f / sqrtf(d);
        qx = qx * inv;
        qy = qy * inv;
        qz = qz * inv;
        qw = qw * inv;
        attr[0 * N + i] = p[0];
        attr[1 * N + i] = p[1];
        attr[2 * N + i] = p[2];
        attr[3 * N + i] = qw;
        attr[4 * N + i] = qx;
        attr[5 * N + i] = qy;
        attr[6 * N + i] = qz;
        attr[7 * N + i] = r[lay.base[3]];
        attr[8 * N + i] = r[lay.base[4]];
        attr[9 * N + i] = r[lay.base[5]];
        attr[10 * N + i] = r[lay.base[6]];
        sh[0 * N + i] = r[lay.base[11]];
        sh[1 * N + i] = r[lay.base[12]];
        sh[2 * N + i] = r[lay.base[13]];
        const uint32_t m = lay.k - 1;
        for (uint32_t j = 0; j < m; ++j)
            for (uint32_t c = 0; c < 3; ++c) sh[((j + 1) * 3 + c) * N + i] = r[lay.rest[c * m + j]];
    }
    // Bounds: warp min / max, one atomic per warp and axis.
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const bool ok = valid && p[k] == p[k];
        uint32_t lo = ok ? ordered(p[k]) : 0xffffffffu;
        uint32_t hi = ok ? ordered(p[k]) : 0u;
        lo = __reduce_min_sync(0xffffffffu, lo);
        hi = __reduce_max_sync(0xffffffffu, hi);
        if ((threadIdx.x & 31u) == 0) {
            if (lo != 0xffffffffu) atomicMin(bounds_u + k, lo);
            if (hi != 0u) atomicMax(bounds_u + 3 + k, hi);
        }
    }
}

}  // namespace
}  // namespace sfk

using namespace sfk;

extern "C" {

int sf_ply_inspect(const void* bytes, size_t len, uint32_t* n, uint32_t* sh_per_ch) {
    try {
        if (!bytes && len) return set_error(SF_ERR_ARG, "null bytes");
        Header h;
        const int rc = parse_header(static_cast<const uint8_t*>(bytes), len, &h);
        if (rc != SF_OK) return rc;
        if (n) *n = (uint32_t)h.n;
        if (sh_per_ch) *sh_per_ch = h.lay.k;
        return SF_OK;
    } catch (const std::bad_alloc&) {
        return set_error(SF_ERR_NOMEM, "host allocation failed");
    }
}

int sf_ply_load(sf_ctx ctx, const void* bytes, size_t len, sf_splats* out) {
    try {
        if (!ctx || !out || (!bytes && len)) return set_error(SF_ERR_ARG, "null argument");
        *out = nullptr;
        Header h;
        int rc = parse_header(static_cast<const uint8_t*>(bytes), len, &h);
        if (rc != SF_OK) return rc;
        int cur = -1;
        cudaError_t e = cudaGetDevice(&cur);
        if (e == cudaSuccess && cur != ctx->device) e = cudaSetDevice(ctx->device);
        const uint32_t n = (uint32_t)h.n;
        const size_t row_bytes = (size_t)n * h.lay.stride * 4;
        float* rows = nullptr;
        uint32_t* bounds_u = nullptr;
        auto* s = new sf_splats_t();
        s->ctx = ctx;
        s->n = n;
        s->K = h.lay.k;
        if (e == cudaSuccess) e = cudaMalloc(&rows, row_bytes);
        if (e == cudaSuccess) e = cudaMalloc(&s->attr, (size_t)11 * n * 4);
        if (e == cudaSuccess) e = cudaMalloc(&s->sh, (size_t)3 * h.lay.k * n * 4);
        if (e == cudaSuccess) e = cudaMalloc(&s->geom, (size_t)kGeomPlanes * n * 4);
        if (e == cudaSuccess) e = cudaMalloc(&bounds_u, 6 * 4);
        if (e == cudaSuccess)
            e = cudaMemcpy(rows, static_cast<const uint8_t*>(bytes) + h.data_off, row_bytes, cudaMemcpyHostToDevice);
        const uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
        if (e == cudaSuccess) e = cudaMemcpy(bounds_u, init, sizeof(init), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) {
            ply_planes_kernel<<<(n + 255) / 256, 256>>>(rows, n, h.lay, s->attr, s->sh, bounds_u);
            note_launches(1);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = launch_splat_geom(s->attr, n, s->geom, nullptr);
        uint32_t bu[6] = {0, 0, 0, 0, 0, 0};
        if (e == cudaSuccess) e = cudaMemcpy(bu, bounds_u, sizeof(bu), cudaMemcpyDeviceToHost);
        if (rows) cudaFree(rows);
        if (bounds_u) cudaFree(bounds_u);
        if (e != cudaSuccess) {
            if (s->attr) cudaFree(s->attr);
            if (s->sh) cudaFree(s->sh);
            if (s->geom) cudaFree(s->geom);
            delete s;
            return set_error(e == cudaErrorMemoryAllocation ? SF_ERR_NOMEM : SF_ERR_CUDA, cudaGetErrorString(e));
        }
        for (int k = 0; k < 3; ++k) {
            // All positions NaN: the host path's +/-FLT_MAX start values.
            const uint32_t lo = bu[k], hi = bu[3 + k];
            auto unord = [](uint32_t u) {
                const uint32_t b = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
                float f;
                std::memcpy(&f, &b, 4);
                return f;
            };
            s->bounds[k] = lo == 0xffffffffu ? 3.4028235e38f : unord(lo);
            s->bounds[3 + k] = hi == 0u ? -3.4028235e38f : unord(hi);
        }
        *out = s;
        return SF_OK;
    } catch (const std::bad_alloc&) {
        return set_error(SF_ERR_NOMEM, "host allocation failed");
    }
}

int sf_ply_load_file(sf_ctx ctx, const char* path, sf_splats* out) {
    try {
        if (!path) return set_error(SF_ERR_ARG, "null path");
        std::ifstream f(path, std::ios::binary | std::ios::ate);
        if (!f) return set_error(SF_ERR_ARG, std::string("cannot open ") + path);
        const std::streamsize size = f.tellg();
        f.seekg(0);
        std::vector<uint8_t> bytes((size_t)std::max<std::streamsize>(size, 0));
        if (size > 0 && !f.read(reinterpret_cast<char*>(bytes.data()), size))
            return set_error(SF_ERR_ARG, std::string("cannot read ") + path);
        return sf_ply_load(ctx, bytes.data(), bytes.size(), out);
    } catch (const std::bad_alloc&) {
        return set_error(SF_ERR_NOMEM, "host allocation failed");
    }
}

int sf_ply_write(const float* attr, const float* sh, uint32_t n, uint32_t sh_per_ch, void* out, size_t cap,
                 size_t* len) {
    try {
        if (!attr || !sh || !len) return set_error(SF_ERR_ARG, "null argument");
        if (n == 0) return set_error(SF_ERR_SHAPE, "no splats to write");
        if (sh_per_ch == 0) return set_error(SF_ERR_SHAPE, "sh_per_ch must be positive");
        const uint32_t rest = (sh_per_ch - 1) * 3;
        std::string header = "ply\nformat binary_little_endian 1.0\nelement vertex " + std::to_string(n) + "\n";
        const char* head[] = {"x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"};
        for (const char* p : head) header += std::string("property float ") + p + "\n";
        for (uint32_t j = 0; j < rest; ++j) header += "property float f_rest_" + std::to_string(j) + "\n";
        const char* tail[] = {"opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"};
        for (const char* p : tail) header += std::string("property float ") + p + "\n";
        header += "end_header\n";
        const size_t floats = 17 + rest;
        const size_t total = header.size() + (size_t)n * floats * 4;
        *len = total;
        if (!out) return SF_OK;
        if (cap < total) return set_error(SF_ERR_SHAPE, "output buffer too small");
        uint8_t* o = static_cast<uint8_t*>(out);
        std::memcpy(o, header.data(), header.size());
        o += header.size();
        std::vector<float> row(floats);
        const size_t N = n;
        for (size_t i = 0; i < N; ++i) {
            auto a = [&](int plane) { return attr[plane * N + i]; };
            row[0] = a(0);
            row[1] = a(1);
            row[2] = a(2);
            row[3] = row[4] = row[5] = 0.0f;
            row[6] = sh[i];
            row[7] = sh[N + i];
            row[8] = sh[2 * N + i];
            const uint32_t per = rest / 3;
            for (uint32_t j = 0; j < rest; ++j) {
                const uint32_t c = j / per, coef = j % per;
                row[9 + j] = sh[((coef + 1) * 3 + c) * N + i];
            }
            row[9 + rest] = a(10);
            row[10 + rest] = a(7);
            row[11 + rest] = a(8);
            row[12 + rest] = a(9);
            row[13 + rest] = a(3);
            row[14 + rest] = a(4);
            row[15 + rest] = a(5);
            row[16 + rest] = a(6);
            std::memcpy(o, row.data(), floats * 4);
            o += floats * 4;
        }
        return SF_OK;
    } catch (const std::bad_alloc&) {
        return set_error(SF_ERR_NOMEM, "host allocation failed");
    }
}

}  // extern "C"
