// SOG scenes (parse_sog, src/sog.rs:97-198): a zip archive holding
// meta.json and lossless WebP planes, one pixel per splat.
//
// Host: the zip central directory is read (stored and deflate entries; raw
// deflate through zlib), meta.json is parsed with a small JSON reader, and
// each plane is decoded by the WebP decoder of sf_webp.cpp. The checks and
// their messages are the reference's (missing entries, plane sizes below the
// splat count, codebooks of 256 floats, rotation tags 252-255, shN bands
// 1..3, shN labels inside the palette). Device: the decoded RGBA planes go
// up as bytes (24 B per splat, a tenth of the float planes they become) and
// one kernel dequantises them into the field-major attribute and SH planes:
//  * means: t = (lo | hi << 8) / 65535 per axis, v = min + span * t, then
//    inv_log(v) = sign(v) * expm1(|v|) (sog.rs:114-130, 68-70);
//  * log-scales and SH DC from their 256-entry codebooks (:132-138, :161-167);
//  * rotations: three components in [-1/sqrt 2, 1/sqrt 2] and the omitted
//    one from the unit norm, placed by the tag (:80-93, :140-149);
//  * opacity = logit(alpha / 255) clamped to [1e-6, 1 - 1e-6] (:73-76);
//  * higher SH from the centroid palette addressed by each splat's 16-bit
//    label (:169-193, palette_offset :202-205).
#include <cuda_runtime.h>
#include <zlib.h>
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <string>
#include <vector>
#include "sf_handles.h"

namespace sfk {
namespace webp {
int decode(const uint8_t* p, size_t n, uint32_t* w, uint32_t* h, std::vector<uint32_t>* argb, std::string* err);
}

namespace {

struct SogFail {
    std::string msg;
};

// ---------------------------------------------------------------- zip

uint32_t rd16(const uint8_t* p) { return (uint32_t)p[0] | (uint32_t)p[1] << 8; }
uint32_t rd32(const uint8_t* p) { return rd16(p) | rd16(p + 2) << 16; }

struct ZipEntry {
    uint32_t method = 0, csize = 0, usize = 0, local = 0;
};

std::map<std::string, ZipEntry> zip_directory(const uint8_t* p, size_t n) {
    // End of central directory: the last signature within the final 64 KiB.
    if (n < 22) throw SogFail{"not a SOG archive"};
    size_t eocd = n;
    for (size_t i = n - 22 + 1; i-- > 0 && n - i <= 22 + 65535;) {
        if (rd32(p + i) == 0x06054b50u) {
            eocd = i;
            break;
        }
    }
    if (eocd == n) throw SogFail{"not a SOG archive"};
    const uint32_t count = rd16(p + eocd + 10);
    const uint32_t cd_off = rd32(p + eocd + 16);
    std::map<std::string, ZipEntry> dir;
    size_t off = cd_off;
    for (uint32_t k = 0; k < count; ++k) {
        if (off + 46 > n || rd32(p + off) != 0x02014b50u) throw SogFail{"not a SOG archive"};
        ZipEntry e;
        e.method = rd16(p + off + 10);
        e.csize = rd32(p + off + 20);
        e.usize = rd32(p + off + 24);
        const uint32_t name_len = rd16(p + off + 28), extra = rd16(p + off + 30), comment = rd16(p + off + 32);
        e.local = rd32(p + off + 42);
        if (off + 46 + name_len > n) throw SogFail{"not a SOG archive"};
        dir[std::string(reinterpret_cast<const char*>(p + off + 46), name_len)] = e;
        off += 46 + (size_t)name_len + extra + comment;
    }
    return dir;
}

std::vector<uint8_t> zip_read(const uint8_t* p, size_t n, const std::map<std::string, ZipEntry>& dir,
                              const std::string& name) {
    auto it = dir.find(name);
    if (it == dir.end()) throw SogFail{"missing " + name};
    const ZipEntry& e = it->second;
    if ((size_t)e.local + 30 > n || rd32(p + e.local) != 0x04034b50u) throw SogFail{"missing " + name};
    const size_t data = (size_t)e.local + 30 + rd16(p + e.local + 26) + rd16(p + e.local + 28);
    if (data + e.csize > n) throw SogFail{"missing " + name};
    std::vector<uint8_t> out(e.usize);
    if (e.method == 0) {
        if (e.csize != e.usize) throw SogFail{"missing " + name};
        std::memcpy(out.data(), p + data, e.usize);
    } else if (e.method == 8) {
        z_stream zs{};
        if (inflateInit2(&zs, -MAX_WBITS) != Z_OK) throw SogFail{"inflate " + name};
        zs.next_in = const_cast<Bytef*>(p + data);
        zs.avail_in = e.csize;
        zs.next_out = out.data();
        zs.avail_out = e.usize;
        const int rc = inflate(&zs, Z_FINISH);
        const bool ok = rc == Z_STREAM_END && zs.total_out == e.usize;
        inflateEnd(&zs);
        if (!ok) throw SogFail{"inflate " + name};
    } else {
        throw SogFail{name + ": unsupported zip compression method " + std::to_string(e.method)};
    }
    return out;
}

// ---------------------------------------------------------------- JSON

struct Json {
    enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
    double num = 0.0;
    bool b = false;
    std::string str;
    std::vector<Json> arr;
    std::vector<std::pair<std::string, Json>> obj;
    const Json* get(const std::string& k) const {
        for (const auto& kv : obj)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
};

class JsonReader {
   public:
    JsonReader(const std::vector<uint8_t>& s) : s_(s) {}
    Json parse() {
        Json v = value();
        ws();
        if (i_ != s_.size()) bad();
        return v;
    }

   private:
    [[noreturn]] void bad() { throw SogFail{"invalid meta.json"}; }
    void ws() {
        while (i_ < s_.size() && (s_[i_] == ' ' || s_[i_] == '\n' || s_[i_] == '\r' || s_[i_] == '\t')) ++i_;
    }
    bool lit(const char* t) {
        const size_t k = std::strlen(t);
        if (i_ + k <= s_.size() && std::memcmp(s_.data() + i_, t, k) == 0) {
            i_ += k;
            return true;
        }
        return false;
    }
    std::string string() {
        if (i_ >= s_.size() || s_[i_] != '"') bad();
        ++i_;
        std::string out;
        while (i_ < s_.size() && s_[i_] != '"') {
            char c = (char)s_[i_++];
            if (c == '\\') {
                if (i_ >= s_.size()) bad();
                const char e = (char)s_[i_++];
                switch (e) {
                    case '"': case '\\': case '/': out += e; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'n': out += '\n'; break;
                    case 'r': out += '\r'; break;
                    case 't': out += '\t'; break;
                    case 'u': {
                        if (i_ + 4 > s_.size()) bad();
                        const uint32_t cp = (uint32_t)std::stoul(std::string(s_.begin() + i_, s_.begin() + i_ + 4), nullptr, 16);
                        i_ += 4;
                        if (cp < 0x80) out += (char)cp;
                        else if (cp < 0x800) { out += (char)(0xc0 | (cp >> 6)); out += (char)(0x80 | (cp & 0x3f)); }
                        else { out += (char)(0xe0 | (cp >> 12)); out += (char)(0x80 | ((cp >> 6) & 0x3f)); out += (char)(0x80 | (cp & 0x3f)); }
                        break;
                    }
                    default: bad();
                }
            } else {
                out += c;
            }
        }
        if (i_ >= s_.size()) bad();
        ++i_;
        return out;
    }
    Json value() {
        ws();
        if (i_ >= s_.size()) bad();
        Json v;
        const char c = (char)s_[i_];
        if (c == '{') {
            ++i_;
            v.kind = Json::Obj;
            ws();
            if (i_ < s_.size() && s_[i_] == '}') { ++i_; return v; }
            for (;;) {
                ws();
                std::string k = string();
                ws();
                if (i_ >= s_.size() || s_[i_] != ':') bad();
                ++i_;
                v.obj.emplace_back(std::move(k), value());
                ws();
                if (i_ < s_.size() && s_[i_] == ',') { ++i_; continue; }
                if (i_ < s_.size() && s_[i_] == '}') { ++i_; return v; }
                bad();
            }
        }
        if (c == '[') {
            ++i_;
            v.kind = Json::Arr;
            ws();
            if (i_ < s_.size() && s_[i_] == ']') { ++i_; return v; }
            for (;;) {
                v.arr.push_back(value());
                ws();
                if (i_ < s_.size() && s_[i_] == ',') { ++i_; continue; }
                if (i_ < s_.size() && s_[i_] == ']') { ++i_; return v; }
                bad();
            }
        }
        if (c == '"') {
            v.kind = Json::Str;
            v.str = string();
            return v;
        }
        if (lit("true")) { v.kind = Json::Bool; v.b = true; return v; }
        if (lit("false")) { v.kind = Json::Bool; return v; }
        if (lit("null")) return v;
        const size_t start = i_;
        while (i_ < s_.size() && (std::isdigit(s_[i_]) || s_[i_] == '-' || s_[i_] == '+' || s_[i_] == '.' ||
                                  s_[i_] == 'e' || s_[i_] == 'E'))
            ++i_;
        if (i_ == start) bad();
        const std::string num(s_.begin() + start, s_.begin() + i_);
        char* end = nullptr;
        v.num = std::strtod(num.c_str(), &end);
        if (!end || *end) bad();
        v.kind = Json::Num;
        return v;
    }
    const std::vector<uint8_t>& s_;
    size_t i_ = 0;
};

// serde's view of the reference's Meta (sog.rs:8-42): required fields,
// fixed-length file lists where the reference has arrays.
const Json& field(const Json& o, const char* k) {
    if (o.kind != Json::Obj) throw SogFail{"invalid meta.json"};
    const Json* v = o.get(k);
    if (!v) throw SogFail{"invalid meta.json"};
    return *v;
}
double number(const Json& v) {
    if (v.kind != Json::Num) throw SogFail{"invalid meta.json"};
    return v.num;
}
std::vector<float> floats(const Json& v) {
    if (v.kind != Json::Arr) throw SogFail{"invalid meta.json"};
    std::vector<float> out;
    for (const auto& x : v.arr) out.push_back((float)number(x));
    return out;
}
std::vector<std::string> files(const Json& v, size_t exact) {
    if (v.kind != Json::Arr || (exact && v.arr.size() != exact)) throw SogFail{"invalid meta.json"};
    std::vector<std::string> out;
    for (const auto& x : v.arr) {
        if (x.kind != Json::Str) throw SogFail{"invalid meta.json"};
        out.push_back(x.str);
    }
    return out;
}
uint64_t count_of(const Json& v) {
    const double d = number(v);
    if (!(d >= 0.0) || d != std::floor(d) || d > 4294967295.0) throw SogFail{"invalid meta.json"};
    return (uint64_t)d;
}

struct Meta {
    uint64_t count = 0;
    float mins[3], maxs[3];
    std::string means[2], scales, quats, sh0;
    std::vector<float> scales_cb, sh0_cb, shn_cb;
    bool has_shn = false;
    uint64_t bands = 0;
    std::string shn[2];
};

Meta parse_meta(const std::vector<uint8_t>& text) {
    const Json root = JsonReader(text).parse();
    Meta m;
    m.count = count_of(field(root, "count"));
    const Json& means = field(root, "means");
    const auto mins = floats(field(means, "mins")), maxs = floats(field(means, "maxs"));
    if (mins.size() != 3 || maxs.size() != 3) throw SogFail{"invalid meta.json"};
    for (int k = 0; k < 3; ++k) {
        m.mins[k] = mins[k];
        m.maxs[k] = maxs[k];
    }
    const auto mf = files(field(means, "files"), 2);
    m.means[0] = mf[0];
    m.means[1] = mf[1];
    const Json& scales = field(root, "scales");
    m.scales_cb = floats(field(scales, "codebook"));
    const auto sf = files(field(scales, "files"), 0);
    if (sf.empty()) throw SogFail{"invalid meta.json"};
    m.scales = sf[0];
    m.quats = files(field(field(root, "quats"), "files"), 1)[0];
    const Json& sh0 = field(root, "sh0");
    m.sh0_cb = floats(field(sh0, "codebook"));
    const auto s0 = files(field(sh0, "files"), 0);
    if (s0.empty()) throw SogFail{"invalid meta.json"};
    m.sh0 = s0[0];
    const Json* shn = root.get("shN");
    if (shn && shn->kind != Json::Null) {
        m.has_shn = true;
        m.bands = count_of(field(*shn, "bands"));
        m.shn_cb = floats(field(*shn, "codebook"));
        const auto f = files(field(*shn, "files"), 2);
        m.shn[0] = f[0];
        m.shn[1] = f[1];
    }
    return m;
}

struct Plane {
    uint32_t w = 0, h = 0;
    std::vector<uint32_t> rgba;  // bytes r, g, b, a per pixel (little-endian word)
};

// decode_rgba (sog.rs:44-66).
Plane decode_rgba(const uint8_t* p, size_t n, const std::map<std::string, ZipEntry>& dir, const std::string& name,
                  uint64_t min_pixels) {
    const std::vector<uint8_t> bytes = zip_read(p, n, dir, name);
    Plane pl;
    std::vector<uint32_t> argb;
    std::string err;
    if (webp::decode(bytes.data(), bytes.size(), &pl.w, &pl.h, &argb, &err) != SF_OK)
        throw SogFail{"decode " + name + ": " + err};
    if ((uint64_t)pl.w * pl.h < min_pixels)
        throw SogFail{name + ": " + std::to_string(pl.w) + "x" + std::to_string(pl.h) + " < " +
                      std::to_string(min_pixels) + " pixels"};
    pl.rgba.resize(argb.size());
    for (size_t i = 0; i < argb.size(); ++i) {
        const uint32_t v = argb[i];
        pl.rgba[i] = ((v >> 16) & 0xffu) | (v & 0xff00u) << 0 | ((v & 0xffu) << 16) | (v & 0xff000000u);
    }
    return pl;
}

void codebook_check(const std::vector<float>& cb, const char* what) {
    if (cb.size() != 256)
        throw SogFail{std::string(what) + " codebook: 256 floats expected, got " + std::to_string(cb.size())};
}

uint32_t sh_per_ch_of(const Meta& m) {
    if (!m.has_shn) return 1;
    if (m.bands == 1) return 4;
    if (m.bands == 2) return 9;
    if (m.bands == 3) return 16;
    throw SogFail{"shN.bands " + std::to_string(m.bands) + " outside 1..=3"};
}

struct SogArgs {
    uint32_t n, k;
    float mins[3], spans[3];
    const uint32_t *lo, *hi, *scales, *quats, *sh0, *labels, *centroids;
    const float *scales_cb, *sh0_cb, *shn_cb;
    uint32_t cw;  // centroid sheet width
};

__device__ __forceinline__ uint32_t byte_of(uint32_t w, int k) { return (w >> (8 * k)) & 0xffu; }

__device__ __forceinline__ float inv_log(float v) {
    // Rust f32::signum: 1 for +0 and positives, -1 for -0 and negatives.
    const float s = signbit(v) ? -1.0f : 1.0f;
    return v != v ? v : s * expm1f(fabsf(v));
}

__device__ __forceinline__ uint32_t ordered(float v) {
    const uint32_t b = __float_as_uint(v);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__global__ void sog_planes_kernel(SogArgs a, float* __restrict__ attr, float* __restrict__ sh,
                                  uint32_t* bounds_u) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < a.n;
    float p[3] = {0.0f, 0.0f, 0.0f};
    if (valid) {
        const size_t N = a.n;
        const uint32_t lo = a.lo[i], hi = a.hi[i];
        for (int k = 0; k < 3; ++k) {
            const float t = (float)(byte_of(lo, k) | (byte_of(hi, k) << 8)) / 65535.0f;
            p[k] = inv_log(a.mins[k] + a.spans[k] * t);
            attr[k * N + i] = p[k];
        }
        const uint32_t sc = a.scales[i];
        for (int k = 0; k < 3; ++k) attr[(7 + k) * N + i] = a.scales_cb[byte_of(sc, k)];
        const uint32_t qc = a.quats[i];
        auto u = [](uint32_t v) { return ((float)v / 255.0f * 2.0f - 1.0f) / 1.41421356237309504880f; };
        const float qa = u(byte_of(qc, 0)), qb = u(byte_of(qc, 1)), qcc = u(byte_of(qc, 2));
        const float d = sqrtf(fmaxf(((1.0f - qa * qa) - qb * qb) - qcc * qcc, 0.0f));
        float q[4];
        switch (byte_of(qc, 3)) {
            case 252: q[0] = d; q[1] = qa; q[2] = qb; q[3] = qcc; break;
            case 253: q[0] = qa; q[1] = d; q[2] = qb; q[3] = qcc; break;
            case 254: q[0] = qa; q[1] = qb; q[2] = d; q[3] = qcc; break;
            default: q[0] = qa; q[1] = qb; q[2] = qcc; q[3] = d; break;
        }
        for (int k = 0; k < 4; ++k) attr[(3 + k) * N + i] = q[k];
        const uint32_t c0 = a.sh0[i];
        for (int k = 0; k < 3; ++k) sh[k * N + i] = a.sh0_cb[byte_of(c0, k)];
        const float y = (float)byte_of(c0, 3) / 255.0f;
        const float e = fminf(fmaxf(y, 1e-6f), 1.0f - 1e-6f);
        attr[10 * N + i] = logf(e / (1.0f - e));
        if (a.k > 1) {
            const uint32_t m = a.k - 1;
            const uint32_t lw = a.labels[i];
            const uint32_t label = byte_of(lw, 0) | (byte_of(lw, 1) << 8);
            const uint32_t per_row = a.cw / m;
            const uint32_t bx = label % per_row * m, by = label / per_row;
            for (uint32_t j = 0; j < m; ++j) {
                const uint32_t c = a.centroids[(size_t)by * a.cw + bx + j];
                for (int k = 0; k < 3; ++k) sh[((j + 1) * 3 + k) * N + i] = a.shn_cb[byte_of(c, k)];
            }
        }
    }
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

// Everything parse_sog checks, on the host; the decoded planes.
struct Sog {
    Meta meta;
    uint32_t n = 0, k = 1;
    Plane lo, hi, scales, quats, sh0, centroids, labels;
};

Sog read_sog(const uint8_t* p, size_t len, bool decode_planes) {
    Sog s;
    const auto dir = zip_directory(p, len);
    if (!dir.count("meta.json")) throw SogFail{"missing meta.json"};
    s.meta = parse_meta(zip_read(p, len, dir, "meta.json"));
    const Meta& m = s.meta;
    if (m.count == 0) throw SogFail{"SOG contains no splats"};
    s.n = (uint32_t)m.count;
    s.k = sh_per_ch_of(m);
    if (!decode_planes) return s;
    s.lo = decode_rgba(p, len, dir, m.means[0], m.count);
    s.hi = decode_rgba(p, len, dir, m.means[1], m.count);
    s.scales = decode_rgba(p, len, dir, m.scales, m.count);
    codebook_check(m.scales_cb, "scales");
    s.quats = decode_rgba(p, len, dir, m.quats, m.count);
    for (uint32_t i = 0; i < s.n; ++i) {
        const uint32_t tag = s.quats.rgba[i] >> 24;
        if (tag < 252) throw SogFail{"quats: invalid rotation tag " + std::to_string(tag)};
    }
    s.sh0 = decode_rgba(p, len, dir, m.sh0, m.count);
    codebook_check(m.sh0_cb, "sh0");
    if (m.has_shn) {
        const uint32_t per = s.k - 1;
        s.centroids = decode_rgba(p, len, dir, m.shn[0], 1);
        s.labels = decode_rgba(p, len, dir, m.shn[1], m.count);
        codebook_check(m.shn_cb, "shN");
        const uint64_t palettes = (uint64_t)s.centroids.w * s.centroids.h / per;
        const uint32_t per_row = s.centroids.w / per;
        for (uint32_t i = 0; i < s.n; ++i) {
            const uint32_t w = s.labels.rgba[i];
            const uint32_t label = (w & 0xffu) | (w & 0xff00u);
            if (label >= palettes)
                throw SogFail{"shN label " + std::to_string(label) + " >= palette size " + std::to_string(palettes)};
            // palette_offset (sog.rs:202-205) must land inside the sheet.
            const uint64_t end = (per_row ? (uint64_t)(label / per_row) * s.centroids.w + label % per_row * per : ~0ull) + per;
            if (per_row == 0 || end > (uint64_t)s.centroids.w * s.centroids.h)
                throw SogFail{"shN label " + std::to_string(label) + " outside the centroid sheet"};
        }
    }
    return s;
}

int sog_fail(int code, const std::string& msg) { return set_error(code, "SOG: " + msg); }

}  // namespace
}  // namespace sfk

using namespace sfk;

extern "C" {

int sf_sog_inspect(const void* bytes, size_t len, uint32_t* n, uint32_t* sh_per_ch) {
    try {
        if (!bytes) return sog_fail(SF_ERR_ARG, "null bytes");
        const Sog s = read_sog(static_cast<const uint8_t*>(bytes), len, false);
        if (n) *n = s.n;
        if (sh_per_ch) *sh_per_ch = s.k;
        return SF_OK;
    } catch (const SogFail& f) {
        return sog_fail(SF_ERR_ARG, f.msg);
    } catch (const std::bad_alloc&) {
        return sog_fail(SF_ERR_NOMEM, "host allocation failed");
    } catch (const std::exception&) {
        return sog_fail(SF_ERR_ARG, "invalid meta.json");
    }
}

int sf_sog_load(sf_ctx ctx, const void* bytes, size_t len, sf_splats* out) {
    try {
        if (!ctx || !out || !bytes) return sog_fail(SF_ERR_ARG, "null argument");
        *out = nullptr;
        const Sog s = read_sog(static_cast<const uint8_t*>(bytes), len, true);
        const uint32_t n = s.n;
        int cur = -1;
        cudaError_t e = cudaGetDevice(&cur);
        if (e == cudaSuccess && cur != ctx->device) e = cudaSetDevice(ctx->device);
        // Device staging: six n-word planes (labels only with shN), the
        // centroid sheet, three codebooks, the bounds words.
        const int nplanes = s.k > 1 ? 6 : 5;
        uint32_t* planes = nullptr;
        uint32_t* cent = nullptr;
        float* cbs = nullptr;
        uint32_t* bounds_u = nullptr;
        auto* sp = new sf_splats_t();
        sp->ctx = ctx;
        sp->n = n;
        sp->K = s.k;
        if (e == cudaSuccess) e = cudaMalloc(&planes, (size_t)nplanes * n * 4);
        if (e == cudaSuccess) e = cudaMalloc(&cent, std::max<size_t>(s.centroids.rgba.size(), 1) * 4);
        if (e == cudaSuccess) e = cudaMalloc(&cbs, 3 * 256 * 4);
        if (e == cudaSuccess) e = cudaMalloc(&bounds_u, 6 * 4);
        if (e == cudaSuccess) e = cudaMalloc(&sp->attr, (size_t)11 * n * 4);
        if (e == cudaSuccess) e = cudaMalloc(&sp->sh, (size_t)3 * s.k * n * 4);
        if (e == cudaSuccess) e = cudaMalloc(&sp->geom, (size_t)kGeomPlanes * n * 4);
        const Plane* src[6] = {&s.lo, &s.hi, &s.scales, &s.quats, &s.sh0, &s.labels};
        for (int k = 0; k < nplanes && e == cudaSuccess; ++k)
            e = cudaMemcpy(planes + (size_t)k * n, src[k]->rgba.data(), (size_t)n * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !s.centroids.rgba.empty())
            e = cudaMemcpy(cent, s.centroids.rgba.data(), s.centroids.rgba.size() * 4, cudaMemcpyHostToDevice);
        std::vector<float> cb(3 * 256, 0.0f);
        std::copy(s.meta.scales_cb.begin(), s.meta.scales_cb.end(), cb.begin());
        std::copy(s.meta.sh0_cb.begin(), s.meta.sh0_cb.end(), cb.begin() + 256);
        if (s.meta.has_shn) std::copy(s.meta.shn_cb.begin(), s.meta.shn_cb.end(), cb.begin() + 512);
        if (e == cudaSuccess) e = cudaMemcpy(cbs, cb.data(), cb.size() * 4, cudaMemcpyHostToDevice);
        const uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
        if (e == cudaSuccess) e = cudaMemcpy(bounds_u, init, sizeof(init), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) {
            SogArgs a{};
            a.n = n;
            a.k = s.k;
            for (int k = 0; k < 3; ++k) {
                a.mins[k] = s.meta.mins[k];
                a.spans[k] = s.meta.maxs[k] - s.meta.mins[k];
            }
            a.lo = planes;
            a.hi = planes + (size_t)n;
            a.scales = planes + 2 * (size_t)n;
            a.quats = planes + 3 * (size_t)n;
            a.sh0 = planes + 4 * (size_t)n;
            a.labels = s.k > 1 ? planes + 5 * (size_t)n : nullptr;
            a.centroids = cent;
            a.scales_cb = cbs;
            a.sh0_cb = cbs + 256;
            a.shn_cb = cbs + 512;
            a.cw = s.centroids.w;
            sog_planes_kernel<<<(n + 255) / 256, 256>>>(a, sp->attr, sp->sh, bounds_u);
            note_launches(1);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = launch_splat_geom(sp->attr, n, sp->geom, nullptr);
        uint32_t bu[6] = {0, 0, 0, 0, 0, 0};
        if (e == cudaSuccess) e = cudaMemcpy(bu, bounds_u, sizeof(bu), cudaMemcpyDeviceToHost);
        if (planes) cudaFree(planes);
        if (cent) cudaFree(cent);
        if (cbs) cudaFree(cbs);
        if (bounds_u) cudaFree(bounds_u);
        if (e != cudaSuccess) {
            if (sp->attr) cudaFree(sp->attr);
            if (sp->sh) cudaFree(sp->sh);
            if (sp->geom) cudaFree(sp->geom);
            delete sp;
            return sog_fail(e == cudaErrorMemoryAllocation ? SF_ERR_NOMEM : SF_ERR_CUDA, cudaGetErrorString(e));
        }
        for (int k = 0; k < 3; ++k) {
            auto unord = [](uint32_t u) {
                const uint32_t b = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
                float f;
                std::memcpy(&f, &b, 4);
                return f;
            };
            sp->bounds[k] = bu[k] == 0xffffffffu ? 3.4028235e38f : unord(bu[k]);
            sp->bounds[3 + k] = bu[3 + k] == 0u ? -3.4028235e38f : unord(bu[3 + k]);
        }
        *out = sp;
        return SF_OK;
    } catch (const SogFail& f) {
        return sog_fail(SF_ERR_ARG, f.msg);
    } catch (const std::bad_alloc&) {
        return sog_fail(SF_ERR_NOMEM, "host allocation failed");
    } catch (const std::exception&) {
        return sog_fail(SF_ERR_ARG, "invalid meta.json");
    }
}

int sf_sog_load_file(sf_ctx ctx, const char* path, sf_splats* out) {
    try {
        if (!path) return sog_fail(SF_ERR_ARG, "null path");
        std::ifstream f(path, std::ios::binary | std::ios::ate);
        if (!f) return sog_fail(SF_ERR_ARG, std::string("cannot open ") + path);
        const std::streamsize size = f.tellg();
        f.seekg(0);
        std::vector<uint8_t> bytes((size_t)std::max<std::streamsize>(size, 0));
        if (size > 0 && !f.read(reinterpret_cast<char*>(bytes.data()), size))
            return sog_fail(SF_ERR_ARG, std::string("cannot read ") + path);
        return sf_sog_load(ctx, bytes.data(), bytes.size(), out);
    } catch (const std::bad_alloc&) {
        return sog_fail(SF_ERR_NOMEM, "host allocation failed");
    }
}

}  // extern "C"
