// Lossless WebP decoder (host), for the SOG scene loader.
//
// The reference decodes SOG planes with the `image` crate (src/sog.rs:44-66);
// that decoder is a third-party dependency and not part of the reference, so
// this file restates the published format instead: the RIFF container
// ("RIFF" size "WEBP", a "VP8L" chunk, optionally behind a "VP8X" header) and
// the VP8L lossless bitstream of RFC 9649 ("WebP Image Format"), section 3:
//  * bits are read least-significant first;
//  * prefix codes are canonical (DEFLATE-style: shorter codes first, ties by
//    symbol), read either as "simple" (1-2 literal symbols) or as code
//    lengths coded with a 19-symbol code-length code and repeat codes 16-18;
//  * an entropy-coded image is a sequence of literal ARGB pixels, LZ77
//    backward references (length and distance through prefix values with
//    extra bits; distances 1..120 map to 2-D neighbour offsets) and
//    color-cache hits (hash 0x1e35a7bd * argb >> (32 - cache_bits));
//  * the main image may use several prefix-code groups, chosen per block by
//    an entropy sub-image;
//  * transforms (predictor with 14 modes, cross colour, subtract green and
//    colour indexing with pixel bundling) are undone in reverse order.
// Lossy ("VP8 ") images are refused: SOG planes are lossless.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include "sf_handles.h"

namespace sfk {
namespace webp {
namespace {

struct Fail {
    std::string msg;
};

// Least-significant-bit-first reader. Past the end it reads zeros; a read
// or skip that consumes bits past the end of the data throws.
class Bits {
   public:
    Bits(const uint8_t* p, size_t n) : p_(p), n_(n) {}
    uint32_t read(int k) {
        const uint32_t v = peek(k);
        skip(k);
        return v;
    }
    uint32_t peek(int k) {
        if (have_ < k) fill();
        return (uint32_t)(buf_ & ((1ull << k) - 1));
    }
    void skip(int k) {
        if (have_ < k) fill();
        buf_ >>= k;
        have_ -= k;
        used_ += (uint64_t)k;
        if (used_ > 8 * (uint64_t)n_) throw Fail{"truncated bitstream"};
    }

   private:
    void fill() {
        while (have_ <= 56) {
            const uint64_t byte = pos_ < n_ ? p_[pos_] : 0u;
            buf_ |= byte << have_;
            have_ += 8;
            ++pos_;
        }
    }
    const uint8_t* p_;
    size_t n_;
    size_t pos_ = 0;
    uint64_t buf_ = 0;
    int have_ = 0;
    uint64_t used_ = 0;
};

// Canonical prefix code with an 8-bit root table and second-level tables.
class Code {
   public:
    static constexpr int kRoot = 8;
    void build(const std::vector<uint8_t>& len) {
        const int n = (int)len.size();
        int count[16] = {0};
        int used = 0, last = 0;
        for (int s = 0; s < n; ++s) {
            if (len[s] > 15) throw Fail{"code length above 15"};
            if (len[s]) {
                ++count[len[s]];
                ++used;
                last = s;
            }
        }
        root_.assign(1 << kRoot, Entry{0, 0, 0});
        sub_.clear();
        single_ = -1;
        if (used == 0) throw Fail{"empty prefix code"};
        if (used == 1) {
            single_ = last;  // one symbol: zero bits per symbol
            return;
        }
        // Canonical codes, checked for over-subscription.
        int next[16] = {0};
        int code = 0;
        for (int l = 1; l <= 15; ++l) {
            code = (code + count[l - 1]) << 1;
            next[l] = code;
            if (next[l] + count[l] > (1 << l)) throw Fail{"over-subscribed prefix code"};
        }
        next[0] = 0;
        std::vector<uint32_t> rev(n, 0);
        int maxsub[1 << kRoot];
        for (int i = 0; i < (1 << kRoot); ++i) maxsub[i] = 0;
        for (int s = 0; s < n; ++s) {
            const int l = len[s];
            if (!l) continue;
            const uint32_t c = (uint32_t)next[l]++;
            uint32_t r = 0;
            for (int b = 0; b < l; ++b) r |= ((c >> b) & 1u) << (l - 1 - b);
            rev[s] = r;
            if (l <= kRoot) {
                for (uint32_t i = r; i < (1u << kRoot); i += 1u << l) root_[i] = Entry{(uint16_t)s, (uint8_t)l, 0};
            } else {
                const int ri = (int)(r & ((1u << kRoot) - 1));
                maxsub[ri] = std::max(maxsub[ri], l - kRoot);
            }
        }
        for (int ri = 0; ri < (1 << kRoot); ++ri) {
            if (!maxsub[ri]) continue;
            root_[ri] = Entry{(uint16_t)sub_.size(), 0, (uint8_t)maxsub[ri]};
            sub_.resize(sub_.size() + (1u << maxsub[ri]), Entry{0, 0xff, 0});
        }
        for (int s = 0; s < n; ++s) {
            const int l = len[s];
            if (l <= kRoot) continue;
            const Entry& re = root_[rev[s] & ((1u << kRoot) - 1)];
            const uint32_t hi = rev[s] >> kRoot;
            for (uint32_t i = hi; i < (1u << re.sub); i += 1u << (l - kRoot))
                sub_[re.sym + i] = Entry{(uint16_t)s, (uint8_t)(l - kRoot), 0};
        }
        // Root slots no code reaches stay unusable.
        for (auto& e : root_)
            if (e.len == 0 && e.sub == 0) e.len = 0xff;
    }
    int read(Bits& b) const {
        if (single_ >= 0) return single_;
        const uint32_t v = b.peek(15);
        const Entry& e = root_[v & ((1u << kRoot) - 1)];
        if (e.sub == 0) {
            if (e.len == 0xff) throw Fail{"invalid prefix code"};
            b.skip(e.len);
            return e.sym;
        }
        const Entry& s = sub_[e.sym + ((v >> kRoot) & ((1u << e.sub) - 1))];
        if (s.len == 0xff) throw Fail{"invalid prefix code"};
        b.skip(kRoot + s.len);
        return s.sym;
    }

   private:
    struct Entry {
        uint16_t sym;
        uint8_t len;  // bits consumed (0xff: no code)
        uint8_t sub;  // root entries: bits of the second-level table
    };
    std::vector<Entry> root_, sub_;
    int single_ = -1;
};

const int kCodeLengthOrder[19] = {17, 18, 0, 1, 2, 3, 4, 5, 16, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15};

Code read_code(Bits& b, int alphabet) {
    std::vector<uint8_t> len(alphabet, 0);
    if (b.read(1)) {
        // Simple code: one or two symbols.
        const int count = (int)b.read(1) + 1;
        const int first_bits = b.read(1) ? 8 : 1;
        const int s0 = (int)b.read(first_bits);
        if (s0 >= alphabet) throw Fail{"simple code symbol out of range"};
        len[s0] = 1;
        if (count == 2) {
            const int s1 = (int)b.read(8);
            if (s1 >= alphabet) throw Fail{"simple code symbol out of range"};
            len[s1] = 1;
        }
    } else {
        std::vector<uint8_t> cl(19, 0);
        const int ncl = 4 + (int)b.read(4);
        for (int i = 0; i < ncl; ++i) cl[kCodeLengthOrder[i]] = (uint8_t)b.read(3);
        Code clc;
        clc.build(cl);
        int max_symbol = alphabet;
        if (b.read(1)) {
            const int nbits = 2 + 2 * (int)b.read(3);
            max_symbol = 2 + (int)b.read(nbits);
            if (max_symbol > alphabet) throw Fail{"code length count above the alphabet"};
        }
        int prev = 8;
        int s = 0;
        while (s < alphabet) {
            if (max_symbol-- == 0) break;
            const int c = clc.read(b);
            if (c < 16) {
                len[s++] = (uint8_t)c;
                if (c) prev = c;
            } else {
                int rep, val;
                if (c == 16) {
                    rep = 3 + (int)b.read(2);
                    val = prev;
                } else if (c == 17) {
                    rep = 3 + (int)b.read(3);
                    val = 0;
                } else {
                    rep = 11 + (int)b.read(7);
                    val = 0;
                }
                if (s + rep > alphabet) throw Fail{"code length repeat past the alphabet"};
                for (int k = 0; k < rep; ++k) len[s++] = (uint8_t)val;
            }
        }
    }
    Code code;
    code.build(len);
    return code;
}

struct Group {
    Code g, r, b, a, d;  // green+length+cache, red, blue, alpha, distance
};

uint32_t prefix_value(Bits& b, int prefix) {
    if (prefix < 4) return (uint32_t)prefix + 1;
    const int extra = (prefix - 2) >> 1;
    const uint32_t offset = (uint32_t)(2 + (prefix & 1)) << extra;
    return offset + b.read(extra) + 1;
}

// The 120 short distance codes: (dx, dy) neighbour offsets, the distance
// being dx + dy * width (at least 1).
const int8_t kDistXY[120][2] = {
    {0, 1},  {1, 0},  {1, 1},  {-1, 1}, {0, 2},  {2, 0},  {1, 2},  {-1, 2}, {2, 1},  {-2, 1}, {2, 2},  {-2, 2},
    {0, 3},  {3, 0},  {1, 3},  {-1, 3}, {3, 1},  {-3, 1}, {2, 3},  {-2, 3}, {3, 2},  {-3, 2}, {0, 4},  {4, 0},
    {1, 4},  {-1, 4}, {4, 1},  {-4, 1}, {3, 3},  {-3, 3}, {2, 4},  {-2, 4}, {4, 2},  {-4, 2}, {0, 5},  {3, 4},
    {-3, 4}, {4, 3},  {-4, 3}, {5, 0},  {1, 5},  {-1, 5}, {5, 1},  {-5, 1}, {2, 5},  {-2, 5}, {5, 2},  {-5, 2},
    {4, 4},  {-4, 4}, {3, 5},  {-3, 5}, {5, 3},  {-5, 3}, {0, 6},  {6, 0},  {1, 6},  {-1, 6}, {6, 1},  {-6, 1},
    {2, 6},  {-2, 6}, {6, 2},  {-6, 2}, {4, 5},  {-4, 5}, {5, 4},  {-5, 4}, {3, 6},  {-3, 6}, {6, 3},  {-6, 3},
    {0, 7},  {7, 0},  {1, 7},  {-1, 7}, {5, 5},  {-5, 5}, {7, 1},  {-7, 1}, {4, 6},  {-4, 6}, {6, 4},  {-6, 4},
    {2, 7},  {-2, 7}, {7, 2},  {-7, 2}, {3, 7},  {-3, 7}, {7, 3},  {-7, 3}, {5, 6},  {-5, 6}, {6, 5},  {-6, 5},
    {8, 0},  {4, 7},  {-4, 7}, {7, 4},  {-7, 4}, {8, 1},  {8, 2},  {6, 6},  {-6, 6}, {8, 3},  {5, 7},  {-5, 7},
    {7, 5},  {-7, 5}, {8, 4},  {6, 7},  {-6, 7}, {7, 6},  {-7, 6}, {8, 5},  {7, 7},  {-7, 7}, {8, 6},  {8, 7}};

inline uint32_t div_up(uint32_t v, int bits) { return (v + (1u << bits) - 1) >> bits; }

// One entropy-coded image of w x h pixels. level0: the main image, which
// may carry prefix-code groups chosen by an entropy sub-image.
std::vector<uint32_t> decode_entropy_image(Bits& b, uint32_t w, uint32_t h, bool level0);

std::vector<uint32_t> decode_sub_image(Bits& b, uint32_t w, uint32_t h) {
    return decode_entropy_image(b, w, h, false);
}

std::vector<uint32_t> decode_entropy_image(Bits& b, uint32_t w, uint32_t h, bool level0) {
    int cache_bits = 0;
    if (b.read(1)) {
        cache_bits = (int)b.read(4);
        if (cache_bits < 1 || cache_bits > 11) throw Fail{"colour cache size out of range"};
    }
    int prefix_bits = 0;
    std::vector<uint32_t> entropy;
    uint32_t groups_n = 1, ew = 0;
    if (level0 && b.read(1)) {
        prefix_bits = (int)b.read(3) + 2;
        ew = div_up(w, prefix_bits);
        entropy = decode_sub_image(b, ew, div_up(h, prefix_bits));
        for (auto& v : entropy) {
            v = (v >> 8) & 0xffffu;
            groups_n = std::max(groups_n, v + 1);
        }
    }
    const int cache_size = cache_bits ? (1 << cache_bits) : 0;
    std::vector<Group> groups(groups_n);
    for (auto& g : groups) {
        g.g = read_code(b, 256 + 24 + cache_size);
        g.r = read_code(b, 256);
        g.b = read_code(b, 256);
        g.a = read_code(b, 256);
        g.d = read_code(b, 40);
    }
    const size_t total = (size_t)w * h;
    std::vector<uint32_t> px(total);
    std::vector<uint32_t> cache(cache_size ? cache_size : 1, 0);
    size_t pos = 0, cached = 0;
    auto insert = [&](size_t upto) {
        if (!cache_size) return;
        for (; cached < upto; ++cached)
            cache[(0x1e35a7bdu * px[cached]) >> (32 - cache_bits)] = px[cached];
    };
    while (pos < total) {
        const uint32_t x = (uint32_t)(pos % w), y = (uint32_t)(pos / w);
        const Group& g = prefix_bits ? groups[entropy[(size_t)(y >> prefix_bits) * ew + (x >> prefix_bits)]]
                                     : groups[0];
        const int s = g.g.read(b);
        if (s < 256) {
            const uint32_t red = (uint32_t)g.r.read(b);
            const uint32_t blue = (uint32_t)g.b.read(b);
            const uint32_t alpha = (uint32_t)g.a.read(b);
            px[pos++] = (alpha << 24) | (red << 16) | ((uint32_t)s << 8) | blue;
        } else if (s < 256 + 24) {
            const uint32_t length = prefix_value(b, s - 256);
            const int ds = g.d.read(b);
            const uint32_t dcode = prefix_value(b, ds);
            int64_t dist;
            if (dcode > 120) {
                dist = (int64_t)dcode - 120;
            } else {
                const int8_t* xy = kDistXY[dcode - 1];
                dist = (int64_t)xy[0] + (int64_t)xy[1] * w;
                if (dist < 1) dist = 1;
            }
            if ((uint64_t)dist > pos || pos + length > total) throw Fail{"backward reference out of range"};
            for (uint32_t k = 0; k < length; ++k, ++pos) px[pos] = px[pos - (size_t)dist];
        } else {
            const int key = s - 280;
            if (key >= cache_size) throw Fail{"colour cache index out of range"};
            insert(pos);
            px[pos++] = cache[key];
        }
        insert(pos);
    }
    return px;
}

inline uint32_t add_px(uint32_t a, uint32_t b) {
    const uint32_t ag = (a & 0xff00ff00u) + (b & 0xff00ff00u);
    const uint32_t rb = (a & 0x00ff00ffu) + (b & 0x00ff00ffu);
    return (ag & 0xff00ff00u) | (rb & 0x00ff00ffu);
}
inline uint32_t avg2(uint32_t a, uint32_t b) { return (((a ^ b) & 0xfefefefeu) >> 1) + (a & b); }
inline int ch(uint32_t p, int k) { return (int)((p >> (8 * k)) & 0xffu); }
inline uint32_t clamp_px(int a, int r, int g, int b) {
    auto c = [](int v) { return (uint32_t)(v < 0 ? 0 : v > 255 ? 255 : v); };
    return (c(a) << 24) | (c(r) << 16) | (c(g) << 8) | c(b);
}
uint32_t select_px(uint32_t L, uint32_t T, uint32_t TL) {
    int pl = 0, pt = 0;
    for (int k = 0; k < 4; ++k) {
        const int p = ch(L, k) + ch(T, k) - ch(TL, k);
        pl += std::abs(p - ch(L, k));
        pt += std::abs(p - ch(T, k));
    }
    return pl < pt ? L : T;
}
uint32_t clamp_add_sub_full(uint32_t a, uint32_t b, uint32_t c) {
    return clamp_px(ch(a, 3) + ch(b, 3) - ch(c, 3), ch(a, 2) + ch(b, 2) - ch(c, 2), ch(a, 1) + ch(b, 1) - ch(c, 1),
                    ch(a, 0) + ch(b, 0) - ch(c, 0));
}
uint32_t clamp_add_sub_half(uint32_t a, uint32_t b) {
    auto h = [&](int k) { return ch(a, k) + (ch(a, k) - ch(b, k)) / 2; };
    return clamp_px(h(3), h(2), h(1), h(0));
}

uint32_t predict(int mode, const uint32_t* cur, const uint32_t* up) {
    const uint32_t L = cur[-1], T = up[0], TL = up[-1], TR = up[1];
    switch (mode) {
        case 0: return 0xff000000u;
        case 1: return L;
        case 2: return T;
        case 3: return TR;
        case 4: return TL;
        case 5: return avg2(avg2(L, TR), T);
        case 6: return avg2(L, TL);
        case 7: return avg2(L, T);
        case 8: return avg2(TL, T);
        case 9: return avg2(T, TR);
        case 10: return avg2(avg2(L, TL), avg2(T, TR));
        case 11: return select_px(L, T, TL);
        case 12: return clamp_add_sub_full(L, T, TL);
        case 13: return clamp_add_sub_half(avg2(L, T), TL);
        default: return 0xff000000u;  // modes 14 and 15: as mode 0
    }
}

struct Transform {
    int type;
    int bits;
    uint32_t w_before;  // image width before this transform's packing
    std::vector<uint32_t> data;
};

void undo_predictor(std::vector<uint32_t>& px, uint32_t w, uint32_t h, const Transform& t) {
    const uint32_t bw = div_up(w, t.bits);
    for (uint32_t y = 0; y < h; ++y) {
        uint32_t* row = px.data() + (size_t)y * w;
        for (uint32_t x = 0; x < w; ++x) {
            uint32_t pred;
            if (y == 0) pred = x == 0 ? 0xff000000u : row[x - 1];
            else if (x == 0) pred = row[-(int64_t)w];
            else pred = predict((int)((t.data[(size_t)(y >> t.bits) * bw + (x >> t.bits)] >> 8) & 0xfu), row + x,
                                row + x - w);
            row[x] = add_px(row[x], pred);
        }
    }
}

inline int delta(int8_t t, int8_t c) { return ((int)t * (int)c) >> 5; }

void undo_cross_colour(std::vector<uint32_t>& px, uint32_t w, uint32_t h, const Transform& t) {
    const uint32_t bw = div_up(w, t.bits);
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x) {
            const uint32_t m = t.data[(size_t)(y >> t.bits) * bw + (x >> t.bits)];
            const int8_t g2r = (int8_t)(m & 0xff), g2b = (int8_t)((m >> 8) & 0xff), r2b = (int8_t)((m >> 16) & 0xff);
            uint32_t& p = px[(size_t)y * w + x];
            const int8_t green = (int8_t)((p >> 8) & 0xff);
            int red = (int)((p >> 16) & 0xff), blue = (int)(p & 0xff);
            red = (red + delta(g2r, green)) & 0xff;
            blue = (blue + delta(g2b, green)) & 0xff;
            blue = (blue + delta(r2b, (int8_t)red)) & 0xff;
            p = (p & 0xff00ff00u) | ((uint32_t)red << 16) | (uint32_t)blue;
        }
}

void undo_subtract_green(std::vector<uint32_t>& px) {
    for (auto& p : px) {
        const uint32_t g = (p >> 8) & 0xff;
        const uint32_t rb = ((p & 0x00ff00ffu) + ((g << 16) | g)) & 0x00ff00ffu;
        p = (p & 0xff00ff00u) | rb;
    }
}

// Colour indexing: packed index pixels (width pw) -> colours (width w).
std::vector<uint32_t> undo_colour_index(const std::vector<uint32_t>& px, uint32_t pw, uint32_t w, uint32_t h,
                                        const Transform& t) {
    std::vector<uint32_t> out((size_t)w * h);
    const int per = 1 << t.bits;          // indices per packed pixel
    const int nbits = 8 >> t.bits;        // bits per index
    const uint32_t mask = (1u << nbits) - 1;
    const size_t table_n = t.data.size();
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x) {
            const uint32_t packed = (px[(size_t)y * pw + (x >> t.bits)] >> 8) & 0xff;
            const uint32_t idx = (packed >> (nbits * (int)(x & (uint32_t)(per - 1)))) & mask;
            out[(size_t)y * w + x] = idx < table_n ? t.data[idx] : 0u;
        }
    return out;
}

std::vector<uint32_t> decode_vp8l(const uint8_t* p, size_t n, uint32_t* w_out, uint32_t* h_out) {
    if (n < 5 || p[0] != 0x2f) throw Fail{"not a lossless WebP bitstream (VP8L signature)"};
    Bits b(p + 1, n - 1);
    const uint32_t w = b.read(14) + 1, h = b.read(14) + 1;
    b.read(1);  // alpha hint
    if (b.read(3) != 0) throw Fail{"unknown VP8L version"};
    std::vector<Transform> ts;
    uint32_t cw = w;
    int seen = 0;
    while (b.read(1)) {
        Transform t{};
        t.type = (int)b.read(2);
        if (seen & (1 << t.type)) throw Fail{"transform repeated"};
        seen |= 1 << t.type;
        t.w_before = cw;
        if (t.type == 0 || t.type == 1) {
            t.bits = (int)b.read(3) + 2;
            t.data = decode_sub_image(b, div_up(cw, t.bits), div_up(h, t.bits));
        } else if (t.type == 3) {
            const uint32_t size = b.read(8) + 1;
            t.data = decode_sub_image(b, size, 1);
            for (uint32_t i = 1; i < size; ++i) t.data[i] = add_px(t.data[i], t.data[i - 1]);
            t.bits = size <= 2 ? 3 : size <= 4 ? 2 : size <= 16 ? 1 : 0;
            cw = div_up(cw, t.bits);
        }
        ts.push_back(std::move(t));
    }
    std::vector<uint32_t> px = decode_entropy_image(b, cw, h, true);
    for (auto it = ts.rbegin(); it != ts.rend(); ++it) {
        switch (it->type) {
            case 0: undo_predictor(px, cw, h, *it); break;
            case 1: undo_cross_colour(px, cw, h, *it); break;
            case 2: undo_subtract_green(px); break;
            case 3:
                px = undo_colour_index(px, cw, it->w_before, h, *it);
                cw = it->w_before;
                break;
        }
    }
    *w_out = w;
    *h_out = h;
    return px;
}

uint32_t le32(const uint8_t* p) { return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24; }

}  // namespace

// RIFF container -> ARGB pixels (row-major, 0xAARRGGBB).
int decode(const uint8_t* p, size_t n, uint32_t* w, uint32_t* h, std::vector<uint32_t>* argb, std::string* err) {
    try {
        if (n < 12 || std::memcmp(p, "RIFF", 4) != 0 || std::memcmp(p + 8, "WEBP", 4) != 0)
            throw Fail{"not a WebP file (RIFF/WEBP header)"};
        size_t off = 12;
        const size_t end = std::min(n, (size_t)le32(p + 4) + 8);
        while (off + 8 <= end) {
            const uint8_t* c = p + off;
            const uint32_t size = le32(c + 4);
            if (off + 8 + (size_t)size > end) throw Fail{"truncated RIFF chunk"};
            if (std::memcmp(c, "VP8L", 4) == 0) {
                *argb = decode_vp8l(c + 8, size, w, h);
                return SF_OK;
            }
            if (std::memcmp(c, "VP8 ", 4) == 0) throw Fail{"lossy WebP is not supported (SOG planes are lossless)"};
            off += 8 + (size_t)size + (size & 1u);
        }
        throw Fail{"no VP8L chunk"};
    } catch (const Fail& f) {
        *err = f.msg;
        return SF_ERR_ARG;
    }
}

}  // namespace webp
}  // namespace sfk

extern "C" int sf_webp_decode(const void* bytes, size_t len, uint32_t* w, uint32_t* h, uint8_t* rgba, size_t cap) {
    try {
        if (!bytes || !w || !h) return sfk::set_error(SF_ERR_ARG, "null argument");
        std::vector<uint32_t> argb;
        std::string err;
        const int rc = sfk::webp::decode(static_cast<const uint8_t*>(bytes), len, w, h, &argb, &err);
        if (rc != SF_OK) return sfk::set_error(rc, "WebP: " + err);
        if (!rgba) return SF_OK;
        if (cap < argb.size() * 4) return sfk::set_error(SF_ERR_SHAPE, "output smaller than w * h * 4 bytes");
        for (size_t i = 0; i < argb.size(); ++i) {
            const uint32_t v = argb[i];
            rgba[4 * i + 0] = (uint8_t)(v >> 16);
            rgba[4 * i + 1] = (uint8_t)(v >> 8);
            rgba[4 * i + 2] = (uint8_t)v;
            rgba[4 * i + 3] = (uint8_t)(v >> 24);
        }
        return SF_OK;
    } catch (const std::bad_alloc&) {
        return sfk::set_error(SF_ERR_NOMEM, "host allocation failed");
    }
}
