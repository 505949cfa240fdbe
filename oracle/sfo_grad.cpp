// Oracle FP64 twin of the render path and its exact adjoint (TEST
// INFRASTRUCTURE ONLY; the reference has no backward pass).
//
// Forward: the same steps as sfo_render.cpp (src/project.rs:235-327,
// src/raster.rs:88-230) in double with libm exp/log. Backward: reverse-mode
// derivative of that forward for L = sum_p <dl_drgba[p], rgba[p]>, with
//   alpha = min(op*exp(-power), 0.999)  (zero gradient where the clamp binds),
//   pairs with alpha < 1/255 skipped, a pixel stopping after the contributor
//   that takes T below 1/255 (src/raster.rs:212-218),
//   the 1.3x FOV clamp on u, v (src/project.rs:192-195), the det floor 1e-6
//   (:225) and the +0.3 dilation (:217-219) differentiated as written,
//   culling and tile binning treated as constants.
// The per-pixel backward keeps each pixel's contributor list (exact, no
// transmittance division), so it is an independent check of the GPU adjoint
// that replays from the stored final T.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include <omp.h>
#include "sfo.h"

namespace {

constexpr double kAlphaCutoff = (double)(10.0f / 255.0f);
constexpr double C0 = 0.2820948, C1 = 0.48860252, C20 = 0.9461747, C21 = 0.31539157,
                 C22 = -1.0925485, C23 = 0.54627424;
constexpr double K3 = -0.5900436, A3 = -2.285229, B3 = 0.4570458, E3 = 1.8658817,
                 F3 = 1.119529, G3 = 1.4453057;

struct View64 {
    double rot[3][3], trans[3], focal[2], world_pos[3], img[2];
    uint32_t tiles_x, tiles_y;
};

View64 make_view(const sfo_camera* cam, uint32_t w, uint32_t h) {
    sfo_view v;
    sfo_view_for_camera(cam, w, h, &v);
    View64 o;
    for (int j = 0; j < 3; ++j) {
        o.rot[0][j] = v.rot0[j]; o.rot[1][j] = v.rot1[j]; o.rot[2][j] = v.rot2[j];
        o.trans[j] = v.trans[j]; o.world_pos[j] = v.world_pos[j];
    }
    o.focal[0] = v.focal[0]; o.focal[1] = v.focal[1];
    o.img[0] = w; o.img[1] = h;
    o.tiles_x = (w + 15) / 16; o.tiles_y = (h + 15) / 16;
    return o;
}

// SH basis values B[k] (colour = sum_k B[k]*sh[k][c] + 0.5) and their
// gradients dB[k][3] with respect to the unit direction, in the reference's
// exact polynomial forms (src/project.rs:344-388).
void sh_basis(uint32_t K, const double d[3], double B[16], double dB[16][3]) {
    const double x = d[0], y = d[1], z = d[2];
    for (int k = 0; k < 16; ++k) { B[k] = 0; dB[k][0] = dB[k][1] = dB[k][2] = 0; }
    B[0] = C0;
    if (K >= 4) {
        B[1] = -C1 * y; dB[1][1] = -C1;
        B[2] = C1 * z;  dB[2][2] = C1;
        B[3] = -C1 * x; dB[3][0] = -C1;
    }
    if (K >= 9) {
        B[4] = 2 * C23 * x * y; dB[4][0] = 2 * C23 * y; dB[4][1] = 2 * C23 * x;
        B[5] = C22 * z * y;     dB[5][1] = C22 * z;     dB[5][2] = C22 * y;
        B[6] = C20 * z * z - C21; dB[6][2] = 2 * C20 * z;
        B[7] = C22 * z * x;     dB[7][0] = C22 * z;     dB[7][2] = C22 * x;
        B[8] = C23 * (x * x - y * y); dB[8][0] = 2 * C23 * x; dB[8][1] = -2 * C23 * y;
    }
    if (K >= 16) {
        const double c1x = x * x - y * y, c1y = 2 * x * y, t0 = A3 * z * z + B3;
        B[9] = K3 * x * c1y + y * c1x;
        dB[9][0] = 4 * K3 * x * y + 2 * x * y;
        dB[9][1] = 2 * K3 * x * x + x * x - 3 * y * y;
        B[10] = K3 * x * c1x - y * c1y;
        dB[10][0] = 3 * K3 * x * x - K3 * y * y - 2 * y * y;
        dB[10][1] = -2 * K3 * x * y - 4 * x * y;
        B[11] = t0 * y; dB[11][1] = t0; dB[11][2] = 2 * A3 * z * y;
        B[12] = t0 * x; dB[12][0] = t0; dB[12][2] = 2 * A3 * z * x;
        B[13] = z * (E3 * z * z - F3); dB[13][2] = 3 * E3 * z * z - F3;
        B[14] = G3 * z * c1y; dB[14][0] = 2 * G3 * z * y; dB[14][1] = 2 * G3 * z * x;
        dB[14][2] = G3 * c1y;
        B[15] = G3 * z * c1x; dB[15][0] = 2 * G3 * z * x; dB[15][1] = -2 * G3 * z * y;
        dB[15][2] = G3 * c1x;
    }
}

// Everything the adjoint needs from one splat's projection.
struct Proj {
    bool vis = false;
    double mean[3], q[4], s[3], op;
    double cam[3], iz;
    double R[3][3], M[3][3];
    double u, v; bool u_clamp, v_clamp;
    double t0[3], t1[3], j0[3], j1[3];
    double cov[3], D; bool det_floor;
    double conic[3], m2[2];
    double dir[3], vlen, B[16], dB[16][3], color[3];
    uint32_t bb[2];
};

void project64(const View64& v, const double* attr, const double* sh, uint32_t n, uint32_t K,
               uint32_t i, Proj& p) {
    const size_t N = n;
    for (int j = 0; j < 3; ++j) p.mean[j] = attr[j * N + i];
    for (int j = 0; j < 4; ++j) p.q[j] = attr[(3 + j) * N + i];  // w x y z
    for (int j = 0; j < 3; ++j) p.s[j] = std::exp(attr[(7 + j) * N + i]);
    p.op = 1.0 / (1.0 + std::exp(-attr[10 * N + i]));
    p.vis = false;
    if (!(p.op >= kAlphaCutoff)) return;
    for (int r = 0; r < 3; ++r)
        p.cam[r] = v.rot[r][0] * p.mean[0] + v.rot[r][1] * p.mean[1] + v.rot[r][2] * p.mean[2] +
                   v.trans[r];
    if (!(p.cam[2] > 0.1)) return;
    p.vis = true;
    p.iz = 1.0 / p.cam[2];
    const double w = p.q[0], x = p.q[1], y = p.q[2], z = p.q[3];
    const double R[3][3] = {{1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)},
                            {2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)},
                            {2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)}};
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) { p.R[a][b] = R[a][b]; p.M[a][b] = R[a][b] * p.s[b]; }
    const double lim_x = 1.3 * v.img[0] / (2 * v.focal[0]);
    const double lim_y = 1.3 * v.img[1] / (2 * v.focal[1]);
    const double u0 = p.cam[0] * p.iz, v0 = p.cam[1] * p.iz;
    p.u_clamp = (u0 < -lim_x) || (u0 > lim_x);
    p.v_clamp = (v0 < -lim_y) || (v0 > lim_y);
    p.u = std::min(std::max(u0, -lim_x), lim_x);
    p.v = std::min(std::max(v0, -lim_y), lim_y);
    for (int j = 0; j < 3; ++j) {
        p.t0[j] = v.focal[0] * p.iz * (v.rot[0][j] - p.u * v.rot[2][j]);
        p.t1[j] = v.focal[1] * p.iz * (v.rot[1][j] - p.v * v.rot[2][j]);
    }
    for (int j = 0; j < 3; ++j) {
        p.j0[j] = p.t0[0] * p.M[0][j] + p.t0[1] * p.M[1][j] + p.t0[2] * p.M[2][j];
        p.j1[j] = p.t1[0] * p.M[0][j] + p.t1[1] * p.M[1][j] + p.t1[2] * p.M[2][j];
    }
    auto dot = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
    p.cov[0] = dot(p.j0, p.j0) + 0.3;
    p.cov[1] = dot(p.j0, p.j1);
    p.cov[2] = dot(p.j1, p.j1) + 0.3;
    const double det = p.cov[0] * p.cov[2] - p.cov[1] * p.cov[1];
    p.det_floor = !(det >= 1e-6);
    p.D = p.det_floor ? 1e-6 : det;
    p.conic[0] = p.cov[2] / p.D;
    p.conic[1] = -p.cov[1] / p.D;
    p.conic[2] = p.cov[0] / p.D;
    double dv[3] = {p.mean[0] - v.world_pos[0], p.mean[1] - v.world_pos[1],
                    p.mean[2] - v.world_pos[2]};
    p.vlen = std::sqrt(dot(dv, dv));
    for (int j = 0; j < 3; ++j) p.dir[j] = dv[j] / p.vlen;
    sh_basis(K, p.dir, p.B, p.dB);
    for (int c = 0; c < 3; ++c) {
        double acc = 0;
        for (uint32_t k = 0; k < K; ++k) acc += p.B[k] * sh[((size_t)k * 3 + c) * N + i];
        p.color[c] = acc + 0.5;
    }
    p.m2[0] = v.focal[0] * p.cam[0] * p.iz + v.img[0] * 0.5;
    p.m2[1] = v.focal[1] * p.cam[1] * p.iz + v.img[1] * 0.5;
    const double cutoff = std::log(p.op / kAlphaCutoff);
    const double ex = std::sqrt(2 * cutoff * p.cov[0]), ey = std::sqrt(2 * cutoff * p.cov[2]);
    auto clampu = [](double val, double hi) -> uint32_t {
        if (!(val > 0)) return 0;
        if (val > hi) val = hi;
        return (uint32_t)val;
    };
    const uint32_t min_x = clampu((p.m2[0] - ex) / 16.0, v.tiles_x);
    const uint32_t min_y = clampu((p.m2[1] - ey) / 16.0, v.tiles_y);
    const uint32_t max_x = clampu((p.m2[0] + ex) / 16.0 + 1.0, v.tiles_x);
    const uint32_t max_y = clampu((p.m2[1] + ey) / 16.0 + 1.0, v.tiles_y);
    p.bb[0] = min_x | (min_y << 16);
    p.bb[1] = max_x | (max_y << 16);
}

struct Binned {
    std::vector<Proj> proj;
    std::vector<std::vector<uint32_t>> tiles;  // per tile: splat ids, depth order
};

void bin64(const View64& v, const double* attr, const double* sh, uint32_t n, uint32_t K,
           Binned& out) {
    out.proj.assign(n, Proj());
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) project64(v, attr, sh, n, K, (uint32_t)i, out.proj[i]);
    std::vector<uint32_t> order;
    for (uint32_t i = 0; i < n; ++i)
        if (out.proj[i].vis) order.push_back(i);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        return out.proj[a].cam[2] < out.proj[b].cam[2];
    });
    out.tiles.assign((size_t)v.tiles_x * v.tiles_y, {});
    for (uint32_t id : order) {
        const Proj& p = out.proj[id];
        for (uint32_t ty = p.bb[0] >> 16; ty < (p.bb[1] >> 16); ++ty)
            for (uint32_t tx = p.bb[0] & 0xffff; tx < (p.bb[1] & 0xffff); ++tx)
                out.tiles[(size_t)ty * v.tiles_x + tx].push_back(id);
    }
}

struct Contrib { uint32_t id; double alpha, T, G; bool clamped; };

// One pixel's front-to-back walk; returns the final transmittance.
double walk_pixel(const Binned& bn, const std::vector<uint32_t>& list, double px, double py,
                  std::vector<Contrib>* contribs, double rgb[3]) {
    double T = 1.0;
    rgb[0] = rgb[1] = rgb[2] = 0;
    for (uint32_t id : list) {
        const Proj& p = bn.proj[id];
        const double dx = p.m2[0] - px, dy = p.m2[1] - py;
        const double power = 0.5 * (p.conic[0] * dx * dx + p.conic[2] * dy * dy) + p.conic[1] * dx * dy;
        const double G = std::exp(-power);
        const double raw = p.op * G;
        const bool clamped = raw > 0.999;
        const double alpha = clamped ? 0.999 : raw;
        if (!(alpha >= 1.0 / 255.0)) continue;
        const double vis = alpha * T;
        for (int c = 0; c < 3; ++c) rgb[c] += p.color[c] * vis;
        if (contribs) contribs->push_back({id, alpha, T, G, clamped});
        T *= 1.0 - alpha;
        if (T < 1.0 / 255.0) break;
    }
    return T;
}

}  // namespace

extern "C" int sfo64_render(const sfo_camera* cam, uint32_t w, uint32_t h, const double* attributes,
                            const double* sh, uint32_t n, uint32_t sh_per_ch, double* rgba) {
    const View64 v = make_view(cam, w, h);
    Binned bn;
    bin64(v, attributes, sh, n, sh_per_ch, bn);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t pix = 0; pix < (int64_t)w * h; ++pix) {
        const uint32_t px = (uint32_t)(pix % w), py = (uint32_t)(pix / w);
        const auto& list = bn.tiles[(size_t)(py / 16) * v.tiles_x + px / 16];
        double rgb[3];
        const double T = walk_pixel(bn, list, px + 0.5, py + 0.5, nullptr, rgb);
        for (int c = 0; c < 3; ++c) rgba[4 * pix + c] = rgb[c];
        rgba[4 * pix + 3] = 1.0 - T;
    }
    return 0;
}

extern "C" int sfo64_render_backward(const sfo_camera* cam, uint32_t w, uint32_t h,
                                     const double* attributes, const double* sh, uint32_t n,
                                     uint32_t K, const double* dl_drgba, double* d_attr,
                                     double* d_sh) {
    const View64 v = make_view(cam, w, h);
    Binned bn;
    bin64(v, attributes, sh, n, K, bn);
    // Per-splat 2D adjoints: mean2d (2), conic (3), colour (3), opacity (1).
    const int nthreads = omp_get_max_threads();
    std::vector<double> acc((size_t)nthreads * n * 9, 0.0);
#pragma omp parallel num_threads(nthreads)
    {
        double* my = acc.data() + (size_t)omp_get_thread_num() * n * 9;
        std::vector<Contrib> cs;
#pragma omp for schedule(dynamic, 16)
        for (int64_t pix = 0; pix < (int64_t)w * h; ++pix) {
            const uint32_t px = (uint32_t)(pix % w), py = (uint32_t)(pix / w);
            const auto& list = bn.tiles[(size_t)(py / 16) * v.tiles_x + px / 16];
            cs.clear();
            double rgb[3];
            const double pxc = px + 0.5, pyc = py + 0.5;
            const double t_final = walk_pixel(bn, list, pxc, pyc, &cs, rgb);
            const double* g = dl_drgba + 4 * pix;
            double S[3] = {0, 0, 0};  // colour behind, normalised by T_{k+1}
            for (int64_t k = (int64_t)cs.size() - 1; k >= 0; --k) {
                const Contrib& c = cs[k];
                const Proj& p = bn.proj[c.id];
                double* a = my + (size_t)c.id * 9;
                // alpha channel a = 1 - T_final: d a / d alpha_k = T_final / (1 - alpha_k)
                double dalpha = g[3] * t_final / (1.0 - c.alpha);
                for (int ch = 0; ch < 3; ++ch) {
                    a[5 + ch] += g[ch] * c.alpha * c.T;
                    dalpha += g[ch] * c.T * (p.color[ch] - S[ch]);
                }
                for (int ch = 0; ch < 3; ++ch) S[ch] = c.alpha * p.color[ch] + (1 - c.alpha) * S[ch];
                if (c.clamped) continue;
                a[8] += dalpha * c.G;                // d op
                const double dpower = -dalpha * c.alpha;
                const double dx = p.m2[0] - pxc, dy = p.m2[1] - pyc;
                a[2] += dpower * 0.5 * dx * dx;      // d conic.x
                a[3] += dpower * dx * dy;            // d conic.y
                a[4] += dpower * 0.5 * dy * dy;      // d conic.z
                a[0] += dpower * (p.conic[0] * dx + p.conic[1] * dy);
                a[1] += dpower * (p.conic[2] * dy + p.conic[1] * dx);
            }
        }
    }
    std::memset(d_attr, 0, sizeof(double) * 11 * n);
    std::memset(d_sh, 0, sizeof(double) * 3 * K * n);
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        const uint32_t i = (uint32_t)ii;
        const Proj& p = bn.proj[i];
        if (!p.vis) continue;
        double g[9] = {0};
        for (int t = 0; t < nthreads; ++t)
            for (int k = 0; k < 9; ++k) g[k] += acc[((size_t)t * n + i) * 9 + k];
        const size_t N = n;
        // opacity logit
        d_attr[10 * N + i] = g[8] * p.op * (1 - p.op);
        // SH coefficients and the view direction
        double ddir[3] = {0, 0, 0};
        for (uint32_t k = 0; k < K; ++k) {
            double wsum = 0;
            for (int c = 0; c < 3; ++c) {
                d_sh[((size_t)k * 3 + c) * N + i] = g[5 + c] * p.B[k];
                wsum += g[5 + c] * sh[((size_t)k * 3 + c) * N + i];
            }
            for (int j = 0; j < 3; ++j) ddir[j] += wsum * p.dB[k][j];
        }
        double dmean[3];
        const double dd = ddir[0] * p.dir[0] + ddir[1] * p.dir[1] + ddir[2] * p.dir[2];
        for (int j = 0; j < 3; ++j) dmean[j] = (ddir[j] - p.dir[j] * dd) / p.vlen;
        // conic -> cov
        double dcov[3];
        {
            const double a = p.cov[0], b = p.cov[1], c = p.cov[2], D = p.D;
            const double gx = g[2], gy = g[3], gz = g[4];
            if (p.det_floor) {
                dcov[0] = gz / D; dcov[1] = -gy / D; dcov[2] = gx / D;
            } else {
                const double D2 = D * D;
                dcov[0] = gx * (-c * c / D2) + gy * (b * c / D2) + gz * (1 / D - a * c / D2);
                dcov[1] = gx * (2 * b * c / D2) + gy * (-1 / D - 2 * b * b / D2) + gz * (2 * a * b / D2);
                dcov[2] = gx * (1 / D - a * c / D2) + gy * (a * b / D2) + gz * (-a * a / D2);
            }
        }
        double dj0[3], dj1[3];
        for (int j = 0; j < 3; ++j) {
            dj0[j] = 2 * dcov[0] * p.j0[j] + dcov[1] * p.j1[j];
            dj1[j] = dcov[1] * p.j0[j] + 2 * dcov[2] * p.j1[j];
        }
        // j = M^T t  ->  dt = M dj, dM[k][j] = t_k dj_j
        double dt0[3], dt1[3], dM[3][3];
        for (int k = 0; k < 3; ++k) {
            dt0[k] = p.M[k][0] * dj0[0] + p.M[k][1] * dj0[1] + p.M[k][2] * dj0[2];
            dt1[k] = p.M[k][0] * dj1[0] + p.M[k][1] * dj1[1] + p.M[k][2] * dj1[2];
            for (int j = 0; j < 3; ++j) dM[k][j] = p.t0[k] * dj0[j] + p.t1[k] * dj1[j];
        }
        // M = R diag(s)
        double dR[3][3], ds[3] = {0, 0, 0};
        for (int k = 0; k < 3; ++k)
            for (int j = 0; j < 3; ++j) {
                dR[k][j] = dM[k][j] * p.s[j];
                ds[j] += dM[k][j] * p.R[k][j];
            }
        for (int j = 0; j < 3; ++j) d_attr[(7 + j) * N + i] = ds[j] * p.s[j];
        {
            const double w = p.q[0], x = p.q[1], y = p.q[2], z = p.q[3];
            const double dRw[3][3] = {{0, -2 * z, 2 * y}, {2 * z, 0, -2 * x}, {-2 * y, 2 * x, 0}};
            const double dRx[3][3] = {{0, 2 * y, 2 * z}, {2 * y, -4 * x, -2 * w}, {2 * z, 2 * w, -4 * x}};
            const double dRy[3][3] = {{-4 * y, 2 * x, 2 * w}, {2 * x, 0, 2 * z}, {-2 * w, 2 * z, -4 * y}};
            const double dRz[3][3] = {{-4 * z, -2 * w, 2 * x}, {2 * w, -4 * z, 2 * y}, {2 * x, 2 * y, 0}};
            double dq[4] = {0, 0, 0, 0};
            for (int k = 0; k < 3; ++k)
                for (int j = 0; j < 3; ++j) {
                    dq[0] += dR[k][j] * dRw[k][j];
                    dq[1] += dR[k][j] * dRx[k][j];
                    dq[2] += dR[k][j] * dRy[k][j];
                    dq[3] += dR[k][j] * dRz[k][j];
                }
            for (int j = 0; j < 4; ++j) d_attr[(3 + j) * N + i] = dq[j];
        }
        // t0 = fx*iz*(rot0 - u rot2), t1 = fy*iz*(rot1 - v rot2)
        double dcam[3] = {0, 0, 0};
        {
            const double fx = v.focal[0], fy = v.focal[1], iz = p.iz;
            double du = 0, dvv = 0, diz = 0;
            for (int j = 0; j < 3; ++j) {
                du += dt0[j] * (-fx * iz * v.rot[2][j]);
                dvv += dt1[j] * (-fy * iz * v.rot[2][j]);
                diz += dt0[j] * fx * (v.rot[0][j] - p.u * v.rot[2][j]) +
                       dt1[j] * fy * (v.rot[1][j] - p.v * v.rot[2][j]);
            }
            if (!p.u_clamp) { dcam[0] += du * iz; diz += du * p.cam[0]; }
            if (!p.v_clamp) { dcam[1] += dvv * iz; diz += dvv * p.cam[1]; }
            // mean2d
            dcam[0] += g[0] * fx * iz;
            dcam[1] += g[1] * fy * iz;
            diz += g[0] * fx * p.cam[0] + g[1] * fy * p.cam[1];
            dcam[2] += diz * (-iz * iz);
        }
        for (int j = 0; j < 3; ++j)
            dmean[j] += v.rot[0][j] * dcam[0] + v.rot[1][j] * dcam[1] + v.rot[2][j] * dcam[2];
        for (int j = 0; j < 3; ++j) d_attr[j * N + i] = dmean[j];
    }
    return 0;
}

// ---- FP64 L2 loss over a tile region, for central differences on large
// scenes (TEST INFRASTRUCTURE). The splat set is projected once
// (sfo64_probe_open). sfo64_probe_loss re-projects only the probed splat with
// one parameter replaced, lists the splats whose tile box meets the region
// in the forward's order (visible splats stably sorted by camera depth, as
// bin64), and sums (rgba - target)^2 over the region's pixels. A splat only
// reaches the pixels of its own tile box, so for a region holding the probed
// splat's boxes at both ends of a difference, L(+h) - L(-h) over the region
// equals that of the whole image.
namespace {
struct ProbeSession {
    View64 v;
    uint32_t w = 0, h = 0, n = 0, K = 1;
    std::vector<double> attr, sh;
    std::vector<double> target;  // [h][w][4]
    std::vector<Proj> proj;
};
}  // namespace

extern "C" void* sfo64_probe_open(const sfo_camera* cam, uint32_t w, uint32_t h, const double* attributes,
                                  const double* sh, uint32_t n, uint32_t K, const double* target_rgba) {
    auto* s = new ProbeSession();
    s->v = make_view(cam, w, h);
    s->w = w; s->h = h; s->n = n; s->K = K;
    s->attr.assign(attributes, attributes + (size_t)11 * n);
    s->sh.assign(sh, sh + (size_t)3 * K * n);
    s->target.assign(target_rgba, target_rgba + (size_t)4 * w * h);
    s->proj.assign(n, Proj());
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i)
        project64(s->v, s->attr.data(), s->sh.data(), n, K, (uint32_t)i, s->proj[i]);
    return s;
}

extern "C" void sfo64_probe_close(void* handle) { delete static_cast<ProbeSession*>(handle); }

// Whether splat i is visible and its packed tile box (min, max) at the base
// parameters.
extern "C" int sfo64_probe_bbox(void* handle, uint32_t i, uint32_t out[2]) {
    const auto* s = static_cast<ProbeSession*>(handle);
    const Proj& p = s->proj[i];
    out[0] = p.vis ? p.bb[0] : 0;
    out[1] = p.vis ? p.bb[1] : 0;
    return p.vis ? 1 : 0;
}

// param < 11: attribute plane `param` of splat i; otherwise SH coefficient
// (param - 11) = k * 3 + c. Region: tiles [tx0, tx1) x [ty0, ty1).
extern "C" double sfo64_probe_loss(void* handle, uint32_t i, uint32_t param, double value, uint32_t tx0,
                                   uint32_t ty0, uint32_t tx1, uint32_t ty1) {
    auto* s = static_cast<ProbeSession*>(handle);
    const size_t N = s->n;
    double* slot = param < 11 ? &s->attr[(size_t)param * N + i] : &s->sh[(size_t)(param - 11) * N + i];
    const double keep = *slot;
    *slot = value;
    Proj local;
    project64(s->v, s->attr.data(), s->sh.data(), s->n, s->K, i, local);
    *slot = keep;
    auto P = [&](uint32_t id) -> const Proj& { return id == i ? local : s->proj[id]; };
    std::vector<uint32_t> ids;
    for (uint32_t id = 0; id < s->n; ++id) {
        const Proj& p = P(id);
        if (!p.vis) continue;
        const uint32_t bx0 = p.bb[0] & 0xffff, by0 = p.bb[0] >> 16, bx1 = p.bb[1] & 0xffff, by1 = p.bb[1] >> 16;
        if (bx0 < tx1 && bx1 > tx0 && by0 < ty1 && by1 > ty0) ids.push_back(id);
    }
    std::stable_sort(ids.begin(), ids.end(), [&](uint32_t a, uint32_t b) { return P(a).cam[2] < P(b).cam[2]; });
    Binned bn;
    bn.proj.reserve(ids.size());
    for (uint32_t id : ids) bn.proj.push_back(P(id));
    const uint32_t rw = tx1 - tx0, rh = ty1 - ty0;
    bn.tiles.assign((size_t)rw * rh, {});
    for (uint32_t k = 0; k < ids.size(); ++k) {
        const Proj& p = bn.proj[k];
        const uint32_t bx0 = std::max(p.bb[0] & 0xffff, tx0), by0 = std::max(p.bb[0] >> 16, ty0);
        const uint32_t bx1 = std::min(p.bb[1] & 0xffff, tx1), by1 = std::min(p.bb[1] >> 16, ty1);
        for (uint32_t ty = by0; ty < by1; ++ty)
            for (uint32_t tx = bx0; tx < bx1; ++tx) bn.tiles[(size_t)(ty - ty0) * rw + (tx - tx0)].push_back(k);
    }
    double loss = 0.0;
    const int64_t pixels = (int64_t)rw * 16 * rh * 16;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : loss)
    for (int64_t q = 0; q < pixels; ++q) {
        const uint32_t px = tx0 * 16 + (uint32_t)(q % (rw * 16)), py = ty0 * 16 + (uint32_t)(q / (rw * 16));
        if (px >= s->w || py >= s->h) continue;
        const auto& list = bn.tiles[(size_t)(py / 16 - ty0) * rw + (px / 16 - tx0)];
        double rgb[3];
        const double T = walk_pixel(bn, list, px + 0.5, py + 0.5, nullptr, rgb);
        const double* t = &s->target[4 * ((size_t)py * s->w + px)];
        const double d[4] = {rgb[0] - t[0], rgb[1] - t[1], rgb[2] - t[2], (1.0 - T) - t[3]};
        loss += d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + d[3] * d[3];
    }
    return loss;
}
