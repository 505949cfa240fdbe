// Adjoint of the splat render (no counterpart in the reference, which has no
// backward pass): dL/d(means, log-scales, quaternions, opacity logits, SH)
// for L = sum_p <dL/d rgba_p, rgba_p>.
//
// raster_bwd_kernel replays each pixel's contributors back to front from the
// forward's stored final transmittance and last-contributor index,
// recomputing alpha with the forward's exact arithmetic (so the contributor
// set is the forward's) and the transmittance before each contributor as
// T_k = T_{k+1} / (1 - alpha_k). Per pixel and contributor k:
//   dL/dc_k     = g_rgb * alpha_k T_k
//   dL/dalpha_k = T_k <g_rgb, c_k - S_k> + g_a T_final / (1 - alpha_k),
// with S_k the colour behind k normalised by T_{k+1}
// (S_{k-1} = alpha_k c_k + (1 - alpha_k) S_k); alpha = min(op e^-power, 0.999)
// passes the gradient only where the clamp does not bind. The nine per-splat
// 2D adjoints (mean2d xy, conic xyz, colour rgb, opacity) are reduced per
// warp, per tile in shared memory, and added to global memory once per
// (tile, splat).
// project_bwd_kernel recomputes each splat's projection (src/project.rs:
// 176-327) and applies the chain rule through conic -> cov2d (det floor,
// +0.3 dilation), the Jacobian with its 1.3x FOV clamp, R(q) diag(exp s),
// sigmoid opacity and the SH basis (src/project.rs:344-388) to the view
// direction.
#include <cstdint>
#include "sf_internal.h"
#include "sf_math.cuh"

namespace sfk {

namespace {

using namespace sfm;

constexpr float kAlphaCutoff = 10.0f / 255.0f;
constexpr float C0 = 0.2820948f, C1 = 0.48860252f, C20 = 0.9461747f, C21 = 0.31539157f,
                C22 = -1.0925485f, C23 = 0.54627424f;
constexpr float K3 = -0.5900436f, A3 = -2.285229f, B3 = 0.4570458f, E3 = 1.8658817f,
                F3 = 1.119529f, G3 = 1.4453057f;

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ __launch_bounds__(256) void raster_bwd_kernel(BwdArgs a) {
    __shared__ float4 s_g0[256];
    __shared__ float4 s_g1[256];
    __shared__ float4 s_col[256];
    __shared__ uint32_t s_gid[256];
    __shared__ float s_grad[9][256];
    __shared__ uint32_t s_max_last;

    const uint32_t tile = blockIdx.x;
    const uint32_t tx = tile % a.tiles_x, ty = tile / a.tiles_x;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint32_t px = tx * 16 + (warp & 1u) * 8 + (lane & 7u);
    const uint32_t py = ty * 16 + (warp >> 1) * 4 + (lane >> 3);
    const bool in_bounds = px < a.w && py < a.h;
    const uint32_t start = a.tile_start[tile];
    const float fx = (float)px + 0.5f, fy = (float)py + 0.5f;
    float T = 1.0f, t_final = 1.0f;
    uint32_t last = 0;
    float4 g = make_float4(0.f, 0.f, 0.f, 0.f);
    if (in_bounds) {
        const size_t pix = (size_t)py * a.w + px;
        T = t_final = a.final_t[pix];
        last = a.n_contrib[pix];
        g = a.dl[pix];
    }
    if (tid == 0) s_max_last = 0;
    for (int k = 0; k < 9; ++k) s_grad[k][tid] = 0.0f;
    __syncthreads();
    const uint32_t wmax = __reduce_max_sync(0xffffffffu, last);
    if (lane == 0) atomicMax(&s_max_last, wmax);
    __syncthreads();
    const uint32_t max_last = s_max_last;
    float Sr = 0.f, Sg = 0.f, Sb = 0.f;
    const float inv255 = 1.0f / 255.0f;

    for (int64_t c0 = (int64_t)((max_last + 255u) / 256u) * 256 - 256; c0 >= 0; c0 -= 256) {
        __syncthreads();
        const uint32_t e_stage = (uint32_t)c0 + tid;
        if (e_stage < max_last) {
            const uint32_t gid = a.gaussian_ids[start + e_stage];
            s_gid[tid] = gid;
            s_g0[tid] = a.geo0[gid];
            s_g1[tid] = a.geo1[gid];
            s_col[tid] = a.color[gid];
        }
        __syncthreads();
        const uint32_t cnt = min(256u, max_last - (uint32_t)c0);
        for (int j = (int)cnt - 1; j >= 0; --j) {
            const uint32_t e = (uint32_t)c0 + (uint32_t)j;
            float d[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            bool hit = false;
            if (e < last) {
                const float4 g0 = s_g0[j];
                const float4 g1 = s_g1[j];
                const float dx = g0.x - fx, dy = g0.y - fy;
                const float power = fma_(g0.z * dx, dx, fma_(g1.x * dy, dy, (g0.w * dx) * dy));
                if (!(power > g1.z)) {
                    const float G = exp_neg_(-power);
                    const float raw = g1.y * G;
                    const float alpha = fminf(raw, 0.999f);
                    if (alpha >= inv255) {
                        hit = true;
                        const float4 c = s_col[j];
                        const float inv = 1.0f / (1.0f - alpha);
                        const float Tk = T * inv;
                        float dalpha = g.w * t_final * inv;
                        dalpha += Tk * ((g.x * (c.x - Sr) + g.y * (c.y - Sg)) + g.z * (c.z - Sb));
                        const float w = alpha * Tk;
                        d[5] = g.x * w;
                        d[6] = g.y * w;
                        d[7] = g.z * w;
                        Sr = alpha * c.x + (1.0f - alpha) * Sr;
                        Sg = alpha * c.y + (1.0f - alpha) * Sg;
                        Sb = alpha * c.z + (1.0f - alpha) * Sb;
                        T = Tk;
                        if (raw <= 0.999f) {
                            d[8] = dalpha * G;
                            const float dp = -dalpha * alpha;
                            d[2] = dp * 0.5f * dx * dx;
                            d[3] = dp * dx * dy;
                            d[4] = dp * 0.5f * dy * dy;
                            d[0] = dp * (2.0f * g0.z * dx + g0.w * dy);
                            d[1] = dp * (2.0f * g1.x * dy + g0.w * dx);
                        }
                    }
                }
            }
            if (__any_sync(0xffffffffu, hit)) {
#pragma unroll
                for (int k = 0; k < 9; ++k) {
                    const float s = warp_sum(d[k]);
                    if (lane == 0 && s != 0.0f) atomicAdd(&s_grad[k][j], s);
                }
            }
        }
        __syncthreads();
        if (tid < cnt) {
            float* dst = a.d2d + (size_t)s_gid[tid] * 9;
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                const float v = s_grad[k][tid];
                if (v != 0.0f) atomicAdd(dst + k, v);
                s_grad[k][tid] = 0.0f;
            }
        }
    }
}

// Adjoint of a per-splat scalar feature f: the render F(p) = sum_k f_k
// alpha_k T_k over pixel p's contributors has dF(p)/df_k = alpha_k T_k, so
// for L = sum_p w(p) F(p) the feature gradient is dL/df_i = sum_p w(p)
// alpha_i T_i(p): splat i's responsibility weighted by w. Two weights at
// once, w_fg = mask(p) and w_bg = 1 - mask(p) (all ones without a mask),
// give the real-valued fg / bg responsibilities that the u32 evidence lift
// truncates per pixel. The walk is the adjoint replay of raster_bwd_kernel
// (back to front from the forward's final T and last contributor, T_k =
// T_{k+1} / (1 - alpha_k)), with nothing but the two feature sums; the
// forward state comes from the transmittance-only raster mode. Float sums
// are reduced per warp, per tile in shared memory, then added to global
// memory once per (tile, splat); their order of addition is not fixed.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Chunks of 256 entries walked from the last down to the first; the records
// of chunk c - 1 are copied (cp.async, double-buffered) while chunk c is
// replayed, and the ids of chunk c - 2 are loaded a chunk ahead.
__global__ __launch_bounds__(256) void feature_bwd_kernel(FeatureBwdArgs a) {
    __shared__ float4 s_g0[2][256];
    __shared__ float4 s_g1[2][256];
    __shared__ uint32_t s_gid[2][256];
    __shared__ float s_fg[2][256];
    __shared__ float s_bg[2][256];
    __shared__ uint32_t s_max_last;

    const uint32_t tile = blockIdx.x;
    const uint32_t tx = tile % a.tiles_x, ty = tile / a.tiles_x;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint32_t px = tx * 16 + (warp & 1u) * 8 + (lane & 7u);
    const uint32_t py = ty * 16 + (warp >> 1) * 4 + (lane >> 3);
    const bool in_bounds = px < a.w && py < a.h;
    const uint32_t start = a.tile_start[tile];
    const float fx = (float)px + 0.5f, fy = (float)py + 0.5f;
    float T = 1.0f;
    uint32_t last = 0;
    float wf = 0.0f, wb = 0.0f;
    if (in_bounds) {
        const size_t pix = (size_t)py * a.w + px;
        T = a.final_t[pix];
        last = a.n_contrib[pix];
        const bool inside = a.mask ? ((a.mask[px / 32 + py * a.mask_wpr] >> (px % 32)) & 1u) != 0u : true;
        wf = inside ? 1.0f : 0.0f;
        wb = 1.0f - wf;
    }
    if (tid == 0) s_max_last = 0;
    s_fg[0][tid] = s_fg[1][tid] = 0.0f;
    s_bg[0][tid] = s_bg[1][tid] = 0.0f;
    __syncthreads();
    const uint32_t wmax = __reduce_max_sync(0xffffffffu, last);
    if (lane == 0) atomicMax(&s_max_last, wmax);
    __syncthreads();
    const uint32_t max_last = s_max_last;
    const uint32_t nch = (max_last + 255u) / 256u;
    if (nch == 0) return;
    const float inv255 = 1.0f / 255.0f;
    uint32_t g_next = 0;
    auto load_id = [&](uint32_t c) {
        const uint32_t e = c * 256u + tid;
        g_next = e < max_last ? a.gaussian_ids[start + e] : 0u;
    };
    auto issue = [&](uint32_t c, uint32_t b) {
        if (c * 256u + tid < max_last) {
            cp_async16(&s_g0[b][tid], a.geo0 + g_next);
            cp_async16(&s_g1[b][tid], a.geo1 + g_next);
            s_gid[b][tid] = g_next;
        }
    };
    auto flush = [&](uint32_t b, uint32_t cnt) {
        if (tid < cnt) {
            const uint32_t g = s_gid[b][tid];
            const float f = s_fg[b][tid], bb = s_bg[b][tid];
            if (f != 0.0f) atomicAdd(a.fg + g, f);
            if (bb != 0.0f) atomicAdd(a.bg + g, bb);
            s_fg[b][tid] = 0.0f;
            s_bg[b][tid] = 0.0f;
        }
    };
    load_id(nch - 1);
    issue(nch - 1, 0);
    cp_async_commit();
    if (nch > 1) load_id(nch - 2);
    for (uint32_t k = 0; k < nch; ++k) {
        const uint32_t ci = nch - 1 - k, b = k & 1u;
        // The replay of chunk ci + 1 is over: its buffer may be refilled
        // and its sums are complete.
        __syncthreads();
        if (k > 0) flush(b ^ 1u, min(256u, max_last - (ci + 1) * 256u));
        if (ci > 0) {
            issue(ci - 1, b ^ 1u);
            if (ci > 1) load_id(ci - 2);
        }
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const uint32_t c0 = ci * 256u;
        const uint32_t cnt = min(256u, max_last - c0);
        for (int j = (int)cnt - 1; j >= 0; --j) {
            const uint32_t e = c0 + (uint32_t)j;
            float w = 0.0f;
            if (e < last) {
                const float4 g0 = s_g0[b][j];
                const float4 g1 = s_g1[b][j];
                const float dx = g0.x - fx, dy = g0.y - fy;
                const float power = fma_(g0.z * dx, dx, fma_(g1.x * dy, dy, (g0.w * dx) * dy));
                if (!(power > g1.z)) {
                    const float alpha = fminf(g1.y * exp_neg_(-power), 0.999f);
                    if (alpha >= inv255) {
                        const float Tk = T / (1.0f - alpha);
                        w = alpha * Tk;
                        T = Tk;
                    }
                }
            }
            if (__any_sync(0xffffffffu, w != 0.0f)) {
                const float sf = warp_sum(wf * w);
                const float sb = warp_sum(wb * w);
                if (lane == 0) {
                    if (sf != 0.0f) atomicAdd(&s_fg[b][j], sf);
                    if (sb != 0.0f) atomicAdd(&s_bg[b][j], sb);
                }
            }
        }
    }
    __syncthreads();
    flush((nch - 1) & 1u, min(256u, max_last));
}

struct V3 { float x, y, z; };
__device__ __forceinline__ float dot3(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

template <int K>
__global__ __launch_bounds__(256) void project_bwd_kernel(sf_view v, const float* __restrict__ attr,
                                                          const float* __restrict__ shs, uint32_t n,
                                                          const float* __restrict__ d2d,
                                                          float* __restrict__ d_attr,
                                                          float* __restrict__ d_sh) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t N = n;
    float a[11];
#pragma unroll
    for (int k = 0; k < 11; ++k) a[k] = __ldg(attr + k * N + i);
    const float opacity = sigmoid_(a[10]);
    const V3 mean{a[0], a[1], a[2]};
    const V3 rot0{v.rot0[0], v.rot0[1], v.rot0[2]};
    const V3 rot1{v.rot1[0], v.rot1[1], v.rot1[2]};
    const V3 rot2{v.rot2[0], v.rot2[1], v.rot2[2]};
    const float cam_z = dot3(rot2, mean) + v.trans[2];
    if (!(opacity >= kAlphaCutoff) || !(cam_z > 0.1f)) {
#pragma unroll
        for (int k = 0; k < 11; ++k) d_attr[k * N + i] = 0.0f;
#pragma unroll
        for (int k = 0; k < 3 * K; ++k) d_sh[k * N + i] = 0.0f;
        return;
    }
    float g[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) g[k] = d2d[(size_t)i * 9 + k];
    const float cam_x = dot3(rot0, mean) + v.trans[0];
    const float cam_y = dot3(rot1, mean) + v.trans[1];
    const float qw = a[3], qx = a[4], qy = a[5], qz = a[6];
    const float s0 = exp_(a[7]), s1 = exp_(a[8]), s2 = exp_(a[9]);
    const float s[3] = {s0, s1, s2};
    const float iz = 1.0f / cam_z;
    const float R[3][3] = {{1.0f - 2.0f * (qy * qy + qz * qz), 2.0f * (qx * qy - qw * qz), 2.0f * (qx * qz + qw * qy)},
                           {2.0f * (qx * qy + qw * qz), 1.0f - 2.0f * (qx * qx + qz * qz), 2.0f * (qy * qz - qw * qx)},
                           {2.0f * (qx * qz - qw * qy), 2.0f * (qy * qz + qw * qx), 1.0f - 2.0f * (qx * qx + qy * qy)}};
    float M[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) M[r][c] = R[r][c] * s[c];
    const float lim_x = (1.3f * v.img[0]) / (2.0f * v.focal[0]);
    const float lim_y = (1.3f * v.img[1]) / (2.0f * v.focal[1]);
    const float u0 = cam_x * iz, v0 = cam_y * iz;
    const bool u_clamp = u0 < -lim_x || u0 > lim_x;
    const bool v_clamp = v0 < -lim_y || v0 > lim_y;
    const float u = clamp_(u0, -lim_x, lim_x), vv = clamp_(v0, -lim_y, lim_y);
    const float rw[3][3] = {{rot0.x, rot0.y, rot0.z}, {rot1.x, rot1.y, rot1.z}, {rot2.x, rot2.y, rot2.z}};
    float t0[3], t1[3], j0[3], j1[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        t0[c] = v.focal[0] * iz * (rw[0][c] - u * rw[2][c]);
        t1[c] = v.focal[1] * iz * (rw[1][c] - vv * rw[2][c]);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        j0[c] = t0[0] * M[0][c] + t0[1] * M[1][c] + t0[2] * M[2][c];
        j1[c] = t1[0] * M[0][c] + t1[1] * M[1][c] + t1[2] * M[2][c];
    }
    const float ca = j0[0] * j0[0] + j0[1] * j0[1] + j0[2] * j0[2] + 0.3f;
    const float cb = j0[0] * j1[0] + j0[1] * j1[1] + j0[2] * j1[2];
    const float cc = j1[0] * j1[0] + j1[1] * j1[1] + j1[2] * j1[2] + 0.3f;
    const float det = ca * cc - cb * cb;
    const bool floor_det = !(det >= 1e-6f);
    const float D = floor_det ? 1e-6f : det;

    // opacity logit
    d_attr[10 * N + i] = g[8] * opacity * (1.0f - opacity);

    // SH coefficients and the view direction
    V3 dv{mean.x - v.world_pos[0], mean.y - v.world_pos[1], mean.z - v.world_pos[2]};
    const float vlen = sqrtf(dot3(dv, dv));
    const float dx = dv.x / vlen, dy = dv.y / vlen, dz = dv.z / vlen;
    float B[16], dB[16][3];
#pragma unroll
    for (int k = 0; k < 16; ++k) { B[k] = 0.f; dB[k][0] = dB[k][1] = dB[k][2] = 0.f; }
    B[0] = C0;
    if (K >= 4) {
        B[1] = -C1 * dy; dB[1][1] = -C1;
        B[2] = C1 * dz;  dB[2][2] = C1;
        B[3] = -C1 * dx; dB[3][0] = -C1;
    }
    if (K >= 9) {
        B[4] = 2.f * C23 * dx * dy; dB[4][0] = 2.f * C23 * dy; dB[4][1] = 2.f * C23 * dx;
        B[5] = C22 * dz * dy;       dB[5][1] = C22 * dz;       dB[5][2] = C22 * dy;
        B[6] = C20 * dz * dz - C21; dB[6][2] = 2.f * C20 * dz;
        B[7] = C22 * dz * dx;       dB[7][0] = C22 * dz;       dB[7][2] = C22 * dx;
        B[8] = C23 * (dx * dx - dy * dy); dB[8][0] = 2.f * C23 * dx; dB[8][1] = -2.f * C23 * dy;
    }
    if (K >= 16) {
        const float c1x = dx * dx - dy * dy, c1y = 2.f * dx * dy, t0c = A3 * dz * dz + B3;
        B[9] = K3 * dx * c1y + dy * c1x;
        dB[9][0] = 4.f * K3 * dx * dy + 2.f * dx * dy;
        dB[9][1] = 2.f * K3 * dx * dx + dx * dx - 3.f * dy * dy;
        B[10] = K3 * dx * c1x - dy * c1y;
        dB[10][0] = 3.f * K3 * dx * dx - K3 * dy * dy - 2.f * dy * dy;
        dB[10][1] = -2.f * K3 * dx * dy - 4.f * dx * dy;
        B[11] = t0c * dy; dB[11][1] = t0c; dB[11][2] = 2.f * A3 * dz * dy;
        B[12] = t0c * dx; dB[12][0] = t0c; dB[12][2] = 2.f * A3 * dz * dx;
        B[13] = dz * (E3 * dz * dz - F3); dB[13][2] = 3.f * E3 * dz * dz - F3;
        B[14] = G3 * dz * c1y; dB[14][0] = 2.f * G3 * dz * dy; dB[14][1] = 2.f * G3 * dz * dx;
        dB[14][2] = G3 * c1y;
        B[15] = G3 * dz * c1x; dB[15][0] = 2.f * G3 * dz * dx; dB[15][1] = -2.f * G3 * dz * dy;
        dB[15][2] = G3 * c1x;
    }
    float ddir[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int k = 0; k < K; ++k) {
        float wsum = 0.f;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            d_sh[(size_t)(k * 3 + c) * N + i] = g[5 + c] * B[k];
            wsum += g[5 + c] * __ldg(shs + (size_t)(k * 3 + c) * N + i);
        }
        ddir[0] += wsum * dB[k][0];
        ddir[1] += wsum * dB[k][1];
        ddir[2] += wsum * dB[k][2];
    }
    const float dd = ddir[0] * dx + ddir[1] * dy + ddir[2] * dz;
    float dmean[3] = {(ddir[0] - dx * dd) / vlen, (ddir[1] - dy * dd) / vlen, (ddir[2] - dz * dd) / vlen};

    // conic -> cov2d
    float dcov0, dcov1, dcov2;
    {
        const float gx = g[2], gy = g[3], gz = g[4];
        if (floor_det) {
            dcov0 = gz / D; dcov1 = -gy / D; dcov2 = gx / D;
        } else {
            const float D2 = D * D;
            dcov0 = gx * (-cc * cc / D2) + gy * (cb * cc / D2) + gz * (1.0f / D - ca * cc / D2);
            dcov1 = gx * (2.f * cb * cc / D2) + gy * (-1.0f / D - 2.f * cb * cb / D2) + gz * (2.f * ca * cb / D2);
            dcov2 = gx * (1.0f / D - ca * cc / D2) + gy * (ca * cb / D2) + gz * (-ca * ca / D2);
        }
    }
    float dj0[3], dj1[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        dj0[c] = 2.f * dcov0 * j0[c] + dcov1 * j1[c];
        dj1[c] = dcov1 * j0[c] + 2.f * dcov2 * j1[c];
    }
    float dt0[3], dt1[3], dR[3][3], ds[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        dt0[r] = M[r][0] * dj0[0] + M[r][1] * dj0[1] + M[r][2] * dj0[2];
        dt1[r] = M[r][0] * dj1[0] + M[r][1] * dj1[1] + M[r][2] * dj1[2];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float dM = t0[r] * dj0[c] + t1[r] * dj1[c];
            dR[r][c] = dM * s[c];
            ds[c] += dM * R[r][c];
        }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) d_attr[(7 + c) * N + i] = ds[c] * s[c];
    {
        const float w = qw, x = qx, y = qy, z = qz;
        const float dRw[3][3] = {{0.f, -2.f * z, 2.f * y}, {2.f * z, 0.f, -2.f * x}, {-2.f * y, 2.f * x, 0.f}};
        const float dRx[3][3] = {{0.f, 2.f * y, 2.f * z}, {2.f * y, -4.f * x, -2.f * w}, {2.f * z, 2.f * w, -4.f * x}};
        const float dRy[3][3] = {{-4.f * y, 2.f * x, 2.f * w}, {2.f * x, 0.f, 2.f * z}, {-2.f * w, 2.f * z, -4.f * y}};
        const float dRz[3][3] = {{-4.f * z, -2.f * w, 2.f * x}, {2.f * w, -4.f * z, 2.f * y}, {2.f * x, 2.f * y, 0.f}};
        float dq[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                dq[0] += dR[r][c] * dRw[r][c];
                dq[1] += dR[r][c] * dRx[r][c];
                dq[2] += dR[r][c] * dRy[r][c];
                dq[3] += dR[r][c] * dRz[r][c];
            }
#pragma unroll
        for (int k = 0; k < 4; ++k) d_attr[(3 + k) * N + i] = dq[k];
    }
    // t0 = fx iz (rot0 - u rot2), t1 = fy iz (rot1 - v rot2); mean2d
    float dcam[3] = {0.f, 0.f, 0.f};
    {
        const float fx = v.focal[0], fy = v.focal[1];
        float du = 0.f, dvv = 0.f, diz = 0.f;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            du += dt0[c] * (-fx * iz * rw[2][c]);
            dvv += dt1[c] * (-fy * iz * rw[2][c]);
            diz += dt0[c] * fx * (rw[0][c] - u * rw[2][c]) + dt1[c] * fy * (rw[1][c] - vv * rw[2][c]);
        }
        if (!u_clamp) { dcam[0] += du * iz; diz += du * cam_x; }
        if (!v_clamp) { dcam[1] += dvv * iz; diz += dvv * cam_y; }
        dcam[0] += g[0] * fx * iz;
        dcam[1] += g[1] * fy * iz;
        diz += g[0] * fx * cam_x + g[1] * fy * cam_y;
        dcam[2] += diz * (-iz * iz);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c)
        d_attr[c * N + i] = dmean[c] + rw[0][c] * dcam[0] + rw[1][c] * dcam[1] + rw[2][c] * dcam[2];
}

}  // namespace

cudaError_t launch_raster_bwd(const BwdArgs& a, cudaStream_t stream) {
    const uint32_t tiles = a.tiles_x * a.tiles_y;
    if (tiles == 0) return cudaSuccess;
    raster_bwd_kernel<<<tiles, 256, 0, stream>>>(a);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_feature_bwd(const FeatureBwdArgs& a, cudaStream_t stream) {
    const uint32_t tiles = a.tiles_x * a.tiles_y;
    if (tiles == 0) return cudaSuccess;
    feature_bwd_kernel<<<tiles, 256, 0, stream>>>(a);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_project_bwd(const sf_view& view, const float* attr, const float* sh, uint32_t n,
                               uint32_t sh_per_ch, const float* d2d, float* d_attr, float* d_sh,
                               cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    const uint32_t grid = (n + 255) / 256;
    // Coefficients past the largest whole SH degree are never read by the
    // forward (the reference's `chs >= 4/9/16` tests): zero gradient.
    const uint32_t used = sh_degree_coeffs(sh_per_ch);
    if (used < sh_per_ch) {
        cudaError_t e = cudaMemsetAsync(d_sh + (size_t)3 * used * n, 0, (size_t)3 * (sh_per_ch - used) * n * 4,
                                        stream);
        if (e != cudaSuccess) return e;
    }
    switch (used) {
        case 1: project_bwd_kernel<1><<<grid, 256, 0, stream>>>(view, attr, sh, n, d2d, d_attr, d_sh); break;
        case 4: project_bwd_kernel<4><<<grid, 256, 0, stream>>>(view, attr, sh, n, d2d, d_attr, d_sh); break;
        case 9: project_bwd_kernel<9><<<grid, 256, 0, stream>>>(view, attr, sh, n, d2d, d_attr, d_sh); break;
        case 16: project_bwd_kernel<16><<<grid, 256, 0, stream>>>(view, attr, sh, n, d2d, d_attr, d_sh); break;
        default: return cudaErrorInvalidValue;
    }
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace sfk
