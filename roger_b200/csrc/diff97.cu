// Differentiable 9/7 path: transposes (adjoints) of the forward and inverse 9/7 DWT, and the
// relaxed dead-zone quantiser with its backward.  No counterpart in the reference.
//
// Adjoint of one lifting step.  A forward step updates the samples of parity p:
//     x_i += c * (x_{m(i-1)} + x_{m(i+1)})          (m = whole-sample symmetric mirror)
// Its transpose updates the other parity q = 1-p with the same coefficient:
//     g_j += c * (s_{j-1} + s_{j+1}),   s_k = g_k, except s_k = 0 outside [0, n) and
//     s_k = 2 g_k for the boundary samples k = 0 and k = n-1 when they have parity p
// (the mirrored references fold back onto them).  Scalings are diagonal (their own transpose).
//   forward level  = deinterleave . S . L3 . L2 . L1 . L0   per axis, columns then rows
//   fwd adjoint    = (per level, deepest first) rows then columns of
//                    L0^T L1^T L2^T L3^T S interleave       -> tile structure of the inverse
//   inverse level  = L0' L1' L2' L3' . S' . interleave       per axis, rows then columns
//   inv adjoint    = (per level, finest first) columns then rows of
//                    deinterleave . S' . L3'^T L2'^T L1'^T L0'^T  -> tile structure of the forward
// Arithmetic is FP32 with separately rounded operations; the checks are against the FP64
// oracle (or_dwt97_*_adj_f64) and against finite differences.
//
// Relaxed quantiser (value domain): t = y/step + u, y_hat = t*step, rate = log2(1+|t|),
// u ~ U[-1/2, 1/2) from Philox4x32-10 keyed by (seed, image) and counted by the sample's
// position in its Mallat plane (the oracle draws the same stream).
#include <cmath>

#include "j2k_internal.cuh"

namespace {

constexpr float P1 = -1.586134342f, U1 = -0.05298011854f, P2 = 0.8829110762f, U2 = 0.4435068522f;
constexpr float KMUL = 1.23017410491400f, KDIV = 0.81289306611596153187273657637352f;
constexpr int TW = 64, TH = 64, HALO = 4, NX = TW + 2 * HALO, NY = TH + 2 * HALO, SS = NX + 1;

// Transposed step sequences (parity updated, coefficient):
//   forward adjoint (after the forward scaling): (odd, U2), (even, P2), (odd, U1), (even, P1)
//   inverse adjoint (before the inverse scaling): (even, -P1), (odd, -U1), (even, -P2), (odd, -U2)

// One transposed step along columns (VERT) or rows of the shared tile: positions along the
// step axis in [LO, HI) (tile coordinates), across it in [OLO, OHI).  Absolute coordinate of
// tile index 0 along the axis: a0; n: line length.  EDGE: the tile touches the image boundary
// along this axis (only then are the zero-extension and boundary doubling applied).
template <bool VERT, bool FWD, int K, int LO, int HI, int OLO, int OHI, bool EDGE>
__device__ __forceinline__ void adj_step(float* s, int a0, int n) {
    constexpr int span = OHI - OLO, cnt = (HI - LO) * span;
    const int par = FWD ? (K == 0 || K == 2 ? 1 : 0) : (K == 0 || K == 2 ? 0 : 1);
    const float c = FWD ? (K == 0 ? U2 : K == 1 ? P2 : K == 2 ? U1 : P1)
                        : (K == 0 ? -P1 : K == 1 ? -U1 : K == 2 ? -P2 : -U2);
    constexpr int st = VERT ? SS : 1;
    const int first = LO + (((a0 + LO) & 1) != par);  // first position of the updated parity
    const int na = first < HI ? (HI - first + 1) / 2 : 0;
    for (int e = threadIdx.x; e < na * span; e += blockDim.x) {
        const int a = first + 2 * (e / span), o = OLO + e % span;
        float* p = s + (VERT ? a * SS + o : o * SS + a);
        float left = p[-st], right = p[st];
        if (EDGE) {
            const int abs_a = a0 + a;
            if (abs_a < 0 || abs_a >= n) continue;
            if (abs_a - 1 < 0) left = 0.0f;
            else if (abs_a - 1 == 0) left *= 2.0f;        // sample 0 has the source parity here
            if (abs_a + 1 >= n) right = 0.0f;
            else if (abs_a + 1 == n - 1) right *= 2.0f;   // so does sample n-1
        }
        *p = __fadd_rn(*p, __fmul_rn(c, __fadd_rn(left, right)));
    }
    (void)cnt;
}

template <bool VERT, bool FWD, int OLO, int OHI, bool EDGE>
__device__ __forceinline__ void adj_steps(float* s, int a0, int n) {
    constexpr int L = VERT ? NY : NX;
    adj_step<VERT, FWD, 0, 1, L - 1, OLO, OHI, EDGE>(s, a0, n);
    __syncthreads();
    adj_step<VERT, FWD, 1, 2, L - 2, OLO, OHI, EDGE>(s, a0, n);
    __syncthreads();
    adj_step<VERT, FWD, 2, 3, L - 3, OLO, OHI, EDGE>(s, a0, n);
    __syncthreads();
    adj_step<VERT, FWD, 3, 4, L - 4, OLO, OHI, EDGE>(s, a0, n);
    __syncthreads();
}

// Adjoint of one forward level: subband gradients (Mallat positions of `gsrc`, LL from `gll`
// with pitch llpitch) -> gradient of the level input (w x h) in `gout`.
__global__ void __launch_bounds__(256)
fwd_adj_level(const float* __restrict__ gsrc, size_t spitch, const float* __restrict__ gll, size_t llpitch,
              int w, int h, float* __restrict__ gout, size_t opitch, size_t zs, size_t zll, size_t zo) {
    __shared__ float s[NY * SS];
    gsrc += blockIdx.z * zs;
    gll += blockIdx.z * zll;
    gout += blockIdx.z * zo;
    const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
    const int ax0 = x0 - HALO, ay0 = y0 - HALO;
    const int wl = (w + 1) >> 1, hl = (h + 1) >> 1;
    for (int e = threadIdx.x; e < NX * NY; e += blockDim.x) {
        const int r = e / NX, c = e % NX;
        const int gy = ay0 + r, gx = ax0 + c;
        float v = 0.0f;
        if (gx >= 0 && gx < w && gy >= 0 && gy < h) {
            const int qx = gx & 1, qy = gy & 1;
            const int sx = (gx >> 1) + (qx ? wl : 0), sy = (gy >> 1) + (qy ? hl : 0);
            v = (!qx && !qy) ? gll[(size_t)(gy >> 1) * llpitch + (gx >> 1)] : gsrc[(size_t)sy * spitch + sx];
        }
        s[r * SS + c] = v;
    }
    __syncthreads();
    const bool edge_x = ax0 <= 0 || ax0 + NX >= w, edge_y = ay0 <= 0 || ay0 + NY >= h;
    // rows (the forward applied them last): scale by the forward factors, then the L^T steps
    if (w > 1) {
        for (int e = threadIdx.x; e < NX * NY; e += blockDim.x) {
            const int r = e / NX, c = e % NX;
            s[r * SS + c] = __fmul_rn(s[r * SS + c], ((ax0 + c) & 1) ? KMUL : KDIV);
        }
        __syncthreads();
        if (edge_x) adj_steps<false, true, 0, NY, true>(s, ax0, w);
        else adj_steps<false, true, 0, NY, false>(s, ax0, w);
    }
    if (h > 1) {
        for (int e = threadIdx.x; e < NX * NY; e += blockDim.x) {
            const int r = e / NX, c = e % NX;
            s[r * SS + c] = __fmul_rn(s[r * SS + c], ((ay0 + r) & 1) ? KMUL : KDIV);
        }
        __syncthreads();
        if (edge_y) adj_steps<true, true, HALO, HALO + TW, true>(s, ay0, h);
        else adj_steps<true, true, HALO, HALO + TW, false>(s, ay0, h);
    }
    for (int e = threadIdx.x; e < TW * TH; e += blockDim.x) {
        const int i = e % TW, j = e / TW;
        const int x = x0 + i, y = y0 + j;
        if (x < w && y < h) gout[(size_t)y * opitch + x] = s[(HALO + j) * SS + HALO + i];
    }
}

// Adjoint of one inverse level: gradient of the reconstructed level (w x h, natural order,
// `gin`) -> subband gradients (details into the Mallat plane `gdst`, LL into `gll`).
__global__ void __launch_bounds__(256)
inv_adj_level(const float* __restrict__ gin, size_t ipitch, int w, int h, float* __restrict__ gdst, size_t dpitch,
              float* __restrict__ gll, size_t llpitch, size_t zi, size_t zd, size_t zll) {
    __shared__ float s[NY * SS];
    gin += blockIdx.z * zi;
    gdst += blockIdx.z * zd;
    gll += blockIdx.z * zll;
    const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
    const int ax0 = x0 - HALO, ay0 = y0 - HALO;
    for (int e = threadIdx.x; e < NX * NY; e += blockDim.x) {
        const int r = e / NX, c = e % NX;
        const int gy = ay0 + r, gx = ax0 + c;
        s[r * SS + c] = (gx >= 0 && gx < w && gy >= 0 && gy < h) ? gin[(size_t)gy * ipitch + gx] : 0.0f;
    }
    __syncthreads();
    const bool edge_x = ax0 <= 0 || ax0 + NX >= w, edge_y = ay0 <= 0 || ay0 + NY >= h;
    // columns first (the inverse applied them last)
    if (h > 1) {
        if (edge_y) adj_steps<true, false, 0, NX, true>(s, ay0, h);
        else adj_steps<true, false, 0, NX, false>(s, ay0, h);
        for (int e = threadIdx.x; e < NX * NY; e += blockDim.x) {
            const int r = e / NX, c = e % NX;
            s[r * SS + c] = __fmul_rn(s[r * SS + c], ((ay0 + r) & 1) ? KDIV : KMUL);
        }
        __syncthreads();
    }
    if (w > 1) {
        if (edge_x) adj_steps<false, false, HALO, HALO + TH, true>(s, ax0, w);
        else adj_steps<false, false, HALO, HALO + TH, false>(s, ax0, w);
    }
    const int wl = (w + 1) >> 1, hl = (h + 1) >> 1;
    for (int e = threadIdx.x; e < TW * TH; e += blockDim.x) {
        const int i = e % TW, j = e / TW;
        const int x = x0 + i, y = y0 + j;
        if (x >= w || y >= h) continue;
        float v = s[(HALO + j) * SS + HALO + i];
        if (w > 1) v = __fmul_rn(v, (x & 1) ? KDIV : KMUL);
        const int qx = x & 1, qy = y & 1;
        if (!qx && !qy) gll[(size_t)(y >> 1) * llpitch + (x >> 1)] = v;
        else gdst[(size_t)((y >> 1) + (qy ? hl : 0)) * dpitch + (x >> 1) + (qx ? wl : 0)] = v;
    }
}

__global__ void copy_f(const float* __restrict__ a, size_t ap, float* __restrict__ b, size_t bp, int w, int h) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x < w && y < h) b[(size_t)y * bp + x] = a[(size_t)y * ap + x];
}

// ---- Philox4x32-10 (Salmon et al., SC'11) -------------------------------------------------------
__device__ __forceinline__ float philox_uniform(uint64_t seed, uint64_t i) {
    uint32_t c0 = (uint32_t)i, c1 = (uint32_t)(i >> 32), c2 = 0, c3 = 0;
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return __fmul_rn((float)(c0 >> 8), 1.0f / 16777216.0f) - 0.5f;
}

// band geometry of one Mallat plane, in QCD order
struct Bands {
    int nb;
    int x0[3 * 16 + 1], y0[3 * 16 + 1], bw[3 * 16 + 1], bh[3 * 16 + 1];
};

// grid: (tiles of 256 samples within the band, band, image).  Each CTA writes one partial sum
// per output (rate) so that the host-side reduction is in a fixed order.
__global__ void __launch_bounds__(256)
relaxed_quant_fwd(const float* __restrict__ y, float* __restrict__ yhat, int w, int h, size_t plane,
                  Bands B, const float* __restrict__ log_steps, uint64_t seed, float* __restrict__ rate_part,
                  int parts_per_band) {
    const int b = blockIdx.y, img = blockIdx.z;
    const int n = B.bw[b] * B.bh[b];
    const float step = expf(log_steps[b]);
    const float inv_ln2 = 1.4426950408889634f;
    float acc = 0.0f;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int xx = B.x0[b] + e % B.bw[b], yy = B.y0[b] + e / B.bw[b];
        const size_t idx = (size_t)img * plane + (size_t)yy * w + xx;
        const float u = philox_uniform(seed + (uint64_t)img, (uint64_t)yy * w + xx);
        const float t = __fadd_rn(__fdiv_rn(y[idx], step), u);
        yhat[idx] = __fmul_rn(t, step);
        acc += log1pf(fabsf(t)) * inv_ln2;
    }
    __shared__ float red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 128; o; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) rate_part[((size_t)img * B.nb + b) * parts_per_band + blockIdx.x] = red[0];
}

// g_y = g_yhat + lam * dr/dt / step;  g_logstep[b] += g_yhat * u * step + lam * dr/dt * (-y/step)
__global__ void __launch_bounds__(256)
relaxed_quant_bwd(const float* __restrict__ y, const float* __restrict__ gyhat, float* __restrict__ gy, int w, int h,
                  size_t plane, Bands B, const float* __restrict__ log_steps, uint64_t seed, float lam,
                  float* __restrict__ gls_part, int parts_per_band) {
    const int b = blockIdx.y, img = blockIdx.z;
    const int n = B.bw[b] * B.bh[b];
    const float step = expf(log_steps[b]);
    const float inv_ln2 = 1.4426950408889634f;
    float acc = 0.0f;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int xx = B.x0[b] + e % B.bw[b], yy = B.y0[b] + e / B.bw[b];
        const size_t idx = (size_t)img * plane + (size_t)yy * w + xx;
        const float u = philox_uniform(seed + (uint64_t)img, (uint64_t)yy * w + xx);
        const float yv = y[idx];
        const float t = __fadd_rn(__fdiv_rn(yv, step), u);
        const float sg = t > 0.0f ? 1.0f : (t < 0.0f ? -1.0f : 0.0f);
        const float drdt = lam * inv_ln2 * sg / (1.0f + fabsf(t));
        const float g = gyhat[idx];
        gy[idx] = g + drdt / step;
        acc += g * u * step - drdt * yv / step;
    }
    __shared__ float red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 128; o; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) gls_part[((size_t)img * B.nb + b) * parts_per_band + blockIdx.x] = red[0];
}

Bands make_bands(int w, int h, int levels) {
    Bands B{};
    j2k_band_rect r[3 * 16 + 1];
    B.nb = j2k_band_rects(w, h, levels, r);
    for (int b = 0; b < B.nb; ++b) {
        B.x0[b] = (int)r[b].x0;
        B.y0[b] = (int)r[b].y0;
        B.bw[b] = (int)r[b].w;
        B.bh[b] = (int)r[b].h;
    }
    return B;
}

j2k_status check_common(j2k_ctx* ctx, const void* a, const void* b, int n, size_t w, size_t h, int levels) {
    if (!ctx) return J2K_ERR_INVALID_ARG;
    if (!a || !b || n <= 0 || w == 0 || h == 0 || w > 65535 || h > 65535 || levels < 0 || levels > 16)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "differentiable 9/7: bad pointer, size or levels (0..16)");
    return J2K_OK;
}

}  // namespace

extern "C" {

j2k_status j2k_dwt97_forward_adjoint(j2k_ctx* ctx, const float* g_coef, float* g_img, int n, size_t w, size_t h,
                                     int levels) {
    J2K_TRY(check_common(ctx, g_coef, g_img, n, w, h, levels));
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    int ws[20], hs[20];
    ws[0] = (int)w;
    hs[0] = (int)h;
    for (int k = 1; k <= levels; ++k) { ws[k] = (ws[k - 1] + 1) / 2; hs[k] = (hs[k - 1] + 1) / 2; }
    const size_t plane = w * h, zlev = (size_t)ws[1] * hs[1];
    if (levels == 0) {
        for (int img = 0; img < n; ++img)
            copy_f<<<dim3((unsigned)((w + 255) / 256), (unsigned)h), 256, 0, st>>>(g_coef + img * plane, w,
                                                                                  g_img + img * plane, w, (int)w,
                                                                                  (int)h);
        J2K_CUDA(ctx, cudaGetLastError());
        return J2K_OK;
    }
    float* s0 = (float*)j2k_scratch(ctx, SCR_LL0, zlev * n * 4 + 64);
    float* s1 = (float*)j2k_scratch(ctx, SCR_LL1, zlev * n * 4 + 64);
    if (!s0 || !s1) return J2K_ERR_OUT_OF_MEMORY;
    // deepest level first; level k's LL gradient is level k+1's output
    const float* ll = g_coef;  // LL_L lives in the top-left of each Mallat plane
    size_t llp = w, llz = plane;
    for (int k = levels - 1; k >= 0; --k) {
        float* out = k == 0 ? g_img : ((levels - 1 - k) % 2 == 0 ? s0 : s1);
        const size_t op = k == 0 ? w : (size_t)ws[k], oz = k == 0 ? plane : zlev;
        dim3 g((ws[k] + TW - 1) / TW, (hs[k] + TH - 1) / TH, n);
        fwd_adj_level<<<g, 256, 0, st>>>(g_coef, w, ll, llp, ws[k], hs[k], out, op, plane, llz, oz);
        J2K_CUDA(ctx, cudaGetLastError());
        ll = out;
        llp = op;
        llz = oz;
    }
    return J2K_OK;
}

j2k_status j2k_dwt97_inverse_adjoint(j2k_ctx* ctx, const float* g_img, float* g_coef, int n, size_t w, size_t h,
                                     int levels) {
    J2K_TRY(check_common(ctx, g_img, g_coef, n, w, h, levels));
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    int ws[20], hs[20];
    ws[0] = (int)w;
    hs[0] = (int)h;
    for (int k = 1; k <= levels; ++k) { ws[k] = (ws[k - 1] + 1) / 2; hs[k] = (hs[k - 1] + 1) / 2; }
    const size_t plane = w * h, zlev = (size_t)ws[1] * hs[1];
    if (levels == 0) {
        for (int img = 0; img < n; ++img)
            copy_f<<<dim3((unsigned)((w + 255) / 256), (unsigned)h), 256, 0, st>>>(g_img + img * plane, w,
                                                                                  g_coef + img * plane, w, (int)w,
                                                                                  (int)h);
        J2K_CUDA(ctx, cudaGetLastError());
        return J2K_OK;
    }
    float* s0 = (float*)j2k_scratch(ctx, SCR_LL0, zlev * n * 4 + 64);
    float* s1 = (float*)j2k_scratch(ctx, SCR_LL1, zlev * n * 4 + 64);
    if (!s0 || !s1) return J2K_ERR_OUT_OF_MEMORY;
    const float* in = g_img;
    size_t ip = w, iz = plane;
    for (int k = 0; k < levels; ++k) {
        const bool last = k == levels - 1;
        float* ll = last ? g_coef : (k % 2 == 0 ? s0 : s1);
        const size_t llp = last ? w : (size_t)ws[k + 1], llz = last ? plane : zlev;
        dim3 g((ws[k] + TW - 1) / TW, (hs[k] + TH - 1) / TH, n);
        inv_adj_level<<<g, 256, 0, st>>>(in, ip, ws[k], hs[k], g_coef, w, ll, llp, iz, plane, llz);
        J2K_CUDA(ctx, cudaGetLastError());
        in = ll;
        ip = llp;
        iz = llz;
    }
    return J2K_OK;
}

j2k_status j2k_relaxed_quant_forward(j2k_ctx* ctx, const float* y, float* y_hat, int n, size_t w, size_t h,
                                     int levels, const float* log_steps, uint64_t seed, float* rate_partials,
                                     int parts_per_band) {
    J2K_TRY(check_common(ctx, y, y_hat, n, w, h, levels));
    if (!log_steps || !rate_partials || parts_per_band <= 0 || parts_per_band > 65535)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "relaxed quantiser: bad log_steps/partials");
    cudaSetDevice(ctx->device);
    Bands B = make_bands((int)w, (int)h, levels);
    dim3 g((unsigned)parts_per_band, (unsigned)B.nb, (unsigned)n);
    relaxed_quant_fwd<<<g, 256, 0, ctx->stream>>>(y, y_hat, (int)w, (int)h, w * h, B, log_steps, seed, rate_partials,
                                                  parts_per_band);
    J2K_CUDA(ctx, cudaGetLastError());
    return J2K_OK;
}

j2k_status j2k_relaxed_quant_backward(j2k_ctx* ctx, const float* y, const float* g_yhat, float* g_y, int n,
                                      size_t w, size_t h, int levels, const float* log_steps, uint64_t seed,
                                      float lam, float* g_logstep_partials, int parts_per_band) {
    J2K_TRY(check_common(ctx, y, g_y, n, w, h, levels));
    if (!g_yhat || !log_steps || !g_logstep_partials || parts_per_band <= 0 || parts_per_band > 65535)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "relaxed quantiser backward: bad arguments");
    cudaSetDevice(ctx->device);
    Bands B = make_bands((int)w, (int)h, levels);
    dim3 g((unsigned)parts_per_band, (unsigned)B.nb, (unsigned)n);
    relaxed_quant_bwd<<<g, 256, 0, ctx->stream>>>(y, g_yhat, g_y, (int)w, (int)h, w * h, B, log_steps, seed, lam,
                                                  g_logstep_partials, parts_per_band);
    J2K_CUDA(ctx, cudaGetLastError());
    return J2K_OK;
}

}  // extern "C"
