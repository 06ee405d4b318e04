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
#include <atomic>
#include <cmath>

#include "lift.cuh"

namespace {

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

// out = a - (*scale) * alpha * b (natural order, n planes back to back); the small-level
// fallback of the fused residual forms below
__global__ void axpy_f(const float* a, const float* b, const float* scale, float alpha, float* out, size_t count) {
    const float sc = __fmul_rn(scale ? *scale : 1.0f, alpha);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
        out[i] = __fsub_rn(a[i], __fmul_rn(sc, b[i]));
}

// d = xh - x over the same 248 x 16 tiles as the strip kernel, one partial sum of d^2 per tile
__global__ void residual_tiles(const float* xh, const float* x, float* d, int w, int h, float* part) {
    const size_t plane = (size_t)w * h;
    xh += blockIdx.z * plane;
    x += blockIdx.z * plane;
    d += blockIdx.z * plane;
    float sq = 0.0f;
    for (int e = threadIdx.x; e < FTW * STH; e += blockDim.x) {
        const int xx = blockIdx.x * FTW + e % FTW, yy = blockIdx.y * STH + e / FTW;
        if (xx < w && yy < h) {
            const size_t i = (size_t)yy * w + xx;
            const float v = __fsub_rn(xh[i], x[i]);
            d[i] = v;
            sq = __fmaf_rn(v, v, sq);
        }
    }
    __shared__ float red[256];
    red[threadIdx.x] = sq;
    __syncthreads();
    for (int o = 128; o; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = red[0];
}

// ---- Philox4x32-10 (Salmon et al., SC'11) -------------------------------------------------------
__device__ __forceinline__ void philox4(uint64_t key, uint64_t ctr, uint32_t (&o)[4]) {
    uint32_t c0 = (uint32_t)ctr, c1 = (uint32_t)(ctr >> 32), c2 = 0, c3 = 0;
    uint32_t k0 = (uint32_t)key, k1 = (uint32_t)(key >> 32);
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
    o[0] = c0;
    o[1] = c1;
    o[2] = c2;
    o[3] = c3;
}
__device__ __forceinline__ float noise_of(uint32_t word) {
    return __fmul_rn((float)(word >> 8), 1.0f / 16777216.0f) - 0.5f;
}

// Level widths/heights of one Mallat plane: W[0] = w, W[k] = ceil(W[k-1]/2).
struct Levels {
    int L;
    int W[17], H[17];
};
// depth of a coordinate: how many of the levels keep it in their low half
__device__ __forceinline__ int depth_of(int v, const int* lim, int L) {
    int d = 0;
#pragma unroll
    for (int k = 1; k <= 16; ++k)
        if (k <= L) d += v < lim[k];
    return d;
}
// QCD band index of the Mallat sample with depths (dx, dy): LL = 0, level d's HL/LH/HH at
// 1 + 3(L - d) + {0, 1, 2}
__device__ __forceinline__ int band_of(int dx, int dy, int L) {
    const int m = min(dx, dy);
    if (m == L) return 0;
    const int o = (dx == m && dy == m) ? 2 : (dx == m ? 0 : 1);
    return 1 + 3 * (L - (m + 1)) + o;
}

#include "rowband.cuh"

// Relaxed quantiser over whole Mallat planes.  grid (parts, images); CTA p takes rows
// [p*rows, (p+1)*rows) of its image, thread i the 4-sample groups i, i+256, ... of each row.
// Noise: one Philox4x32-10 call per group (key seed + image, counter y*ceil(w/4) + x/4), word
// x%4 for sample x.  Per-band sums are kept per thread in shared memory and reduced in a
// fixed order, so the partials are deterministic.
// NZ: the forward also writes the noise u of every sample to nz, and the backward reads it from
// there instead of regenerating it.
template <bool BWD, bool NZ>
__global__ void __launch_bounds__(256, 3)
relaxed_quant_k(const float* __restrict__ y, const float* __restrict__ gin, float* __restrict__ out, int w, int h,
                size_t plane, Levels lv, const float* __restrict__ log_steps, uint64_t seed, float lam,
                const float* __restrict__ gscale, float alpha, float* __restrict__ part, int rows, int vec,
                float* __restrict__ nz) {
    extern __shared__ float acc[];  // [band][256]
    __shared__ float stp[49], rstp[49];
    __shared__ int wlim[17], hlim[17];
    griddep_launch_dependents();
    griddep_wait();  // launched as a dependent: the previous kernel's writes are visible from here
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5, img = blockIdx.y;
    const int L = lv.L, nb = 3 * L + 1;
    for (int b = 0; b < nb; ++b) acc[b * 256 + t] = 0.0f;
    if (t < nb) {
        stp[t] = expf(log_steps[t]);
        rstp[t] = __frcp_rn(stp[t]);
    }
    if (t <= L) {
        wlim[t] = lv.W[t];
        hlim[t] = lv.H[t];
    }
    __syncthreads();
    const float inv_ln2 = 1.4426950408889634f;
    float G = 1.0f, lamG = lam;
    if (BWD) {
        const float s = gscale ? *gscale : 1.0f;
        G = __fmul_rn(s, alpha);
        lamG = __fmul_rn(s, lam);
    }
    const int groups = (w + 3) >> 2;
    const uint64_t key = seed + (uint64_t)img;
    const int r0 = blockIdx.x * rows, r1 = min(h, r0 + rows);
    const size_t ib = (size_t)img * plane;
    constexpr int RB = BWD ? 2 : 4;  // rows per batch: all their loads are issued before any use
    for (int g = t; g < groups; g += 256) {
        const int x = 4 * g;
        const bool full = vec && x + 4 <= w;
        int dx[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) dx[k] = depth_of(x + k, wlim, L);
        for (int y0 = r0; y0 < r1; y0 += RB) {
            float v[RB][4], gi[RB][4], un[RB][4];
#pragma unroll
            for (int i = 0; i < RB; ++i) {
                const size_t rb = ib + (size_t)(y0 + i) * w + x;
                if (y0 + i >= r1) break;
                if (full) {
                    *reinterpret_cast<float4*>(v[i]) = __ldg(reinterpret_cast<const float4*>(y + rb));
                    if (BWD) *reinterpret_cast<float4*>(gi[i]) = __ldg(reinterpret_cast<const float4*>(gin + rb));
                    if (BWD && NZ) *reinterpret_cast<float4*>(un[i]) = __ldg(reinterpret_cast<const float4*>(nz + rb));
                } else {
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        v[i][k] = x + k < w ? y[rb + k] : 0.0f;
                        if (BWD) gi[i][k] = x + k < w ? gin[rb + k] : 0.0f;
                        if (BWD && NZ) un[i][k] = x + k < w ? nz[rb + k] : 0.0f;
                    }
                }
            }
#pragma unroll
            for (int i = 0; i < RB; ++i) {
                const int yy = y0 + i;
                if (yy >= r1) break;
                const int dy = depth_of(yy, hlim, L);
                uint32_t o[4] = {0u, 0u, 0u, 0u};
                if (!(BWD && NZ)) philox4(key, (uint64_t)yy * groups + g, o);
                float r[4], uo[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    r[k] = 0.0f;
                    if (x + k >= w) continue;
                    const int b = band_of(dx[k], dy, L);
                    const float step = stp[b], rs = rstp[b], u = (BWD && NZ) ? un[i][k] : noise_of(o[k]);
                    uo[k] = u;
                    const float tt = __fadd_rn(__fmul_rn(v[i][k], rs), u);
                    if (!BWD) {
                        r[k] = __fmul_rn(tt, step);
                        acc[b * 256 + t] += __log2f(__fadd_rn(1.0f, fabsf(tt)));
                    } else {
                        const float sg = tt > 0.0f ? 1.0f : (tt < 0.0f ? -1.0f : 0.0f);
                        const float drdt = __fdividef(lamG * inv_ln2 * sg, 1.0f + fabsf(tt));
                        const float gg = __fmul_rn(G, gi[i][k]);
                        r[k] = __fadd_rn(gg, __fmul_rn(drdt, rs));
                        acc[b * 256 + t] += gg * u * step - drdt * v[i][k] * rs;
                    }
                }
                const size_t rb = ib + (size_t)yy * w + x;
                if (full) {
                    *reinterpret_cast<float4*>(out + rb) = *reinterpret_cast<float4*>(r);
                    if (!BWD && NZ) *reinterpret_cast<float4*>(nz + rb) = *reinterpret_cast<float4*>(uo);
                } else {
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (x + k < w) {
                            out[rb + k] = r[k];
                            if (!BWD && NZ) nz[rb + k] = uo[k];
                        }
                }
            }
        }
    }
    __syncthreads();
    for (int b = warp; b < nb; b += 8) {
        float a = 0.0f;
#pragma unroll
        for (int i = 0; i < 8; ++i) a += acc[b * 256 + lane + 32 * i];
#pragma unroll
        for (int o = 16; o; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if (lane == 0) part[((size_t)img * nb + b) * gridDim.x + blockIdx.x] = a;
    }
}

Levels make_levels(int w, int h, int levels) {
    Levels lv{};
    lv.L = levels;
    lv.W[0] = w;
    lv.H[0] = h;
    for (int k = 1; k <= levels; ++k) {
        lv.W[k] = (lv.W[k - 1] + 1) / 2;
        lv.H[k] = (lv.H[k - 1] + 1) / 2;
    }
    return lv;
}

// ---- row-band level launches ------------------------------------------------------------------
static_assert(RB_BH == STH, "the band kernels keep the strip kernels' 16-row partial-sum layout");

bool rb_width_ok(int w) { return w == 64 || w == 128 || w == 256 || w == 512 || w == 1024; }
bool rb_level_ok(const j2k_ctx* ctx, int w, int h) { return ctx->dwt97_rows && rb_width_ok(w) && h >= 2; }
// how many levels, finest first, the band kernels take (widths halve, so they are a prefix)
int rb_levels(const j2k_ctx* ctx, const int* ws, const int* hs, int levels) {
    int k = 0;
    while (k < levels && rb_level_ok(ctx, ws[k], hs[k])) ++k;
    return k;
}

// Each kernel opts in to its dynamic shared memory once per device (with its static arrays the
// total can pass 48 KB even when the dynamic part does not).
template <typename K>
cudaError_t rb_optin(K* k, size_t smem, std::atomic<uint32_t>& mask, int dev) {
    const uint32_t bit = 1u << (dev & 31);
    if (mask.load() & bit) return cudaSuccess;
    const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) mask.fetch_or(bit);
    return e;
}

template <int MODE, int SPL, int QB>
cudaError_t rb_ana_go(j2k_ctx* ctx, int h, int n, bool pdl, const float* in, size_t ip, size_t iz, float* dst,
                      size_t dp, size_t dz, float* lld, size_t llp, size_t llz, int last, const RbQ& q) {
    static std::atomic<uint32_t> optin{0};
    const size_t smem = (size_t)RB_BH * RB<SPL>::W * sizeof(float);
    const cudaError_t e = rb_optin(rb_ana<MODE, SPL, QB>, smem, optin, ctx->device);
    if (e != cudaSuccess) return e;
    const dim3 g((unsigned)((h + RB_BH - 1) / RB_BH), (unsigned)n);
    return launch_pdl_smem(rb_ana<MODE, SPL, QB>, g, dim3(RB<SPL>::NT), smem, ctx->stream, pdl, in, ip, iz, h, dst,
                           dp, dz, lld, llp, llz, last, q);
}

// One analysis-shape level of width w (rb_width_ok) and height h over n images.
template <int MODE, int QB>
j2k_status rb_ana_level(j2k_ctx* ctx, int w, int h, int n, bool pdl, const float* in, size_t ip, size_t iz,
                        float* dst, size_t dp, size_t dz, float* lld, size_t llp, size_t llz, int last,
                        const RbQ& q) {
    cudaError_t e = cudaErrorInvalidValue;
    switch (w) {
        case 64: e = rb_ana_go<MODE, 2, QB>(ctx, h, n, pdl, in, ip, iz, dst, dp, dz, lld, llp, llz, last, q); break;
        case 128: e = rb_ana_go<MODE, 4, QB>(ctx, h, n, pdl, in, ip, iz, dst, dp, dz, lld, llp, llz, last, q); break;
        case 256: e = rb_ana_go<MODE, 8, QB>(ctx, h, n, pdl, in, ip, iz, dst, dp, dz, lld, llp, llz, last, q); break;
        case 512: e = rb_ana_go<MODE, 16, QB>(ctx, h, n, pdl, in, ip, iz, dst, dp, dz, lld, llp, llz, last, q); break;
        case 1024: e = rb_ana_go<MODE, 32, QB>(ctx, h, n, pdl, in, ip, iz, dst, dp, dz, lld, llp, llz, last, q); break;
        default: return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "band kernels: level width not a power of two in 64..1024");
    }
    J2K_CUDA(ctx, e);
    return J2K_OK;
}

template <int MODE, int SPL, bool LQ, int EXTRA>
cudaError_t rb_syn_go(j2k_ctx* ctx, int h, int n, bool pdl, const float* src, size_t sp, size_t sz,
                      const float* lls, size_t llp, size_t llz, float* out, size_t op, size_t oz,
                      const SynExtra& ex, const RbQ& q, int deepest) {
    static std::atomic<uint32_t> optin{0};
    const size_t smem = (size_t)(RB_BH + 2 * RB_HV) * RB<SPL>::W * sizeof(float);
    const cudaError_t e = rb_optin(rb_syn<MODE, SPL, LQ, EXTRA>, smem, optin, ctx->device);
    if (e != cudaSuccess) return e;
    const dim3 g((unsigned)((h + RB_BH - 1) / RB_BH), (unsigned)n);
    return launch_pdl_smem(rb_syn<MODE, SPL, LQ, EXTRA>, g, dim3(RB<SPL>::NT), smem, ctx->stream, pdl, src, sp, sz,
                           lls, llp, llz, h, out, op, oz, ex, q, deepest);
}

// One synthesis-shape level of width w (rb_width_ok) and height h over n images.
template <int MODE, bool LQ, int EXTRA>
j2k_status rb_syn_level(j2k_ctx* ctx, int w, int h, int n, bool pdl, const float* src, size_t sp, size_t sz,
                        const float* lls, size_t llp, size_t llz, float* out, size_t op, size_t oz,
                        const SynExtra& ex, const RbQ& q, int deepest) {
    cudaError_t e = cudaErrorInvalidValue;
#define RB_SYN(SPL_) rb_syn_go<MODE, SPL_, LQ, EXTRA>(ctx, h, n, pdl, src, sp, sz, lls, llp, llz, out, op, oz, ex, q, deepest)
    switch (w) {
        case 64: e = RB_SYN(2); break;
        case 128: e = RB_SYN(4); break;
        case 256: e = RB_SYN(8); break;
        case 512: e = RB_SYN(16); break;
        case 1024: e = RB_SYN(32); break;
        default: return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "band kernels: level width not a power of two in 64..1024");
    }
#undef RB_SYN
    J2K_CUDA(ctx, e);
    return J2K_OK;
}

// the quantiser operands of level k (partials, steps and planes as the call needs them)
RbQ rb_q(const float* log_steps, uint64_t seed, const float* u, const float* y, float lam, const float* gscale,
         float alpha, float* part, int kp, int levels, int k, size_t w) {
    RbQ q{};
    q.log_steps = log_steps;
    q.seed = seed;
    q.u = const_cast<float*>(u);
    q.y = y;
    q.lam = lam;
    q.gscale = gscale;
    q.alpha = alpha;
    q.part = part;
    q.kp = kp;
    q.levels = levels;
    q.level = k;
    q.groups = (int)((w + 3) / 4);
    return q;
}

j2k_status check_common(j2k_ctx* ctx, const void* a, const void* b, int n, size_t w, size_t h, int levels) {
    if (!ctx) return J2K_ERR_INVALID_ARG;
    if (!a || !b || n <= 0 || n > 65535 || w == 0 || h == 0 || w > 65535 || h > 65535 || levels < 0 ||
        levels > 16)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "differentiable 9/7: bad pointer, size or levels (0..16)");
    return J2K_OK;
}

// Transpose of the forward DWT, deepest level first.  With `ex` (EXTRA 2) the level-0 output
// is g_img = DWT^T(g_coef) - (*scale) * alpha * sub.
j2k_status fwd_adj_run(j2k_ctx* ctx, const float* g_coef, float* g_img, int n, size_t w, size_t h, int levels,
                       const SynExtra* ex) {
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    int ws[20] = {}, hs[20] = {};
    ws[0] = (int)w;
    hs[0] = (int)h;
    for (int k = 1; k <= levels; ++k) { ws[k] = (ws[k - 1] + 1) / 2; hs[k] = (hs[k - 1] + 1) / 2; }
    const size_t plane = w * h, zlev = (size_t)ws[1] * hs[1];
    if (levels == 0) {
        if (ex) {
            axpy_f<<<ctx->sm_count * 4, 256, 0, st>>>(g_coef, ex->sub, ex->scale, ex->alpha, g_img, plane * n);
        } else {
            for (int img = 0; img < n; ++img)
                copy_f<<<dim3((unsigned)((w + 255) / 256), (unsigned)h), 256, 0, st>>>(
                    g_coef + img * plane, w, g_img + img * plane, w, (int)w, (int)h);
        }
        J2K_CUDA(ctx, cudaGetLastError());
        return J2K_OK;
    }
    float* s0 = (float*)j2k_scratch(ctx, SCR_LL0, zlev * n * 4 + 64);
    float* s1 = (float*)j2k_scratch(ctx, SCR_LL1, zlev * n * 4 + 64);
    if (!s0 || !s1) return J2K_ERR_OUT_OF_MEMORY;
    const float* ll = g_coef;  // LL_L lives in the top-left of each Mallat plane
    size_t llp = w, llz = plane;
    for (int k = levels - 1; k >= 0; --k) {
        float* out = k == 0 ? g_img : ((levels - 1 - k) % 2 == 0 ? s0 : s1);
        const size_t op = k == 0 ? w : (size_t)ws[k], oz = k == 0 ? plane : zlev;
        const bool fused = k == 0 && ex;
        if (rb_level_ok(ctx, ws[k], hs[k])) {
            const bool pdl = k < levels - 1;  // every launch of the chain but the first
            const RbQ q = rb_q(nullptr, 0, nullptr, nullptr, 0.0f, nullptr, 1.0f, nullptr, 0, levels, k, w);
            if (fused)
                J2K_TRY((rb_syn_level<1, false, 2>(ctx, ws[k], hs[k], n, pdl, g_coef, w, plane, ll, llp, llz, out, op, oz,
                                                    *ex, q, 0)));
            else
                J2K_TRY((rb_syn_level<1, false, 0>(ctx, ws[k], hs[k], n, pdl, g_coef, w, plane, ll, llp, llz, out, op, oz,
                                                    SynExtra{}, q, 0)));
        } else if (ws[k] >= 8 && hs[k] >= 2) {
            const int wl = (ws[k] + 1) / 2;
            const int vec = (((uintptr_t)g_coef & 7) == 0) && ((w & 1) == 0) && ((plane & 1) == 0) &&
                            (((uintptr_t)ll & 7) == 0) && ((llp & 1) == 0) && ((llz & 1) == 0) && ((wl & 1) == 0);
            const dim3 fg((ws[k] + FTW - 1) / FTW, (hs[k] + STH - 1) / STH, n);
            const ZStride zs{plane, oz, llz};
            if (fused)
                J2K_CUDA(ctx, launch_pdl(dwt_syn_fast<97, 1, float, false, false, 2>, fg, dim3(256), st, false, g_coef, w,
                                         ll, llp, ws[k], hs[k], out, op, Steps4{}, zs, vec, *ex));
            else
                J2K_CUDA(ctx, launch_pdl(dwt_syn_fast<97, 1, float, false, false, 0>, fg, dim3(256), st, false, g_coef, w,
                                         ll, llp, ws[k], hs[k], out, op, Steps4{}, zs, vec, SynExtra{}));
        } else {
            dim3 g((ws[k] + TW - 1) / TW, (hs[k] + TH - 1) / TH, n);
            fwd_adj_level<<<g, 256, 0, st>>>(g_coef, w, ll, llp, ws[k], hs[k], out, op, plane, llz, oz);
            if (fused)
                axpy_f<<<ctx->sm_count * 4, 256, 0, st>>>(g_img, ex->sub, ex->scale, ex->alpha, g_img, plane * n);
        }
        J2K_CUDA(ctx, cudaGetLastError());
        ll = out;
        llp = op;
        llz = oz;
    }
    return J2K_OK;
}

j2k_status quant_run(j2k_ctx* ctx, bool bwd, const float* y, const float* gin, float* out, int n, size_t w,
                     size_t h, int levels, const float* log_steps, uint64_t seed, float lam, const float* gscale,
                     float alpha, float* partials, int parts, float* noise) {
    J2K_TRY(check_common(ctx, y, out, n, w, h, levels));
    if (!log_steps || !partials || parts <= 0 || parts > 65535 || (bwd && !gin))
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "relaxed quantiser: bad log_steps, partials or parts");
    cudaSetDevice(ctx->device);
    const int nb = 3 * levels + 1;
    const size_t smem = (size_t)nb * 256 * 4;
    const int rows = (int)((h + parts - 1) / parts);
    const size_t plane = w * h;
    const int vec = (((uintptr_t)y & 15) == 0) && (((uintptr_t)out & 15) == 0) && (!bwd || ((uintptr_t)gin & 15) == 0) &&
                    (!noise || ((uintptr_t)noise & 15) == 0) && ((w & 3) == 0);
    const dim3 g((unsigned)parts, (unsigned)n);
    const Levels lv = make_levels((int)w, (int)h, levels);
#define RQ_LAUNCH(B_, N_)                                                                                     \
    do {                                                                                                       \
        if (smem > 48 * 1024)                                                                                  \
            J2K_CUDA(ctx, cudaFuncSetAttribute(relaxed_quant_k<B_, N_>,                                        \
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));       \
        J2K_CUDA(ctx, launch_pdl_smem(relaxed_quant_k<B_, N_>, g, dim3(256), smem, ctx->stream, false, y, gin, out, \
                                      (int)w, (int)h, plane, lv, log_steps, seed, lam, gscale, alpha, partials,    \
                                      rows, vec, noise));                                                          \
    } while (0)
    if (bwd) {
        if (noise) RQ_LAUNCH(true, true);
        else RQ_LAUNCH(true, false);
    } else {
        if (noise) RQ_LAUNCH(false, true);
        else RQ_LAUNCH(false, false);
    }
#undef RQ_LAUNCH
    J2K_CUDA(ctx, cudaGetLastError());
    return J2K_OK;
}

}  // namespace

namespace {

// Sum of a float array by one CTA (blockDim a power of two), in a fixed order (strided per thread, then a
// fixed tree), so repeated steps give the same bits.
__device__ float cta_sum(const float* __restrict__ a, size_t n, float* sh) {
    float v0 = 0.0f, v1 = 0.0f, v2 = 0.0f, v3 = 0.0f;  // four independent chains of loads
    const size_t step = blockDim.x;
    size_t i = threadIdx.x;
    for (; i + 3 * step < n; i += 4 * step) {
        v0 += a[i];
        v1 += a[i + step];
        v2 += a[i + 2 * step];
        v3 += a[i + 3 * step];
    }
    for (; i < n; i += step) v0 += a[i];
    sh[threadIdx.x] = (v0 + v1) + (v2 + v3);
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    const float r = sh[0];
    __syncthreads();
    return r;
}

// loss = sum(sq) * inv_count + lam * sum(rate)
__global__ void __launch_bounds__(1024) rd_finalize_kernel(const float* __restrict__ rate, size_t nrate,
                                                          const float* __restrict__ sq, size_t nsq, double inv_count,
                                                          float lam, float* __restrict__ loss) {
    __shared__ float sh[1024];
    griddep_launch_dependents();
    griddep_wait();
    const float r = cta_sum(rate, nrate, sh);
    const float q = cta_sum(sq, nsq, sh);
    if (threadIdx.x == 0) *loss = (float)((double)q * inv_count) + lam * r;
}

// out[b] = sum over images i and parts j of parts[(i * nb + b) * k + j]; one CTA per band
__global__ void __launch_bounds__(256) band_sum_kernel(const float* __restrict__ parts, int n, int nb, int k,
                                                       float* __restrict__ out) {
    __shared__ float sh[256];
    griddep_launch_dependents();
    griddep_wait();
    const int b = blockIdx.x;
    float v = 0.0f;
    for (int t = threadIdx.x; t < n * k; t += blockDim.x) v += parts[((size_t)(t / k) * nb + b) * k + (t % k)];
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[b] = sh[0];
}

}  // namespace

namespace {

// Inverse 9/7 of the Mallat planes y with the residual d = IDWT(y) - x fused into level 0, for
// planes whose finest kr >= 1 levels the band kernels take; the deeper levels, if any, run as one
// strip-kernel transform of the planes' top-left corner.  lq (kr == levels only): y holds the
// coefficients with their noise q.u, every band entering as y_hat.  pdl: the first launch is a
// programmatic dependent too.
j2k_status inv_residual_rb(j2k_ctx* ctx, const float* y, const float* x, float* d, int n, size_t w, size_t h,
                           int levels, float* sq_partials, const RbQ* lq, bool pdl) {
    cudaStream_t st = ctx->stream;
    const size_t plane = w * h;
    int ws[20] = {}, hs[20] = {};
    ws[0] = (int)w;
    hs[0] = (int)h;
    for (int k = 1; k <= levels; ++k) { ws[k] = (ws[k - 1] + 1) / 2; hs[k] = (hs[k - 1] + 1) / 2; }
    const int kr = rb_levels(ctx, ws, hs, levels);
    if (kr < 1 || (lq && kr < levels)) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "band inverse: level shapes");
    float *bufA = nullptr, *bufB = nullptr;
    if (levels > 1) {
        const size_t z1 = (size_t)ws[1] * hs[1] * (size_t)n * 4 + 64;
        bufA = (float*)j2k_scratch(ctx, SCR_RES, z1);
        bufB = (float*)j2k_scratch(ctx, SCR_LL1, z1);
        if (!bufA || !bufB) return J2K_ERR_OUT_OF_MEMORY;
    }
    const float* ll = y;
    size_t llp = w, llz = plane;
    if (kr < levels) {
        // levels kr .. L-1: the top-left ws[kr] x hs[kr] of each plane is their own Mallat plane
        void* a = j2k_scratch(ctx, SCR_LL0, (size_t)ws[kr + 1] * hs[kr + 1] * (size_t)n * 4 + 64);
        if (!a) return J2K_ERR_OUT_OF_MEMORY;
        const size_t zk = (size_t)ws[kr] * hs[kr];
        J2K_TRY(j2k_dwt_inv_impl(ctx, J2K_W97, J2K_ORDER_T800, y, w, bufA, ws[kr], ws[kr], hs[kr], levels - kr, nullptr,
                                 a, bufB, j2k_dwt_tile{64, 64}, st, n, plane, zk));
        ll = bufA;
        llp = (size_t)ws[kr];
        llz = zk;
        pdl = true;
    }
    for (int k = kr - 1; k >= 0; --k) {
        const int deepest = k == levels - 1;
        RbQ q = lq ? *lq : rb_q(nullptr, 0, nullptr, nullptr, 0.0f, nullptr, 1.0f, nullptr, 0, levels, k, w);
        q.level = k;
        if (k == 0) {
            const SynExtra ex{x, w, plane, nullptr, 1.0f, sq_partials, (int)((w + FTW - 1) / FTW)};
            if (lq)
                J2K_TRY((rb_syn_level<0, true, 1>(ctx, ws[0], hs[0], n, pdl, y, w, plane, ll, llp, llz, d, w, plane, ex, q,
                                                   deepest)));
            else
                J2K_TRY((rb_syn_level<0, false, 1>(ctx, ws[0], hs[0], n, pdl, y, w, plane, ll, llp, llz, d, w, plane, ex,
                                                    q, deepest)));
        } else {
            float* out = ll == bufA ? bufB : bufA;
            const size_t op = (size_t)ws[k], oz = (size_t)ws[k] * hs[k];
            if (lq)
                J2K_TRY((rb_syn_level<0, true, 0>(ctx, ws[k], hs[k], n, pdl, y, w, plane, ll, llp, llz, out, op, oz,
                                                   SynExtra{}, q, deepest)));
            else
                J2K_TRY((rb_syn_level<0, false, 0>(ctx, ws[k], hs[k], n, pdl, y, w, plane, ll, llp, llz, out, op, oz,
                                                    SynExtra{}, q, deepest)));
            ll = out;
            llp = op;
            llz = oz;
        }
        pdl = true;
    }
    return J2K_OK;
}

}  // namespace

extern "C" {

j2k_status j2k_dwt97_rd_finalize(j2k_ctx* ctx, const float* rate_partials, size_t nrate, const float* sq_partials,
                                 size_t nsq, double inv_count, float lam, float* loss) {
    J2K_API_BEGIN
    if (!ctx || !loss || (!rate_partials && nrate) || (!sq_partials && nsq)) return J2K_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    J2K_CUDA(ctx, launch_pdl(rd_finalize_kernel, dim3(1), dim3(1024), ctx->stream, false, rate_partials, nrate,
                             sq_partials, nsq, inv_count, lam, loss));
    J2K_CUDA(ctx, cudaGetLastError());
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_dwt97_band_sum(j2k_ctx* ctx, const float* partials, int n, int nb, int k, float* out) {
    J2K_API_BEGIN
    if (!ctx || !partials || !out || n < 1 || nb < 1 || k < 1) return J2K_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    J2K_CUDA(ctx, launch_pdl(band_sum_kernel, dim3((unsigned)nb), dim3(256), ctx->stream, false, partials, n, nb, k,
                             out));
    J2K_CUDA(ctx, cudaGetLastError());
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_dwt97_forward_adjoint(j2k_ctx* ctx, const float* g_coef, float* g_img, int n, size_t w, size_t h,
                                     int levels) {
    J2K_API_BEGIN
    J2K_TRY(check_common(ctx, g_coef, g_img, n, w, h, levels));
    return fwd_adj_run(ctx, g_coef, g_img, n, w, h, levels, nullptr);
    J2K_API_END
}

j2k_status j2k_dwt97_forward_adjoint_residual(j2k_ctx* ctx, const float* g_coef, const float* sub,
                                              const float* scale, float alpha, float* g_img, int n, size_t w,
                                              size_t h, int levels) {
    J2K_API_BEGIN
    J2K_TRY(check_common(ctx, g_coef, g_img, n, w, h, levels));
    if (!sub) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "forward adjoint residual: sub is NULL");
    const SynExtra ex{sub, w, w * h, scale, alpha, nullptr};
    return fwd_adj_run(ctx, g_coef, g_img, n, w, h, levels, &ex);
    J2K_API_END
}

j2k_status j2k_dwt97_inverse_adjoint(j2k_ctx* ctx, const float* g_img, float* g_coef, int n, size_t w, size_t h,
                                     int levels) {
    J2K_API_BEGIN
    J2K_TRY(check_common(ctx, g_img, g_coef, n, w, h, levels));
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    int ws[20] = {}, hs[20] = {};
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
        if (rb_level_ok(ctx, ws[k], hs[k])) {
            const RbQ q = rb_q(nullptr, 0, nullptr, nullptr, 0.0f, nullptr, 1.0f, nullptr, 0, levels, k, w);
            J2K_TRY((rb_ana_level<2, 0>(ctx, ws[k], hs[k], n, k > 0, in, ip, iz, g_coef, w, plane, ll, llp, llz, 0, q)));
        } else if (ws[k] >= 8 && hs[k] >= 2) {
            const int vin = (((uintptr_t)in & 15) == 0) && ((ip & 3) == 0) && ((iz & 3) == 0);
            const int vout = (((uintptr_t)g_coef & 7) == 0) && ((w & 1) == 0) && ((plane & 1) == 0) &&
                             (((uintptr_t)ll & 7) == 0) && ((llp & 1) == 0) && ((llz & 1) == 0);
            const dim3 fg((ws[k] + FTW - 1) / FTW, (hs[k] + STH - 1) / STH, n);
            J2K_CUDA(ctx, launch_pdl(iadj_ana_fast, fg, dim3(256), st, false, in, ip, ws[k], hs[k], g_coef, w, ll, llp,
                                     ZStride{iz, plane, llz}, vin, vout));
        } else {
            dim3 g((ws[k] + TW - 1) / TW, (hs[k] + TH - 1) / TH, n);
            inv_adj_level<<<g, 256, 0, st>>>(in, ip, ws[k], hs[k], g_coef, w, ll, llp, iz, plane, llz);
        }
        J2K_CUDA(ctx, cudaGetLastError());
        in = ll;
        ip = llp;
        iz = llz;
    }
    return J2K_OK;
    J2K_API_END
}

size_t j2k_dwt97_residual_partials(size_t w, size_t h, int n) {
    return ((w + FTW - 1) / FTW) * ((h + STH - 1) / STH) * (size_t)(n > 0 ? n : 0);
}

j2k_status j2k_dwt97_inverse_residual(j2k_ctx* ctx, const float* y, const float* x, float* d, int n, size_t w,
                                      size_t h, int levels, float* sq_partials) {
    J2K_API_BEGIN
    J2K_TRY(check_common(ctx, y, d, n, w, h, levels));
    if (!x || !sq_partials) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "inverse residual: NULL x or partials");
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const size_t plane = w * h;
    const dim3 fg((unsigned)((w + FTW - 1) / FTW), (unsigned)((h + STH - 1) / STH), (unsigned)n);
    if (levels == 0 || w < 8 || h < 2) {
        // small planes: plain inverse into d, then the residual pass over the same tiles
        J2K_TRY(j2k_dwt_inverse_batch(ctx, J2K_W97, J2K_ORDER_T800, y, w, plane, d, w, plane, n, w, h, levels,
                                      nullptr));
        residual_tiles<<<fg, 256, 0, st>>>(d, x, d, (int)w, (int)h, sq_partials);
        J2K_CUDA(ctx, cudaGetLastError());
        return J2K_OK;
    }
    {
        int ws[20] = {}, hs[20] = {};
        ws[0] = (int)w;
        hs[0] = (int)h;
        for (int k = 1; k <= levels; ++k) { ws[k] = (ws[k - 1] + 1) / 2; hs[k] = (hs[k - 1] + 1) / 2; }
        if (rb_levels(ctx, ws, hs, levels) >= 1)
            return inv_residual_rb(ctx, y, x, d, n, w, h, levels, sq_partials, nullptr, false);
    }
    // levels L..2 reconstruct LL_1 (the top-left ceil(w/2) x ceil(h/2) of each Mallat plane is
    // itself the Mallat plane of LL_1's (L-1)-level transform) into scratch; level 1 runs fused
    const size_t w1 = (w + 1) / 2, h1 = (h + 1) / 2;
    const float* ll = y;
    size_t llp = w, llz = plane;
    if (levels > 1) {
        float* buf = (float*)j2k_scratch(ctx, SCR_RES, w1 * h1 * (size_t)n * 4 + 64);
        if (!buf) return J2K_ERR_OUT_OF_MEMORY;
        size_t w2 = (w1 + 1) / 2, h2 = (h1 + 1) / 2;
        void* a = j2k_scratch(ctx, SCR_LL0, w2 * h2 * (size_t)n * 4 + 64);
        void* b = j2k_scratch(ctx, SCR_LL1, ((w2 + 1) / 2) * ((h2 + 1) / 2) * (size_t)n * 4 + 64);
        if (!a || !b) return J2K_ERR_OUT_OF_MEMORY;
        J2K_TRY(j2k_dwt_inv_impl(ctx, J2K_W97, J2K_ORDER_T800, y, w, buf, w1, w1, h1, levels - 1, nullptr, a, b,
                                 j2k_dwt_tile{64, 64}, st, n, plane, w1 * h1));
        ll = buf;
        llp = w1;
        llz = w1 * h1;
    }
    const int wl = (int)w1;
    const int vec = (((uintptr_t)y & 7) == 0) && ((w & 1) == 0) && ((plane & 1) == 0) && (((uintptr_t)ll & 7) == 0) &&
                    ((llp & 1) == 0) && ((llz & 1) == 0) && ((wl & 1) == 0);
    const SynExtra ex{x, w, plane, nullptr, 1.0f, sq_partials};
    J2K_CUDA(ctx, launch_pdl(dwt_syn_fast<97, 0, float, false, false, 1>, fg, dim3(256), st, false, y, w, ll, llp,
                             (int)w, (int)h, d, w, Steps4{}, ZStride{plane, plane, llz}, vec, ex));
    J2K_CUDA(ctx, cudaGetLastError());
    return J2K_OK;
    J2K_API_END
}

// The fused step runs when the band kernels take every level.
static bool rd_fused(const j2k_ctx* ctx, size_t w, size_t h, int levels, int* ws, int* hs) {
    ws[0] = (int)w;
    hs[0] = (int)h;
    for (int k = 1; k <= levels; ++k) { ws[k] = (ws[k - 1] + 1) / 2; hs[k] = (hs[k - 1] + 1) / 2; }
    return levels >= 1 && rb_levels(ctx, ws, hs, levels) == levels;
}

size_t j2k_dwt97_rd_parts(j2k_ctx* ctx, size_t w, size_t h, int levels) {
    if (!ctx || w == 0 || h == 0 || w > 65535 || h > 65535 || levels < 0 || levels > 16) return 0;
    int ws[20] = {}, hs[20] = {};
    if (rd_fused(ctx, w, h, levels, ws, hs)) return (h + RB_BH - 1) / RB_BH;
    return h < 64 ? h : 64;  // the quantiser kernels' row ranges
}

j2k_status j2k_dwt97_rd_forward(j2k_ctx* ctx, const float* x, float* y, float* u, float* d, int n, size_t w,
                                size_t h, int levels, const float* log_steps, uint64_t seed, float* rate_partials,
                                float* sq_partials) {
    J2K_API_BEGIN
    J2K_TRY(check_common(ctx, x, y, n, w, h, levels));
    if (!u || !d || !log_steps || !rate_partials || !sq_partials)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "rd forward: NULL noise, residual, log steps or partials");
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const size_t plane = w * h;
    const int nb = 3 * levels + 1;
    int ws[20] = {}, hs[20] = {};
    const int kp = (int)j2k_dwt97_rd_parts(ctx, w, h, levels);
    if (!rd_fused(ctx, w, h, levels, ws, hs)) {
        // the separate passes: forward DWT, quantiser keeping its noise (y_hat in scratch), inverse
        // with the residual
        float* yh = (float*)j2k_scratch(ctx, SCR_PLANE, plane * (size_t)n * 4 + 64);
        if (!yh) return J2K_ERR_OUT_OF_MEMORY;
        J2K_TRY(j2k_dwt_forward_batch(ctx, J2K_W97, J2K_ORDER_T800, x, w, plane, y, w, plane, n, w, h, levels, nullptr));
        J2K_TRY(quant_run(ctx, false, y, nullptr, yh, n, w, h, levels, log_steps, seed, 0.0f, nullptr, 1.0f,
                          rate_partials, kp, u));
        return j2k_dwt97_inverse_residual(ctx, yh, x, d, n, w, h, levels, sq_partials);
    }
    // forward levels with the quantiser in their band writes (y and u; rate partials), every
    // level after the first a programmatic dependent of the one before
    J2K_CUDA(ctx, cudaMemsetAsync(rate_partials, 0, (size_t)n * nb * kp * sizeof(float), st));
    const size_t zlev = (size_t)ws[1] * hs[1];
    float* s0 = (float*)j2k_scratch(ctx, SCR_LL0, zlev * n * 4 + 64);
    float* s1 = (float*)j2k_scratch(ctx, SCR_LL1, zlev * n * 4 + 64);
    if (!s0 || !s1) return J2K_ERR_OUT_OF_MEMORY;
    const float* in = x;
    size_t ip = w, iz = plane;
    for (int k = 0; k < levels; ++k) {
        const int last = k == levels - 1;
        float* lld = last ? y : (k % 2 == 0 ? s0 : s1);
        const size_t llp = last ? w : (size_t)ws[k + 1], llz = last ? plane : zlev;
        const RbQ q = rb_q(log_steps, seed, u, nullptr, 0.0f, nullptr, 1.0f, rate_partials, kp, levels, k, w);
        J2K_TRY((rb_ana_level<3, 1>(ctx, ws[k], hs[k], n, k > 0, in, ip, iz, y, w, plane, lld, llp, llz, last, q)));
        in = lld;
        ip = llp;
        iz = llz;
    }
    // inverse of y_hat = (y / step + u) * step, formed as the bands are loaded, residual at level 0
    const RbQ q = rb_q(log_steps, seed, u, nullptr, 0.0f, nullptr, 1.0f, nullptr, 0, levels, 0, w);
    return inv_residual_rb(ctx, y, x, d, n, w, h, levels, sq_partials, &q, true);
    J2K_API_END
}

j2k_status j2k_dwt97_rd_backward(j2k_ctx* ctx, const float* y, const float* u, const float* d, const float* log_steps,
                                 float lam, const float* scale, float alpha, float* g_y, float* g_x, int n, size_t w,
                                 size_t h, int levels, float* ls_partials) {
    J2K_API_BEGIN
    J2K_TRY(check_common(ctx, y, g_x, n, w, h, levels));
    if (!u || !d || !log_steps || !g_y || !ls_partials)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "rd backward: NULL noise, residual, log steps or buffers");
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const size_t plane = w * h;
    const int nb = 3 * levels + 1;
    int ws[20] = {}, hs[20] = {};
    const int kp = (int)j2k_dwt97_rd_parts(ctx, w, h, levels);
    const SynExtra ex{d, w, plane, scale, alpha, nullptr, 0};
    if (!rd_fused(ctx, w, h, levels, ws, hs)) {
        // the separate passes: inverse adjoint of d (into scratch), quantiser backward into g_y,
        // forward adjoint with the residual term
        float* gr = (float*)j2k_scratch(ctx, SCR_PLANE, plane * (size_t)n * 4 + 64);
        if (!gr) return J2K_ERR_OUT_OF_MEMORY;
        J2K_TRY(j2k_dwt97_inverse_adjoint(ctx, d, gr, n, w, h, levels));
        J2K_TRY(quant_run(ctx, true, y, gr, g_y, n, w, h, levels, log_steps, 0, lam, scale, alpha, ls_partials, kp,
                          const_cast<float*>(u)));
        return fwd_adj_run(ctx, g_y, g_x, n, w, h, levels, &ex);
    }
    // transpose of the inverse, level by level, with the quantiser backward in the band writes
    J2K_CUDA(ctx, cudaMemsetAsync(ls_partials, 0, (size_t)n * nb * kp * sizeof(float), st));
    const size_t zlev = (size_t)ws[1] * hs[1];
    float* s0 = (float*)j2k_scratch(ctx, SCR_LL0, zlev * n * 4 + 64);
    float* s1 = (float*)j2k_scratch(ctx, SCR_LL1, zlev * n * 4 + 64);
    if (!s0 || !s1) return J2K_ERR_OUT_OF_MEMORY;
    const float* in = d;
    size_t ip = w, iz = plane;
    for (int k = 0; k < levels; ++k) {
        const int last = k == levels - 1;
        float* lld = last ? g_y : (k % 2 == 0 ? s0 : s1);
        const size_t llp = last ? w : (size_t)ws[k + 1], llz = last ? plane : zlev;
        const RbQ q = rb_q(log_steps, 0, u, y, lam, scale, alpha, ls_partials, kp, levels, k, w);
        J2K_TRY((rb_ana_level<2, 2>(ctx, ws[k], hs[k], n, k > 0, in, ip, iz, g_y, w, plane, lld, llp, llz, last, q)));
        in = lld;
        ip = llp;
        iz = llz;
    }
    // transpose of the forward, with the -scale * alpha * d term at level 0
    return fwd_adj_run(ctx, g_y, g_x, n, w, h, levels, &ex);
    J2K_API_END
}

j2k_status j2k_relaxed_quant_forward(j2k_ctx* ctx, const float* y, float* y_hat, int n, size_t w, size_t h,
                                     int levels, const float* log_steps, uint64_t seed, float* rate_partials,
                                     int parts_per_band) {
    J2K_API_BEGIN
    return quant_run(ctx, false, y, nullptr, y_hat, n, w, h, levels, log_steps, seed, 0.0f, nullptr, 1.0f,
                     rate_partials, parts_per_band, nullptr);
    J2K_API_END
}

j2k_status j2k_relaxed_quant_forward_noise(j2k_ctx* ctx, const float* y, float* y_hat, float* noise, int n, size_t w,
                                           size_t h, int levels, const float* log_steps, uint64_t seed,
                                           float* rate_partials, int parts_per_band) {
    J2K_API_BEGIN
    if (!noise) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "relaxed quantiser: noise buffer is NULL");
    return quant_run(ctx, false, y, nullptr, y_hat, n, w, h, levels, log_steps, seed, 0.0f, nullptr, 1.0f,
                     rate_partials, parts_per_band, noise);
    J2K_API_END
}

j2k_status j2k_relaxed_quant_backward(j2k_ctx* ctx, const float* y, const float* g_yhat, float* g_y, int n,
                                      size_t w, size_t h, int levels, const float* log_steps, uint64_t seed,
                                      float lam, float* g_logstep_partials, int parts_per_band) {
    J2K_API_BEGIN
    return quant_run(ctx, true, y, g_yhat, g_y, n, w, h, levels, log_steps, seed, lam, nullptr, 1.0f,
                     g_logstep_partials, parts_per_band, nullptr);
    J2K_API_END
}

j2k_status j2k_relaxed_quant_backward_scaled(j2k_ctx* ctx, const float* y, const float* g_in, float* g_y, int n,
                                             size_t w, size_t h, int levels, const float* log_steps, uint64_t seed,
                                             const float* noise, float lam, const float* scale, float alpha,
                                             float* g_logstep_partials, int parts_per_band) {
    J2K_API_BEGIN
    return quant_run(ctx, true, y, g_in, g_y, n, w, h, levels, log_steps, seed, lam, scale, alpha,
                     g_logstep_partials, parts_per_band, const_cast<float*>(noise));
    J2K_API_END
}

}  // extern "C"
