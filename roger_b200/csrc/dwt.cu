// Forward and inverse 2-D lifting DWT, reversible 5/3 (int32) and irreversible 9/7 (fp32),
// one launch per decomposition level, Mallat output.
//
// Reference: src/CL/ocldwt53.cl:167-292 (5/3, rows in registers then columns in local memory,
// whole-sample symmetric extension through a MIRRORED_REPEAT sampler, :86) and
// src/CL/ocldwt97.cl:196-420 / :487-716 (9/7 with fused "quantisation"), level recursion
// src/OCLDWTForward.cpp:124-137.  Differences by design:
//   * each CTA stages a (TW+2H) x (TH+2H) tile (H = 2 for 5/3, 4 for 9/7) in shared memory,
//     extension is done by mirroring the load coordinates (parity preserving), and every lifting
//     step of both axes runs in shared memory with the tile shrinking by one sample per step;
//   * the row/column order is a template parameter: J2K_ORDER_REF (rows first, the reference)
//     or J2K_ORDER_T800 (columns first, T.800 F.4.2);
//   * odd sizes follow T.800 (ceil(n/2) low samples; a 1-sample axis is left untransformed);
//   * 9/7 arithmetic is the reference's horizontal pipeline order (ocldwt97.cl:248-310:
//     x + c*(left+right), then low*1/K, high*K after each 1-D pass) with every operation
//     rounded separately, which makes it bit-comparable with the CPU oracle;
//   * the dead-zone quantiser (T.800 E.1) is fused into the writes of the final subbands; the
//     inverse fuses the midpoint dequantiser into its loads.
// HBM roofline per level: read c*n + write c*n bytes (c = 4), n = samples of the level.
#include <algorithm>

#include <cuda.h>  // CUtensorMap (the encoder is reached through the runtime's entry points)
#include <cudaTypedefs.h>

#include "lift.cuh"
#include "mct.cuh"

namespace {

// Shared tile geometry
template <int KERN, int TW, int TH>
struct Tile {
    static constexpr int H = KT<KERN>::H;
    static constexpr int NX = TW + 2 * H, NY = TH + 2 * H;
    static constexpr int S = NX + 1;  // odd stride: column sweeps hit distinct banks
};

// One lifting step along columns (vertical): rows of the step's parity in
// [STEP+1, NY-STEP-1), columns [C0, C1).  All bounds are compile-time constants.
template <int KERN, int TW, int TH, bool INV, int STEP, int C0, int C1>
__device__ __forceinline__ void vstep(typename KT<KERN>::T* s) {
    using G = Tile<KERN, TW, TH>;
    constexpr int PAR = INV ? (STEP & 1) : 1 - (STEP & 1);
    constexpr int LO = STEP + 1, HI = G::NY - STEP - 1;
    constexpr int FIRST = LO + ((LO & 1) != PAR);
    constexpr int NR = FIRST < HI ? (HI - FIRST + 1) / 2 : 0;
    constexpr int NCOL = C1 - C0;
    for (int e = threadIdx.x; e < NR * NCOL; e += blockDim.x) {
        int r = FIRST + 2 * (e / NCOL), c = C0 + e % NCOL;
        auto* p = s + r * G::S + c;
        *p = KT<KERN>::op(INV, STEP, *p, p[-G::S], p[G::S]);
    }
}

// One lifting step along rows (horizontal): columns of the step's parity, rows [R0, R1).
template <int KERN, int TW, int TH, bool INV, int STEP, int R0, int R1>
__device__ __forceinline__ void hstep(typename KT<KERN>::T* s) {
    using G = Tile<KERN, TW, TH>;
    constexpr int PAR = INV ? (STEP & 1) : 1 - (STEP & 1);
    constexpr int LO = STEP + 1, HI = G::NX - STEP - 1;
    constexpr int FIRST = LO + ((LO & 1) != PAR);
    constexpr int NC = FIRST < HI ? (HI - FIRST + 1) / 2 : 0;
    constexpr int NROW = R1 - R0;
    for (int e = threadIdx.x; e < NROW * NC; e += blockDim.x) {
        int c = FIRST + 2 * (e % NC), r = R0 + e / NC;
        auto* p = s + r * G::S + c;
        *p = KT<KERN>::op(INV, STEP, *p, p[-1], p[1]);
    }
}

template <int KERN, int TW, int TH, bool INV, int C0, int C1, int K = 0>
__device__ __forceinline__ void vsteps(typename KT<KERN>::T* s) {
    if constexpr (K < KT<KERN>::NSTEP) {
        vstep<KERN, TW, TH, INV, K, C0, C1>(s);
        __syncthreads();
        vsteps<KERN, TW, TH, INV, C0, C1, K + 1>(s);
    }
}
template <int KERN, int TW, int TH, bool INV, int R0, int R1, int K = 0>
__device__ __forceinline__ void hsteps(typename KT<KERN>::T* s) {
    if constexpr (K < KT<KERN>::NSTEP) {
        hstep<KERN, TW, TH, INV, K, R0, R1>(s);
        __syncthreads();
        hsteps<KERN, TW, TH, INV, R0, R1, K + 1>(s);
    }
}

// 9/7 scaling sweeps (forward: low*KDIV, high*KMUL; inverse: low*KMUL, high*KDIV).
// VERT: factor by row parity, else by column parity.  Region [C0,C1) x [R0,R1).
template <int KERN, int TW, int TH, bool INV, bool VERT, int C0, int C1, int R0, int R1>
__device__ __forceinline__ void scale97(typename KT<KERN>::T* s) {
    if constexpr (KERN == 97) {
        using G = Tile<KERN, TW, TH>;
        constexpr int NCOL = C1 - C0, N = (R1 - R0) * NCOL;
        for (int e = threadIdx.x; e < N; e += blockDim.x) {
            int r = R0 + e / NCOL, c = C0 + e % NCOL;
            int odd = VERT ? (r & 1) : (c & 1);
            float f = odd ? (INV ? KDIV : KMUL) : (INV ? KMUL : KDIV);
            s[r * G::S + c] = __fmul_rn(s[r * G::S + c], f);
        }
        __syncthreads();
    }
}

// ---- forward level ----------------------------------------------------------------------------
// src: level input (w x h).  Detail subbands go to dst at Mallat positions (dst is the full
// output plane); LL goes to ll_dst (T) unless QLL, in which case it is quantised into dst.
template <int KERN, int ORDER, int TW, int TH, typename TD, bool QUANT, bool QLL>
__device__ __forceinline__ void fwd_tile(typename KT<KERN>::T* s, const typename KT<KERN>::T* __restrict__ src,
                                         size_t spitch, int w, int h, typename KT<KERN>::T* __restrict__ ll_dst,
                                         size_t llpitch, TD* __restrict__ dst, size_t dpitch, Steps4 st, int x0,
                                         int y0) {
    using T = typename KT<KERN>::T;
    using G = Tile<KERN, TW, TH>;
    constexpr int H = G::H;
    for (int e = threadIdx.x; e < G::NX * G::NY; e += blockDim.x) {
        int r = e / G::NX, c = e % G::NX;
        int gy = mirror(y0 - H + r, h), gx = mirror(x0 - H + c, w);
        s[r * G::S + c] = __ldcg(src + (size_t)gy * spitch + gx);  // L2 only, as fwd_fast_tile_reg
    }
    __syncthreads();
    const bool dov = h > 1, doh = w > 1;
    if (ORDER == J2K_ORDER_T800) {
        if (dov) {
            vsteps<KERN, TW, TH, false, 0, G::NX>(s);
            scale97<KERN, TW, TH, false, true, 0, G::NX, H, H + TH>(s);
        }
        if (doh) hsteps<KERN, TW, TH, false, H, H + TH>(s);
    } else {
        if (doh) {
            hsteps<KERN, TW, TH, false, 0, G::NY>(s);
            scale97<KERN, TW, TH, false, false, H, H + TW, 0, G::NY>(s);
        }
        if (dov) vsteps<KERN, TW, TH, false, H, H + TW>(s);
    }
    // write the four subbands; the second pass's scaling is applied here
    const int wl = (w + 1) >> 1, hl = (h + 1) >> 1;
    constexpr int SW = TW / 2, SH = TH / 2;
#pragma unroll 1
    for (int q = 0; q < 4; ++q) {
        const int qx = q & 1, qy = q >> 1;
        float f = 1.0f;
        if (KERN == 97) {
            if (ORDER == J2K_ORDER_T800) f = doh ? (qx ? KMUL : KDIV) : 1.0f;
            else f = dov ? (qy ? KMUL : KDIV) : 1.0f;
        }
        const float step = q == 0 ? st.ll : (q == 1 ? st.hl : (q == 2 ? st.lh : st.hh));
        for (int e = threadIdx.x; e < SW * SH; e += blockDim.x) {
            int i = e % SW, j = e / SW;
            int x = x0 + 2 * i + qx, y = y0 + 2 * j + qy;
            if (x >= w || y >= h) continue;
            T v = s[(H + 2 * j + qy) * G::S + H + 2 * i + qx];
            if (KERN == 97) v = (T)__fmul_rn((float)v, f);
            int sx = (x >> 1) + (qx ? wl : 0), sy = (y >> 1) + (qy ? hl : 0);
            if (q == 0 && !QLL) {
                ll_dst[(size_t)sy * llpitch + sx] = v;
            } else if (QUANT) {
                dst[(size_t)sy * dpitch + sx] = (TD)quantize((float)v, step);
            } else {
                dst[(size_t)sy * dpitch + sx] = (TD)v;
            }
        }
    }
}

template <int KERN, int ORDER, int TW, int TH, typename TD, bool QUANT, bool QLL>
__global__ void __launch_bounds__(256)
dwt_fwd_level(const typename KT<KERN>::T* __restrict__ src, size_t spitch, int w, int h,
              typename KT<KERN>::T* __restrict__ ll_dst, size_t llpitch, TD* __restrict__ dst,
              size_t dpitch, Steps4 st, ZStride z) {
    using G = Tile<KERN, TW, TH>;
    __shared__ typename KT<KERN>::T s[G::NY * G::S];
    src += blockIdx.z * z.src;
    dst += blockIdx.z * z.dst;
    ll_dst += blockIdx.z * z.ll;
    fwd_tile<KERN, ORDER, TW, TH, TD, QUANT, QLL>(s, src, spitch, w, h, ll_dst, llpitch, dst, dpitch, st,
                                                 blockIdx.x * TW, blockIdx.y * TH);
}

// Batched forward level: CTA b takes tile b of a flattened tile list covering many images
// (owner[b] = image slot, tiles numbered row-major within each image from d.tile0).
template <int KERN, int ORDER, int TW, int TH>
__global__ void __launch_bounds__(256)
dwt_fwd_batched(const j2k_dwt_level_desc* __restrict__ descs, const uint32_t* __restrict__ owner) {
    using T = typename KT<KERN>::T;
    using G = Tile<KERN, TW, TH>;
    __shared__ T s[G::NY * G::S];
    const j2k_dwt_level_desc d = descs[owner[blockIdx.x]];
    const int t = (int)(blockIdx.x - d.tile0);
    const int x0 = (t % d.tiles_x) * TW, y0 = (t / d.tiles_x) * TH;
    const Steps4 st{d.s_ll, d.s_hl, d.s_lh, d.s_hh};
    if (KERN == 97 && (d.flags & 1)) {
        if (d.flags & 2)
            fwd_tile<KERN, ORDER, TW, TH, int32_t, true, true>(s, (const T*)d.src, d.spitch, d.w, d.h, (T*)d.ll_dst,
                                                                d.llpitch, (int32_t*)d.dst, d.dpitch, st, x0, y0);
        else
            fwd_tile<KERN, ORDER, TW, TH, int32_t, true, false>(s, (const T*)d.src, d.spitch, d.w, d.h, (T*)d.ll_dst,
                                                                 d.llpitch, (int32_t*)d.dst, d.dpitch, st, x0, y0);
    } else {
        fwd_tile<KERN, ORDER, TW, TH, T, false, false>(s, (const T*)d.src, d.spitch, d.w, d.h, (T*)d.ll_dst,
                                                        d.llpitch, (T*)d.dst, d.dpitch, st, x0, y0);
    }
}

// ---- fast forward level (T.800 order) ------------------------------------------------------------
// One CTA produces a 248 x 32 tile of level outputs from a 256-column x (32 + 2*HV)-row strip:
//   * rows are loaded with 16-byte vectors (mirrored scalar loads only where the strip leaves
//     the image), columns x0-4 .. x0+251;
//   * the vertical lifting runs in registers, one thread per column, the whole column unrolled;
//   * the horizontal lifting runs in registers, 8 samples per lane, neighbours exchanged with
//     warp shuffles (the 4-column halo absorbs the missing neighbours at the warp ends);
//   * subbands are written straight from registers (8-byte vectors when aligned).
// Same arithmetic, operation order and rounding as dwt_fwd_level, so the outputs are identical.

// Step 3 of the fast forward level: horizontal lifting of the FTH vertically lifted rows held in
// shared memory (strip row r at s[r - RO]), 8 samples per lane (tile columns 8*lane ..
// 8*lane+7), and the writes of the four subbands (dead-zone indices when QUANT) straight from
// registers.  Shared by the register-load and the TMA-staged forms of the level kernel.
template <int KERN, typename TD, bool QUANT, bool QLL, int FTH, int RO>
__device__ __forceinline__ void fwd_fast_rows(typename KT<KERN>::T (*s)[FNX], int x0, int y0, int w, int h,
                                              typename KT<KERN>::T* __restrict__ ll_dst, size_t llpitch,
                                              TD* __restrict__ dst, size_t dpitch, Steps4 st, int vec_out) {
    using T = typename KT<KERN>::T;
    constexpr int HV = KT<KERN>::H;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wl = (w + 1) >> 1, hl = (h + 1) >> 1;
    const bool doh = w > 1;
#pragma unroll
    for (int i = 0; i < FTH / 8; ++i) {
        const int r = HV + warp + 8 * i;
        const int y = y0 + r - HV;
        if (y >= h) break;
        T v[8];
        *reinterpret_cast<uint4*>(&v[0]) = *reinterpret_cast<const uint4*>(&s[r - RO][8 * lane]);
        *reinterpret_cast<uint4*>(&v[4]) = *reinterpret_cast<const uint4*>(&s[r - RO][8 * lane + 4]);
        if (doh) {
#pragma unroll
            for (int k = 0; k < KT<KERN>::NSTEP; ++k) {
                if ((k & 1) == 0) {  // odd samples from their even neighbours
                    const T nx = __shfl_down_sync(0xffffffffu, v[0], 1);
                    v[1] = KT<KERN>::op(false, k, v[1], v[0], v[2]);
                    v[3] = KT<KERN>::op(false, k, v[3], v[2], v[4]);
                    v[5] = KT<KERN>::op(false, k, v[5], v[4], v[6]);
                    v[7] = KT<KERN>::op(false, k, v[7], v[6], nx);
                } else {             // even samples from their odd neighbours
                    const T pv = __shfl_up_sync(0xffffffffu, v[7], 1);
                    v[0] = KT<KERN>::op(false, k, v[0], pv, v[1]);
                    v[2] = KT<KERN>::op(false, k, v[2], v[1], v[3]);
                    v[4] = KT<KERN>::op(false, k, v[4], v[3], v[5]);
                    v[6] = KT<KERN>::op(false, k, v[6], v[5], v[7]);
                }
            }
            if (KERN == 97) {
#pragma unroll
                for (int j = 0; j < 8; ++j) v[j] = (T)__fmul_rn((float)v[j], (j & 1) ? KMUL : KDIV);
            }
        }
        // subband rows: even y -> LL / HL, odd y -> LH / HH
        const int qy = y & 1;
        const int sy = (y >> 1) + (qy ? hl : 0);
        const int xs = x0 - 4 + 8 * lane;  // absolute x of v[0] (even)
#pragma unroll
        for (int half = 0; half < 2; ++half) {  // samples v[4*half .. 4*half+3]
            const int e0 = 8 * lane + 4 * half;  // tile column of the first sample
            const int xa = xs + 4 * half;
            if (e0 + 4 <= 4 || e0 >= 252) continue;  // halo columns
            for (int qx = 0; qx < 2; ++qx) {
                const bool isll = (qx == 0 && qy == 0);
                T a = v[4 * half + qx], b = v[4 * half + 2 + qx];
                const int sx = (xa >> 1) + (qx ? wl : 0);  // band index of a (b is sx+1)
                const bool va = xa + qx < w, vb = xa + 2 + qx < w;
                if (isll && !QLL) {
                    T* p = ll_dst + (size_t)sy * llpitch + sx;
                    if (vec_out && va && vb) {
                        T pr[2] = {a, b};
                        *reinterpret_cast<uint2*>(p) = *reinterpret_cast<uint2*>(pr);
                    } else {
                        if (va) p[0] = a;
                        if (vb) p[1] = b;
                    }
                } else {
                    const float step = isll ? st.ll : (qx && qy ? st.hh : (qx ? st.hl : st.lh));
                    TD oa, ob;
                    if (QUANT) {
                        oa = (TD)quantize((float)a, step);
                        ob = (TD)quantize((float)b, step);
                    } else {
                        oa = (TD)a;
                        ob = (TD)b;
                    }
                    TD* p = dst + (size_t)sy * dpitch + sx;
                    if (vec_out && va && vb && ((sx & 1) == 0)) {
                        TD pr[2] = {oa, ob};
                        *reinterpret_cast<uint2*>(p) = *reinterpret_cast<uint2*>(pr);
                    } else {
                        if (va) p[0] = oa;
                        if (vb) p[1] = ob;
                    }
                }
            }
        }
    }
}

// One 248 x FTH output tile of a forward level in the register-load form: each thread loads its
// column of the strip (columns x0-4 .. x0+251, rows y0-HV .. y0+FTH+HV-1, mirrored at the image
// edges) straight into registers, lifts it vertically there, and the FTH lifted rows go through
// s (FTH x FNX) to the horizontal pass and the subband writes (fwd_fast_rows).
template <int KERN, typename TD, bool QUANT, bool QLL, int FTH>
__device__ __forceinline__ void fwd_fast_tile_reg(typename KT<KERN>::T (*s)[FNX],
                                                  const typename KT<KERN>::T* __restrict__ src, size_t spitch,
                                                  int w, int h, typename KT<KERN>::T* __restrict__ ll_dst,
                                                  size_t llpitch, TD* __restrict__ dst, size_t dpitch, Steps4 st,
                                                  int vec_out, int x0, int y0) {
    using T = typename KT<KERN>::T;
    constexpr int HV = KT<KERN>::H, NY = FTH + 2 * HV;
    const int t = threadIdx.x;
    const bool inner_x = (x0 - 4 >= 0) && (x0 + 252 <= w);
    const bool inner_y = (y0 - HV >= 0) && (y0 + FTH + HV <= h);
    T c[NY];
    // 1. column t of the strip.  Loads cached in L2 only: a level launched as a programmatic
    // dependent may start while the previous level still runs on the same SMs, so lines of
    // its input buffer that an earlier level read could still sit in an SM's L1
    const int gx = x0 - 4 + t;
    const T* colp = src + (inner_x ? gx : mirror(gx, w));
#pragma unroll
    for (int r = 0; r < NY; ++r) {
        const int gy = inner_y ? y0 - HV + r : mirror(y0 - HV + r, h);
        c[r] = __ldcg(colp + (size_t)gy * spitch);
    }
    // 2. vertical lifting of column t in registers
    if (h > 1) {
#pragma unroll
        for (int k = 0; k < KT<KERN>::NSTEP; ++k) {
            const int par = 1 - (k & 1);
#pragma unroll
            for (int r = k + 1; r < NY - k - 1; ++r)
                if ((r & 1) == par) c[r] = KT<KERN>::op(false, k, c[r], c[r - 1], c[r + 1]);
        }
    }
#pragma unroll
    for (int r = HV; r < HV + FTH; ++r) {
        T v = c[r];
        if (KERN == 97 && h > 1) v = (T)__fmul_rn((float)v, (r & 1) ? KMUL : KDIV);
        s[r - HV][t] = v;
    }
    __syncthreads();
    // 3. horizontal lifting and the subband writes
    fwd_fast_rows<KERN, TD, QUANT, QLL, FTH, HV>(s, x0, y0, w, h, ll_dst, llpitch, dst, dpitch, st, vec_out);
}

// REG: each thread loads its column of the strip straight from global memory into registers
// (coalesced 4-byte loads, all NY in flight at once), so the strip is never staged in shared
// memory; only the FTH vertically lifted rows go through shared memory to the horizontal pass.
template <int KERN, typename TD, bool QUANT, bool QLL, int FTH, bool REG>
__global__ void __launch_bounds__(256, REG ? (FTH == 16 ? 6 : 4) : ((KERN == 53 && FTH == 16) ? 8 : 6))
dwt_fwd_fast(const typename KT<KERN>::T* __restrict__ src, size_t spitch, int w, int h,
             typename KT<KERN>::T* __restrict__ ll_dst, size_t llpitch, TD* __restrict__ dst, size_t dpitch,
             Steps4 st, int vec_out, ZStride z) {
    using T = typename KT<KERN>::T;
    griddep_launch_dependents();
    griddep_wait();  // a level launched as a dependent reads the previous level's LL band
    src += blockIdx.z * z.src;
    dst += blockIdx.z * z.dst;
    ll_dst += blockIdx.z * z.ll;
    constexpr int HV = KT<KERN>::H, NY = FTH + 2 * HV;
    constexpr int SR = REG ? FTH : NY, RO = REG ? HV : 0;  // shared rows; strip row r at s[r - RO]
    __shared__ __align__(16) T s[SR][FNX];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, t = threadIdx.x;
    const int x0 = blockIdx.x * FTW, y0 = blockIdx.y * FTH;
    if constexpr (REG) {
        fwd_fast_tile_reg<KERN, TD, QUANT, QLL, FTH>(s, src, spitch, w, h, ll_dst, llpitch, dst, dpitch, st,
                                                     vec_out, x0, y0);
        return;
    }
    const bool inner_x = (x0 - 4 >= 0) && (x0 + 252 <= w);
    T c[NY];
    {
        // 1. load the strip: every copy of the CTA in flight at once (cp.async, no register staging)
        for (int r = warp; r < NY; r += 8) {
            const T* row = src + (size_t)mirror(y0 - HV + r, h) * spitch;
#pragma unroll
            for (int q2 = 0; q2 < 2; ++q2) {
                const int q = lane + 32 * q2;
                const int gx = x0 - 4 + 4 * q;
                if (inner_x) {
                    cp_async16(&s[r][4 * q], row + gx);
                } else {
#pragma unroll
                    for (int k = 0; k < 4; ++k) cp_async4(&s[r][4 * q + k], row + mirror(gx + k, w));
                }
            }
        }
        cp_async_wait_all();
        __syncthreads();
#pragma unroll
        for (int r = 0; r < NY; ++r) c[r] = s[r][t];
        __syncthreads();
    }
    // 2. vertical lifting of column t in registers
    if (h > 1) {
#pragma unroll
        for (int k = 0; k < KT<KERN>::NSTEP; ++k) {
            const int par = 1 - (k & 1);
#pragma unroll
            for (int r = k + 1; r < NY - k - 1; ++r)
                if ((r & 1) == par) c[r] = KT<KERN>::op(false, k, c[r], c[r - 1], c[r + 1]);
        }
    }
#pragma unroll
    for (int r = HV; r < HV + FTH; ++r) {
        T v = c[r];
        if (KERN == 97 && h > 1) v = (T)__fmul_rn((float)v, (r & 1) ? KMUL : KDIV);
        s[r - RO][t] = v;
    }
    __syncthreads();
    // 3. horizontal lifting and the subband writes
    fwd_fast_rows<KERN, TD, QUANT, QLL, FTH, RO>(s, x0, y0, w, h, ll_dst, llpitch, dst, dpitch, st, vec_out);
}

// ---- first level straight from interleaved 8-bit pixels -----------------------------------------
// Level 0 of NC components (1: gray, 3: colour) read from the pixels themselves.  CTA x takes
// component x % NC of tile x / NC, so the NC CTAs of a tile run side by side and the two that come
// second find the tile's pixel lines in L2.  The strip's rows (NC * 256 bytes each, for columns
// x0-4 .. x0+251) come in as aligned 32-bit words, every word of the strip requested before any is
// used, and go to shared memory; a tile whose strip leaves the image at the left or right edge
// loads its mirrored columns byte by byte instead.  Each thread then forms the level-shifted,
// colour-transformed samples of its column and component in registers (mct_component: the planar
// split's arithmetic) and runs the tile of dwt_fwd_fast on them (vertical lifting in registers,
// horizontal lifting and the subband writes in fwd_fast_rows).  The component planes are never
// stored: per pixel the level reads NC bytes where the planar split wrote, and the level read
// back, 4 NC bytes.  Component c writes dst + c * dst_z and ll_dst + c * ll_z.
// It is an encoder option (J2K_TUNE_DWT_PX), off by default: the plane kernel is issue-bound
// already, and this one moves a third of the bytes in 2.4x the instructions (176 us for the
// 4096x4096 RGB level 0, against 45 + 85 us for the planar split and the level over the planes).
// Words are read only where they hold a byte of the row's strip; such an aligned word never
// leaves the page of that byte.
template <int KERN, int NC, int MCT, typename TD, bool QUANT, bool QLL>
__global__ void __launch_bounds__(256, 6)
dwt_fwd_fast_px(const uint8_t* __restrict__ px, size_t pitch, int w, int h, typename KT<KERN>::T* __restrict__ ll_dst,
                size_t llpitch, size_t ll_z, TD* __restrict__ dst, size_t dpitch, size_t dst_z, Steps4 st,
                int vec_out) {
    using T = typename KT<KERN>::T;
    constexpr int FTH = 16, HV = KT<KERN>::H, NY = FTH + 2 * HV;
    constexpr int RW = (NC * FNX) / 4 + 1;  // words per strip row: NC * 256 bytes from any byte offset
    __shared__ __align__(16) T s[FTH][FNX];
    __shared__ uint32_t rows[NY][RW];
    __shared__ int lead[NY];                // byte offset of column x0-4 in each row's first word
    const int t = threadIdx.x;
    const int c = (int)(blockIdx.x % NC);
    const int x0 = (int)(blockIdx.x / NC) * FTW, y0 = blockIdx.y * FTH;
    const bool inner_x = (x0 - 4 >= 0) && (x0 + 252 <= w);
    const bool inner_y = (y0 - HV >= 0) && (y0 + FTH + HV <= h);
    T col[NY];
    if (inner_x) {
        // words of row r: from the one holding byte b0 = gy * pitch + NC * (x0 - 4) to the one
        // holding b0 + NC * 256 - 1 (each holds at least one byte of the row's strip)
        const uint8_t* base = px + (size_t)NC * (x0 - 4);
#pragma unroll 4
        for (int i = t; i < NY * RW; i += 256) {
            const int r = i / RW, k = i % RW;
            const int gy = inner_y ? y0 - HV + r : mirror(y0 - HV + r, h);
            const uintptr_t b0 = (uintptr_t)(base + (size_t)gy * pitch);
            const uintptr_t a0 = b0 & ~(uintptr_t)3;
            if (a0 + 4 * (uintptr_t)k <= b0 + NC * FNX - 1) rows[r][k] = __ldg(reinterpret_cast<const uint32_t*>(a0) + k);
            if (k == 0) lead[r] = (int)(b0 & 3);
        }
        __syncthreads();
        const uint8_t* rb = reinterpret_cast<const uint8_t*>(&rows[0][0]);
#pragma unroll
        for (int r = 0; r < NY; ++r) {
            const uint8_t* q = rb + r * RW * 4 + lead[r] + NC * t;
            uint32_t v = q[0];
            if constexpr (NC == 3) v |= ((uint32_t)q[1] << 8) | ((uint32_t)q[2] << 16);
            col[r] = mct_component<T, NC, MCT>(v, c);
        }
    } else {
        const uint8_t* colp = px + (size_t)mirror(x0 - 4 + t, w) * NC;
#pragma unroll
        for (int r = 0; r < NY; ++r) {
            const int gy = inner_y ? y0 - HV + r : mirror(y0 - HV + r, h);
            const uint8_t* p = colp + (size_t)gy * pitch;
            uint32_t v = __ldg(p);
            if constexpr (NC == 3) v |= ((uint32_t)__ldg(p + 1) << 8) | ((uint32_t)__ldg(p + 2) << 16);
            col[r] = mct_component<T, NC, MCT>(v, c);
        }
    }
    if (h > 1) {
#pragma unroll
        for (int k = 0; k < KT<KERN>::NSTEP; ++k) {
            const int par = 1 - (k & 1);
#pragma unroll
            for (int r = k + 1; r < NY - k - 1; ++r)
                if ((r & 1) == par) col[r] = KT<KERN>::op(false, k, col[r], col[r - 1], col[r + 1]);
        }
    }
#pragma unroll
    for (int r = HV; r < HV + FTH; ++r) {
        T v = col[r];
        if (KERN == 97 && h > 1) v = (T)__fmul_rn((float)v, (r & 1) ? KMUL : KDIV);
        s[r - HV][t] = v;
    }
    __syncthreads();
    fwd_fast_rows<KERN, TD, QUANT, QLL, FTH, HV>(s, x0, y0, w, h, ll_dst + c * ll_z, llpitch, dst + c * dst_z, dpitch,
                                                 st, vec_out);
}

// The batched level in the register-lifting form (T.800 order): CTA b takes tile b - d.tile0 of
// its image's level (248 output columns x 16 rows, tiles row-major), and runs the same tile as
// dwt_fwd_fast.  A level narrower than 8 or lower than 2 samples takes the shared-memory tile
// instead (fwd_tile, 64 x 16 sub-tiles over the CTA's 248 x 16 region).  The descriptor's flags:
// 1 quantise the details (9/7), 2 last level (LL quantised into dst), 4 8-byte vector stores.
constexpr int kBatchFastTh = 16;

template <int KERN>
__global__ void __launch_bounds__(256, 6)
dwt_fwd_batched_fast(const j2k_dwt_level_desc* __restrict__ descs, const uint32_t* __restrict__ owner) {
    using T = typename KT<KERN>::T;
    __shared__ __align__(16) T s[kBatchFastTh][FNX];
    griddep_launch_dependents();
    griddep_wait();  // a level launched as a dependent reads the previous level's LL band
    const j2k_dwt_level_desc d = descs[owner[blockIdx.x]];
    const int t = (int)(blockIdx.x - d.tile0);
    const int x0 = (t % d.tiles_x) * FTW, y0 = (t / d.tiles_x) * kBatchFastTh;
    const Steps4 st{d.s_ll, d.s_hl, d.s_lh, d.s_hh};
    const int vec = (d.flags >> 2) & 1;
    const T* src = (const T*)d.src;
    T* lld = (T*)d.ll_dst;
    if (d.w < 8 || d.h < 2) {
        using G = Tile<KERN, 64, kBatchFastTh>;
        T* ts = reinterpret_cast<T*>(&s[0][0]);
        static_assert(G::NY * G::S <= kBatchFastTh * FNX, "fallback tile must fit the shared rows");
        for (int sx = x0; sx < x0 + FTW && sx < d.w; sx += 64) {
            if (KERN == 97 && (d.flags & 1)) {
                if (d.flags & 2)
                    fwd_tile<KERN, J2K_ORDER_T800, 64, kBatchFastTh, int32_t, true, true>(
                        ts, src, d.spitch, d.w, d.h, lld, d.llpitch, (int32_t*)d.dst, d.dpitch, st, sx, y0);
                else
                    fwd_tile<KERN, J2K_ORDER_T800, 64, kBatchFastTh, int32_t, true, false>(
                        ts, src, d.spitch, d.w, d.h, lld, d.llpitch, (int32_t*)d.dst, d.dpitch, st, sx, y0);
            } else {
                fwd_tile<KERN, J2K_ORDER_T800, 64, kBatchFastTh, T, false, false>(
                    ts, src, d.spitch, d.w, d.h, lld, d.llpitch, (T*)d.dst, d.dpitch, st, sx, y0);
            }
            __syncthreads();
        }
        return;
    }
    if (KERN == 97 && (d.flags & 1)) {
        if (d.flags & 2)
            fwd_fast_tile_reg<KERN, int32_t, true, true, kBatchFastTh>(s, src, d.spitch, d.w, d.h, lld, d.llpitch,
                                                                      (int32_t*)d.dst, d.dpitch, st, vec, x0, y0);
        else
            fwd_fast_tile_reg<KERN, int32_t, true, false, kBatchFastTh>(s, src, d.spitch, d.w, d.h, lld, d.llpitch,
                                                                       (int32_t*)d.dst, d.dpitch, st, vec, x0, y0);
    } else {
        fwd_fast_tile_reg<KERN, T, false, false, kBatchFastTh>(s, src, d.spitch, d.w, d.h, lld, d.llpitch, (T*)d.dst,
                                                              d.dpitch, st, vec, x0, y0);
    }
}

// ---- fused deep levels ---------------------------------------------------------------------------
// The deep levels of a forward transform are under one wave each (config 1's levels 3-5: 96 to 24
// CTAs), so each costs a tile's latency plus a launch.  dwt_fwd_tail runs levels k0 .. k1-1 in one
// cooperative launch: every CTA takes tiles of a level in turn (the register-lifting tile of
// dwt_fwd_fast), then all CTAs meet at a grid barrier before the next level reads the LL band
// they wrote.  The barrier is an arrival counter and a generation word in global memory; a CTA
// waits for the generation with a bounded spin and, when the bound runs out, sets the timeout
// error and leaves.  Loads are L2-only (fwd_fast_tile_reg), so no SM reads a stale L1 line of
// the band the level before wrote.
constexpr int kTailLevels = 8;
struct TailLevel {
    const void* src;
    void* lld;
    size_t spitch, llp, src_z, ll_z;
    int w, h, tiles_x, tiles_y, vec, last;
    Steps4 st;
};
struct TailPlan {
    TailLevel lv[kTailLevels];
    int nlev, nz;
};

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// All CTAs of the (co-resident) grid; false when the wait for the others gave up.
__device__ __forceinline__ bool tail_barrier(uint32_t* bar, uint32_t gen) {
    __syncthreads();
    int ok = 1;
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t arrived = atomicAdd(&bar[0], 1u) + 1u;
        if (arrived == gridDim.x) {
            atomicExch(&bar[0], 0u);
            __threadfence();
            atomicAdd(&bar[1], 1u);
        } else {
            int spin = 0;
            while (ld_acquire_u32(&bar[1]) < gen && spin < (1 << 22)) ++spin;
            ok = spin < (1 << 22);
        }
    }
    return __syncthreads_and(ok) != 0;
}

template <int KERN, bool QUANT>
__global__ void __launch_bounds__(256, 4)
dwt_fwd_tail(const TailPlan plan, void* __restrict__ dst, size_t dpitch, size_t dst_z, uint32_t* __restrict__ bar,
             uint32_t* __restrict__ err) {
    using T = typename KT<KERN>::T;
    __shared__ __align__(16) T s[16][FNX];
    for (int li = 0; li < plan.nlev; ++li) {
        const TailLevel& L = plan.lv[li];
        const int per = L.tiles_x * L.tiles_y, ntiles = per * plan.nz;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
            const int tz = tile / per, r = tile % per;
            const int x0 = (r % L.tiles_x) * FTW, y0 = (r / L.tiles_x) * 16;
            const T* src = (const T*)L.src + tz * L.src_z;
            T* lld = (T*)L.lld + tz * L.ll_z;
            if (QUANT && L.last)
                fwd_fast_tile_reg<KERN, int32_t, true, true, 16>(s, src, L.spitch, L.w, L.h, lld, L.llp,
                                                                 (int32_t*)dst + tz * dst_z, dpitch, L.st, L.vec, x0,
                                                                 y0);
            else if (QUANT)
                fwd_fast_tile_reg<KERN, int32_t, true, false, 16>(s, src, L.spitch, L.w, L.h, lld, L.llp,
                                                                  (int32_t*)dst + tz * dst_z, dpitch, L.st, L.vec, x0,
                                                                  y0);
            else
                fwd_fast_tile_reg<KERN, T, false, false, 16>(s, src, L.spitch, L.w, L.h, lld, L.llp,
                                                             (T*)dst + tz * dst_z, dpitch, L.st, L.vec, x0, y0);
            __syncthreads();  // s is reused by the next tile
        }
        if (li + 1 < plan.nlev && !tail_barrier(bar, (uint32_t)li + 1u)) {
            if (threadIdx.x == 0) atomicCAS(err, 0u, (uint32_t)J2K_DEVERR_TIMEOUT);
            return;
        }
    }
}

// The same deep levels with one thread-block cluster per plane (cluster size = gridDim.x, plane =
// blockIdx.z): CTA r of a cluster takes tiles r, r + gridDim.x, ... of its plane's level, and the
// cluster's hardware barrier (arrive.release / wait.acquire at cluster scope, after a fence) sits
// between levels, so no global counter is spun on.  Every CTA of a cluster runs every level and
// every barrier (the plan is a kernel parameter and there is no early exit), and the CTAs of a
// cluster are scheduled together, so each barrier is reached by all of them.
__device__ __forceinline__ void cluster_barrier_rel_acq() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

template <int KERN, bool QUANT>
__global__ void __launch_bounds__(256)
dwt_fwd_ctail(const TailPlan plan, void* __restrict__ dst, size_t dpitch, size_t dst_z) {
    using T = typename KT<KERN>::T;
    __shared__ __align__(16) T s[16][FNX];
    griddep_launch_dependents();
    griddep_wait();  // launched as a dependent: the level before has finished and its LL is visible
    const int tz = blockIdx.z, cs = (int)gridDim.x;
    for (int li = 0; li < plan.nlev; ++li) {
        const TailLevel& L = plan.lv[li];
        const int per = L.tiles_x * L.tiles_y;
        const T* src = (const T*)L.src + tz * L.src_z;
        T* lld = (T*)L.lld + tz * L.ll_z;
        for (int r = (int)blockIdx.x; r < per; r += cs) {
            const int x0 = (r % L.tiles_x) * FTW, y0 = (r / L.tiles_x) * 16;
            if (QUANT && L.last)
                fwd_fast_tile_reg<KERN, int32_t, true, true, 16>(s, src, L.spitch, L.w, L.h, lld, L.llp,
                                                                 (int32_t*)dst + tz * dst_z, dpitch, L.st, L.vec, x0,
                                                                 y0);
            else if (QUANT)
                fwd_fast_tile_reg<KERN, int32_t, true, false, 16>(s, src, L.spitch, L.w, L.h, lld, L.llp,
                                                                  (int32_t*)dst + tz * dst_z, dpitch, L.st, L.vec, x0,
                                                                  y0);
            else
                fwd_fast_tile_reg<KERN, T, false, false, 16>(s, src, L.spitch, L.w, L.h, lld, L.llp,
                                                             (T*)dst + tz * dst_z, dpitch, L.st, L.vec, x0, y0);
            __syncthreads();  // s is reused by the next tile
        }
        if (li + 1 < plan.nlev) {
            __threadfence();
            __syncthreads();
            cluster_barrier_rel_acq();
        }
    }
}

// ---- TMA-staged forward level -----------------------------------------------------------------
// Persistent CTAs walk the tiles (248 output columns x 16 rows of one plane) in a fixed order.
// A tile's strip (256 columns x 16 + 2*HV rows, halo included) comes into shared memory by one
// tensor copy (cp.async.bulk.tensor, TMA) that one thread issues, two stages deep: the next
// tile's copy is in flight while the current tile is lifted.  Strip samples outside the plane
// arrive as zeros and are never used: every thread reads its column through the mirror map
// (whole-sample symmetric extension), and the mirrored sample of every row and column an output
// depends on lies inside the strip.  Vertical lifting then runs per column in registers, the
// lifted rows go back into the strip in place, and the horizontal pass is fwd_fast_rows on the
// strip, as in dwt_fwd_fast, so the outputs are identical.  Shared memory is the two strips
// alone (40 KB for 5/3, 48 KB for 9/7).  No multicast: each copy reads this GPU's plane into this
// CTA's shared memory.
constexpr int kTmaTh = 16;

template <int KERN>
struct TmaStrip {
    static constexpr int NY = kTmaTh + 2 * KT<KERN>::H;
    static constexpr int BYTES = NY * FNX * 4;
    static constexpr int SMEM = 2 * BYTES + 16;  // two strips, two barriers
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

template <int KERN, typename TD, bool QUANT, bool QLL>
__global__ void __launch_bounds__(256)
dwt_fwd_tma(const __grid_constant__ CUtensorMap tmap, int w, int h, int nz, int tiles_x, int tiles_y,
            typename KT<KERN>::T* __restrict__ ll_dst, size_t llpitch, TD* __restrict__ dst, size_t dpitch,
            Steps4 st, int vec_out, ZStride z, uint32_t* __restrict__ err) {
    using T = typename KT<KERN>::T;
    constexpr int HV = KT<KERN>::H, NY = TmaStrip<KERN>::NY;
    extern __shared__ __align__(128) unsigned char dsm[];
    T(*stg)[NY][FNX] = reinterpret_cast<T(*)[NY][FNX]>(dsm);                             // [2][NY][FNX]
    uint64_t* bar = reinterpret_cast<uint64_t*>(dsm + 2 * TmaStrip<KERN>::BYTES);  // [2]
    const int t = threadIdx.x;
    const int ntiles = tiles_x * tiles_y * nz;
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    griddep_launch_dependents();
    griddep_wait();  // a level launched as a dependent reads the previous level's LL band
    auto issue = [&](int tile, int stage) {
        const int tx = tile % tiles_x, rest = tile / tiles_x;
        const int ty = rest % tiles_y, tz = rest / tiles_y;
        const int x = tx * FTW - 4, y = ty * kTmaTh - HV;  // x a multiple of 4: 16-byte aligned
        const uint32_t b = smem_u32(&bar[stage]);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b),
                     "r"((uint32_t)TmaStrip<KERN>::BYTES)
                     : "memory");
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
            "[%5];" ::"r"(smem_u32(&stg[stage][0][0])),
            "l"(reinterpret_cast<uint64_t>(&tmap)), "r"(x), "r"(y), "r"(tz), "r"(b)
            : "memory");
    };
    if (t == 0 && (int)blockIdx.x < ntiles) issue(blockIdx.x, 0);
    int it = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
        const int stage = it & 1;
        if (t == 0 && tile + (int)gridDim.x < ntiles) issue(tile + gridDim.x, stage ^ 1);
        // this tile's strip: wait on its barrier's phase (bounded; a copy that never lands
        // sets the timeout error and the CTA leaves)
        auto wait_bar = [&](int sg, uint32_t par) -> bool {
            const uint32_t b = smem_u32(&bar[sg]);
            uint32_t ok = 0;
            for (int spin = 0; spin < (1 << 22) && !ok; ++spin)
                asm volatile(
                    "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                    : "=r"(ok)
                    : "r"(b), "r"(par)
                    : "memory");
            return ok != 0;
        };
        if (__syncthreads_or(!wait_bar(stage, (uint32_t)(it >> 1) & 1u))) {
            // the whole CTA leaves together; first the copy of the next tile, if one was
            // issued, is waited for (bounded), so that nothing lands after the CTA is gone
            if (t == 0) {
                atomicCAS(err, 0u, (uint32_t)J2K_DEVERR_TIMEOUT);
                if (tile + (int)gridDim.x < ntiles) wait_bar(stage ^ 1, (uint32_t)((it + 1) >> 1) & 1u);
            }
            return;
        }
        const int tx = tile % tiles_x, rest = tile / tiles_x;
        const int ty = rest % tiles_y, tz = rest / tiles_y;
        const int x0 = tx * FTW, y0 = ty * kTmaTh;
        // 1. column t of the strip, through the mirror map at the plane's edges
        int sx = mirror(x0 - 4 + t, w) - (x0 - 4);
        sx = min(max(sx, 0), FNX - 1);  // columns no output depends on: any sample
        const bool inner_y = (y0 - HV >= 0) && (y0 + kTmaTh + HV <= h);
        T c[NY];
#pragma unroll
        for (int r = 0; r < NY; ++r) {
            int sy = r;
            if (!inner_y) sy = min(max(mirror(y0 - HV + r, h) - (y0 - HV), 0), NY - 1);
            c[r] = stg[stage][sy][sx];
        }
        __syncthreads();  // every column read (mirrored reads cross columns) before any write-back
        // 2. vertical lifting of column t in registers
        if (h > 1) {
#pragma unroll
            for (int k = 0; k < KT<KERN>::NSTEP; ++k) {
                const int par = 1 - (k & 1);
#pragma unroll
                for (int r = k + 1; r < NY - k - 1; ++r)
                    if ((r & 1) == par) c[r] = KT<KERN>::op(false, k, c[r], c[r - 1], c[r + 1]);
            }
        }
#pragma unroll
        for (int r = HV; r < HV + kTmaTh; ++r) {
            T v = c[r];
            if (KERN == 97 && h > 1) v = (T)__fmul_rn((float)v, (r & 1) ? KMUL : KDIV);
            stg[stage][r][t] = v;  // the lifted rows go back into the strip, in place
        }
        __syncthreads();
        // 3. horizontal lifting and the subband writes, from the strip's rows HV .. HV+15
        fwd_fast_rows<KERN, TD, QUANT, QLL, kTmaTh, 0>(stg[stage], x0, y0, w, h, ll_dst + tz * z.ll, llpitch,
                                                       dst + tz * z.dst, dpitch, st, vec_out);
        __syncthreads();  // the strip is free for the copy issued at the top of the next tile
    }
}

// ---- pipelined fast forward level ------------------------------------------------------------
// Same tile computation as dwt_fwd_fast, but each CTA walks a column strip band by band
// (bands blockIdx.y, blockIdx.y + gridDim.y, ...) with two shared strips: while band i is
// lifted, band i+1 streams into the other strip with cp.async (16-byte copies in the interior,
// 4-byte mirrored copies at the image border), so loads are always in flight.
template <int KERN, typename TD, bool QUANT, bool QLL, int FTH>
__global__ void __launch_bounds__(256)
dwt_fwd_pipe(const typename KT<KERN>::T* __restrict__ src, size_t spitch, int w, int h,
             typename KT<KERN>::T* __restrict__ ll_dst, size_t llpitch, TD* __restrict__ dst, size_t dpitch,
             Steps4 st, int vec_out, int nbands) {
    using T = typename KT<KERN>::T;
    constexpr int HV = KT<KERN>::H, NY = FTH + 2 * HV;
    __shared__ __align__(16) T sb[2][NY][FNX];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, t = threadIdx.x;
    const int x0 = blockIdx.x * FTW;
    const bool inner_x = (x0 - 4 >= 0) && (x0 + 252 <= w);
    const int wl = (w + 1) >> 1, hl = (h + 1) >> 1;
    auto issue = [&](int band, int buf) {
        const int y0 = band * FTH;
        for (int e = t; e < NY * 64; e += 256) {
            const int r = e >> 6, q = e & 63;
            const T* row = src + (size_t)mirror(y0 - HV + r, h) * spitch;
            const int gx = x0 - 4 + 4 * q;
            T* d = &sb[buf][r][4 * q];
            if (inner_x) {
                cp_async16(d, row + gx);
            } else {
#pragma unroll
                for (int k = 0; k < 4; ++k) cp_async4(d + k, row + mirror(gx + k, w));
            }
        }
    };
    int band = blockIdx.y;
    if (band < nbands) issue(band, 0);
    cp_async_commit();
    for (int it = 0; band < nbands; ++it, band += gridDim.y) {
        const int buf = it & 1;
        const int next = band + gridDim.y;
        if (next < nbands) issue(next, buf ^ 1);
        cp_async_commit();
        cp_async_wait1();
        __syncthreads();
        auto& s = sb[buf];
        const int y0 = band * FTH;
        if (h > 1) {
            T c[NY];
#pragma unroll
            for (int r = 0; r < NY; ++r) c[r] = s[r][t];
#pragma unroll
            for (int k = 0; k < KT<KERN>::NSTEP; ++k) {
                const int par = 1 - (k & 1);
#pragma unroll
                for (int r = k + 1; r < NY - k - 1; ++r)
                    if ((r & 1) == par) c[r] = KT<KERN>::op(false, k, c[r], c[r - 1], c[r + 1]);
            }
#pragma unroll
            for (int r = HV; r < HV + FTH; ++r) {
                T v = c[r];
                if (KERN == 97) v = (T)__fmul_rn((float)v, (r & 1) ? KMUL : KDIV);
                s[r][t] = v;
            }
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < FTH / 8; ++i) {
            const int r = HV + warp + 8 * i;
            const int y = y0 + r - HV;
            if (y >= h) break;
            T v[8];
            *reinterpret_cast<uint4*>(&v[0]) = *reinterpret_cast<const uint4*>(&s[r][8 * lane]);
            *reinterpret_cast<uint4*>(&v[4]) = *reinterpret_cast<const uint4*>(&s[r][8 * lane + 4]);
            if (w > 1) {
#pragma unroll
                for (int k = 0; k < KT<KERN>::NSTEP; ++k) {
                    if ((k & 1) == 0) {
                        const T nx = __shfl_down_sync(0xffffffffu, v[0], 1);
                        v[1] = KT<KERN>::op(false, k, v[1], v[0], v[2]);
                        v[3] = KT<KERN>::op(false, k, v[3], v[2], v[4]);
                        v[5] = KT<KERN>::op(false, k, v[5], v[4], v[6]);
                        v[7] = KT<KERN>::op(false, k, v[7], v[6], nx);
                    } else {
                        const T pv = __shfl_up_sync(0xffffffffu, v[7], 1);
                        v[0] = KT<KERN>::op(false, k, v[0], pv, v[1]);
                        v[2] = KT<KERN>::op(false, k, v[2], v[1], v[3]);
                        v[4] = KT<KERN>::op(false, k, v[4], v[3], v[5]);
                        v[6] = KT<KERN>::op(false, k, v[6], v[5], v[7]);
                    }
                }
                if (KERN == 97) {
#pragma unroll
                    for (int j = 0; j < 8; ++j) v[j] = (T)__fmul_rn((float)v[j], (j & 1) ? KMUL : KDIV);
                }
            }
            const int qy = y & 1;
            const int sy = (y >> 1) + (qy ? hl : 0);
            const int xs = x0 - 4 + 8 * lane;
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                const int e0 = 8 * lane + 4 * half;
                const int xa = xs + 4 * half;
                if (e0 + 4 <= 4 || e0 >= 252) continue;
#pragma unroll
                for (int qx = 0; qx < 2; ++qx) {
                    const bool isll = (qx == 0 && qy == 0);
                    T a = v[4 * half + qx], b = v[4 * half + 2 + qx];
                    const int sx = (xa >> 1) + (qx ? wl : 0);
                    const bool va = xa + qx < w, vb = xa + 2 + qx < w;
                    if (isll && !QLL) {
                        T* p = ll_dst + (size_t)sy * llpitch + sx;
                        if (vec_out && va && vb) {
                            T pr[2] = {a, b};
                            *reinterpret_cast<uint2*>(p) = *reinterpret_cast<uint2*>(pr);
                        } else {
                            if (va) p[0] = a;
                            if (vb) p[1] = b;
                        }
                    } else {
                        const float stp = isll ? st.ll : (qx && qy ? st.hh : (qx ? st.hl : st.lh));
                        TD oa, ob;
                        if (QUANT) {
                            oa = (TD)quantize((float)a, stp);
                            ob = (TD)quantize((float)b, stp);
                        } else {
                            oa = (TD)a;
                            ob = (TD)b;
                        }
                        TD* p = dst + (size_t)sy * dpitch + sx;
                        if (vec_out && va && vb && ((sx & 1) == 0)) {
                            TD pr[2] = {oa, ob};
                            *reinterpret_cast<uint2*>(p) = *reinterpret_cast<uint2*>(pr);
                        } else {
                            if (va) p[0] = oa;
                            if (vb) p[1] = ob;
                        }
                    }
                }
            }
        }
        __syncthreads();  // strip `buf` is refilled two bands later
    }
    cp_async_wait1();
}

// ---- inverse level ----------------------------------------------------------------------------
// Reconstructs the w x h region of level k-1 from the detail subbands of `src` (Mallat plane,
// optionally int32 indices when DEQ) and the LL band (ll_src, or src itself when DEQLL).
template <int KERN, int ORDER, int TW, int TH, typename TS, bool DEQ, bool DEQLL>
__global__ void __launch_bounds__(256)
dwt_inv_level(const TS* __restrict__ src, size_t spitch,
              const typename KT<KERN>::T* __restrict__ ll_src, size_t llpitch, int w, int h,
              typename KT<KERN>::T* __restrict__ out, size_t opitch, Steps4 st, ZStride z) {
    src += blockIdx.z * z.src;
    ll_src += blockIdx.z * z.ll;
    out += blockIdx.z * z.dst;
    using T = typename KT<KERN>::T;
    using G = Tile<KERN, TW, TH>;
    constexpr int H = G::H;
    __shared__ T s[G::NY * G::S];
    const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
    const int wl = (w + 1) >> 1, hl = (h + 1) >> 1;
    for (int e = threadIdx.x; e < G::NX * G::NY; e += blockDim.x) {
        int r = e / G::NX, c = e % G::NX;
        int gy = mirror(y0 - H + r, h), gx = mirror(x0 - H + c, w);
        int qx = gx & 1, qy = gy & 1;
        int sx = (gx >> 1) + (qx ? wl : 0), sy = (gy >> 1) + (qy ? hl : 0);
        T v;
        if (!qx && !qy) {
            if (DEQLL) v = (T)dequantize((int32_t)src[(size_t)sy * spitch + sx], st.ll);
            else v = ll_src[(size_t)sy * llpitch + sx];
        } else {
            TS raw = src[(size_t)sy * spitch + sx];
            if (DEQ) v = (T)dequantize((int32_t)raw, qx && qy ? st.hh : (qx ? st.hl : st.lh));
            else v = (T)raw;
        }
        s[r * G::S + c] = v;
    }
    __syncthreads();
    const bool dov = h > 1, doh = w > 1;
    if (ORDER == J2K_ORDER_T800) {
        // undo rows first (all rows of the tile are needed by the column pass)
        if (doh) {
            scale97<KERN, TW, TH, true, false, 0, G::NX, 0, G::NY>(s);
            hsteps<KERN, TW, TH, true, 0, G::NY>(s);
        }
        if (dov) {
            scale97<KERN, TW, TH, true, true, H, H + TW, 0, G::NY>(s);
            vsteps<KERN, TW, TH, true, H, H + TW>(s);
        }
    } else {
        if (dov) {
            scale97<KERN, TW, TH, true, true, 0, G::NX, 0, G::NY>(s);
            vsteps<KERN, TW, TH, true, 0, G::NX>(s);
        }
        if (doh) {
            scale97<KERN, TW, TH, true, false, 0, G::NX, H, H + TH>(s);
            hsteps<KERN, TW, TH, true, H, H + TH>(s);
        }
    }
    for (int e = threadIdx.x; e < TW * TH; e += blockDim.x) {
        int i = e % TW, j = e / TW;
        int x = x0 + i, y = y0 + j;
        if (x < w && y < h) out[(size_t)y * opitch + x] = s[(H + j) * G::S + H + i];
    }
}

// levels == 0: plain copy, or quantisation of the single LL band
template <typename TI, typename TO, bool Q>
__global__ void copy_plane(const TI* __restrict__ in, size_t ip, TO* __restrict__ out, size_t op,
                           int w, int h, float step, ZStride z) {
    in += blockIdx.z * z.src;
    out += blockIdx.z * z.dst;
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= w || y >= h) return;
    TI v = in[(size_t)y * ip + x];
    if (Q) out[(size_t)y * op + x] = (TO)quantize((float)v, step);
    else out[(size_t)y * op + x] = (TO)v;
}
template <typename TI, typename TO, bool DQ>
__global__ void copy_plane_deq(const TI* __restrict__ in, size_t ip, TO* __restrict__ out,
                               size_t op, int w, int h, float step, ZStride z) {
    in += blockIdx.z * z.src;
    out += blockIdx.z * z.dst;
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= w || y >= h) return;
    TI v = in[(size_t)y * ip + x];
    if (DQ) out[(size_t)y * op + x] = (TO)dequantize((int32_t)v, step);
    else out[(size_t)y * op + x] = (TO)v;
}

// cuTensorMapEncodeTiled through the runtime (no link dependency on the driver library)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
        return (PFN_cuTensorMapEncodeTiled_v12000)f;
    }();
    return fn;
}

// One forward level by the TMA-staged kernel: n planes of w x h at src (pitch and plane stride
// in elements, both multiples of 4 so that rows and planes start on 16-byte boundaries).
template <int KERN, typename TD, bool QUANT, bool QLL>
static j2k_status launch_fwd_tma(j2k_ctx* ctx, const void* src, size_t spitch, size_t src_z, int w, int h, int n,
                                 typename KT<KERN>::T* lld, size_t llp, TD* out, size_t out_pitch, Steps4 st, int vec,
                                 ZStride zs, cudaStream_t stream, bool pdl) {
    auto enc = tensor_map_encoder();
    if (!enc) return j2k_fail(ctx, J2K_ERR_UNSUPPORTED, "no tensor-map encoder in this driver");
    CUtensorMap tm;
    const cuuint64_t dims[3] = {(cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)n};
    const cuuint64_t strides[2] = {(cuuint64_t)spitch * 4, (cuuint64_t)(n > 1 ? src_z : spitch * h) * 4};
    const cuuint32_t box[3] = {(cuuint32_t)FNX, (cuuint32_t)TmaStrip<KERN>::NY, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = enc(&tm, KERN == 53 ? CU_TENSOR_MAP_DATA_TYPE_INT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                           const_cast<void*>(src), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return j2k_fail(ctx, J2K_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    auto kern = dwt_fwd_tma<KERN, TD, QUANT, QLL>;
    constexpr int smem = TmaStrip<KERN>::SMEM;
    static int per_sm = 0;  // resident CTAs per SM of this instantiation (set once)
    if (per_sm == 0) {
        J2K_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        int v = 0;
        J2K_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kern, 256, smem));
        per_sm = std::max(v, 1);
    }
    const int tiles_x = (w + FTW - 1) / FTW, tiles_y = (h + kTmaTh - 1) / kTmaTh;
    const long ntiles = (long)tiles_x * tiles_y * n;
    const int grid = (int)std::min<long>(ntiles, (long)per_sm * ctx->sm_count);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = pdl ? at : nullptr;
    cfg.numAttrs = pdl ? 1 : 0;
    J2K_CUDA(ctx, cudaLaunchKernelEx(&cfg, kern, tm, w, h, n, tiles_x, tiles_y, lld, llp, out, out_pitch, st, vec, zs,
                                     ctx->d_err));
    return J2K_OK;
}

// Levels k .. of the transform whose level-k input is cw x chh (n planes) by one cooperative
// dwt_fwd_tail launch, when they are few tiles: from the first level with at most two tiles per
// resident CTA, through the last level at least 8 x 2 samples.  *used = the levels it covered
// (0: none, the caller launches level k itself).
template <int KERN>
static j2k_status fwd_tail_launch(j2k_ctx* ctx, int k, int levels, int cw, int chh, int n,
                                  const typename KT<KERN>::T* src, size_t spitch, size_t src_z, void* out,
                                  size_t out_pitch, size_t out_z, const float* steps, void* ll0, void* ll1,
                                  size_t z0, size_t z1, cudaStream_t stream, int* used) {
    using T = typename KT<KERN>::T;
    *used = 0;
    const bool quant = (KERN == 97) && steps != nullptr;
    static int per_sm_q = 0, per_sm_f = 0;  // resident CTAs per SM of each instantiation (set once)
    int& per_sm = quant ? per_sm_q : per_sm_f;
    if (per_sm == 0) {
        int v = 0;
        J2K_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                          &v, quant ? dwt_fwd_tail<KERN, true> : dwt_fwd_tail<KERN, false>, 256, 0));
        per_sm = std::max(v, 1);
    }
    const long cap = (long)per_sm * ctx->sm_count;
    const long tiles_k = (long)((cw + FTW - 1) / FTW) * ((chh + 15) / 16) * n;
    // form 1: cooperative launch over the GPU; 2..5: one cluster per plane (size 16, 16, 8, 16)
    // from the first level with at most 96, 32, 96, 320 tiles per plane
    const int form = ctx->dwt_tail;
    static const int kCs[6] = {0, 0, 16, 16, 8, 16}, kThr[6] = {0, 0, 96, 32, 96, 320};
    if (form >= 2) {
        if (tiles_k > (long)kThr[form] * n) return J2K_OK;
    } else if (tiles_k > 2 * cap) {
        return J2K_OK;  // a full-size level: its own launch
    }
    TailPlan plan{};
    plan.nz = n;
    int w = cw, h = chh;
    const T* s = src;
    size_t sp = spitch, sz = src_z;
    long maxt = 0;
    for (int q = k; q < levels && plan.nlev < kTailLevels; ++q) {
        if (w < 8 || h < 2) break;
        const bool last = q == levels - 1;
        TailLevel& L = plan.lv[plan.nlev];
        L.src = s;
        L.spitch = sp;
        L.src_z = sz;
        L.w = w;
        L.h = h;
        if (last) {
            L.lld = out;
            L.llp = out_pitch;
            L.ll_z = out_z;
        } else {
            L.lld = q % 2 == 0 ? ll0 : ll1;
            L.llp = (size_t)((w + 1) / 2);
            L.ll_z = q % 2 == 0 ? z0 : z1;
        }
        L.last = last;
        L.tiles_x = (w + FTW - 1) / FTW;
        L.tiles_y = (h + 15) / 16;
        L.vec = (((uintptr_t)out & 7) == 0) && ((out_pitch & 1) == 0) && (((uintptr_t)L.lld & 7) == 0) &&
                ((L.llp & 1) == 0);
        const int bt = 1 + 3 * (levels - (q + 1));
        L.st = quant ? Steps4{steps[0], steps[bt], steps[bt + 1], steps[bt + 2]} : Steps4{1.f, 1.f, 1.f, 1.f};
        maxt = std::max(maxt, (long)L.tiles_x * L.tiles_y * n);
        ++plan.nlev;
        s = (const T*)L.lld;
        sp = L.llp;
        sz = L.ll_z;
        w = (w + 1) / 2;
        h = (h + 1) / 2;
        if (last) break;
    }
    if (plan.nlev < 2) return J2K_OK;  // one level gains nothing
    if (form >= 2) {
        const int cs = kCs[form];
        auto kern = quant ? dwt_fwd_ctail<KERN, true> : dwt_fwd_ctail<KERN, false>;
        if (cs > 8) J2K_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(cs, 1, n);
        cfg.blockDim = dim3(256);
        cfg.stream = stream;
        cudaLaunchAttribute at[2];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = cs;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[1].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = 2;
        int clusters = 0;
        J2K_CUDA(ctx, cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg));
        if (clusters < 1) return J2K_OK;  // no room for a cluster of this size: level by level
        J2K_CUDA(ctx, cudaLaunchKernelEx(&cfg, kern, plan, out, out_pitch, out_z));
        *used = plan.nlev;
        return J2K_OK;
    }
    uint32_t* bar = (uint32_t*)j2k_scratch(ctx, SCR_BARRIER, 64);
    if (!bar) return J2K_ERR_OUT_OF_MEMORY;
    J2K_CUDA(ctx, cudaMemsetAsync(bar, 0, 8, stream));
    const int grid = (int)std::min<long>(maxt, cap);
    void* args[] = {(void*)&plan, (void*)&out, (void*)&out_pitch, (void*)&out_z, (void*)&bar, (void*)&ctx->d_err};
    if (quant)
        J2K_CUDA(ctx, cudaLaunchCooperativeKernel((const void*)dwt_fwd_tail<KERN, true>, dim3(grid), dim3(256), args, 0,
                                                  stream));
    else
        J2K_CUDA(ctx, cudaLaunchCooperativeKernel((const void*)dwt_fwd_tail<KERN, false>, dim3(grid), dim3(256), args,
                                                  0, stream));
    *used = plan.nlev;
    return J2K_OK;
}

template <int KERN, int ORDER, int TW, int TH>
j2k_status fwd_levels(j2k_ctx* ctx, const void* in, size_t in_pitch, void* out, size_t out_pitch,
                      int w, int h, int levels, const float* steps, void* ll0, void* ll1,
                      cudaStream_t stream, int n, size_t in_z, size_t out_z) {
    using T = typename KT<KERN>::T;
    const bool quant = (KERN == 97) && steps != nullptr;
    if (levels == 0) {
        dim3 g((w + 255) / 256, h, n);
        const ZStride zc{in_z, out_z, 0};
        if (quant)
            copy_plane<float, int32_t, true><<<g, 256, 0, stream>>>((const float*)in, in_pitch, (int32_t*)out, out_pitch, w, h, steps[0], zc);
        else
            copy_plane<T, T, false><<<g, 256, 0, stream>>>((const T*)in, in_pitch, (T*)out, out_pitch, w, h, 1.0f, zc);
        J2K_CUDA(ctx, cudaGetLastError());
        return J2K_OK;
    }
    int cw = w, chh = h;
    const T* src = (const T*)in;
    size_t spitch = in_pitch;
    // per-image strides of the two LL scratch buffers (sized for level 0 / level 1 outputs)
    const size_t z0 = (size_t)((w + 1) / 2) * ((h + 1) / 2);
    const size_t z1 = (size_t)(((w + 1) / 2 + 1) / 2) * (((h + 1) / 2 + 1) / 2);
    size_t src_z = in_z;
    for (int k = 0; k < levels; ++k) {
        bool last = (k == levels - 1);
        if (ctx && ctx->dwt_tail && ORDER == J2K_ORDER_T800 && ctx->dwt_fast_th == 16 && k >= 1 && !ctx->dwt_tma) {
            int used = 0;
            J2K_TRY((fwd_tail_launch<KERN>(ctx, k, levels, cw, chh, n, src, spitch, src_z, out, out_pitch, out_z,
                                           steps, ll0, ll1, z0, z1, stream, &used)));
            if (used > 0) {
                for (int q = 0; q < used; ++q) {
                    src = (const T*)((k + q) % 2 == 0 ? ll0 : ll1);
                    spitch = (size_t)((cw + 1) / 2);
                    src_z = (k + q) % 2 == 0 ? z0 : z1;
                    cw = (cw + 1) / 2;
                    chh = (chh + 1) / 2;
                }
                k += used - 1;
                continue;
            }
        }
        dim3 grid((cw + TW - 1) / TW, (chh + TH - 1) / TH, n);
        T* lld;
        size_t llp, ll_z;
        if (last) {
            lld = (T*)out;
            llp = out_pitch;
            ll_z = out_z;
        } else {
            int nw = (cw + 1) / 2;
            lld = (T*)((k % 2 == 0) ? ll0 : ll1);
            llp = (size_t)nw;  // the next level's input pitch
            ll_z = (k % 2 == 0) ? z0 : z1;
        }
        const ZStride zs{src_z, out_z, ll_z};
        // subband indices of this level in QCD order: level L-k's triple
        int dl = k + 1;  // decomposition level produced
        int bt = 1 + 3 * (levels - dl);
        Steps4 st{1.f, 1.f, 1.f, 1.f};
        if (quant) st = Steps4{steps[0], steps[bt], steps[bt + 1], steps[bt + 2]};
        // every image of the batch starts 16-byte aligned (the cp.async form copies 16-byte chunks)
        const bool fast_ok = ORDER == J2K_ORDER_T800 && ((uintptr_t)src & 15) == 0 && (spitch & 3) == 0 &&
                             (n == 1 || (src_z & 3) == 0) && cw >= 8 && chh >= 2 &&
                             (!ctx || ctx->dwt_fast_th != 0);
        if (fast_ok) {
            const int fth = ctx ? ctx->dwt_fast_th : 32;
            dim3 fg((cw + FTW - 1) / FTW, (chh + fth - 1) / fth, n);
            const int vec = (((uintptr_t)out & 7) == 0) && ((out_pitch & 1) == 0) &&
                            (((uintptr_t)lld & 7) == 0) && ((llp & 1) == 0) &&
                            (n == 1 || ((out_z & 1) == 0 && (ll_z & 1) == 0));
#define FAST(TH_, REG_)                                                                                  \
    do {                                                                                                 \
        if (quant) {                                                                                     \
            if (last)                                                                                    \
                dwt_fwd_fast<KERN, int32_t, true, true, TH_, REG_><<<fg, 256, 0, stream>>>(              \
                    src, spitch, cw, chh, lld, llp, (int32_t*)out, out_pitch, st, vec, zs);             \
            else                                                                                         \
                dwt_fwd_fast<KERN, int32_t, true, false, TH_, REG_><<<fg, 256, 0, stream>>>(             \
                    src, spitch, cw, chh, lld, llp, (int32_t*)out, out_pitch, st, vec, zs);             \
        } else {                                                                                         \
            dwt_fwd_fast<KERN, T, false, false, TH_, REG_><<<fg, 256, 0, stream>>>(                      \
                src, spitch, cw, chh, lld, llp, (T*)out, out_pitch, st, vec, zs);                        \
        }                                                                                                \
    } while (0)
            const bool tma_ok = ctx && ctx->dwt_tma && (n == 1 || (src_z & 3) == 0) && cw >= 16;
            if (tma_ok) {
                const bool pdl = k > 0;
                if (quant && last)
                    J2K_TRY((launch_fwd_tma<KERN, int32_t, true, true>(ctx, src, spitch, src_z, cw, chh, n, lld, llp,
                                                                      (int32_t*)out, out_pitch, st, vec, zs, stream,
                                                                      pdl)));
                else if (quant)
                    J2K_TRY((launch_fwd_tma<KERN, int32_t, true, false>(ctx, src, spitch, src_z, cw, chh, n, lld, llp,
                                                                       (int32_t*)out, out_pitch, st, vec, zs, stream,
                                                                       pdl)));
                else
                    J2K_TRY((launch_fwd_tma<KERN, T, false, false>(ctx, src, spitch, src_z, cw, chh, n, lld, llp,
                                                                  (T*)out, out_pitch, st, vec, zs, stream, pdl)));
            } else if (ctx && ctx->dwt_pipe && n == 1) {
                const int bands = (chh + 16 - 1) / 16;
                const int tx = (cw + FTW - 1) / FTW;
                const int want = std::max(1, (ctx->sm_count * 4 + tx - 1) / tx);
                dim3 pg(tx, std::min(bands, want));
                if (quant) {
                    if (last)
                        dwt_fwd_pipe<KERN, int32_t, true, true, 16><<<pg, 256, 0, stream>>>(
                            src, spitch, cw, chh, lld, llp, (int32_t*)out, out_pitch, st, vec, bands);
                    else
                        dwt_fwd_pipe<KERN, int32_t, true, false, 16><<<pg, 256, 0, stream>>>(
                            src, spitch, cw, chh, lld, llp, (int32_t*)out, out_pitch, st, vec, bands);
                } else {
                    dwt_fwd_pipe<KERN, T, false, false, 16><<<pg, 256, 0, stream>>>(
                        src, spitch, cw, chh, lld, llp, (T*)out, out_pitch, st, vec, bands);
                }
            } else if (ctx && !ctx->dwt_reg) {
                if (fth == 16) FAST(16, false); else FAST(32, false);
            } else {
                // the default path: every level after the first is a programmatic dependent of
                // the one before, so its launch overlaps the previous level's last CTAs
                const bool pdl = k > 0;
                const dim3 b(256);
                cudaError_t le;
                if (quant && last)
                    le = fth == 16 ? launch_pdl(dwt_fwd_fast<KERN, int32_t, true, true, 16, true>, fg, b, stream, pdl,
                                                src, spitch, cw, chh, lld, llp, (int32_t*)out, out_pitch, st, vec, zs)
                                   : launch_pdl(dwt_fwd_fast<KERN, int32_t, true, true, 32, true>, fg, b, stream, pdl,
                                                src, spitch, cw, chh, lld, llp, (int32_t*)out, out_pitch, st, vec, zs);
                else if (quant)
                    le = fth == 16 ? launch_pdl(dwt_fwd_fast<KERN, int32_t, true, false, 16, true>, fg, b, stream, pdl,
                                                src, spitch, cw, chh, lld, llp, (int32_t*)out, out_pitch, st, vec, zs)
                                   : launch_pdl(dwt_fwd_fast<KERN, int32_t, true, false, 32, true>, fg, b, stream, pdl,
                                                src, spitch, cw, chh, lld, llp, (int32_t*)out, out_pitch, st, vec, zs);
                else
                    le = fth == 16 ? launch_pdl(dwt_fwd_fast<KERN, T, false, false, 16, true>, fg, b, stream, pdl,
                                                src, spitch, cw, chh, lld, llp, (T*)out, out_pitch, st, vec, zs)
                                   : launch_pdl(dwt_fwd_fast<KERN, T, false, false, 32, true>, fg, b, stream, pdl,
                                                src, spitch, cw, chh, lld, llp, (T*)out, out_pitch, st, vec, zs);
                J2K_CUDA(ctx, le);
            }
#undef FAST
        } else if (quant) {
            if (last)
                dwt_fwd_level<KERN, ORDER, TW, TH, int32_t, true, true><<<grid, 256, 0, stream>>>(
                    src, spitch, cw, chh, lld, llp, (int32_t*)out, out_pitch, st, zs);
            else
                dwt_fwd_level<KERN, ORDER, TW, TH, int32_t, true, false><<<grid, 256, 0, stream>>>(
                    src, spitch, cw, chh, lld, llp, (int32_t*)out, out_pitch, st, zs);
        } else {
            dwt_fwd_level<KERN, ORDER, TW, TH, T, false, false><<<grid, 256, 0, stream>>>(
                src, spitch, cw, chh, lld, llp, (T*)out, out_pitch, st, zs);
        }
        J2K_CUDA(ctx, cudaGetLastError());
        src = lld;
        spitch = llp;
        src_z = ll_z;
        cw = (cw + 1) / 2;
        chh = (chh + 1) / 2;
    }
    return J2K_OK;
}

template <int KERN, int ORDER, int TW, int TH>
j2k_status inv_levels(j2k_ctx* ctx, const void* in, size_t in_pitch, void* out, size_t out_pitch,
                      int w, int h, int levels, const float* steps, void* ll0, void* ll1,
                      cudaStream_t stream, int n, size_t in_z, size_t out_z) {
    using T = typename KT<KERN>::T;
    const bool deq = (KERN == 97) && steps != nullptr;
    if (levels == 0) {
        dim3 g((w + 255) / 256, h, n);
        const ZStride zc{in_z, out_z, 0};
        if (deq)
            copy_plane_deq<int32_t, float, true><<<g, 256, 0, stream>>>((const int32_t*)in, in_pitch, (float*)out, out_pitch, w, h, steps[0], zc);
        else
            copy_plane_deq<T, T, false><<<g, 256, 0, stream>>>((const T*)in, in_pitch, (T*)out, out_pitch, w, h, 1.0f, zc);
        J2K_CUDA(ctx, cudaGetLastError());
        return J2K_OK;
    }
    int ws[40], hs[40];
    ws[0] = w;
    hs[0] = h;
    for (int k = 1; k <= levels; ++k) { ws[k] = (ws[k - 1] + 1) / 2; hs[k] = (hs[k - 1] + 1) / 2; }
    // per-image strides of the two LL scratch buffers: odd levels use ll0 (level-1 size),
    // even levels >= 2 use ll1 (level-2 size)
    const size_t z0 = (size_t)ws[1] * hs[1];
    const size_t z1 = levels >= 2 ? (size_t)ws[2] * hs[2] : 0;
    for (int k = levels - 1; k >= 0; --k) {
        int cw = ws[k], chh = hs[k];
        dim3 grid((cw + TW - 1) / TW, (chh + TH - 1) / TH, n);
        T* o = (k == 0) ? (T*)out : (T*)((k % 2 == 1) ? ll0 : ll1);
        size_t op = (k == 0) ? out_pitch : (size_t)cw;
        const size_t o_z = (k == 0) ? out_z : ((k % 2 == 1) ? z0 : z1);
        const T* lls = (k == levels - 1) ? (const T*)in : (const T*)((k % 2 == 1) ? ll1 : ll0);
        size_t llp = (k == levels - 1) ? in_pitch : (size_t)ws[k + 1];
        const size_t l_z = (k == levels - 1) ? in_z : ((k % 2 == 1) ? z1 : z0);
        const ZStride zs{in_z, o_z, l_z};
        int bt = 1 + 3 * (levels - (k + 1));
        Steps4 st{1.f, 1.f, 1.f, 1.f};
        if (deq) st = Steps4{steps[0], steps[bt], steps[bt + 1], steps[bt + 2]};
        const bool fast_ok = ORDER == J2K_ORDER_T800 && cw >= 8 && chh >= 2 && (!ctx || ctx->dwt_fast_th != 0);
        if (fast_ok) {
            // register-lifting strip kernel; 8-byte band loads when every row start is aligned
            const int wl = (cw + 1) / 2;
            const int vec = (((uintptr_t)in & 7) == 0) && ((in_pitch & 1) == 0) && ((in_z & 1) == 0) &&
                            (((uintptr_t)lls & 7) == 0) && ((llp & 1) == 0) && ((l_z & 1) == 0) &&
                            ((wl & 1) == 0);
            const dim3 fg((cw + FTW - 1) / FTW, (chh + STH - 1) / STH, n);
            const SynExtra ex{};
            // (not programmatic dependents: these kernels read their input through the read-only
            // cache, which the previous level writes)
            const dim3 b(256);
            cudaError_t le;
            if (deq) {
                if (k == levels - 1)
                    le = launch_pdl(dwt_syn_fast<KERN, 0, int32_t, true, true, 0>, fg, b, stream, false,
                                    (const int32_t*)in, in_pitch, lls, llp, cw, chh, o, op, st, zs, vec, ex);
                else
                    le = launch_pdl(dwt_syn_fast<KERN, 0, int32_t, true, false, 0>, fg, b, stream, false,
                                    (const int32_t*)in, in_pitch, lls, llp, cw, chh, o, op, st, zs, vec, ex);
            } else {
                le = launch_pdl(dwt_syn_fast<KERN, 0, T, false, false, 0>, fg, b, stream, false, (const T*)in,
                                in_pitch, lls, llp, cw, chh, o, op, st, zs, vec, ex);
            }
            J2K_CUDA(ctx, le);
        } else if (deq) {
            if (k == levels - 1)
                dwt_inv_level<KERN, ORDER, TW, TH, int32_t, true, true><<<grid, 256, 0, stream>>>(
                    (const int32_t*)in, in_pitch, lls, llp, cw, chh, o, op, st, zs);
            else
                dwt_inv_level<KERN, ORDER, TW, TH, int32_t, true, false><<<grid, 256, 0, stream>>>(
                    (const int32_t*)in, in_pitch, lls, llp, cw, chh, o, op, st, zs);
        } else {
            dwt_inv_level<KERN, ORDER, TW, TH, T, false, false><<<grid, 256, 0, stream>>>(
                (const T*)in, in_pitch, lls, llp, cw, chh, o, op, st, zs);
        }
        J2K_CUDA(ctx, cudaGetLastError());
    }
    return J2K_OK;
}

template <int KERN, int TW, int TH>
j2k_status fwd_dispatch_order(j2k_ctx* ctx, int order, const void* in, size_t ip, void* out,
                              size_t op, int w, int h, int levels, const float* steps, void* a,
                              void* b, cudaStream_t st, int n, size_t iz, size_t oz) {
    if (order == J2K_ORDER_REF) return fwd_levels<KERN, J2K_ORDER_REF, TW, TH>(ctx, in, ip, out, op, w, h, levels, steps, a, b, st, n, iz, oz);
    return fwd_levels<KERN, J2K_ORDER_T800, TW, TH>(ctx, in, ip, out, op, w, h, levels, steps, a, b, st, n, iz, oz);
}
template <int KERN, int TW, int TH>
j2k_status inv_dispatch_order(j2k_ctx* ctx, int order, const void* in, size_t ip, void* out,
                              size_t op, int w, int h, int levels, const float* steps, void* a,
                              void* b, cudaStream_t st, int n, size_t iz, size_t oz) {
    if (order == J2K_ORDER_REF) return inv_levels<KERN, J2K_ORDER_REF, TW, TH>(ctx, in, ip, out, op, w, h, levels, steps, a, b, st, n, iz, oz);
    return inv_levels<KERN, J2K_ORDER_T800, TW, TH>(ctx, in, ip, out, op, w, h, levels, steps, a, b, st, n, iz, oz);
}

}  // namespace

// Tile shapes offered to callers (and the autotuner): 64x64, 128x32, 32x128 (input samples).
#define J2K_TILE_DISPATCH(FN, KERN, ...)                                                      \
    (tile.tw == 128 && tile.th == 32)   ? FN<KERN, 128, 32>(__VA_ARGS__)                      \
    : (tile.tw == 32 && tile.th == 128) ? FN<KERN, 32, 128>(__VA_ARGS__)                      \
                                        : FN<KERN, 64, 64>(__VA_ARGS__)

bool j2k_dwt_fwd_px_ok(int kernel, int ncomp, int mct, size_t w, size_t h) {
    const bool pair = ncomp == 1 ? mct == J2K_MCT_NONE
                                 : ncomp == 3 && mct == (kernel == J2K_W53 ? J2K_MCT_RCT : J2K_MCT_ICT);
    return pair && w >= 8 && h >= 2 && w <= 0x7FFFFFFF && h <= 0x7FFFFFFF;
}

j2k_status j2k_dwt_fwd_px_launch(j2k_ctx* ctx, int kernel, int ncomp, int mct, const uint8_t* px, size_t pitch,
                                 size_t w, size_t h, int levels, const float* steps, void* ll, size_t llpitch,
                                 size_t ll_z, void* out, size_t out_pitch, size_t out_z, cudaStream_t stream) {
    if (!j2k_dwt_fwd_px_ok(kernel, ncomp, mct, w, h) || levels < 1)
        return j2k_fail(ctx, J2K_ERR_UNSUPPORTED, "dwt from pixels: unsupported shape or colour transform");
    const bool quant = kernel == J2K_W97 && steps != nullptr;
    const bool last = levels == 1;
    if (last) {  // one level: the LL band goes to the output plane (quantised into it when quant)
        ll = out;
        llpitch = out_pitch;
        ll_z = out_z;
    }
    Steps4 st{1.f, 1.f, 1.f, 1.f};
    if (quant) {
        const int bt = 1 + 3 * (levels - 1);  // the level-1 subbands in QCD order
        st = Steps4{steps[0], steps[bt], steps[bt + 1], steps[bt + 2]};
    }
    // 8-byte stores only where every component's plane keeps them aligned
    const int vec = (((uintptr_t)out & 7) == 0) && ((out_pitch & 1) == 0) && (ncomp == 1 || (out_z & 1) == 0) &&
                    (((uintptr_t)ll & 7) == 0) && ((llpitch & 1) == 0) && (ncomp == 1 || (ll_z & 1) == 0);
    const dim3 g((unsigned)((w + FTW - 1) / FTW * ncomp), (unsigned)((h + 15) / 16), 1), b(256);
    const int iw = (int)w, ih = (int)h;
    if (kernel == J2K_W53) {
        int32_t* l = (int32_t*)ll;
        int32_t* o = (int32_t*)out;
        if (ncomp == 1)
            dwt_fwd_fast_px<53, 1, J2K_MCT_NONE, int32_t, false, false><<<g, b, 0, stream>>>(
                px, pitch, iw, ih, l, llpitch, ll_z, o, out_pitch, out_z, st, vec);
        else
            dwt_fwd_fast_px<53, 3, J2K_MCT_RCT, int32_t, false, false><<<g, b, 0, stream>>>(
                px, pitch, iw, ih, l, llpitch, ll_z, o, out_pitch, out_z, st, vec);
    } else {
        float* l = (float*)ll;
#define PX97(NC_, MCT_)                                                                                              \
    do {                                                                                                             \
        if (!quant)                                                                                                  \
            dwt_fwd_fast_px<97, NC_, MCT_, float, false, false><<<g, b, 0, stream>>>(                                \
                px, pitch, iw, ih, l, llpitch, ll_z, (float*)out, out_pitch, out_z, st, vec);                        \
        else if (last)                                                                                               \
            dwt_fwd_fast_px<97, NC_, MCT_, int32_t, true, true><<<g, b, 0, stream>>>(                                \
                px, pitch, iw, ih, l, llpitch, ll_z, (int32_t*)out, out_pitch, out_z, st, vec);                      \
        else                                                                                                         \
            dwt_fwd_fast_px<97, NC_, MCT_, int32_t, true, false><<<g, b, 0, stream>>>(                               \
                px, pitch, iw, ih, l, llpitch, ll_z, (int32_t*)out, out_pitch, out_z, st, vec);                      \
    } while (0)
        if (ncomp == 1) PX97(1, J2K_MCT_NONE);
        else PX97(3, J2K_MCT_ICT);
#undef PX97
    }
    J2K_CUDA(ctx, cudaGetLastError());
    return J2K_OK;
}

j2k_status j2k_dwt_fwd_impl(j2k_ctx* ctx, int kernel, int order, const void* in, size_t in_pitch,
                            void* out, size_t out_pitch, size_t w, size_t h, int levels,
                            const float* steps, void* ll0, void* ll1, j2k_dwt_tile tile,
                            cudaStream_t st, int n, size_t in_z, size_t out_z) {
    if (kernel == J2K_W53)
        return J2K_TILE_DISPATCH(fwd_dispatch_order, 53, ctx, order, in, in_pitch, out, out_pitch,
                                 (int)w, (int)h, levels, steps, ll0, ll1, st, n, in_z, out_z);
    return J2K_TILE_DISPATCH(fwd_dispatch_order, 97, ctx, order, in, in_pitch, out, out_pitch,
                             (int)w, (int)h, levels, steps, ll0, ll1, st, n, in_z, out_z);
}

j2k_status j2k_dwt_inv_impl(j2k_ctx* ctx, int kernel, int order, const void* in, size_t in_pitch,
                            void* out, size_t out_pitch, size_t w, size_t h, int levels,
                            const float* steps, void* ll0, void* ll1, j2k_dwt_tile tile,
                            cudaStream_t st, int n, size_t in_z, size_t out_z) {
    if (kernel == J2K_W53)
        return J2K_TILE_DISPATCH(inv_dispatch_order, 53, ctx, order, in, in_pitch, out, out_pitch,
                                 (int)w, (int)h, levels, steps, ll0, ll1, st, n, in_z, out_z);
    return J2K_TILE_DISPATCH(inv_dispatch_order, 97, ctx, order, in, in_pitch, out, out_pitch,
                             (int)w, (int)h, levels, steps, ll0, ll1, st, n, in_z, out_z);
}

j2k_status j2k_dwt_fwd_batched_launch(j2k_ctx* ctx, int kernel, int order, j2k_dwt_tile tile,
                                      const j2k_dwt_level_desc* d_descs, const uint32_t* d_owner,
                                      unsigned ntiles, cudaStream_t st) {
    if (ntiles == 0) return J2K_OK;
    if (tile.tw == FTW && tile.th == kBatchFastTh && order == J2K_ORDER_T800) {
        // the register-lifting form, launched as a programmatic dependent of the previous level
        if (kernel == J2K_W53)
            J2K_CUDA(ctx, launch_pdl(dwt_fwd_batched_fast<53>, dim3(ntiles), dim3(256), st, true, d_descs, d_owner));
        else
            J2K_CUDA(ctx, launch_pdl(dwt_fwd_batched_fast<97>, dim3(ntiles), dim3(256), st, true, d_descs, d_owner));
        return J2K_OK;
    }
#define BL(K, O, TW_, TH_) dwt_fwd_batched<K, O, TW_, TH_><<<ntiles, 256, 0, st>>>(d_descs, d_owner)
#define BL_ORDER(K, TW_, TH_)                          \
    do {                                               \
        if (order == J2K_ORDER_REF) BL(K, J2K_ORDER_REF, TW_, TH_); \
        else BL(K, J2K_ORDER_T800, TW_, TH_);          \
    } while (0)
#define BL_TILE(K)                                                          \
    do {                                                                    \
        if (tile.tw == 128 && tile.th == 32) BL_ORDER(K, 128, 32);          \
        else if (tile.tw == 32 && tile.th == 128) BL_ORDER(K, 32, 128);     \
        else BL_ORDER(K, 64, 64);                                           \
    } while (0)
    if (kernel == J2K_W53) BL_TILE(53);
    else BL_TILE(97);
#undef BL_TILE
#undef BL_ORDER
#undef BL
    J2K_CUDA(ctx, cudaGetLastError());
    return J2K_OK;
}
