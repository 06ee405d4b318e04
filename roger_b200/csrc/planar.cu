// RGB -> planar split fused with the level shift and the RCT/ICT colour transforms, and its
// inverse.  Reference: src/CL/oclplanar.cl:23-40 (one read, one write per channel, no colour
// transform) driven by src/OCLRGBtoPlanar.cpp:36-44.  The colour transforms follow
// ITU-T T.800 Annex G (G.2 RCT, G.3 ICT), with every float operation rounded separately
// (__fmul_rn/__fadd_rn) in the order the CPU oracle uses.
//
// HBM-bound: algorithmic bytes per pixel = ncomp (uint8 in) + 4*ncomp (planes out).  The fast
// kernel moves 16 pixels per thread with 16-byte loads and stores.
#include "j2k_internal.cuh"
#include "mct.cuh"

namespace {

// one pixel, generic path
template <typename TO>
__device__ __forceinline__ void fwd_pixel(const uint8_t* px, int ncomp, int mct, TO* dst,
                                          size_t idx, size_t stride) {
    if (mct != J2K_MCT_NONE) {
        int r = (int)px[0] - 128, g = (int)px[1] - 128, b = (int)px[2] - 128;
        if (mct == J2K_MCT_RCT) {
            dst[idx] = (TO)((r + 2 * g + b) >> 2);
            dst[idx + stride] = (TO)(b - g);
            dst[idx + 2 * stride] = (TO)(r - g);
        } else {
            float fr = (float)r, fg = (float)g, fb = (float)b;
            dst[idx] = (TO)dot3(YR, fr, YG, fg, YB, fb);
            dst[idx + stride] = (TO)dot3(BR, fr, BG, fg, BB, fb);
            dst[idx + 2 * stride] = (TO)dot3(RR, fr, RG, fg, RB, fb);
        }
        for (int c = 3; c < ncomp; ++c) dst[idx + c * stride] = (TO)((int)px[c] - 128);
    } else {
        for (int c = 0; c < ncomp; ++c) dst[idx + c * stride] = (TO)((int)px[c] - 128);
    }
}

template <typename TO>
__global__ void planar_fwd_generic(const uint8_t* __restrict__ in, size_t in_pitch, int ncomp,
                                   int mct, TO* __restrict__ planes, size_t pitch, size_t stride,
                                   int w, int h) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    if (x >= w || y >= h) return;
    fwd_pixel<TO>(in + (size_t)y * in_pitch + (size_t)x * ncomp, ncomp, mct, planes,
                  (size_t)y * pitch + x, stride);
}

// Fast path: contiguous rows and planes, 16 pixels per thread.
template <int NC, typename TO>
__global__ void __launch_bounds__(256) planar_fwd_vec16(const uint8_t* __restrict__ in, int mct,
                                                        TO* __restrict__ planes, size_t stride,
                                                        size_t ngroups) {
    size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ngroups) return;
    uint8_t px[16 * NC];
    const uint4* src = reinterpret_cast<const uint4*>(in + g * 16 * NC);
#pragma unroll
    for (int i = 0; i < NC; ++i) *reinterpret_cast<uint4*>(px + 16 * i) = __ldcs(src + i);
    TO o[NC][16];
#pragma unroll
    for (int p = 0; p < 16; ++p) {
        const uint8_t* q = px + p * NC;
        bool done = false;
        if constexpr (NC >= 3) {
            if (mct == J2K_MCT_RCT) {
                int r = (int)q[0] - 128, gg = (int)q[1] - 128, b = (int)q[2] - 128;
                o[0][p] = (TO)((r + 2 * gg + b) >> 2);
                o[1][p] = (TO)(b - gg);
                o[2][p] = (TO)(r - gg);
#pragma unroll
                for (int c = 3; c < NC; ++c) o[c][p] = (TO)((int)q[c] - 128);
                done = true;
            } else if (mct == J2K_MCT_ICT) {
                float r = (float)((int)q[0] - 128), gg = (float)((int)q[1] - 128),
                      b = (float)((int)q[2] - 128);
                o[0][p] = (TO)dot3(YR, r, YG, gg, YB, b);
                o[1][p] = (TO)dot3(BR, r, BG, gg, BB, b);
                o[2][p] = (TO)dot3(RR, r, RG, gg, RB, b);
#pragma unroll
                for (int c = 3; c < NC; ++c) o[c][p] = (TO)((int)q[c] - 128);
                done = true;
            }
        }
        if (!done) {
#pragma unroll
            for (int c = 0; c < NC; ++c) o[c][p] = (TO)((int)q[c] - 128);
        }
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        uint4* dst = reinterpret_cast<uint4*>(planes + c * stride + g * 16);
#pragma unroll
        for (int k = 0; k < 4; ++k) __stcs(dst + k, *reinterpret_cast<const uint4*>(&o[c][4 * k]));
    }
}

// The same flat path, 4 pixels per thread and step (their 4 NC bytes are NC aligned 32-bit
// words): consecutive threads take consecutive 4-pixel groups, so each plane's store of a warp
// is one contiguous 512-byte run of 16-byte streaming stores, and the loads of a warp cover
// 128 NC contiguous bytes.  Each thread takes U groups (groups g0 + 256 j of the CTA's 256 U),
// all of whose words are requested before any is used.
template <int NC, typename TO, int U>
__global__ void __launch_bounds__(256) planar_fwd_c4(const uint8_t* __restrict__ in, int mct,
                                                     TO* __restrict__ planes, size_t stride, size_t ngroups) {
    const size_t g0 = (size_t)blockIdx.x * (256 * U) + threadIdx.x;
    const uint32_t* in32 = reinterpret_cast<const uint32_t*>(in);
    uint32_t raw[U][NC];
#pragma unroll
    for (int j = 0; j < U; ++j) {
        const size_t g = g0 + (size_t)j * 256;
        if (g < ngroups) {
#pragma unroll
            for (int i = 0; i < NC; ++i) raw[j][i] = __ldcs(in32 + g * NC + i);
        }
    }
#pragma unroll
    for (int j = 0; j < U; ++j) {
        const size_t g = g0 + (size_t)j * 256;
        if (g >= ngroups) break;
        const uint8_t* px = reinterpret_cast<const uint8_t*>(raw[j]);
        TO o[NC][4];
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const uint8_t* q = px + p * NC;
            bool done = false;
            if constexpr (NC >= 3) {
                if (mct == J2K_MCT_RCT) {
                    const int r = (int)q[0] - 128, gg = (int)q[1] - 128, b = (int)q[2] - 128;
                    o[0][p] = (TO)((r + 2 * gg + b) >> 2);
                    o[1][p] = (TO)(b - gg);
                    o[2][p] = (TO)(r - gg);
#pragma unroll
                    for (int c = 3; c < NC; ++c) o[c][p] = (TO)((int)q[c] - 128);
                    done = true;
                } else if (mct == J2K_MCT_ICT) {
                    const float r = (float)((int)q[0] - 128), gg = (float)((int)q[1] - 128),
                                b = (float)((int)q[2] - 128);
                    o[0][p] = (TO)dot3(YR, r, YG, gg, YB, b);
                    o[1][p] = (TO)dot3(BR, r, BG, gg, BB, b);
                    o[2][p] = (TO)dot3(RR, r, RG, gg, RB, b);
#pragma unroll
                    for (int c = 3; c < NC; ++c) o[c][p] = (TO)((int)q[c] - 128);
                    done = true;
                }
            }
            if (!done) {
#pragma unroll
                for (int c = 0; c < NC; ++c) o[c][p] = (TO)((int)q[c] - 128);
            }
        }
#pragma unroll
        for (int c = 0; c < NC; ++c)
            __stcs(reinterpret_cast<uint4*>(planes + c * stride + g * 4), *reinterpret_cast<const uint4*>(o[c]));
    }
}

__device__ __forceinline__ uint8_t clamp_u8i(int v) { return (uint8_t)min(max(v, 0), 255); }
__device__ __forceinline__ uint8_t round_u8f(float v) {
    float r = rintf(__fadd_rn(v, 128.0f));
    r = fminf(fmaxf(r, 0.0f), 255.0f);
    return (uint8_t)(int)r;
}

template <typename T> struct is_int_t { static constexpr bool v = false; };
template <> struct is_int_t<int32_t> { static constexpr bool v = true; };

template <typename TI>
__device__ __forceinline__ void inv_pixel(const TI* src, size_t idx, size_t stride, int ncomp,
                                          int mct, uint8_t* px) {
    if (mct == J2K_MCT_RCT) {
        int Y = (int)src[idx], U = (int)src[idx + stride], V = (int)src[idx + 2 * stride];
        int g = Y - ((U + V) >> 2);
        px[0] = clamp_u8i(V + g + 128);
        px[1] = clamp_u8i(g + 128);
        px[2] = clamp_u8i(U + g + 128);
        for (int c = 3; c < ncomp; ++c) px[c] = clamp_u8i((int)src[idx + c * stride] + 128);
    } else if (mct == J2K_MCT_ICT) {
        float Y = (float)src[idx], U = (float)src[idx + stride], V = (float)src[idx + 2 * stride];
        px[0] = round_u8f(__fadd_rn(Y, __fmul_rn(IRV, V)));
        px[1] = round_u8f(__fadd_rn(__fadd_rn(Y, __fmul_rn(IGU, U)), __fmul_rn(IGV, V)));
        px[2] = round_u8f(__fadd_rn(Y, __fmul_rn(IBU, U)));
        for (int c = 3; c < ncomp; ++c) px[c] = round_u8f((float)src[idx + c * stride]);
    } else {
        for (int c = 0; c < ncomp; ++c) {
            if constexpr (is_int_t<TI>::v) px[c] = clamp_u8i((int)src[idx + c * stride] + 128);
            else px[c] = round_u8f((float)src[idx + c * stride]);
        }
    }
}

template <typename TI>
__global__ void planar_inv_generic(const TI* __restrict__ planes, size_t pitch, size_t stride,
                                   int ncomp, int mct, uint8_t* __restrict__ out, size_t out_pitch,
                                   int w, int h) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y;
    if (x >= w || y >= h) return;
    inv_pixel<TI>(planes, (size_t)y * pitch + x, stride, ncomp, mct,
                  out + (size_t)y * out_pitch + (size_t)x * ncomp);
}

template <int NC, typename TI>
__global__ void __launch_bounds__(256) planar_inv_vec16(const TI* __restrict__ planes,
                                                        size_t stride, int mct,
                                                        uint8_t* __restrict__ out,
                                                        size_t ngroups) {
    size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ngroups) return;
    TI v[NC][16];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const uint4* s = reinterpret_cast<const uint4*>(planes + c * stride + g * 16);
#pragma unroll
        for (int k = 0; k < 4; ++k) *reinterpret_cast<uint4*>(&v[c][4 * k]) = __ldcs(s + k);
    }
    uint8_t px[16 * NC];
#pragma unroll
    for (int p = 0; p < 16; ++p) {
        TI tmp[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) tmp[c] = v[c][p];
        inv_pixel<TI>(tmp, 0, 1, NC, mct, px + p * NC);
    }
    uint4* dst = reinterpret_cast<uint4*>(out + g * 16 * NC);
#pragma unroll
    for (int i = 0; i < NC; ++i) __stcs(dst + i, *reinterpret_cast<const uint4*>(px + 16 * i));
}

template <typename TS, typename TD>
__global__ void cast_kernel(const TS* __restrict__ s, TD* __restrict__ d, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) d[i] = (TD)s[i];
}

template <typename T>
__global__ void mct_planes_kernel(T* p, size_t stride, size_t n, int mct) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (mct == J2K_MCT_RCT) {
        int r = (int)p[i], g = (int)p[i + stride], b = (int)p[i + 2 * stride];
        p[i] = (T)((r + 2 * g + b) >> 2);
        p[i + stride] = (T)(b - g);
        p[i + 2 * stride] = (T)(r - g);
    } else {
        float r = (float)p[i], g = (float)p[i + stride], b = (float)p[i + 2 * stride];
        p[i] = (T)dot3(YR, r, YG, g, YB, b);
        p[i + stride] = (T)dot3(BR, r, BG, g, BB, b);
        p[i + 2 * stride] = (T)dot3(RR, r, RG, g, RB, b);
    }
}

inline bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

}  // namespace

j2k_status j2k_launch_planar_fwd(j2k_ctx* ctx, const uint8_t* in, size_t in_pitch, int ncomp,
                                 int mct, int out_dtype, void* planes, size_t plane_pitch,
                                 size_t plane_stride, size_t w, size_t h, cudaStream_t st) {
    size_t n = w * h;
    bool flat = in_pitch == w * (size_t)ncomp && plane_pitch == w && (n % 16) == 0 &&
                aligned16(in) && aligned16(planes) && (plane_stride * 4) % 16 == 0 &&
                (ncomp == 1 || ncomp == 3 || ncomp == 4);
    if (flat) {
        size_t groups = n / 16;
        const int form = ctx->planar_form;  // 0: 16 pixels per thread; 1, 2: 4 pixels per step, U = 4 or 8
        const size_t g4 = n / 4;
        const int U = form == 2 ? 8 : 4;
        unsigned blocks = form == 0 ? (unsigned)((groups + 255) / 256) : (unsigned)((g4 + 256 * U - 1) / (256 * U));
#define PF(NC, T)                                                                                   \
    do {                                                                                            \
        if (form == 0)                                                                              \
            planar_fwd_vec16<NC, T><<<blocks, 256, 0, st>>>(in, mct, (T*)planes, plane_stride, groups); \
        else if (form == 1)                                                                         \
            planar_fwd_c4<NC, T, 4><<<blocks, 256, 0, st>>>(in, mct, (T*)planes, plane_stride, g4);    \
        else                                                                                        \
            planar_fwd_c4<NC, T, 8><<<blocks, 256, 0, st>>>(in, mct, (T*)planes, plane_stride, g4);    \
    } while (0)
        if (out_dtype == J2K_I32) {
            if (ncomp == 1) PF(1, int32_t); else if (ncomp == 3) PF(3, int32_t); else PF(4, int32_t);
        } else {
            if (ncomp == 1) PF(1, float); else if (ncomp == 3) PF(3, float); else PF(4, float);
        }
#undef PF
    } else {
        dim3 grid((unsigned)((w + 255) / 256), (unsigned)h);
        if (out_dtype == J2K_I32)
            planar_fwd_generic<int32_t><<<grid, 256, 0, st>>>(in, in_pitch, ncomp, mct, (int32_t*)planes,
                                                              plane_pitch, plane_stride, (int)w, (int)h);
        else
            planar_fwd_generic<float><<<grid, 256, 0, st>>>(in, in_pitch, ncomp, mct, (float*)planes,
                                                            plane_pitch, plane_stride, (int)w, (int)h);
    }
    J2K_CUDA(ctx, cudaGetLastError());
    return J2K_OK;
}

j2k_status j2k_launch_planar_inv(j2k_ctx* ctx, const void* planes, int in_dtype,
                                 size_t plane_pitch, size_t plane_stride, int ncomp, int mct,
                                 uint8_t* out, size_t out_pitch, size_t w, size_t h,
                                 cudaStream_t st) {
    size_t n = w * h;
    bool flat = out_pitch == w * (size_t)ncomp && plane_pitch == w && (n % 16) == 0 &&
                aligned16(out) && aligned16(planes) && (plane_stride * 4) % 16 == 0 &&
                (ncomp == 1 || ncomp == 3 || ncomp == 4);
    if (flat) {
        size_t groups = n / 16;
        unsigned blocks = (unsigned)((groups + 255) / 256);
#define PI(NC, T)                                                                              \
    planar_inv_vec16<NC, T><<<blocks, 256, 0, st>>>((const T*)planes, plane_stride, mct, out, groups)
        if (in_dtype == J2K_I32) {
            if (ncomp == 1) PI(1, int32_t); else if (ncomp == 3) PI(3, int32_t); else PI(4, int32_t);
        } else {
            if (ncomp == 1) PI(1, float); else if (ncomp == 3) PI(3, float); else PI(4, float);
        }
#undef PI
    } else {
        dim3 grid((unsigned)((w + 255) / 256), (unsigned)h);
        if (in_dtype == J2K_I32)
            planar_inv_generic<int32_t><<<grid, 256, 0, st>>>((const int32_t*)planes, plane_pitch,
                                                              plane_stride, ncomp, mct, out,
                                                              out_pitch, (int)w, (int)h);
        else
            planar_inv_generic<float><<<grid, 256, 0, st>>>((const float*)planes, plane_pitch,
                                                            plane_stride, ncomp, mct, out,
                                                            out_pitch, (int)w, (int)h);
    }
    J2K_CUDA(ctx, cudaGetLastError());
    return J2K_OK;
}

j2k_status j2k_launch_cast_planes(j2k_ctx* ctx, const void* src, int sd, void* dst, int dd,
                                  size_t n, cudaStream_t st) {
    unsigned blocks = (unsigned)((n + 255) / 256);
    if (sd == J2K_I16 && dd == J2K_I32) cast_kernel<int16_t, int32_t><<<blocks, 256, 0, st>>>((const int16_t*)src, (int32_t*)dst, n);
    else if (sd == J2K_I16 && dd == J2K_F32) cast_kernel<int16_t, float><<<blocks, 256, 0, st>>>((const int16_t*)src, (float*)dst, n);
    else if (sd == J2K_I32 && dd == J2K_F32) cast_kernel<int32_t, float><<<blocks, 256, 0, st>>>((const int32_t*)src, (float*)dst, n);
    else if (sd == J2K_F32 && dd == J2K_I32) cast_kernel<float, int32_t><<<blocks, 256, 0, st>>>((const float*)src, (int32_t*)dst, n);
    else if (sd == dd) {
        J2K_CUDA(ctx, cudaMemcpyAsync(dst, src, n * 4, cudaMemcpyDeviceToDevice, st));
        return J2K_OK;
    } else return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "cast: unsupported dtype pair");
    J2K_CUDA(ctx, cudaGetLastError());
    return J2K_OK;
}

j2k_status j2k_launch_mct_planes(j2k_ctx* ctx, void* planes, int dtype, size_t stride, size_t n,
                                 int mct, cudaStream_t st) {
    unsigned blocks = (unsigned)((n + 255) / 256);
    if (dtype == J2K_I32) mct_planes_kernel<int32_t><<<blocks, 256, 0, st>>>((int32_t*)planes, stride, n, mct);
    else mct_planes_kernel<float><<<blocks, 256, 0, st>>>((float*)planes, stride, n, mct);
    J2K_CUDA(ctx, cudaGetLastError());
    return J2K_OK;
}

// ---- batched planar split: one launch for many images ------------------------------------------
// Each CTA converts a chunk of 4096 pixels of one image; chunks of all images are listed in `work`
// as (image, first pixel).  A thread takes 4 pixels in each of 4 steps (pixels first + 1024 j +
// 4 t .. + 3), so each plane's store of a warp is one contiguous run of 16-byte streaming stores
// and the loads are aligned 32-bit words (image inputs start 16-byte aligned, planes on
// 16-element boundaries); a last group of fewer than 4 pixels goes pixel by pixel.
namespace {
template <typename TO>
__global__ void __launch_bounds__(256) planar_fwd_batched(const j2k_batch_planar_desc* __restrict__ descs,
                                                          const uint2* __restrict__ work,
                                                          const uint8_t* __restrict__ in_base,
                                                          TO* __restrict__ plane_base) {
    const uint2 wk = work[blockIdx.x];
    const j2k_batch_planar_desc d = descs[wk.x];
    const uint8_t* in = in_base + d.in_off;
    TO* out = plane_base + d.plane_off;
    const int nc = d.ncomp;
    uint32_t raw[4][3];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const size_t p = (size_t)wk.y + (size_t)j * 1024 + (size_t)threadIdx.x * 4;
        if (p + 4 > d.n) continue;
        if (nc == 3) {
            const uint32_t* src = reinterpret_cast<const uint32_t*>(in + p * 3);
#pragma unroll
            for (int i = 0; i < 3; ++i) raw[j][i] = __ldcs(src + i);
        } else if (nc == 1) {
            raw[j][0] = __ldcs(reinterpret_cast<const uint32_t*>(in + p));
        }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const size_t p = (size_t)wk.y + (size_t)j * 1024 + (size_t)threadIdx.x * 4;
        if (p >= d.n) break;
        if (p + 4 <= d.n && nc == 3) {
            const uint8_t* px = reinterpret_cast<const uint8_t*>(raw[j]);
            TO o[3][4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const uint8_t* q = px + 3 * k;
                if (d.mct == J2K_MCT_RCT) {
                    const int r = (int)q[0] - 128, g = (int)q[1] - 128, b = (int)q[2] - 128;
                    o[0][k] = (TO)((r + 2 * g + b) >> 2);
                    o[1][k] = (TO)(b - g);
                    o[2][k] = (TO)(r - g);
                } else if (d.mct == J2K_MCT_ICT) {
                    const float r = (float)((int)q[0] - 128), g = (float)((int)q[1] - 128),
                                b = (float)((int)q[2] - 128);
                    o[0][k] = (TO)dot3(YR, r, YG, g, YB, b);
                    o[1][k] = (TO)dot3(BR, r, BG, g, BB, b);
                    o[2][k] = (TO)dot3(RR, r, RG, g, RB, b);
                } else {
#pragma unroll
                    for (int c = 0; c < 3; ++c) o[c][k] = (TO)((int)q[c] - 128);
                }
            }
#pragma unroll
            for (int c = 0; c < 3; ++c)
                __stcs(reinterpret_cast<uint4*>(out + c * d.stride + p), *reinterpret_cast<const uint4*>(o[c]));
        } else if (p + 4 <= d.n && nc == 1) {
            const uint8_t* px = reinterpret_cast<const uint8_t*>(raw[j]);
            TO o[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) o[k] = (TO)((int)px[k] - 128);
            __stcs(reinterpret_cast<uint4*>(out + p), *reinterpret_cast<const uint4*>(o));
        } else {
            const size_t pe = min(p + 4, d.n);
            for (size_t q = p; q < pe; ++q) fwd_pixel<TO>(in + q * nc, nc, d.mct, out, q, d.stride);
        }
    }
}
}  // namespace

j2k_status j2k_launch_planar_batched(j2k_ctx* ctx, const j2k_batch_planar_desc* d_descs, const uint2* d_work,
                                     unsigned nwork, const uint8_t* in_base, void* plane_base, int float_out,
                                     cudaStream_t st) {
    if (!nwork) return J2K_OK;
    if (float_out)
        planar_fwd_batched<float><<<nwork, 256, 0, st>>>(d_descs, d_work, in_base, (float*)plane_base);
    else
        planar_fwd_batched<int32_t><<<nwork, 256, 0, st>>>(d_descs, d_work, in_base, (int32_t*)plane_base);
    J2K_CUDA(ctx, cudaGetLastError());
    return J2K_OK;
}
