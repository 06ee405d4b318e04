/*
 * CPU oracle for the JPEG 2000 hot path — test infrastructure only (see j2k_oracle.h for what
 * each part restates and where).  Built with -ffp-contract=off so that every float operation
 * rounds exactly once, in the order written; the CUDA kernels use the same order with
 * explicitly rounded intrinsics, which makes the FP32 9/7 path bit-comparable.
 */
#include "j2k_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ============================================================================================
 * Planar split + level shift + colour transforms (src/CL/oclplanar.cl:23-40, T.800 Annex G)
 * ========================================================================================== */

/* ICT coefficients, T.800 G.3 (forward) / G.3 (inverse). */
#define ICT_YR 0.299f
#define ICT_YG 0.587f
#define ICT_YB 0.114f
#define ICT_BR (-0.16875f)
#define ICT_BG (-0.33126f)
#define ICT_BB 0.5f
#define ICT_RR 0.5f
#define ICT_RG (-0.41869f)
#define ICT_RB (-0.08131f)
#define ICTI_RV 1.402f
#define ICTI_GU (-0.34413f)
#define ICTI_GV (-0.71414f)
#define ICTI_BU 1.772f

void or_planar_fwd_i32(const uint8_t* src, size_t w, size_t h, size_t src_pitch, int ncomp,
                       int mct, int32_t* dst, size_t dst_pitch, size_t plane_stride) {
    for (size_t y = 0; y < h; ++y) {
        const uint8_t* row = src + y * src_pitch;
        for (size_t x = 0; x < w; ++x) {
            const uint8_t* px = row + x * (size_t)ncomp;
            if (mct == OR_MCT_RCT && ncomp >= 3) {
                int32_t r = (int32_t)px[0] - 128, g = (int32_t)px[1] - 128, b = (int32_t)px[2] - 128;
                dst[0 * plane_stride + y * dst_pitch + x] = (r + 2 * g + b) >> 2;
                dst[1 * plane_stride + y * dst_pitch + x] = b - g;
                dst[2 * plane_stride + y * dst_pitch + x] = r - g;
                for (int c = 3; c < ncomp; ++c)
                    dst[(size_t)c * plane_stride + y * dst_pitch + x] = (int32_t)px[c] - 128;
            } else {
                for (int c = 0; c < ncomp; ++c)
                    dst[(size_t)c * plane_stride + y * dst_pitch + x] = (int32_t)px[c] - 128;
            }
        }
    }
}

void or_planar_fwd_f32(const uint8_t* src, size_t w, size_t h, size_t src_pitch, int ncomp,
                       int mct, float* dst, size_t dst_pitch, size_t plane_stride) {
    for (size_t y = 0; y < h; ++y) {
        const uint8_t* row = src + y * src_pitch;
        for (size_t x = 0; x < w; ++x) {
            const uint8_t* px = row + x * (size_t)ncomp;
            if (mct == OR_MCT_ICT && ncomp >= 3) {
                float r = (float)((int)px[0] - 128), g = (float)((int)px[1] - 128),
                      b = (float)((int)px[2] - 128);
                dst[0 * plane_stride + y * dst_pitch + x] = (ICT_YR * r + ICT_YG * g) + ICT_YB * b;
                dst[1 * plane_stride + y * dst_pitch + x] = (ICT_BR * r + ICT_BG * g) + ICT_BB * b;
                dst[2 * plane_stride + y * dst_pitch + x] = (ICT_RR * r + ICT_RG * g) + ICT_RB * b;
                for (int c = 3; c < ncomp; ++c)
                    dst[(size_t)c * plane_stride + y * dst_pitch + x] = (float)((int)px[c] - 128);
            } else {
                for (int c = 0; c < ncomp; ++c)
                    dst[(size_t)c * plane_stride + y * dst_pitch + x] = (float)((int)px[c] - 128);
            }
        }
    }
}

static uint8_t clamp_u8(int32_t v) { return (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v)); }

void or_planar_inv_i32(const int32_t* src, size_t src_pitch, size_t plane_stride, size_t w,
                       size_t h, int ncomp, int mct, uint8_t* dst, size_t dst_pitch) {
    for (size_t y = 0; y < h; ++y) {
        for (size_t x = 0; x < w; ++x) {
            uint8_t* px = dst + y * dst_pitch + x * (size_t)ncomp;
            if (mct == OR_MCT_RCT && ncomp >= 3) {
                int32_t Y = src[y * src_pitch + x], U = src[plane_stride + y * src_pitch + x],
                        V = src[2 * plane_stride + y * src_pitch + x];
                int32_t g = Y - ((U + V) >> 2);
                px[0] = clamp_u8(V + g + 128);
                px[1] = clamp_u8(g + 128);
                px[2] = clamp_u8(U + g + 128);
                for (int c = 3; c < ncomp; ++c)
                    px[c] = clamp_u8(src[(size_t)c * plane_stride + y * src_pitch + x] + 128);
            } else {
                for (int c = 0; c < ncomp; ++c)
                    px[c] = clamp_u8(src[(size_t)c * plane_stride + y * src_pitch + x] + 128);
            }
        }
    }
}

static uint8_t round_clamp_u8(float v) {
    float r = rintf(v + 128.0f);
    return (uint8_t)(r < 0.0f ? 0 : (r > 255.0f ? 255 : (int)r));
}

void or_planar_inv_f32(const float* src, size_t src_pitch, size_t plane_stride, size_t w,
                       size_t h, int ncomp, int mct, uint8_t* dst, size_t dst_pitch) {
    for (size_t y = 0; y < h; ++y) {
        for (size_t x = 0; x < w; ++x) {
            uint8_t* px = dst + y * dst_pitch + x * (size_t)ncomp;
            if (mct == OR_MCT_ICT && ncomp >= 3) {
                float Y = src[y * src_pitch + x], U = src[plane_stride + y * src_pitch + x],
                      V = src[2 * plane_stride + y * src_pitch + x];
                px[0] = round_clamp_u8(Y + ICTI_RV * V);
                px[1] = round_clamp_u8((Y + ICTI_GU * U) + ICTI_GV * V);
                px[2] = round_clamp_u8(Y + ICTI_BU * U);
                for (int c = 3; c < ncomp; ++c)
                    px[c] = round_clamp_u8(src[(size_t)c * plane_stride + y * src_pitch + x]);
            } else {
                for (int c = 0; c < ncomp; ++c)
                    px[c] = round_clamp_u8(src[(size_t)c * plane_stride + y * src_pitch + x]);
            }
        }
    }
}

/* ============================================================================================
 * 1-D lifting kernels.  Whole-sample symmetric extension (src/CL/ocldwt53.cl:86 sampler);
 * the extension preserves parity, so lifted intermediates are mirrored with the same rule.
 * ========================================================================================== */

static long mirror_idx(long i, long n) {
    if (n == 1) return 0;
    long p = 2 * (n - 1);
    i %= p;
    if (i < 0) i += p;
    if (i >= n) i = p - i;
    return i;
}

/* 5/3: src/CL/ocldwt53.cl:223 (predict) and :228 (update). */
static void fwd53_1d(int32_t* s, long n, int32_t* tmp) {
    if (n == 1) return;
    for (long i = 1; i < n; i += 2) s[i] -= (s[mirror_idx(i - 1, n)] + s[mirror_idx(i + 1, n)]) >> 1;
    for (long i = 0; i < n; i += 2) s[i] += (s[mirror_idx(i - 1, n)] + s[mirror_idx(i + 1, n)] + 2) >> 2;
    long nl = (n + 1) / 2;
    for (long i = 0; i < n; ++i) tmp[(i & 1) ? nl + i / 2 : i / 2] = s[i];
    memcpy(s, tmp, (size_t)n * sizeof(int32_t));
}

static void inv53_1d(int32_t* s, long n, int32_t* tmp) {
    if (n == 1) return;
    long nl = (n + 1) / 2;
    for (long i = 0; i < n; ++i) tmp[i] = s[(i & 1) ? nl + i / 2 : i / 2];
    for (long i = 0; i < n; i += 2) tmp[i] -= (tmp[mirror_idx(i - 1, n)] + tmp[mirror_idx(i + 1, n)] + 2) >> 2;
    for (long i = 1; i < n; i += 2) tmp[i] += (tmp[mirror_idx(i - 1, n)] + tmp[mirror_idx(i + 1, n)]) >> 1;
    memcpy(s, tmp, (size_t)n * sizeof(int32_t));
}

/* 9/7 constants exactly as written in src/CL/ocldwt97.cl:69-78. */
#define P1F (-1.586134342f)
#define U1F (-0.05298011854f)
#define P2F 0.8829110762f
#define U2F 0.4435068522f
#define KMULF 1.23017410491400f
#define KDIVF 0.81289306611596153187273657637352f
#define P1D (-1.586134342)
#define U1D (-0.05298011854)
#define P2D 0.8829110762
#define U2D 0.4435068522
#define KMULD 1.23017410491400
#define KDIVD 0.81289306611596153187273657637352

#define DEF_97(T, SUF, P1, U1, P2, U2, KM, KD)                                                 \
    static void lift_##SUF(T* s, long n, int par, T a) {                                      \
        for (long i = par; i < n; i += 2) {                                                   \
            T t = s[mirror_idx(i - 1, n)] + s[mirror_idx(i + 1, n)];                          \
            t = a * t;                                                                        \
            s[i] = s[i] + t;                                                                  \
        }                                                                                     \
    }                                                                                         \
    static void fwd97_1d_##SUF(T* s, long n, T* tmp) {                                        \
        if (n == 1) return;                                                                   \
        lift_##SUF(s, n, 1, P1);                                                              \
        lift_##SUF(s, n, 0, U1);                                                              \
        lift_##SUF(s, n, 1, P2);                                                              \
        lift_##SUF(s, n, 0, U2);                                                              \
        long nl = (n + 1) / 2;                                                                \
        for (long i = 0; i < n; ++i) tmp[(i & 1) ? nl + i / 2 : i / 2] = s[i] * ((i & 1) ? KM : KD); \
        memcpy(s, tmp, (size_t)n * sizeof(T));                                                \
    }                                                                                         \
    static void inv97_1d_##SUF(T* s, long n, T* tmp) {                                        \
        if (n == 1) return;                                                                   \
        long nl = (n + 1) / 2;                                                                \
        for (long i = 0; i < n; ++i) tmp[i] = s[(i & 1) ? nl + i / 2 : i / 2] * ((i & 1) ? KD : KM); \
        lift_##SUF(tmp, n, 0, -(U2));                                                         \
        lift_##SUF(tmp, n, 1, -(P2));                                                         \
        lift_##SUF(tmp, n, 0, -(U1));                                                         \
        lift_##SUF(tmp, n, 1, -(P1));                                                         \
        memcpy(s, tmp, (size_t)n * sizeof(T));                                                \
    }

DEF_97(float, f32, P1F, U1F, P2F, U2F, KMULF, KDIVF)
DEF_97(double, f64, P1D, U1D, P2D, U2D, KMULD, KDIVD)

/* ============================================================================================
 * 2-D multi-level drivers.  Level sizes follow ceil(n/2) (src/OCLDWTForward.cpp:124-137);
 * Mallat placement as src/CL/ocldwt53.cl:110-160,174 (low half first on both axes).
 * ========================================================================================== */

#define DEF_PASSES(T, TAG, F1D, I1D)                                                          \
    static void rows_##TAG(T* d, size_t pitch, size_t w, size_t h, T* tmp, T* tmp2, int inv) { \
        for (size_t y = 0; y < h; ++y) {                                                      \
            memcpy(tmp, d + y * pitch, w * sizeof(T));                                        \
            if (inv) I1D(tmp, (long)w, tmp2); else F1D(tmp, (long)w, tmp2);                   \
            memcpy(d + y * pitch, tmp, w * sizeof(T));                                        \
        }                                                                                     \
    }                                                                                         \
    static void cols_##TAG(T* d, size_t pitch, size_t w, size_t h, T* tmp, T* tmp2, int inv) { \
        for (size_t x = 0; x < w; ++x) {                                                      \
            for (size_t y = 0; y < h; ++y) tmp[y] = d[y * pitch + x];                         \
            if (inv) I1D(tmp, (long)h, tmp2); else F1D(tmp, (long)h, tmp2);                   \
            for (size_t y = 0; y < h; ++y) d[y * pitch + x] = tmp[y];                         \
        }                                                                                     \
    }

#define DEF_2D(T, TAG, NAME_F, NAME_I)                                                        \
    void NAME_F(const T* in, size_t in_pitch, T* out, size_t out_pitch, size_t w, size_t h,   \
                int levels, int order) {                                                      \
        size_t m = (w > h ? w : h) + 8;                                                       \
        T* tmp = (T*)malloc(m * sizeof(T));                                                   \
        T* tmp2 = (T*)malloc(m * sizeof(T));                                                  \
        for (size_t y = 0; y < h; ++y) memcpy(out + y * out_pitch, in + y * in_pitch, w * sizeof(T)); \
        size_t cw = w, ch = h;                                                                \
        for (int l = 0; l < levels; ++l) {                                                    \
            if (order == OR_ORDER_REF) {                                                      \
                rows_##TAG(out, out_pitch, cw, ch, tmp, tmp2, 0);                          \
                cols_##TAG(out, out_pitch, cw, ch, tmp, tmp2, 0);                          \
            } else {                                                                          \
                cols_##TAG(out, out_pitch, cw, ch, tmp, tmp2, 0);                          \
                rows_##TAG(out, out_pitch, cw, ch, tmp, tmp2, 0);                          \
            }                                                                                 \
            cw = (cw + 1) / 2;                                                                \
            ch = (ch + 1) / 2;                                                                \
        }                                                                                     \
        free(tmp);                                                                            \
        free(tmp2);                                                                           \
    }                                                                                         \
    void NAME_I(const T* in, size_t in_pitch, T* out, size_t out_pitch, size_t w, size_t h,   \
                int levels, int order) {                                                      \
        size_t m = (w > h ? w : h) + 8;                                                       \
        T* tmp = (T*)malloc(m * sizeof(T));                                                   \
        T* tmp2 = (T*)malloc(m * sizeof(T));                                                  \
        for (size_t y = 0; y < h; ++y) memcpy(out + y * out_pitch, in + y * in_pitch, w * sizeof(T)); \
        for (int l = levels - 1; l >= 0; --l) {                                               \
            size_t cw = w, ch = h;                                                            \
            for (int k = 0; k < l; ++k) { cw = (cw + 1) / 2; ch = (ch + 1) / 2; }             \
            if (order == OR_ORDER_REF) {                                                      \
                cols_##TAG(out, out_pitch, cw, ch, tmp, tmp2, 1);                          \
                rows_##TAG(out, out_pitch, cw, ch, tmp, tmp2, 1);                          \
            } else {                                                                          \
                rows_##TAG(out, out_pitch, cw, ch, tmp, tmp2, 1);                          \
                cols_##TAG(out, out_pitch, cw, ch, tmp, tmp2, 1);                          \
            }                                                                                 \
        }                                                                                     \
        free(tmp);                                                                            \
        free(tmp2);                                                                           \
    }

DEF_PASSES(int32_t, i53, fwd53_1d, inv53_1d)
DEF_PASSES(float, f97, fwd97_1d_f32, inv97_1d_f32)
DEF_PASSES(double, d97, fwd97_1d_f64, inv97_1d_f64)
DEF_2D(int32_t, i53, or_dwt53_fwd, or_dwt53_inv)
DEF_2D(float, f97, or_dwt97_fwd_f32, or_dwt97_inv_f32)
DEF_2D(double, d97, or_dwt97_fwd_f64, or_dwt97_inv_f64)

/* ---- adjoints of the FP64 9/7 transforms (T800 order) ------------------------------------ */

/* transpose of lift_f64(s, n, par, a): every `par` position i scatters a*g[i] to its two
 * (mirrored) neighbours; `par` positions themselves are unchanged. */
static void lift_adj_f64(double* g, long n, int par, double a) {
    for (long i = par; i < n; i += 2) {
        double v = a * g[i];
        g[mirror_idx(i - 1, n)] += v;
        g[mirror_idx(i + 1, n)] += v;
    }
}

/* adjoint of fwd97_1d_f64: g holds the gradient in deinterleaved (low|high) order. */
static void fwd97_adj_1d(double* g, long n, double* tmp) {
    if (n == 1) return;
    long nl = (n + 1) / 2;
    for (long i = 0; i < n; ++i) tmp[i] = g[(i & 1) ? nl + i / 2 : i / 2] * ((i & 1) ? KMULD : KDIVD);
    lift_adj_f64(tmp, n, 0, U2D);
    lift_adj_f64(tmp, n, 1, P2D);
    lift_adj_f64(tmp, n, 0, U1D);
    lift_adj_f64(tmp, n, 1, P1D);
    memcpy(g, tmp, (size_t)n * sizeof(double));
}

/* adjoint of inv97_1d_f64: g holds the gradient in natural order, result deinterleaved. */
static void inv97_adj_1d(double* g, long n, double* tmp) {
    if (n == 1) return;
    lift_adj_f64(g, n, 1, -P1D);
    lift_adj_f64(g, n, 0, -U1D);
    lift_adj_f64(g, n, 1, -P2D);
    lift_adj_f64(g, n, 0, -U2D);
    long nl = (n + 1) / 2;
    for (long i = 0; i < n; ++i) tmp[(i & 1) ? nl + i / 2 : i / 2] = g[i] * ((i & 1) ? KDIVD : KMULD);
    memcpy(g, tmp, (size_t)n * sizeof(double));
}

DEF_PASSES(double, adj, fwd97_adj_1d, inv97_adj_1d)

void or_dwt97_fwd_adj_f64(const double* g_out, size_t gpitch, double* g_in, size_t ipitch,
                          size_t w, size_t h, int levels) {
    /* forward = per level: columns, then rows.  Adjoint: deepest level first, per level the
     * row adjoint then the column adjoint. */
    size_t m = (w > h ? w : h) + 8;
    double* tmp = (double*)malloc(m * sizeof(double));
    double* tmp2 = (double*)malloc(m * sizeof(double));
    for (size_t y = 0; y < h; ++y) memcpy(g_in + y * ipitch, g_out + y * gpitch, w * sizeof(double));
    for (int l = levels - 1; l >= 0; --l) {
        size_t cw = w, ch = h;
        for (int k = 0; k < l; ++k) { cw = (cw + 1) / 2; ch = (ch + 1) / 2; }
        rows_adj(g_in, ipitch, cw, ch, tmp, tmp2, 0);
        cols_adj(g_in, ipitch, cw, ch, tmp, tmp2, 0);
    }
    free(tmp);
    free(tmp2);
}

void or_dwt97_inv_adj_f64(const double* g_img, size_t gpitch, double* g_coef, size_t cpitch,
                          size_t w, size_t h, int levels) {
    /* inverse = deepest level first, per level rows^-1 then cols^-1.  Adjoint: level 0 first,
     * per level the column adjoint then the row adjoint. */
    size_t m = (w > h ? w : h) + 8;
    double* tmp = (double*)malloc(m * sizeof(double));
    double* tmp2 = (double*)malloc(m * sizeof(double));
    for (size_t y = 0; y < h; ++y) memcpy(g_coef + y * cpitch, g_img + y * gpitch, w * sizeof(double));
    size_t cw = w, ch = h;
    for (int l = 0; l < levels; ++l) {
        cols_adj(g_coef, cpitch, cw, ch, tmp, tmp2, 1);
        rows_adj(g_coef, cpitch, cw, ch, tmp, tmp2, 1);
        cw = (cw + 1) / 2;
        ch = (ch + 1) / 2;
    }
    free(tmp);
    free(tmp2);
}

/* ============================================================================================
 * Subband geometry and the dead-zone quantiser (T.800 E.1)
 * ========================================================================================== */

int or_subband_rect(size_t w, size_t h, int levels, int b, size_t* x0, size_t* y0, size_t* sw,
                    size_t* sh, int* orient, int* level) {
    size_t ws[40], hs[40];
    ws[0] = w;
    hs[0] = h;
    for (int k = 1; k <= levels; ++k) { ws[k] = (ws[k - 1] + 1) / 2; hs[k] = (hs[k - 1] + 1) / 2; }
    if (b == 0) {
        *x0 = 0; *y0 = 0; *sw = ws[levels]; *sh = hs[levels]; *orient = OR_LL; *level = levels;
    } else {
        int k = levels - (b - 1) / 3;      /* decomposition level of this triple */
        int o = 1 + (b - 1) % 3;           /* 1 HL, 2 LH, 3 HH */
        size_t lw = ws[k], lh = hs[k], pw = ws[k - 1], ph = hs[k - 1];
        *orient = o;
        *level = k;
        *x0 = (o == OR_HL || o == OR_HH) ? lw : 0;
        *y0 = (o == OR_LH || o == OR_HH) ? lh : 0;
        *sw = (o == OR_HL || o == OR_HH) ? pw - lw : lw;
        *sh = (o == OR_LH || o == OR_HH) ? ph - lh : lh;
    }
    return 3 * levels + 1;
}

void or_quantize_f32(const float* in, size_t in_pitch, int32_t* q, size_t q_pitch, size_t w,
                     size_t h, int levels, const float* steps) {
    int nb = 3 * levels + 1;
    for (int b = 0; b < nb; ++b) {
        size_t x0, y0, sw, sh;
        int o, l;
        or_subband_rect(w, h, levels, b, &x0, &y0, &sw, &sh, &o, &l);
        float st = steps[b];
        for (size_t y = y0; y < y0 + sh; ++y)
            for (size_t x = x0; x < x0 + sw; ++x) {
                float v = in[y * in_pitch + x];
                float a = fabsf(v) / st;
                int32_t m = (int32_t)floorf(a);
                q[y * q_pitch + x] = v < 0.0f ? -m : m;
            }
    }
}

void or_dequantize_f32(const int32_t* q, size_t q_pitch, float* out, size_t out_pitch, size_t w,
                       size_t h, int levels, const float* steps) {
    int nb = 3 * levels + 1;
    for (int b = 0; b < nb; ++b) {
        size_t x0, y0, sw, sh;
        int o, l;
        or_subband_rect(w, h, levels, b, &x0, &y0, &sw, &sh, &o, &l);
        float st = steps[b];
        for (size_t y = y0; y < y0 + sh; ++y)
            for (size_t x = x0; x < x0 + sw; ++x) {
                int32_t v = q[y * q_pitch + x];
                int32_t m = v < 0 ? -v : v;
                float r = m ? ((float)m + 0.5f) * st : 0.0f;
                out[y * out_pitch + x] = v < 0 ? -r : r;
            }
    }
}

/* ============================================================================================
 * MQ arithmetic coder, T.800 Annex C (Table C.2 probability states; C.2 encoder incl. the
 * FLUSH of C.2.9; C.3 decoder).
 * ========================================================================================== */

static const uint16_t MQ_QE[47] = {
    0x5601, 0x3401, 0x1801, 0x0AC1, 0x0521, 0x0221, 0x5601, 0x5401, 0x4801, 0x3801, 0x3001, 0x2401,
    0x1C01, 0x1601, 0x5601, 0x5401, 0x5101, 0x4801, 0x3801, 0x3401, 0x3001, 0x2801, 0x2401, 0x2201,
    0x1C01, 0x1801, 0x1601, 0x1401, 0x1201, 0x1101, 0x0AC1, 0x09C1, 0x08A1, 0x0521, 0x0441, 0x02A1,
    0x0221, 0x0141, 0x0111, 0x0085, 0x0049, 0x0025, 0x0015, 0x0009, 0x0005, 0x0001, 0x5601};
static const uint8_t MQ_NMPS[47] = {1,  2,  3,  4,  5,  38, 7,  8,  9,  10, 11, 12, 13, 29, 15, 16,
                                    17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32,
                                    33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 44, 45, 45, 46};
static const uint8_t MQ_NLPS[47] = {1,  6,  9,  12, 29, 33, 6,  14, 14, 14, 17, 18, 20, 21, 14, 14,
                                    15, 16, 17, 18, 19, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29,
                                    30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 46};
static const uint8_t MQ_SW[47] = {1, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                                  0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};

/* Context labels: ZC 0-8, SC 9-13, MR 14-16, run-length 17, uniform 18 (T.800 Table D.7 for
 * the initial states). */
#define CX_RL 17
#define CX_UNI 18
#define NCX 19

typedef struct {
    uint32_t A, C;
    int CT, bp, cap, ovf;
    uint8_t* out;
    uint8_t st[NCX], mps[NCX];
    uint8_t* syms;
    int sym_cap, nsyms;
} mqe_t;

static void mq_reset_states(uint8_t* st, uint8_t* mps) {
    for (int i = 0; i < NCX; ++i) { st[i] = 0; mps[i] = 0; }
    st[0] = 4;
    st[CX_RL] = 3;
    st[CX_UNI] = 46;
}

/* INITENC (C.2.8) of a codeword segment starting at `out`; the context states are kept */
static void mqe_start(mqe_t* e, uint8_t* out, int cap) {
    e->A = 0x8000;
    e->C = 0;
    e->CT = 12;
    e->bp = -1;
    e->out = out;
    e->cap = cap;
}

static void mqe_init(mqe_t* e, uint8_t* out, int cap) {
    mqe_start(e, out, cap);
    e->ovf = 0;
    e->nsyms = 0;
    mq_reset_states(e->st, e->mps);
}

static void mqe_put(mqe_t* e, int idx, uint8_t v) {
    if (idx < e->cap) e->out[idx] = v; else e->ovf = 1;
}
static uint8_t mqe_get(mqe_t* e, int idx) {
    if (idx < 0) return 0;
    return idx < e->cap ? e->out[idx] : 0;
}

static void mqe_byteout(mqe_t* e) {
    if (mqe_get(e, e->bp) == 0xFF) {
        e->bp++;
        mqe_put(e, e->bp, (uint8_t)(e->C >> 20));
        e->C &= 0xFFFFF;
        e->CT = 7;
    } else if (e->C < 0x8000000) {
        e->bp++;
        mqe_put(e, e->bp, (uint8_t)(e->C >> 19));
        e->C &= 0x7FFFF;
        e->CT = 8;
    } else {
        uint8_t b = (uint8_t)(mqe_get(e, e->bp) + 1);
        if (e->bp >= 0) mqe_put(e, e->bp, b);
        if (b == 0xFF) {
            e->C &= 0x7FFFFFF;
            e->bp++;
            mqe_put(e, e->bp, (uint8_t)(e->C >> 20));
            e->C &= 0xFFFFF;
            e->CT = 7;
        } else {
            e->bp++;
            mqe_put(e, e->bp, (uint8_t)(e->C >> 19));
            e->C &= 0x7FFFF;
            e->CT = 8;
        }
    }
}

static void mqe_renorm(mqe_t* e) {
    do {
        e->A <<= 1;
        e->C <<= 1;
        e->CT--;
        if (e->CT == 0) mqe_byteout(e);
    } while ((e->A & 0x8000) == 0);
}

static void mqe_encode(mqe_t* e, int cx, int d) {
    if (e->syms) {
        if (e->nsyms < e->sym_cap) e->syms[e->nsyms] = (uint8_t)(cx | (d ? 0x80 : 0));
    }
    e->nsyms++;
    int s = e->st[cx];
    uint32_t qe = MQ_QE[s];
    e->A -= qe;
    if (d == e->mps[cx]) {
        if ((e->A & 0x8000) == 0) {
            if (e->A < qe) e->A = qe; else e->C += qe;
            e->st[cx] = MQ_NMPS[s];
            mqe_renorm(e);
        } else {
            e->C += qe;
        }
    } else {
        if (e->A < qe) e->C += qe; else e->A = qe;
        if (MQ_SW[s]) e->mps[cx] ^= 1;
        e->st[cx] = MQ_NLPS[s];
        mqe_renorm(e);
    }
}

static int mqe_flush(mqe_t* e) {
    uint32_t tempc = e->C + e->A;
    e->C |= 0xFFFF;
    if (e->C >= tempc) e->C -= 0x8000;
    e->C <<= e->CT;
    mqe_byteout(e);
    e->C <<= e->CT;
    mqe_byteout(e);
    /* a codeword never ends with 0xFF: the last 0xFF byte is dropped */
    int len = e->bp + 1;
    if (len > 0 && mqe_get(e, e->bp) == 0xFF) len--;
    return len;
}

/* Raw (bypass) segments, T.800 D.6: decisions written as bits, most significant bit of each
 * byte first; a byte that follows 0xFF carries 7 bits (its top bit is a stuffed 0).  At the
 * end of a segment the bits of a partial byte are padded with 0s, and a last byte of 0xFF is
 * dropped (a decoder reads 0xFF past the end of a segment, as the MQ decoder does). */
typedef struct {
    uint8_t* out;
    int cap, pos, ovf;
    uint32_t c;
    int ct, lastff;
} rawe_t;

static void rawe_start(rawe_t* r, uint8_t* out, int cap) {
    r->out = out;
    r->cap = cap;
    r->pos = 0;
    r->ovf = 0;
    r->c = 0;
    r->ct = 8;
    r->lastff = 0;
}

static void rawe_byte(rawe_t* r, uint8_t b) {
    if (r->pos < r->cap) r->out[r->pos] = b; else r->ovf = 1;
    r->pos++;
    r->lastff = b == 0xFF;
    r->ct = r->lastff ? 7 : 8;
    r->c = 0;
}

static void rawe_put(rawe_t* r, int bit) {
    r->c = (r->c << 1) | (uint32_t)(bit & 1);
    if (--r->ct == 0) rawe_byte(r, (uint8_t)r->c);
}

static int rawe_flush(rawe_t* r) {
    if (r->ct < (r->lastff ? 7 : 8)) rawe_byte(r, (uint8_t)(r->c << r->ct));
    int len = r->pos;
    if (len > 0 && len <= r->cap && r->out[len - 1] == 0xFF) len--;
    return len;
}

typedef struct {
    const uint8_t* data;
    int len, pos, ct, lastff;
    uint32_t c;
} rawd_t;

static void rawd_start(rawd_t* r, const uint8_t* data, int len) {
    r->data = data;
    r->len = len;
    r->pos = 0;
    r->ct = 0;
    r->lastff = 0;
    r->c = 0;
}

static int rawd_get(rawd_t* r) {
    if (r->ct == 0) {
        uint8_t b = r->pos < r->len ? r->data[r->pos] : 0xFF;
        r->pos++;
        r->ct = r->lastff ? 7 : 8;
        r->lastff = b == 0xFF;
        r->c = b;
    }
    r->ct--;
    return (int)((r->c >> r->ct) & 1);
}

typedef struct {
    const uint8_t* data;
    int len, bp;
    uint32_t A, C;
    int CT;
    uint8_t st[NCX], mps[NCX];
} mqd_t;

static uint8_t mqd_byte(const mqd_t* d, int i) { return i < d->len ? d->data[i] : 0xFF; }

static void mqd_bytein(mqd_t* d) {
    if (mqd_byte(d, d->bp) == 0xFF) {
        if (mqd_byte(d, d->bp + 1) > 0x8F) {
            d->C += 0xFF00;
            d->CT = 8;
        } else {
            d->bp++;
            d->C += (uint32_t)mqd_byte(d, d->bp) << 9;
            d->CT = 7;
        }
    } else {
        d->bp++;
        d->C += (uint32_t)mqd_byte(d, d->bp) << 8;
        d->CT = 8;
    }
}

/* INITDEC (C.3.5) on a codeword segment; the context states are kept */
static void mqd_start(mqd_t* d, const uint8_t* data, int len) {
    d->data = data;
    d->len = len;
    d->bp = 0;
    d->C = (uint32_t)mqd_byte(d, 0) << 16;
    mqd_bytein(d);
    d->C <<= 7;
    d->CT -= 7;
    d->A = 0x8000;
}

static void mqd_init(mqd_t* d, const uint8_t* data, int len) {
    mqd_start(d, data, len);
    mq_reset_states(d->st, d->mps);
}

static void mqd_renorm(mqd_t* d) {
    do {
        if (d->CT == 0) mqd_bytein(d);
        d->A <<= 1;
        d->C <<= 1;
        d->CT--;
    } while ((d->A & 0x8000) == 0);
}

static int mqd_decode(mqd_t* d, int cx) {
    int s = d->st[cx];
    uint32_t qe = MQ_QE[s];
    int D;
    d->A -= qe;
    if ((d->C >> 16) < qe) {
        /* LPS exchange */
        if (d->A < qe) {
            d->A = qe;
            D = d->mps[cx];
            d->st[cx] = MQ_NMPS[s];
        } else {
            d->A = qe;
            D = 1 - d->mps[cx];
            if (MQ_SW[s]) d->mps[cx] ^= 1;
            d->st[cx] = MQ_NLPS[s];
        }
        mqd_renorm(d);
    } else {
        d->C -= qe << 16;
        if ((d->A & 0x8000) == 0) {
            /* MPS exchange */
            if (d->A < qe) {
                D = 1 - d->mps[cx];
                if (MQ_SW[s]) d->mps[cx] ^= 1;
                d->st[cx] = MQ_NLPS[s];
            } else {
                D = d->mps[cx];
                d->st[cx] = MQ_NMPS[s];
            }
            mqd_renorm(d);
        } else {
            D = d->mps[cx];
        }
    }
    return D;
}

/* ============================================================================================
 * EBCOT tier-1 (scan order and passes: src/CL/oclbpc.cl:19-111; context tables :205-275 and
 * T.800 Tables D.1-D.4; run-length mode D.3.4).
 * ========================================================================================== */

#define F_SIG 1   /* sigma: significant */
#define F_REF 2   /* sigma': refined at least once */
#define F_VIS 4   /* eta: coded in this plane's significance propagation pass */
#define F_NEG 8   /* sign (1 = negative) */

typedef struct {
    int cw, ch, stride; /* state grid has a one-sample border */
    uint8_t* f;
} t1st_t;

#define FLAG(t, x, y) ((t)->f[((y) + 1) * (t)->stride + (x) + 1])

static int sig_at(const t1st_t* t, int x, int y) { return FLAG(t, x, y) & F_SIG; }

static void nbr_counts(const t1st_t* t, int x, int y, int* h, int* v, int* d) {
    *h = (sig_at(t, x - 1, y) != 0) + (sig_at(t, x + 1, y) != 0);
    *v = (sig_at(t, x, y - 1) != 0) + (sig_at(t, x, y + 1) != 0);
    *d = (sig_at(t, x - 1, y - 1) != 0) + (sig_at(t, x + 1, y - 1) != 0) +
         (sig_at(t, x - 1, y + 1) != 0) + (sig_at(t, x + 1, y + 1) != 0);
}

/* Zero-coding label, T.800 Table D.1.  The HL band (horizontally high-pass) uses the LL/LH
 * table with the horizontal and vertical counts exchanged. */
static int zc_label(int orient, int h, int v, int d) {
    if (orient == OR_HH) {
        int hv = h + v;
        if (d >= 3) return 8;
        if (d == 2) return hv >= 1 ? 7 : 6;
        if (d == 1) return hv >= 2 ? 5 : (hv == 1 ? 4 : 3);
        return hv >= 2 ? 2 : (hv == 1 ? 1 : 0);
    }
    if (orient == OR_HL) { int tt = h; h = v; v = tt; }
    if (h == 2) return 8;
    if (h == 1) return v >= 1 ? 7 : (d >= 1 ? 6 : 5);
    if (v == 2) return 4;
    if (v == 1) return 3;
    return d >= 2 ? 2 : d;
}

static int sgn_contrib(const t1st_t* t, int x, int y) {
    uint8_t f = FLAG(t, x, y);
    if (!(f & F_SIG)) return 0;
    return (f & F_NEG) ? -1 : 1;
}

/* Sign-coding label and XOR bit, T.800 Tables D.2/D.3.  The table is symmetric under negating
 * both contributions with the XOR bit flipped, so it is folded onto hc >= 0. */
static int sc_label(const t1st_t* t, int x, int y, int* xorbit) {
    int hc = sgn_contrib(t, x - 1, y) + sgn_contrib(t, x + 1, y);
    int vc = sgn_contrib(t, x, y - 1) + sgn_contrib(t, x, y + 1);
    hc = hc < -1 ? -1 : (hc > 1 ? 1 : hc);
    vc = vc < -1 ? -1 : (vc > 1 ? 1 : vc);
    *xorbit = 0;
    if (hc < 0 || (hc == 0 && vc < 0)) { hc = -hc; vc = -vc; *xorbit = 1; }
    if (hc == 0) return vc ? 10 : 9;
    return 12 + vc;
}

static int mr_label(const t1st_t* t, int x, int y) {
    if (FLAG(t, x, y) & F_REF) return 16;
    int h, v, d;
    nbr_counts(t, x, y, &h, &v, &d);
    return (h + v + d) ? 15 : 14;
}

static int t1_alloc(t1st_t* t, int cw, int ch) {
    t->cw = cw;
    t->ch = ch;
    t->stride = cw + 2;
    t->f = (uint8_t*)calloc((size_t)(cw + 2) * (ch + 2), 1);
    return t->f != NULL;
}

/* ---- code-block styles (T.800 Table A.19, D.6): which passes are raw-coded, and after which
 * passes the codeword is terminated (a new codeword segment starts with the next pass). */
int or_t1_pass_raw(int style, int pass) {
    return (style & OR_STYLE_BYPASS) && pass >= 10 && pass % 3 != 0;
}

int or_t1_pass_terminated(int style, int pass, int npasses) {
    if (pass >= npasses - 1 || (style & OR_STYLE_TERMALL)) return 1;
    return or_t1_pass_raw(style, pass) != or_t1_pass_raw(style, pass + 1);
}

/* Tier-1 coder of one code-block: MQ or raw per pass, segments terminated per the style. */
typedef struct {
    mqe_t e;
    rawe_t r;
    int style, raw, open;
    uint8_t* out;
    int cap, base, ovf;
} t1e_t;

static void t1e_bit(t1e_t* E, int cx, int d) {
    if (E->raw) rawe_put(&E->r, d); else mqe_encode(&E->e, cx, d);
}

/* sign of a newly significant sample: MQ codes it XOR the context's bit, raw codes it as is */
static void t1e_sign(t1e_t* E, int cx, int xb, int neg) {
    if (E->raw) rawe_put(&E->r, neg); else mqe_encode(&E->e, cx, neg ^ xb);
}

static void t1e_begin(t1e_t* E, int pass) {
    if (pass > 0 && (E->style & OR_STYLE_RESET)) mq_reset_states(E->e.st, E->e.mps);
    E->raw = or_t1_pass_raw(E->style, pass);
    if (!E->open) {
        if (E->raw) rawe_start(&E->r, E->out + E->base, E->cap - E->base);
        else mqe_start(&E->e, E->out + E->base, E->cap - E->base);
        E->open = 1;
    }
}

/* bytes of the codeword so far (exact once the segment is terminated) */
static int t1e_end(t1e_t* E, int pass, int npasses) {
    if (or_t1_pass_terminated(E->style, pass, npasses)) {
        int len;
        if (E->raw) {
            len = rawe_flush(&E->r);
            E->ovf |= E->r.ovf;
        } else {
            len = mqe_flush(&E->e);
        }
        E->base += len;
        E->open = 0;
        return E->base;
    }
    return E->base + (E->raw ? E->r.pos : E->e.bp + 1);
}

static int t1_encode_core(const int32_t* coeff, size_t pitch, int cw, int ch, int orient, int style, uint8_t* out,
                          int cap, uint8_t* syms, int sym_cap, or_t1_info* info, int* pass_end) {
    t1st_t t;
    if (!t1_alloc(&t, cw, ch)) return -1;
    uint32_t* mag = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)cw * ch);
    uint32_t mx = 0;
    for (int y = 0; y < ch; ++y)
        for (int x = 0; x < cw; ++x) {
            int32_t v = coeff[(size_t)y * pitch + x];
            uint32_t m = v < 0 ? (uint32_t)(-(int64_t)v) : (uint32_t)v;
            mag[y * cw + x] = m;
            if (v < 0) FLAG(&t, x, y) |= F_NEG;
            if (m > mx) mx = m;
        }
    int nbps = 0;
    while (nbps < 32 && (mx >> nbps)) nbps++;
    const int total = nbps ? 3 * nbps - 2 : 0;
    t1e_t E;
    mqe_init(&E.e, out, cap);
    E.e.syms = syms;
    E.e.sym_cap = sym_cap;
    E.style = style;
    E.raw = 0;
    E.open = 0;
    E.out = out;
    E.cap = cap;
    E.base = 0;
    E.ovf = 0;
    int npasses = 0, len = 0;
    for (int p = nbps - 1; p >= 0; --p) {
        int first = (p == nbps - 1);
        if (!first) {
            /* significance propagation pass */
            t1e_begin(&E, npasses);
            for (int y0 = 0; y0 < ch; y0 += 4)
                for (int x = 0; x < cw; ++x)
                    for (int y = y0; y < y0 + 4 && y < ch; ++y) {
                        uint8_t f = FLAG(&t, x, y);
                        if (f & F_SIG) continue;
                        int h, v, d;
                        nbr_counts(&t, x, y, &h, &v, &d);
                        if (h + v + d == 0) continue;
                        int bit = (mag[y * cw + x] >> p) & 1;
                        t1e_bit(&E, zc_label(orient, h, v, d), bit);
                        FLAG(&t, x, y) |= F_VIS;
                        if (bit) {
                            int xb;
                            int cx = sc_label(&t, x, y, &xb);
                            t1e_sign(&E, cx, xb, (FLAG(&t, x, y) & F_NEG) ? 1 : 0);
                            FLAG(&t, x, y) |= F_SIG;
                        }
                    }
            len = t1e_end(&E, npasses, total);
            if (pass_end) pass_end[npasses] = len;
            npasses++;
            /* magnitude refinement pass */
            t1e_begin(&E, npasses);
            for (int y0 = 0; y0 < ch; y0 += 4)
                for (int x = 0; x < cw; ++x)
                    for (int y = y0; y < y0 + 4 && y < ch; ++y) {
                        uint8_t f = FLAG(&t, x, y);
                        if (!(f & F_SIG) || (f & F_VIS)) continue;
                        t1e_bit(&E, mr_label(&t, x, y), (mag[y * cw + x] >> p) & 1);
                        FLAG(&t, x, y) |= F_REF;
                    }
            len = t1e_end(&E, npasses, total);
            if (pass_end) pass_end[npasses] = len;
            npasses++;
        }
        /* cleanup pass (never raw-coded) */
        t1e_begin(&E, npasses);
        for (int y0 = 0; y0 < ch; y0 += 4)
            for (int x = 0; x < cw; ++x) {
                int start = y0;
                if (y0 + 3 < ch) {
                    int rl = 1;
                    for (int y = y0; y < y0 + 4 && rl; ++y) {
                        uint8_t f = FLAG(&t, x, y);
                        int h, v, d;
                        nbr_counts(&t, x, y, &h, &v, &d);
                        if ((f & (F_SIG | F_VIS)) || h + v + d) rl = 0;
                    }
                    if (rl) {
                        int idx = -1;
                        for (int k = 0; k < 4; ++k)
                            if ((mag[(y0 + k) * cw + x] >> p) & 1) { idx = k; break; }
                        t1e_bit(&E, CX_RL, idx >= 0);
                        if (idx < 0) continue;
                        t1e_bit(&E, CX_UNI, (idx >> 1) & 1);
                        t1e_bit(&E, CX_UNI, idx & 1);
                        int y = y0 + idx, xb;
                        int cx = sc_label(&t, x, y, &xb);
                        t1e_sign(&E, cx, xb, (FLAG(&t, x, y) & F_NEG) ? 1 : 0);
                        FLAG(&t, x, y) |= F_SIG;
                        start = y + 1;
                    }
                }
                for (int y = start; y < y0 + 4 && y < ch; ++y) {
                    uint8_t f = FLAG(&t, x, y);
                    if (f & (F_SIG | F_VIS)) continue;
                    int h, v, d;
                    nbr_counts(&t, x, y, &h, &v, &d);
                    int bit = (mag[y * cw + x] >> p) & 1;
                    t1e_bit(&E, zc_label(orient, h, v, d), bit);
                    if (bit) {
                        int xb;
                        int cx = sc_label(&t, x, y, &xb);
                        t1e_sign(&E, cx, xb, (FLAG(&t, x, y) & F_NEG) ? 1 : 0);
                        FLAG(&t, x, y) |= F_SIG;
                    }
                }
            }
        if (info && nbps - 1 - p < 32) info->plane_bytes[nbps - 1 - p] = E.base + E.e.bp + 1;
        len = t1e_end(&E, npasses, total);
        if (pass_end) pass_end[npasses] = len;
        npasses += 1;
        for (int y = 0; y < ch; ++y)
            for (int x = 0; x < cw; ++x) FLAG(&t, x, y) &= (uint8_t)~F_VIS;
    }
    len = nbps ? E.base : 0;
    free(mag);
    free(t.f);
    if (info) {
        info->numbps = nbps;
        info->npasses = npasses;
        info->length = len;
        info->nsyms = E.e.nsyms;
    }
    if (E.e.ovf || E.ovf || (syms && E.e.nsyms > sym_cap)) return -1;
    return len;
}

int or_t1_encode(const int32_t* coeff, size_t pitch, int cw, int ch, int orient, uint8_t* out,
                 int cap, uint8_t* syms, int sym_cap, or_t1_info* info) {
    return t1_encode_core(coeff, pitch, cw, ch, orient, 0, out, cap, syms, sym_cap, info, NULL);
}

int or_t1_encode_styled(const int32_t* coeff, size_t pitch, int cw, int ch, int orient, int style, uint8_t* out,
                        int cap, or_t1_info* info, int* pass_end) {
    return t1_encode_core(coeff, pitch, cw, ch, orient, style, out, cap, NULL, 0, info, pass_end);
}

/* Tier-1 decoder of one code-block: segments located by the pass ends, MQ or raw per pass. */
typedef struct {
    mqd_t d;
    rawd_t r;
    int style, raw, npasses;
    const uint8_t* data;
    int len;
    const int* pass_end;
} t1d_t;

static int t1d_bit(t1d_t* D, int cx) { return D->raw ? rawd_get(&D->r) : mqd_decode(&D->d, cx); }

static int t1d_sign(t1d_t* D, int cx, int xb) { return D->raw ? rawd_get(&D->r) : (mqd_decode(&D->d, cx) ^ xb); }

static void t1d_begin(t1d_t* D, int pass) {
    if (pass > 0 && (D->style & OR_STYLE_RESET)) mq_reset_states(D->d.st, D->d.mps);
    D->raw = or_t1_pass_raw(D->style, pass);
    if (pass == 0 || or_t1_pass_terminated(D->style, pass - 1, D->npasses)) {
        /* a new segment: from the end of the previous one to the end of its last pass */
        int b0 = pass == 0 ? 0 : (D->pass_end ? D->pass_end[pass - 1] : 0);
        int q = pass;
        while (!or_t1_pass_terminated(D->style, q, D->npasses)) q++;
        int b1 = D->pass_end ? D->pass_end[q] : D->len;
        if (b0 < 0) b0 = 0;
        if (b1 > D->len) b1 = D->len;
        if (b1 < b0) b1 = b0;
        if (D->raw) rawd_start(&D->r, D->data + b0, b1 - b0);
        else mqd_start(&D->d, D->data + b0, b1 - b0);
    }
}

static int t1_decode_core(const uint8_t* data, int len, const int* pass_end, int numbps, int npasses, int orient,
                          int style, int32_t* coeff, size_t pitch, int cw, int ch) {
    for (int y = 0; y < ch; ++y)
        for (int x = 0; x < cw; ++x) coeff[(size_t)y * pitch + x] = 0;
    if (numbps == 0 || npasses == 0) return 0;
    t1st_t t;
    if (!t1_alloc(&t, cw, ch)) return -1;
    uint32_t* mag = (uint32_t*)calloc((size_t)cw * ch, sizeof(uint32_t));
    t1d_t D;
    D.style = style;
    D.npasses = npasses;
    D.data = data;
    D.len = len;
    D.pass_end = pass_end;
    D.raw = 0;
    mq_reset_states(D.d.st, D.d.mps);
    int pass = 0;
    for (int p = numbps - 1; p >= 0 && pass < npasses; --p) {
        int first = (p == numbps - 1);
        if (!first) {
            t1d_begin(&D, pass);
            for (int y0 = 0; y0 < ch; y0 += 4)
                for (int x = 0; x < cw; ++x)
                    for (int y = y0; y < y0 + 4 && y < ch; ++y) {
                        uint8_t f = FLAG(&t, x, y);
                        if (f & F_SIG) continue;
                        int h, v, dd;
                        nbr_counts(&t, x, y, &h, &v, &dd);
                        if (h + v + dd == 0) continue;
                        int bit = t1d_bit(&D, zc_label(orient, h, v, dd));
                        FLAG(&t, x, y) |= F_VIS;
                        if (bit) {
                            int xb;
                            int cx = sc_label(&t, x, y, &xb);
                            int s = t1d_sign(&D, cx, xb);
                            FLAG(&t, x, y) |= (uint8_t)(F_SIG | (s ? F_NEG : 0));
                            mag[y * cw + x] |= 1u << p;
                        }
                    }
            if (++pass >= npasses) break;
            t1d_begin(&D, pass);
            for (int y0 = 0; y0 < ch; y0 += 4)
                for (int x = 0; x < cw; ++x)
                    for (int y = y0; y < y0 + 4 && y < ch; ++y) {
                        uint8_t f = FLAG(&t, x, y);
                        if (!(f & F_SIG) || (f & F_VIS)) continue;
                        int bit = t1d_bit(&D, mr_label(&t, x, y));
                        if (bit) mag[y * cw + x] |= 1u << p;
                        FLAG(&t, x, y) |= F_REF;
                    }
            if (++pass >= npasses) break;
        }
        t1d_begin(&D, pass);
        for (int y0 = 0; y0 < ch; y0 += 4)
            for (int x = 0; x < cw; ++x) {
                int start = y0;
                if (y0 + 3 < ch) {
                    int rl = 1;
                    for (int y = y0; y < y0 + 4 && rl; ++y) {
                        uint8_t f = FLAG(&t, x, y);
                        int h, v, dd;
                        nbr_counts(&t, x, y, &h, &v, &dd);
                        if ((f & (F_SIG | F_VIS)) || h + v + dd) rl = 0;
                    }
                    if (rl) {
                        if (!t1d_bit(&D, CX_RL)) continue;
                        int idx = t1d_bit(&D, CX_UNI) << 1;
                        idx |= t1d_bit(&D, CX_UNI);
                        int y = y0 + idx, xb;
                        int cx = sc_label(&t, x, y, &xb);
                        int s = t1d_sign(&D, cx, xb);
                        FLAG(&t, x, y) |= (uint8_t)(F_SIG | (s ? F_NEG : 0));
                        mag[y * cw + x] |= 1u << p;
                        start = y + 1;
                    }
                }
                for (int y = start; y < y0 + 4 && y < ch; ++y) {
                    uint8_t f = FLAG(&t, x, y);
                    if (f & (F_SIG | F_VIS)) continue;
                    int h, v, dd;
                    nbr_counts(&t, x, y, &h, &v, &dd);
                    int bit = t1d_bit(&D, zc_label(orient, h, v, dd));
                    if (bit) {
                        int xb;
                        int cx = sc_label(&t, x, y, &xb);
                        int s = t1d_sign(&D, cx, xb);
                        FLAG(&t, x, y) |= (uint8_t)(F_SIG | (s ? F_NEG : 0));
                        mag[y * cw + x] |= 1u << p;
                    }
                }
            }
        ++pass;
        for (int y = 0; y < ch; ++y)
            for (int x = 0; x < cw; ++x) FLAG(&t, x, y) &= (uint8_t)~F_VIS;
    }
    /* a block cut at the end of a bit-plane above the last one: significant magnitudes are
     * reconstructed at the middle of the interval their undecoded low bits leave */
    uint32_t half = 0;
    if (npasses < 3 * numbps - 2 && (npasses - 1) % 3 == 0) {
        const int plast = numbps - 1 - (npasses - 1) / 3;
        half = plast > 0 ? 1u << (plast - 1) : 0u;
    }
    for (int y = 0; y < ch; ++y)
        for (int x = 0; x < cw; ++x) {
            int32_t m = (int32_t)mag[y * cw + x];
            if (FLAG(&t, x, y) & F_SIG) m += (int32_t)half;
            coeff[(size_t)y * pitch + x] = (FLAG(&t, x, y) & F_NEG) ? -m : m;
        }
    free(mag);
    free(t.f);
    return 0;
}

int or_t1_decode(const uint8_t* data, int len, int numbps, int npasses, int orient,
                 int32_t* coeff, size_t pitch, int cw, int ch) {
    return t1_decode_core(data, len, NULL, numbps, npasses, orient, 0, coeff, pitch, cw, ch);
}

int or_t1_decode_styled(const uint8_t* data, int len, const int* pass_end, int numbps, int npasses, int orient,
                        int style, int32_t* coeff, size_t pitch, int cw, int ch) {
    return t1_decode_core(data, len, pass_end, numbps, npasses, orient, style, coeff, pitch, cw, ch);
}

/* ============================================================================================
 * Tier-2: minimal T.800 codestream (Annex A markers, Annex B packets with tag trees)
 * ========================================================================================== */

typedef struct {
    uint8_t* buf;
    long cap, pos;
    int ovf;
} bytes_t;

static void bput(bytes_t* b, uint8_t v) {
    if (b->pos < b->cap) b->buf[b->pos] = v; else b->ovf = 1;
    b->pos++;
}
static void bput16(bytes_t* b, uint32_t v) { bput(b, (uint8_t)(v >> 8)); bput(b, (uint8_t)v); }
static void bput32(bytes_t* b, uint32_t v) { bput16(b, v >> 16); bput16(b, v & 0xFFFF); }

/* packet-header bit writer with the B.10.1 bit stuffing after 0xFF */
typedef struct {
    bytes_t* out;
    uint32_t acc;
    int nb, room;
} bitw_t;

static void bw_init(bitw_t* w, bytes_t* out) { w->out = out; w->acc = 0; w->nb = 0; w->room = 8; }
static void bw_put(bitw_t* w, int bit) {
    w->acc = (w->acc << 1) | (uint32_t)(bit & 1);
    w->nb++;
    if (w->nb == w->room) {
        bput(w->out, (uint8_t)w->acc);
        w->room = (w->acc == 0xFF) ? 7 : 8;
        w->acc = 0;
        w->nb = 0;
    }
}
static void bw_putn(bitw_t* w, uint32_t v, int n) {
    for (int i = n - 1; i >= 0; --i) bw_put(w, (v >> i) & 1);
}
static void bw_flush(bitw_t* w) {
    int last_ff = 0;
    if (w->nb) {
        uint32_t v = w->acc << (w->room - w->nb);
        bput(w->out, (uint8_t)v);
        last_ff = (v == 0xFF);
    } else {
        last_ff = (w->room == 7);
    }
    if (last_ff) bput(w->out, 0x00);
    w->acc = 0; w->nb = 0; w->room = 8;
}

typedef struct {
    int nw, nh, nlev;
    int lw[20], lh[20], off[20];
    int* val;
    int* low;
    uint8_t* known;
} tagtree_t;

static void tt_init(tagtree_t* t, int nw, int nh, const int* leaves) {
    t->nlev = 0;
    int w = nw, h = nh, total = 0;
    for (;;) {
        t->lw[t->nlev] = w;
        t->lh[t->nlev] = h;
        t->off[t->nlev] = total;
        total += w * h;
        t->nlev++;
        if (w == 1 && h == 1) break;
        w = (w + 1) / 2;
        h = (h + 1) / 2;
    }
    t->val = (int*)malloc(sizeof(int) * total);
    t->low = (int*)calloc(total, sizeof(int));
    t->known = (uint8_t*)calloc(total, 1);
    for (int i = 0; i < nw * nh; ++i) t->val[i] = leaves[i];
    for (int l = 1; l < t->nlev; ++l)
        for (int y = 0; y < t->lh[l]; ++y)
            for (int x = 0; x < t->lw[l]; ++x) {
                int m = 0x7FFFFFFF;
                for (int dy = 0; dy < 2; ++dy)
                    for (int dx = 0; dx < 2; ++dx) {
                        int cx = 2 * x + dx, cy = 2 * y + dy;
                        if (cx < t->lw[l - 1] && cy < t->lh[l - 1]) {
                            int v = t->val[t->off[l - 1] + cy * t->lw[l - 1] + cx];
                            if (v < m) m = v;
                        }
                    }
                t->val[t->off[l] + y * t->lw[l] + x] = m;
            }
}
static void tt_free(tagtree_t* t) { free(t->val); free(t->low); free(t->known); }

/* B.10.2: code whether leaf (x,y) has value < threshold, walking root to leaf. */
static void tt_encode(tagtree_t* t, bitw_t* w, int x, int y, int threshold) {
    int path[20];
    for (int l = 0; l < t->nlev; ++l) {
        path[l] = t->off[l] + y * t->lw[l] + x;
        x >>= 1;
        y >>= 1;
    }
    int low = 0;
    for (int l = t->nlev - 1; l >= 0; --l) {
        int n = path[l];
        if (low > t->low[n]) t->low[n] = low; else low = t->low[n];
        while (low < threshold) {
            if (low >= t->val[n]) {
                if (!t->known[n]) { bw_put(w, 1); t->known[n] = 1; }
                break;
            }
            bw_put(w, 0);
            low++;
        }
        t->low[n] = low;
    }
}

static void put_npasses(bitw_t* w, int n) {
    if (n == 1) bw_put(w, 0);
    else if (n == 2) bw_putn(w, 2, 2);
    else if (n <= 5) { bw_putn(w, 3, 2); bw_putn(w, (uint32_t)(n - 3), 2); }
    else if (n <= 36) { bw_putn(w, 0xF, 4); bw_putn(w, (uint32_t)(n - 6), 5); }
    else { bw_putn(w, 0x1FF, 9); bw_putn(w, (uint32_t)(n - 37), 7); }
}

static int floorlog2(long v) { int l = -1; while (v) { v >>= 1; l++; } return l; }

typedef struct {
    int x0, y0, cw, ch;
    or_t1_info info;
    int pass_end[96];
    uint8_t* data;
} cb_t;

typedef struct {
    int orient, level;
    size_t x0, y0, sw, sh;
    int ncbx, ncby;
    cb_t* cbs;
} band_t;

long or_encode_image(const uint8_t* img, size_t w, size_t h, int ncomp, const or_enc_params* p,
                     uint8_t* out, long cap) {
    int L = p->levels, nb = 3 * L + 1;
    size_t N = w * h;
    int mct = (ncomp >= 3) ? (p->lossless ? OR_MCT_RCT : OR_MCT_ICT) : OR_MCT_NONE;
    float steps[3 * 32 + 1];
    for (int b = 0; b < nb; ++b) {
        size_t a, c, d, e;
        int o, l;
        or_subband_rect(w, h, L, b, &a, &c, &d, &e, &o, &l);
        steps[b] = p->steps ? p->steps[b] : 8.0f * ldexpf(1.0f, -l);
    }
    int32_t* coef = (int32_t*)malloc(sizeof(int32_t) * N * ncomp);
    if (p->lossless) {
        int32_t* planes = (int32_t*)malloc(sizeof(int32_t) * N * ncomp);
        or_planar_fwd_i32(img, w, h, w * ncomp, ncomp, mct, planes, w, N);
        for (int c = 0; c < ncomp; ++c)
            or_dwt53_fwd(planes + c * N, w, coef + c * N, w, w, h, L, p->order);
        free(planes);
    } else {
        float* planes = (float*)malloc(sizeof(float) * N * ncomp);
        float* tr = (float*)malloc(sizeof(float) * N);
        or_planar_fwd_f32(img, w, h, w * ncomp, ncomp, mct, planes, w, N);
        for (int c = 0; c < ncomp; ++c) {
            or_dwt97_fwd_f32(planes + c * N, w, tr, w, w, h, L, OR_ORDER_T800);
            or_quantize_f32(tr, w, coef + c * N, w, w, h, L, steps);
        }
        free(planes);
        free(tr);
    }
    /* tier-1 on every code-block */
    band_t* bands = (band_t*)calloc((size_t)nb * ncomp, sizeof(band_t));
    int maxbps[3 * 32 + 1];
    memset(maxbps, 0, sizeof(maxbps));
    for (int c = 0; c < ncomp; ++c)
        for (int b = 0; b < nb; ++b) {
            band_t* bd = &bands[c * nb + b];
            or_subband_rect(w, h, L, b, &bd->x0, &bd->y0, &bd->sw, &bd->sh, &bd->orient, &bd->level);
            bd->ncbx = bd->sw ? (int)((bd->sw + p->cbw - 1) / p->cbw) : 0;
            bd->ncby = bd->sh ? (int)((bd->sh + p->cbh - 1) / p->cbh) : 0;
            bd->cbs = (cb_t*)calloc((size_t)bd->ncbx * bd->ncby + 1, sizeof(cb_t));
            for (int j = 0; j < bd->ncby; ++j)
                for (int i = 0; i < bd->ncbx; ++i) {
                    cb_t* cb = &bd->cbs[j * bd->ncbx + i];
                    cb->x0 = i * p->cbw;
                    cb->y0 = j * p->cbh;
                    cb->cw = (int)((bd->sw - cb->x0) < (size_t)p->cbw ? bd->sw - cb->x0 : (size_t)p->cbw);
                    cb->ch = (int)((bd->sh - cb->y0) < (size_t)p->cbh ? bd->sh - cb->y0 : (size_t)p->cbh);
                    int ccap = cb->cw * cb->ch * 5 + 64 + 4 * 96;
                    cb->data = (uint8_t*)malloc((size_t)ccap);
                    const int32_t* src = coef + c * N + (bd->y0 + cb->y0) * w + bd->x0 + cb->x0;
                    t1_encode_core(src, w, cb->cw, cb->ch, bd->orient, p->style, cb->data, ccap, NULL, 0, &cb->info,
                                   cb->pass_end);
                    if (cb->info.numbps > maxbps[b]) maxbps[b] = cb->info.numbps;
                }
        }
    if (p->tier1_only) {
        long total = 0;
        for (int i = 0; i < nb * ncomp; ++i) {
            band_t* bd = &bands[i];
            for (int k = 0; k < bd->ncbx * bd->ncby; ++k) {
                total += bd->cbs[k].info.length;
                free(bd->cbs[k].data);
            }
            free(bd->cbs);
        }
        free(bands);
        free(coef);
        return total;
    }
    /* quantisation exponents (eps_b) and guard bits */
    int eps[3 * 32 + 1], mant[3 * 32 + 1], G = 2;
    for (int b = 0; b < nb; ++b) {
        size_t a, c, d, e;
        int o, l;
        or_subband_rect(w, h, L, b, &a, &c, &d, &e, &o, &l);
        int gain = (o == OR_LL) ? 0 : (o == OR_HH ? 2 : 1);
        int Rb = 8 + gain;
        if (p->lossless) {
            eps[b] = Rb + (mct ? 1 : 0);
            mant[b] = 0;
        } else {
            int ex;
            float fr = frexpf(steps[b], &ex); /* steps = fr*2^ex, fr in [0.5,1) */
            int e2 = ex - 1;                  /* step = 2^e2 * (1 + mu/2048) */
            eps[b] = Rb - e2;
            mant[b] = (int)lrintf((fr * 2.0f - 1.0f) * 2048.0f);
            if (mant[b] == 2048) { /* the 11-bit mantissa rounded up: next power of two */
                mant[b] = 0;
                eps[b] -= 1;
            }
        }
        int need = maxbps[b] - eps[b] + 1;
        if (need > G) G = need;
    }
    if (G > 7) G = 7;
    bytes_t o = {out, cap, 0, 0};
    bput16(&o, 0xFF4F);                      /* SOC */
    bput16(&o, 0xFF51);                      /* SIZ */
    bput16(&o, (uint32_t)(38 + 3 * ncomp));
    bput16(&o, 0);
    bput32(&o, (uint32_t)w); bput32(&o, (uint32_t)h);
    bput32(&o, 0); bput32(&o, 0);
    bput32(&o, (uint32_t)w); bput32(&o, (uint32_t)h);
    bput32(&o, 0); bput32(&o, 0);
    bput16(&o, (uint32_t)ncomp);
    for (int c = 0; c < ncomp; ++c) { bput(&o, 7); bput(&o, 1); bput(&o, 1); }
    bput16(&o, 0xFF52);                      /* COD */
    bput16(&o, 12);
    bput(&o, 0);
    bput(&o, 0);                             /* LRCP */
    bput16(&o, 1);                           /* one layer */
    bput(&o, mct ? 1 : 0);
    bput(&o, (uint8_t)L);
    bput(&o, (uint8_t)(floorlog2(p->cbw) - 2));
    bput(&o, (uint8_t)(floorlog2(p->cbh) - 2));
    bput(&o, (uint8_t)p->style);            /* code-block style */
    bput(&o, p->lossless ? 1 : 0);
    bput16(&o, 0xFF5C);                      /* QCD */
    if (p->lossless) {
        bput16(&o, (uint32_t)(3 + nb));
        bput(&o, (uint8_t)(G << 5));
        for (int b = 0; b < nb; ++b) bput(&o, (uint8_t)(eps[b] << 3));
    } else {
        bput16(&o, (uint32_t)(3 + 2 * nb));
        bput(&o, (uint8_t)((G << 5) | 2));
        for (int b = 0; b < nb; ++b) bput16(&o, (uint32_t)((eps[b] << 11) | mant[b]));
    }
    long sot = o.pos;
    bput16(&o, 0xFF90);                      /* SOT */
    bput16(&o, 10);
    bput16(&o, 0);
    bput32(&o, 0);                           /* Psot patched below */
    bput(&o, 0);
    bput(&o, 1);
    bput16(&o, 0xFF93);                      /* SOD */
    /* packets: layer 0, resolutions 0..L, components, one precinct */
    for (int r = 0; r <= L; ++r)
        for (int c = 0; c < ncomp; ++c) {
            int bfirst = (r == 0) ? 0 : 1 + 3 * (r - 1);
            int bcount = (r == 0) ? 1 : 3;
            int any = 0;
            for (int k = 0; k < bcount; ++k) {
                band_t* bd = &bands[c * nb + bfirst + k];
                for (int i = 0; i < bd->ncbx * bd->ncby; ++i) any |= bd->cbs[i].info.npasses > 0;
            }
            bitw_t bw;
            bw_init(&bw, &o);
            if (!any) {
                bw_put(&bw, 0);
                bw_flush(&bw);
                continue;
            }
            bw_put(&bw, 1);
            for (int k = 0; k < bcount; ++k) {
                band_t* bd = &bands[c * nb + bfirst + k];
                int n = bd->ncbx * bd->ncby;
                if (!n) continue;
                int Mb = G + eps[bfirst + k] - 1;
                int* incl = (int*)malloc(sizeof(int) * n);
                int* zbp = (int*)malloc(sizeof(int) * n);
                for (int i = 0; i < n; ++i) {
                    incl[i] = bd->cbs[i].info.npasses > 0 ? 0 : 1;
                    zbp[i] = Mb - bd->cbs[i].info.numbps;
                }
                tagtree_t ti, tz;
                tt_init(&ti, bd->ncbx, bd->ncby, incl);
                tt_init(&tz, bd->ncbx, bd->ncby, zbp);
                for (int j = 0; j < bd->ncby; ++j)
                    for (int i = 0; i < bd->ncbx; ++i) {
                        cb_t* cb = &bd->cbs[j * bd->ncbx + i];
                        tt_encode(&ti, &bw, i, j, 1);
                        if (cb->info.npasses == 0) continue;
                        tt_encode(&tz, &bw, i, j, 0x7FFFFFF);
                        put_npasses(&bw, cb->info.npasses);
                        /* one codeword segment per terminated pass (B.10.7.2): each length in
                         * Lblock + floor(log2(passes of the segment)) bits, Lblock raised once
                         * so that every length fits */
                        int lblock = 3, nseg = 0, seg_np[96], seg_len[96], prev = 0, np0 = 0;
                        for (int q = 0; q < cb->info.npasses; ++q)
                            if (or_t1_pass_terminated(p->style, q, cb->info.npasses)) {
                                seg_np[nseg] = q + 1 - np0;
                                seg_len[nseg] = cb->pass_end[q] - prev;
                                prev = cb->pass_end[q];
                                np0 = q + 1;
                                nseg++;
                            }
                        int inc = 0;
                        for (int q = 0; q < nseg; ++q) {
                            int bits = floorlog2(seg_len[q]) + 1;
                            int avail = lblock + floorlog2(seg_np[q]);
                            if (bits - avail > inc) inc = bits - avail;
                        }
                        for (int q = 0; q < inc; ++q) bw_put(&bw, 1);
                        bw_put(&bw, 0);
                        lblock += inc;
                        for (int q = 0; q < nseg; ++q)
                            bw_putn(&bw, (uint32_t)seg_len[q], lblock + floorlog2(seg_np[q]));
                    }
                tt_free(&ti);
                tt_free(&tz);
                free(incl);
                free(zbp);
            }
            bw_flush(&bw);
            for (int k = 0; k < bcount; ++k) {
                band_t* bd = &bands[c * nb + bfirst + k];
                for (int i = 0; i < bd->ncbx * bd->ncby; ++i)
                    for (int q = 0; q < bd->cbs[i].info.length; ++q) bput(&o, bd->cbs[i].data[q]);
            }
        }
    long psot = o.pos - sot;
    if (sot + 10 <= o.cap) {
        out[sot + 6] = (uint8_t)(psot >> 24);
        out[sot + 7] = (uint8_t)(psot >> 16);
        out[sot + 8] = (uint8_t)(psot >> 8);
        out[sot + 9] = (uint8_t)psot;
    }
    bput16(&o, 0xFFD9);                      /* EOC */
    for (int i = 0; i < nb * ncomp; ++i) {
        band_t* bd = &bands[i];
        for (int k = 0; k < bd->ncbx * bd->ncby; ++k) free(bd->cbs[k].data);
        free(bd->cbs);
    }
    free(bands);
    free(coef);
    return o.ovf ? -1 : o.pos;
}

/* ============================================================================================
 * Differentiable 9/7 step in FP64
 * ========================================================================================== */

static uint32_t mulhilo(uint32_t a, uint32_t b, uint32_t* hi) {
    uint64_t p = (uint64_t)a * b;
    *hi = (uint32_t)(p >> 32);
    return (uint32_t)p;
}

void or_philox4x32(uint32_t k0, uint32_t k1, const uint32_t ctr[4], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, hi1;
        uint32_t lo0 = mulhilo(0xD2511F53u, c0, &hi0);
        uint32_t lo1 = mulhilo(0xCD9E8D57u, c2, &hi1);
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

double or_philox_uniform(uint64_t seed, uint64_t i) {
    uint32_t ctr[4] = {(uint32_t)i, (uint32_t)(i >> 32), 0, 0}, o[4];
    or_philox4x32((uint32_t)seed, (uint32_t)(seed >> 32), ctr, o);
    /* 24-bit uniform in [0,1), shifted to [-0.5, 0.5): exactly representable in float too */
    return (double)(o[0] >> 8) * (1.0 / 16777216.0) - 0.5;
}

double or_rd_noise(uint64_t seed, size_t w, size_t x, size_t y) {
    /* one Philox block per 4 consecutive samples of a plane row: counter y*ceil(w/4) + x/4,
     * output word x%4 */
    uint64_t c = (uint64_t)y * ((w + 3) / 4) + x / 4;
    uint32_t ctr[4] = {(uint32_t)c, (uint32_t)(c >> 32), 0, 0}, o[4];
    or_philox4x32((uint32_t)seed, (uint32_t)(seed >> 32), ctr, o);
    return (double)(o[x & 3] >> 8) * (1.0 / 16777216.0) - 0.5;
}

double or_rd_loss_f64(const double* x, size_t w, size_t h, int levels, const double* log_steps,
                      double lam, uint64_t seed, double* grad_x, double* grad_ls) {
    size_t N = w * h;
    int nb = 3 * levels + 1;
    double* y = (double*)malloc(sizeof(double) * N);
    double* yh = (double*)malloc(sizeof(double) * N);
    double* xh = (double*)malloc(sizeof(double) * N);
    double* gy = (double*)malloc(sizeof(double) * N);
    or_dwt97_fwd_f64(x, w, y, w, w, h, levels, OR_ORDER_T800);
    double rate = 0.0;
    const double inv_ln2 = 1.0 / log(2.0);
    /* relaxed quantiser: t = y/step + u, y_hat = t*step, rate = log2(1+|t|) */
    for (int b = 0; b < nb; ++b) {
        size_t x0, y0, sw, sh;
        int o, l;
        or_subband_rect(w, h, levels, b, &x0, &y0, &sw, &sh, &o, &l);
        double st = exp(log_steps[b]);
        for (size_t yy = y0; yy < y0 + sh; ++yy)
            for (size_t xx = x0; xx < x0 + sw; ++xx) {
                size_t i = yy * w + xx;
                double u = or_rd_noise(seed, w, xx, yy);
                double t = y[i] / st + u;
                yh[i] = t * st;
                rate += log(1.0 + fabs(t)) * inv_ln2;
            }
    }
    or_dwt97_inv_f64(yh, w, xh, w, w, h, levels, OR_ORDER_T800);
    double mse = 0.0;
    for (size_t i = 0; i < N; ++i) { double d = xh[i] - x[i]; mse += d * d; }
    mse /= (double)N;
    double loss = mse + lam * rate;
    if (grad_x || grad_ls) {
        double* gxh = (double*)malloc(sizeof(double) * N);
        double* gyh = (double*)malloc(sizeof(double) * N);
        for (size_t i = 0; i < N; ++i) gxh[i] = 2.0 * (xh[i] - x[i]) / (double)N;
        or_dwt97_inv_adj_f64(gxh, w, gyh, w, w, h, levels);
        for (int b = 0; b < nb; ++b) {
            size_t x0, y0, sw, sh;
            int o, l;
            or_subband_rect(w, h, levels, b, &x0, &y0, &sw, &sh, &o, &l);
            double st = exp(log_steps[b]);
            double gls = 0.0;
            for (size_t yy = y0; yy < y0 + sh; ++yy)
                for (size_t xx = x0; xx < x0 + sw; ++xx) {
                    size_t i = yy * w + xx;
                    double u = or_rd_noise(seed, w, xx, yy);
                    double t = y[i] / st + u;
                    double sg = t > 0 ? 1.0 : (t < 0 ? -1.0 : 0.0);
                    double dr_dt = lam * inv_ln2 * sg / (1.0 + fabs(t));
                    /* y_hat = y + u*st: d/dy = 1, d/dlog(st) = u*st; t = y/st + u */
                    gy[i] = gyh[i] + dr_dt / st;
                    gls += gyh[i] * u * st + dr_dt * (-y[i] / st);
                }
            if (grad_ls) grad_ls[b] = gls;
        }
        if (grad_x) {
            double* gx = grad_x;
            or_dwt97_fwd_adj_f64(gy, w, gx, w, w, h, levels);
            for (size_t i = 0; i < N; ++i) gx[i] += -2.0 * (xh[i] - x[i]) / (double)N;
        }
        free(gxh);
        free(gyh);
    }
    free(y);
    free(yh);
    free(xh);
    free(gy);
    return loss;
}

void or_t1_plane_distortion(const int32_t* coeff, size_t pitch, int cw, int ch, int numbps, double dist[33]) {
    for (int k = 0; k < 33; ++k) dist[k] = 0.0;
    for (int y = 0; y < ch; ++y)
        for (int x = 0; x < cw; ++x) {
            const int32_t v = coeff[(size_t)y * pitch + x];
            const uint64_t m = v < 0 ? (uint64_t)(-(int64_t)v) : (uint64_t)v;
            dist[32] += (double)m * (double)m;
            for (int k = 0; k < numbps && k < 32; ++k) {
                const int p = numbps - 1 - k;
                const uint64_t hi = (m >> p) << p;
                const uint64_t rec = hi ? hi + ((1ull << p) >> 1) : 0;
                const double e = (double)m - (double)rec;
                dist[k] += e * e;
            }
        }
}
