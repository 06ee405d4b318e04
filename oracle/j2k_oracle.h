/*
 * CPU oracle for the JPEG 2000 encode/decode hot path — TEST INFRASTRUCTURE ONLY.
 *
 * This library is the checker for the CUDA product path (roger_b200/csrc).  Only the test
 * suite, the smoke check and the CPU-baseline leg of the benchmark may load it.  The product
 * never links or calls it.
 *
 * What it restates (reference paths are relative to the knopkem/roger source tree):
 *   - planar split            src/CL/oclplanar.cl:23-40 (channel order R,G,B,A -> planes 0..3),
 *                             plus the ITU-T T.800 Annex G level shift, RCT (G.2) and ICT (G.3),
 *                             which the reference never implemented.
 *   - 5/3 forward lifting     src/CL/ocldwt53.cl:223,228 (rows) and :259,273 (columns):
 *                             predict  x_o -= (x_e + x_e') >> 1, update x_e += (x_o + x_o' + 2) >> 2,
 *                             whole-sample symmetric extension (the MIRRORED_REPEAT sampler at
 *                             ocldwt53.cl:86), Mallat output (ocldwt53.cl:110-160,174), level
 *                             recursion on ceil(n/2) (src/OCLDWTForward.cpp:124-137).
 *                             Two orders: J2K_ORDER_REF = rows then columns (the reference),
 *                             J2K_ORDER_T800 = columns then rows (T.800 F.4.2, decodable by any
 *                             conformant decoder).
 *   - 9/7 forward lifting     constants and low*1/K, high*K convention src/CL/ocldwt97.cl:69-78,
 *                             arithmetic order of the horizontal register pipeline :248-310
 *                             (P1, U1, P2, U2, then scaling), applied identically to columns and
 *                             scaled once (the racy double-scaled vertical pass :319-403 and
 *                             :151-157 is not reproduced).  FP32 without contraction, plus FP64.
 *   - inverse DWTs            the reference's ocldwt53rev.cl/ocldwt97rev.cl are forward
 *                             transforms; the inverses here are the exact lifting inverses
 *                             (T.800 F.3).
 *   - dead-zone quantiser     T.800 E.1 (the reference's ceil "quantiser" at ocldwt97.cl:441,447
 *                             is not a dead-zone quantiser); midpoint reconstruction.
 *   - EBCOT tier-1            scan order / state variables / pass definitions of
 *                             src/CL/oclbpc.cl:19-111 and the context tables :205-275, completed
 *                             from T.800 Annex D (context labels, run-length mode, sign coding)
 *                             and Annex C (MQ coder), since the reference kernel codes nothing.
 *   - tier-2                  a minimal T.800 Annex A/B codestream writer (one tile, one layer,
 *                             LRCP, one precinct per resolution) so that an independent decoder
 *                             (OpenJPEG via Pillow) can pin the whole chain.
 *   - relaxed quantiser and   the differentiable 9/7 step (forward noise quantiser, adjoint
 *     adjoint DWT             lifting) in FP64, used for finite-difference and transpose checks.
 */
#ifndef J2K_ORACLE_H
#define J2K_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OR_ORDER_T800 = 0, OR_ORDER_REF = 1 };
enum { OR_MCT_NONE = 0, OR_MCT_RCT = 1, OR_MCT_ICT = 2 };
enum { OR_LL = 0, OR_HL = 1, OR_LH = 2, OR_HH = 3 };

/* ---- planar split + level shift + colour transform ---------------------------------------- */
/* src: interleaved uint8, ncomp samples per pixel, row pitch src_pitch bytes.
 * dst: ncomp planes, plane c at dst + c*plane_stride, row pitch dst_pitch elements. */
void or_planar_fwd_i32(const uint8_t* src, size_t w, size_t h, size_t src_pitch, int ncomp,
                       int mct, int32_t* dst, size_t dst_pitch, size_t plane_stride);
void or_planar_fwd_f32(const uint8_t* src, size_t w, size_t h, size_t src_pitch, int ncomp,
                       int mct, float* dst, size_t dst_pitch, size_t plane_stride);
void or_planar_inv_i32(const int32_t* src, size_t src_pitch, size_t plane_stride, size_t w,
                       size_t h, int ncomp, int mct, uint8_t* dst, size_t dst_pitch);
void or_planar_inv_f32(const float* src, size_t src_pitch, size_t plane_stride, size_t w,
                       size_t h, int ncomp, int mct, uint8_t* dst, size_t dst_pitch);

/* ---- DWT (Mallat layout, out-of-place) ---------------------------------------------------- */
void or_dwt53_fwd(const int32_t* in, size_t in_pitch, int32_t* out, size_t out_pitch, size_t w,
                  size_t h, int levels, int order);
void or_dwt53_inv(const int32_t* in, size_t in_pitch, int32_t* out, size_t out_pitch, size_t w,
                  size_t h, int levels, int order);
void or_dwt97_fwd_f32(const float* in, size_t in_pitch, float* out, size_t out_pitch, size_t w,
                      size_t h, int levels, int order);
void or_dwt97_inv_f32(const float* in, size_t in_pitch, float* out, size_t out_pitch, size_t w,
                      size_t h, int levels, int order);
void or_dwt97_fwd_f64(const double* in, size_t in_pitch, double* out, size_t out_pitch, size_t w,
                      size_t h, int levels, int order);
void or_dwt97_inv_f64(const double* in, size_t in_pitch, double* out, size_t out_pitch, size_t w,
                      size_t h, int levels, int order);
/* Transposes (adjoints) of the FP64 9/7 transforms, T800 order. */
void or_dwt97_fwd_adj_f64(const double* g_out, size_t gpitch, double* g_in, size_t ipitch,
                          size_t w, size_t h, int levels);
void or_dwt97_inv_adj_f64(const double* g_img, size_t gpitch, double* g_coef, size_t cpitch,
                          size_t w, size_t h, int levels);

/* Subband geometry of a Mallat plane.  Subband index b: 0 = LL_L, then for k = L..1 the triple
 * HL_k, LH_k, HH_k (the T.800 QCD order).  Returns the number of subbands (3L+1). */
int or_subband_rect(size_t w, size_t h, int levels, int b, size_t* x0, size_t* y0, size_t* sw,
                    size_t* sh, int* orient, int* level);

/* ---- quantiser ----------------------------------------------------------------------------- */
void or_quantize_f32(const float* in, size_t in_pitch, int32_t* q, size_t q_pitch, size_t w,
                     size_t h, int levels, const float* steps);
void or_dequantize_f32(const int32_t* q, size_t q_pitch, float* out, size_t out_pitch, size_t w,
                       size_t h, int levels, const float* steps);

/* ---- EBCOT tier-1 -------------------------------------------------------------------------- */
typedef struct {
    int numbps;   /* magnitude bit-planes coded (0 = all-zero block) */
    int npasses;  /* 3*numbps-2, or 0 */
    int length;   /* codeword bytes */
    int nsyms;    /* number of MQ symbols coded */
    /* bytes the coder had produced (bytes 0..bp, the last one still open to a carry) when the
     * cleanup pass of bit-plane k (k = 0 for the most significant) ended */
    int plane_bytes[32];
} or_t1_info;
/* Bytes kept when a code-block is truncated after the cleanup pass of bit-plane k (npasses =
 * 3k+1): the bytes produced so far plus OR_TRUNC_EXTRA more of the finished codeword (what the MQ
 * decoder reads ahead of the encoder), never more than the whole codeword. */
#define OR_TRUNC_EXTRA 4
/* Squared reconstruction error of one code-block when it is decoded down to bit-plane k only
 * (dist[k], k = 0 .. numbps-1, k = 0 the most significant; magnitudes below the last decoded
 * plane reconstructed at the middle of their interval), and with nothing decoded (dist[32]). */
void or_t1_plane_distortion(const int32_t* coeff, size_t pitch, int cw, int ch, int numbps, double dist[33]);
/* Encodes one code-block.  coeff: cw x ch int32 values (two's complement) at row pitch `pitch`.
 * out: capacity `cap` bytes.  syms (optional, capacity sym_cap): one byte per MQ symbol,
 * context label in bits 0-4 and the decision in bit 7, in coding order.  Returns the codeword
 * length or -1 on overflow. */
int or_t1_encode(const int32_t* coeff, size_t pitch, int cw, int ch, int orient, uint8_t* out,
                 int cap, uint8_t* syms, int sym_cap, or_t1_info* info);
/* Decodes one code-block back to int32 values (all passes present). 0 = ok. */
int or_t1_decode(const uint8_t* data, int len, int numbps, int npasses, int orient,
                 int32_t* coeff, size_t pitch, int cw, int ch);

/* Code-block styles (T.800 Table A.19, COD SPcod byte): selective arithmetic-coding bypass
 * (the significance-propagation and refinement passes from the fifth bit-plane on are written
 * as raw bits, D.6), context reset at every pass boundary, and termination of the codeword
 * after every pass.  Each terminated segment starts afresh (MQ INITENC, or a new raw byte). */
enum { OR_STYLE_BYPASS = 1, OR_STYLE_RESET = 2, OR_STYLE_TERMALL = 4 };
/* 1 when pass `pass` (0 = the first cleanup pass) is raw-coded under `style` */
int or_t1_pass_raw(int style, int pass);
/* 1 when the codeword is terminated after pass `pass` of a block coded in `npasses` passes */
int or_t1_pass_terminated(int style, int pass, int npasses);
/* or_t1_encode with a code-block style; pass_end (optional, 96 entries) receives, per pass,
 * the codeword bytes when the pass ended (exact where the pass is terminated). */
int or_t1_encode_styled(const int32_t* coeff, size_t pitch, int cw, int ch, int orient, int style, uint8_t* out,
                        int cap, or_t1_info* info, int* pass_end);
/* Decodes a block coded with `style`; the codeword segments are located by pass_end (the
 * encoder's pass ends, exact at terminated passes; NULL for one segment of `len` bytes). */
int or_t1_decode_styled(const uint8_t* data, int len, const int* pass_end, int numbps, int npasses, int orient,
                        int style, int32_t* coeff, size_t pitch, int cw, int ch);

/* ---- whole-image encode (tier-1 + tier-2) --------------------------------------------------- */
typedef struct {
    int levels;
    int cbw, cbh;          /* code-block size (powers of two, 4..64) */
    int lossless;          /* 1: RCT + 5/3, 0: ICT + 9/7 + quantiser */
    int order;             /* OR_ORDER_* for the 5/3 path */
    const float* steps;    /* 3L+1 quantiser steps (lossy); NULL = 8*2^-level */
    int tier1_only;        /* 1: stop after tier-1 (no codestream written; out may be NULL) */
    int style;             /* code-block style, OR_STYLE_* bits (0: none) */
} or_enc_params;
/* Encodes an interleaved uint8 image (ncomp 1 or 3) into a raw J2K codestream.  Returns the
 * codestream length, or -1 when `cap` is too small.  With p->tier1_only the image is coded up
 * to the code-blocks' codewords only (planar, colour transform, DWT, quantiser, tier-1) and the
 * return value is the sum of the codeword lengths. */
long or_encode_image(const uint8_t* img, size_t w, size_t h, int ncomp, const or_enc_params* p,
                     uint8_t* out, long cap);

/* ---- differentiable 9/7 (FP64) ------------------------------------------------------------- */
/* Philox4x32-10 (Salmon et al., SC'11) uniform in [-0.5, 0.5) for element index i. */
double or_philox_uniform(uint64_t seed, uint64_t i);
double or_rd_noise(uint64_t seed, size_t w, size_t x, size_t y);
void or_philox4x32(uint32_t key0, uint32_t key1, const uint32_t ctr[4], uint32_t out[4]);
/* loss = mean((x_hat - x)^2) + lam * sum log2(1 + |y + u*step|/step) over all coefficients,
 * x_hat = IDWT(y + u*step), y = DWT(x); steps = exp(log_steps[b]).  Returns the loss; when
 * grad_x / grad_ls are non-NULL they receive the analytic gradients. */
double or_rd_loss_f64(const double* x, size_t w, size_t h, int levels, const double* log_steps,
                      double lam, uint64_t seed, double* grad_x, double* grad_ls);

#ifdef __cplusplus
}
#endif
#endif
