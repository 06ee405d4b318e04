/*
 * j2k_b200 — C ABI of the B200 (sm_100a) JPEG 2000 encode/decode hot path.
 *
 * This header replaces the OpenCL plumbing of knopkem/roger (OCLDeviceManager, OCLQueue,
 * OCLMemoryManager, OCLKernel; src/ocl_platform.h, src/OCLUtil.h:31-39) with a context that owns
 * a CUDA stream plus grow-only device scratch, and exposes each stage operator of the reference
 * as one call.  Conventions:
 *   - every call returns j2k_status (0 = ok, < 0 = error); j2k_last_error() gives the message.
 *     The reference logged and swallowed cl_int failures (src/OCLUtil.cpp:60-74); here nothing
 *     is swallowed.
 *   - stage operators take DEVICE pointers owned by the caller and are ordered on the context's
 *     stream (j2k_ctx_set_stream to use your own); j2k_stream_sync replaces clFinish
 *     (src/OCLEncodeDecode.cpp:33-36).
 *   - a context is not thread-safe: use one per host thread (as the reference's single in-order
 *     queue, src/OCLUtil.cpp:505-516).
 *   - device code never traps: kernels report through an error word that becomes a status.
 *   - pitches are in ELEMENTS of the buffer's type unless the name says bytes.
 *   - no C++ exceptions cross this boundary.
 */
#ifndef J2K_B200_H
#define J2K_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int j2k_status;
#define J2K_OK 0
#define J2K_ERR_INVALID_ARG (-1)
#define J2K_ERR_CUDA (-2)
#define J2K_ERR_OUT_OF_MEMORY (-3)
#define J2K_ERR_DEVICE (-4)       /* a kernel set its error word (bad descriptor, bound hit) */
#define J2K_ERR_CAPACITY (-5)     /* an output buffer was too small; nothing past it was written */
#define J2K_ERR_UNSUPPORTED (-6)
#define J2K_ERR_TIMEOUT (-7)      /* a bounded device-side wait gave up */
#define J2K_ERR_HOST (-8)         /* a host-side failure other than memory (a host thread could not start) */

enum { J2K_U8 = 0, J2K_I16 = 1, J2K_I32 = 2, J2K_F32 = 3 };
enum { J2K_MCT_NONE = 0, J2K_MCT_RCT = 1, J2K_MCT_ICT = 2 };
/* J2K_ORDER_T800: columns then rows per level (T.800 F.4.2; any conformant decoder inverts it).
 * J2K_ORDER_REF : rows then columns per level (src/CL/ocldwt53.cl:206-277, the reference). */
enum { J2K_ORDER_T800 = 0, J2K_ORDER_REF = 1 };
enum { J2K_W53 = 53, J2K_W97 = 97 };
enum { J2K_BAND_LL = 0, J2K_BAND_HL = 1, J2K_BAND_LH = 2, J2K_BAND_HH = 3 };

typedef struct j2k_ctx j2k_ctx;

/* ---- context: replaces OCLDeviceManager::init/getInfo + ocl_args_d_t ------------------------ */
j2k_status j2k_ctx_create(int device, j2k_ctx** out);
j2k_status j2k_ctx_destroy(j2k_ctx* ctx);
/* Launch on `cuda_stream` from now on (NULL = the CUDA legacy default stream).  A new context
 * uses a non-blocking stream of its own; j2k_ctx_use_own_stream switches back to it. */
j2k_status j2k_ctx_set_stream(j2k_ctx* ctx, void* cuda_stream);
j2k_status j2k_ctx_use_own_stream(j2k_ctx* ctx);
void* j2k_ctx_stream(j2k_ctx* ctx);
j2k_status j2k_stream_sync(j2k_ctx* ctx);                          /* replaces clFinish */
const char* j2k_last_error(const j2k_ctx* ctx);
/* Launch-shape knobs (set by the autotuner; defaults are sensible).  No reference counterpart:
 * the reference fixed its OpenCL work-group shapes in -D build strings (src/OCLEncoder.cpp:27-29). */
enum {
    J2K_TUNE_MQ_LANES = 1,   /* one-lane-per-block MQ kernel: blocks per warp (8, 16 default, 32) after
                                the tiers of J2K_TUNE_MQ_TIER */
    J2K_TUNE_MQ_VARIANT = 2, /* 0: one lane per block (default); 1: state warp + code-register warp */
    J2K_TUNE_DWT_FAST_TH = 3, /* register-lifting forward DWT tile height: 16 (default), 32, 0 = off */
    J2K_TUNE_DWT_PIPE = 4,    /* 1: that kernel streams bands with cp.async double buffering (default 0) */
    J2K_TUNE_DWT_REG = 5,     /* 1 (default): that kernel loads its columns straight into registers;
                                 0: it stages the strip in shared memory with cp.async */
    J2K_TUNE_DWT_TMA = 7,     /* 1: that kernel is the TMA-staged form (persistent CTAs, each strip brought in
                                 by one tensor copy, two stages deep) */
    J2K_TUNE_T1A_CTAS = 8,    /* tier-1 context modelling: resident CTAs per SM its registers are cut for,
                                 2 (default, no spills) or 3 */
    J2K_TUNE_DWT_TAIL = 9,    /* the forward DWT's deep levels in one launch.  1: those with at most two tiles
                                 per resident CTA, one cooperative launch with grid barriers between
                                 levels; 2, 3, 4, 5: from the first level with at most 96, 32, 96, 320
                                 tiles per plane, one thread-block cluster of 16, 16, 8, 16 CTAs per
                                 plane with the cluster barrier between levels.  0 (default): off */
    J2K_TUNE_T1D_LANES = 10,  /* tier-1 decoder: code-blocks decoded side by side in one warp, one per lane
                                 (2, 4 default, 8, 16, 32); 0: one warp per block, lane 0 decoding */
    J2K_TUNE_T1D_STEPS = 11,  /* 1: with 8, 16 or 32 lanes, unstyled blocks are decoded in a loop of one
                                 symbol per step (one MQ decoding site); 0 (default): in the pass /
                                 stripe / column loops */
    J2K_TUNE_PLANAR = 12,     /* interleaved-to-planar split of contiguous images: 0: 16 pixels per thread;
                                 1 (default) / 2: 4 pixels per thread and step, a warp's stores contiguous,
                                 4 / 8 steps per thread with all their loads issued first */
    J2K_TUNE_DWT97_ROWS = 13, /* differentiable 9/7 (j2k_dwt97_*): 1 (default) runs every level whose width is
                                 a power of two in 64..1024 as bands of 16 full rows (a warp per row in
                                 registers, no halo columns); 0: the 248 x 16 strip kernels */
    J2K_TUNE_T1D_ORDER = 14,  /* tier-1 decoder with blocks side by side in a warp: 1 (default) gives the
                                 warps their blocks sorted by codeword length, longest first (the blocks
                                 of a warp then take about as long); 0: list order */
    J2K_TUNE_DWT_PX = 15,     /* encoder of interleaved 8-bit pixels (j2k_encoder_run_interleaved), 1 or 3
                                 components, T.800 order: 1 runs the level shift and colour transform
                                 inside the first DWT level's loads, so the component planes are never
                                 written (a third of the DRAM bytes, but more instructions in a level
                                 kernel that is issue-bound: slower on B200); 0 (default): a planar
                                 split first, then the DWT of the planes.  Same coefficients either way */
    J2K_TUNE_MQ_TIER = 6      /* MQ kernel schedule: value = tier << 24 | lanes << 20 | warps.  The
                                 blocks, longest first, go to up to 4 tiers of `warps` warps with
                                 `lanes` blocks each (lanes 0 ends the list), then to warps of
                                 J2K_TUNE_MQ_LANES blocks, so that the longest serial chains share
                                 their warp with fewer others.  Default: SM-count warps x 1 block,
                                 2 x SM-count warps x 4 blocks */
};
j2k_status j2k_ctx_set_tuning(j2k_ctx* ctx, int key, int value);
const char* j2k_status_string(j2k_status s);
int j2k_version(void);

/* ---- RGB -> planar (+ level shift + RCT/ICT): replaces OCLRGBtoPlanar<T>::run
 *      (src/OCLRGBtoPlanar.cpp:36-44) and kernel src/CL/oclplanar.cl:23-40.
 * in: interleaved uint8, ncomp (1..4) samples per pixel, row pitch in bytes.
 * planes: out_dtype J2K_I32 (mct NONE/RCT) or J2K_F32 (mct NONE/ICT); plane c starts at
 * planes + c*plane_stride elements, rows plane_pitch elements apart.  Subtracts 128. */
j2k_status j2k_rgb_to_planar(j2k_ctx* ctx, const uint8_t* in, size_t in_pitch_bytes, int ncomp,
                             int mct, int out_dtype, void* planes, size_t plane_pitch,
                             size_t plane_stride, size_t w, size_t h);
/* Inverse: planes (+ inverse MCT, + 128, round, clamp) -> interleaved uint8. */
j2k_status j2k_planar_to_rgb(j2k_ctx* ctx, const void* planes, int in_dtype, size_t plane_pitch,
                             size_t plane_stride, int ncomp, int mct, uint8_t* out,
                             size_t out_pitch_bytes, size_t w, size_t h);

/* ---- forward DWT: replaces OCLDWTForward<T>::run (src/OCLDWTForward.cpp:124-137) and kernels
 * src/CL/ocldwt53.cl:167-292 / src/CL/ocldwt97.cl:196-420,487-716.
 * Out-of-place, all `levels` levels, Mallat layout in `out` (low half first on both axes,
 * ceil(n/2) low samples).  kernel 53: in/out int32.  kernel 97: in float32; out float32 when
 * steps == NULL, else int32 dead-zone indices with steps[b] (host array, 3*levels+1 entries in
 * T.800 QCD order: LL_L, then HL,LH,HH for level L..1).  `in` is not modified.
 * Uses context scratch for the intermediate LL bands. */
j2k_status j2k_dwt_forward(j2k_ctx* ctx, int kernel, int order, const void* in, size_t in_pitch,
                           void* out, size_t out_pitch, size_t w, size_t h, int levels,
                           const float* steps);
/* ---- inverse DWT: replaces OCLDWTRev<T>::run (src/OCLDWTRev.cpp:39-58), whose kernels
 * (ocldwt53rev.cl / ocldwt97rev.cl) are forward transforms; this is the true inverse.
 * kernel 97 with steps != NULL reads int32 indices and dequantises ((|q|+1/2)*step). */
j2k_status j2k_dwt_inverse(j2k_ctx* ctx, int kernel, int order, const void* in, size_t in_pitch,
                           void* out, size_t out_pitch, size_t w, size_t h, int levels,
                           const float* steps);

/* ---- allocation-free forward DWT.  No counterpart in the reference (its OCLMemoryManager
 * allocated every image itself).  For callers that cannot allocate device memory — a plugin
 * inside a framework that owns the device heap, or a latency-critical pipeline that must never
 * reach cudaMalloc — this variant of j2k_dwt_forward needs no context and allocates nothing:
 * its intermediate LL bands live in a 5 MiB array reserved in the library's device image,
 * which every GPU that loads the library holds until the process exits.  Limit: the LL bands
 * of the image must fit, i.e. ceil(w/2)*ceil(h/2) + ceil(w/4)*ceil(h/4) <= 1,310,720 samples
 * (2048x2048 at most for square images); larger images return J2K_ERR_CAPACITY.  Arguments
 * and output are those of j2k_dwt_forward, launched on `cuda_stream` (NULL = legacy default
 * stream).  The first call on a device looks up the array's device address; make that first
 * call before any stream capture.  The address is kept per device and CUDA context, so the
 * first call after a cudaDeviceReset (which creates a new context) looks it up again.  All calls share the one array (its contents persist from
 * the previous call and nothing needs clearing), so calls whose execution overlaps on the GPU
 * race: order them on one stream or synchronise between them.  Errors are returned as
 * statuses only (there is no context to hold a message). */
j2k_status j2k_dwt_forward_noalloc(void* cuda_stream, int kernel, int order, const void* in,
                                   size_t in_pitch, void* out, size_t out_pitch, size_t w, size_t h,
                                   int levels, const float* steps);

/* Batched forms: n images, image i at in + i*in_stride / out + i*out_stride elements, one
 * launch per level for the whole batch (the reference transforms one image per call). */
j2k_status j2k_dwt_forward_batch(j2k_ctx* ctx, int kernel, int order, const void* in, size_t in_pitch,
                                 size_t in_stride, void* out, size_t out_pitch, size_t out_stride, int n,
                                 size_t w, size_t h, int levels, const float* steps);
j2k_status j2k_dwt_inverse_batch(j2k_ctx* ctx, int kernel, int order, const void* in, size_t in_pitch,
                                 size_t in_stride, void* out, size_t out_pitch, size_t out_stride, int n,
                                 size_t w, size_t h, int levels, const float* steps);

/* ---- EBCOT tier-1: replaces OCLBPC<T>::run (src/OCLBPC.cpp:38-50) and src/CL/oclbpc.cl:279-746.
 * Code-blocks partition every subband of a Mallat plane (w x h, `levels`) on a cbw x cbh grid
 * anchored at the subband origin, subbands in QCD order, blocks in raster order. */
/* Code-block styles (T.800 Table A.19, the COD code-block style byte), no counterpart in the
 * reference.  BYPASS: the significance-propagation and refinement passes from the fifth
 * bit-plane on are written as raw bits (T.800 D.6).  RESET: the context states start afresh at
 * every pass.  TERMALL: the codeword is terminated after every pass.  With RESET and TERMALL
 * together every pass is an independent codeword segment, which the encoder codes one lane per
 * pass instead of one lane per code-block.  A styled block's codeword is the concatenation of
 * its segments; its pass ends (codeword bytes when each pass ended, exact at terminated passes,
 * J2K_PASS_STRIDE entries per block) locate them. */
#define J2K_CBLK_BYPASS 1
#define J2K_CBLK_RESET 2
#define J2K_CBLK_TERMALL 4
#define J2K_PASS_STRIDE 92
typedef struct {
    uint32_t offset;   /* byte offset of this block's codeword in the bytes buffer */
    int32_t length;    /* codeword bytes (0 for an all-zero block) */
    uint8_t numbps;    /* magnitude bit-planes coded */
    uint8_t npasses;   /* coding passes (3*numbps-2, or 0) */
    uint8_t orient;    /* J2K_BAND_* */
    uint8_t band;      /* subband index in QCD order */
    uint16_t x0, y0;   /* top-left sample in the component's Mallat plane */
    uint16_t cw, ch;   /* block size */
    uint16_t comp;     /* component index */
    uint16_t reserved;
} j2k_cb_desc;

/* Number of code-blocks of the partition above. */
size_t j2k_codeblock_count(size_t w, size_t h, int levels, int cbw, int cbh);
/* Encodes every code-block of `coeff` (int32, device).  descs (device, count entries) and
 * bytes (device, count*cap_per_block bytes) are written; block i's codeword starts at
 * i*cap_per_block.  J2K_ERR_CAPACITY when a block needs more than cap_per_block bytes.
 * cbw, cbh: powers of two in 4..64, cbw*cbh <= 4096. */
j2k_status j2k_bpc_encode(j2k_ctx* ctx, const int32_t* coeff, size_t pitch, size_t w, size_t h,
                          int levels, int cbw, int cbh, j2k_cb_desc* descs, uint8_t* bytes,
                          size_t cap_per_block);
/* Decodes code-blocks (device descs/bytes as produced above) back into an int32 Mallat plane. */
j2k_status j2k_bpc_decode(j2k_ctx* ctx, const j2k_cb_desc* descs, const uint8_t* bytes,
                          size_t count, int32_t* coeff, size_t pitch, size_t w, size_t h,
                          int levels, int cbw, int cbh);

/* ---- whole-image encoder / decoder: replaces OCLEncoder<T>/OCLDecoder<T>
 * (src/OCLEncoder.cpp:43-52, src/OCLDecoder.cpp:35-38, src/OCLEncodeDecode.h:23-38). */
typedef struct j2k_encoder j2k_encoder;
typedef struct {
    int levels;        /* decomposition levels */
    int cbw, cbh;      /* code-block size (default 64x64) */
    int order;         /* J2K_ORDER_* (default T800) */
    const float* steps;/* lossy: 3*levels+1 steps; NULL = 8*2^-level.  Each must fit the QCD's
                          5-bit exponent (about 2^(g-23) <= step < 2^(g+9), g = 0 for LL, 1 for
                          HL/LH, 2 for HH); others are refused with J2K_ERR_INVALID_ARG */
    size_t target_bytes; /* 0: every coding pass kept; else the codestream is cut to at most this many
                            bytes by rate-distortion optimised truncation of the code-blocks (PCRD-opt:
                            bit-plane truncation points, one quality layer).  No counterpart in the
                            reference, which writes no codestream. */
    int layers;          /* > 1: that many quality layers, cut by PCRD-opt to layer_bytes[l] bytes of
                            codestream for layers 0..l (non-decreasing; 0 in the last place keeps
                            every pass: a lossless final layer); target_bytes is then unused */
    const size_t* layer_bytes;
    int cblk_style;      /* J2K_CBLK_* bits (0: none).  Encoding: the code-blocks are coded in that
                            style (rate control and layers are not combined with a style); the
                            pass ends come from j2k_encoder_get_pass_ends.  Decoding: the style
                            the code-blocks were coded in */
    const uint32_t* pass_ends; /* decoding with a style: the blocks' pass ends, J2K_PASS_STRIDE
                                  per block in descriptor order, in the memory the descriptors
                                  are in */
} j2k_enc_params;

j2k_status j2k_encoder_create(j2k_ctx* ctx, int lossy, int output_dwt_only, j2k_encoder** out);
j2k_status j2k_encoder_destroy(j2k_encoder* enc);
/* Reference-shaped entry (OCLEncoder<T>::run(components, w, h, levels, precision)): planar HOST
 * components, already level-shifted (pixel-128) as src/OCLTest.cpp:80-90 builds them, of type
 * dtype (J2K_I16, J2K_I32 or J2K_F32).  ncomp >= 3 applies RCT (lossless) / ICT (lossy) to
 * components 0..2.  precision = bit depth (8). */
j2k_status j2k_encoder_run(j2k_encoder* enc, const void* const* comps, int ncomp, int dtype,
                           size_t w, size_t h, size_t levels, size_t precision,
                           const j2k_enc_params* params);
/* Fast entry: interleaved uint8 pixels (ncomp 1 or 3), on the host (on_device = 0, copied
 * through pinned staging) or already on the device. */
j2k_status j2k_encoder_run_interleaved(j2k_encoder* enc, const uint8_t* pixels, int on_device,
                                       size_t pitch_bytes, int ncomp, size_t w, size_t h,
                                       const j2k_enc_params* params);
/* Host copy of the DWT coefficients (int32 lossless / lossy-quantised, float when
 * output_dwt_only && lossy), planes back to back, row pitch in bytes returned (the reference's
 * OCLEncodeDecode::mapDWTOut dropped it).  Valid until unmap. */
j2k_status j2k_encoder_map_dwt_out(j2k_encoder* enc, void** ptr, size_t* pitch_bytes);
j2k_status j2k_encoder_unmap_dwt_out(j2k_encoder* enc, void* ptr);
/* Code-block results of the last run, copied to the host: *count descriptors (component-major)
 * and their codewords packed back to back (descs[i].offset rewritten to the packed offset).
 * Pass descs/bytes NULL to query count and total bytes. */
j2k_status j2k_encoder_get_codeblocks(j2k_encoder* enc, j2k_cb_desc* descs, size_t* count,
                                      uint8_t* bytes, size_t cap, size_t* used);
/* Times the tier-1 MQ schedules (J2K_TUNE_MQ_TIER / _LANES) on the last run's coefficients and
 * keeps the fastest in the encoder's context; the result stays that of the last run.
 * report (optional, 4 ints): tier-0 warps, tier-1 warps, tier-1 blocks per warp, blocks per warp. */
j2k_status j2k_encoder_autotune(j2k_encoder* enc, int reps, int* report);
/* T.800 codestream (SOC..EOC, one tile, LRCP; one quality layer, or the layers asked for) of the
 * last run.  out NULL: size only. */
j2k_status j2k_encoder_get_codestream(j2k_encoder* enc, uint8_t* out, size_t cap, size_t* len);
/* Pass ends of the last styled encode (j2k_enc_params.cblk_style != 0): for every code-block in
 * job order J2K_PASS_STRIDE entries, entry p the codeword bytes when pass p ended (exact where
 * the style terminates the codeword after pass p; entries past the block's npasses are 0).
 * ends NULL: *count = the number of entries only.  No reference counterpart. */
j2k_status j2k_encoder_get_pass_ends(j2k_encoder* enc, uint32_t* ends, size_t cap, size_t* count);
/* Device-side view of the last run's results (valid until the next run). */
j2k_status j2k_encoder_device_results(j2k_encoder* enc, const j2k_cb_desc** descs,
                                      const uint8_t** bytes, size_t* count,
                                      size_t* cap_per_block);

typedef struct j2k_decoder j2k_decoder;
j2k_status j2k_decoder_create(j2k_ctx* ctx, int lossy, j2k_decoder** out);
j2k_status j2k_decoder_destroy(j2k_decoder* dec);
/* Decodes code-blocks (layout of j2k_encoder_get_codeblocks; host or device memory) to an
 * interleaved uint8 image (host or device). */
j2k_status j2k_decoder_run_codeblocks(j2k_decoder* dec, const j2k_cb_desc* descs,
                                      const uint8_t* bytes, size_t nbytes, int on_device,
                                      int ncomp, size_t w, size_t h, const j2k_enc_params* params,
                                      uint8_t* out, int out_on_device, size_t out_pitch_bytes);

/* Batched decode: the code-blocks of n images (each as j2k_codestream_read returns them, host
 * memory) are uploaded in one copy and tier-1 decoded in one launch; each image then runs its
 * inverse DWT and inverse colour transform, and every image's pixels come back in one copy into
 * its `out` (interleaved uint8, pitch w*ncomp).  The reference decodes nothing
 * (src/OCLDecoder.cpp:35-38). */
typedef struct {
    uint32_t w, h;
    int ncomp;                 /* 1 or 3 (colour transform) */
    int lossless;              /* 1: 5/3 (RCT); 0: 9/7 (ICT) */
    int levels, cbw, cbh;
    const float* steps;        /* lossy: 3*levels+1 steps (QCD order); NULL = 8*2^-level */
    const j2k_cb_desc* descs;  /* job order, count entries */
    size_t count;
    const uint8_t* bytes;      /* codewords, descs[i].offset into it */
    size_t nbytes;
    uint8_t* out;              /* host output */
    int cblk_style;            /* code-block style of the blocks (J2K_CBLK_*) */
    const uint32_t* pass_ends; /* with a style: J2K_PASS_STRIDE pass ends per block (host) */
} j2k_decode_item;
j2k_status j2k_decoder_run_batch(j2k_decoder* dec, const j2k_decode_item* items, int n);
/* The same from codestreams: each stream's tier-2 runs on a pool of host threads (the first
 * max_layers quality layers, 0: all), then the batched decode above; outs[k] receives stream k's
 * pixels (interleaved uint8, w*h*ncomp bytes; j2k_codestream_info gives w, h, ncomp). */
j2k_status j2k_decoder_run_codestreams(j2k_decoder* dec, const uint8_t* const* streams, const size_t* sizes, int n,
                                       int max_layers, uint8_t* const* outs);

/* ---- codestream reading (tier-2 decoding).  No counterpart in the reference, which writes and
 * reads no codestream.  Parses a T.800 codestream of one tile (tile-parts allowed), any number of
 * quality layers, LRCP or RLCP progression, one precinct per resolution, the default code-block style
 * or the bypass / reset / per-pass termination styles (see j2k_codestream_pass_ends),
 * reversible (5/3) or irreversible (9/7) transform with no, derived or expounded quantisation,
 * 1 or 3 (with colour transform) 8-bit components: the subset this library writes and the one
 * OpenJPEG writes by default.  SOP/EPH markers are skipped.  Other streams return
 * J2K_ERR_UNSUPPORTED with the reason in `err`.  Call with descs = bytes = NULL for the stream
 * info, the code-block count and the codeword bytes needed; then with buffers of that size:
 * descs (job order, as j2k_encoder_get_codeblocks) and the codewords packed back to back.  The
 * result feeds j2k_decoder_run_codeblocks (lossy = !info->lossless, steps = info->steps).
 * Host memory only; needs no context. */
#define J2K_MAX_BANDS 97
typedef struct {
    uint32_t w, h;
    int ncomp, levels, cbw, cbh;
    int lossless;      /* 1: reversible 5/3; 0: irreversible 9/7 */
    int mct;           /* colour transform (RCT with 5/3, ICT with 9/7) */
    int guard;         /* guard bits */
    int precision;     /* bits per component sample */
    int layers, progression;
    float steps[J2K_MAX_BANDS];  /* per-subband quantiser steps in QCD order (1 when lossless) */
    int cblk_style;              /* J2K_CBLK_* bits of the code-block style */
} j2k_stream_info;
j2k_status j2k_codestream_read(const uint8_t* cs, size_t n, j2k_stream_info* info, j2k_cb_desc* descs,
                               size_t* count, uint8_t* bytes, size_t cap, size_t* used, char* err,
                               size_t errlen);
/* Tier-2 only: writes the codestream of code-blocks coded elsewhere (this library's encoders,
 * j2k_codestream_read, or another tier-1), host memory, no context.  descs in job order
 * (component, subband in QCD order, raster), codewords in `bytes` at descs[i].offset; lossless
 * selects 5/3 (RCT for 3 components), else 9/7 (ICT) with `steps` (3*levels+1, NULL =
 * 8*2^-level).  layers <= 1 with NULL arrays: one layer holding every block's npasses and
 * length.  Else `layers` quality layers: after layer l block i holds layer_npasses[l*count+i]
 * passes and the first layer_lengths[l*count+i] bytes of its codeword (non-decreasing in l, at
 * most the descriptor's; 0 bytes when 0 passes).  out NULL: size only.  The reference writes no
 * codestream. */
j2k_status j2k_codestream_write(uint32_t w, uint32_t h, int ncomp, int levels, int cbw, int cbh, int lossless,
                                const float* steps, const j2k_cb_desc* descs, size_t count, const uint8_t* bytes,
                                size_t nbytes, int layers, const int32_t* layer_npasses,
                                const int32_t* layer_lengths, uint8_t* out, size_t cap, size_t* len);
/* Only the main header: the stream info without parsing any packet (cheap). */
j2k_status j2k_codestream_info(const uint8_t* cs, size_t n, j2k_stream_info* info, char* err, size_t errlen);
/* Same, keeping only the first max_layers quality layers (0: all): each block's codeword is the
 * concatenation of its segments from those layers and npasses counts their passes, so the
 * result decodes to the image at that layer's quality. */
j2k_status j2k_codestream_read_layers(const uint8_t* cs, size_t n, int max_layers, j2k_stream_info* info,
                                      j2k_cb_desc* descs, size_t* count, uint8_t* bytes, size_t cap,
                                      size_t* used, char* err, size_t errlen);
/* The pass ends of the blocks j2k_codestream_read_layers returns (same stream, same max_layers):
 * J2K_PASS_STRIDE entries per block in job order, for decoding a styled stream
 * (j2k_enc_params.pass_ends); for an unstyled stream every entry is the block's codeword length.
 * ends NULL: *count only.  Streams with the bypass, reset, per-pass or predictable termination
 * styles are read; vertically causal contexts and segmentation symbols are refused. */
j2k_status j2k_codestream_pass_ends(const uint8_t* cs, size_t n, int max_layers, uint32_t* ends, size_t cap,
                                    size_t* count, char* err, size_t errlen);

/* ---- differentiable 9/7 (no counterpart in the reference).  n images of w x h float32,
 * planes back to back (pitch w, plane stride w*h), device pointers, T.800 order.  Used with
 * j2k_dwt_forward / j2k_dwt_inverse (kernel 97, steps NULL) as the forward operators.
 * j2k_dwt97_forward_adjoint: transpose of the forward DWT (Mallat gradient -> image gradient).
 * j2k_dwt97_inverse_adjoint: transpose of the inverse DWT (image gradient -> Mallat gradient).
 * The relaxed quantiser replaces rounding by additive noise of one step: for a coefficient y of
 * subband b (step = exp(log_steps[b]), log_steps a device array of 3L+1 floats),
 *   t = y/step + u, y_hat = t*step, rate = log2(1+|t|), u ~ U[-1/2,1/2): Philox4x32-10 keyed
 *   by seed+image, counter y*ceil(w/4) + x/4 for the Mallat sample (x, y), output word x%4,
 *   u = (word >> 8) * 2^-24 - 1/2.
 * Forward writes y_hat and, per (image, band, part), a partial rate sum: the plane's rows are
 * split into parts_per_band row ranges, partial[(image*(3L+1) + band)*parts_per_band + part],
 * to be summed by the caller in a fixed order.  Backward, for a loss L(y_hat) + lam*sum(rate),
 * writes dL/dy and the same layout of partials of dL/dlog_step.  levels <= 16. */
j2k_status j2k_dwt97_forward_adjoint(j2k_ctx* ctx, const float* g_coef, float* g_img, int n, size_t w,
                                     size_t h, int levels);
j2k_status j2k_dwt97_inverse_adjoint(j2k_ctx* ctx, const float* g_img, float* g_coef, int n, size_t w,
                                     size_t h, int levels);
j2k_status j2k_relaxed_quant_forward(j2k_ctx* ctx, const float* y, float* y_hat, int n, size_t w, size_t h,
                                     int levels, const float* log_steps, uint64_t seed, float* rate_partials,
                                     int parts_per_band);
j2k_status j2k_relaxed_quant_backward(j2k_ctx* ctx, const float* y, const float* g_yhat, float* g_y, int n,
                                      size_t w, size_t h, int levels, const float* log_steps, uint64_t seed,
                                      float lam, float* g_logstep_partials, int parts_per_band);
/* Forward that also writes every sample's noise u to `noise` (n*w*h floats), for a backward that
 * then reads it instead of regenerating it. */
j2k_status j2k_relaxed_quant_forward_noise(j2k_ctx* ctx, const float* y, float* y_hat, float* noise, int n, size_t w,
                                           size_t h, int levels, const float* log_steps, uint64_t seed,
                                           float* rate_partials, int parts_per_band);
/* Backward with the incoming gradient scaled on the device: g_yhat = (*scale) * alpha * g_in and the
 * rate weight (*scale) * lam (scale: device pointer to one float, NULL = 1), so that an autograd
 * backward can pass its output gradient without reading it on the host.  noise: the forward's
 * noise (j2k_relaxed_quant_forward_noise), or NULL to regenerate it from seed. */
j2k_status j2k_relaxed_quant_backward_scaled(j2k_ctx* ctx, const float* y, const float* g_in, float* g_y, int n,
                                             size_t w, size_t h, int levels, const float* log_steps, uint64_t seed,
                                             const float* noise, float lam, const float* scale, float alpha,
                                             float* g_logstep_partials, int parts_per_band);
/* Fused residual forms for a distortion term mean((IDWT(y) - x)^2):
 * j2k_dwt97_inverse_residual writes d = IDWT(y) - x (the reconstruction itself is never stored)
 * and one partial sum of d^2 per 248 x 16 tile of the finest level, j2k_dwt97_residual_partials
 * of them, image-major; j2k_dwt97_forward_adjoint_residual writes
 * g_img = DWT^T(g_coef) - (*scale) * alpha * sub (scale: device pointer or NULL = 1). */
size_t j2k_dwt97_residual_partials(size_t w, size_t h, int n);
/* The scalar of the fused rate-distortion loss from the partial sums above, in one launch:
 * *loss = sum(sq_partials) * inv_count + lam * sum(rate_partials) (device pointers).  And the
 * per-band sums of quantiser partials laid out (image, band, part): out[b] = sum over images and
 * parts (nb entries), e.g. the log-step gradient of j2k_relaxed_quant_backward_scaled. */
j2k_status j2k_dwt97_rd_finalize(j2k_ctx* ctx, const float* rate_partials, size_t nrate, const float* sq_partials,
                                 size_t nsq, double inv_count, float lam, float* loss);
j2k_status j2k_dwt97_band_sum(j2k_ctx* ctx, const float* partials, int n, int nb, int k, float* out);
j2k_status j2k_dwt97_inverse_residual(j2k_ctx* ctx, const float* y, const float* x, float* d, int n, size_t w,
                                      size_t h, int levels, float* sq_partials);
/* The fused rate-distortion step of config 3 (no counterpart in the reference) in two calls.
 * j2k_dwt97_rd_forward: y = DWT(x) with the relaxed quantiser run as each level writes its bands
 * (y and its noise u written; rate partial sums), then the inverse of y_hat = (y/step + u)*step,
 * formed as the bands are loaded, with d = IDWT(y_hat) - x and the partial sums of d^2
 * (j2k_dwt97_residual_partials of them).  rate_partials: n x (3L+1) x j2k_dwt97_rd_parts floats,
 * laid out (image, band, part); j2k_dwt97_rd_finalize turns both sets into the loss.
 * j2k_dwt97_rd_backward: for the loss's gradient (*scale) (device pointer, NULL = 1) and
 * alpha = 2 / (n w h): g_y = dL/dy (the transpose of the inverse with the quantiser backward in
 * its band writes) and g_x = DWT^T(g_y) - (*scale) alpha d; log-step partial sums in the same
 * layout, for j2k_dwt97_band_sum.  y, u and d are the forward's outputs.  When every level's width
 * is a power of two in 64..1024 (J2K_TUNE_DWT97_ROWS on) both run as band kernels; otherwise as
 * the separate passes above.  y, u, d, g_y, g_x: n*w*h floats each. */
size_t j2k_dwt97_rd_parts(j2k_ctx* ctx, size_t w, size_t h, int levels);
j2k_status j2k_dwt97_rd_forward(j2k_ctx* ctx, const float* x, float* y, float* u, float* d, int n, size_t w,
                                size_t h, int levels, const float* log_steps, uint64_t seed, float* rate_partials,
                                float* sq_partials);
j2k_status j2k_dwt97_rd_backward(j2k_ctx* ctx, const float* y, const float* u, const float* d, const float* log_steps,
                                 float lam, const float* scale, float alpha, float* g_y, float* g_x, int n, size_t w,
                                 size_t h, int levels, float* ls_partials);
j2k_status j2k_dwt97_forward_adjoint_residual(j2k_ctx* ctx, const float* g_coef, const float* sub,
                                              const float* scale, float alpha, float* g_img, int n, size_t w,
                                              size_t h, int levels);

/* ---- batched encoder.  No counterpart in the reference, which encodes one image per
 * OCLEncoder<T>::run call (src/OCLEncoder.cpp:43-52).  Many images of uneven size, mixed 5/3 and
 * 9/7, are encoded by one fixed launch sequence (batched planar split, one DWT launch per level
 * and filter, one persistent tier-1 pass over a device-side queue of all code-blocks, one MQ
 * launch), captured once in a CUDA graph and replayed. */
typedef struct {
    uint32_t w, h;
    int ncomp;           /* 1 or 3 */
    int kernel;          /* J2K_W53: lossless (RCT); J2K_W97: ICT + dead-zone quantiser */
    int levels;          /* 1..32 */
    int cb;              /* square code-block side: power of two in 4..64 */
    const float* steps;  /* 9/7: 3*levels+1 steps (copied); NULL = 8*2^-level */
} j2k_batch_image;
typedef struct j2k_batch j2k_batch;
enum {
    J2K_BATCH_USE_GRAPH = 1,     /* 1 (default): capture the launch sequence once, replay it */
    J2K_BATCH_TILE53 = 2,        /* DWT tile shape of 5/3 images: 0 64x64, 1 128x32, 2 32x128 (shared-memory
                                    tiles), 3 (default) 248x16 register lifting */
    J2K_BATCH_TILE97 = 3,        /* same for 9/7 images */
    J2K_BATCH_PHASE_A_ORDER = 4, /* 1: context modelling takes the largest code-blocks first */
    J2K_BATCH_MQ_VARIANT = 5,    /* read-only here; set with j2k_ctx_set_tuning */
    J2K_BATCH_MQ_LANES = 6,
    J2K_BATCH_MQ_TIERS = 7,      /* read-only: 1 when the MQ coder runs the tiered warp schedule */
    J2K_BATCH_GRAPH_KERNELS = 8, /* read-only: kernel launches of one replay of the captured
                                    sequence, this library's own (library sort/scan kernels are
                                    not counted); 0 before the first graph encode */
    J2K_BATCH_STAGES = 9,        /* stages an encode runs, for timing them apart: 1 planar split,
                                    2 DWT, 4 tier-1 (default 7, all).  Without 4 the encode leaves
                                    no code-blocks to read */
    J2K_BATCH_T1A_CTAS = 10      /* read-only: the context modelling's resident CTAs per SM that
                                    the autotuner kept (J2K_TUNE_T1A_CTAS) */
};
j2k_status j2k_batch_create(j2k_ctx* ctx, const j2k_batch_image* images, int n, j2k_batch** out);
j2k_status j2k_batch_destroy(j2k_batch* b);
/* The batch's packed device input buffer and each image's byte offset in it (n+1 entries,
 * the last is the total): interleaved uint8 pixels, rows packed (pitch = w*ncomp). */
j2k_status j2k_batch_input(j2k_batch* b, uint8_t** device_buffer, size_t* offsets);
/* Encodes the batch.  pixels: per-image pointers (host or device) copied into the input buffer
 * first, or NULL when the caller filled the input buffer itself. */
j2k_status j2k_batch_encode(j2k_batch* b, const uint8_t* const* pixels, int on_device);
/* Same, without waiting: the copies and the launch sequence are queued on the context's stream
 * and the device error word is read (and a tier-1 capacity overflow re-run) by the next call
 * that needs the result (j2k_batch_pack, j2k_batch_get_codeblocks, ...).  Host pixels must stay
 * valid until the stream has consumed them (page-locked memory makes the copies asynchronous). */
j2k_status j2k_batch_encode_async(j2k_batch* b, const uint8_t* const* pixels, int on_device);
/* Only the copies of j2k_batch_encode (queued on the context's stream), for callers that upload
 * on a copy stream and encode with pixels = NULL on another. */
j2k_status j2k_batch_upload(j2k_batch* b, const uint8_t* const* pixels, int on_device);
j2k_status j2k_batch_set_option(j2k_batch* b, int key, int value);
j2k_status j2k_batch_get_option(j2k_batch* b, int key, int* value);
/* Times the tile shapes and code-block-to-warp schedules on this batch and keeps the fastest;
 * report (optional, 5 ints): tile53, tile97, phase-A order, MQ variant, MQ blocks per warp. */
j2k_status j2k_batch_autotune(j2k_batch* b, int reps, int* report);
/* Per-image results of the last encode: code-blocks (layout of j2k_encoder_get_codeblocks) and
 * the T.800 codestream. */
j2k_status j2k_batch_get_codeblocks(j2k_batch* b, int image, j2k_cb_desc* descs, size_t* count,
                                    uint8_t* bytes, size_t cap, size_t* used);
j2k_status j2k_batch_get_codestream(j2k_batch* b, int image, uint8_t* out, size_t cap, size_t* len);
/* Bulk readback, for hosts that move whole batches: j2k_batch_pack packs every code-block of the
 * last result back to back on the device (job order: image by image, each in the layout of
 * j2k_encoder_get_codeblocks) and returns the total bytes (it waits for the packing sizes);
 * j2k_batch_read_packed then queues the copies of the descriptors (offsets into the packed
 * bytes) and the bytes to host buffers on the context's stream, without waiting, so that with
 * page-locked buffers they overlap other work; j2k_batch_image_jobs gives each image's first
 * job (n+1 entries, the last = the total count). */
j2k_status j2k_batch_pack(j2k_batch* b, size_t* total);
j2k_status j2k_batch_read_packed(j2k_batch* b, j2k_cb_desc* descs, uint8_t* bytes, size_t cap);
j2k_status j2k_batch_image_jobs(j2k_batch* b, size_t* first);

#ifdef __cplusplus
}
#endif
#endif
