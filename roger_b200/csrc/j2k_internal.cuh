// Internal declarations shared by the CUDA translation units of libj2kb200.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <exception>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "j2k_b200.h"

// Every entry point of the C ABI runs its body between J2K_API_BEGIN and J2K_API_END, so that no
// C++ exception crosses the ABI: a failed host allocation returns J2K_ERR_OUT_OF_MEMORY, any
// other exception J2K_ERR_HOST.
#define J2K_API_BEGIN try {
#define J2K_API_END                          \
    }                                        \
    catch (const std::bad_alloc&) {          \
        return J2K_ERR_OUT_OF_MEMORY;        \
    }                                        \
    catch (...) {                            \
        return J2K_ERR_HOST;                 \
    }

// Runs fn(t) for t in [0, nt): t = 0 and every t whose host thread cannot be started run on the
// calling thread, the rest on their own threads.  Every started thread is joined before this
// returns, also when fn throws on the calling thread (the exception is then rethrown).  fn must
// not throw on the other threads.
template <class F>
void j2k_run_threads(int nt, F fn) {
    std::vector<std::thread> pool;
    std::exception_ptr err;
    int t = 1;
    try {
        pool.reserve(nt > 1 ? (size_t)nt - 1 : 0);
        for (; t < nt; ++t) pool.emplace_back(fn, t);
    } catch (...) {  // no more threads: the remaining shares run here
    }
    try {
        fn(0);
        for (; t < nt; ++t) fn(t);
    } catch (...) {
        err = std::current_exception();
    }
    for (auto& th : pool) th.join();
    if (err) std::rethrow_exception(err);
}

// Device error word values (written by kernels, read back by the host; kernels never trap).
enum : uint32_t {
    J2K_DEVERR_NONE = 0,
    J2K_DEVERR_SYM_CAPACITY = 1,  // symbol buffer of a code-block full
    J2K_DEVERR_OUT_CAPACITY = 2,  // codeword buffer of a code-block full
    J2K_DEVERR_BAD_JOB = 3,       // malformed code-block descriptor
    J2K_DEVERR_TIMEOUT = 4,       // bounded wait expired
    J2K_DEVERR_PLANES = 5,        // more magnitude bit-planes than the coder supports
    J2K_DEVERR_SEG_CAPACITY = 6,  // a coding-pass segment outgrew its slot (code-block styles)
};

constexpr int J2K_SCRATCH_SLOTS = 15;

constexpr int J2K_MQ_TIERS = 4;

struct j2k_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::string err;
    // grow-only device scratch slots (each independently sized)
    void* scratch[J2K_SCRATCH_SLOTS] = {};
    size_t scratch_size[J2K_SCRATCH_SLOTS] = {};
    uint32_t* d_err = nullptr;   // device error word
    void* h_pinned = nullptr;    // pinned staging
    size_t h_pinned_size = 0;
    int sm_count = 148;
    int mq_lanes = 8;            // tier-1 MQ: code-blocks per warp after the schedule's tiers (16 from creation)
    int mq_variant = 0;          // 0: one lane per block, 1: state warp + code warp pair
    int dwt_fast_th = 16;        // fast level-0 DWT tile height (16, 32; 0 = off)
    int dwt_pipe = 0;            // fast level-0 DWT: persistent cp.async double-buffered variant
    // MQ schedule: tiers of warps with fewer blocks each for the longest blocks (lanes 0 ends)
    int mq_tier_warps[4] = {0, 0, 0, 0}, mq_tier_lanes[4] = {1, 0, 0, 0};  // tier 0: sm_count warps
    int dwt_reg = 1;             // fast forward DWT: columns loaded straight into registers (0: cp.async strip)
    int t1_seg_factor = 1;       // styled tier-1: pass-segment slot bytes per symbol (grown on overflow)
    int dwt_tma = 0;             // fast forward DWT: strips staged by TMA tensor copies (persistent CTAs)
    int t1a_ctas = 2;            // tier-1 phase A: resident CTAs per SM its registers are cut for (2 or 3)
    int dwt_tail = 0;            // forward DWT: deep levels in one launch (1 cooperative, 2..5 clusters)
    int t1d_lanes = 4;           // tier-1 decoder: code-blocks per warp (2, 4, 8, 16, 32), 0 = one warp per block
    int t1d_steps = 0;           // tier-1 decoder: unstyled blocks by the one-symbol-per-step loop
    int planar_form = 1;         // planar split: 0 16 pixels per thread; 1 / 2: 4 pixels per thread and step
    int dwt97_rows = 1;          // differentiable 9/7: levels 64..1024 wide (powers of two) as full-row bands
    int t1d_order = 1;           // tier-1 decoder: blocks to lanes by codeword length, longest first
    int dwt_px = 0;              // encoder: first DWT level read straight from interleaved pixels
};

// scratch slot ids
enum { SCR_LL0 = 0, SCR_LL1 = 1, SCR_JOBS = 2, SCR_SYMS = 3, SCR_T1STATE = 4, SCR_MISC = 5,
       SCR_PLANES = 6, SCR_MISC2 = 7, SCR_RES = 8, SCR_UNITS = 9, SCR_SEGS = 10, SCR_BARRIER = 11,
       SCR_PLANE = 12, SCR_DECORD = 13, SCR_LLPX = 14 };

j2k_status j2k_fail(j2k_ctx* ctx, j2k_status s, const std::string& msg);
j2k_status j2k_cuda_check(j2k_ctx* ctx, cudaError_t e, const char* what);
void* j2k_scratch(j2k_ctx* ctx, int slot, size_t bytes);  // nullptr on failure (error set)
void* j2k_pinned(j2k_ctx* ctx, size_t bytes);
j2k_status j2k_read_device_error(j2k_ctx* ctx);             // syncs the stream
j2k_status j2k_clear_device_error(j2k_ctx* ctx);

#define J2K_TRY(x)                              \
    do {                                        \
        j2k_status _s = (x);                    \
        if (_s != J2K_OK) return _s;            \
    } while (0)
#define J2K_CUDA(ctx, call) J2K_TRY(j2k_cuda_check((ctx), (call), #call))

// ---- geometry -------------------------------------------------------------------------------
struct j2k_band_rect {
    size_t x0, y0, w, h;
    int orient, level;
};
int j2k_band_rects(size_t w, size_t h, int levels, j2k_band_rect* out);  // returns 3L+1

// code-block job for the tier-1 kernels (device side)
struct j2k_cb_job {
    uint64_t off;      // element offset of the block's first sample from the coefficient base
    uint32_t pitch;    // row pitch of its plane (elements)
    uint16_t cw, ch;
    uint8_t orient, band;
    uint16_t comp;
    uint16_t px0, py0; // position within the component's Mallat plane
    uint32_t image;    // image index (batched encoder), 0 otherwise
    uint32_t out_cap;  // codeword capacity (bytes, multiple of 16)
    uint32_t sym_cap;  // symbol-stream capacity (bytes, multiple of 16)
    uint64_t out_off;  // codeword byte offset in the output buffer (16-aligned)
    uint64_t sym_off;  // symbol-stream byte offset in the scratch buffer (16-aligned)
};
// Fills out/sym offsets of jobs[first..] uniformly (block i at i*cap) or, when per_sample
// factors are given, proportionally to block area.  Returns total (out, sym) bytes.
void j2k_assign_capacities(std::vector<j2k_cb_job>& jobs, size_t first, size_t out_cap, size_t sym_cap,
                           size_t* out_total, size_t* sym_total);
// Appends the jobs of one component plane, whose sample (0,0) sits at element `base` of the
// coefficient buffer with row pitch `pitch`, to *jobs.
size_t j2k_build_jobs(size_t w, size_t h, int levels, int cbw, int cbh, std::vector<j2k_cb_job>* jobs,
                      int comp = 0, uint64_t base = 0, size_t pitch = 0, uint32_t image = 0);

// ---- launchers (defined in the .cu files) ---------------------------------------------------
j2k_status j2k_launch_planar_fwd(j2k_ctx* ctx, const uint8_t* in, size_t in_pitch, int ncomp,
                                 int mct, int out_dtype, void* planes, size_t plane_pitch,
                                 size_t plane_stride, size_t w, size_t h, cudaStream_t st);
j2k_status j2k_launch_planar_inv(j2k_ctx* ctx, const void* planes, int in_dtype,
                                 size_t plane_pitch, size_t plane_stride, int ncomp, int mct,
                                 uint8_t* out, size_t out_pitch, size_t w, size_t h,
                                 cudaStream_t st);
j2k_status j2k_launch_cast_planes(j2k_ctx* ctx, const void* src, int src_dtype, void* dst,
                                  int dst_dtype, size_t n, cudaStream_t st);
j2k_status j2k_launch_mct_planes(j2k_ctx* ctx, void* planes, int dtype, size_t plane_stride,
                                 size_t n, int mct, cudaStream_t st);

// one image of a batched planar split
struct j2k_batch_planar_desc {
    uint64_t in_off;     // byte offset of the interleaved pixels in the input buffer
    uint64_t plane_off;  // element offset of plane 0 in the plane buffer
    uint64_t stride;     // elements between planes (16-aligned)
    uint64_t n;          // pixels
    int ncomp, mct;
};
j2k_status j2k_launch_planar_batched(j2k_ctx* ctx, const j2k_batch_planar_desc* d_descs, const uint2* d_work,
                                     unsigned nwork, const uint8_t* in_base, void* plane_base, int float_out,
                                     cudaStream_t st);

struct j2k_dwt_tile { int tw, th; };
// one image at one decomposition level, for the batched forward DWT
struct j2k_dwt_level_desc {
    const void* src;    // level input (w x h)
    void* ll_dst;       // LL output (unless flags & 2)
    void* dst;          // full coefficient plane (Mallat positions)
    size_t spitch, llpitch, dpitch;
    int w, h;
    float s_ll, s_hl, s_lh, s_hh;  // quantiser steps (9/7)
    int flags;          // 1: quantise details (9/7), 2: this is the last level (LL quantised into dst),
                        // 4: dst and ll_dst take 8-byte vector stores
    int tiles_x;
    uint32_t tile0;     // first flattened tile index of this image
};
j2k_status j2k_dwt_fwd_batched_launch(j2k_ctx* ctx, int kernel, int order, j2k_dwt_tile tile,
                                      const j2k_dwt_level_desc* d_descs, const uint32_t* d_owner,
                                      unsigned ntiles, cudaStream_t st);
// n images at element strides in_z / out_z (blockIdx.z); the LL scratch holds n images at
// strides ceil(w/2)*ceil(h/2) (ll0) and ceil(w/4)*ceil(h/4) (ll1).
j2k_status j2k_dwt_fwd_impl(j2k_ctx* ctx, int kernel, int order, const void* in, size_t in_pitch,
                            void* out, size_t out_pitch, size_t w, size_t h, int levels,
                            const float* steps, void* ll0, void* ll1, j2k_dwt_tile tile,
                            cudaStream_t st, int n = 1, size_t in_z = 0, size_t out_z = 0);
// Level 0 of ncomp (1 or 3) components read straight from interleaved 8-bit pixels, the colour
// transform (mct) inside the level's loads; T.800 order.  Component c's subbands go to
// out + c * out_z (Mallat positions), its LL band to ll + c * ll_z, or into out when levels == 1
// (quantised when steps are given).  _ok tells whether a shape and transform pair is supported.
bool j2k_dwt_fwd_px_ok(int kernel, int ncomp, int mct, size_t w, size_t h);
j2k_status j2k_dwt_fwd_px_launch(j2k_ctx* ctx, int kernel, int ncomp, int mct, const uint8_t* px, size_t pitch,
                                 size_t w, size_t h, int levels, const float* steps, void* ll, size_t llpitch,
                                 size_t ll_z, void* out, size_t out_pitch, size_t out_z, cudaStream_t stream);
j2k_status j2k_dwt_inv_impl(j2k_ctx* ctx, int kernel, int order, const void* in, size_t in_pitch,
                            void* out, size_t out_pitch, size_t w, size_t h, int levels,
                            const float* steps, void* ll0, void* ll1, j2k_dwt_tile tile,
                            cudaStream_t st, int n = 1, size_t in_z = 0, size_t out_z = 0);

// Tier-1 encode of njobs blocks.  order (device, optional): phase-A processing order (largest
// first); sym_bytes: size of the symbol scratch the jobs' sym_off/sym_cap address.
// plane_bytes (njobs x 32) and dist (njobs x 33), both device, optional: when given, the MQ coder
// records the bytes produced at every bit-plane end and the distortion of every truncation point
// is computed (rate control).
// style: code-block style bits (J2K_CBLK_*; 0 = none).  With a style, pass_ends (device,
// J2K_PASS_STRIDE entries per job) receives each pass's end in codeword bytes (exact where the
// pass is terminated); rate control (plane_bytes, dist) is not combined with a style.
j2k_status j2k_t1_encode_jobs(j2k_ctx* ctx, const int32_t* coeff, const j2k_cb_job* d_jobs, size_t njobs,
                              j2k_cb_desc* descs, uint8_t* bytes, size_t sym_bytes,
                              const uint32_t* d_order, cudaStream_t st, uint32_t* plane_bytes = nullptr,
                              double* dist = nullptr, int style = 0, uint32_t* pass_ends = nullptr);
// Code-block style rules (T.800 Table A.19, D.6), host and device: pass `p` (0 = the first
// cleanup pass) is raw-coded, and the codeword is terminated after pass p of npasses.
__host__ __device__ __forceinline__ bool j2k_pass_raw(int style, int p) {
    return (style & J2K_CBLK_BYPASS) && p >= 10 && p % 3 != 0;
}
__host__ __device__ __forceinline__ bool j2k_pass_terminated(int style, int p, int npasses) {
    if (p >= npasses - 1 || (style & J2K_CBLK_TERMALL)) return true;
    return j2k_pass_raw(style, p) != j2k_pass_raw(style, p + 1);
}

// ---- rate control (PCRD-opt, rate.cpp) -----------------------------------------------------
// Squared-norm gain of the synthesis basis of subband b (QCD order) for the 5/3 or 9/7 inverse
// with `levels` levels: an error e in that band's coefficients costs gain * e^2 in the image.
double j2k_band_gain(int kernel, int levels, int band);
// Truncation choice per code-block for a codeword budget: for block i (numbps nb, codeword
// length len, bit-plane byte positions pb[32], distortions d[33] as from the tier-1 rate path,
// weight w = band gain (* step^2 when lossy)), picks npasses in {0, 1, 4, ..., 3nb-2} and the
// kept length so that the total kept bytes stay within budget and the weighted distortion is
// as low as the convex hulls allow.  Writes descs[i].npasses and descs[i].length.
extern "C" j2k_status j2k_pcrd_truncate(j2k_cb_desc* descs, size_t n, const uint32_t* plane_bytes,
                                        const double* dist, const double* weight, size_t budget);
// The same choice split in three, for callers that try several budgets on one set of blocks:
// build() makes every block's lower convex hull (the budget plays no part), threshold(budget)
// finds the slope below which hull segments are dropped, cut(thr) writes each block's kept
// passes and length.  j2k_pcrd_truncate = build + threshold + cut.
struct j2k_pcrd_hulls {
    struct Seg {
        uint64_t key;  // slope (weighted error drop per byte) as the bits of a positive double
        double dl;     // extra bytes
    };
    size_t n = 0, nseg = 0;
    std::vector<double> L, D;    // block i's hull points in slots [i * 33, i * 33 + cnt[i])
    std::vector<uint8_t> N;      // passes kept at each hull point
    std::vector<uint64_t> S;     // slot q > 0: slope key of the segment from point q - 1 to q
    std::vector<int> cnt;
    std::vector<Seg> cand;       // selection scratch
    double base = 0.0, all = 0.0;  // bytes at every hull's first point; at every last point
    void build(const j2k_cb_desc* descs, size_t n, const uint32_t* plane_bytes, const double* dist,
               const double* weight);
    double threshold(size_t budget);
    void cut(double thr, int32_t* npasses, int32_t* length) const;
};
constexpr int J2K_TRUNC_EXTRA = 4;  // bytes kept beyond those produced at a plane end
// style / pass_ends (device, J2K_PASS_STRIDE per job) locate the codeword segments of styled
// blocks; style 0 decodes one segment of descs[i].length bytes.  job_style (device, one byte per
// job, optional) gives each job its own style (pass ends then needed for every job).
j2k_status j2k_t1_decode_jobs(j2k_ctx* ctx, const j2k_cb_desc* descs, const uint8_t* bytes,
                              const j2k_cb_job* d_jobs, size_t njobs, int32_t* coeff,
                              cudaStream_t st, int style = 0, const uint32_t* pass_ends = nullptr,
                              const uint8_t* job_style = nullptr);

// Expounded quantisation (T.800 A.6.4, E.1.1) for 8-bit samples: step = 2^(Rb - eps) *
// (1 + mant / 2^11), Rb = 8 + the gain of QCD band `band` (0 for LL, 1 for HL and LH, 2 for HH).
// Writes the 5-bit exponent and the 11-bit mantissa of `step`, the mantissa rounded to nearest (a
// carry out of it moves to the exponent); false when the step is not a positive finite number or
// its exponent falls outside 0..31.
bool j2k_qcd_step(float step, int band, int* eps, int* mant);

// host tier-2 writer
struct j2k_t2_block {
    int numbps, npasses, length;
    const uint8_t* data;
    const uint32_t* pass_end = nullptr;  // styled blocks: J2K_PASS_STRIDE pass ends
};
// style: the code-block style written in COD; styled blocks' segments (one per terminated pass)
// get a length each in the packet headers.
std::vector<uint8_t> j2k_t2_write(size_t w, size_t h, int ncomp, int levels, int cbw, int cbh,
                                  int lossless, int mct, const float* steps,
                                  const std::vector<j2k_t2_block>& blocks, int style = 0);
// Parses a codestream (the first max_layers quality layers, 0: all) into descriptors in job order
// and the codewords packed back to back (descs[i].offset into bytes).
j2k_status j2k_t2_parse_packed(const uint8_t* cs, size_t n, int max_layers, j2k_stream_info* info,
                               std::vector<j2k_cb_desc>* descs, std::vector<uint8_t>* bytes, std::string* err,
                               std::vector<uint32_t>* pass_ends = nullptr);
// Size in bytes of the codestream j2k_t2_write would produce (block data is not read).
size_t j2k_t2_size(size_t w, size_t h, int ncomp, int levels, int cbw, int cbh, int lossless, int mct,
                   const float* steps, const std::vector<j2k_t2_block>& blocks, int nlayers = 1,
                   const int32_t* cum_np = nullptr, const int32_t* cum_len = nullptr);
// Quality layers: after layer l block i holds cum_np[l * n + i] passes and the first
// cum_len[l * n + i] bytes of blocks[i].data (both non-decreasing in l).
std::vector<uint8_t> j2k_t2_write_layers(size_t w, size_t h, int ncomp, int levels, int cbw, int cbh,
                                         int lossless, int mct, const float* steps,
                                         const std::vector<j2k_t2_block>& blocks, int nlayers,
                                         const int32_t* cum_np, const int32_t* cum_len);
