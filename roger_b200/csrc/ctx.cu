// Context, error handling, scratch memory and subband / code-block geometry.
// Replaces the reference's OCLDeviceManager (src/OCLDeviceManager.cpp:33-90), the queue
// (src/OCLQueue.cpp) and the image allocations of OCLMemoryManager
// (src/OCLMemoryManager.cpp:56-148) with one CUDA stream and grow-only device buffers.
#include <cstdio>
#include <cstring>
#include <new>

#include "j2k_internal.cuh"

j2k_status j2k_fail(j2k_ctx* ctx, j2k_status s, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return s;
}

j2k_status j2k_cuda_check(j2k_ctx* ctx, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return J2K_OK;
    char buf[512];
    snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    return j2k_fail(ctx, e == cudaErrorMemoryAllocation ? J2K_ERR_OUT_OF_MEMORY : J2K_ERR_CUDA,
                    buf);
}

void* j2k_scratch(j2k_ctx* ctx, int slot, size_t bytes) {
    if (bytes == 0) bytes = 256;
    if (ctx->scratch_size[slot] >= bytes) return ctx->scratch[slot];
    if (ctx->scratch[slot]) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->scratch[slot]);
        ctx->scratch[slot] = nullptr;
        ctx->scratch_size[slot] = 0;
    }
    size_t want = bytes + bytes / 4;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        j2k_cuda_check(ctx, e, "cudaMalloc(scratch)");
        return nullptr;
    }
    ctx->scratch[slot] = p;
    ctx->scratch_size[slot] = want;
    return p;
}

void* j2k_pinned(j2k_ctx* ctx, size_t bytes) {
    if (ctx->h_pinned_size >= bytes) return ctx->h_pinned;
    if (ctx->h_pinned) {
        cudaStreamSynchronize(ctx->stream);
        cudaFreeHost(ctx->h_pinned);
        ctx->h_pinned = nullptr;
        ctx->h_pinned_size = 0;
    }
    void* p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) {
        j2k_fail(ctx, J2K_ERR_OUT_OF_MEMORY, "cudaMallocHost(staging) failed");
        return nullptr;
    }
    ctx->h_pinned = p;
    ctx->h_pinned_size = bytes;
    return p;
}

j2k_status j2k_clear_device_error(j2k_ctx* ctx) {
    J2K_CUDA(ctx, cudaMemsetAsync(ctx->d_err, 0, sizeof(uint32_t), ctx->stream));
    return J2K_OK;
}

j2k_status j2k_read_device_error(j2k_ctx* ctx) {
    uint32_t v = 0;
    J2K_CUDA(ctx, cudaMemcpyAsync(&v, ctx->d_err, sizeof v, cudaMemcpyDeviceToHost, ctx->stream));
    J2K_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    switch (v) {
        case J2K_DEVERR_NONE: return J2K_OK;
        case J2K_DEVERR_SYM_CAPACITY:
            return j2k_fail(ctx, J2K_ERR_CAPACITY, "tier-1 symbol buffer of a code-block is full");
        case J2K_DEVERR_OUT_CAPACITY:
            return j2k_fail(ctx, J2K_ERR_CAPACITY, "code-block codeword exceeds cap_per_block");
        case J2K_DEVERR_BAD_JOB:
            return j2k_fail(ctx, J2K_ERR_DEVICE, "malformed code-block descriptor");
        case J2K_DEVERR_TIMEOUT:
            return j2k_fail(ctx, J2K_ERR_TIMEOUT, "bounded device wait expired");
        case J2K_DEVERR_PLANES:
            return j2k_fail(ctx, J2K_ERR_UNSUPPORTED, "more than 31 magnitude bit-planes");
        case J2K_DEVERR_SEG_CAPACITY:
            return j2k_fail(ctx, J2K_ERR_CAPACITY, "a coding-pass segment outgrew its slot");
        default: return j2k_fail(ctx, J2K_ERR_DEVICE, "device error word " + std::to_string(v));
    }
}

int j2k_band_rects(size_t w, size_t h, int levels, j2k_band_rect* out) {
    size_t ws[40], hs[40];
    ws[0] = w;
    hs[0] = h;
    for (int k = 1; k <= levels; ++k) {
        ws[k] = (ws[k - 1] + 1) / 2;
        hs[k] = (hs[k - 1] + 1) / 2;
    }
    out[0] = {0, 0, ws[levels], hs[levels], J2K_BAND_LL, levels};
    int b = 1;
    for (int k = levels; k >= 1; --k) {
        size_t lw = ws[k], lh = hs[k], pw = ws[k - 1], ph = hs[k - 1];
        out[b++] = {lw, 0, pw - lw, lh, J2K_BAND_HL, k};
        out[b++] = {0, lh, lw, ph - lh, J2K_BAND_LH, k};
        out[b++] = {lw, lh, pw - lw, ph - lh, J2K_BAND_HH, k};
    }
    return b;
}

size_t j2k_build_jobs(size_t w, size_t h, int levels, int cbw, int cbh,
                      std::vector<j2k_cb_job>* jobs, int comp, uint64_t base, size_t pitch, uint32_t image) {
    j2k_band_rect r[3 * 32 + 1];
    int nb = j2k_band_rects(w, h, levels, r);
    if (pitch == 0) pitch = w;
    size_t n = 0;
    for (int b = 0; b < nb; ++b) {
        if (!r[b].w || !r[b].h) continue;
        for (size_t y = 0; y < r[b].h; y += (size_t)cbh)
            for (size_t x = 0; x < r[b].w; x += (size_t)cbw) {
                if (jobs) {
                    j2k_cb_job j;
                    const size_t px = r[b].x0 + x, py = r[b].y0 + y;
                    j.off = base + (uint64_t)py * pitch + px;
                    j.pitch = (uint32_t)pitch;
                    j.px0 = (uint16_t)px;
                    j.py0 = (uint16_t)py;
                    j.comp = (uint16_t)comp;
                    j.image = image;
                    j.cw = (uint16_t)(r[b].w - x < (size_t)cbw ? r[b].w - x : (size_t)cbw);
                    j.ch = (uint16_t)(r[b].h - y < (size_t)cbh ? r[b].h - y : (size_t)cbh);
                    j.orient = (uint8_t)r[b].orient;
                    j.band = (uint8_t)b;
                    jobs->push_back(j);
                }
                ++n;
            }
    }
    return n;
}

void j2k_assign_capacities(std::vector<j2k_cb_job>& jobs, size_t first, size_t out_cap, size_t sym_cap,
                           size_t* out_total, size_t* sym_total) {
    uint64_t o = 0, y = 0;
    for (size_t i = first; i < jobs.size(); ++i) {
        j2k_cb_job& j = jobs[i];
        j.out_cap = (uint32_t)out_cap;
        j.sym_cap = (uint32_t)sym_cap;
        j.out_off = o;
        j.sym_off = y;
        o += out_cap;
        y += sym_cap;
    }
    if (out_total) *out_total = o;
    if (sym_total) *sym_total = y;
}

static bool valid_cb(int v) { return v >= 4 && v <= 64 && (v & (v - 1)) == 0; }

extern "C" {

int j2k_version(void) { return 1; }

const char* j2k_status_string(j2k_status s) {
    switch (s) {
        case J2K_OK: return "ok";
        case J2K_ERR_INVALID_ARG: return "invalid argument";
        case J2K_ERR_CUDA: return "CUDA error";
        case J2K_ERR_OUT_OF_MEMORY: return "out of memory";
        case J2K_ERR_DEVICE: return "device-reported error";
        case J2K_ERR_CAPACITY: return "output capacity exceeded";
        case J2K_ERR_UNSUPPORTED: return "unsupported";
        case J2K_ERR_TIMEOUT: return "device wait timed out";
        case J2K_ERR_HOST: return "host error";
        default: return "unknown status";
    }
}

j2k_status j2k_ctx_create(int device, j2k_ctx** out) {
    J2K_API_BEGIN
    if (!out) return J2K_ERR_INVALID_ARG;
    *out = nullptr;
    j2k_ctx* c = new (std::nothrow) j2k_ctx();
    if (!c) return J2K_ERR_OUT_OF_MEMORY;
    c->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_err, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(c->d_err, 0, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) {
        if (c->own_stream) cudaStreamDestroy(c->own_stream);
        if (c->d_err) cudaFree(c->d_err);
        delete c;
        return J2K_ERR_CUDA;
    }
    c->stream = c->own_stream;
    // MQ schedule (longest blocks first): one warp per SM with one block each, two warps per SM
    // with four blocks each, then 16 blocks per warp
    c->mq_tier_warps[0] = c->sm_count;
    c->mq_tier_lanes[0] = 1;
    c->mq_tier_warps[1] = 2 * c->sm_count;
    c->mq_tier_lanes[1] = 4;
    c->mq_lanes = 16;
    *out = c;
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_ctx_destroy(j2k_ctx* ctx) {
    J2K_API_BEGIN
    if (!ctx) return J2K_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (int i = 0; i < J2K_SCRATCH_SLOTS; ++i)
        if (ctx->scratch[i]) cudaFree(ctx->scratch[i]);
    if (ctx->d_err) cudaFree(ctx->d_err);
    if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_ctx_set_stream(j2k_ctx* ctx, void* s) {
    J2K_API_BEGIN
    if (!ctx) return J2K_ERR_INVALID_ARG;
    ctx->stream = (cudaStream_t)s;  // NULL is the CUDA legacy default stream
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_ctx_use_own_stream(j2k_ctx* ctx) {
    J2K_API_BEGIN
    if (!ctx) return J2K_ERR_INVALID_ARG;
    ctx->stream = ctx->own_stream;
    return J2K_OK;
    J2K_API_END
}

void* j2k_ctx_stream(j2k_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

j2k_status j2k_stream_sync(j2k_ctx* ctx) {
    J2K_API_BEGIN
    if (!ctx) return J2K_ERR_INVALID_ARG;
    J2K_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_ctx_set_tuning(j2k_ctx* ctx, int key, int value) {
    J2K_API_BEGIN
    if (!ctx) return J2K_ERR_INVALID_ARG;
    if (key == J2K_TUNE_MQ_LANES) {
        if (value != 8 && value != 16 && value != 32)
            return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "MQ lanes per warp must be 8, 16 or 32");
        ctx->mq_lanes = value;
        return J2K_OK;
    }
    if (key == J2K_TUNE_MQ_VARIANT) {
        if (value != 0 && value != 1) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "MQ variant must be 0 or 1");
        ctx->mq_variant = value;
        return J2K_OK;
    }
    if (key == J2K_TUNE_DWT_FAST_TH) {
        if (value != 0 && value != 16 && value != 32)
            return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "fast DWT tile height must be 0, 16 or 32");
        ctx->dwt_fast_th = value;
        return J2K_OK;
    }
    if (key == J2K_TUNE_DWT_PIPE) {
        ctx->dwt_pipe = value != 0;
        return J2K_OK;
    }
    if (key == J2K_TUNE_DWT_REG) {
        ctx->dwt_reg = value != 0;
        return J2K_OK;
    }
    if (key == J2K_TUNE_DWT_TMA) {
        ctx->dwt_tma = value != 0;
        return J2K_OK;
    }
    if (key == J2K_TUNE_DWT_TAIL) {
        if (value < 0 || value > 5) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "DWT tail form must be 0..5");
        ctx->dwt_tail = value;
        return J2K_OK;
    }
    if (key == J2K_TUNE_T1D_LANES) {
        if (value != 0 && value != 2 && value != 3 && value != 4 && value != 6 && value != 8 && value != 16 &&
            value != 32)
            return j2k_fail(ctx, J2K_ERR_INVALID_ARG,
                            "tier-1 decoder blocks per warp must be 0, 2, 3, 4, 6, 8, 16 or 32");
        ctx->t1d_lanes = value;
        return J2K_OK;
    }
    if (key == J2K_TUNE_PLANAR) {
        if (value < 0 || value > 2) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "planar form must be 0, 1 or 2");
        ctx->planar_form = value;
        return J2K_OK;
    }
    if (key == J2K_TUNE_DWT_PX) {
        ctx->dwt_px = value != 0;
        return J2K_OK;
    }
    if (key == J2K_TUNE_T1D_ORDER) {
        ctx->t1d_order = value != 0;
        return J2K_OK;
    }
    if (key == J2K_TUNE_DWT97_ROWS) {
        ctx->dwt97_rows = value != 0;
        return J2K_OK;
    }
    if (key == J2K_TUNE_T1D_STEPS) {
        ctx->t1d_steps = value != 0;
        return J2K_OK;
    }
    if (key == J2K_TUNE_T1A_CTAS) {
        if (value != 2 && value != 3) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "phase-A CTAs per SM must be 2 or 3");
        ctx->t1a_ctas = value;
        return J2K_OK;
    }
    if (key == J2K_TUNE_MQ_TIER) {
        const int tier = (value >> 24) & 0x7F, lanes = (value >> 20) & 15, warps = value & 0xFFFFF;
        if (tier >= J2K_MQ_TIERS || lanes > 8 || value < 0)
            return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "MQ tier: tier 0..3, lanes 0..8");
        ctx->mq_tier_warps[tier] = lanes ? warps : 0;
        ctx->mq_tier_lanes[tier] = lanes;
        return J2K_OK;
    }
    return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "unknown tuning key");
    J2K_API_END
}

const char* j2k_last_error(const j2k_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

size_t j2k_codeblock_count(size_t w, size_t h, int levels, int cbw, int cbh) {
    if (!w || !h || levels < 0 || levels > 32 || !valid_cb(cbw) || !valid_cb(cbh)) return 0;
    return j2k_build_jobs(w, h, levels, cbw, cbh, nullptr);
}

j2k_status j2k_rgb_to_planar(j2k_ctx* ctx, const uint8_t* in, size_t in_pitch, int ncomp, int mct,
                             int out_dtype, void* planes, size_t plane_pitch, size_t plane_stride,
                             size_t w, size_t h) {
    J2K_API_BEGIN
    if (!ctx) return J2K_ERR_INVALID_ARG;
    if (!in || !planes || ncomp < 1 || ncomp > 4 || w == 0 || h == 0)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "rgb_to_planar: bad pointer/ncomp/size");
    if (in_pitch < w * (size_t)ncomp || plane_pitch < w || plane_stride < plane_pitch * h)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "rgb_to_planar: pitch too small");
    if (out_dtype != J2K_I32 && out_dtype != J2K_F32)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "rgb_to_planar: out_dtype must be I32 or F32");
    if ((mct == J2K_MCT_RCT && out_dtype != J2K_I32) || (mct == J2K_MCT_ICT && out_dtype != J2K_F32) ||
        mct < 0 || mct > 2 || (mct != J2K_MCT_NONE && ncomp < 3))
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "rgb_to_planar: mct/dtype/ncomp mismatch");
    cudaSetDevice(ctx->device);
    return j2k_launch_planar_fwd(ctx, in, in_pitch, ncomp, mct, out_dtype, planes, plane_pitch,
                                 plane_stride, w, h, ctx->stream);
    J2K_API_END
}

j2k_status j2k_planar_to_rgb(j2k_ctx* ctx, const void* planes, int in_dtype, size_t plane_pitch,
                             size_t plane_stride, int ncomp, int mct, uint8_t* out,
                             size_t out_pitch, size_t w, size_t h) {
    J2K_API_BEGIN
    if (!ctx) return J2K_ERR_INVALID_ARG;
    if (!out || !planes || ncomp < 1 || ncomp > 4 || w == 0 || h == 0)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "planar_to_rgb: bad pointer/ncomp/size");
    if (out_pitch < w * (size_t)ncomp || plane_pitch < w || plane_stride < plane_pitch * h)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "planar_to_rgb: pitch too small");
    if ((in_dtype != J2K_I32 && in_dtype != J2K_F32) ||
        (mct == J2K_MCT_RCT && in_dtype != J2K_I32) || (mct == J2K_MCT_ICT && in_dtype != J2K_F32) ||
        mct < 0 || mct > 2 || (mct != J2K_MCT_NONE && ncomp < 3))
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "planar_to_rgb: mct/dtype/ncomp mismatch");
    cudaSetDevice(ctx->device);
    return j2k_launch_planar_inv(ctx, planes, in_dtype, plane_pitch, plane_stride, ncomp, mct, out,
                                 out_pitch, w, h, ctx->stream);
    J2K_API_END
}

static j2k_status check_dwt_args(j2k_ctx* ctx, int kernel, int order, const void* in,
                                 size_t in_pitch, void* out, size_t out_pitch, size_t w, size_t h,
                                 int levels) {
    if (!in || !out || w == 0 || h == 0 || in_pitch < w || out_pitch < w)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "dwt: bad pointer, size or pitch");
    if (kernel != J2K_W53 && kernel != J2K_W97)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "dwt: kernel must be 53 or 97");
    if (order != J2K_ORDER_T800 && order != J2K_ORDER_REF)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "dwt: bad order");
    if (levels < 0 || levels > 32)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "dwt: levels must be in 0..32");
    if (w > 0x7FFFFFFF || h > 0x7FFFFFFF)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "dwt: dimension too large");
    return J2K_OK;
}

j2k_status j2k_dwt_forward(j2k_ctx* ctx, int kernel, int order, const void* in, size_t in_pitch,
                           void* out, size_t out_pitch, size_t w, size_t h, int levels,
                           const float* steps) {
    J2K_API_BEGIN
    if (!ctx) return J2K_ERR_INVALID_ARG;
    J2K_TRY(check_dwt_args(ctx, kernel, order, in, in_pitch, out, out_pitch, w, h, levels));
    if (kernel == J2K_W53 && steps)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "dwt: the 5/3 path is not quantised");
    cudaSetDevice(ctx->device);
    size_t w1 = (w + 1) / 2, h1 = (h + 1) / 2, w2 = (w1 + 1) / 2, h2 = (h1 + 1) / 2;
    void* ll0 = j2k_scratch(ctx, SCR_LL0, w1 * h1 * 4);
    void* ll1 = j2k_scratch(ctx, SCR_LL1, w2 * h2 * 4);
    if (!ll0 || !ll1) return J2K_ERR_OUT_OF_MEMORY;
    return j2k_dwt_fwd_impl(ctx, kernel, order, in, in_pitch, out, out_pitch, w, h, levels, steps,
                            ll0, ll1, j2k_dwt_tile{64, 64}, ctx->stream);
    J2K_API_END
}

j2k_status j2k_dwt_inverse(j2k_ctx* ctx, int kernel, int order, const void* in, size_t in_pitch,
                           void* out, size_t out_pitch, size_t w, size_t h, int levels,
                           const float* steps) {
    J2K_API_BEGIN
    if (!ctx) return J2K_ERR_INVALID_ARG;
    J2K_TRY(check_dwt_args(ctx, kernel, order, in, in_pitch, out, out_pitch, w, h, levels));
    if (kernel == J2K_W53 && steps)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "dwt: the 5/3 path is not quantised");
    cudaSetDevice(ctx->device);
    size_t w1 = (w + 1) / 2, h1 = (h + 1) / 2, w2 = (w1 + 1) / 2, h2 = (h1 + 1) / 2;
    void* ll0 = j2k_scratch(ctx, SCR_LL0, w1 * h1 * 4);
    void* ll1 = j2k_scratch(ctx, SCR_LL1, w2 * h2 * 4);
    if (!ll0 || !ll1) return J2K_ERR_OUT_OF_MEMORY;
    return j2k_dwt_inv_impl(ctx, kernel, order, in, in_pitch, out, out_pitch, w, h, levels, steps,
                            ll0, ll1, j2k_dwt_tile{64, 64}, ctx->stream);
    J2K_API_END
}

}  // extern "C"

extern "C" j2k_status j2k_dwt_forward_batch(j2k_ctx* ctx, int kernel, int order, const void* in, size_t in_pitch,
                                            size_t in_stride, void* out, size_t out_pitch, size_t out_stride,
                                            int n, size_t w, size_t h, int levels, const float* steps) {
    J2K_API_BEGIN
    if (!ctx) return J2K_ERR_INVALID_ARG;
    J2K_TRY(check_dwt_args(ctx, kernel, order, in, in_pitch, out, out_pitch, w, h, levels));
    if (n <= 0 || n > 65535 || in_stride < in_pitch * h || out_stride < out_pitch * h)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "dwt batch: bad image count or plane stride");
    if (kernel == J2K_W53 && steps)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "dwt: the 5/3 path is not quantised");
    cudaSetDevice(ctx->device);
    size_t w1 = (w + 1) / 2, h1 = (h + 1) / 2, w2 = (w1 + 1) / 2, h2 = (h1 + 1) / 2;
    void* ll0 = j2k_scratch(ctx, SCR_LL0, w1 * h1 * 4 * (size_t)n);
    void* ll1 = j2k_scratch(ctx, SCR_LL1, w2 * h2 * 4 * (size_t)n);
    if (!ll0 || !ll1) return J2K_ERR_OUT_OF_MEMORY;
    return j2k_dwt_fwd_impl(ctx, kernel, order, in, in_pitch, out, out_pitch, w, h, levels, steps, ll0, ll1,
                            j2k_dwt_tile{64, 64}, ctx->stream, n, in_stride, out_stride);
    J2K_API_END
}

extern "C" j2k_status j2k_dwt_inverse_batch(j2k_ctx* ctx, int kernel, int order, const void* in, size_t in_pitch,
                                            size_t in_stride, void* out, size_t out_pitch, size_t out_stride,
                                            int n, size_t w, size_t h, int levels, const float* steps) {
    J2K_API_BEGIN
    if (!ctx) return J2K_ERR_INVALID_ARG;
    J2K_TRY(check_dwt_args(ctx, kernel, order, in, in_pitch, out, out_pitch, w, h, levels));
    if (n <= 0 || n > 65535 || in_stride < in_pitch * h || out_stride < out_pitch * h)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "dwt batch: bad image count or plane stride");
    if (kernel == J2K_W53 && steps)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "dwt: the 5/3 path is not quantised");
    cudaSetDevice(ctx->device);
    size_t w1 = (w + 1) / 2, h1 = (h + 1) / 2, w2 = (w1 + 1) / 2, h2 = (h1 + 1) / 2;
    void* ll0 = j2k_scratch(ctx, SCR_LL0, w1 * h1 * 4 * (size_t)n);
    void* ll1 = j2k_scratch(ctx, SCR_LL1, w2 * h2 * 4 * (size_t)n);
    if (!ll0 || !ll1) return J2K_ERR_OUT_OF_MEMORY;
    return j2k_dwt_inv_impl(ctx, kernel, order, in, in_pitch, out, out_pitch, w, h, levels, steps, ll0, ll1,
                            j2k_dwt_tile{64, 64}, ctx->stream, n, in_stride, out_stride);
    J2K_API_END
}
