// Whole-image encoder / decoder objects and the tier-1 ABI entry points.
//
// Reference: OCLEncoder<T>::run (src/OCLEncoder.cpp:43-52: upload -> DWT -> planar -> BPC),
// OCLDecoder<T>::run (src/OCLDecoder.cpp:35-38), OCLEncodeDecode<T>::mapDWTOut/finish
// (src/OCLEncodeDecode.cpp:33-49) and OCLMemoryManager<T>::init/mapImage
// (src/OCLMemoryManager.cpp:56-190).  The B200 pipeline order is upload -> planar+MCT ->
// DWT (+ quantiser) -> tier-1, all on one stream, with every buffer kept resident and grown
// only when a larger image arrives.  Code-block codewords are packed on the device (prefix
// sum of lengths + gather) so a single device->host copy returns them.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <new>
#include <thread>

#include "j2k_internal.cuh"

namespace {

size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }

bool valid_cb(int v) { return v >= 4 && v <= 64 && (v & (v - 1)) == 0; }

struct DevBuf {
    void* p = nullptr;
    size_t n = 0;
    j2k_status ensure(j2k_ctx* ctx, size_t bytes) {
        if (n >= bytes) return J2K_OK;
        if (p) {
            cudaStreamSynchronize(ctx->stream);
            cudaFree(p);
            p = nullptr;
            n = 0;
        }
        J2K_CUDA(ctx, cudaMalloc(&p, bytes));
        n = bytes;
        return J2K_OK;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

// gather each block's codeword (at i*cap) into a packed buffer at out_off[i]
__global__ void pack_kernel(const j2k_cb_desc* __restrict__ descs, const uint32_t* __restrict__ off,
                            const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, int n) {
    int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (wid >= n) return;
    int len = descs[wid].length;
    const uint8_t* s = src + descs[wid].offset;
    uint8_t* d = dst + off[wid];
    for (int k = lane; k < len; k += 32) d[k] = s[k];
}

__global__ void lengths_kernel(const j2k_cb_desc* __restrict__ descs, uint32_t* __restrict__ len, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) len[i] = (uint32_t)max(descs[i].length, 0);
}

std::vector<float> default_steps(size_t w, size_t h, int levels) {
    std::vector<j2k_band_rect> r(3 * levels + 1);
    j2k_band_rects(w, h, levels, r.data());
    std::vector<float> s(r.size());
    for (size_t b = 0; b < r.size(); ++b) s[b] = 8.0f * std::ldexp(1.0f, -r[b].level);
    return s;
}

// Runs fn(k) for k = 0..n-1 on up to 16 host threads (one thread when the work is small), each
// thread taking every nt-th item; used for the copies between callers' buffers and page-locked
// staging, which one thread does at only a few GB/s.
template <typename F>
void host_parallel(int n, size_t bytes, F fn) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int nt = bytes < ((size_t)8 << 20) ? 1 : (int)std::min<unsigned>((unsigned)n, std::min(16u, hw));
    if (nt <= 1) {
        for (int k = 0; k < n; ++k) fn(k);
        return;
    }
    j2k_run_threads(nt, [&](int t) {
        for (int k = t; k < n; k += nt) fn(k);
    });
}

// A host copy split over up to 16 threads when it is large (one thread copies at a few GB/s).
void parallel_copy(void* dst, const void* src, size_t bytes) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int nt = bytes < ((size_t)8 << 20) ? 1 : (int)std::min(16u, hw);
    const size_t chunk = (bytes + nt - 1) / nt;
    host_parallel(nt, bytes, [&](int t) {
        const size_t a = (size_t)t * chunk, b = std::min(bytes, a + chunk);
        if (a < b) std::memcpy((uint8_t*)dst + a, (const uint8_t*)src + a, b - a);
    });
}

// Host memory that the GPU can copy from or to asynchronously (page-locked or registered).
bool page_locked(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

}  // namespace

struct j2k_encoder {
    j2k_ctx* ctx = nullptr;
    int lossy = 0, dwt_only = 0;
    // geometry of the last run
    size_t w = 0, h = 0;
    int ncomp = 0, levels = 0, cbw = 64, cbh = 64, order = J2K_ORDER_T800, mct = 0;
    std::vector<float> steps;
    DevBuf in, planes, coef, jobs, descs, bytes, lens, offs, packed, cubtmp;
    std::vector<j2k_cb_job> hjobs;
    size_t njobs = 0, cap = 0, sym_cap = 0;
    size_t job_key[6] = {0, 0, 0, 0, 0, 0};
    bool have_result = false;
    bool packed_ok = false;  // the packed codewords of the current result are on the device
    size_t packed_total = 0;
    size_t target_bytes = 0;  // rate control: codestream budget (0 = keep every pass)
    int style = 0;            // code-block style of the last run (J2K_CBLK_*)
    DevBuf pass_ends;         // styled runs: J2K_PASS_STRIDE pass ends per job
    // quality layers: cumulative codestream budgets (0 in the last place: every pass), and per
    // layer l and block i the passes / codeword bytes kept after that layer (lay_*[l * n + i])
    std::vector<size_t> layer_budget;
    std::vector<int32_t> lay_np, lay_len;
    DevBuf rate_pb, rate_dist;
    j2k_pcrd_hulls pcrd;  // the blocks' convex hulls of the last rate-controlled encode
    void* mapped = nullptr;
};

struct j2k_decoder {
    j2k_ctx* ctx = nullptr;
    int lossy = 0;
    DevBuf descs, bytes, coef, planes, out, jobs, pass_ends, job_style;
    std::vector<j2k_cb_job> hjobs;
    size_t job_key[6] = {0, 0, 0, 0, 0, 0};
};

static j2k_status prepare_jobs(j2k_ctx* ctx, std::vector<j2k_cb_job>& hjobs, DevBuf& djobs,
                               size_t* key, size_t w, size_t h, int ncomp, int levels, int cbw,
                               int cbh, size_t* njobs) {
    size_t k[6] = {w, h, (size_t)ncomp, (size_t)levels, (size_t)cbw, (size_t)cbh};
    if (std::equal(k, k + 6, key) && !hjobs.empty()) {
        *njobs = hjobs.size();
        return J2K_OK;
    }
    hjobs.clear();
    for (int c = 0; c < ncomp; ++c) j2k_build_jobs(w, h, levels, cbw, cbh, &hjobs, c, (uint64_t)c * w * h, w);
    J2K_TRY(djobs.ensure(ctx, std::max<size_t>(hjobs.size(), 1) * sizeof(j2k_cb_job)));
    J2K_CUDA(ctx, cudaMemcpyAsync(djobs.p, hjobs.data(), hjobs.size() * sizeof(j2k_cb_job),
                                  cudaMemcpyHostToDevice, ctx->stream));
    std::copy(k, k + 6, key);
    *njobs = hjobs.size();
    return J2K_OK;
}

static j2k_status check_params(j2k_ctx* ctx, const j2k_enc_params* p, size_t w, size_t h,
                               int* levels, int* cbw, int* cbh, int* order) {
    *levels = p ? p->levels : 5;
    *cbw = p && p->cbw ? p->cbw : 64;
    *cbh = p && p->cbh ? p->cbh : 64;
    *order = p ? p->order : J2K_ORDER_T800;
    if (*levels < 0 || *levels > 32) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "levels must be in 0..32");
    if (!valid_cb(*cbw) || !valid_cb(*cbh) || *cbw * *cbh > 4096)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "code-block size must be a power of two in 4..64");
    if (*order != J2K_ORDER_T800 && *order != J2K_ORDER_REF)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "bad order");
    if (w == 0 || h == 0 || w > 65535 || h > 65535)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "image size must be in 1..65535");
    if (p && (p->cblk_style < 0 || p->cblk_style > 7))
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "code-block style: BYPASS, RESET and TERMALL bits only");
    return J2K_OK;
}

// DWT of every component + tier-1 of all blocks.  planes: ncomp planes (int32 or float).
// PCRD-opt truncation of the current tier-1 result to the encoder's byte budget: per-block
// bit-plane byte positions and distortions come from the tier-1 rate path; the chosen passes
// and lengths are written back into the device descriptors, which the packing and the
// codestream writer then follow.  The codestream size (headers included) is checked by writing
// its headers, and the codeword budget lowered by any excess.
static j2k_status rate_control(j2k_encoder* e) {
    j2k_ctx* ctx = e->ctx;
    const size_t n = e->njobs;
    // descriptors, plane-end byte counts and distortions through the context's page-locked
    // staging buffer (the input copy it held is complete: the error word was read after it)
    uint8_t* hp = (uint8_t*)j2k_pinned(ctx, n * (33 * 8 + 32 * 4 + sizeof(j2k_cb_desc)) + 64);
    if (!hp) return J2K_ERR_OUT_OF_MEMORY;
    double* dist = (double*)hp;
    uint32_t* pb = (uint32_t*)(dist + n * 33);
    j2k_cb_desc* dh = (j2k_cb_desc*)(pb + n * 32);
    J2K_CUDA(ctx, cudaMemcpyAsync(dh, e->descs.p, n * sizeof(j2k_cb_desc), cudaMemcpyDeviceToHost, ctx->stream));
    J2K_CUDA(ctx, cudaMemcpyAsync(pb, e->rate_pb.p, n * 32 * 4, cudaMemcpyDeviceToHost, ctx->stream));
    J2K_CUDA(ctx, cudaMemcpyAsync(dist, e->rate_dist.p, n * 33 * 8, cudaMemcpyDeviceToHost, ctx->stream));
    J2K_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    const int kernel = e->lossy ? J2K_W97 : J2K_W53;
    const int nb = 3 * e->levels + 1;
    std::vector<double> gain(nb), w(n);
    for (int b = 0; b < nb; ++b) {
        gain[b] = j2k_band_gain(kernel, e->levels, b);
        if (e->lossy) gain[b] *= (double)e->steps[b] * e->steps[b];
    }
    for (size_t i = 0; i < n; ++i) w[i] = gain[e->hjobs[i].band];
    // the blocks' hulls do not depend on the budget: built once for every layer and try
    j2k_pcrd_hulls& hull = e->pcrd;
    hull.build(dh, n, pb, dist, w.data());
    std::vector<j2k_cb_desc> d(n);
    std::vector<j2k_t2_block> blocks(n);
    for (size_t i = 0; i < n; ++i) blocks[i] = j2k_t2_block{dh[i].numbps, 0, 0, nullptr};
    // one layer per budget (a single target_bytes is one layer); each layer keeps at least what
    // the layer before it kept, and its budget is lowered until the codestream of the layers so
    // far (headers included) fits it
    std::vector<size_t> budgets = e->layer_budget;
    if (budgets.empty()) budgets.push_back(e->target_bytes);
    const int L = (int)budgets.size();
    e->lay_np.assign((size_t)L * n, 0);
    e->lay_len.assign((size_t)L * n, 0);
    for (int l = 0; l < L; ++l) {
        int32_t* np = e->lay_np.data() + (size_t)l * n;
        int32_t* ln = e->lay_len.data() + (size_t)l * n;
        const int32_t* pnp = l ? np - n : nullptr;
        const int32_t* pln = l ? ln - n : nullptr;
        if (budgets[l] == 0) {  // the last layer may keep every pass
            for (size_t i = 0; i < n; ++i) np[i] = dh[i].npasses, ln[i] = std::max(dh[i].length, 0);
            continue;
        }
        size_t budget = budgets[l];
        for (int it = 0; it < 24; ++it) {
            hull.cut(hull.threshold(budget), np, ln);
            if (pnp)
                for (size_t i = 0; i < n; ++i)
                    if (np[i] < pnp[i]) np[i] = pnp[i], ln[i] = pln[i];
            const size_t size = j2k_t2_size(e->w, e->h, e->ncomp, e->levels, e->cbw, e->cbh, !e->lossy,
                                            e->mct != J2K_MCT_NONE, e->steps.data(), blocks, l + 1,
                                            e->lay_np.data(), e->lay_len.data());
            if (size <= budgets[l]) break;
            // the headers of a cut differ from those of the one before: lower the codeword
            // budget by the excess, by more on every try, until the codestream fits (with no
            // codeword bytes left it holds headers only)
            const size_t excess = size - budgets[l] + 16 + (size_t)it * it * 8;
            if (budget == 0) break;
            budget = budget > excess ? budget - excess : 0;
        }
    }
    const int32_t* fnp = e->lay_np.data() + (size_t)(L - 1) * n;
    const int32_t* fln = e->lay_len.data() + (size_t)(L - 1) * n;
    for (size_t i = 0; i < n; ++i) {
        d[i] = dh[i];
        d[i].npasses = (uint8_t)fnp[i];
        d[i].length = fnp[i] ? fln[i] : 0;
    }
    if (L == 1) e->lay_np.clear(), e->lay_len.clear();
    std::memcpy(dh, d.data(), n * sizeof(j2k_cb_desc));
    J2K_CUDA(ctx, cudaMemcpyAsync(e->descs.p, dh, n * sizeof(j2k_cb_desc), cudaMemcpyHostToDevice, ctx->stream));
    J2K_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return J2K_OK;
}

static j2k_status run_tier1(j2k_encoder* e);

static j2k_status encode_planes(j2k_encoder* e) {
    j2k_ctx* ctx = e->ctx;
    const size_t n = e->w * e->h;
    const bool quant = e->lossy && !e->dwt_only;
    const size_t csz = 4;
    J2K_TRY(e->coef.ensure(ctx, n * csz * e->ncomp));
    size_t w1 = (e->w + 1) / 2, h1 = (e->h + 1) / 2, w2 = (w1 + 1) / 2, h2 = (h1 + 1) / 2;
    void* ll0 = j2k_scratch(ctx, SCR_LL0, w1 * h1 * 4);
    void* ll1 = j2k_scratch(ctx, SCR_LL1, w2 * h2 * 4);
    if (!ll0 || !ll1) return J2K_ERR_OUT_OF_MEMORY;
    for (int c = 0; c < e->ncomp; ++c) {
        const char* src = (const char*)e->planes.p + (size_t)c * n * 4;
        char* dst = (char*)e->coef.p + (size_t)c * n * csz;
        J2K_TRY(j2k_dwt_fwd_impl(ctx, e->lossy ? J2K_W97 : J2K_W53, e->lossy ? J2K_ORDER_T800 : e->order,
                                 src, e->w, dst, e->w, e->w, e->h, e->levels,
                                 quant ? e->steps.data() : nullptr, ll0, ll1, j2k_dwt_tile{64, 64},
                                 ctx->stream));
    }
    e->have_result = true;
    if (e->dwt_only) return J2K_OK;
    return run_tier1(e);
}

// The first DWT level reads the interleaved pixels itself (the level shift and colour transform
// inside its loads) when J2K_TUNE_DWT_PX asks for it and the level takes the register-lifting tile
// in the T.800 order.
static bool pixels_to_dwt(const j2k_encoder* e) {
    const j2k_ctx* ctx = e->ctx;
    const int order = e->lossy ? J2K_ORDER_T800 : e->order;
    return ctx->dwt_px && order == J2K_ORDER_T800 && e->levels >= 1 && ctx->dwt_fast_th == 16 && ctx->dwt_reg &&
           !ctx->dwt_tma && !ctx->dwt_pipe &&
           j2k_dwt_fwd_px_ok(e->lossy ? J2K_W97 : J2K_W53, e->ncomp, e->mct, e->w, e->h);
}

// Encode from device pixels: level 0 of every component straight from the pixels (their LL
// bands to a scratch buffer), then the remaining levels of all components in one call with the
// components side by side (gridDim.z), then tier-1.  The same coefficients as the planar split
// followed by encode_planes.
static j2k_status encode_pixels(j2k_encoder* e, const uint8_t* px, size_t pitch) {
    j2k_ctx* ctx = e->ctx;
    const size_t n = e->w * e->h;
    const int nc = e->ncomp;
    const bool quant = e->lossy && !e->dwt_only;
    const int kern = e->lossy ? J2K_W97 : J2K_W53;
    J2K_TRY(e->coef.ensure(ctx, n * 4 * nc));
    const size_t w1 = (e->w + 1) / 2, h1 = (e->h + 1) / 2, w2 = (w1 + 1) / 2, h2 = (h1 + 1) / 2;
    const size_t w3 = (w2 + 1) / 2, h3 = (h2 + 1) / 2;
    void* llpx = j2k_scratch(ctx, SCR_LLPX, w1 * h1 * 4 * nc);
    void* ll0 = j2k_scratch(ctx, SCR_LL0, w2 * h2 * 4 * nc);
    void* ll1 = j2k_scratch(ctx, SCR_LL1, w3 * h3 * 4 * nc);
    if (!llpx || !ll0 || !ll1) return J2K_ERR_OUT_OF_MEMORY;
    const float* steps = quant ? e->steps.data() : nullptr;
    J2K_TRY(j2k_dwt_fwd_px_launch(ctx, kern, nc, e->mct, px, pitch, e->w, e->h, e->levels, steps, llpx, w1, w1 * h1,
                                  e->coef.p, e->w, n, ctx->stream));
    if (e->levels > 1)
        J2K_TRY(j2k_dwt_fwd_impl(ctx, kern, J2K_ORDER_T800, llpx, w1, e->coef.p, e->w, w1, h1, e->levels - 1, steps,
                                 ll0, ll1, j2k_dwt_tile{64, 64}, ctx->stream, nc, w1 * h1, n));
    e->have_result = true;
    if (e->dwt_only) return J2K_OK;
    return run_tier1(e);
}

// Tier-1 of every code-block of the current coefficients (and rate control when asked for).
static j2k_status run_tier1(j2k_encoder* e) {
    j2k_ctx* ctx = e->ctx;
    J2K_TRY(prepare_jobs(ctx, e->hjobs, e->jobs, e->job_key, e->w, e->h, e->ncomp, e->levels, e->cbw,
                         e->cbh, &e->njobs));
    const size_t nblk = (size_t)e->cbw * e->cbh;
    if (e->cap == 0) e->cap = align16(nblk * 2 + 256);
    if (e->sym_cap == 0) e->sym_cap = align16(nblk * 20 + 256);
    for (int attempt = 0; attempt < 6; ++attempt) {
        if (e->hjobs.empty() || e->hjobs[0].out_cap != e->cap || e->hjobs[0].sym_cap != e->sym_cap) {
            j2k_assign_capacities(e->hjobs, 0, e->cap, e->sym_cap, nullptr, nullptr);
            J2K_CUDA(ctx, cudaMemcpyAsync(e->jobs.p, e->hjobs.data(), e->hjobs.size() * sizeof(j2k_cb_job),
                                          cudaMemcpyHostToDevice, ctx->stream));
        }
        J2K_TRY(e->descs.ensure(ctx, std::max<size_t>(e->njobs, 1) * sizeof(j2k_cb_desc)));
        J2K_TRY(e->bytes.ensure(ctx, std::max<size_t>(e->njobs, 1) * e->cap));
        J2K_TRY(j2k_clear_device_error(ctx));
        uint32_t* pb = nullptr;
        double* dist = nullptr;
        if (e->target_bytes || !e->layer_budget.empty()) {
            J2K_TRY(e->rate_pb.ensure(ctx, e->njobs * 32 * 4 + 16));
            J2K_TRY(e->rate_dist.ensure(ctx, e->njobs * 33 * 8 + 16));
            pb = (uint32_t*)e->rate_pb.p;
            dist = (double*)e->rate_dist.p;
        }
        uint32_t* pe = nullptr;
        if (e->style) {
            J2K_TRY(e->pass_ends.ensure(ctx, e->njobs * J2K_PASS_STRIDE * 4 + 16));
            pe = (uint32_t*)e->pass_ends.p;
        }
        J2K_TRY(j2k_t1_encode_jobs(ctx, (const int32_t*)e->coef.p, (const j2k_cb_job*)e->jobs.p,
                                   e->njobs, (j2k_cb_desc*)e->descs.p, (uint8_t*)e->bytes.p,
                                   e->njobs * e->sym_cap, nullptr, ctx->stream, pb, dist, e->style, pe));
        j2k_status s = j2k_read_device_error(ctx);
        if (s == J2K_OK) return (e->target_bytes || !e->layer_budget.empty()) ? rate_control(e) : J2K_OK;
        if (s != J2K_ERR_CAPACITY) return s;
        // grow whichever capacity overflowed and retry
        if (ctx->err.find("symbol") != std::string::npos) e->sym_cap = align16(e->sym_cap * 2);
        else if (ctx->err.find("segment") != std::string::npos) ctx->t1_seg_factor *= 2;
        else e->cap = align16(e->cap * 2);
    }
    return j2k_fail(ctx, J2K_ERR_CAPACITY, "tier-1 capacities kept overflowing");
}

// pack codewords on the device: descs[i].offset -> packed offsets; returns total bytes
static j2k_status pack_blocks(j2k_encoder* e, size_t* total) {
    j2k_ctx* ctx = e->ctx;
    if (e->packed_ok) {  // already packed for this result (size query, then copy)
        *total = e->packed_total;
        return J2K_OK;
    }
    int n = (int)e->njobs;
    J2K_TRY(e->lens.ensure(ctx, (size_t)(n + 1) * 4));
    J2K_TRY(e->offs.ensure(ctx, (size_t)(n + 1) * 4));
    lengths_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>((const j2k_cb_desc*)e->descs.p, (uint32_t*)e->lens.p, n);
    J2K_CUDA(ctx, cudaMemsetAsync((uint32_t*)e->lens.p + n, 0, 4, ctx->stream));
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, (uint32_t*)e->lens.p, (uint32_t*)e->offs.p, n + 1, ctx->stream);
    J2K_TRY(e->cubtmp.ensure(ctx, tmp + 16));
    J2K_CUDA(ctx, cub::DeviceScan::ExclusiveSum(e->cubtmp.p, tmp, (uint32_t*)e->lens.p,
                                                (uint32_t*)e->offs.p, n + 1, ctx->stream));
    uint32_t tot = 0;
    J2K_CUDA(ctx, cudaMemcpyAsync(&tot, (uint32_t*)e->offs.p + n, 4, cudaMemcpyDeviceToHost, ctx->stream));
    J2K_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    J2K_TRY(e->packed.ensure(ctx, (size_t)tot + 16));
    pack_kernel<<<(n * 32 + 255) / 256, 256, 0, ctx->stream>>>((const j2k_cb_desc*)e->descs.p,
                                                               (const uint32_t*)e->offs.p,
                                                               (const uint8_t*)e->bytes.p,
                                                               (uint8_t*)e->packed.p, n);
    J2K_CUDA(ctx, cudaGetLastError());
    *total = tot;
    e->packed_total = tot;
    e->packed_ok = true;
    return J2K_OK;
}

extern "C" {

j2k_status j2k_bpc_encode(j2k_ctx* ctx, const int32_t* coeff, size_t pitch, size_t w, size_t h,
                          int levels, int cbw, int cbh, j2k_cb_desc* descs, uint8_t* bytes,
                          size_t cap_per_block) {
    J2K_API_BEGIN
    if (!ctx) return J2K_ERR_INVALID_ARG;
    if (!coeff || !descs || !bytes || pitch < w || w == 0 || h == 0 || w > 65535 || h > 65535)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "bpc_encode: bad pointer/size/pitch");
    if (levels < 0 || levels > 32 || !valid_cb(cbw) || !valid_cb(cbh) || cbw * cbh > 4096)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "bpc_encode: bad levels or code-block size");
    if (cap_per_block == 0 || cap_per_block % 16)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "bpc_encode: cap_per_block must be a positive multiple of 16");
    cudaSetDevice(ctx->device);
    std::vector<j2k_cb_job> jobs;
    j2k_build_jobs(w, h, levels, cbw, cbh, &jobs, 0, 0, pitch);
    j2k_cb_job* dj = (j2k_cb_job*)j2k_scratch(ctx, SCR_JOBS, jobs.size() * sizeof(j2k_cb_job) + 16);
    if (!dj) return J2K_ERR_OUT_OF_MEMORY;
    size_t sym_cap = align16((size_t)cbw * cbh * 20 + 256);
    for (int attempt = 0; attempt < 6; ++attempt) {
        j2k_assign_capacities(jobs, 0, cap_per_block, sym_cap, nullptr, nullptr);
        J2K_CUDA(ctx, cudaMemcpyAsync(dj, jobs.data(), jobs.size() * sizeof(j2k_cb_job), cudaMemcpyHostToDevice, ctx->stream));
        J2K_TRY(j2k_clear_device_error(ctx));
        J2K_TRY(j2k_t1_encode_jobs(ctx, coeff, dj, jobs.size(), descs, bytes, jobs.size() * sym_cap, nullptr,
                                   ctx->stream));
        j2k_status s = j2k_read_device_error(ctx);
        if (s == J2K_OK) return J2K_OK;
        if (s == J2K_ERR_CAPACITY && ctx->err.find("symbol") != std::string::npos) {
            sym_cap = align16(sym_cap * 2);
            continue;
        }
        return s;
    }
    return j2k_fail(ctx, J2K_ERR_CAPACITY, "tier-1 symbol capacity kept overflowing");
    J2K_API_END
}

j2k_status j2k_bpc_decode(j2k_ctx* ctx, const j2k_cb_desc* descs, const uint8_t* bytes,
                          size_t count, int32_t* coeff, size_t pitch, size_t w, size_t h,
                          int levels, int cbw, int cbh) {
    J2K_API_BEGIN
    if (!ctx) return J2K_ERR_INVALID_ARG;
    if (!coeff || !descs || !bytes || pitch < w || w == 0 || h == 0 || w > 65535 || h > 65535)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "bpc_decode: bad pointer/size/pitch");
    if (levels < 0 || levels > 32 || !valid_cb(cbw) || !valid_cb(cbh) || cbw * cbh > 4096)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "bpc_decode: bad levels or code-block size");
    cudaSetDevice(ctx->device);
    std::vector<j2k_cb_job> jobs;
    j2k_build_jobs(w, h, levels, cbw, cbh, &jobs, 0, 0, pitch);
    if (jobs.size() != count)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "bpc_decode: count does not match the partition");
    j2k_cb_job* dj = (j2k_cb_job*)j2k_scratch(ctx, SCR_JOBS, jobs.size() * sizeof(j2k_cb_job) + 16);
    if (!dj) return J2K_ERR_OUT_OF_MEMORY;
    J2K_CUDA(ctx, cudaMemcpyAsync(dj, jobs.data(), jobs.size() * sizeof(j2k_cb_job), cudaMemcpyHostToDevice, ctx->stream));
    J2K_TRY(j2k_clear_device_error(ctx));
    J2K_TRY(j2k_t1_decode_jobs(ctx, descs, bytes, dj, jobs.size(), coeff, ctx->stream));
    return j2k_read_device_error(ctx);
    J2K_API_END
}

j2k_status j2k_encoder_create(j2k_ctx* ctx, int lossy, int output_dwt_only, j2k_encoder** out) {
    J2K_API_BEGIN
    if (!ctx || !out) return J2K_ERR_INVALID_ARG;
    j2k_encoder* e = new (std::nothrow) j2k_encoder();
    if (!e) return J2K_ERR_OUT_OF_MEMORY;
    e->ctx = ctx;
    e->lossy = lossy ? 1 : 0;
    e->dwt_only = output_dwt_only ? 1 : 0;
    *out = e;
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_encoder_destroy(j2k_encoder* e) {
    J2K_API_BEGIN
    if (!e) return J2K_ERR_INVALID_ARG;
    cudaSetDevice(e->ctx->device);
    cudaStreamSynchronize(e->ctx->stream);
    for (DevBuf* b : {&e->in, &e->planes, &e->coef, &e->jobs, &e->descs, &e->bytes, &e->lens, &e->offs,
                      &e->packed, &e->cubtmp})
        b->release();
    if (e->mapped) cudaFreeHost(e->mapped);
    delete e;
    return J2K_OK;
    J2K_API_END
}

static j2k_status setup_run(j2k_encoder* e, int ncomp, size_t w, size_t h, const j2k_enc_params* p) {
    j2k_ctx* ctx = e->ctx;
    int levels, cbw, cbh, order;
    J2K_TRY(check_params(ctx, p, w, h, &levels, &cbw, &cbh, &order));
    if (ncomp != 1 && ncomp != 3)
        return j2k_fail(ctx, J2K_ERR_UNSUPPORTED, "encoder supports 1 or 3 components");
    e->target_bytes = p ? p->target_bytes : 0;
    e->style = p ? p->cblk_style : 0;
    if (e->style && (e->target_bytes || (p && p->layers > 1)))
        return j2k_fail(ctx, J2K_ERR_UNSUPPORTED, "rate control and layers are not combined with a code-block style");
    e->layer_budget.clear();
    e->lay_np.clear();
    e->lay_len.clear();
    if (p && p->layers > 1) {
        if (!p->layer_bytes || p->layers > 64)
            return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "layers > 1 needs layer_bytes (at most 64 layers)");
        for (int l = 0; l < p->layers; ++l) {
            const size_t b = p->layer_bytes[l];
            if (b == 0 && l != p->layers - 1)
                return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "only the last layer budget may be 0 (every pass)");
            if (l && b && b < p->layer_bytes[l - 1])
                return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "layer budgets must not decrease");
            e->layer_budget.push_back(b);
        }
    }
    e->w = w;
    e->h = h;
    e->ncomp = ncomp;
    e->levels = levels;
    e->cbw = cbw;
    e->cbh = cbh;
    e->order = order;
    e->mct = ncomp >= 3 ? (e->lossy ? J2K_MCT_ICT : J2K_MCT_RCT) : J2K_MCT_NONE;
    if (e->lossy) {
        if (p && p->steps) e->steps.assign(p->steps, p->steps + 3 * levels + 1);
        else e->steps = default_steps(w, h, levels);
        for (int b = 0; b < (int)e->steps.size(); ++b) {
            int ex, mt;
            if (!j2k_qcd_step(e->steps[b], b, &ex, &mt))
                return j2k_fail(ctx, J2K_ERR_INVALID_ARG,
                                "quantiser step " + std::to_string(b) + " is not positive or out of the QCD range");
        }
    } else {
        e->steps.clear();
    }
    J2K_TRY(e->planes.ensure(ctx, w * h * 4 * (size_t)ncomp));
    e->have_result = false;
    e->packed_ok = false;
    return J2K_OK;
}

j2k_status j2k_encoder_run_interleaved(j2k_encoder* e, const uint8_t* pixels, int on_device,
                                       size_t pitch, int ncomp, size_t w, size_t h,
                                       const j2k_enc_params* p) {
    J2K_API_BEGIN
    if (!e) return J2K_ERR_INVALID_ARG;
    j2k_ctx* ctx = e->ctx;
    if (!pixels) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "pixels is NULL");
    if (pitch == 0) pitch = w * (size_t)ncomp;
    if (pitch < w * (size_t)ncomp) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "pitch too small");
    cudaSetDevice(ctx->device);
    J2K_TRY(setup_run(e, ncomp, w, h, p));
    const uint8_t* src = pixels;
    if (!on_device) {
        J2K_TRY(e->in.ensure(ctx, pitch * h + 16));
        J2K_CUDA(ctx, cudaMemcpyAsync(e->in.p, pixels, pitch * h, cudaMemcpyHostToDevice, ctx->stream));
        src = (const uint8_t*)e->in.p;
    }
    if (pixels_to_dwt(e)) return encode_pixels(e, src, pitch);
    J2K_TRY(j2k_launch_planar_fwd(ctx, src, pitch, ncomp, e->mct, e->lossy ? J2K_F32 : J2K_I32, e->planes.p,
                                  w, w * h, w, h, ctx->stream));
    return encode_planes(e);
    J2K_API_END
}

j2k_status j2k_encoder_run(j2k_encoder* e, const void* const* comps, int ncomp, int dtype, size_t w,
                           size_t h, size_t levels, size_t precision, const j2k_enc_params* p) {
    J2K_API_BEGIN
    if (!e) return J2K_ERR_INVALID_ARG;
    j2k_ctx* ctx = e->ctx;
    if (!comps) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "components is NULL");
    if (dtype != J2K_I16 && dtype != J2K_I32 && dtype != J2K_F32)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "component dtype must be I16, I32 or F32");
    if (precision != 8) return j2k_fail(ctx, J2K_ERR_UNSUPPORTED, "only 8-bit precision is supported");
    j2k_enc_params q{};
    if (p) q = *p;
    q.levels = (int)levels;
    cudaSetDevice(ctx->device);
    J2K_TRY(setup_run(e, ncomp, w, h, &q));
    const size_t n = w * h, esz = dtype == J2K_I16 ? 2 : 4;
    J2K_TRY(e->in.ensure(ctx, n * esz * ncomp + 16));
    int pd = e->lossy ? J2K_F32 : J2K_I32;
    for (int c = 0; c < ncomp; ++c) {
        if (!comps[c]) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "component pointer is NULL");
        char* staged = (char*)e->in.p + (size_t)c * n * esz;
        J2K_CUDA(ctx, cudaMemcpyAsync(staged, comps[c], n * esz, cudaMemcpyHostToDevice, ctx->stream));
        J2K_TRY(j2k_launch_cast_planes(ctx, staged, dtype, (char*)e->planes.p + (size_t)c * n * 4, pd, n, ctx->stream));
    }
    if (e->mct != J2K_MCT_NONE) J2K_TRY(j2k_launch_mct_planes(ctx, e->planes.p, pd, n, n, e->mct, ctx->stream));
    return encode_planes(e);
    J2K_API_END
}

j2k_status j2k_encoder_map_dwt_out(j2k_encoder* e, void** ptr, size_t* pitch_bytes) {
    J2K_API_BEGIN
    if (!e || !ptr) return J2K_ERR_INVALID_ARG;
    j2k_ctx* ctx = e->ctx;
    if (!e->have_result) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "no encoder run yet");
    size_t bytes = e->w * e->h * 4 * e->ncomp;
    if (!e->mapped) J2K_CUDA(ctx, cudaMallocHost(&e->mapped, bytes));
    J2K_CUDA(ctx, cudaMemcpyAsync(e->mapped, e->coef.p, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    J2K_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *ptr = e->mapped;
    if (pitch_bytes) *pitch_bytes = e->w * 4;
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_encoder_unmap_dwt_out(j2k_encoder* e, void* ptr) {
    J2K_API_BEGIN
    if (!e) return J2K_ERR_INVALID_ARG;
    if (ptr && ptr == e->mapped) {
        cudaFreeHost(e->mapped);
        e->mapped = nullptr;
    }
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_encoder_get_codeblocks(j2k_encoder* e, j2k_cb_desc* descs, size_t* count,
                                      uint8_t* bytes, size_t cap, size_t* used) {
    J2K_API_BEGIN
    if (!e || !count) return J2K_ERR_INVALID_ARG;
    j2k_ctx* ctx = e->ctx;
    if (!e->have_result || e->dwt_only) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "no tier-1 result");
    cudaSetDevice(ctx->device);
    size_t total = 0;
    J2K_TRY(pack_blocks(e, &total));
    if (used) *used = total;
    if (!descs && !bytes) {
        *count = e->njobs;
        return J2K_OK;
    }
    if (descs && *count < e->njobs) return j2k_fail(ctx, J2K_ERR_CAPACITY, "descs array too small");
    if (bytes && cap < total) return j2k_fail(ctx, J2K_ERR_CAPACITY, "bytes buffer too small");
    *count = e->njobs;
    // a large pageable destination is filled through the page-locked staging buffer by host
    // threads (a pageable download is much slower than a page-locked one)
    uint8_t* hs = nullptr;
    if (bytes && total >= ((size_t)8 << 20) && !page_locked(bytes)) {
        hs = (uint8_t*)j2k_pinned(ctx, total + 16);
        if (!hs) return J2K_ERR_OUT_OF_MEMORY;
    }
    if (bytes) J2K_CUDA(ctx, cudaMemcpyAsync(hs ? hs : bytes, e->packed.p, total, cudaMemcpyDeviceToHost, ctx->stream));
    if (descs) {
        J2K_CUDA(ctx, cudaMemcpyAsync(descs, e->descs.p, e->njobs * sizeof(j2k_cb_desc), cudaMemcpyDeviceToHost,
                                      ctx->stream));
    }
    J2K_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (hs) parallel_copy(bytes, hs, total);
    if (descs) {
        uint32_t acc = 0;
        for (size_t i = 0; i < e->njobs; ++i) {
            descs[i].offset = acc;
            acc += (uint32_t)std::max(descs[i].length, 0);
        }
    }
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_encoder_autotune(j2k_encoder* e, int reps, int* report) {
    J2K_API_BEGIN
    if (!e) return J2K_ERR_INVALID_ARG;
    j2k_ctx* ctx = e->ctx;
    if (!e->have_result || e->dwt_only || e->njobs == 0)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "autotune needs the tier-1 result of a run");
    cudaSetDevice(ctx->device);
    reps = std::max(reps, 1);
    // candidates: {tier-0 warps per SM, tier-1 warps per SM, tier-1 blocks per warp, blocks per
    // warp after the tiers}; 0 warps: no tier
    const int cand[8][4] = {{1, 2, 4, 16}, {1, 2, 4, 8}, {1, 2, 4, 32}, {1, 0, 0, 8},
                            {1, 0, 0, 16}, {0, 0, 0, 8}, {2, 2, 4, 16}, {1, 2, 8, 16}};
    cudaEvent_t e0, e1;
    J2K_CUDA(ctx, cudaEventCreate(&e0));
    J2K_CUDA(ctx, cudaEventCreate(&e1));
    const int variant = ctx->mq_variant;
    ctx->mq_variant = 0;
    auto apply = [&](const int* c) {
        for (int k = 0; k < J2K_MQ_TIERS; ++k) ctx->mq_tier_warps[k] = 0, ctx->mq_tier_lanes[k] = 0;
        if (c[0]) ctx->mq_tier_warps[0] = c[0] * ctx->sm_count, ctx->mq_tier_lanes[0] = 1;
        if (c[0] && c[1]) ctx->mq_tier_warps[1] = c[1] * ctx->sm_count, ctx->mq_tier_lanes[1] = c[2];
        ctx->mq_lanes = c[3];
    };
    j2k_status s = J2K_OK;
    int best = 0;
    float best_t = 1e30f;
    for (int c = 0; c < 8 && s == J2K_OK; ++c) {
        apply(cand[c]);
        float tmin = 1e30f;
        for (int r = 0; r <= reps && s == J2K_OK; ++r) {  // the first run warms up
            cudaEventRecord(e0, ctx->stream);
            s = j2k_t1_encode_jobs(ctx, (const int32_t*)e->coef.p, (const j2k_cb_job*)e->jobs.p, e->njobs,
                                   (j2k_cb_desc*)e->descs.p, (uint8_t*)e->bytes.p, e->njobs * e->sym_cap, nullptr,
                                   ctx->stream);
            cudaEventRecord(e1, ctx->stream);
            if (s == J2K_OK) s = j2k_read_device_error(ctx);
            float t = 0;
            if (s == J2K_OK && cudaEventElapsedTime(&t, e0, e1) == cudaSuccess && r > 0) tmin = std::min(tmin, t);
        }
        if (s == J2K_OK && tmin < best_t) best_t = tmin, best = c;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    apply(cand[best]);
    ctx->mq_variant = variant;
    if (report) {
        report[0] = ctx->mq_tier_warps[0];
        report[1] = ctx->mq_tier_warps[1];
        report[2] = ctx->mq_tier_lanes[1];
        report[3] = ctx->mq_lanes;
    }
    // the result again, as the encoder left it (rate control included)
    e->packed_ok = false;
    if (s == J2K_OK) s = run_tier1(e);
    return s;
    J2K_API_END
}

j2k_status j2k_encoder_get_codestream(j2k_encoder* e, uint8_t* out, size_t cap, size_t* len) {
    J2K_API_BEGIN
    if (!e || !len) return J2K_ERR_INVALID_ARG;
    j2k_ctx* ctx = e->ctx;
    size_t count = 0, total = 0;
    J2K_TRY(j2k_encoder_get_codeblocks(e, nullptr, &count, nullptr, 0, &total));
    std::vector<j2k_cb_desc> d(count);
    std::vector<uint8_t> b(total + 1);
    J2K_TRY(j2k_encoder_get_codeblocks(e, d.data(), &count, b.data(), b.size(), &total));
    std::vector<uint32_t> pe;
    if (e->style) {  // the segments of styled blocks are located by their pass ends
        pe.resize(count * J2K_PASS_STRIDE);
        J2K_CUDA(ctx, cudaMemcpyAsync(pe.data(), e->pass_ends.p, pe.size() * 4, cudaMemcpyDeviceToHost, ctx->stream));
        J2K_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    std::vector<j2k_t2_block> blocks(count);
    for (size_t i = 0; i < count; ++i)
        blocks[i] = j2k_t2_block{d[i].numbps, d[i].npasses, d[i].length, b.data() + d[i].offset,
                                 e->style ? pe.data() + i * J2K_PASS_STRIDE : nullptr};
    const int L = (int)(e->lay_np.size() / std::max<size_t>(count, 1));
    std::vector<uint8_t> cs =
        L > 1 && e->lay_np.size() == (size_t)L * count
            ? j2k_t2_write_layers(e->w, e->h, e->ncomp, e->levels, e->cbw, e->cbh, !e->lossy,
                                  e->mct != J2K_MCT_NONE, e->steps.data(), blocks, L, e->lay_np.data(),
                                  e->lay_len.data())
            : j2k_t2_write(e->w, e->h, e->ncomp, e->levels, e->cbw, e->cbh, !e->lossy, e->mct != J2K_MCT_NONE,
                           e->steps.data(), blocks, e->style);
    *len = cs.size();
    if (!out) return J2K_OK;
    if (cap < cs.size()) return j2k_fail(ctx, J2K_ERR_CAPACITY, "codestream buffer too small");
    std::memcpy(out, cs.data(), cs.size());
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_encoder_get_pass_ends(j2k_encoder* e, uint32_t* ends, size_t cap, size_t* count) {
    J2K_API_BEGIN
    if (!e || !count) return J2K_ERR_INVALID_ARG;
    j2k_ctx* ctx = e->ctx;
    if (!e->have_result || e->dwt_only || !e->style)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "no styled tier-1 result");
    *count = e->njobs * J2K_PASS_STRIDE;
    if (!ends) return J2K_OK;
    if (cap < *count) return j2k_fail(ctx, J2K_ERR_CAPACITY, "pass-end buffer too small");
    cudaSetDevice(ctx->device);
    J2K_CUDA(ctx, cudaMemcpyAsync(ends, e->pass_ends.p, *count * 4, cudaMemcpyDeviceToHost, ctx->stream));
    J2K_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_encoder_device_results(j2k_encoder* e, const j2k_cb_desc** descs, const uint8_t** bytes,
                                      size_t* count, size_t* cap_per_block) {
    J2K_API_BEGIN
    if (!e) return J2K_ERR_INVALID_ARG;
    if (!e->have_result || e->dwt_only) return j2k_fail(e->ctx, J2K_ERR_INVALID_ARG, "no tier-1 result");
    if (descs) *descs = (const j2k_cb_desc*)e->descs.p;
    if (bytes) *bytes = (const uint8_t*)e->bytes.p;
    if (count) *count = e->njobs;
    if (cap_per_block) *cap_per_block = e->cap;
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_decoder_create(j2k_ctx* ctx, int lossy, j2k_decoder** out) {
    J2K_API_BEGIN
    if (!ctx || !out) return J2K_ERR_INVALID_ARG;
    j2k_decoder* d = new (std::nothrow) j2k_decoder();
    if (!d) return J2K_ERR_OUT_OF_MEMORY;
    d->ctx = ctx;
    d->lossy = lossy ? 1 : 0;
    *out = d;
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_decoder_destroy(j2k_decoder* d) {
    J2K_API_BEGIN
    if (!d) return J2K_ERR_INVALID_ARG;
    cudaSetDevice(d->ctx->device);
    cudaStreamSynchronize(d->ctx->stream);
    for (DevBuf* b : {&d->descs, &d->bytes, &d->coef, &d->planes, &d->out, &d->jobs, &d->pass_ends, &d->job_style})
        b->release();
    delete d;
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_decoder_run_batch(j2k_decoder* d, const j2k_decode_item* items, int n) {
    J2K_API_BEGIN
    if (!d || (!items && n > 0) || n < 0) return J2K_ERR_INVALID_ARG;
    j2k_ctx* ctx = d->ctx;
    if (n == 0) return J2K_OK;
    cudaSetDevice(ctx->device);
    // jobs of every image into one coefficient buffer; descriptors rebased into one byte buffer
    std::vector<j2k_cb_job> jobs;
    std::vector<size_t> coef_off(n), out_off(n + 1, 0), job0(n + 1, 0), byte0(n + 1, 0);
    std::vector<int> lv(n), cbw(n), cbh(n);
    size_t coef_total = 0, desc_total = 0, max_ll0 = 16, max_ll1 = 16;
    bool any_style = false;
    for (int k = 0; k < n; ++k) {
        const j2k_decode_item& it = items[k];
        if (!it.descs || (!it.bytes && it.nbytes) || !it.out)
            return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "NULL pointer in item " + std::to_string(k));
        if (it.ncomp != 1 && it.ncomp != 3)
            return j2k_fail(ctx, J2K_ERR_UNSUPPORTED, "decoder supports 1 or 3 components");
        j2k_enc_params p{};
        p.levels = it.levels;
        p.cbw = it.cbw;
        p.cbh = it.cbh;
        int order;
        J2K_TRY(check_params(ctx, &p, it.w, it.h, &lv[k], &cbw[k], &cbh[k], &order));
        coef_off[k] = coef_total;
        job0[k] = jobs.size();
        for (int c = 0; c < it.ncomp; ++c)
            j2k_build_jobs(it.w, it.h, lv[k], cbw[k], cbh[k], &jobs, c, coef_total + (uint64_t)c * it.w * it.h,
                           it.w, (uint32_t)k);
        job0[k + 1] = jobs.size();
        if (it.count != job0[k + 1] - job0[k])
            return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "item " + std::to_string(k) + ": descriptor count does not "
                                                      "match the image's code-blocks");
        if (it.cblk_style < 0 || it.cblk_style > 7 || (it.cblk_style && !it.pass_ends))
            return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "item " + std::to_string(k) + ": bad code-block style or "
                                                      "no pass ends");
        for (size_t i = 0; i < it.count; ++i) {
            const j2k_cb_desc& q = it.descs[i];
            if (q.length < 0 || (size_t)q.offset + (size_t)q.length > it.nbytes || q.numbps > 31 ||
                q.npasses > 3 * q.numbps)
                return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "item " + std::to_string(k) + ": code-block descriptor " +
                                                              std::to_string(i) + " is out of range");
        }
        any_style |= it.cblk_style != 0;
        coef_total += (size_t)it.w * it.h * it.ncomp;
        byte0[k + 1] = byte0[k] + it.nbytes;
        out_off[k + 1] = out_off[k] + (size_t)it.w * it.h * it.ncomp;
        const size_t w1 = (it.w + 1) / 2, h1 = (it.h + 1) / 2;
        max_ll0 = std::max(max_ll0, w1 * h1 * 4);
        max_ll1 = std::max(max_ll1, ((w1 + 1) / 2) * ((h1 + 1) / 2) * 4);
        desc_total += it.count;
    }
    // one upload: descriptors and codewords through the page-locked staging buffer
    const size_t nbytes = byte0[n], dbytes = desc_total * sizeof(j2k_cb_desc);
    const size_t stage = std::max(align16(dbytes) + nbytes, out_off[n]) + 16;
    uint8_t* hs = (uint8_t*)j2k_pinned(ctx, stage);
    if (!hs) return J2K_ERR_OUT_OF_MEMORY;
    j2k_cb_desc* hd = (j2k_cb_desc*)hs;
    uint8_t* hb = hs + align16(dbytes);
    host_parallel(n, byte0[n], [&](int k) {
        const j2k_decode_item& it = items[k];
        for (size_t i = 0; i < it.count; ++i) {
            j2k_cb_desc q = it.descs[i];
            q.offset = (uint32_t)(byte0[k] + q.offset);
            hd[job0[k] + i] = q;
        }
        if (it.nbytes) std::memcpy(hb + byte0[k], it.bytes, it.nbytes);
    });
    if (nbytes + 16 > 0xFFFFFFFFull) return j2k_fail(ctx, J2K_ERR_UNSUPPORTED, "more than 4 GiB of codewords");
    J2K_TRY(d->descs.ensure(ctx, dbytes + 16));
    J2K_TRY(d->bytes.ensure(ctx, nbytes + 16));
    J2K_TRY(d->jobs.ensure(ctx, jobs.size() * sizeof(j2k_cb_job) + 16));
    J2K_TRY(d->coef.ensure(ctx, coef_total * 4 + 16));
    J2K_TRY(d->planes.ensure(ctx, coef_total * 4 + 16));
    J2K_TRY(d->out.ensure(ctx, out_off[n] + 16));
    d->job_key[0] = 0;  // the per-image job cache no longer describes d->jobs
    d->hjobs.clear();
    J2K_CUDA(ctx, cudaMemcpyAsync(d->descs.p, hd, dbytes, cudaMemcpyHostToDevice, ctx->stream));
    J2K_CUDA(ctx, cudaMemcpyAsync(d->bytes.p, hb, nbytes, cudaMemcpyHostToDevice, ctx->stream));
    J2K_CUDA(ctx, cudaMemcpyAsync(d->jobs.p, jobs.data(), jobs.size() * sizeof(j2k_cb_job), cudaMemcpyHostToDevice,
                                  ctx->stream));
    J2K_TRY(j2k_clear_device_error(ctx));
    const uint32_t* dpe = nullptr;
    const uint8_t* djs = nullptr;
    if (any_style) {
        // a style per job, and pass ends for every job (an unstyled block: one segment of its
        // whole codeword, the end of its last pass)
        const size_t nj = jobs.size();
        std::vector<uint32_t> pe(nj * J2K_PASS_STRIDE, 0);
        std::vector<uint8_t> js(nj, 0);
        for (int k = 0; k < n; ++k) {
            const j2k_decode_item& it = items[k];
            for (size_t i = 0; i < it.count; ++i) {
                uint32_t* row = pe.data() + (job0[k] + i) * J2K_PASS_STRIDE;
                js[job0[k] + i] = (uint8_t)it.cblk_style;
                if (it.cblk_style) std::memcpy(row, it.pass_ends + i * J2K_PASS_STRIDE, J2K_PASS_STRIDE * 4);
                else
                    for (int q = 0; q < J2K_PASS_STRIDE; ++q) row[q] = (uint32_t)std::max(it.descs[i].length, 0);
            }
        }
        J2K_TRY(d->pass_ends.ensure(ctx, pe.size() * 4 + 16));
        J2K_TRY(d->job_style.ensure(ctx, nj + 16));
        J2K_CUDA(ctx, cudaMemcpyAsync(d->pass_ends.p, pe.data(), pe.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
        J2K_CUDA(ctx, cudaMemcpyAsync(d->job_style.p, js.data(), nj, cudaMemcpyHostToDevice, ctx->stream));
        J2K_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // the host vectors go out of scope
        dpe = (const uint32_t*)d->pass_ends.p;
        djs = (const uint8_t*)d->job_style.p;
    }
    // tier-1 of every block of every image in one launch
    J2K_TRY(j2k_t1_decode_jobs(ctx, (const j2k_cb_desc*)d->descs.p, (const uint8_t*)d->bytes.p,
                               (const j2k_cb_job*)d->jobs.p, jobs.size(), (int32_t*)d->coef.p, ctx->stream, 0, dpe,
                               djs));
    void* ll0 = j2k_scratch(ctx, SCR_LL0, max_ll0);
    void* ll1 = j2k_scratch(ctx, SCR_LL1, max_ll1);
    if (!ll0 || !ll1) return J2K_ERR_OUT_OF_MEMORY;
    for (int k = 0; k < n; ++k) {
        const j2k_decode_item& it = items[k];
        const bool lossy = !it.lossless;
        const size_t w = it.w, h = it.h, px = w * h;
        std::vector<float> steps;
        if (lossy) {
            if (it.steps) steps.assign(it.steps, it.steps + 3 * lv[k] + 1);
            else steps = default_steps(w, h, lv[k]);
        }
        for (int c = 0; c < it.ncomp; ++c)
            J2K_TRY(j2k_dwt_inv_impl(ctx, lossy ? J2K_W97 : J2K_W53, J2K_ORDER_T800,
                                     (const char*)d->coef.p + (coef_off[k] + (size_t)c * px) * 4, w,
                                     (char*)d->planes.p + (coef_off[k] + (size_t)c * px) * 4, w, w, h, lv[k],
                                     lossy ? steps.data() : nullptr, ll0, ll1, j2k_dwt_tile{64, 64}, ctx->stream));
        const int mct = it.ncomp >= 3 ? (lossy ? J2K_MCT_ICT : J2K_MCT_RCT) : J2K_MCT_NONE;
        J2K_TRY(j2k_launch_planar_inv(ctx, (const char*)d->planes.p + coef_off[k] * 4, lossy ? J2K_F32 : J2K_I32, w,
                                      px, it.ncomp, mct, (uint8_t*)d->out.p + out_off[k], w * it.ncomp, w, h,
                                      ctx->stream));
    }
    // one read-back of every image's pixels
    J2K_CUDA(ctx, cudaMemcpyAsync(hs, d->out.p, out_off[n], cudaMemcpyDeviceToHost, ctx->stream));
    J2K_TRY(j2k_read_device_error(ctx));
    host_parallel(n, out_off[n], [&](int k) { std::memcpy(items[k].out, hs + out_off[k], out_off[k + 1] - out_off[k]); });
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_decoder_run_codestreams(j2k_decoder* d, const uint8_t* const* streams, const size_t* sizes, int n,
                                       int max_layers, uint8_t* const* outs) {
    J2K_API_BEGIN
    if (!d || n < 0 || (n > 0 && (!streams || !sizes || !outs)) || max_layers < 0) return J2K_ERR_INVALID_ARG;
    j2k_ctx* ctx = d->ctx;
    if (n == 0) return J2K_OK;
    // tier-2 of every stream on host threads, then one batched device decode
    std::vector<j2k_stream_info> info(n);
    std::vector<std::vector<j2k_cb_desc>> descs(n);
    std::vector<std::vector<uint8_t>> bytes(n);
    std::vector<std::vector<uint32_t>> ends(n);
    std::vector<j2k_status> st(n, J2K_OK);
    std::vector<std::string> msg(n);
    const int nt = (int)std::min<unsigned>((unsigned)n, std::max(1u, std::min(16u, std::thread::hardware_concurrency())));
    auto work = [&](int t) {
        for (int k = t; k < n; k += nt) {
            if (!streams[k]) {
                st[k] = J2K_ERR_INVALID_ARG;
                msg[k] = "NULL stream";
                continue;
            }
            try {
                st[k] = j2k_t2_parse_packed(streams[k], sizes[k], max_layers, &info[k], &descs[k], &bytes[k],
                                            &msg[k], &ends[k]);
            } catch (...) {  // a host allocation failed
                st[k] = J2K_ERR_OUT_OF_MEMORY;
            }
        }
    };
    j2k_run_threads(nt, work);
    std::vector<j2k_decode_item> items(n);
    for (int k = 0; k < n; ++k) {
        if (st[k] != J2K_OK) return j2k_fail(ctx, st[k], "stream " + std::to_string(k) + ": " + msg[k]);
        const j2k_stream_info& I = info[k];
        if (I.precision != 8) return j2k_fail(ctx, J2K_ERR_UNSUPPORTED, "stream " + std::to_string(k) + ": precision");
        items[k] = j2k_decode_item{I.w, I.h, I.ncomp, I.lossless, I.levels, I.cbw, I.cbh,
                                   I.lossless ? nullptr : I.steps, descs[k].data(), descs[k].size(),
                                   bytes[k].data(), bytes[k].size(), outs[k], I.cblk_style,
                                   I.cblk_style ? ends[k].data() : nullptr};
    }
    return j2k_decoder_run_batch(d, items.data(), n);
    J2K_API_END
}

j2k_status j2k_decoder_run_codeblocks(j2k_decoder* d, const j2k_cb_desc* descs, const uint8_t* bytes,
                                      size_t nbytes, int on_device, int ncomp, size_t w, size_t h,
                                      const j2k_enc_params* p, uint8_t* out, int out_on_device,
                                      size_t out_pitch) {
    J2K_API_BEGIN
    if (!d) return J2K_ERR_INVALID_ARG;
    j2k_ctx* ctx = d->ctx;
    if (!descs || !bytes || !out) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "NULL pointer");
    if (ncomp != 1 && ncomp != 3) return j2k_fail(ctx, J2K_ERR_UNSUPPORTED, "decoder supports 1 or 3 components");
    int levels, cbw, cbh, order;
    J2K_TRY(check_params(ctx, p, w, h, &levels, &cbw, &cbh, &order));
    if (out_pitch == 0) out_pitch = w * (size_t)ncomp;
    cudaSetDevice(ctx->device);
    size_t njobs = 0;
    J2K_TRY(prepare_jobs(ctx, d->hjobs, d->jobs, d->job_key, w, h, ncomp, levels, cbw, cbh, &njobs));
    const j2k_cb_desc* dd = descs;
    const uint8_t* db = bytes;
    const int style = p ? p->cblk_style : 0;
    const uint32_t* dpe = style ? p->pass_ends : nullptr;
    if (style && !dpe) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "a styled decode needs the pass ends");
    if (style && !on_device) {
        J2K_TRY(d->pass_ends.ensure(ctx, njobs * J2K_PASS_STRIDE * 4 + 16));
        J2K_CUDA(ctx, cudaMemcpyAsync(d->pass_ends.p, dpe, njobs * J2K_PASS_STRIDE * 4, cudaMemcpyHostToDevice,
                                      ctx->stream));
        dpe = (const uint32_t*)d->pass_ends.p;
    }
    if (!on_device) {
        // host descriptors are validated before any kernel reads through them
        for (size_t i = 0; i < njobs; ++i) {
            const j2k_cb_desc& q = descs[i];
            if (q.length < 0 || (size_t)q.offset + (size_t)q.length > nbytes || q.numbps > 31 ||
                q.npasses > 3 * q.numbps)
                return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "code-block descriptor " + std::to_string(i) +
                                                              " is out of range");
        }
        J2K_TRY(d->descs.ensure(ctx, njobs * sizeof(j2k_cb_desc) + 16));
        J2K_TRY(d->bytes.ensure(ctx, nbytes + 16));
        J2K_CUDA(ctx, cudaMemcpyAsync(d->descs.p, descs, njobs * sizeof(j2k_cb_desc), cudaMemcpyHostToDevice, ctx->stream));
        // (pageable uploads are left to the driver, which pipelines its own staging)
        J2K_CUDA(ctx, cudaMemcpyAsync(d->bytes.p, bytes, nbytes, cudaMemcpyHostToDevice, ctx->stream));
        dd = (const j2k_cb_desc*)d->descs.p;
        db = (const uint8_t*)d->bytes.p;
    }
    const size_t n = w * h;
    J2K_TRY(d->coef.ensure(ctx, n * 4 * ncomp));
    J2K_TRY(d->planes.ensure(ctx, n * 4 * ncomp));
    J2K_TRY(j2k_clear_device_error(ctx));
    J2K_TRY(j2k_t1_decode_jobs(ctx, dd, db, (const j2k_cb_job*)d->jobs.p, njobs, (int32_t*)d->coef.p, ctx->stream,
                               style, dpe));
    std::vector<float> steps;
    if (d->lossy) {
        if (p && p->steps) steps.assign(p->steps, p->steps + 3 * levels + 1);
        else steps = default_steps(w, h, levels);
    }
    size_t w1 = (w + 1) / 2, h1 = (h + 1) / 2, w2 = (w1 + 1) / 2, h2 = (h1 + 1) / 2;
    void* ll0 = j2k_scratch(ctx, SCR_LL0, w1 * h1 * 4);
    void* ll1 = j2k_scratch(ctx, SCR_LL1, w2 * h2 * 4);
    if (!ll0 || !ll1) return J2K_ERR_OUT_OF_MEMORY;
    for (int c = 0; c < ncomp; ++c) {
        J2K_TRY(j2k_dwt_inv_impl(ctx, d->lossy ? J2K_W97 : J2K_W53, d->lossy ? J2K_ORDER_T800 : order,
                                 (const char*)d->coef.p + (size_t)c * n * 4, w,
                                 (char*)d->planes.p + (size_t)c * n * 4, w, w, h, levels,
                                 d->lossy ? steps.data() : nullptr, ll0, ll1, j2k_dwt_tile{64, 64}, ctx->stream));
    }
    int mct = ncomp >= 3 ? (d->lossy ? J2K_MCT_ICT : J2K_MCT_RCT) : J2K_MCT_NONE;
    uint8_t* dst = out;
    if (!out_on_device) {
        J2K_TRY(d->out.ensure(ctx, out_pitch * h + 16));
        dst = (uint8_t*)d->out.p;
    }
    J2K_TRY(j2k_launch_planar_inv(ctx, d->planes.p, d->lossy ? J2K_F32 : J2K_I32, w, n, ncomp, mct, dst,
                                  out_pitch, w, h, ctx->stream));
    if (!out_on_device) {
        const size_t ob = out_pitch * h;
        if (ob >= ((size_t)8 << 20) && !page_locked(out)) {
            // pageable output: through the page-locked staging buffer, emptied by host threads
            // (a pageable download is much slower than a page-locked one and a parallel copy)
            uint8_t* hs = (uint8_t*)j2k_pinned(ctx, ob + 16);
            if (!hs) return J2K_ERR_OUT_OF_MEMORY;
            J2K_CUDA(ctx, cudaMemcpyAsync(hs, dst, ob, cudaMemcpyDeviceToHost, ctx->stream));
            J2K_TRY(j2k_read_device_error(ctx));
            parallel_copy(out, hs, ob);
            return J2K_OK;
        }
        J2K_CUDA(ctx, cudaMemcpyAsync(out, dst, ob, cudaMemcpyDeviceToHost, ctx->stream));
    }
    return j2k_read_device_error(ctx);
    J2K_API_END
}

}  // extern "C"
