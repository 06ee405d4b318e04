// Batched encoder: many images of uneven size, mixed 5/3 (lossless, RCT) and 9/7 (ICT +
// dead-zone quantiser), encoded by a fixed launch sequence that does not grow with the number
// of images:
//   2 planar launches (int32 / float planes)  ->  per decomposition level, one forward-DWT launch
//   per filter over a flattened tile list of every image and component at that level  ->
//   one persistent tier-1 context-modelling launch pulling code-blocks of all images from a
//   device-side queue (largest first)  ->  radix sort of the symbol counts  ->  one MQ launch.
// The sequence is captured once into a CUDA graph and replayed per batch.  The autotuner picks
// the DWT tile shape per filter and the code-block-to-warp schedule (phase-A order, MQ variant
// and blocks per warp) by timing the candidates on the batch itself.
//
// The reference has no batching: OCLEncoder<T>::run encodes one image per call
// (src/OCLEncoder.cpp:43-52), which is the "per-image" path this is measured against.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <numeric>

#include <cub/cub.cuh>

#include "j2k_internal.cuh"

namespace {

size_t a16(size_t v) { return (v + 15) & ~(size_t)15; }
bool pow2cb(int v) { return v >= 4 && v <= 64 && (v & (v - 1)) == 0; }

struct Buf {
    void* p = nullptr;
    size_t n = 0;
    j2k_status ensure(j2k_ctx* ctx, size_t bytes) {
        if (bytes == 0) bytes = 16;
        if (n >= bytes) return J2K_OK;
        if (p) {
            cudaStreamSynchronize(ctx->stream);
            cudaFree(p);
        }
        p = nullptr;
        n = 0;
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

struct ImgPlan {
    j2k_batch_image d;
    std::vector<float> steps;
    size_t n = 0;             // pixels
    size_t in_off = 0;        // bytes in the packed input buffer
    size_t plane_off = 0;     // elements in the plane / coefficient buffers
    size_t stride = 0;        // elements between component planes
    size_t ll_off = 0;        // elements in the LL scratch (per component: ll0 then ll1)
    size_t ll_stride = 0;
    size_t job0 = 0, njobs = 0;
};

// tile shapes of the batched forward DWT: 0-2 the shared-memory tile kernel, 3 the
// register-lifting kernel (248 output columns x 16 rows, the form the per-image path uses)
j2k_dwt_tile tile_of(int code) {
    return code == 1 ? j2k_dwt_tile{128, 32}
                     : (code == 2 ? j2k_dwt_tile{32, 128} : (code == 3 ? j2k_dwt_tile{248, 16} : j2k_dwt_tile{64, 64}));
}

}  // namespace

struct j2k_batch {
    j2k_ctx* ctx = nullptr;
    std::vector<ImgPlan> img;
    size_t in_bytes = 0, plane_elems = 0, ll_elems = 0;
    Buf in, planes, coef, ll, jobs, order, descs, bytes, pdesc, pwork53, pwork97, ldesc, lowner;
    unsigned nwork53 = 0, nwork97 = 0;
    int lmax = 0;
    // per level: [filter 0 = 5/3, 1 = 9/7] -> (first desc, count, first owner, tile count)
    std::vector<size_t> ldesc_first[2], ldesc_count[2], lowner_first[2], lowner_count[2];
    std::vector<j2k_cb_job> hjobs;
    size_t out_bytes = 0, sym_bytes = 0;
    double out_factor = 2.0, sym_factor = 20.0;  // capacity per sample (grown on overflow)
    // tuning
    int tile_code[2] = {3, 3};
    int phase_a_order = 1;  // 1: largest blocks first, 0: natural order
    bool use_graph = true;
    int stages = 7;  // J2K_BATCH_STAGES: 1 planar, 2 DWT, 4 tier-1
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    cudaStream_t cap_stream = nullptr;  // capture stream (the caller's may be the legacy stream)
    bool have_result = false;
    bool pending = false;  // enqueued by j2k_batch_encode_async, device error word not read yet
    std::string err;
    // packed results (j2k_batch_pack): every block's codeword back to back, in job order
    Buf plens, poffs, ptmp, packed, pdescs;
    size_t packed_total = 0;
};

namespace {
__global__ void batch_lengths_kernel(const j2k_cb_desc* __restrict__ d, uint32_t* __restrict__ len, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) len[i] = (uint32_t)max(d[i].length, 0);
}
// one warp per block: codeword to its packed offset, descriptor with the packed offset
__global__ void batch_pack_kernel(const j2k_cb_desc* __restrict__ d, const uint32_t* __restrict__ off,
                                  const uint8_t* __restrict__ src, uint8_t* __restrict__ dst,
                                  j2k_cb_desc* __restrict__ out, int n) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= n) return;
    const int len = max(d[w].length, 0);
    const uint8_t* a = src + d[w].offset;
    uint8_t* b = dst + off[w];
    for (int k = lane; k < len; k += 32) b[k] = a[k];
    if (lane == 0) {
        j2k_cb_desc x = d[w];
        x.offset = off[w];
        out[w] = x;
    }
}
}  // namespace

static void drop_graph(j2k_batch* b) {
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->gexec = nullptr;
    b->graph = nullptr;
}

// lays out the tier-1 jobs' symbol / codeword capacities (proportional to block area)
static j2k_status layout_t1(j2k_batch* b) {
    j2k_ctx* ctx = b->ctx;
    uint64_t o = 0, y = 0;
    for (auto& j : b->hjobs) {
        const double area = (double)j.cw * j.ch;
        j.out_cap = (uint32_t)a16((size_t)(area * b->out_factor) + 256);
        j.sym_cap = (uint32_t)a16((size_t)(area * b->sym_factor) + 256);
        j.out_off = o;
        j.sym_off = y;
        o += j.out_cap;
        y += j.sym_cap;
    }
    b->out_bytes = o;
    b->sym_bytes = y;
    J2K_TRY(b->jobs.ensure(ctx, b->hjobs.size() * sizeof(j2k_cb_job)));
    J2K_CUDA(ctx, cudaMemcpy(b->jobs.p, b->hjobs.data(), b->hjobs.size() * sizeof(j2k_cb_job), cudaMemcpyHostToDevice));
    J2K_TRY(b->bytes.ensure(ctx, o + 64));
    J2K_TRY(b->descs.ensure(ctx, b->hjobs.size() * sizeof(j2k_cb_desc)));
    // scratch used by the tier-1 launcher, sized now so that graph capture never allocates
    if (!j2k_scratch(ctx, SCR_SYMS, y + 64)) return J2K_ERR_OUT_OF_MEMORY;
    return J2K_OK;
}

static j2k_status plan(j2k_batch* b) {
    j2k_ctx* ctx = b->ctx;
    size_t in_off = 0, pe = 0, lle = 0;
    b->lmax = 0;
    for (auto& im : b->img) {
        const j2k_batch_image& d = im.d;
        im.n = (size_t)d.w * d.h;
        im.in_off = in_off;
        in_off += a16(im.n * d.ncomp);
        im.stride = a16(im.n);
        im.plane_off = pe;
        pe += im.stride * d.ncomp;
        const size_t w1 = (d.w + 1) / 2, h1 = (d.h + 1) / 2, w2 = (w1 + 1) / 2, h2 = (h1 + 1) / 2;
        im.ll_stride = a16(w1 * h1) + a16(w2 * h2);
        im.ll_off = lle;
        lle += im.ll_stride * d.ncomp;
        b->lmax = std::max(b->lmax, d.levels);
    }
    b->in_bytes = in_off;
    b->plane_elems = pe;
    b->ll_elems = lle;
    J2K_TRY(b->in.ensure(ctx, in_off + 64));
    J2K_TRY(b->planes.ensure(ctx, pe * 4 + 64));
    J2K_TRY(b->coef.ensure(ctx, pe * 4 + 64));
    J2K_TRY(b->ll.ensure(ctx, lle * 4 + 64));
    // planar work lists
    std::vector<j2k_batch_planar_desc> pd(b->img.size());
    std::vector<uint2> w53, w97;
    for (size_t i = 0; i < b->img.size(); ++i) {
        const ImgPlan& im = b->img[i];
        const bool lossy = im.d.kernel == J2K_W97;
        pd[i] = j2k_batch_planar_desc{im.in_off, im.plane_off, im.stride, im.n, im.d.ncomp,
                                      im.d.ncomp >= 3 ? (lossy ? J2K_MCT_ICT : J2K_MCT_RCT) : J2K_MCT_NONE};
        for (size_t p = 0; p < im.n; p += 4096) (lossy ? w97 : w53).push_back(make_uint2((unsigned)i, (unsigned)p));
    }
    b->nwork53 = (unsigned)w53.size();
    b->nwork97 = (unsigned)w97.size();
    J2K_TRY(b->pdesc.ensure(ctx, pd.size() * sizeof(pd[0])));
    J2K_TRY(b->pwork53.ensure(ctx, w53.size() * sizeof(uint2)));
    J2K_TRY(b->pwork97.ensure(ctx, w97.size() * sizeof(uint2)));
    J2K_CUDA(ctx, cudaMemcpy(b->pdesc.p, pd.data(), pd.size() * sizeof(pd[0]), cudaMemcpyHostToDevice));
    if (!w53.empty()) J2K_CUDA(ctx, cudaMemcpy(b->pwork53.p, w53.data(), w53.size() * sizeof(uint2), cudaMemcpyHostToDevice));
    if (!w97.empty()) J2K_CUDA(ctx, cudaMemcpy(b->pwork97.p, w97.data(), w97.size() * sizeof(uint2), cudaMemcpyHostToDevice));
    return J2K_OK;
}

// DWT level descriptors + tile owners for the current tile shapes
static j2k_status plan_dwt(j2k_batch* b) {
    j2k_ctx* ctx = b->ctx;
    std::vector<j2k_dwt_level_desc> all;
    std::vector<uint32_t> owners;
    int32_t* coef = (int32_t*)b->coef.p;
    int32_t* planes = (int32_t*)b->planes.p;
    int32_t* llb = (int32_t*)b->ll.p;
    for (int f = 0; f < 2; ++f) {
        b->ldesc_first[f].assign(b->lmax, 0);
        b->ldesc_count[f].assign(b->lmax, 0);
        b->lowner_first[f].assign(b->lmax, 0);
        b->lowner_count[f].assign(b->lmax, 0);
    }
    for (int k = 0; k < b->lmax; ++k)
        for (int f = 0; f < 2; ++f) {
            const int kern = f ? J2K_W97 : J2K_W53;
            const j2k_dwt_tile t = tile_of(b->tile_code[f]);
            b->ldesc_first[f][k] = all.size();
            b->lowner_first[f][k] = owners.size();
            for (const ImgPlan& im : b->img) {
                if (im.d.kernel != kern || im.d.levels <= k) continue;
                int ws[40], hs[40];
                ws[0] = (int)im.d.w;
                hs[0] = (int)im.d.h;
                for (int q = 1; q <= im.d.levels; ++q) { ws[q] = (ws[q - 1] + 1) / 2; hs[q] = (hs[q - 1] + 1) / 2; }
                const bool last = k == im.d.levels - 1;
                for (int c = 0; c < im.d.ncomp; ++c) {
                    int32_t* plane = planes + im.plane_off + (size_t)c * im.stride;
                    int32_t* cf = coef + im.plane_off + (size_t)c * im.stride;
                    int32_t* l0 = llb + im.ll_off + (size_t)c * im.ll_stride;
                    int32_t* l1 = l0 + a16((size_t)ws[1] * hs[1]);
                    j2k_dwt_level_desc d{};
                    d.src = k == 0 ? (const void*)plane : (const void*)((k - 1) % 2 == 0 ? l0 : l1);
                    d.spitch = k == 0 ? im.d.w : (size_t)ws[k];
                    d.w = ws[k];
                    d.h = hs[k];
                    d.dst = cf;
                    d.dpitch = im.d.w;
                    if (last) {
                        d.ll_dst = cf;
                        d.llpitch = im.d.w;
                    } else {
                        d.ll_dst = k % 2 == 0 ? l0 : l1;
                        d.llpitch = (size_t)ws[k + 1];
                    }
                    d.flags = 0;
                    if (kern == J2K_W97) {
                        const int bt = 1 + 3 * (im.d.levels - (k + 1));
                        d.s_ll = im.steps[0];
                        d.s_hl = im.steps[bt];
                        d.s_lh = im.steps[bt + 1];
                        d.s_hh = im.steps[bt + 2];
                        d.flags = 1 | (last ? 2 : 0);
                    }
                    if ((((uintptr_t)d.dst & 7) == 0) && ((d.dpitch & 1) == 0) && (((uintptr_t)d.ll_dst & 7) == 0) &&
                        ((d.llpitch & 1) == 0))
                        d.flags |= 4;  // 8-byte vector stores of sample pairs
                    d.tiles_x = (d.w + t.tw - 1) / t.tw;
                    const int ty = (d.h + t.th - 1) / t.th;
                    d.tile0 = (uint32_t)(owners.size() - b->lowner_first[f][k]);  // launch-relative
                    const uint32_t slot = (uint32_t)all.size();
                    for (int q = 0; q < d.tiles_x * ty; ++q) owners.push_back(slot);
                    all.push_back(d);
                }
            }
            b->ldesc_count[f][k] = all.size() - b->ldesc_first[f][k];
            b->lowner_count[f][k] = owners.size() - b->lowner_first[f][k];
        }
    J2K_TRY(b->ldesc.ensure(ctx, all.size() * sizeof(j2k_dwt_level_desc)));
    J2K_TRY(b->lowner.ensure(ctx, owners.size() * sizeof(uint32_t)));
    if (!all.empty())
        J2K_CUDA(ctx, cudaMemcpy(b->ldesc.p, all.data(), all.size() * sizeof(all[0]), cudaMemcpyHostToDevice));
    if (!owners.empty())
        J2K_CUDA(ctx, cudaMemcpy(b->lowner.p, owners.data(), owners.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    return J2K_OK;
}

static j2k_status plan_t1(j2k_batch* b) {
    j2k_ctx* ctx = b->ctx;
    b->hjobs.clear();
    for (size_t i = 0; i < b->img.size(); ++i) {
        ImgPlan& im = b->img[i];
        im.job0 = b->hjobs.size();
        for (int c = 0; c < im.d.ncomp; ++c)
            j2k_build_jobs(im.d.w, im.d.h, im.d.levels, im.d.cb, im.d.cb, &b->hjobs, c,
                           im.plane_off + (size_t)c * im.stride, im.d.w, (uint32_t)i);
        im.njobs = b->hjobs.size() - im.job0;
    }
    J2K_TRY(layout_t1(b));
    // phase-A order: largest blocks first (ties by position)
    std::vector<uint32_t> ord(b->hjobs.size());
    std::iota(ord.begin(), ord.end(), 0u);
    std::stable_sort(ord.begin(), ord.end(), [&](uint32_t x, uint32_t y) {
        return (uint32_t)b->hjobs[x].cw * b->hjobs[x].ch > (uint32_t)b->hjobs[y].cw * b->hjobs[y].ch;
    });
    J2K_TRY(b->order.ensure(ctx, ord.size() * 4));
    J2K_CUDA(ctx, cudaMemcpy(b->order.p, ord.data(), ord.size() * 4, cudaMemcpyHostToDevice));
    return J2K_OK;
}

// the device pipeline of one batch (input already in b->in), on ctx->stream
static j2k_status enqueue(j2k_batch* b, bool do_planar, bool do_dwt, bool do_t1) {
    j2k_ctx* ctx = b->ctx;
    cudaStream_t st = ctx->stream;
    if (do_planar) {
        J2K_TRY(j2k_launch_planar_batched(ctx, (const j2k_batch_planar_desc*)b->pdesc.p, (const uint2*)b->pwork53.p,
                                          b->nwork53, (const uint8_t*)b->in.p, b->planes.p, 0, st));
        J2K_TRY(j2k_launch_planar_batched(ctx, (const j2k_batch_planar_desc*)b->pdesc.p, (const uint2*)b->pwork97.p,
                                          b->nwork97, (const uint8_t*)b->in.p, b->planes.p, 1, st));
    }
    if (do_dwt)
        for (int k = 0; k < b->lmax; ++k)
            for (int f = 0; f < 2; ++f) {
                if (!b->lowner_count[f][k]) continue;
                const j2k_dwt_level_desc* d = (const j2k_dwt_level_desc*)b->ldesc.p;
                const uint32_t* own = (const uint32_t*)b->lowner.p + b->lowner_first[f][k];
                // this launch covers owner entries [first, first+count); descriptors' tile0 are
                // relative to `first`
                J2K_TRY(j2k_dwt_fwd_batched_launch(ctx, f ? J2K_W97 : J2K_W53, J2K_ORDER_T800,
                                                   tile_of(b->tile_code[f]), d, own,
                                                   (unsigned)b->lowner_count[f][k], st));
            }
    if (do_t1)
        J2K_TRY(j2k_t1_encode_jobs(ctx, (const int32_t*)b->coef.p, (const j2k_cb_job*)b->jobs.p, b->hjobs.size(),
                                   (j2k_cb_desc*)b->descs.p, (uint8_t*)b->bytes.p, b->sym_bytes,
                                   b->phase_a_order ? (const uint32_t*)b->order.p : nullptr, st));
    return J2K_OK;
}

// Kernel nodes of a captured graph whose kernels are this library's (CUB's sort and scan
// kernels, which the tier-1 order uses, are left out); -1 when the graph cannot be read.
static int count_own_kernel_nodes(cudaGraph_t g) {
    size_t n = 0;
    if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess) return -1;
    std::vector<cudaGraphNode_t> nodes(n);
    if (n && cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return -1;
    int count = 0;
    for (size_t i = 0; i < n; ++i) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nodes[i], &t) != cudaSuccess || t != cudaGraphNodeTypeKernel) continue;
        cudaKernelNodeParams kp;
        if (cudaGraphKernelNodeGetParams(nodes[i], &kp) != cudaSuccess) continue;
        const char* name = nullptr;
        if (cudaFuncGetName(&name, kp.func) != cudaSuccess || !name) continue;
        if (std::strstr(name, "cub") != nullptr) continue;
        ++count;
    }
    return count;
}

static j2k_status run_once(j2k_batch* b) {
    j2k_ctx* ctx = b->ctx;
    if (b->use_graph) {
        if (!b->gexec) {
            // warm every launch path once outside capture (lazy module loading, scratch sizing)
            J2K_TRY(enqueue(b, b->stages & 1, b->stages & 2, b->stages & 4));
            J2K_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            if (!b->cap_stream) J2K_CUDA(ctx, cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking));
            cudaStream_t caller = ctx->stream;
            ctx->stream = b->cap_stream;
            cudaError_t eb = cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal);
            if (eb != cudaSuccess) {
                ctx->stream = caller;
                J2K_CUDA(ctx, eb);
            }
            j2k_status s = enqueue(b, b->stages & 1, b->stages & 2, b->stages & 4);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(b->cap_stream, &g);
            ctx->stream = caller;
            if (s != J2K_OK) {
                if (g) cudaGraphDestroy(g);
                return s;
            }
            J2K_CUDA(ctx, e);
            b->graph = g;
            J2K_CUDA(ctx, cudaGraphInstantiate(&b->gexec, g, 0));
        }
        J2K_CUDA(ctx, cudaGraphLaunch(b->gexec, ctx->stream));
        return J2K_OK;
    }
    return enqueue(b, b->stages & 1, b->stages & 2, b->stages & 4);
}

extern "C" {

j2k_status j2k_batch_create(j2k_ctx* ctx, const j2k_batch_image* images, int n, j2k_batch** out) {
    J2K_API_BEGIN
    if (!ctx || !out || !images || n <= 0) return J2K_ERR_INVALID_ARG;
    *out = nullptr;
    j2k_batch* b = new (std::nothrow) j2k_batch();
    if (!b) return J2K_ERR_OUT_OF_MEMORY;
    b->ctx = ctx;
    cudaSetDevice(ctx->device);
    for (int i = 0; i < n; ++i) {
        const j2k_batch_image& d = images[i];
        if (d.w == 0 || d.h == 0 || d.w > 65535 || d.h > 65535 || (d.ncomp != 1 && d.ncomp != 3) ||
            (d.kernel != J2K_W53 && d.kernel != J2K_W97) || d.levels < 1 || d.levels > 32 || !pow2cb(d.cb)) {
            delete b;
            return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "batch image " + std::to_string(i) + " has a bad descriptor");
        }
        ImgPlan im;
        im.d = d;
        if (d.kernel == J2K_W97) {
            std::vector<j2k_band_rect> r(3 * d.levels + 1);
            j2k_band_rects(d.w, d.h, d.levels, r.data());
            im.steps.resize(r.size());
            for (size_t q = 0; q < r.size(); ++q) {
                im.steps[q] = d.steps ? d.steps[q] : 8.0f * std::ldexp(1.0f, -r[q].level);
                int ex, mt;
                if (!j2k_qcd_step(im.steps[q], (int)q, &ex, &mt)) {
                    delete b;
                    return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "batch image " + std::to_string(i) +
                                                                   ": a quantiser step is not positive or out of the QCD range");
                }
            }
        }
        im.d.steps = nullptr;
        b->img.push_back(im);
    }
    j2k_status s = plan(b);
    if (s == J2K_OK) s = plan_dwt(b);
    if (s == J2K_OK) s = plan_t1(b);
    if (s != J2K_OK) {
        j2k_batch_destroy(b);
        return s;
    }
    *out = b;
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_batch_destroy(j2k_batch* b) {
    J2K_API_BEGIN
    if (!b) return J2K_ERR_INVALID_ARG;
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    drop_graph(b);
    if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
    for (Buf* x : {&b->in, &b->planes, &b->coef, &b->ll, &b->jobs, &b->order, &b->descs, &b->bytes, &b->pdesc,
                   &b->pwork53, &b->pwork97, &b->ldesc, &b->lowner})
        x->release();
    delete b;
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_batch_input(j2k_batch* b, uint8_t** device_buffer, size_t* offsets) {
    J2K_API_BEGIN
    if (!b) return J2K_ERR_INVALID_ARG;
    if (device_buffer) *device_buffer = (uint8_t*)b->in.p;
    if (offsets) {
        for (size_t i = 0; i < b->img.size(); ++i) offsets[i] = b->img[i].in_off;
        offsets[b->img.size()] = b->in_bytes;
    }
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_batch_set_option(j2k_batch* b, int key, int value) {
    J2K_API_BEGIN
    if (!b) return J2K_ERR_INVALID_ARG;
    j2k_ctx* ctx = b->ctx;
    switch (key) {
        case J2K_BATCH_USE_GRAPH: b->use_graph = value != 0; break;
        case J2K_BATCH_TILE53:
        case J2K_BATCH_TILE97:
            if (value < 0 || value > 3) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "tile code must be 0, 1, 2 or 3");
            b->tile_code[key == J2K_BATCH_TILE97] = value;
            J2K_TRY(plan_dwt(b));
            break;
        case J2K_BATCH_PHASE_A_ORDER: b->phase_a_order = value != 0; break;
        case J2K_BATCH_STAGES:
            if (value < 1 || value > 7) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "stage mask must be 1..7");
            b->stages = value;
            break;
        default: return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "unknown batch option");
    }
    drop_graph(b);
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_batch_get_option(j2k_batch* b, int key, int* value) {
    J2K_API_BEGIN
    if (!b || !value) return J2K_ERR_INVALID_ARG;
    switch (key) {
        case J2K_BATCH_USE_GRAPH: *value = b->use_graph; break;
        case J2K_BATCH_TILE53: *value = b->tile_code[0]; break;
        case J2K_BATCH_TILE97: *value = b->tile_code[1]; break;
        case J2K_BATCH_PHASE_A_ORDER: *value = b->phase_a_order; break;
        case J2K_BATCH_MQ_VARIANT: *value = b->ctx->mq_variant; break;
        case J2K_BATCH_MQ_LANES: *value = b->ctx->mq_lanes; break;
        case J2K_BATCH_MQ_TIERS: *value = b->ctx->mq_tier_lanes[0] > 0 && b->ctx->mq_tier_warps[0] > 0; break;
        case J2K_BATCH_GRAPH_KERNELS: *value = b->graph ? count_own_kernel_nodes(b->graph) : 0; break;
        case J2K_BATCH_STAGES: *value = b->stages; break;
        case J2K_BATCH_T1A_CTAS: *value = b->ctx->t1a_ctas; break;
        default: return J2K_ERR_INVALID_ARG;
    }
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_batch_upload(j2k_batch* b, const uint8_t* const* pixels, int on_device) {
    J2K_API_BEGIN
    if (!b || !pixels) return J2K_ERR_INVALID_ARG;
    j2k_ctx* ctx = b->ctx;
    cudaSetDevice(ctx->device);
    for (size_t i = 0; i < b->img.size(); ++i)
        if (!pixels[i]) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "pixel pointer is NULL");
    for (size_t i = 0; i < b->img.size(); ++i) {
        const ImgPlan& im = b->img[i];
        J2K_CUDA(ctx, cudaMemcpyAsync((uint8_t*)b->in.p + im.in_off, pixels[i], im.n * im.d.ncomp,
                                      on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream));
    }
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_batch_encode_async(j2k_batch* b, const uint8_t* const* pixels, int on_device) {
    J2K_API_BEGIN
    if (!b) return J2K_ERR_INVALID_ARG;
    j2k_ctx* ctx = b->ctx;
    cudaSetDevice(ctx->device);
    b->have_result = false;
    b->pending = false;
    if (pixels) J2K_TRY(j2k_batch_upload(b, pixels, on_device));
    J2K_TRY(j2k_clear_device_error(ctx));
    J2K_TRY(run_once(b));
    b->pending = true;
    return J2K_OK;
    J2K_API_END
}

}  // extern "C"

// Reads the device error word of a pending run (one stream synchronisation); a capacity
// overflow grows the tier-1 buffers and re-runs from the input still on the device.
static j2k_status batch_finish(j2k_batch* b) {
    if (!b->pending) return J2K_OK;
    j2k_ctx* ctx = b->ctx;
    b->pending = false;
    for (int attempt = 0; attempt < 6; ++attempt) {
        j2k_status s = j2k_read_device_error(ctx);
        if (s == J2K_OK) {
            b->have_result = (b->stages & 4) != 0;  // code-blocks exist only when tier-1 ran
            return J2K_OK;
        }
        if (s != J2K_ERR_CAPACITY) return s;
        if (ctx->err.find("symbol") != std::string::npos) b->sym_factor *= 2; else b->out_factor *= 2;
        drop_graph(b);
        J2K_TRY(layout_t1(b));
        J2K_TRY(j2k_clear_device_error(ctx));
        J2K_TRY(run_once(b));
    }
    return j2k_fail(ctx, J2K_ERR_CAPACITY, "tier-1 capacities kept overflowing");
}

extern "C" {

j2k_status j2k_batch_encode(j2k_batch* b, const uint8_t* const* pixels, int on_device) {
    J2K_API_BEGIN
    J2K_TRY(j2k_batch_encode_async(b, pixels, on_device));
    return batch_finish(b);
    J2K_API_END
}

// Times each candidate on this batch (CUDA events around the stage it affects) and keeps the
// fastest: DWT tile shape per filter, then phase-A order, then the MQ schedule.
j2k_status j2k_batch_autotune(j2k_batch* b, int reps, int* report) {
    J2K_API_BEGIN
    if (!b) return J2K_ERR_INVALID_ARG;
    j2k_ctx* ctx = b->ctx;
    cudaSetDevice(ctx->device);
    reps = std::max(reps, 1);
    J2K_TRY(batch_finish(b));
    const bool graph = b->use_graph;
    b->use_graph = false;
    drop_graph(b);
    cudaEvent_t e0, e1;
    J2K_CUDA(ctx, cudaEventCreate(&e0));
    J2K_CUDA(ctx, cudaEventCreate(&e1));
    auto time_stage = [&](bool pl, bool dw, bool t1, float* ms) -> j2k_status {
        J2K_TRY(enqueue(b, true, true, true));  // warm / produce inputs of later stages
        J2K_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        float best = 1e30f;
        for (int r = 0; r < reps; ++r) {
            J2K_CUDA(ctx, cudaEventRecord(e0, ctx->stream));
            J2K_TRY(enqueue(b, pl, dw, t1));
            J2K_CUDA(ctx, cudaEventRecord(e1, ctx->stream));
            J2K_CUDA(ctx, cudaEventSynchronize(e1));
            float t = 0;
            J2K_CUDA(ctx, cudaEventElapsedTime(&t, e0, e1));
            best = std::min(best, t);
        }
        *ms = best;
        return j2k_read_device_error(ctx);
    };
    j2k_status s = J2K_OK;
    float t;
    for (int f = 0; f < 2 && s == J2K_OK; ++f) {
        int best_code = 0;
        float best_t = 1e30f;
        for (int code = 0; code < 4 && s == J2K_OK; ++code) {
            b->tile_code[f] = code;
            s = plan_dwt(b);
            if (s == J2K_OK) s = time_stage(false, true, false, &t);
            if (s == J2K_OK && t < best_t) { best_t = t; best_code = code; }
        }
        b->tile_code[f] = best_code;
        if (s == J2K_OK) s = plan_dwt(b);
    }
    // MQ candidates: {variant, blocks per warp, tiered schedule on}; the tiers are the context's
    // (by default one warp per SM with one block, two per SM with four blocks)
    const int cand[7][3] = {{0, 8, 1}, {0, 16, 1}, {0, 32, 1}, {0, 8, 0}, {0, 16, 0}, {0, 32, 0}, {1, 32, 0}};
    int tw[J2K_MQ_TIERS], tl[J2K_MQ_TIERS];
    std::copy(ctx->mq_tier_warps, ctx->mq_tier_warps + J2K_MQ_TIERS, tw);
    std::copy(ctx->mq_tier_lanes, ctx->mq_tier_lanes + J2K_MQ_TIERS, tl);
    auto set_tiers = [&](bool on) {
        for (int k = 0; k < J2K_MQ_TIERS; ++k) {
            ctx->mq_tier_warps[k] = on ? tw[k] : 0;
            ctx->mq_tier_lanes[k] = on ? tl[k] : 0;
        }
    };
    int best_order = 1, best_c = 0;
    float best_t = 1e30f;
    for (int ord = 0; ord < 2 && s == J2K_OK; ++ord)
        for (int c = 0; c < 7 && s == J2K_OK; ++c) {
            b->phase_a_order = ord;
            ctx->mq_variant = cand[c][0];
            ctx->mq_lanes = cand[c][1];
            set_tiers(cand[c][2] != 0);
            s = time_stage(false, false, true, &t);
            if (s == J2K_OK && t < best_t) { best_t = t; best_order = ord; best_c = c; }
        }
    b->phase_a_order = best_order;
    ctx->mq_variant = cand[best_c][0];
    ctx->mq_lanes = cand[best_c][1];
    set_tiers(cand[best_c][2] != 0);
    // phase A's register budget: 2 or 3 resident CTAs per SM
    {
        int best_occ = ctx->t1a_ctas;
        float occ_t = best_t;
        for (int occ = 2; occ <= 3 && s == J2K_OK; ++occ) {
            if (occ == best_occ) continue;
            const int keep = ctx->t1a_ctas;
            ctx->t1a_ctas = occ;
            s = time_stage(false, false, true, &t);
            if (s == J2K_OK && t < occ_t) occ_t = t, best_occ = occ;
            ctx->t1a_ctas = keep;
        }
        ctx->t1a_ctas = best_occ;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->use_graph = graph;
    if (report) {
        report[0] = b->tile_code[0];
        report[1] = b->tile_code[1];
        report[2] = b->phase_a_order;
        report[3] = ctx->mq_variant;
        report[4] = ctx->mq_lanes;
    }
    return s;
    J2K_API_END
}

j2k_status j2k_batch_get_codeblocks(j2k_batch* b, int image, j2k_cb_desc* descs, size_t* count,
                                    uint8_t* bytes, size_t cap, size_t* used) {
    J2K_API_BEGIN
    if (!b || !count || image < 0 || image >= (int)b->img.size()) return J2K_ERR_INVALID_ARG;
    j2k_ctx* ctx = b->ctx;
    J2K_TRY(batch_finish(b));
    if (!b->have_result) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "no batch result yet");
    const ImgPlan& im = b->img[image];
    std::vector<j2k_cb_desc> d(im.njobs);
    J2K_CUDA(ctx, cudaMemcpy(d.data(), (j2k_cb_desc*)b->descs.p + im.job0, im.njobs * sizeof(j2k_cb_desc),
                             cudaMemcpyDeviceToHost));
    size_t total = 0;
    for (auto& x : d) total += (size_t)std::max(x.length, 0);
    if (used) *used = total;
    if (!descs && !bytes) {
        *count = im.njobs;
        return J2K_OK;
    }
    if ((descs && *count < im.njobs) || (bytes && cap < total))
        return j2k_fail(ctx, J2K_ERR_CAPACITY, "output arrays too small");
    *count = im.njobs;
    size_t acc = 0;
    for (size_t i = 0; i < im.njobs; ++i) {
        if (bytes && d[i].length > 0)
            J2K_CUDA(ctx, cudaMemcpyAsync(bytes + acc, (const uint8_t*)b->bytes.p + d[i].offset, d[i].length,
                                          cudaMemcpyDeviceToHost, ctx->stream));
        d[i].offset = (uint32_t)acc;
        acc += (size_t)std::max(d[i].length, 0);
    }
    J2K_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (descs) std::memcpy(descs, d.data(), im.njobs * sizeof(j2k_cb_desc));
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_batch_get_codestream(j2k_batch* b, int image, uint8_t* out, size_t cap, size_t* len) {
    J2K_API_BEGIN
    if (!b || !len) return J2K_ERR_INVALID_ARG;
    size_t count = 0, total = 0;
    J2K_TRY(j2k_batch_get_codeblocks(b, image, nullptr, &count, nullptr, 0, &total));
    std::vector<j2k_cb_desc> d(count);
    std::vector<uint8_t> bytes(total + 1);
    J2K_TRY(j2k_batch_get_codeblocks(b, image, d.data(), &count, bytes.data(), bytes.size(), &total));
    const ImgPlan& im = b->img[image];
    std::vector<j2k_t2_block> blocks(count);
    for (size_t i = 0; i < count; ++i) blocks[i] = j2k_t2_block{d[i].numbps, d[i].npasses, d[i].length, bytes.data() + d[i].offset};
    std::vector<uint8_t> cs = j2k_t2_write(im.d.w, im.d.h, im.d.ncomp, im.d.levels, im.d.cb, im.d.cb,
                                           im.d.kernel == J2K_W53, im.d.ncomp >= 3, im.steps.data(), blocks);
    *len = cs.size();
    if (!out) return J2K_OK;
    if (cap < cs.size()) return j2k_fail(b->ctx, J2K_ERR_CAPACITY, "codestream buffer too small");
    std::memcpy(out, cs.data(), cs.size());
    return J2K_OK;
    J2K_API_END
}

}  // extern "C"


extern "C" {

j2k_status j2k_batch_pack(j2k_batch* b, size_t* total) {
    J2K_API_BEGIN
    if (!b || !total) return J2K_ERR_INVALID_ARG;
    j2k_ctx* ctx = b->ctx;
    cudaSetDevice(ctx->device);
    J2K_TRY(batch_finish(b));
    if (!b->have_result) return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "no batch result yet");
    const int n = (int)b->hjobs.size();
    cudaStream_t st = ctx->stream;
    J2K_TRY(b->plens.ensure(ctx, (size_t)(n + 1) * 4));
    J2K_TRY(b->poffs.ensure(ctx, (size_t)(n + 1) * 4));
    J2K_TRY(b->pdescs.ensure(ctx, (size_t)std::max(n, 1) * sizeof(j2k_cb_desc)));
    batch_lengths_kernel<<<(n + 255) / 256, 256, 0, st>>>((const j2k_cb_desc*)b->descs.p, (uint32_t*)b->plens.p, n);
    J2K_CUDA(ctx, cudaMemsetAsync((uint32_t*)b->plens.p + n, 0, 4, st));
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, (uint32_t*)b->plens.p, (uint32_t*)b->poffs.p, n + 1, st);
    J2K_TRY(b->ptmp.ensure(ctx, tmp + 16));
    J2K_CUDA(ctx, cub::DeviceScan::ExclusiveSum(b->ptmp.p, tmp, (uint32_t*)b->plens.p, (uint32_t*)b->poffs.p,
                                                n + 1, st));
    uint32_t tot = 0;
    J2K_CUDA(ctx, cudaMemcpyAsync(&tot, (uint32_t*)b->poffs.p + n, 4, cudaMemcpyDeviceToHost, st));
    J2K_CUDA(ctx, cudaStreamSynchronize(st));
    J2K_TRY(b->packed.ensure(ctx, (size_t)tot + 16));
    batch_pack_kernel<<<(unsigned)(((size_t)n * 32 + 255) / 256), 256, 0, st>>>(
        (const j2k_cb_desc*)b->descs.p, (const uint32_t*)b->poffs.p, (const uint8_t*)b->bytes.p,
        (uint8_t*)b->packed.p, (j2k_cb_desc*)b->pdescs.p, n);
    J2K_CUDA(ctx, cudaGetLastError());
    b->packed_total = tot;
    *total = tot;
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_batch_read_packed(j2k_batch* b, j2k_cb_desc* descs, uint8_t* bytes, size_t cap) {
    J2K_API_BEGIN
    if (!b || !descs || !bytes) return J2K_ERR_INVALID_ARG;
    j2k_ctx* ctx = b->ctx;
    if (cap < b->packed_total) return j2k_fail(ctx, J2K_ERR_CAPACITY, "bytes buffer smaller than the packed total");
    cudaSetDevice(ctx->device);
    J2K_CUDA(ctx, cudaMemcpyAsync(descs, b->pdescs.p, b->hjobs.size() * sizeof(j2k_cb_desc), cudaMemcpyDeviceToHost,
                                  ctx->stream));
    if (b->packed_total)
        J2K_CUDA(ctx, cudaMemcpyAsync(bytes, b->packed.p, b->packed_total, cudaMemcpyDeviceToHost, ctx->stream));
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_batch_image_jobs(j2k_batch* b, size_t* first) {
    J2K_API_BEGIN
    if (!b || !first) return J2K_ERR_INVALID_ARG;
    for (size_t i = 0; i < b->img.size(); ++i) first[i] = b->img[i].job0;
    first[b->img.size()] = b->hjobs.size();
    return J2K_OK;
    J2K_API_END
}

}  // extern "C"
