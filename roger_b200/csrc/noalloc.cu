// Allocation-free forward DWT entry point.
//
// j2k_dwt_forward needs two intermediate LL buffers (a quarter and a sixteenth of the image)
// and takes them from a j2k_ctx, which allocates them with cudaMalloc on first use.  Some
// callers cannot allocate device memory at all: a plugin hosted inside a framework that owns
// the device heap and forbids allocations outside its pool, or a latency-critical pipeline that
// reserves every byte up front and must not hit cudaMalloc (which can synchronise the device).
// j2k_dwt_forward_noalloc serves them: the intermediate LL bands live in the file-scope array
// below, reserved once in every process that loads the library and held until exit, so the
// call allocates nothing and needs no context.  The caller still passes input and output.
#include <cudaTypedefs.h>

#include <mutex>

#include "j2k_internal.cuh"

namespace {

// Capacity in 4-byte samples: the LL bands of one 2048x2048 level-0 plane
// (1024*1024 + 512*512).  Larger images are rejected.
constexpr size_t kNoallocElems = (size_t)1024 * 1024 + (size_t)512 * 512;

static __device__ __align__(256) uint32_t g_dwt_scratch[kNoallocElems];

constexpr int kMaxDevices = 64;
std::mutex g_mu;

// The array's device address per device, and the id of the CUDA context it was looked up in.
// A cudaDeviceReset destroys the context and unloads the module; the next context gets a new
// id (context ids are unique for the life of the process), so the address is looked up again.
struct ScratchSlot {
    unsigned long long ctx_id;
    void* ptr;
};
ScratchSlot g_slot[kMaxDevices] = {};

// Driver entry points for the current context's id, resolved once through the runtime (no link
// dependency on libcuda).  When they are unavailable the address is looked up on every call.
PFN_cuCtxGetCurrent_v4000 g_get_current = nullptr;
PFN_cuCtxGetId_v12000 g_get_id = nullptr;
bool g_resolved = false;

void resolve_entry_points() {
    if (g_resolved) return;
    g_resolved = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_get_current = (PFN_cuCtxGetCurrent_v4000)f;
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_get_id = (PFN_cuCtxGetId_v12000)f;
    if (!g_get_current || !g_get_id) g_get_current = nullptr, g_get_id = nullptr;
}

// Id of the current context, 0 when there is none yet or it cannot be read.
unsigned long long current_ctx_id() {
    if (!g_get_current) return 0;
    CUcontext c = nullptr;
    if (g_get_current(&c) != CUDA_SUCCESS || !c) return 0;
    unsigned long long id = 0;
    if (g_get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of g_dwt_scratch on `device` (which is current).  In host code the array's
// name is only a host-side stand-in, so the address must come from cudaGetSymbolAddress: once
// per device and context (the first call on a device, and again after a device reset).
j2k_status scratch_address(int device, void** out) {
    if (device < 0 || device >= kMaxDevices) return J2K_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_mu);
    resolve_entry_points();
    ScratchSlot& s = g_slot[device];
    unsigned long long id = current_ctx_id();
    if (id != 0 && s.ptr && s.ctx_id == id) {
        *out = s.ptr;
        return J2K_OK;
    }
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_dwt_scratch);  // loads the module in this context
    if (e != cudaSuccess || !p) return J2K_ERR_CUDA;
    if (id == 0) id = current_ctx_id();  // the lookup made the device's context current
    s.ctx_id = id;
    s.ptr = id != 0 ? p : nullptr;  // without a context id, look it up again next time
    *out = p;
    return J2K_OK;
}

}  // namespace

extern "C" j2k_status j2k_dwt_forward_noalloc(void* cuda_stream, int kernel, int order, const void* in,
                                              size_t in_pitch, void* out, size_t out_pitch, size_t w,
                                              size_t h, int levels, const float* steps) {
    J2K_API_BEGIN
    if (!in || !out || w == 0 || h == 0 || in_pitch < w || out_pitch < w) return J2K_ERR_INVALID_ARG;
    if (w > 0x7FFFFFFF || h > 0x7FFFFFFF) return J2K_ERR_INVALID_ARG;
    if (kernel != J2K_W53 && kernel != J2K_W97) return J2K_ERR_INVALID_ARG;
    if (order != J2K_ORDER_T800 && order != J2K_ORDER_REF) return J2K_ERR_INVALID_ARG;
    if (levels < 0 || levels > 32 || (kernel == J2K_W53 && steps)) return J2K_ERR_INVALID_ARG;
    const size_t w1 = (w + 1) / 2, h1 = (h + 1) / 2, w2 = (w1 + 1) / 2, h2 = (h1 + 1) / 2;
    const size_t need0 = w1 * h1, need1 = w2 * h2;
    if (need0 + need1 > kNoallocElems) return J2K_ERR_CAPACITY;  // beyond the reserved maximum
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return J2K_ERR_CUDA;
    void* base = nullptr;
    j2k_status s = scratch_address(device, &base);
    if (s != J2K_OK) return s;
    // LL of even levels in the first region, odd levels in the second (no clearing needed:
    // every sample is written before it is read)
    void* ll0 = base;
    void* ll1 = (char*)base + ((need0 * 4 + 255) & ~(size_t)255);
    if (((need0 * 4 + 255) & ~(size_t)255) / 4 + need1 > kNoallocElems) ll1 = (char*)base + need0 * 4;
    return j2k_dwt_fwd_impl(nullptr, kernel, order, in, in_pitch, out, out_pitch, w, h, levels, steps, ll0, ll1,
                            j2k_dwt_tile{64, 64}, (cudaStream_t)cuda_stream);
    J2K_API_END
}
