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
#include <mutex>

#include "j2k_internal.cuh"

namespace {

// Capacity in 4-byte samples: the LL bands of one 2048x2048 level-0 plane
// (1024*1024 + 512*512).  Larger images are rejected.
constexpr size_t kNoallocElems = (size_t)1024 * 1024 + (size_t)512 * 512;

static __device__ __align__(256) uint32_t g_dwt_scratch[kNoallocElems];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_dwt_scratch on `device` (which is current).  In host code the array's
// name is only a host-side stand-in, so the address must come from cudaGetSymbolAddress, once
// per device.
j2k_status scratch_address(int device, void** out) {
    if (device < 0 || device >= kMaxDevices) return J2K_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_dwt_scratch);
        if (e != cudaSuccess || !p) return J2K_ERR_CUDA;
        g_scratch_ptr[device] = p;
    }
    *out = g_scratch_ptr[device];
    return J2K_OK;
}

}  // namespace

extern "C" j2k_status j2k_dwt_forward_noalloc(void* cuda_stream, int kernel, int order, const void* in,
                                              size_t in_pitch, void* out, size_t out_pitch, size_t w,
                                              size_t h, int levels, const float* steps) {
    J2K_API_BEGIN
    if (!in || !out || w == 0 || h == 0 || in_pitch < w || out_pitch < w) return J2K_ERR_INVALID_ARG;
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
