// Header-only C++ drop-in for knopkem/roger's operator classes, over the j2k_b200 C ABI.
//
// The class names, template parameter and method signatures follow the reference:
//   OCLEncodeDecode<T>   src/OCLEncodeDecode.h:23-38 (mapDWTOut, unmapDWTOut, finish)
//   OCLEncoder<T>        src/OCLEncoder.h:27-37      (run(components, w, h, levels, precision))
//   OCLDecoder<T>        src/OCLDecoder.h:25-34
//   OCLDWTForward<T>     src/OCLDWTForward.h:31      (run(lossy, w, h, windowX, windowY, level, levels))
//   OCLDWTRev<T>         src/OCLDWTRev.h:31          (run(lossy, w, h, windowX, windowY))
//   OCLRGBtoPlanar<T>    src/OCLRGBtoPlanar.h:28     (run())
//   OCLBPC<T>            src/OCLBPC.h:28             (run(codeblockX, codeblockY))
//   OCLMemoryManager<T>  src/OCLMemoryManager.h:24-88 (device planes shared by the operators)
// `ocl_args_d_t` (src/OCLUtil.h:31-39) becomes DeviceContext; tDeviceRC/DeviceSuccess
// (src/ocl_platform.h:22-24) map to j2k_status/J2K_OK.  Unlike the reference, failures are not
// swallowed: run() methods throw roger_b200::Error carrying the status and message.
// T is the host component type of the reference's harness (short or float, level-shifted).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../j2k_b200.h"

namespace roger_b200 {

typedef j2k_status tDeviceRC;
static const tDeviceRC DeviceSuccess = J2K_OK;

struct Error : std::runtime_error {
    tDeviceRC status;
    Error(tDeviceRC s, const std::string& m) : std::runtime_error(m), status(s) {}
};

class DeviceContext {
public:
    explicit DeviceContext(int device = 0) {
        tDeviceRC s = j2k_ctx_create(device, &ctx_);
        if (s != J2K_OK) throw Error(s, "j2k_ctx_create failed");
    }
    ~DeviceContext() { if (ctx_) j2k_ctx_destroy(ctx_); }
    DeviceContext(const DeviceContext&) = delete;
    DeviceContext& operator=(const DeviceContext&) = delete;
    j2k_ctx* get() const { return ctx_; }
    void check(tDeviceRC s) const {
        if (s != J2K_OK) throw Error(s, std::string(j2k_status_string(s)) + ": " + j2k_last_error(ctx_));
    }
private:
    j2k_ctx* ctx_ = nullptr;
};

template <typename T> struct dtype_of;
template <> struct dtype_of<short> { static const int value = J2K_I16; };
template <> struct dtype_of<int> { static const int value = J2K_I32; };
template <> struct dtype_of<float> { static const int value = J2K_F32; };

// Device planes shared by the stage operators (the OCLMemoryManager<T> role).
template <typename T> class OCLMemoryManager {
public:
    OCLMemoryManager(DeviceContext* ocl, bool lossy, bool outputDwt)
        : ocl_(ocl), lossy_(lossy), onlyDwtOut_(outputDwt) {}
    ~OCLMemoryManager() { release(); }
    // uploads level-shifted planar host components; int32 planes for 5/3, float for 9/7
    void init(std::vector<T*> components, size_t w, size_t h, size_t levels, size_t precision) {
        width_ = w; height_ = h; levels_ = levels; precision_ = precision;
        numComponents_ = components.size();
        size_t n = w * h;
        ensure(&dwtIn_, &inBytes_, n * 4 * numComponents_);
        ensure(&dwtOut_, &outBytes_, n * 4 * numComponents_);
        std::vector<float> tmpf;
        std::vector<int32_t> tmpi;
        for (size_t c = 0; c < numComponents_; ++c) {
            const T* src = components[c];
            char* dst = (char*)dwtIn_ + c * n * 4;
            if (lossy_) {
                tmpf.assign(src, src + n);
                ocl_->check(cudaMemcpy(dst, tmpf.data(), n * 4, cudaMemcpyHostToDevice) == cudaSuccess
                                ? J2K_OK : J2K_ERR_CUDA);
            } else {
                tmpi.assign(src, src + n);
                ocl_->check(cudaMemcpy(dst, tmpi.data(), n * 4, cudaMemcpyHostToDevice) == cudaSuccess
                                ? J2K_OK : J2K_ERR_CUDA);
            }
        }
    }
    size_t getWidth() const { return width_; }
    size_t getHeight() const { return height_; }
    size_t getNumLevels() const { return levels_; }
    size_t getPrecision() const { return precision_; }
    size_t getNumComponents() const { return numComponents_; }
    bool isOnlyDwtOut() const { return onlyDwtOut_; }
    bool isLossy() const { return lossy_; }
    void* getDwtIn(size_t channel = 0) const { return (char*)dwtIn_ + channel * width_ * height_ * 4; }
    void* getDWTOutByChannel(size_t channel) const {
        return channel < numComponents_ ? (char*)dwtOut_ + channel * width_ * height_ * 4 : nullptr;
    }
    DeviceContext* context() const { return ocl_; }
private:
    void ensure(void** p, size_t* have, size_t bytes) {
        if (*have >= bytes) return;
        if (*p) cudaFree(*p);
        *p = nullptr;
        if (cudaMalloc(p, bytes) != cudaSuccess) throw Error(J2K_ERR_OUT_OF_MEMORY, "cudaMalloc failed");
        *have = bytes;
    }
    void release() {
        if (dwtIn_) cudaFree(dwtIn_);
        if (dwtOut_) cudaFree(dwtOut_);
        dwtIn_ = dwtOut_ = nullptr;
    }
    DeviceContext* ocl_;
    bool lossy_, onlyDwtOut_;
    size_t width_ = 0, height_ = 0, levels_ = 0, precision_ = 8, numComponents_ = 0;
    void *dwtIn_ = nullptr, *dwtOut_ = nullptr;
    size_t inBytes_ = 0, outBytes_ = 0;
};

// Forward DWT of every component of the memory manager (dwtIn -> dwtOut), all levels from
// `level`.  The window sizes were the OpenCL work-group shape and are ignored.
template <typename T> class OCLDWTForward {
public:
    OCLDWTForward(DeviceContext* ocl, OCLMemoryManager<T>* memMgr, int order = J2K_ORDER_REF)
        : ocl_(ocl), mm_(memMgr), order_(order) {}
    void run(bool lossy, size_t w, size_t h, size_t /*windowX*/, size_t /*windowY*/, size_t level,
             size_t levels, const float* steps = nullptr) {
        for (size_t c = 0; c < mm_->getNumComponents(); ++c)
            ocl_->check(j2k_dwt_forward(ocl_->get(), lossy ? J2K_W97 : J2K_W53, order_, mm_->getDwtIn(c), w,
                                        mm_->getDWTOutByChannel(c), w, w, h, (int)(levels - level), steps));
    }
private:
    DeviceContext* ocl_;
    OCLMemoryManager<T>* mm_;
    int order_;
};

// True inverse DWT (the reference's "reverse" kernels are forward transforms): dwtOut -> dwtIn.
template <typename T> class OCLDWTRev {
public:
    OCLDWTRev(DeviceContext* ocl, OCLMemoryManager<T>* memMgr, int order = J2K_ORDER_REF)
        : ocl_(ocl), mm_(memMgr), order_(order) {}
    void run(bool lossy, size_t w, size_t h, size_t /*windowX*/, size_t /*windowY*/,
             const float* steps = nullptr) {
        for (size_t c = 0; c < mm_->getNumComponents(); ++c)
            ocl_->check(j2k_dwt_inverse(ocl_->get(), lossy ? J2K_W97 : J2K_W53, order_,
                                        mm_->getDWTOutByChannel(c), w, mm_->getDwtIn(c), w, w, h,
                                        (int)mm_->getNumLevels(), steps));
    }
private:
    DeviceContext* ocl_;
    OCLMemoryManager<T>* mm_;
    int order_;
};

// Interleaved uint8 device image -> planes of the memory manager (+ level shift + RCT/ICT).
template <typename T> class OCLRGBtoPlanar {
public:
    OCLRGBtoPlanar(DeviceContext* ocl, OCLMemoryManager<T>* memMgr) : ocl_(ocl), mm_(memMgr) {}
    void run(const uint8_t* interleaved_device, int ncomp) {
        size_t w = mm_->getWidth(), h = mm_->getHeight();
        int mct = ncomp >= 3 ? (mm_->isLossy() ? J2K_MCT_ICT : J2K_MCT_RCT) : J2K_MCT_NONE;
        ocl_->check(j2k_rgb_to_planar(ocl_->get(), interleaved_device, w * ncomp, ncomp, mct,
                                      mm_->isLossy() ? J2K_F32 : J2K_I32, mm_->getDwtIn(0), w, w * h, w, h));
    }
private:
    DeviceContext* ocl_;
    OCLMemoryManager<T>* mm_;
};

// EBCOT tier-1 of one component's coefficient plane; results stay on the device.
template <typename T> class OCLBPC {
public:
    OCLBPC(DeviceContext* ocl, OCLMemoryManager<T>* memMgr) : ocl_(ocl), mm_(memMgr) {}
    ~OCLBPC() {
        if (descs_) cudaFree(descs_);
        if (bytes_) cudaFree(bytes_);
    }
    void run(size_t codeblockX, size_t codeblockY, size_t channel = 0) {
        size_t w = mm_->getWidth(), h = mm_->getHeight();
        int L = (int)mm_->getNumLevels();
        count_ = j2k_codeblock_count(w, h, L, (int)codeblockX, (int)codeblockY);
        cap_ = ((codeblockX * codeblockY * 2 + 256) + 15) / 16 * 16;
        if (descs_) cudaFree(descs_);
        if (bytes_) cudaFree(bytes_);
        if (cudaMalloc(&descs_, count_ * sizeof(j2k_cb_desc)) != cudaSuccess ||
            cudaMalloc(&bytes_, count_ * cap_) != cudaSuccess)
            throw Error(J2K_ERR_OUT_OF_MEMORY, "cudaMalloc failed");
        ocl_->check(j2k_bpc_encode(ocl_->get(), (const int32_t*)mm_->getDWTOutByChannel(channel), w, w, h, L,
                                   (int)codeblockX, (int)codeblockY, descs_, bytes_, cap_));
    }
    const j2k_cb_desc* deviceDescs() const { return descs_; }
    const uint8_t* deviceBytes() const { return bytes_; }
    size_t count() const { return count_; }
private:
    DeviceContext* ocl_;
    OCLMemoryManager<T>* mm_;
    j2k_cb_desc* descs_ = nullptr;
    uint8_t* bytes_ = nullptr;
    size_t count_ = 0, cap_ = 0;
};

template <typename T> class OCLEncodeDecode {
public:
    OCLEncodeDecode(DeviceContext* ocl, bool isLossy, bool outputDwt)
        : _ocl(ocl), lossy(isLossy), outputDwt_(outputDwt) {}
    virtual ~OCLEncodeDecode() {}
    void finish() { _ocl->check(j2k_stream_sync(_ocl->get())); }
protected:
    DeviceContext* _ocl;
    bool lossy;
    bool outputDwt_;
};

template <typename T> class OCLEncoder : public OCLEncodeDecode<T> {
public:
    OCLEncoder(DeviceContext* ocl, bool isLossy, bool outputDwt) : OCLEncodeDecode<T>(ocl, isLossy, outputDwt) {
        this->_ocl->check(j2k_encoder_create(ocl->get(), isLossy, outputDwt, &enc_));
    }
    ~OCLEncoder() { if (enc_) j2k_encoder_destroy(enc_); }
    // components: planar, level-shifted (pixel - 128), 1 or 3 of them (src/OCLTest.cpp:80-90)
    void run(std::vector<T*> components, size_t w, size_t h, size_t levels, size_t precision,
             const j2k_enc_params* params = nullptr) {
        std::vector<const void*> p(components.begin(), components.end());
        this->_ocl->check(j2k_encoder_run(enc_, p.data(), (int)p.size(), dtype_of<T>::value, w, h, levels,
                                          precision, params));
    }
    tDeviceRC mapDWTOut(void** mappedPtr, size_t* pitchBytes = nullptr) {
        return j2k_encoder_map_dwt_out(enc_, mappedPtr, pitchBytes);
    }
    tDeviceRC unmapDWTOut(void* mappedPtr) { return j2k_encoder_unmap_dwt_out(enc_, mappedPtr); }
    void codeblocks(std::vector<j2k_cb_desc>* descs, std::vector<uint8_t>* bytes) {
        size_t n = 0, used = 0;
        this->_ocl->check(j2k_encoder_get_codeblocks(enc_, nullptr, &n, nullptr, 0, &used));
        descs->resize(n);
        bytes->resize(used + 1);
        this->_ocl->check(j2k_encoder_get_codeblocks(enc_, descs->data(), &n, bytes->data(), bytes->size(), &used));
        bytes->resize(used);
    }
    std::vector<uint8_t> codestream() {
        size_t n = 0;
        this->_ocl->check(j2k_encoder_get_codestream(enc_, nullptr, 0, &n));
        std::vector<uint8_t> out(n);
        this->_ocl->check(j2k_encoder_get_codestream(enc_, out.data(), out.size(), &n));
        return out;
    }
    j2k_encoder* handle() const { return enc_; }
private:
    j2k_encoder* enc_ = nullptr;
};

template <typename T> class OCLDecoder : public OCLEncodeDecode<T> {
public:
    OCLDecoder(DeviceContext* ocl, bool isLossy) : OCLEncodeDecode<T>(ocl, isLossy, false) {
        this->_ocl->check(j2k_decoder_create(ocl->get(), isLossy, &dec_));
    }
    ~OCLDecoder() { if (dec_) j2k_decoder_destroy(dec_); }
    // decodes code-blocks (as returned by OCLEncoder::codeblocks) to interleaved uint8 pixels
    std::vector<uint8_t> run(const std::vector<j2k_cb_desc>& descs, const std::vector<uint8_t>& bytes,
                             size_t w, size_t h, int ncomp, size_t levels, const j2k_enc_params* params = nullptr) {
        std::vector<uint8_t> out(w * h * ncomp);
        j2k_enc_params p{};
        if (params) p = *params;
        p.levels = (int)levels;
        this->_ocl->check(j2k_decoder_run_codeblocks(dec_, descs.data(), bytes.data(), bytes.size(), 0, ncomp, w,
                                                     h, &p, out.data(), 0, w * ncomp));
        return out;
    }
private:
    j2k_decoder* dec_ = nullptr;
};

}  // namespace roger_b200
