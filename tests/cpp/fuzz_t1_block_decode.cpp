// Random-input fuzzer for the tier-1 block decoder, through its host entry point
// j2k_t1_decode_block_host, which runs the same __host__ __device__ decode_block_steps as the
// default device kernel.  Built with AddressSanitizer and UBSan together with t1dec.cu itself.  Each block gets
// a random size (1..64 a side, at most 4096 samples), orientation, bit-plane count, a pass count
// the kernel's descriptor check admits (0..3*numbps) and a codeword of random, all-0xFF or
// sparse bytes held in a buffer of exactly its length, so that any read past the codeword's end
// is a sanitizer report.  Every other block is decoded as coded in a random code-block style
// with random pass ends (j2k_t1_decode_block_styled_host); the others by both unstyled forms,
// which must give the same output.  Prints "decoded N" and exits 0.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

extern "C" int j2k_t1_decode_block_host(const uint8_t* data, int len, int numbps, int npasses, int orient,
                                        int cw, int ch, int32_t* out, size_t pitch);
extern "C" int j2k_t1_decode_block_steps_host(const uint8_t* data, int len, int numbps, int npasses, int orient,
                                              int cw, int ch, int32_t* out, size_t pitch);
extern "C" int j2k_t1_decode_block_styled_host(const uint8_t* data, int len, const uint32_t* pass_ends, int numbps,
                                               int npasses, int orient, int style, int cw, int ch, int32_t* out,
                                               size_t pitch);

int main(int argc, char** argv) {
    const int iters = argc > 1 ? std::atoi(argv[1]) : 1000;
    std::mt19937_64 rng(12345);
    const int sizes[] = {4, 8, 16, 32, 64};
    int decoded = 0;
    for (int it = 0; it < iters; ++it) {
        const int cw = (rng() % 3 == 0) ? 1 + (int)(rng() % 64) : sizes[rng() % 5];
        const int ch = (rng() % 3 == 0) ? 1 + (int)(rng() % 64) : sizes[rng() % 5];
        if (cw * ch > 4096) continue;
        const int numbps = (int)(rng() % 32);
        const int npasses = numbps ? (int)(rng() % (3 * numbps + 1)) : 0;
        const int len = (rng() % 4 == 0) ? (int)(rng() % 8) : (int)(rng() % 6000);
        std::vector<uint8_t> data(len);
        const int mode = (int)(rng() % 3);
        for (auto& b : data) b = mode == 0 ? (uint8_t)rng() : mode == 1 ? 0xFF : (uint8_t)(rng() & 0x8F);
        std::vector<int32_t> out((size_t)ch * cw);
        if (it % 2 == 1 && npasses <= 91) {
            // a code-block style, with pass ends that need not make sense (out of order, past
            // the codeword, zero)
            std::vector<uint32_t> pe(92);
            uint32_t at = 0;
            for (auto& e : pe) {
                const int k = (int)(rng() % 8);
                e = k == 0 ? (uint32_t)rng() : k == 1 ? 0u : (at += (uint32_t)(rng() % 200));
            }
            if (j2k_t1_decode_block_styled_host(len ? data.data() : nullptr, len, pe.data(), numbps, npasses,
                                                (int)(rng() % 4), 1 + (int)(rng() % 7), cw, ch, out.data(),
                                                (size_t)cw) != 0) {
                std::printf("refused styled block %d\n", it);
                return 1;
            }
        } else {
            // the default per-lane loops and the one-symbol-per-step loop on the same block must
            // agree, bit for bit, whatever the bytes
            const int orient = (int)(rng() % 4);
            std::vector<int32_t> out2((size_t)ch * cw);
            if (j2k_t1_decode_block_host(len ? data.data() : nullptr, len, numbps, npasses, orient, cw, ch, out.data(),
                                         (size_t)cw) != 0 ||
                j2k_t1_decode_block_steps_host(len ? data.data() : nullptr, len, numbps, npasses, orient, cw, ch,
                                               out2.data(), (size_t)cw) != 0) {
                std::printf("refused block %d\n", it);
                return 1;
            }
            if (out != out2) {
                std::printf("decoder forms differ on block %d\n", it);
                return 1;
            }
        }
        ++decoded;
    }
    std::printf("decoded %d\n", decoded);
    return 0;
}
