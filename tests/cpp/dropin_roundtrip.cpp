// Exercises the header-only C++ drop-in the way the reference's harness uses its OpenCL
// classes (src/OCLTest.cpp:80-120): planar level-shifted components -> OCLEncoder<short>::run
// -> code-blocks -> OCLDecoder<short>::run, and requires the exact pixels back.  Also runs
// OCLDWTForward / OCLDWTRev over the shared memory manager.  Exit code 0 = pass.
#include <cstdio>
#include <vector>

#include "roger_b200/ocl_dropin.hpp"

using namespace roger_b200;

int main(int argc, char** argv) {
    const size_t w = argc > 1 ? std::atoi(argv[1]) : 301, h = argc > 2 ? std::atoi(argv[2]) : 197;
    const size_t levels = 5;
    std::vector<unsigned char> rgb(w * h * 3);
    for (size_t y = 0; y < h; ++y)
        for (size_t x = 0; x < w; ++x)
            for (int c = 0; c < 3; ++c)
                rgb[(y * w + x) * 3 + c] = (unsigned char)((x * (3 + c) + y * (5 - c) + ((x * y) >> (c + 2))) & 255);
    std::vector<std::vector<short>> planes(3, std::vector<short>(w * h));
    for (size_t i = 0; i < w * h; ++i)
        for (int c = 0; c < 3; ++c) planes[c][i] = (short)(rgb[i * 3 + c] - 128);  // level shift
    std::vector<short*> comps = {planes[0].data(), planes[1].data(), planes[2].data()};
    try {
        DeviceContext dev(0);
        OCLEncoder<short> enc(&dev, false, false);
        enc.run(comps, w, h, levels, 8);
        std::vector<j2k_cb_desc> descs;
        std::vector<uint8_t> bytes;
        enc.codeblocks(&descs, &bytes);
        std::vector<uint8_t> cs = enc.codestream();
        OCLDecoder<short> dec(&dev, false);
        std::vector<uint8_t> out = dec.run(descs, bytes, w, h, 3, levels);
        if (out != rgb) {
            std::fprintf(stderr, "round trip mismatch\n");
            return 1;
        }
        if (cs.size() < 100 || cs[0] != 0xFF || cs[1] != 0x4F) {
            std::fprintf(stderr, "bad codestream\n");
            return 1;
        }
        std::printf("ok %zu blocks, %zu codeword bytes, %zu codestream bytes\n", descs.size(), bytes.size(),
                    cs.size());
    } catch (const Error& e) {
        std::fprintf(stderr, "error %d: %s\n", e.status, e.what());
        return 1;
    }
    return 0;
}
