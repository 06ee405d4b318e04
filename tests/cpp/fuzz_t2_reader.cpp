// Mutation fuzzer for the host tier-2 reader (j2k_codestream_info, j2k_codestream_read_layers),
// built with AddressSanitizer and UBSan together with t2.cpp itself.  Each seed codestream given
// on the command line is truncated or has bytes overwritten, set to 0xFF or deleted; every
// mutant must be refused with a status or parse into descriptors whose codeword ranges lie
// inside the returned bytes.  Headers that claim more than 2^20 code-blocks are only sized.
// Prints "parsed P refused R huge H" and exits 0; a sanitizer report or a bad descriptor ends
// it with a non-zero status.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iterator>
#include <random>
#include <vector>

#include "j2k_b200.h"

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s iterations seed.j2k...\n", argv[0]);
        return 2;
    }
    const int iters = std::atoi(argv[1]);
    size_t parsed = 0, refused = 0, huge = 0;
    for (int s = 2; s < argc; ++s) {
        std::ifstream f(argv[s], std::ios::binary);
        const std::vector<uint8_t> cs((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
        std::mt19937_64 rng(7919u * (unsigned)s);
        for (int it = 0; it < iters; ++it) {
            std::vector<uint8_t> m = cs;
            if (it % 5 == 0) {
                m.resize(rng() % (m.size() + 1));
            } else {
                const int k = 1 + (int)(rng() % 5);
                for (int q = 0; q < k && !m.empty(); ++q) {
                    // the first 200 bytes (the main header) are hit as often as the rest
                    const size_t hi = (rng() & 1) ? std::min<size_t>(m.size(), 200) : m.size();
                    const size_t p = rng() % hi;
                    const int kind = (int)(rng() % 10);
                    if (kind < 6) m[p] = (uint8_t)rng();
                    else if (kind < 8) m[p] = 0xFF;
                    else m.erase(m.begin() + p, m.begin() + std::min(m.size(), p + 1 + rng() % 8));
                }
            }
            j2k_stream_info info;
            char err[256];
            if (j2k_codestream_info(m.data(), m.size(), &info, err, sizeof err) != J2K_OK) {
                ++refused;
                continue;
            }
            size_t nb = 0;
            for (int c = 0; c < info.ncomp; ++c)
                nb += (size_t)((info.w + info.cbw - 1) / info.cbw) * (size_t)((info.h + info.cbh - 1) / info.cbh);
            if (nb > ((size_t)1 << 20)) {
                ++huge;
                continue;
            }
            size_t cnt = 0, used = 0;
            if (j2k_codestream_read_layers(m.data(), m.size(), 0, &info, nullptr, &cnt, nullptr, 0, &used, err,
                                           sizeof err) != J2K_OK) {
                ++refused;
                continue;
            }
            std::vector<j2k_cb_desc> d(cnt + 1);
            std::vector<uint8_t> b(used + 1);
            if (j2k_codestream_read_layers(m.data(), m.size(), 0, &info, d.data(), &cnt, b.data(), b.size(), &used,
                                           err, sizeof err) != J2K_OK) {
                ++refused;
                continue;
            }
            for (size_t i = 0; i < cnt; ++i)
                if (d[i].length < 0 || (size_t)d[i].offset + (size_t)d[i].length > used || d[i].numbps > 31 ||
                    d[i].npasses > 3 * d[i].numbps) {
                    std::printf("bad descriptor %zu of mutant %d of %s\n", i, it, argv[s]);
                    return 1;
                }
            ++parsed;
        }
    }
    std::printf("parsed %zu refused %zu huge %zu\n", parsed, refused, huge);
    return 0;
}
