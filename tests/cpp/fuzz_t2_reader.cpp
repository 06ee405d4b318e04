// Mutation fuzzer for the host tier-2 reader (j2k_codestream_info, j2k_codestream_read_layers),
// built with AddressSanitizer and UBSan together with t2.cpp itself.  Each seed codestream given
// on the command line is truncated or has bytes overwritten, set to 0xFF or deleted; every
// mutant must be refused with a status or parse into descriptors whose codeword ranges lie
// inside the returned bytes.  Headers that claim more than 2^20 code-blocks are only sized.
// Every parsed mutant is also written back as one layer by j2k_codestream_write (which may
// refuse blocks the writer does not produce, e.g. a cut inside a bit-plane); a written stream
// must read back to the same blocks and codeword bytes.
// Prints "parsed P refused R huge H rewritten W" and exits 0; a sanitizer report, a bad
// descriptor or a round trip that differs ends it with a non-zero status.
#include <algorithm>
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
    size_t parsed = 0, refused = 0, huge = 0, rewritten = 0;
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
            // write the parsed blocks back (one layer) and read them again
            size_t wl = 0;
            const float* st = info.lossless ? nullptr : info.steps;
            if (j2k_codestream_write(info.w, info.h, info.ncomp, info.levels, info.cbw, info.cbh, info.lossless, st,
                                     d.data(), cnt, b.data(), used, 1, nullptr, nullptr, nullptr, 0, &wl) != J2K_OK)
                continue;
            std::vector<uint8_t> w2(wl);
            if (j2k_codestream_write(info.w, info.h, info.ncomp, info.levels, info.cbw, info.cbh, info.lossless, st,
                                     d.data(), cnt, b.data(), used, 1, nullptr, nullptr, w2.data(), w2.size(),
                                     &wl) != J2K_OK) {
                std::printf("second write of mutant %d of %s failed\n", it, argv[s]);
                return 1;
            }
            j2k_stream_info i2;
            size_t c2 = 0, u2 = 0;
            if (j2k_codestream_read_layers(w2.data(), wl, 0, &i2, nullptr, &c2, nullptr, 0, &u2, err, sizeof err) !=
                    J2K_OK || c2 != cnt || u2 != used) {
                std::printf("written stream of mutant %d of %s does not read back: %s\n", it, argv[s], err);
                return 1;
            }
            std::vector<j2k_cb_desc> d2(c2 + 1);
            std::vector<uint8_t> b2(u2 + 1);
            if (j2k_codestream_read_layers(w2.data(), wl, 0, &i2, d2.data(), &c2, b2.data(), b2.size(), &u2, err,
                                           sizeof err) != J2K_OK) {
                std::printf("written stream of mutant %d of %s does not read back: %s\n", it, argv[s], err);
                return 1;
            }
            for (size_t i = 0; i < cnt; ++i)
                if (d2[i].numbps != d[i].numbps || d2[i].npasses != d[i].npasses || d2[i].length != d[i].length ||
                    !std::equal(b.begin() + d[i].offset, b.begin() + d[i].offset + d[i].length,
                                b2.begin() + d2[i].offset)) {
                    std::printf("block %zu of mutant %d of %s differs after the round trip\n", i, it, argv[s]);
                    return 1;
                }
            ++rewritten;
        }
    }
    std::printf("parsed %zu refused %zu huge %zu rewritten %zu\n", parsed, refused, huge, rewritten);
    return 0;
}
