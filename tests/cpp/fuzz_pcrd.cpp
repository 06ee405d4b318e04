// Random-input fuzzer for PCRD-opt (rate.cpp: j2k_pcrd_hulls and j2k_pcrd_truncate), built with
// AddressSanitizer and UBSan together with rate.cpp itself.  Block sets of 0 to 9000 blocks (so
// that the threaded hull build runs too) get random bit-plane counts (0..31), pass counts up to
// 3*numbps, lengths, plane-end byte positions (not necessarily increasing), distortions (zeros
// and repeats included) and weights; every budget from 0 to past the total must give a cut that
// keeps whole passes, stays within the block's codeword, and fits the budget.  Prints "cuts N"
// and exits 0.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "j2k_internal.cuh"

int main(int argc, char** argv) {
    const int sets = argc > 1 ? std::atoi(argv[1]) : 50;
    std::mt19937_64 rng(777);
    long cuts = 0;
    for (int t = 0; t < sets; ++t) {
        const size_t n = t % 10 == 9 ? 4096 + rng() % 5000 : rng() % 700;
        std::vector<j2k_cb_desc> d(n);
        std::vector<uint32_t> pb(n * 32);
        std::vector<double> dist(n * 33), w(n);
        size_t full = 0;
        for (size_t i = 0; i < n; ++i) {
            d[i] = j2k_cb_desc{};
            const int nb = (int)(rng() % 32);
            d[i].numbps = (uint8_t)nb;
            d[i].npasses = (uint8_t)(nb ? rng() % (3 * nb + 1) : 0);
            d[i].length = (int32_t)(rng() % 5000);
            full += (size_t)d[i].length;
            for (int k = 0; k < 32; ++k) pb[i * 32 + k] = (uint32_t)(rng() % 6000);
            if (rng() % 16 == 0) {  // coded passes with no bytes (a codeword of length 0)
                d[i].length = 0;
                for (int k = 0; k < 32; ++k) pb[i * 32 + k] = 0;
            }
            for (int k = 0; k < 33; ++k) dist[i * 33 + k] = (rng() % 4 == 0) ? 0.0 : (double)(rng() % 1000000);
            w[i] = (rng() % 8 == 0) ? 0.0 : 0.1 + (double)(rng() % 100) / 10.0;
        }
        for (size_t budget : {(size_t)0, full / 10, full / 3, full / 2, full, full + 1000}) {
            std::vector<j2k_cb_desc> c = d;
            if (j2k_pcrd_truncate(n ? c.data() : nullptr, n, n ? pb.data() : nullptr, n ? dist.data() : nullptr,
                                  n ? w.data() : nullptr, budget) != J2K_OK) {
                std::printf("set %d: refused\n", t);
                return 1;
            }
            size_t kept = 0;
            for (size_t i = 0; i < n; ++i) {
                const int np = c[i].npasses;
                if (np > d[i].npasses || (np && np % 3 != 1) || c[i].length < 0 || c[i].length > d[i].length ||
                    (np == 0 && c[i].length != 0) || (np != 0 && c[i].length == 0)) {
                    std::printf("set %d block %zu: bad cut (%d passes, %d bytes)\n", t, i, np, c[i].length);
                    return 1;
                }
                kept += (size_t)c[i].length;
            }
            if (kept > budget && kept > 0) {
                std::printf("set %d: %zu bytes kept for a budget of %zu\n", t, kept, budget);
                return 1;
            }
            ++cuts;
        }
    }
    std::printf("cuts %ld\n", cuts);
    return 0;
}
