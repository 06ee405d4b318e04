// Rate control: post-compression rate-distortion optimised truncation (PCRD-opt) of the
// code-blocks to a byte budget, single quality layer.  No counterpart in the reference.
//
// Truncation points of a block are the ends of its bit-planes (after each cleanup pass:
// npasses = 1, 4, 7, ..., 3nb-2) and "nothing" (npasses = 0).  At the end of bit-plane k the
// kept length is the bytes the MQ coder had produced (the last one still open to a carry) plus
// J2K_TRUNC_EXTRA bytes of the finished codeword, which covers what the MQ decoder reads ahead
// of the encoder; the decoder reconstructs the undecoded low bits at the middle of their
// interval.  Distortions are squared errors in coefficient units, weighted by the squared norm
// of the subband's synthesis basis (and the step squared for quantised coefficients), so that
// blocks of different bands compare in image units.  Each block's points are reduced to their
// lower convex hull; over all hull segments in order of decreasing slope, those before the first
// one that no longer fits the budget are kept (a threshold on the slope, found by a weighted
// selection), so that every block keeps a prefix of its hull.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <thread>
#include <vector>

#include "j2k_internal.cuh"

namespace {

// one level of the 1-D inverse lifting (linear 5/3 or 9/7) of s (low) and d (high) -> x
void inv_level(std::vector<double>& x, const std::vector<double>& lo, const std::vector<double>& hi, int kernel) {
    const int n = (int)(lo.size() + hi.size());
    x.assign(n, 0.0);
    for (size_t i = 0; i < lo.size(); ++i) x[2 * i] = lo[i];
    for (size_t i = 0; i < hi.size(); ++i) x[2 * i + 1] = hi[i];
    auto at = [&](int i) {  // whole-sample symmetric extension
        if (n == 1) return 0;
        const int p = 2 * (n - 1);
        i %= p;
        if (i < 0) i += p;
        return i >= n ? p - i : i;
    };
    auto step = [&](int parity, double c) {
        for (int i = parity; i < n; i += 2) x[i] += c * (x[at(i - 1)] + x[at(i + 1)]);
    };
    if (kernel == J2K_W53) {
        step(0, -0.25);
        step(1, 0.5);
    } else {
        const double P1 = -1.586134342, U1 = -0.05298011854, P2 = 0.8829110762, U2 = 0.4435068522,
                     K = 1.230174104914;
        for (int i = 0; i < n; ++i) x[i] *= (i & 1) ? 1.0 / K : K;
        step(0, -U2);
        step(1, -P2);
        step(0, -U1);
        step(1, -P1);
    }
}

// squared norm of the 1-D synthesis basis of a coefficient in the low (high = false) or high
// band of decomposition level `lev` (1 = finest), computed from an impulse far from the edges
double gain_1d(int kernel, int lev, bool high) {
    const int n = 64 << lev;
    std::vector<double> lo(n >> lev, 0.0), hi;
    int cur = lev;
    // band of level lev: impulse at the middle of its low or high half
    std::vector<double> bl(n >> lev, 0.0), bh(n >> lev, 0.0);
    (high ? bh : bl)[(n >> lev) / 2] = 1.0;
    std::vector<double> x;
    inv_level(x, bl, bh, kernel);
    for (cur = lev - 1; cur >= 1; --cur) {
        std::vector<double> z(x.size(), 0.0), y;
        inv_level(y, x, z, kernel);
        x.swap(y);
    }
    double s = 0.0;
    for (double v : x) s += v * v;
    return s;
}

}  // namespace

double j2k_band_gain(int kernel, int levels, int band) {
    if (band == 0) {
        const double g = gain_1d(kernel, levels, false);
        return g * g;
    }
    const int lev = levels - (band - 1) / 3;  // decomposition level of the band
    const int o = (band - 1) % 3;             // 0 HL, 1 LH, 2 HH
    const double gl = gain_1d(kernel, lev, false), gh = gain_1d(kernel, lev, true);
    return o == 0 ? gh * gl : (o == 1 ? gl * gh : gh * gh);
}

extern "C" void j2k_pcrd_truncate(j2k_cb_desc* descs, size_t n, const uint32_t* plane_bytes, const double* dist,
                                  const double* weight, size_t budget) {
    // hull points of every block: block i owns slots [i * 33, i * 33 + cnt[i]) (scratch kept per
    // thread between calls); the blocks' hulls are independent and built on host threads
    static thread_local std::vector<double> HL, HD;
    static thread_local std::vector<uint8_t> HN;
    static thread_local std::vector<int> cnt;
    HL.resize(n * 33);
    HD.resize(n * 33);
    HN.resize(n * 33);
    cnt.assign(n, 0);
    double* const hlp = HL.data();
    double* const hdp = HD.data();
    uint8_t* const hnp = HN.data();
    int* const cntp = cnt.data();
    auto hulls = [&](size_t i0, size_t i1) {
        for (size_t i = i0; i < i1; ++i) {
            const j2k_cb_desc& d = descs[i];
            const int nb = d.numbps;
            const double w = weight[i];
            double pl[33], pd[33];
            int pn[33], m = 0;
            pl[m] = 0.0, pd[m] = dist[i * 33 + 32] * w, pn[m++] = 0;
            for (int k = 0; k < nb && k < 31; ++k) {
                const int np = 3 * k + 1;
                if (np > d.npasses) break;
                pl[m] = k == nb - 1 ? (double)d.length
                                    : std::min<double>(d.length, (double)plane_bytes[i * 32 + k] + J2K_TRUNC_EXTRA);
                pd[m] = dist[i * 33 + k] * w;
                pn[m++] = np;
            }
            // lower convex hull in (L, D): slopes (D drop per byte) strictly decreasing
            double* hl = hlp + i * 33;
            double* hd = hdp + i * 33;
            uint8_t* hn = hnp + i * 33;
            int h = 0;
            for (int q = 0; q < m; ++q) {
                if (h && pl[q] <= hl[h - 1]) {  // no extra bytes: keep the better point
                    if (pd[q] < hd[h - 1]) hl[h - 1] = pl[q], hd[h - 1] = pd[q], hn[h - 1] = (uint8_t)pn[q];
                    continue;
                }
                if (h && pd[q] >= hd[h - 1]) continue;  // no improvement
                // drop the last hull point while the new point's slope is not below its slope
                // (cross-multiplied: both byte differences are positive)
                while (h >= 2 && (hd[h - 1] - pd[q]) * (hl[h - 1] - hl[h - 2]) >=
                                     (hd[h - 2] - hd[h - 1]) * (pl[q] - hl[h - 1]))
                    --h;
                hl[h] = pl[q], hd[h] = pd[q], hn[h++] = (uint8_t)pn[q];
            }
            cntp[i] = h;
        }
    };
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t nt = n < 4096 ? 1 : std::min<size_t>(std::min(16u, hw), n / 1024);
    if (nt <= 1) {
        hulls(0, n);
    } else {
        std::vector<std::thread> pool;
        const size_t per = (n + nt - 1) / nt;
        for (size_t t = 1; t < nt; ++t) pool.emplace_back(hulls, std::min(n, t * per), std::min(n, (t + 1) * per));
        hulls(0, std::min(n, per));
        for (auto& th : pool) th.join();
    }
    double base = 0.0;  // bytes of every hull's first point (L = 0)
    for (size_t i = 0; i < n; ++i) base += HL[i * 33];
    // every hull segment (slope, extra bytes); a block's segments have decreasing slopes, so
    // keeping the segments of slope above a threshold keeps a prefix of every hull
    struct Seg {
        double s, dl;
    };
    static thread_local std::vector<Seg> seg;
    seg.clear();
    double all = base;
    for (size_t i = 0; i < n; ++i)
        for (size_t q = i * 33 + 1; q < i * 33 + (size_t)cnt[i]; ++q) {
            const double dl = HL[q] - HL[q - 1];
            seg.push_back({(HD[q - 1] - HD[q]) / dl, dl});
            all += dl;
        }
    // Threshold: in the order of decreasing slope, the slope of the first segment that no longer
    // fits the budget; segments of that slope or less are dropped (ties together).  Found by a
    // weighted quickselect, linear in the number of segments on average.
    double thr = -1.0;  // keep everything
    if (all > (double)budget) {
        double room = (double)budget - base;
        size_t a = 0, b = seg.size();
        uint64_t rng = 0x9E3779B97F4A7C15ull;
        thr = std::numeric_limits<double>::infinity();
        while (a < b) {
            rng ^= rng << 13, rng ^= rng >> 7, rng ^= rng << 17;
            const double piv = seg[a + rng % (b - a)].s;
            // [a, g): slope > piv, [g, e): slope == piv, [e, b): slope < piv
            auto g = std::partition(seg.begin() + a, seg.begin() + b, [piv](const Seg& x) { return x.s > piv; });
            auto e = std::partition(g, seg.begin() + b, [piv](const Seg& x) { return x.s == piv; });
            double sg = 0.0, se = 0.0;
            for (auto it = seg.begin() + a; it != g; ++it) sg += it->dl;
            if (sg > room) {
                b = (size_t)(g - seg.begin());
                continue;
            }
            room -= sg;
            for (auto it = g; it != e; ++it) se += it->dl;
            if (se > room) {
                thr = piv;
                break;
            }
            room -= se;
            a = (size_t)(e - seg.begin());
        }
    }
    for (size_t i = 0; i < n; ++i) {
        size_t q = i * 33;
        const size_t qe = i * 33 + (size_t)cnt[i];
        while (q + 1 < qe && (HD[q] - HD[q + 1]) / (HL[q + 1] - HL[q]) > thr) ++q;
        descs[i].npasses = HN[q];
        descs[i].length = HN[q] ? (int32_t)HL[q] : 0;
    }
}
