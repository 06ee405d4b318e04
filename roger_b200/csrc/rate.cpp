// Rate control: post-compression rate-distortion optimised truncation (PCRD-opt) of the
// code-blocks to a byte budget (each quality layer of a layered stream is one such cut, at its
// cumulative budget).  No counterpart in the reference.
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
// one that no longer fits the budget are kept (a threshold on the slope, found by a radix
// selection over the slopes' bits weighted by their bytes), so that every block keeps a prefix
// of its hull.  The hulls do not depend on the budget: j2k_pcrd_hulls builds them once for every
// budget a caller tries.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
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

void j2k_pcrd_hulls::build(const j2k_cb_desc* descs, size_t nblocks, const uint32_t* plane_bytes,
                           const double* dist, const double* weight) {
    n = nblocks;
    L.resize(n * 33);
    D.resize(n * 33);
    N.resize(n * 33);
    S.resize(n * 33);
    cnt.assign(n, 0);
    double* const hlp = L.data();
    double* const hdp = D.data();
    uint8_t* const hnp = N.data();
    uint64_t* const hsp = S.data();
    int* const cntp = cnt.data();
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t nt = n < 4096 ? 1 : std::min<size_t>(std::min(16u, hw), n / 1024);
    std::vector<double> part_base(nt, 0.0), part_all(nt, 0.0);
    std::vector<size_t> part_ns(nt, 0);
    auto hulls = [=, &part_base, &part_all, &part_ns](size_t t, size_t i0, size_t i1) {
        double sb = 0.0, sa = 0.0;
        size_t ns = 0;
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
                // a later cut never keeps fewer bytes (the coder's output only grows); held for
                // any input, so that the kept lengths add up along every hull
                pl[m] = std::max(pl[m], pl[m - 1]);
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
                    // (never in place of the empty cut: coded passes need bytes, so a cut of
                    // passes with no bytes, which only a malformed input gives, is skipped)
                    if (h > 1 && pd[q] < hd[h - 1]) hl[h - 1] = pl[q], hd[h - 1] = pd[q], hn[h - 1] = (uint8_t)pn[q];
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
            // slopes of the hull segments as ordered keys: positive doubles order as their bits
            uint64_t* hs = hsp + i * 33;
            for (int q = 1; q < h; ++q) {
                const double sl = (hd[q - 1] - hd[q]) / (hl[q] - hl[q - 1]);
                std::memcpy(&hs[q], &sl, 8);
            }
            sb += hl[0];
            sa += hl[h - 1];
            ns += (size_t)(h - 1);
        }
        part_base[t] = sb, part_all[t] = sa, part_ns[t] = ns;
    };
    const size_t per = (n + nt - 1) / nt;
    j2k_run_threads((int)nt, [&](int t) { hulls(t, std::min(n, t * per), std::min(n, (t + 1) * per)); });
    // byte counts are whole numbers, so these sums are exact in any order
    base = all = 0.0;
    nseg = 0;
    for (size_t t = 0; t < nt; ++t) base += part_base[t], all += part_all[t], nseg += part_ns[t];
}

double j2k_pcrd_hulls::threshold(size_t budget) {
    // In the order of decreasing slope, the slope of the first segment that no longer fits the
    // budget; segments of that slope or less are dropped (ties together): the slope v with
    // bytes(slope > v) <= room < bytes(slope >= v).  Found by a radix selection on the slopes'
    // bits, 11 bits per pass from the top: each pass sums the candidates' extra bytes per digit,
    // keeps the candidates of the digit where the running sum from the top passes the room, and
    // takes the bytes of the digits above it off the room.  Byte counts are whole numbers, so
    // every sum is exact and the result does not depend on the order of the segments.
    if (all <= (double)budget) return -1.0;  // keep everything
    double room = (double)budget - base;
    if (room < 0.0 || nseg == 0) return std::numeric_limits<double>::infinity();
    constexpr int kBits = 11, kBins = 1 << kBits;
    double hist[kBins];
    // first pass over every hull segment, in place (a negative slope cannot occur: hull points'
    // distortions strictly decrease); the sign bit is 0, so digit 0 is bits 62..52
    std::memset(hist, 0, sizeof(hist));
    const double* hl = L.data();
    const uint64_t* hs = S.data();
    for (size_t i = 0; i < n; ++i) {
        const size_t b0 = i * 33;
        for (int q = 1; q < cnt[i]; ++q) hist[(hs[b0 + q] >> 52) & (kBins - 1)] += hl[b0 + q] - hl[b0 + q - 1];
    }
    auto pick = [&](const double* hh) {
        double above = 0.0;
        for (int b = kBins - 1; b >= 0; --b) {
            if (above + hh[b] > room) {
                room -= above;
                return b;
            }
            above += hh[b];
        }
        return -1;  // cannot happen: the candidates' bytes exceed the room
    };
    int dig = pick(hist);
    if (dig < 0) return std::numeric_limits<double>::infinity();
    uint64_t prefix = (uint64_t)dig << 52;
    int shift = 52;  // bits below the digits fixed so far
    cand.clear();
    for (size_t i = 0; i < n; ++i) {
        const size_t b0 = i * 33;
        for (int q = 1; q < cnt[i]; ++q)
            if ((hs[b0 + q] >> 52) == (uint64_t)dig) cand.push_back(Seg{hs[b0 + q], hl[b0 + q] - hl[b0 + q - 1]});
    }
    while (shift > 0) {
        const int bits = std::min(kBits, shift);
        shift -= bits;
        const uint64_t mask = ((uint64_t)1 << bits) - 1;
        std::memset(hist, 0, sizeof(hist));
        for (const Seg& c : cand) hist[(c.key >> shift) & mask] += c.dl;
        double above = 0.0;
        int b = (int)mask;
        for (; b >= 0; --b) {
            if (above + hist[b] > room) break;
            above += hist[b];
        }
        if (b < 0) return std::numeric_limits<double>::infinity();
        room -= above;
        prefix |= (uint64_t)b << shift;
        size_t k = 0;
        for (const Seg& c : cand)
            if (((c.key >> shift) & mask) == (uint64_t)b) cand[k++] = c;
        cand.resize(k);
    }
    double thr;
    std::memcpy(&thr, &prefix, 8);
    return thr;
}

void j2k_pcrd_hulls::cut(double thr, int32_t* npasses, int32_t* length) const {
    const double* hl = L.data();
    const uint64_t* hs = S.data();
    const uint8_t* hn = N.data();
    uint64_t tk;  // slopes compare as their bits; a threshold of -1 keeps every segment
    std::memcpy(&tk, &thr, 8);
    const bool all_kept = thr < 0.0;
    for (size_t i = 0; i < n; ++i) {
        const size_t b0 = i * 33;
        int q = 0;
        while (q + 1 < cnt[i] && (all_kept || hs[b0 + q + 1] > tk)) ++q;
        npasses[i] = hn[b0 + q];
        length[i] = hn[b0 + q] ? (int32_t)hl[b0 + q] : 0;
    }
}

extern "C" j2k_status j2k_pcrd_truncate(j2k_cb_desc* descs, size_t n, const uint32_t* plane_bytes,
                                        const double* dist, const double* weight, size_t budget) {
    J2K_API_BEGIN
    if (n && (!descs || !plane_bytes || !dist || !weight)) return J2K_ERR_INVALID_ARG;
    static thread_local j2k_pcrd_hulls hulls;  // scratch kept per thread between calls
    static thread_local std::vector<int32_t> np, len;
    j2k_pcrd_hulls& h = hulls;
    h.build(descs, n, plane_bytes, dist, weight);
    const double thr = h.threshold(budget);
    np.resize(n);
    len.resize(n);
    h.cut(thr, np.data(), len.data());
    for (size_t i = 0; i < n; ++i) descs[i].npasses = (uint8_t)np[i], descs[i].length = len[i];
    return J2K_OK;
    J2K_API_END
}
