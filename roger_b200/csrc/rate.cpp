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
// lower convex hull; a bisection on the slope lambda keeps, in every block, the last hull point
// whose rate-distortion slope is at least lambda.
#include <algorithm>
#include <cmath>
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

void j2k_pcrd_truncate(j2k_cb_desc* descs, size_t n, const uint32_t* plane_bytes, const double* dist,
                       const double* weight, size_t budget) {
    struct Pt {
        double L, D;
        int np;
    };
    std::vector<std::vector<Pt>> hull(n);
    for (size_t i = 0; i < n; ++i) {
        const j2k_cb_desc& d = descs[i];
        const int nb = d.numbps;
        const double w = weight[i];
        std::vector<Pt> pts;
        pts.push_back({0.0, dist[i * 33 + 32] * w, 0});
        for (int k = 0; k < nb && k < 31; ++k) {
            const int np = 3 * k + 1;
            if (np > d.npasses) break;
            double L = k == nb - 1 ? (double)d.length
                                   : std::min<double>(d.length, (double)plane_bytes[i * 32 + k] + J2K_TRUNC_EXTRA);
            pts.push_back({L, dist[i * 33 + k] * w, np});
        }
        // lower convex hull in (L, D): slopes (D drop per byte) strictly decreasing
        std::vector<Pt> h;
        for (const Pt& p : pts) {
            if (!h.empty() && p.L <= h.back().L) {  // no extra bytes: keep the better point
                if (p.D < h.back().D) h.back() = p;
                continue;
            }
            if (!h.empty() && p.D >= h.back().D) continue;  // no improvement
            while (h.size() >= 2) {
                const Pt& a = h[h.size() - 2];
                const Pt& b = h.back();
                const double s1 = (a.D - b.D) / (b.L - a.L), s2 = (b.D - p.D) / (p.L - b.L);
                if (s2 >= s1) h.pop_back();
                else break;
            }
            h.push_back(p);
        }
        hull[i].swap(h);
    }
    auto choose = [&](double lam, std::vector<int>* pick) {
        double total = 0.0;
        for (size_t i = 0; i < n; ++i) {
            const std::vector<Pt>& h = hull[i];
            size_t j = 0;
            while (j + 1 < h.size() && (h[j].D - h[j + 1].D) / (h[j + 1].L - h[j].L) >= lam) ++j;
            if (pick) (*pick)[i] = (int)j;
            total += h[j].L;
        }
        return total;
    };
    std::vector<int> pick(n, 0);
    double lo = 0.0, hi = 1.0;
    if (choose(0.0, nullptr) <= (double)budget) {
        choose(0.0, &pick);
    } else {
        while (choose(hi, nullptr) > (double)budget && hi < 1e300) hi *= 16.0;
        for (int it = 0; it < 200; ++it) {
            const double mid = 0.5 * (lo + hi);
            if (choose(mid, nullptr) > (double)budget) lo = mid;
            else hi = mid;
        }
        choose(hi, &pick);
    }
    for (size_t i = 0; i < n; ++i) {
        const Pt& p = hull[i][pick[i]];
        descs[i].npasses = (uint8_t)p.np;
        descs[i].length = (int32_t)p.L;
        if (p.np == 0) descs[i].length = 0;
    }
}
