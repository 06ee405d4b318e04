// Tier-2: T.800 codestream assembly on the host (Annex A markers, Annex B packets).
// One tile, one quality layer, LRCP progression, one precinct per resolution, code-blocks of
// one codeword segment each (all passes included).  The reference has no tier-2 at all.
#include <cmath>
#include <cstring>
#include <vector>

#include "j2k_internal.cuh"

namespace {

struct Bytes {
    std::vector<uint8_t> v;
    void u8(uint32_t x) { v.push_back((uint8_t)x); }
    void u16(uint32_t x) { u8(x >> 8); u8(x); }
    void u32(uint32_t x) { u16(x >> 16); u16(x & 0xFFFF); }
};

// packet-header bit writer; after a 0xFF byte the next byte carries 7 bits (B.10.1)
struct BitWriter {
    Bytes& out;
    uint32_t acc = 0;
    int nb = 0, room = 8;
    explicit BitWriter(Bytes& o) : out(o) {}
    void bit(int b) {
        acc = (acc << 1) | (uint32_t)(b & 1);
        if (++nb == room) {
            out.u8(acc);
            room = (acc == 0xFF) ? 7 : 8;
            acc = 0;
            nb = 0;
        }
    }
    void bits(uint32_t v, int n) {
        for (int i = n - 1; i >= 0; --i) bit((v >> i) & 1);
    }
    void flush() {
        bool last_ff;
        if (nb) {
            uint32_t v = acc << (room - nb);
            out.u8(v);
            last_ff = (v == 0xFF);
        } else {
            last_ff = (room == 7);
        }
        if (last_ff) out.u8(0);  // a packet header never ends in 0xFF
        acc = 0;
        nb = 0;
        room = 8;
    }
};

// B.10.2 tag tree
struct TagTree {
    std::vector<int> lw, lh, off, val, low;
    std::vector<uint8_t> known;
    int nlev = 0;
    TagTree(int nw, int nh, const std::vector<int>& leaves) {
        int w = nw, h = nh, total = 0;
        for (;;) {
            lw.push_back(w);
            lh.push_back(h);
            off.push_back(total);
            total += w * h;
            ++nlev;
            if (w == 1 && h == 1) break;
            w = (w + 1) / 2;
            h = (h + 1) / 2;
        }
        val.assign(total, 0);
        low.assign(total, 0);
        known.assign(total, 0);
        for (int i = 0; i < nw * nh; ++i) val[i] = leaves[i];
        for (int l = 1; l < nlev; ++l)
            for (int y = 0; y < lh[l]; ++y)
                for (int x = 0; x < lw[l]; ++x) {
                    int m = 0x7FFFFFFF;
                    for (int dy = 0; dy < 2; ++dy)
                        for (int dx = 0; dx < 2; ++dx) {
                            int cx = 2 * x + dx, cy = 2 * y + dy;
                            if (cx < lw[l - 1] && cy < lh[l - 1])
                                m = std::min(m, val[off[l - 1] + cy * lw[l - 1] + cx]);
                        }
                    val[off[l] + y * lw[l] + x] = m;
                }
    }
    void encode(BitWriter& bw, int x, int y, int threshold) {
        int path[40];
        for (int l = 0; l < nlev; ++l) {
            path[l] = off[l] + y * lw[l] + x;
            x >>= 1;
            y >>= 1;
        }
        int lo = 0;
        for (int l = nlev - 1; l >= 0; --l) {
            int n = path[l];
            if (lo > low[n]) low[n] = lo; else lo = low[n];
            while (lo < threshold) {
                if (lo >= val[n]) {
                    if (!known[n]) {
                        bw.bit(1);
                        known[n] = 1;
                    }
                    break;
                }
                bw.bit(0);
                ++lo;
            }
            low[n] = lo;
        }
    }
};

int floorlog2(long v) {
    int l = -1;
    while (v) {
        v >>= 1;
        ++l;
    }
    return l;
}

void put_npasses(BitWriter& bw, int n) {  // Table B.4
    if (n == 1) bw.bit(0);
    else if (n == 2) bw.bits(2, 2);
    else if (n <= 5) { bw.bits(3, 2); bw.bits((uint32_t)(n - 3), 2); }
    else if (n <= 36) { bw.bits(0xF, 4); bw.bits((uint32_t)(n - 6), 5); }
    else { bw.bits(0x1FF, 9); bw.bits((uint32_t)(n - 37), 7); }
}

}  // namespace

// blocks: component-major, then subbands in QCD order, then raster order within each subband
// (exactly the order of j2k_build_jobs).
std::vector<uint8_t> j2k_t2_write(size_t w, size_t h, int ncomp, int levels, int cbw, int cbh,
                                  int lossless, int mct, const float* steps,
                                  const std::vector<j2k_t2_block>& blocks) {
    const int nb = 3 * levels + 1;
    std::vector<j2k_band_rect> rects(nb);
    j2k_band_rects(w, h, levels, rects.data());
    // index of the first block of each (component, band)
    std::vector<size_t> first((size_t)ncomp * nb + 1);
    std::vector<int> ncbx(nb), ncby(nb);
    size_t k = 0;
    for (int c = 0; c < ncomp; ++c)
        for (int b = 0; b < nb; ++b) {
            first[(size_t)c * nb + b] = k;
            ncbx[b] = rects[b].w ? (int)((rects[b].w + cbw - 1) / cbw) : 0;
            ncby[b] = rects[b].h ? (int)((rects[b].h + cbh - 1) / cbh) : 0;
            if (!rects[b].w || !rects[b].h) ncbx[b] = ncby[b] = 0;
            k += (size_t)ncbx[b] * ncby[b];
        }
    first[(size_t)ncomp * nb] = k;
    // exponents / mantissas and guard bits
    std::vector<int> eps(nb), mant(nb), maxbps(nb, 0);
    for (int c = 0; c < ncomp; ++c)
        for (int b = 0; b < nb; ++b)
            for (size_t i = first[(size_t)c * nb + b]; i < first[(size_t)c * nb + b + 1]; ++i)
                maxbps[b] = std::max(maxbps[b], blocks[i].numbps);
    int G = 2;
    for (int b = 0; b < nb; ++b) {
        int o = rects[b].orient;
        int gain = o == J2K_BAND_LL ? 0 : (o == J2K_BAND_HH ? 2 : 1);
        int Rb = 8 + gain;
        if (lossless) {
            eps[b] = Rb + (mct ? 1 : 0);
            mant[b] = 0;
        } else {
            int ex;
            float fr = std::frexp(steps[b], &ex);
            eps[b] = Rb - (ex - 1);
            mant[b] = (int)std::lrint((fr * 2.0f - 1.0f) * 2048.0f);
        }
        G = std::max(G, maxbps[b] - eps[b] + 1);
    }
    G = std::min(G, 7);
    Bytes o;
    o.u16(0xFF4F);  // SOC
    o.u16(0xFF51);  // SIZ
    o.u16((uint32_t)(38 + 3 * ncomp));
    o.u16(0);
    o.u32((uint32_t)w); o.u32((uint32_t)h); o.u32(0); o.u32(0);
    o.u32((uint32_t)w); o.u32((uint32_t)h); o.u32(0); o.u32(0);
    o.u16((uint32_t)ncomp);
    for (int c = 0; c < ncomp; ++c) { o.u8(7); o.u8(1); o.u8(1); }
    o.u16(0xFF52);  // COD
    o.u16(12);
    o.u8(0);
    o.u8(0);        // LRCP
    o.u16(1);       // one layer
    o.u8(mct ? 1 : 0);
    o.u8((uint32_t)levels);
    o.u8((uint32_t)(floorlog2(cbw) - 2));
    o.u8((uint32_t)(floorlog2(cbh) - 2));
    o.u8(0);
    o.u8(lossless ? 1 : 0);
    o.u16(0xFF5C);  // QCD
    if (lossless) {
        o.u16((uint32_t)(3 + nb));
        o.u8((uint32_t)(G << 5));
        for (int b = 0; b < nb; ++b) o.u8((uint32_t)(eps[b] << 3));
    } else {
        o.u16((uint32_t)(3 + 2 * nb));
        o.u8((uint32_t)((G << 5) | 2));
        for (int b = 0; b < nb; ++b) o.u16((uint32_t)((eps[b] << 11) | mant[b]));
    }
    size_t sot = o.v.size();
    o.u16(0xFF90);  // SOT
    o.u16(10);
    o.u16(0);
    o.u32(0);       // Psot, patched
    o.u8(0);
    o.u8(1);
    o.u16(0xFF93);  // SOD
    for (int r = 0; r <= levels; ++r)
        for (int c = 0; c < ncomp; ++c) {
            int b0 = r == 0 ? 0 : 1 + 3 * (r - 1);  // resolution r holds level L-r+1
            int bcount = r == 0 ? 1 : 3;
            bool any = false;
            for (int q = 0; q < bcount; ++q)
                for (size_t i = first[(size_t)c * nb + b0 + q]; i < first[(size_t)c * nb + b0 + q + 1]; ++i)
                    any |= blocks[i].npasses > 0;
            BitWriter bw(o);
            if (!any) {
                bw.bit(0);
                bw.flush();
                continue;
            }
            bw.bit(1);
            for (int q = 0; q < bcount; ++q) {
                int b = b0 + q;
                int n = ncbx[b] * ncby[b];
                if (!n) continue;
                size_t f = first[(size_t)c * nb + b];
                int Mb = G + eps[b] - 1;
                std::vector<int> incl(n), zbp(n);
                for (int i = 0; i < n; ++i) {
                    incl[i] = blocks[f + i].npasses > 0 ? 0 : 1;
                    zbp[i] = Mb - blocks[f + i].numbps;
                }
                TagTree ti(ncbx[b], ncby[b], incl), tz(ncbx[b], ncby[b], zbp);
                for (int j = 0; j < ncby[b]; ++j)
                    for (int i = 0; i < ncbx[b]; ++i) {
                        const j2k_t2_block& cb = blocks[f + (size_t)j * ncbx[b] + i];
                        ti.encode(bw, i, j, 1);
                        if (cb.npasses == 0) continue;
                        tz.encode(bw, i, j, 0x7FFFFFF);
                        put_npasses(bw, cb.npasses);
                        int lblock = 3;
                        int bits = floorlog2(cb.length) + 1;
                        int avail = lblock + floorlog2(cb.npasses);
                        int inc = bits > avail ? bits - avail : 0;
                        for (int t = 0; t < inc; ++t) bw.bit(1);
                        bw.bit(0);
                        lblock += inc;
                        bw.bits((uint32_t)cb.length, lblock + floorlog2(cb.npasses));
                    }
            }
            bw.flush();
            // the header of the NEXT packet needs the band's Lblock state only within this
            // packet: with one layer every block appears at most once, so no state is kept.
            for (int q = 0; q < bcount; ++q)
                for (size_t i = first[(size_t)c * nb + b0 + q]; i < first[(size_t)c * nb + b0 + q + 1]; ++i)
                    o.v.insert(o.v.end(), blocks[i].data, blocks[i].data + blocks[i].length);
        }
    uint32_t psot = (uint32_t)(o.v.size() - sot);
    o.v[sot + 6] = (uint8_t)(psot >> 24);
    o.v[sot + 7] = (uint8_t)(psot >> 16);
    o.v[sot + 8] = (uint8_t)(psot >> 8);
    o.v[sot + 9] = (uint8_t)psot;
    o.u16(0xFFD9);  // EOC
    return o.v;
}
