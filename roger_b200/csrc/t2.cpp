// Tier-2: T.800 codestream assembly and parsing on the host (Annex A markers, Annex B packets).
// Writer: one tile, LRCP progression, one precinct per resolution, one or more quality layers,
// each block's codeword one segment (the default code-block style).  Reader: the same subset,
// LRCP or RLCP, any number of layers.  The reference has no tier-2 at all.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <string>
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
    // the n low bits of v, most significant first (n <= 32), a byte's worth at a time
    void bits(uint32_t v, int n) {
        while (n > 0) {
            const int take = std::min(room - nb, n);
            n -= take;
            acc = (acc << take) | ((v >> n) & ((1u << take) - 1));
            nb += take;
            if (nb == room) {
                out.u8(acc);
                room = (acc == 0xFF) ? 7 : 8;
                acc = 0;
                nb = 0;
            }
        }
    }
    void zeros(int n) {
        for (; n > 24; n -= 24) bits(0, 24);
        bits(0, n);
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
            // a 0 for every step from lo up to the node's value (or the threshold), then a 1
            // once the value is reached below the threshold, if not sent before
            if (lo < threshold) {
                const int v = val[n];
                if (v > lo) {
                    const int stop = std::min(v, threshold);
                    bw.zeros(stop - lo);
                    lo = stop;
                }
                if (lo < threshold && !known[n]) {
                    bw.bit(1);
                    known[n] = 1;
                }
            }
            low[n] = lo;
        }
    }
};

int floorlog2(long v) {  // -1 for 0
    return v > 0 ? 63 - __builtin_clzl((unsigned long)v) : -1;
}

void put_npasses(BitWriter& bw, int n) {  // Table B.4
    if (n == 1) bw.bit(0);
    else if (n == 2) bw.bits(2, 2);
    else if (n <= 5) { bw.bits(3, 2); bw.bits((uint32_t)(n - 3), 2); }
    else if (n <= 36) { bw.bits(0xF, 4); bw.bits((uint32_t)(n - 6), 5); }
    else { bw.bits(0x1FF, 9); bw.bits((uint32_t)(n - 37), 7); }
}

}  // namespace

namespace {

bool j2k_qcd_step_impl(float step, int band, int* eps, int* mant) {
    if (!(step > 0.0f) || !std::isfinite(step)) return false;
    const int gain = band == 0 ? 0 : ((band - 1) % 3 == 2 ? 2 : 1);
    int ex;
    const float fr = std::frexp(step, &ex);  // step = fr * 2^ex, fr in [0.5, 1)
    int e = 8 + gain - (ex - 1);
    int m = (int)std::lrint((fr * 2.0f - 1.0f) * 2048.0f);
    if (m == 2048) {  // rounded up to the next power of two
        m = 0;
        e -= 1;
    }
    if (e < 0 || e > 31) return false;
    *eps = e;
    *mant = m;
    return true;
}

// Writes the codestream into `o`; without bodies only the markers and packet headers are
// written and the returned size still counts every block's codeword bytes.  nlayers quality
// layers: after layer l block i has cum_np[l * n + i] passes and cum_len[l * n + i] bytes of its
// codeword (non-decreasing in l); cum_np / cum_len NULL means one layer holding what
// blocks[i] says.
size_t t2_emit(Bytes& o, size_t w, size_t h, int ncomp, int levels, int cbw, int cbh, int lossless, int mct,
               const float* steps, const std::vector<j2k_t2_block>& blocks, bool bodies, int nlayers = 1,
               const int32_t* cum_np = nullptr, const int32_t* cum_len = nullptr, int style = 0) {
    const size_t nblk = blocks.size();
    if (!cum_np || !cum_len) nlayers = 1;
    // passes / bytes of block i after layer l (l = -1: nothing)
    auto NP = [&](int l, size_t i) -> int {
        if (l < 0) return 0;
        return cum_np ? cum_np[(size_t)l * nblk + i] : blocks[i].npasses;
    };
    auto LEN = [&](int l, size_t i) -> int {
        if (l < 0) return 0;
        return cum_len ? cum_len[(size_t)l * nblk + i] : std::max(blocks[i].length, 0);
    };
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
        } else if (!j2k_qcd_step(steps[b], b, &eps[b], &mant[b])) {  // callers refuse such steps
            eps[b] = 31;
            mant[b] = 0;
        }
        G = std::max(G, maxbps[b] - eps[b] + 1);
    }
    G = std::min(G, 7);
    size_t body = 0;
    for (size_t i = 0; i < nblk; ++i) body += (size_t)LEN(nlayers - 1, i);
    o.v.reserve(256 + (size_t)nb * 4 + blocks.size() * 10 + (bodies ? body : 0));
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
    o.u16((uint32_t)nlayers);
    o.u8(mct ? 1 : 0);
    o.u8((uint32_t)levels);
    o.u8((uint32_t)(floorlog2(cbw) - 2));
    o.u8((uint32_t)(floorlog2(cbh) - 2));
    o.u8((uint32_t)style);  // code-block style
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
    // tag trees (inclusion: first layer holding a pass of the block; zero bit-planes) and the
    // Lblock state of every block persist from layer to layer
    std::vector<TagTree> incl, zbp;
    incl.reserve((size_t)ncomp * nb);
    zbp.reserve((size_t)ncomp * nb);
    for (int c = 0; c < ncomp; ++c)
        for (int b = 0; b < nb; ++b) {
            const int n = ncbx[b] * ncby[b];
            const size_t f = first[(size_t)c * nb + b];
            const int Mb = G + eps[b] - 1;
            std::vector<int> li(std::max(n, 1), nlayers), lz(std::max(n, 1), 0);
            for (int i = 0; i < n; ++i) {
                for (int l = 0; l < nlayers; ++l)
                    if (NP(l, f + i) > 0) {
                        li[i] = l;
                        break;
                    }
                lz[i] = Mb - blocks[f + i].numbps;
            }
            incl.emplace_back(std::max(ncbx[b], 1), std::max(ncby[b], 1), li);
            zbp.emplace_back(std::max(ncbx[b], 1), std::max(ncby[b], 1), lz);
        }
    std::vector<int> lblock(nblk, 3);
    // packet (layer l, resolution r, component c): its header, then (with bodies) its codeword
    // segments.  Within a layer the packets touch disjoint bands, tag trees and blocks.
    auto packet = [&](Bytes& out, int l, int r, int c) {
        int b0 = r == 0 ? 0 : 1 + 3 * (r - 1);  // resolution r holds level L-r+1
        int bcount = r == 0 ? 1 : 3;
        bool any = false;
        for (int q = 0; q < bcount; ++q)
            for (size_t i = first[(size_t)c * nb + b0 + q]; i < first[(size_t)c * nb + b0 + q + 1]; ++i)
                any |= NP(l, i) > NP(l - 1, i);
        if (!any) {
            BitWriter bw(out);
            bw.bit(0);
            bw.flush();
            return;
        }
        if (bodies) {  // room for the header (a few bytes a block) and the segments
            size_t need = 64;
            for (int q = 0; q < bcount; ++q)
                for (size_t i = first[(size_t)c * nb + b0 + q]; i < first[(size_t)c * nb + b0 + q + 1]; ++i)
                    need += 16 + (size_t)(LEN(l, i) - LEN(l - 1, i));
            out.v.reserve(out.v.size() + need);
        }
        BitWriter bw(out);
        bw.bit(1);
        for (int q = 0; q < bcount; ++q) {
            int b = b0 + q;
            if (ncbx[b] == 0 || ncby[b] == 0) continue;
            size_t f = first[(size_t)c * nb + b];
            TagTree& ti = incl[(size_t)c * nb + b];
            TagTree& tz = zbp[(size_t)c * nb + b];
            for (int j = 0; j < ncby[b]; ++j)
                for (int i = 0; i < ncbx[b]; ++i) {
                    const size_t k = f + (size_t)j * ncbx[b] + i;
                    const int prev = NP(l - 1, k), cur = NP(l, k);
                    if (prev == 0) {  // not included before: inclusion tag tree up to layer l
                        ti.encode(bw, i, j, l + 1);
                        if (cur == 0) continue;
                        tz.encode(bw, i, j, 0x7FFFFFF);
                    } else {
                        bw.bit(cur > prev);
                        if (cur == prev) continue;
                    }
                    const int newp = cur - prev;
                    put_npasses(bw, newp);
                    // the new passes as pieces of codeword segments (B.10.7.2): one piece per
                    // segment the style terminates within them, and the rest; each piece's
                    // length in Lblock + floor(log2(its passes)) bits, Lblock raised once so
                    // that every length fits
                    int pnp[J2K_PASS_STRIDE + 1], plen[J2K_PASS_STRIDE + 1], npc = 0;
                    if (style) {
                        const j2k_t2_block& B = blocks[k];
                        int at = LEN(l - 1, k), start = prev;
                        for (int q = prev; q < cur; ++q) {
                            const bool term = j2k_pass_terminated(style, q, B.npasses);
                            if (!term && q != cur - 1) continue;
                            const int end = term && B.pass_end ? (int)B.pass_end[q] : LEN(l, k);
                            pnp[npc] = q + 1 - start;
                            plen[npc++] = end - at;
                            at = end;
                            start = q + 1;
                        }
                    } else {
                        pnp[0] = newp;
                        plen[0] = LEN(l, k) - LEN(l - 1, k);
                        npc = 1;
                    }
                    int inc = 0;
                    for (int q = 0; q < npc; ++q)
                        inc = std::max(inc, floorlog2(plen[q]) + 1 - (lblock[k] + floorlog2(pnp[q])));
                    bw.bits(((1u << inc) - 1) << 1, inc + 1);  // inc ones, then a zero
                    lblock[k] += inc;
                    for (int q = 0; q < npc; ++q) bw.bits((uint32_t)plen[q], lblock[k] + floorlog2(pnp[q]));
                }
        }
        bw.flush();
        if (bodies)
            for (int q = 0; q < bcount; ++q)
                for (size_t i = first[(size_t)c * nb + b0 + q]; i < first[(size_t)c * nb + b0 + q + 1]; ++i)
                    if (NP(l, i) > NP(l - 1, i))
                        out.v.insert(out.v.end(), blocks[i].data + LEN(l - 1, i), blocks[i].data + LEN(l, i));
    };
    // many blocks: a layer's packets on host threads (largest first, taken from a shared
    // counter) into their own buffers, appended in LRCP order
    const int npk = (levels + 1) * ncomp;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int nt = nblk < 4096 ? 1 : (int)std::min<unsigned>(std::min(16u, hw), (unsigned)npk);
    std::vector<Bytes> pk(nt > 1 ? npk : 0);
    std::vector<int> order(npk);
    for (int i = 0; i < npk; ++i) order[i] = i;
    auto blocks_of = [&](int i) {  // packet i = r * ncomp + c
        const int r = i / ncomp, c = i % ncomp;
        const int b0 = r == 0 ? 0 : 1 + 3 * (r - 1), bcount = r == 0 ? 1 : 3;
        return first[(size_t)c * nb + b0 + bcount] - first[(size_t)c * nb + b0];
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return blocks_of(a) > blocks_of(b); });
    for (int l = 0; l < nlayers; ++l) {
        if (nt <= 1) {
            for (int r = 0; r <= levels; ++r)
                for (int c = 0; c < ncomp; ++c) packet(o, l, r, c);
            continue;
        }
        std::atomic<int> next{0};
        std::atomic<bool> failed{false};
        j2k_run_threads(nt, [&](int) {
            for (int i; (i = next.fetch_add(1)) < npk;) {
                const int p = order[i];
                pk[p].v.clear();
                try {
                    packet(pk[p], l, p / ncomp, p % ncomp);
                } catch (...) {  // a host allocation failed: reported after the join
                    failed = true;
                }
            }
        });
        if (failed) throw std::bad_alloc();
        // append the packets in order; with codeword bytes (over 4 MB) each packet is copied by
        // one of the threads
        std::vector<size_t> at(npk + 1, o.v.size());
        for (int p = 0; p < npk; ++p) at[p + 1] = at[p] + pk[p].v.size();
        if (at[npk] - at[0] < ((size_t)4 << 20)) {
            for (int p = 0; p < npk; ++p) o.v.insert(o.v.end(), pk[p].v.begin(), pk[p].v.end());
            continue;
        }
        o.v.resize(at[npk]);
        next = 0;
        j2k_run_threads(nt, [&](int) {
            for (int i; (i = next.fetch_add(1)) < npk;) {
                const int p = order[i];
                if (!pk[p].v.empty()) std::memcpy(o.v.data() + at[p], pk[p].v.data(), pk[p].v.size());
            }
        });
    }
    const size_t extra = bodies ? 0 : body;
    uint32_t psot = (uint32_t)(o.v.size() + extra - sot);
    o.v[sot + 6] = (uint8_t)(psot >> 24);
    o.v[sot + 7] = (uint8_t)(psot >> 16);
    o.v[sot + 8] = (uint8_t)(psot >> 8);
    o.v[sot + 9] = (uint8_t)psot;
    o.u16(0xFFD9);  // EOC
    return o.v.size() + extra;
}

}  // namespace

bool j2k_qcd_step(float step, int band, int* eps, int* mant) { return j2k_qcd_step_impl(step, band, eps, mant); }

// blocks: component-major, then subbands in QCD order, then raster order within each subband
// (exactly the order of j2k_build_jobs).
std::vector<uint8_t> j2k_t2_write(size_t w, size_t h, int ncomp, int levels, int cbw, int cbh,
                                  int lossless, int mct, const float* steps,
                                  const std::vector<j2k_t2_block>& blocks, int style) {
    Bytes o;
    t2_emit(o, w, h, ncomp, levels, cbw, cbh, lossless, mct, steps, blocks, true, 1, nullptr, nullptr, style);
    return std::move(o.v);
}

size_t j2k_t2_size(size_t w, size_t h, int ncomp, int levels, int cbw, int cbh, int lossless, int mct,
                   const float* steps, const std::vector<j2k_t2_block>& blocks, int nlayers,
                   const int32_t* cum_np, const int32_t* cum_len) {
    static thread_local Bytes o;
    o.v.clear();
    return t2_emit(o, w, h, ncomp, levels, cbw, cbh, lossless, mct, steps, blocks, false, nlayers, cum_np, cum_len);
}

std::vector<uint8_t> j2k_t2_write_layers(size_t w, size_t h, int ncomp, int levels, int cbw, int cbh,
                                         int lossless, int mct, const float* steps,
                                         const std::vector<j2k_t2_block>& blocks, int nlayers,
                                         const int32_t* cum_np, const int32_t* cum_len) {
    Bytes o;
    t2_emit(o, w, h, ncomp, levels, cbw, cbh, lossless, mct, steps, blocks, true, nlayers, cum_np, cum_len);
    return std::move(o.v);
}

// ---- tier-2 reading (codestream parser) -----------------------------------------------------
namespace {

struct ReadErr {
    j2k_status s;
    const char* msg;
};

struct Cursor {
    const uint8_t* p;
    size_t n, i = 0;
    uint32_t u8() {
        if (i >= n) throw ReadErr{J2K_ERR_INVALID_ARG, "codestream truncated"};
        return p[i++];
    }
    uint32_t u16() { uint32_t a = u8(); return (a << 8) | u8(); }
    uint32_t u32() { uint32_t a = u16(); return (a << 16) | u16(); }
};

// packet-header bit reader: after a 0xFF byte the next byte carries 7 bits (B.10.1)
struct BitReader {
    const uint8_t* p;
    size_t n, i;
    uint32_t cur = 0;
    int left = 0;
    bool last_ff = false;
    BitReader(const uint8_t* d, size_t len, size_t start) : p(d), n(len), i(start) {}
    int bit() {
        if (left == 0) {
            if (i >= n) throw ReadErr{J2K_ERR_INVALID_ARG, "packet header truncated"};
            cur = p[i++];
            left = last_ff ? 7 : 8;
            last_ff = (cur == 0xFF);
        }
        --left;
        return (int)((cur >> left) & 1);
    }
    uint32_t bits(int k) {
        uint32_t v = 0;
        while (k--) v = (v << 1) | (uint32_t)bit();
        return v;
    }
    // end of header: byte aligned; a header whose last byte is 0xFF is followed by one more
    size_t end() {
        if (last_ff) {
            if (i >= n) throw ReadErr{J2K_ERR_INVALID_ARG, "packet header truncated"};
            ++i;
        }
        return i;
    }
};

// B.10.2 tag tree, decoding side
struct TagTreeDec {
    std::vector<int> lw, lh, off, low, val;
    std::vector<uint8_t> known;
    int nlev = 0;
    TagTreeDec(int nw, int nh) {
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
        low.assign(total, 0);
        val.assign(total, 0);
        known.assign(total, 0);
    }
    // value of leaf (x, y) if it is below `threshold`, else `threshold`
    int decode(BitReader& br, int x, int y, int threshold) {
        const int leaf = y * lw[0] + x;  // level 0 starts at offset 0
        int path[40];
        for (int l = 0; l < nlev; ++l) {
            path[l] = off[l] + y * lw[l] + x;
            x >>= 1;
            y >>= 1;
        }
        int lo = 0;
        for (int l = nlev - 1; l >= 0; --l) {
            const int q = path[l];
            if (low[q] < lo) low[q] = lo;
            while (!known[q] && low[q] < threshold) {
                if (br.bit()) {
                    known[q] = 1;
                    val[q] = low[q];
                } else {
                    ++low[q];
                }
            }
            lo = low[q];
        }
        return (known[leaf] && val[leaf] < threshold) ? val[leaf] : threshold;
    }
};

int get_npasses(BitReader& br) {  // Table B.4
    if (!br.bit()) return 1;
    if (!br.bit()) return 2;
    uint32_t v = br.bits(2);
    if (v < 3) return 3 + (int)v;
    v = br.bits(5);
    if (v < 31) return 6 + (int)v;
    return 37 + (int)br.bits(7);
}

}  // namespace

extern "C" j2k_status j2k_codestream_write(uint32_t w, uint32_t h, int ncomp, int levels, int cbw, int cbh,
                                           int lossless, const float* steps, const j2k_cb_desc* descs,
                                           size_t count, const uint8_t* bytes, size_t nbytes, int layers,
                                           const int32_t* layer_npasses, const int32_t* layer_lengths, uint8_t* out,
                                           size_t cap, size_t* len) {
    J2K_API_BEGIN
    if (!len || (!descs && count) || (!bytes && nbytes)) return J2K_ERR_INVALID_ARG;
    auto pow2 = [](int v) { return v >= 4 && v <= 64 && (v & (v - 1)) == 0; };
    if (w == 0 || h == 0 || w > 65535 || h > 65535 || (ncomp != 1 && ncomp != 3) || levels < 0 || levels > 32 ||
        !pow2(cbw) || !pow2(cbh) || cbw * cbh > 4096)
        return J2K_ERR_INVALID_ARG;
    if (count != j2k_build_jobs(w, h, levels, cbw, cbh, nullptr) * (size_t)ncomp) return J2K_ERR_INVALID_ARG;
    const bool layered = layers > 1 || (layers == 1 && layer_npasses && layer_lengths);
    if (layers < 0 || layers > 64 || (layered && (!layer_npasses || !layer_lengths))) return J2K_ERR_INVALID_ARG;
    const int nl = layered ? layers : 1;
    std::vector<j2k_t2_block> blocks(count);
    for (size_t i = 0; i < count; ++i) {
        const j2k_cb_desc& d = descs[i];
        if (d.numbps > 31 || d.length < 0 || (d.numbps && d.npasses > 3 * d.numbps - 2) || (!d.numbps && d.npasses) ||
            (size_t)d.offset + (size_t)d.length > nbytes)
            return J2K_ERR_INVALID_ARG;
        blocks[i] = j2k_t2_block{d.numbps, d.npasses, d.length, bytes ? bytes + d.offset : nullptr};
        if (layered) {
            int pn = 0, pl = 0;
            for (int l = 0; l < nl; ++l) {
                const int np = layer_npasses[(size_t)l * count + i], ln = layer_lengths[(size_t)l * count + i];
                if (np < pn || ln < pl || np > d.npasses || ln > d.length || (np == 0 && ln != 0))
                    return J2K_ERR_INVALID_ARG;
                pn = np;
                pl = ln;
            }
        }
    }
    std::vector<float> st;
    if (!lossless) {
        const int nb = 3 * levels + 1;
        if (steps) {
            st.assign(steps, steps + nb);
        } else {
            std::vector<j2k_band_rect> r(nb);
            j2k_band_rects(w, h, levels, r.data());
            st.resize(nb);
            for (int b = 0; b < nb; ++b) st[b] = 8.0f * std::ldexp(1.0f, -r[b].level);
        }
        for (int b = 0; b < (int)st.size(); ++b) {
            int e, m;
            if (!j2k_qcd_step(st[b], b, &e, &m)) return J2K_ERR_INVALID_ARG;
        }
    }
    // a block's bit-planes must fit its band's exponent and at most 7 guard bits (the zero
    // bit-plane count Mb - numbps is not negative, Mb = guard + eps - 1)
    {
        std::vector<j2k_cb_job> jobs;
        for (int c = 0; c < ncomp; ++c) j2k_build_jobs(w, h, levels, cbw, cbh, &jobs, c);
        for (size_t i = 0; i < count; ++i) {
            const int b = jobs[i].band;
            const int gain = b == 0 ? 0 : ((b - 1) % 3 == 2 ? 2 : 1);
            int e = 8 + gain + (ncomp == 3 ? 1 : 0), m;
            if (!lossless) j2k_qcd_step(st[b], b, &e, &m);
            if (descs[i].numbps > e + 6) return J2K_ERR_INVALID_ARG;
        }
    }
    Bytes o;
    t2_emit(o, w, h, ncomp, levels, cbw, cbh, lossless ? 1 : 0, ncomp == 3, lossless ? nullptr : st.data(), blocks,
            true, nl, layered ? layer_npasses : nullptr, layered ? layer_lengths : nullptr);
    *len = o.v.size();
    if (!out) return J2K_OK;
    if (cap < o.v.size()) return J2K_ERR_CAPACITY;
    std::memcpy(out, o.v.data(), o.v.size());
    return J2K_OK;
    J2K_API_END
}

namespace {

// Parses a codestream into stream parameters, one descriptor per code-block (job order:
// component, subband in QCD order, raster) and the packet bytes of the tile (tile-parts
// concatenated); src_off[i] is block i's codeword offset within tile_bytes.
// Quality layers: the packets of every layer are parsed (the tag-tree, Lblock and inclusion state
// carries from layer to layer); a block's codeword is the concatenation of its segments from
// the first `max_layers` layers (0: all), segs[i] listing (offset in tile_bytes, length).
j2k_status t2_read(const uint8_t* cs, size_t n, int max_layers, j2k_stream_info* info,
                   std::vector<j2k_cb_desc>* descs, std::vector<std::vector<std::pair<uint32_t, int>>>* segs,
                   std::vector<uint8_t>* tile_bytes, std::string* err, bool header_only = false,
                   std::vector<uint32_t>* pass_ends = nullptr) {
    try {
        Cursor c{cs, n};
        if (c.u16() != 0xFF4F) throw ReadErr{J2K_ERR_INVALID_ARG, "no SOC marker"};
        j2k_stream_info I{};
        int ncomp = 0, levels = -1, prog = 0, layers = 0, mct = 0, cbw = 0, cbh = 0, sty = 0, xform = 0, scod = 0;
        int qstyle = -1, guard = 0;
        std::vector<int> eps, mant;
        uint32_t tw = 0, th = 0;
        std::vector<uint8_t> data;  // packet bytes of tile 0, tile-parts concatenated
        bool in_tile = false;
        for (;;) {
            const uint32_t m = c.u16();
            if (m == 0xFFD9) break;  // EOC
            if (m == 0xFF93) {       // SOD: read to the end of the tile-part
                throw ReadErr{J2K_ERR_INVALID_ARG, "SOD outside a tile-part"};
            }
            const size_t seg_start = c.i;
            const uint32_t L = c.u16();
            if (L < 2 || seg_start + L > n) throw ReadErr{J2K_ERR_INVALID_ARG, "bad marker segment length"};
            const size_t seg_end = seg_start + L;
            if (m == 0xFF51) {  // SIZ
                c.u16();
                const uint32_t xs = c.u32(), ys = c.u32(), x0 = c.u32(), y0 = c.u32();
                tw = c.u32();
                th = c.u32();
                const uint32_t tx0 = c.u32(), ty0 = c.u32();
                ncomp = (int)c.u16();
                if (x0 || y0 || tx0 || ty0) throw ReadErr{J2K_ERR_UNSUPPORTED, "image or tile offsets"};
                // code-block positions are kept in 16 bits, as the writer's limit
                if (xs == 0 || ys == 0 || xs > 65535 || ys > 65535)
                    throw ReadErr{J2K_ERR_UNSUPPORTED, "image width or height outside 1..65535"};
                if (tw < xs || th < ys) throw ReadErr{J2K_ERR_UNSUPPORTED, "more than one tile"};
                if (ncomp != 1 && ncomp != 3) throw ReadErr{J2K_ERR_UNSUPPORTED, "component count other than 1 or 3"};
                for (int k = 0; k < ncomp; ++k) {
                    const uint32_t ssiz = c.u8(), dx = c.u8(), dy = c.u8();
                    if (ssiz != 7 || dx != 1 || dy != 1)
                        throw ReadErr{J2K_ERR_UNSUPPORTED, "components other than 8-bit unsigned, unsubsampled"};
                }
                I.w = xs;
                I.h = ys;
                I.ncomp = ncomp;
                I.precision = 8;
            } else if (m == 0xFF52) {  // COD
                scod = (int)c.u8();
                prog = (int)c.u8();
                layers = (int)c.u16();
                mct = (int)c.u8();
                levels = (int)c.u8();
                const int xcb = (int)c.u8(), ycb = (int)c.u8();  // exponents - 2 (A.6.1)
                if (xcb > 8 || ycb > 8) throw ReadErr{J2K_ERR_INVALID_ARG, "code-block size exponent"};
                cbw = 1 << (xcb + 2);
                cbh = 1 << (ycb + 2);
                sty = (int)c.u8();
                xform = (int)c.u8();
                if (scod & 1) throw ReadErr{J2K_ERR_UNSUPPORTED, "user-defined precincts"};
                if (layers < 1) throw ReadErr{J2K_ERR_INVALID_ARG, "no quality layer"};
                if (prog != 0 && prog != 1) throw ReadErr{J2K_ERR_UNSUPPORTED, "progression other than LRCP/RLCP"};
                // bypass, reset, per-pass termination and predictable termination (which needs
                // nothing of a decoder) are read; vertically causal contexts and segmentation
                // symbols are not
                if (sty & 0x08) throw ReadErr{J2K_ERR_UNSUPPORTED, "vertically causal code-block contexts"};
                if (sty & 0x20) throw ReadErr{J2K_ERR_UNSUPPORTED, "code-block segmentation symbols"};
                if (sty & ~0x3F) throw ReadErr{J2K_ERR_INVALID_ARG, "code-block style"};
                if (levels > 32 || cbw > 64 || cbh > 64 || cbw * cbh > 4096)
                    throw ReadErr{J2K_ERR_UNSUPPORTED, "code-block size or decomposition levels"};
            } else if (m == 0xFF5C) {  // QCD
                const uint32_t sq = c.u8();
                guard = (int)(sq >> 5);
                qstyle = (int)(sq & 31);
                const size_t nbytes = seg_end - c.i;
                if (qstyle == 0) {
                    for (size_t k = 0; k < nbytes; ++k) {
                        eps.push_back((int)(c.u8() >> 3));
                        mant.push_back(0);
                    }
                } else if (qstyle == 1 || qstyle == 2) {
                    for (size_t k = 0; k + 1 < nbytes; k += 2) {
                        const uint32_t v = c.u16();
                        eps.push_back((int)(v >> 11));
                        mant.push_back((int)(v & 0x7FF));
                    }
                } else {
                    throw ReadErr{J2K_ERR_UNSUPPORTED, "quantisation style"};
                }
            } else if (m == 0xFF53 || m == 0xFF5D || m == 0xFF5E || m == 0xFF60 || m == 0xFF61) {
                throw ReadErr{J2K_ERR_UNSUPPORTED, "COC, QCC, RGN, PPM or PPT marker"};
            } else if (m == 0xFF90) {  // SOT
                if (header_only) break;
                const uint32_t isot = c.u16(), psot = c.u32();
                c.u8();
                c.u8();
                if (isot != 0) throw ReadErr{J2K_ERR_UNSUPPORTED, "more than one tile"};
                // tile-part header markers up to SOD
                size_t end = psot ? seg_start - 2 + psot : n - 2;
                if (end > n) throw ReadErr{J2K_ERR_INVALID_ARG, "bad Psot"};
                c.i = seg_end;
                for (;;) {
                    const uint32_t mm = c.u16();
                    if (mm == 0xFF93) break;
                    const size_t s2 = c.i;
                    const uint32_t L2 = c.u16();
                    if (mm == 0xFF52 || mm == 0xFF5C || mm == 0xFF53 || mm == 0xFF5D || mm == 0xFF61)
                        throw ReadErr{J2K_ERR_UNSUPPORTED, "coding or quantisation markers in a tile-part header"};
                    c.i = s2 + L2;
                }
                if (c.i > end) throw ReadErr{J2K_ERR_INVALID_ARG, "bad tile-part"};
                data.insert(data.end(), cs + c.i, cs + end);
                c.i = end;
                in_tile = true;
                continue;
            }
            c.i = seg_end;
        }
        (void)in_tile;
        if (!ncomp || levels < 0 || qstyle < 0) throw ReadErr{J2K_ERR_INVALID_ARG, "missing SIZ, COD or QCD"};
        if (ncomp == 3 && !mct) throw ReadErr{J2K_ERR_UNSUPPORTED, "three components without a colour transform"};
        if (ncomp == 1 && mct) throw ReadErr{J2K_ERR_INVALID_ARG, "colour transform on one component"};
        const int nb = 3 * levels + 1;
        if (qstyle == 1) {  // derived: every band from the LL exponent (E.1.1.1)
            if (eps.empty()) throw ReadErr{J2K_ERR_INVALID_ARG, "empty QCD"};
            const int e0 = eps[0], m0 = mant[0];
            eps.assign(nb, 0);
            mant.assign(nb, m0);
            for (int b = 0; b < nb; ++b) {
                const int lev = b == 0 ? levels : levels - (b - 1) / 3;  // decomposition level of band b
                eps[b] = e0 - (levels - lev);
            }
        }
        if ((int)eps.size() < nb) throw ReadErr{J2K_ERR_INVALID_ARG, "QCD lists fewer bands than the transform has"};
        I.levels = levels;
        I.cbw = cbw;
        I.cbh = cbh;
        I.lossless = xform == 1;
        I.mct = mct;
        I.guard = guard;
        I.layers = layers;
        I.progression = prog;
        I.cblk_style = sty & (J2K_CBLK_BYPASS | J2K_CBLK_RESET | J2K_CBLK_TERMALL);
        const int style = I.cblk_style;
        std::vector<j2k_band_rect> rects(nb);
        j2k_band_rects(I.w, I.h, levels, rects.data());
        for (int b = 0; b < nb && b < J2K_MAX_BANDS; ++b) {
            const int o = rects[b].orient;
            const int gain = o == J2K_BAND_LL ? 0 : (o == J2K_BAND_HH ? 2 : 1);
            I.steps[b] = I.lossless ? 1.0f : std::ldexp(1.0f + mant[b] / 2048.0f, 8 + gain - eps[b]);
        }
        if (header_only) {
            *info = I;
            return J2K_OK;
        }
        // code-blocks in job order (component, band, raster) and the packets of the tile
        std::vector<size_t> first((size_t)ncomp * nb + 1);
        std::vector<int> ncbx(nb), ncby(nb);
        size_t k = 0;
        for (int cc = 0; cc < ncomp; ++cc)
            for (int b = 0; b < nb; ++b) {
                first[(size_t)cc * nb + b] = k;
                ncbx[b] = (rects[b].w && rects[b].h) ? (int)((rects[b].w + cbw - 1) / cbw) : 0;
                ncby[b] = (rects[b].w && rects[b].h) ? (int)((rects[b].h + cbh - 1) / cbh) : 0;
                k += (size_t)ncbx[b] * ncby[b];
            }
        first[(size_t)ncomp * nb] = k;
        descs->assign(k, j2k_cb_desc{});
        segs->assign(k, {});
        for (int cc = 0; cc < ncomp; ++cc)
            for (int b = 0; b < nb; ++b)
                for (int j = 0; j < ncby[b]; ++j)
                    for (int i = 0; i < ncbx[b]; ++i) {
                        j2k_cb_desc& d = (*descs)[first[(size_t)cc * nb + b] + (size_t)j * ncbx[b] + i];
                        d.orient = (uint8_t)rects[b].orient;
                        d.band = (uint8_t)b;
                        d.x0 = (uint16_t)(rects[b].x0 + (size_t)i * cbw);
                        d.y0 = (uint16_t)(rects[b].y0 + (size_t)j * cbh);
                        d.cw = (uint16_t)std::min<size_t>(cbw, rects[b].w - (size_t)i * cbw);
                        d.ch = (uint16_t)std::min<size_t>(cbh, rects[b].h - (size_t)j * cbh);
                        d.comp = (uint16_t)cc;
                    }
        // per (component, band) tag trees and per block Lblock / inclusion state, kept across layers
        std::vector<TagTreeDec> incl, zbp;
        incl.reserve((size_t)ncomp * nb);
        zbp.reserve((size_t)ncomp * nb);
        for (int cc = 0; cc < ncomp; ++cc)
            for (int b = 0; b < nb; ++b) {
                incl.emplace_back(std::max(ncbx[b], 1), std::max(ncby[b], 1));
                zbp.emplace_back(std::max(ncbx[b], 1), std::max(ncby[b], 1));
            }
        std::vector<int> lblock(k, 3), tot_np(k, 0);
        if (pass_ends) pass_ends->assign(style ? k * J2K_PASS_STRIDE : 0, 0u);
        std::vector<uint8_t> included(k, 0);  // 0, or the block's bit-plane count once included
        const int keep = max_layers > 0 ? std::min(max_layers, layers) : layers;
        size_t pos = 0;
        const uint8_t* pd = data.data();
        const size_t pn = data.size();
        auto packet = [&](int l, int r, int cc) {
            if (scod & 2) {  // SOP marker segment before the packet
                if (pos + 6 <= pn && pd[pos] == 0xFF && pd[pos + 1] == 0x91) pos += 6;
            }
            const int b0 = r == 0 ? 0 : 1 + 3 * (r - 1);  // resolution r holds level L-r+1
            const int bcount = r == 0 ? 1 : 3;
            BitReader br(pd, pn, pos);
            std::vector<std::pair<size_t, int>> body;  // (block index, length) in packet order
            if (br.bit()) {
                for (int q = 0; q < bcount; ++q) {
                    const int b = b0 + q;
                    const int nbx = ncbx[b], nby = ncby[b];
                    if (!nbx || !nby) continue;
                    TagTreeDec& ti = incl[(size_t)cc * nb + b];
                    TagTreeDec& tz = zbp[(size_t)cc * nb + b];
                    const int Mb = guard + eps[b] - 1;
                    for (int j = 0; j < nby; ++j)
                        for (int i = 0; i < nbx; ++i) {
                            const size_t idx = first[(size_t)cc * nb + b] + (size_t)j * nbx + i;
                            j2k_cb_desc& d = (*descs)[idx];
                            if (!included[idx]) {
                                if (ti.decode(br, i, j, l + 1) >= l + 1) continue;  // not included yet
                                int z = 0;
                                while ((z = tz.decode(br, i, j, 1 << 30)) == (1 << 30)) {
                                }
                                const int nbps = Mb - z;
                                if (nbps < 1 || nbps > 31)
                                    throw ReadErr{J2K_ERR_INVALID_ARG, "inconsistent bit-planes"};
                                included[idx] = (uint8_t)nbps;
                            } else if (!br.bit()) {
                                continue;  // no new passes in this layer
                            }
                            const int np = get_npasses(br);
                            while (br.bit()) ++lblock[idx];
                            const int p0 = tot_np[idx];
                            tot_np[idx] += np;
                            if (tot_np[idx] > 3 * included[idx] - 2)
                                throw ReadErr{J2K_ERR_INVALID_ARG, "more passes than bit-planes allow"};
                            // the new passes as pieces of codeword segments (B.10.7.2): a piece
                            // ends where the style terminates the codeword, and at the last new
                            // pass; each has a length of Lblock + floor(log2(its passes)) bits
                            int64_t acc = 0;
                            int start = p0;
                            for (int q = p0; q < p0 + np; ++q) {
                                const bool term = style && q + 1 < 3 * included[idx] - 2 &&
                                                  j2k_pass_terminated(style, q, q + 2);
                                if (!term && q != p0 + np - 1) continue;
                                const int lbits = lblock[idx] + floorlog2(q + 1 - start);
                                if (lbits > 31)
                                    throw ReadErr{J2K_ERR_INVALID_ARG, "code-block length field too long"};
                                acc += (int64_t)br.bits(lbits);
                                if (acc + d.length > 0x7FFFFFFF)
                                    throw ReadErr{J2K_ERR_INVALID_ARG, "code-block length"};
                                if (pass_ends && style && l < keep)
                                    (*pass_ends)[idx * J2K_PASS_STRIDE + q] = (uint32_t)(d.length + acc);
                                start = q + 1;
                            }
                            const int len = (int)acc;
                            if (l < keep) {
                                d.numbps = included[idx];
                                d.npasses = (uint8_t)(d.npasses + np);
                                d.length += len;
                                body.push_back({idx, len});
                            } else {
                                body.push_back({(size_t)-1, len});
                            }
                        }
                }
            }
            pos = br.end();
            if (scod & 4) {  // EPH
                if (pos + 2 <= pn && pd[pos] == 0xFF && pd[pos + 1] == 0x92) pos += 2;
            }
            for (auto& e : body) {
                if (pos + (size_t)e.second > pn) throw ReadErr{J2K_ERR_INVALID_ARG, "packet body truncated"};
                if (e.first != (size_t)-1 && e.second > 0) (*segs)[e.first].push_back({(uint32_t)pos, e.second});
                pos += (size_t)e.second;
            }
        };
        if (prog == 0) {
            for (int l = 0; l < layers && l < keep; ++l)
                for (int r = 0; r <= levels; ++r)
                    for (int cc = 0; cc < ncomp; ++cc) packet(l, r, cc);
        } else {
            for (int r = 0; r <= levels; ++r)
                for (int l = 0; l < layers; ++l)
                    for (int cc = 0; cc < ncomp; ++cc) packet(l, r, cc);
        }
        *info = I;
        tile_bytes->swap(data);
        return J2K_OK;
    } catch (const ReadErr& e) {
        if (err) *err = e.msg;
        return e.s;
    }
}

}  // namespace

extern "C" j2k_status j2k_codestream_read_layers(const uint8_t* cs, size_t n, int max_layers, j2k_stream_info* info,
                                                 j2k_cb_desc* descs, size_t* count, uint8_t* bytes, size_t cap,
                                                 size_t* used, char* err, size_t errlen) {
    J2K_API_BEGIN
    if (!cs || !info || !count || !used || max_layers < 0) return J2K_ERR_INVALID_ARG;
    std::vector<j2k_cb_desc> d;
    std::vector<std::vector<std::pair<uint32_t, int>>> segs;
    std::vector<uint8_t> tile;
    std::string msg;
    j2k_status s = t2_read(cs, n, max_layers, info, &d, &segs, &tile, &msg);
    if (s != J2K_OK) {
        if (err && errlen) {
            std::strncpy(err, msg.c_str(), errlen - 1);
            err[errlen - 1] = 0;
        }
        return s;
    }
    size_t total = 0;
    for (const auto& x : d) total += (size_t)x.length;
    *count = d.size();
    *used = total;
    if (!descs && !bytes) return J2K_OK;
    if (!descs || !bytes || cap < total) return J2K_ERR_CAPACITY;
    size_t o = 0;
    for (size_t i = 0; i < d.size(); ++i) {
        d[i].offset = (uint32_t)o;
        for (const auto& sg : segs[i]) {
            std::memcpy(bytes + o, tile.data() + sg.first, (size_t)sg.second);
            o += (size_t)sg.second;
        }
        descs[i] = d[i];
    }
    return J2K_OK;
    J2K_API_END
}

j2k_status j2k_t2_parse_packed(const uint8_t* cs, size_t n, int max_layers, j2k_stream_info* info,
                               std::vector<j2k_cb_desc>* descs, std::vector<uint8_t>* bytes, std::string* err,
                               std::vector<uint32_t>* pass_ends) {
    std::vector<std::vector<std::pair<uint32_t, int>>> segs;
    std::vector<uint8_t> tile;
    J2K_TRY(t2_read(cs, n, max_layers, info, descs, &segs, &tile, err, false, pass_ends));
    size_t total = 0;
    for (const auto& x : *descs) total += (size_t)x.length;
    bytes->resize(total + 1);
    size_t o = 0;
    for (size_t i = 0; i < descs->size(); ++i) {
        (*descs)[i].offset = (uint32_t)o;
        for (const auto& sg : segs[i]) {
            std::memcpy(bytes->data() + o, tile.data() + sg.first, (size_t)sg.second);
            o += (size_t)sg.second;
        }
    }
    bytes->resize(o);
    return J2K_OK;
}

extern "C" j2k_status j2k_codestream_pass_ends(const uint8_t* cs, size_t n, int max_layers, uint32_t* ends,
                                               size_t cap, size_t* count, char* err, size_t errlen) {
    J2K_API_BEGIN
    if (!cs || !count || max_layers < 0) return J2K_ERR_INVALID_ARG;
    j2k_stream_info info{};
    std::vector<j2k_cb_desc> d;
    std::vector<std::vector<std::pair<uint32_t, int>>> segs;
    std::vector<uint8_t> tile;
    std::vector<uint32_t> pe;
    std::string msg;
    j2k_status s = t2_read(cs, n, max_layers, &info, &d, &segs, &tile, &msg, false, &pe);
    if (s != J2K_OK) {
        if (err && errlen) {
            std::strncpy(err, msg.c_str(), errlen - 1);
            err[errlen - 1] = 0;
        }
        return s;
    }
    *count = d.size() * J2K_PASS_STRIDE;
    if (!ends) return J2K_OK;
    if (cap < *count) return J2K_ERR_CAPACITY;
    if (pe.empty()) {  // no style: one segment per block, its whole codeword
        for (size_t i = 0; i < d.size(); ++i)
            for (int q = 0; q < J2K_PASS_STRIDE; ++q) ends[i * J2K_PASS_STRIDE + q] = (uint32_t)d[i].length;
    } else {
        std::memcpy(ends, pe.data(), pe.size() * 4);
    }
    return J2K_OK;
    J2K_API_END
}

extern "C" j2k_status j2k_codestream_info(const uint8_t* cs, size_t n, j2k_stream_info* info, char* err,
                                          size_t errlen) {
    J2K_API_BEGIN
    if (!cs || !info) return J2K_ERR_INVALID_ARG;
    std::string msg;
    j2k_status s = t2_read(cs, n, 0, info, nullptr, nullptr, nullptr, &msg, true);
    if (s != J2K_OK && err && errlen) {
        std::strncpy(err, msg.c_str(), errlen - 1);
        err[errlen - 1] = 0;
    }
    return s;
    J2K_API_END
}

extern "C" j2k_status j2k_codestream_read(const uint8_t* cs, size_t n, j2k_stream_info* info, j2k_cb_desc* descs,
                                          size_t* count, uint8_t* bytes, size_t cap, size_t* used, char* err,
                                          size_t errlen) {
    J2K_API_BEGIN
    return j2k_codestream_read_layers(cs, n, 0, info, descs, count, bytes, cap, used, err, errlen);
    J2K_API_END
}
