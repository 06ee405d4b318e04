// EBCOT tier-1 decoder (T.800 Annex D context modelling + Annex C.3 MQ decoder).
//
// The reference has no decoder for this stage (src/OCLDecoder.cpp:35-38 runs only the "reverse"
// DWT).  Decoding is serial per code-block: every context depends on the bits decoded before it.
// The default kernel runs one code-block per LANE: a warp decodes 8, 16 or 32 blocks side by side,
// each lane with its own MQ registers and its own 64-bit row masks of significance / sign /
// refined / visited in shared memory (interleaved by lane, so that the warp's accesses to any rows
// fall in distinct banks).  Lanes that take the same branch of the pass / stripe / column loops
// issue together; the decoder is bound by the latency of each decision's dependent chain, not by
// instruction issue, so a warp instruction that serves many blocks is what makes it fast.  The
// warp clears its blocks' output regions first and applies the signs at the end, cooperatively;
// magnitude bits go to the output plane by fire-and-forget atomic ORs (each block owns its region).
// The older form, one warp per block with lane 0 decoding, stays as a tuning choice.
#include <atomic>

#include <cub/cub.cuh>

#include "j2k_internal.cuh"

namespace {

constexpr int kWarps = 4;

// T.800 Table C.2 (probability estimation), device and host copies
__constant__ uint16_t d_qe[47] = {
    0x5601, 0x3401, 0x1801, 0x0AC1, 0x0521, 0x0221, 0x5601, 0x5401, 0x4801, 0x3801, 0x3001, 0x2401,
    0x1C01, 0x1601, 0x5601, 0x5401, 0x5101, 0x4801, 0x3801, 0x3401, 0x3001, 0x2801, 0x2401, 0x2201,
    0x1C01, 0x1801, 0x1601, 0x1401, 0x1201, 0x1101, 0x0AC1, 0x09C1, 0x08A1, 0x0521, 0x0441, 0x02A1,
    0x0221, 0x0141, 0x0111, 0x0085, 0x0049, 0x0025, 0x0015, 0x0009, 0x0005, 0x0001, 0x5601};
__constant__ uint8_t d_nmps[47] = {
    1,  2,  3,  4,  5,  38, 7,  8,  9,  10, 11, 12, 13, 29, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24,
    25, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 44, 45, 45, 46};
__constant__ uint8_t d_nlps[47] = {
    1,  6,  9,  12, 29, 33, 6,  14, 14, 14, 17, 18, 20, 21, 14, 14, 15, 16, 17, 18, 19, 19, 20, 21,
    22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 46};
[[maybe_unused]] static const uint16_t h_qe[47] = {
    0x5601, 0x3401, 0x1801, 0x0AC1, 0x0521, 0x0221, 0x5601, 0x5401, 0x4801, 0x3801, 0x3001, 0x2401,
    0x1C01, 0x1601, 0x5601, 0x5401, 0x5101, 0x4801, 0x3801, 0x3401, 0x3001, 0x2801, 0x2401, 0x2201,
    0x1C01, 0x1801, 0x1601, 0x1401, 0x1201, 0x1101, 0x0AC1, 0x09C1, 0x08A1, 0x0521, 0x0441, 0x02A1,
    0x0221, 0x0141, 0x0111, 0x0085, 0x0049, 0x0025, 0x0015, 0x0009, 0x0005, 0x0001, 0x5601};
[[maybe_unused]] static const uint8_t h_nmps[47] = {
    1,  2,  3,  4,  5,  38, 7,  8,  9,  10, 11, 12, 13, 29, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24,
    25, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 44, 45, 45, 46};
[[maybe_unused]] static const uint8_t h_nlps[47] = {
    1,  6,  9,  12, 29, 33, 6,  14, 14, 14, 17, 18, 20, 21, 14, 14, 15, 16, 17, 18, 19, 19, 20, 21,
    22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 46};
#ifdef __CUDA_ARCH__
#define QE(i) d_qe[i]
#define NMPS(i) d_nmps[i]
#define NLPS(i) d_nlps[i]
#else
#define QE(i) h_qe[i]
#define NMPS(i) h_nmps[i]
#define NLPS(i) h_nlps[i]
#endif

__host__ __device__ __forceinline__ int zc_label_calc(int orient, int h, int v, int d) {
    if (orient == J2K_BAND_HH) {
        int hv = h + v;
        if (d >= 3) return 8;
        if (d == 2) return hv >= 1 ? 7 : 6;
        if (d == 1) return hv >= 2 ? 5 : (hv == 1 ? 4 : 3);
        return hv >= 2 ? 2 : (hv == 1 ? 1 : 0);
    }
    if (orient == J2K_BAND_HL) { int t = h; h = v; v = t; }
    if (h == 2) return 8;
    if (h == 1) return v >= 1 ? 7 : (d >= 1 ? 6 : 5);
    if (v == 2) return 4;
    if (v == 1) return 3;
    return d >= 2 ? 2 : d;
}

// Lookup tables shared by the warps of a CTA (the host path builds its own copy).
//   zc[o][n9]: zero-coding label for orientation o and the 9-bit significance neighbourhood n9
//              (bits 0-2: row above, columns x-1..x+1; 3-5: own row; 6-8: row below; the
//              sample's own bit 4 is ignored; a significant neighbour is n9 & 0x1EF != 0)
//   sc[n8]:    sign-coding label | xor bit << 7 for n8 = sigL negL sigR negR sigU negU sigD negD
//   mq[i]:     Qe | NMPS << 16 | NLPS << 22 | SWITCH << 28 of probability state i (Table C.2)
struct DecTables {
    uint8_t zc[4][512];
    uint8_t sc[256];
    uint32_t mq[47];
};

__host__ __device__ inline void fill_tables_entry(DecTables& T, int i) {
    if (i < 4 * 512) {
        const int o = i >> 9, n = i & 511;
        const int h = ((n >> 3) & 1) + ((n >> 5) & 1), v = ((n >> 1) & 1) + ((n >> 7) & 1);
        const int d = (n & 1) + ((n >> 2) & 1) + ((n >> 6) & 1) + ((n >> 8) & 1);
        T.zc[o][n] = (uint8_t)zc_label_calc(o, h, v, d);
    }
    if (i < 256) {
        auto c = [&](int sh) { return ((i >> sh) & 1) ? (((i >> (sh + 1)) & 1) ? -1 : 1) : 0; };
        int hc = max(-1, min(1, c(0) + c(2))), vc = max(-1, min(1, c(4) + c(6)));
        int xr = 0;
        if (hc < 0 || (hc == 0 && vc < 0)) { hc = -hc; vc = -vc; xr = 1; }
        T.sc[i] = (uint8_t)((hc == 0 ? (vc ? 10 : 9) : 12 + vc) | (xr << 7));
    }
    if (i < 47)
        T.mq[i] = (uint32_t)QE(i) | ((uint32_t)NMPS(i) << 16) | ((uint32_t)NLPS(i) << 22) |
                  ((uint32_t)(i == 0 || i == 6 || i == 14) << 28);
}

__host__ __device__ __forceinline__ int clz32(uint32_t v) {
#ifdef __CUDA_ARCH__
    return __clz(v);
#else
    return v ? __builtin_clz(v) : 32;
#endif
}

// Decoder state of one code-block: rows of 64-bit masks (row r + 1 holds block row r; rows 0
// and 65 are the zero border) and the 19 MQ context states.
struct DecSmem {
    uint64_t sig_[66], neg_[66], ref_[66], vis_[66];
    uint8_t st_[19];
    __host__ __device__ uint64_t& sig(int r) { return sig_[r]; }
    __host__ __device__ uint64_t& neg(int r) { return neg_[r]; }
    __host__ __device__ uint64_t& ref(int r) { return ref_[r]; }
    __host__ __device__ uint64_t& vis(int r) { return vis_[r]; }
    __host__ __device__ uint8_t& st(int k) { return st_[k]; }
};

// The same state for the lanes of a warp that decode L blocks side by side: word (a, r, lane) of
// mask array a at base[(a * 66 + r) * L + lane], context state k at stb[k * L + lane].
template <int L>
struct LaneState {
    uint64_t* base;
    uint8_t* stb;
    int lane;
    __device__ uint64_t& sig(int r) { return base[(0 * 66 + r) * L + lane]; }
    __device__ uint64_t& neg(int r) { return base[(1 * 66 + r) * L + lane]; }
    __device__ uint64_t& ref(int r) { return base[(2 * 66 + r) * L + lane]; }
    __device__ uint64_t& vis(int r) { return base[(3 * 66 + r) * L + lane]; }
    __device__ uint8_t& st(int k) { return stb[k * L + lane]; }
};
template <int L>
__host__ __device__ constexpr size_t lane_state_bytes() {  // one warp's share: the masks, then the context states
    return (size_t)4 * 66 * L * 8 + (((size_t)19 * L + 15) & ~(size_t)15);
}

struct Mqd {
    const uint8_t* data;
    int len, bp, CT;
    uint32_t A, C;
    __host__ __device__ uint32_t byte(int i) const { return i < len ? data[i] : 0xFFu; }
    __host__ __device__ void bytein() {
        if (byte(bp) == 0xFF) {
            if (byte(bp + 1) > 0x8F) {
                C += 0xFF00;
                CT = 8;
            } else {
                ++bp;
                C += byte(bp) << 9;
                CT = 7;
            }
        } else {
            ++bp;
            C += byte(bp) << 8;
            CT = 8;
        }
    }
    __host__ __device__ void init(const uint8_t* d, int n) {
        data = d;
        len = n;
        bp = 0;
        C = byte(0) << 16;
        bytein();
        C <<= 7;
        CT -= 7;
        A = 0x8000;
    }
    // renormalisation by the leading-zero count at once, stopping for a byte-in whenever CT
    // runs out (the same steps as the bit-by-bit loop of C.3.3)
    __host__ __device__ __forceinline__ void renorm() {
        int sh = clz32(A) - 16;
        while (sh > 0) {
            if (CT == 0) bytein();
            const int k = min(sh, CT);
            A <<= k;
            C <<= k;
            CT -= k;
            sh -= k;
        }
    }
    __host__ __device__ int decode(uint8_t& st, const uint32_t* mq) {
        const uint32_t sv = st;
        const uint32_t e = mq[sv >> 1];
        const uint32_t qe = e & 0xFFFF;
        const int mps = sv & 1;
        A -= qe;
        int D, nm = mps;
        uint32_t nidx;
        if ((C >> 16) >= qe) {
            C -= qe << 16;
            if (A & 0x8000) return mps;  // MPS, no renormalisation
            if (A < qe) {                // conditional exchange: LPS
                D = 1 - mps;
                nm ^= (int)(e >> 28);
                nidx = (e >> 22) & 63;
            } else {
                D = mps;
                nidx = (e >> 16) & 63;
            }
        } else {
            if (A < qe) {  // conditional exchange: MPS
                D = mps;
                nidx = (e >> 16) & 63;
            } else {
                D = 1 - mps;
                nm ^= (int)(e >> 28);
                nidx = (e >> 22) & 63;
            }
            A = qe;
        }
        st = (uint8_t)((nidx << 1) | nm);
        renorm();
        return D;
    }
};

// bits x-1, x, x+1 of a row mask (bit 0 = column x-1); columns outside 0..63 read as 0
__host__ __device__ __forceinline__ int ctz64(uint64_t v) {
#ifdef __CUDA_ARCH__
    return __ffsll((long long)v) - 1;
#else
    return __builtin_ctzll(v);
#endif
}
__host__ __device__ __forceinline__ uint32_t nb3(uint64_t m, int x) {
    return (uint32_t)(x > 0 ? (m >> (x - 1)) & 7 : (m << 1) & 7);
}

// sign-coding neighbourhood of stripe row k of a column whose significance / sign neighbourhoods
// are W / NW (bits 3r..3r+2: columns x-1..x+1 of window row r): sigL negL sigR negR sigU negU
// sigD negD
__host__ __device__ __forceinline__ uint32_t sign_nbhd(uint32_t W, uint32_t NW, int k) {
    const int b = 3 * k;
    return ((W >> (b + 3)) & 1) | (((NW >> (b + 3)) & 1) << 1) | (((W >> (b + 5)) & 1) << 2) |
           (((NW >> (b + 5)) & 1) << 3) | (((W >> (b + 1)) & 1) << 4) | (((NW >> (b + 1)) & 1) << 5) |
           (((W >> (b + 7)) & 1) << 6) | (((NW >> (b + 7)) & 1) << 7);
}

// Raw (bypass) segment reader, T.800 D.6: bits most significant first; a byte after 0xFF holds
// 7 bits (its top bit is a stuffed 0); past the end of the segment 0xFF is read.
struct RawD {
    const uint8_t* data;
    int len, pos, ct;
    uint32_t c;
    bool lastff;
    __host__ __device__ void init(const uint8_t* d, int n) {
        data = d;
        len = n;
        pos = 0;
        ct = 0;
        c = 0;
        lastff = false;
    }
    __host__ __device__ int bit() {
        if (ct == 0) {
            const uint32_t b = pos < len ? data[pos] : 0xFFu;
            ++pos;
            ct = lastff ? 7 : 8;
            lastff = b == 0xFF;
            c = b;
        }
        --ct;
        return (int)((c >> ct) & 1);
    }
};

// Serial decode of one code-block into magnitudes (blk, pre-zeroed) and sign/state masks in S
// (a DecSmem, or a LaneState of a block decoded beside others in the same warp).  Host-callable
// so that the exact device logic can be checked on the CPU.  STYLED: the block was coded with
// code-block style `style` (contexts reset per pass, a new codeword segment after every
// terminated pass, located by the pass ends `pe`; raw-coded passes read as bits).  RED: magnitude
// bits are set by atomic ORs whose result is not read (device only).
template <bool STYLED = false, bool RED = false, class State>
__host__ __device__ void decode_block(State& S, const DecTables& T, const uint8_t* data, int len, int numbps,
                                      int npasses, int orient, int cw, int ch, int32_t* blk, size_t pitch,
                                      int style = 0, const uint32_t* pe = nullptr) {
        const uint8_t* zct = T.zc[orient];
        const uint32_t* mq = T.mq;

        auto reset_states = [&]() {
            for (int k = 0; k < 19; ++k) S.st(k) = 0;
            S.st(0) = 4 << 1;
            S.st(17) = 3 << 1;
            S.st(18) = 46 << 1;
        };
        reset_states();
        Mqd m;
        RawD rd;
        bool raw = false;
        if (!STYLED) m.init(data, len);
        // the start of pass q of a styled block: context reset, and a new segment after a
        // terminated pass
        auto begin = [&](int q) {
            if (!STYLED) return;
            if (q > 0 && (style & J2K_CBLK_RESET)) reset_states();
            raw = j2k_pass_raw(style, q);
            if (q == 0 || j2k_pass_terminated(style, q - 1, npasses)) {
                int e = q;
                while (!j2k_pass_terminated(style, e, npasses)) ++e;
                int b0 = q ? (int)min(pe[q - 1], (uint32_t)len) : 0;
                int b1 = (int)min(pe[e], (uint32_t)len);
                if (b1 < b0) b1 = b0;
                if (raw) rd.init(data + b0, b1 - b0);
                else m.init(data + b0, b1 - b0);
            }
        };
        // one decision in context cx, and one sign in sign context sc (label | xor << 7)
        auto dec = [&](int cx) -> int {
            if (STYLED && raw) return rd.bit();
            return m.decode(S.st(cx), mq);
        };
        auto dsign = [&](int sc) -> int {
            if (STYLED && raw) return rd.bit();
            return m.decode(S.st(sc & 31), mq) ^ (sc >> 7);
        };
        int pass = 0;
        const int nb = numbps, np = npasses;
        // a stripe column's neighbourhood, packed: bits 3r..3r+2 hold columns x-1..x+1 of block row
        // y0-1+r (r = 0..5), from the significance (or sign) rows; stripe row k's 9-bit
        // neighbourhood is then (W >> 3k) & 511 and its own bit 3k+4
        auto colw = [&](int y0, int x) -> uint32_t {
            uint32_t w = 0;
#ifdef __CUDA_ARCH__
            if (x > 0) {  // bits x-1..x+1 of each row: one funnel shift of its two halves
                const int s5 = (x - 1) & 31;
                const bool hiw = x - 1 >= 32;
                for (int r = 0; r < 6; ++r) {
                    const uint64_t m = S.sig(y0 + r);
                    const uint32_t lo = (uint32_t)m, hi = (uint32_t)(m >> 32);
                    const uint32_t t = hiw ? (hi >> s5) : __funnelshift_r(lo, hi, s5);
                    w |= (t & 7u) << (3 * r);
                }
                return w;
            }
#endif
            for (int r = 0; r < 6; ++r) w |= nb3(S.sig(y0 + r), x) << (3 * r);
            return w;
        };
        // the sign bits sign_nbhd reads for stripe row k of column x (left and right in its row,
        // above and below), from the sign rows as they are now
        auto negnb = [&](int y0, int x, int k) -> uint32_t {
            const uint64_t nu = S.neg(y0 + k), no = S.neg(y0 + k + 1), nd = S.neg(y0 + k + 2);
            const uint32_t l = x > 0 ? (uint32_t)(no >> (x - 1)) & 1u : 0u;
            const uint32_t r = x < 63 ? (uint32_t)(no >> (x + 1)) & 1u : 0u;
            return (((uint32_t)(nu >> x) & 1u) << (3 * k + 1)) | (l << (3 * k + 3)) | (r << (3 * k + 5)) |
                   (((uint32_t)(nd >> x) & 1u) << (3 * k + 7));
        };
        auto add_bit = [&](int x, int y, int p) {
#ifdef __CUDA_ARCH__
            if (RED) {
                atomicOr(reinterpret_cast<unsigned int*>(blk + (size_t)y * pitch + x), 1u << p);
                return;
            }
#endif
            blk[(size_t)y * pitch + x] |= 1 << p;
        };
        auto n8of = [](uint32_t W, uint32_t NW, int k) { return sign_nbhd(W, NW, k); };
        auto set_sig = [&](int x, int y, int neg, int p) {
            S.sig(y + 1) |= 1ull << x;
            if (neg) S.neg(y + 1) |= 1ull << x;
            add_bit(x, y, p);
        };
        const uint64_t cols = cw >= 64 ? ~0ull : ((1ull << cw) - 1);
        for (int p = nb - 1; p >= 0 && pass < np; --p) {
            if (p != nb - 1) {
                // significance propagation: only columns next to a significant sample can hold a
                // decision; a column joins when its left neighbour gains a significant sample
                begin(pass);
                for (int y0 = 0; y0 < ch; y0 += 4) {
                    const int ny = min(4, ch - y0);
                    uint64_t cm = 0;
                    for (int y = y0; y < y0 + ny; ++y) {
                        const uint64_t own = S.sig(y + 1);
                        uint64_t nbm = S.sig(y) | own | S.sig(y + 2);
                        nbm |= (nbm << 1) | (nbm >> 1);
                        cm |= ~own & nbm;
                    }
                    cm &= cols;
                    uint64_t vacc[4] = {0, 0, 0, 0};  // this stripe's visits, stored once at its end
                    while (cm) {
                        const int x = ctz64(cm);
                        cm &= cm - 1;
                        uint32_t W = colw(y0, x), vb = 0;
                        for (int k = 0; k < ny; ++k) {  // one decoding site: not unrolled
                            if ((W >> (3 * k + 4)) & 1) continue;  // significant already
                            const uint32_t n9 = (W >> (3 * k)) & 511;
                            if (!(n9 & 0x1EF)) continue;           // no significant neighbour
                            const int bit = dec(zct[n9]);
                            vb |= 1u << k;
                            if (bit) {
                                const int sc = T.sc[n8of(W, negnb(y0, x, k), k)];
                                const int sg = dsign(sc);
                                set_sig(x, y0 + k, sg, p);
                                W |= 1u << (3 * k + 4);
                                cm |= (2ull << x) & cols;
                            }
                        }
#pragma unroll
                        for (int k = 0; k < 4; ++k) vacc[k] |= (uint64_t)((vb >> k) & 1) << x;
                    }
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (k < ny) S.vis(y0 + k + 1) |= vacc[k];
                }
                if (++pass >= np) break;
                // magnitude refinement: significant samples not visited in this plane
                begin(pass);
                for (int y0 = 0; y0 < ch; y0 += 4) {
                    const int ny = min(4, ch - y0);
                    // per stripe row k, as masks over the columns (this pass changes none of
                    // them): the samples to refine (significant, not visited in this plane), the
                    // ones refined before (label 16), and the ones with a significant neighbour
                    // (label 15, else 14)
                    uint64_t mr[4] = {0, 0, 0, 0}, rf[4] = {0, 0, 0, 0}, nbs[4] = {0, 0, 0, 0};
                    uint64_t rm = 0;
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        if (k >= ny) break;
                        const uint64_t own = S.sig(y0 + k + 1), v3 = S.sig(y0 + k) | S.sig(y0 + k + 2);
                        mr[k] = own & ~S.vis(y0 + k + 1) & cols;
                        rf[k] = S.ref(y0 + k + 1);
                        nbs[k] = v3 | (v3 << 1) | (v3 >> 1) | (own << 1) | (own >> 1);
                        rm |= mr[k];
                    }
                    while (rm) {
                        const int x = ctz64(rm);
                        rm &= rm - 1;
                        uint32_t mb = 0, rb = 0, nbb = 0;  // the column's rows, as 4-bit masks
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            mb |= (uint32_t)((mr[k] >> x) & 1) << k;
                            rb |= (uint32_t)((rf[k] >> x) & 1) << k;
                            nbb |= (uint32_t)((nbs[k] >> x) & 1) << k;
                        }
                        while (mb) {  // one decoding site
                            const int k = ctz64(mb);
                            mb &= mb - 1;
                            const int lab = ((rb >> k) & 1) ? 16 : (((nbb >> k) & 1) ? 15 : 14);
                            if (dec(lab)) add_bit(x, y0 + k, p);
                        }
                    }
                    // every sample of mr was refined in this pass
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (k < ny) S.ref(y0 + k + 1) = rf[k] | mr[k];
                }
                if (++pass >= np) break;
            }
            // cleanup: every insignificant sample not visited in this plane
            begin(pass);
            for (int y0 = 0; y0 < ch; y0 += 4) {
                const int ny = min(4, ch - y0);
                // per stripe row k: the samples this pass codes (insignificant, not visited in
                // this plane); a sample that becomes significant here is the one being coded, so
                // the masks hold for the whole pass
                uint64_t un[4] = {0, 0, 0, 0};
                uint64_t um = 0;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (k >= ny) break;
                    un[k] = ~S.sig(y0 + k + 1) & ~S.vis(y0 + k + 1) & cols;
                    um |= un[k];
                }
                while (um) {
                    const int x = ctz64(um);
                    um &= um - 1;
                    uint32_t W = colw(y0, x), U = 0;  // U: rows of the column to code
#pragma unroll
                    for (int k = 0; k < 4; ++k) U |= (uint32_t)((un[k] >> x) & 1) << k;
                    int start = 0;
                    if (ny == 4 && W == 0 && U == 15) {
                        // run-length mode: four insignificant, unvisited samples, no significant
                        // neighbour (every bit of the column's neighbourhood is zero)
                        if (!dec(17)) continue;
                        int idx = dec(18) << 1;
                        idx |= dec(18);
                        const int sc = T.sc[0];
                        const int sg = dsign(sc);
                        set_sig(x, y0 + idx, sg, p);
                        W |= 1u << (3 * idx + 4);
                        start = idx + 1;
                    }
                    for (int k = start; k < ny; ++k) {
                        if (!((U >> k) & 1)) continue;
                        if (dec(zct[(W >> (3 * k)) & 511])) {
                            const int sc = T.sc[n8of(W, negnb(y0, x, k), k)];
                            const int sg = dsign(sc);
                            set_sig(x, y0 + k, sg, p);
                            W |= 1u << (3 * k + 4);
                        }
                    }
                }
            }
            ++pass;
            for (int r = 0; r < 66; ++r) S.vis(r) = 0;
        }
}

// the checks a decoder kernel makes of a job before touching its region
__device__ __forceinline__ bool dec_job_ok(const j2k_cb_job& J, const j2k_cb_desc& D, bool styled) {
    return !(J.cw == 0 || J.ch == 0 || J.cw > 64 || J.ch > 64 || J.orient > 3 || D.numbps > 31 ||
             D.npasses > 3 * D.numbps || D.length < 0 || (styled && D.npasses > J2K_PASS_STRIDE - 1));
}

// magnitude offset of a block cut at the end of a bit-plane above the last one (rate control):
// significant magnitudes are reconstructed at the middle of the interval their undecoded bits leave
__host__ __device__ __forceinline__ int32_t cut_half(int numbps, int npasses) {
    if (npasses < 3 * numbps - 2 && (npasses - 1) % 3 == 0) {
        const int plast = numbps - 1 - (npasses - 1) / 3;
        return plast > 0 ? 1 << (plast - 1) : 0;
    }
    return 0;
}

template <bool STYLED>
__global__ void __launch_bounds__(kWarps * 32)
t1_decode_kernel(const j2k_cb_desc* __restrict__ descs, const uint8_t* __restrict__ bytes,
                 const j2k_cb_job* __restrict__ jobs, int njobs, int32_t* __restrict__ coeff,
                 uint32_t* __restrict__ err, int style, const uint32_t* __restrict__ pass_ends,
                 const uint8_t* __restrict__ job_style) {
    __shared__ DecSmem smem[kWarps];
    __shared__ DecTables tabs;
    for (int i = threadIdx.x; i < 4 * 512; i += blockDim.x) fill_tables_entry(tabs, i);
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int jid = blockIdx.x * kWarps + wid;
    if (jid >= njobs) return;
    DecSmem& S = smem[wid];
    const j2k_cb_job J = jobs[jid];
    const j2k_cb_desc D = descs[jid];
    const int cw = J.cw, ch = J.ch, orient = J.orient;
    // (a styled block's passes index its pass ends: at most 3 * 31 - 2 of them)
    if (!dec_job_ok(J, D, STYLED)) {
        if (lane == 0) atomicCAS(err, 0u, (uint32_t)J2K_DEVERR_BAD_JOB);
        return;
    }
    const size_t pitch = J.pitch;
    int32_t* blk = coeff + J.off;
    for (int r = 0; r < ch; ++r)
        for (int x = lane; x < cw; x += 32) blk[(size_t)r * pitch + x] = 0;
    for (int r = lane; r < 66; r += 32) { S.sig_[r] = 0; S.neg_[r] = 0; S.ref_[r] = 0; S.vis_[r] = 0; }
    if (lane < 19) S.st_[lane] = 0;
    __syncwarp();
    if (lane == 0 && D.numbps > 0 && D.npasses > 0)
        decode_block<STYLED>(S, tabs, bytes + D.offset, D.length, D.numbps, D.npasses, orient, cw, ch, blk, pitch,
                             job_style ? (int)job_style[jid] : style,
                             STYLED ? pass_ends + (size_t)jid * J2K_PASS_STRIDE : nullptr);
    __syncwarp();
    const int32_t half = cut_half(D.numbps, D.npasses);
    for (int r = 0; r < ch; ++r)
        for (int x = lane; x < cw; x += 32) {
            int32_t v = blk[(size_t)r * pitch + x];
            if ((S.sig_[r + 1] >> x) & 1) v += half;
            if ((S.neg_[r + 1] >> x) & 1) v = -v;
            blk[(size_t)r * pitch + x] = v;
        }
}


constexpr size_t kTablesBytes = (sizeof(DecTables) + 15) & ~(size_t)15;
// warps per CTA of the lane-per-block decoders for L blocks per warp: 32 blocks per CTA for
// L >= 8, four warps for smaller L (so that a CTA's shared-memory state stays near 70 KB or less)
template <int L>
__host__ __device__ constexpr int cta_warps() {
    return L >= 8 ? 32 / L : 4;
}

template <int L>
__host__ __device__ constexpr size_t lanes_smem_bytes() {
    return kTablesBytes + (size_t)cta_warps<L>() * lane_state_bytes<L>();
}

// One code-block per lane: a CTA takes 32 consecutive jobs (of `order` when given: the jobs
// sorted by codeword length, longest first, so that the blocks sharing a warp take about as long
// and the longest start first) in 32 / L warps of L (lanes 0..L-1 of a warp decode, one block each); every lane of the warp helps clear its blocks' regions first
// and apply the signs at the end.  Dynamic shared memory: the tables, then each warp's
// LaneState<L> area.
template <bool STYLED, int L>
__global__ void __launch_bounds__(32 * cta_warps<L>())
t1_decode_lanes_kernel(const j2k_cb_desc* __restrict__ descs, const uint8_t* __restrict__ bytes,
                       const j2k_cb_job* __restrict__ jobs, int njobs, int32_t* __restrict__ coeff,
                       uint32_t* __restrict__ err, int style, const uint32_t* __restrict__ pass_ends,
                       const uint8_t* __restrict__ job_style, const uint32_t* __restrict__ order) {
    extern __shared__ __align__(16) uint8_t dsm[];
    DecTables& tabs = *reinterpret_cast<DecTables*>(dsm);
    for (int i = threadIdx.x; i < 4 * 512; i += blockDim.x) fill_tables_entry(tabs, i);
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int j0 = (blockIdx.x * cta_warps<L>() + wid) * L;
    if (j0 >= njobs) return;
    const int nb = min(L, njobs - j0);
    uint8_t* wsm = dsm + kTablesBytes + (size_t)wid * lane_state_bytes<L>();
    uint64_t* base = reinterpret_cast<uint64_t*>(wsm);
    uint8_t* stb = wsm + (size_t)4 * 66 * L * 8;
    j2k_cb_job J{};
    j2k_cb_desc D{};
    bool ok = false;
    // this lane's job: position j0 + lane of the order (longest codewords first), or of the list
    const int jid = lane < nb ? (order ? (int)order[j0 + lane] : j0 + lane) : 0;
    if (lane < nb) {
        J = jobs[jid];
        D = descs[jid];
        ok = dec_job_ok(J, D, STYLED);
        if (!ok) atomicCAS(err, 0u, (uint32_t)J2K_DEVERR_BAD_JOB);
    }
    const unsigned okmask = __ballot_sync(~0u, ok);
    for (int i = lane; i < 4 * 66 * L; i += 32) base[i] = 0;
    for (int b = 0; b < nb; ++b) {
        if (!((okmask >> b) & 1)) continue;
        const int cw = __shfl_sync(~0u, (int)J.cw, b), ch = __shfl_sync(~0u, (int)J.ch, b);
        const size_t pitch = __shfl_sync(~0u, J.pitch, b);
        int32_t* blk = coeff + __shfl_sync(~0u, (unsigned long long)J.off, b);
        for (int r = 0; r < ch; ++r)
            for (int x = lane; x < cw; x += 32) blk[(size_t)r * pitch + x] = 0;
    }
    __syncwarp();
    if (ok && D.numbps > 0 && D.npasses > 0) {
        LaneState<L> S{base, stb, lane};
        decode_block<STYLED, true>(S, tabs, bytes + D.offset, D.length, D.numbps, D.npasses, J.orient, J.cw, J.ch,
                                   coeff + J.off, J.pitch, job_style ? (int)job_style[jid] : style,
                                   STYLED ? pass_ends + (size_t)jid * J2K_PASS_STRIDE : nullptr);
    }
    __syncwarp();
    const int32_t my_half = ok ? cut_half(D.numbps, D.npasses) : 0;
    for (int b = 0; b < nb; ++b) {
        if (!((okmask >> b) & 1)) continue;
        const int cw = __shfl_sync(~0u, (int)J.cw, b), ch = __shfl_sync(~0u, (int)J.ch, b);
        const size_t pitch = __shfl_sync(~0u, J.pitch, b);
        int32_t* blk = coeff + __shfl_sync(~0u, (unsigned long long)J.off, b);
        const int32_t half = __shfl_sync(~0u, my_half, b);
        for (int r = 0; r < ch; ++r) {
            const uint64_t sg = base[(0 * 66 + r + 1) * L + b], ng = base[(1 * 66 + r + 1) * L + b];
            for (int x = lane; x < cw; x += 32) {
                int32_t v = __ldcg(blk + (size_t)r * pitch + x);
                if ((sg >> x) & 1) v += half;
                if ((ng >> x) & 1) v = -v;
                blk[(size_t)r * pitch + x] = v;
            }
        }
    }
}


// symbol kinds, pass kinds and pending symbols of decode_block_steps
enum : int { kSymZC = 0, kSymSign = 1, kSymMR = 2, kSymRL = 3, kSymUni = 4 };
enum : int { kPassCU = 0, kPassSP = 1, kPassMR = 2 };
enum : int { kPendNone = 0, kPendSign = 1, kPendUni1 = 2, kPendUni2 = 3 };

// The same decode as decode_block (unstyled blocks), written as a loop of one symbol per step:
// (1) advance the cursor (pass, stripe, column, row) to the next sample that codes a symbol in its
// pass, or take the pending sign / run-length index symbol, (2) decode that one symbol -- the MQ
// decoder's only call site -- and (3) apply it.  Lanes of a warp that decode different blocks
// with it stay together on the decoding step whatever pass or column each is in.  The scan
// order, contexts and pass rules are T.800 D.3-D.5 (significance propagation, magnitude
// refinement and cleanup passes, stripes of four rows scanned column by column, the cleanup
// pass's run-length mode).  Host-callable, for the tests.
template <bool RED = false, class State>
__host__ __device__ void decode_block_steps(State& S, const DecTables& tabs, const uint8_t* data, int len, int numbps,
                                            int npasses, int orient, int cw, int ch, int32_t* blk, size_t pitch,
                                            bool active = true) {
    auto add_bit = [&](int x, int y, int p) {
#ifdef __CUDA_ARCH__
        if (RED) {
            atomicOr(reinterpret_cast<unsigned int*>(blk + (size_t)y * pitch + x), 1u << p);
            return;
        }
#endif
        blk[(size_t)y * pitch + x] |= 1 << p;
    };
    const uint8_t* zct = tabs.zc[orient & 3];
    const uint32_t* mq = tabs.mq;
    const int np = npasses;
    const uint64_t cols = cw >= 64 ? ~0ull : ((1ull << cw) - 1);
    Mqd m;
    if (active) {
        for (int c = 0; c < 19; ++c) S.st(c) = 0;
        S.st(0) = 4 << 1;
        S.st(17) = 3 << 1;
        S.st(18) = 46 << 1;
        m.init(data, len);
    }
    // cursor
    int pass = 0, ptype = kPassCU, p = numbps - 1, y0 = 0, x = 0, k = 4, ny = min(4, ch);
    int pending = kPendNone, idx = 0;
    bool colstart = false, nwv = false;
    uint32_t W = 0, NW = 0, V = 0, R = 0;
    uint64_t cm = 0;
    // candidate columns of the stripe at y0 in the current pass
    auto stripe_setup = [&]() {
        ny = min(4, ch - y0);
        uint64_t c = 0;
        for (int r = 0; r < ny; ++r) {
            const uint64_t own = S.sig(y0 + r + 1);
            if (ptype == kPassSP) {
                uint64_t nbm = S.sig(y0 + r) | own | S.sig(y0 + r + 2);
                nbm |= (nbm << 1) | (nbm >> 1);
                c |= ~own & nbm;
            } else {
                const uint64_t vis = S.vis(y0 + r + 1);
                c |= (ptype == kPassMR ? own : ~own) & ~vis;
            }
        }
        cm = c & cols;
    };
    auto colw = [&](bool negs) -> uint32_t {
        uint32_t w = 0;
        for (int r = 0; r < 6; ++r) w |= nb3(negs ? S.neg(y0 + r) : S.sig(y0 + r), x) << (3 * r);
        return w;
    };
    if (active) stripe_setup();
    // rows of the current column, from row k on, that code a symbol in this pass
    auto cand_rows = [&]() -> uint32_t {
        const uint32_t s4 = ((W >> 4) & 1) | ((W >> 6) & 2) | ((W >> 8) & 4) | ((W >> 10) & 8);
        uint32_t rows;
        if (ptype == kPassSP) {
            uint32_t n4 = 0;
            for (int r = 0; r < 4; ++r) n4 |= (uint32_t)(((W >> (3 * r)) & 0x1EF) != 0) << r;
            rows = ~s4 & n4;
        } else {
            rows = (ptype == kPassMR ? s4 : ~s4) & ~V;
        }
        return rows & ((1u << ny) - 1) & (0xFu << k);
    };
    // On the device every lane of the warp runs this loop (lanes without a block, or done with
    // theirs, inactive), and the vote at the top of each step brings the lanes back together
    // before the next symbol, however their searches diverged.
#ifdef __CUDA_ARCH__
    while (__any_sync(0xffffffffu, active)) {
        if (!active) continue;
#else
    while (active) {
#endif
        int kind = kSymUni;
        if (pending == kPendSign) {
            kind = kSymSign;
        } else if (pending == kPendNone) {
            bool done = false;
            for (;;) {
                if (k < 4) {
                    if (ptype == kPassCU && colstart && ny == 4 && W == 0 && V == 0) {
                        kind = kSymRL;  // run-length mode: no significant sample around the column
                        break;
                    }
                    const uint32_t rows = cand_rows();
                    if (rows) {
                        k = ctz64(rows);
                        kind = ptype == kPassMR ? kSymMR : kSymZC;
                        break;
                    }
                    k = 4;
                }
                if (cm) {  // next column of the stripe that holds a candidate
                    x = ctz64(cm);
                    cm &= cm - 1;
                    W = colw(false);
                    nwv = false;
                    V = 0;
                    R = 0;
                    if (ptype != kPassSP)
                        for (int r = 0; r < ny; ++r) V |= (uint32_t)((S.vis(y0 + r + 1) >> x) & 1) << r;
                    if (ptype == kPassMR)
                        for (int r = 0; r < ny; ++r) R |= (uint32_t)((S.ref(y0 + r + 1) >> x) & 1) << r;
                    k = 0;
                    colstart = true;
                    continue;
                }
                if (y0 + 4 < ch) {  // next stripe
                    y0 += 4;
                    stripe_setup();
                    continue;
                }
                // end of the pass
                if (ptype == kPassCU)
                    for (int r = 0; r < 66; ++r) S.vis(r) = 0;
                if (++pass >= np || (ptype == kPassCU && p == 0)) {  // (the last plane's cleanup ends it)
                    done = true;
                    break;
                }
                if (ptype == kPassCU) {
                    --p;
                    ptype = kPassSP;
                } else {
                    ptype = ptype == kPassSP ? kPassMR : kPassCU;
                }
                y0 = 0;
                stripe_setup();
            }
            if (done) {
                active = false;
                continue;
            }
        }
        // the symbol's context (sign symbols: label | xor bit << 7)
        int cx, xr = 0;
        if (kind == kSymZC) {
            cx = zct[(W >> (3 * k)) & 511];
        } else if (kind == kSymMR) {
            cx = ((R >> k) & 1) ? 16 : (((W >> (3 * k)) & 0x1EF) ? 15 : 14);
        } else if (kind == kSymSign) {
            if (!nwv && W) {  // (with no significant neighbour the signs around do not matter)
                NW = colw(true);
                nwv = true;
            }
            const int sc = tabs.sc[sign_nbhd(W, NW, k)];
            cx = sc & 31;
            xr = sc >> 7;
        } else {
            cx = kind == kSymRL ? 17 : 18;
        }
        const int d = m.decode(S.st(cx), mq) ^ xr;
        if (kind == kSymZC) {
            if (ptype == kPassSP) S.vis(y0 + k + 1) |= 1ull << x;
            if (d) pending = kPendSign;
            else ++k;
            colstart = false;
        } else if (kind == kSymSign) {
            const int y = y0 + k;
            S.sig(y + 1) |= 1ull << x;
            if (d) S.neg(y + 1) |= 1ull << x;
            add_bit(x, y, p);
            W |= 1u << (3 * k + 4);
            NW |= (uint32_t)d << (3 * k + 4);
            if (ptype == kPassSP) cm |= (2ull << x) & cols;
            pending = kPendNone;
            ++k;
        } else if (kind == kSymMR) {
            const int y = y0 + k;
            if (d) add_bit(x, y, p);
            S.ref(y + 1) |= 1ull << x;
            ++k;
        } else if (kind == kSymRL) {
            colstart = false;
            if (d) pending = kPendUni1;
            else k = 4;
        } else if (pending == kPendUni1) {
            idx = d << 1;
            pending = kPendUni2;
        } else {
            k = idx | d;
            pending = kPendSign;
        }
    }
}

// One code-block per lane, each decoded by decode_block_steps.

template <int L>
__global__ void __launch_bounds__(32 * cta_warps<L>())
t1_decode_steps_kernel(const j2k_cb_desc* __restrict__ descs, const uint8_t* __restrict__ bytes,
                       const j2k_cb_job* __restrict__ jobs, int njobs, int32_t* __restrict__ coeff,
                       uint32_t* __restrict__ err) {
    extern __shared__ __align__(16) uint8_t dsm[];
    DecTables& tabs = *reinterpret_cast<DecTables*>(dsm);
    for (int i = threadIdx.x; i < 4 * 512; i += blockDim.x) fill_tables_entry(tabs, i);
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int j0 = (blockIdx.x * cta_warps<L>() + wid) * L;
    if (j0 >= njobs) return;
    const int nb = min(L, njobs - j0);
    uint8_t* wsm = dsm + kTablesBytes + (size_t)wid * lane_state_bytes<L>();
    uint64_t* base = reinterpret_cast<uint64_t*>(wsm);
    uint8_t* stb = wsm + (size_t)4 * 66 * L * 8;
    j2k_cb_job J{};
    j2k_cb_desc D{};
    bool ok = false;
    if (lane < nb) {
        J = jobs[j0 + lane];
        D = descs[j0 + lane];
        ok = dec_job_ok(J, D, false);
        if (!ok) atomicCAS(err, 0u, (uint32_t)J2K_DEVERR_BAD_JOB);
    }
    const unsigned okmask = __ballot_sync(~0u, ok);
    for (int i = lane; i < 4 * 66 * L; i += 32) base[i] = 0;
    for (int b = 0; b < nb; ++b) {
        if (!((okmask >> b) & 1)) continue;
        const int cw = __shfl_sync(~0u, (int)J.cw, b), ch = __shfl_sync(~0u, (int)J.ch, b);
        const size_t pitch = __shfl_sync(~0u, J.pitch, b);
        int32_t* blk = coeff + __shfl_sync(~0u, (unsigned long long)J.off, b);
        for (int r = 0; r < ch; ++r)
            for (int x = lane; x < cw; x += 32) blk[(size_t)r * pitch + x] = 0;
    }
    __syncwarp();
    {  // every lane of the warp takes part in the step loop, whether or not it has a block
        LaneState<L> S{base, stb, lane < L ? lane : 0};
        const bool act = ok && D.numbps > 0 && D.npasses > 0;
        decode_block_steps<true>(S, tabs, bytes + D.offset, D.length, D.numbps, D.npasses, J.orient, J.cw, J.ch,
                                 coeff + J.off, J.pitch, act);
    }
    __syncwarp();
    const int32_t my_half = ok ? cut_half(D.numbps, D.npasses) : 0;
    for (int b = 0; b < nb; ++b) {
        if (!((okmask >> b) & 1)) continue;
        const int cw = __shfl_sync(~0u, (int)J.cw, b), ch = __shfl_sync(~0u, (int)J.ch, b);
        const size_t pitch = __shfl_sync(~0u, J.pitch, b);
        int32_t* blk = coeff + __shfl_sync(~0u, (unsigned long long)J.off, b);
        const int32_t half = __shfl_sync(~0u, my_half, b);
        for (int r = 0; r < ch; ++r) {
            const uint64_t sg = base[(0 * 66 + r + 1) * L + b], ng = base[(1 * 66 + r + 1) * L + b];
            for (int x = lane; x < cw; x += 32) {
                int32_t v = __ldcg(blk + (size_t)r * pitch + x);
                if ((sg >> x) & 1) v += half;
                if ((ng >> x) & 1) v = -v;
                blk[(size_t)r * pitch + x] = v;
            }
        }
    }
}

}  // namespace

// Host execution of the device decoder logic for one block (used by the test suite): the pass /
// stripe / column loops that the default decoder kernel runs in each lane, or (steps != 0) the
// one-symbol-per-step loop of J2K_TUNE_T1D_STEPS.
static int decode_block_host(const uint8_t* data, int len, int numbps, int npasses, int orient, int cw, int ch,
                             int32_t* out, size_t pitch, bool steps) {
    if (cw < 1 || ch < 1 || cw > 64 || ch > 64 || orient < 0 || orient > 3 || numbps < 0 || numbps > 31 ||
        npasses < 0 || npasses > 3 * numbps || len < 0 || (len > 0 && !data) || !out || pitch < (size_t)cw)
        return -1;  // the checks the kernel makes of a descriptor, and the host buffers
    DecSmem S;
    for (int r = 0; r < 66; ++r) S.sig_[r] = S.neg_[r] = S.ref_[r] = S.vis_[r] = 0;
    for (int k = 0; k < 19; ++k) S.st_[k] = 0;
    static const DecTables T = [] {  // built once, thread-safely
        DecTables t{};
        for (int i = 0; i < 4 * 512; ++i) fill_tables_entry(t, i);
        return t;
    }();
    for (int y = 0; y < ch; ++y)
        for (int x = 0; x < cw; ++x) out[(size_t)y * pitch + x] = 0;
    if (numbps > 0 && npasses > 0) {
        if (steps) decode_block_steps(S, T, data, len, numbps, npasses, orient, cw, ch, out, pitch);
        else decode_block(S, T, data, len, numbps, npasses, orient, cw, ch, out, pitch);
    }
    for (int y = 0; y < ch; ++y)
        for (int x = 0; x < cw; ++x)
            if ((S.neg_[y + 1] >> x) & 1) out[(size_t)y * pitch + x] = -out[(size_t)y * pitch + x];
    return 0;
}

extern "C" int j2k_t1_decode_block_host(const uint8_t* data, int len, int numbps, int npasses, int orient,
                                        int cw, int ch, int32_t* out, size_t pitch) {
    return decode_block_host(data, len, numbps, npasses, orient, cw, ch, out, pitch, false);
}

extern "C" int j2k_t1_decode_block_steps_host(const uint8_t* data, int len, int numbps, int npasses, int orient,
                                              int cw, int ch, int32_t* out, size_t pitch) {
    return decode_block_host(data, len, numbps, npasses, orient, cw, ch, out, pitch, true);
}

// The same for a block coded with a code-block style, its segments located by pass_ends
// (J2K_PASS_STRIDE entries; values past len are clamped to it, as the kernel does).
extern "C" int j2k_t1_decode_block_styled_host(const uint8_t* data, int len, const uint32_t* pass_ends, int numbps,
                                               int npasses, int orient, int style, int cw, int ch, int32_t* out,
                                               size_t pitch) {
    if (cw < 1 || ch < 1 || cw > 64 || ch > 64 || orient < 0 || orient > 3 || numbps < 0 || numbps > 31 ||
        npasses < 0 || npasses > 3 * numbps || npasses > J2K_PASS_STRIDE - 1 || len < 0 || (len > 0 && !data) ||
        !out || pitch < (size_t)cw || !pass_ends || style < 0 || style > 7)
        return -1;
    DecSmem S;
    for (int r = 0; r < 66; ++r) S.sig_[r] = S.neg_[r] = S.ref_[r] = S.vis_[r] = 0;
    for (int k = 0; k < 19; ++k) S.st_[k] = 0;
    static const DecTables T = [] {
        DecTables t{};
        for (int i = 0; i < 4 * 512; ++i) fill_tables_entry(t, i);
        return t;
    }();
    for (int y = 0; y < ch; ++y)
        for (int x = 0; x < cw; ++x) out[(size_t)y * pitch + x] = 0;
    if (numbps > 0 && npasses > 0)
        decode_block<true>(S, T, data, len, numbps, npasses, orient, cw, ch, out, pitch, style, pass_ends);
    for (int y = 0; y < ch; ++y)
        for (int x = 0; x < cw; ++x)
            if ((S.neg_[y + 1] >> x) & 1) out[(size_t)y * pitch + x] = -out[(size_t)y * pitch + x];
    return 0;
}

template <bool STYLED, int L>
static j2k_status launch_lanes(j2k_ctx* ctx, cudaStream_t st, const j2k_cb_desc* descs,
                               const uint8_t* bytes, const j2k_cb_job* d_jobs, size_t njobs, int32_t* coeff,
                               int style, const uint32_t* pass_ends, const uint8_t* job_style,
                               const uint32_t* order) {
    constexpr size_t smem = lanes_smem_bytes<L>();
    const unsigned grid = (unsigned)((njobs + L * cta_warps<L>() - 1) / (L * cta_warps<L>()));
    static std::atomic<uint64_t> attr_set{0};  // devices whose attribute is set, per instantiation
    const uint64_t bit = 1ull << (ctx->device & 63);
    if (!(attr_set.load() & bit)) {
        J2K_CUDA(ctx, cudaFuncSetAttribute(t1_decode_lanes_kernel<STYLED, L>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr_set.fetch_or(bit);
    }
    t1_decode_lanes_kernel<STYLED, L><<<grid, 32 * cta_warps<L>(), smem, st>>>(
        descs, bytes, d_jobs, (int)njobs, coeff, ctx->d_err, style, pass_ends, job_style, order);
    J2K_CUDA(ctx, cudaGetLastError());
    return J2K_OK;
}

// keys[i] = codeword length of job i, ids[i] = i
__global__ void t1d_order_keys(const j2k_cb_desc* __restrict__ descs, int n, uint32_t* __restrict__ keys,
                               uint32_t* __restrict__ ids) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t len = descs[i].length;
    keys[i] = len > 0 ? (uint32_t)len : 0u;
    ids[i] = (uint32_t)i;
}

// The jobs sorted by codeword length, longest first (a stable radix sort: equal lengths keep
// their list order), in scratch; nullptr with the error set when scratch runs out.
static const uint32_t* decode_order(j2k_ctx* ctx, cudaStream_t st, const j2k_cb_desc* descs, size_t njobs) {
    const int n = (int)njobs;
    size_t tmp = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                              (const uint32_t*)nullptr, (uint32_t*)nullptr, n, 0, 32, st);
    const size_t words = 4 * njobs + 64;
    uint32_t* w = (uint32_t*)j2k_scratch(ctx, SCR_DECORD, words * 4 + tmp + 64);
    if (!w) return nullptr;
    uint32_t *keys_in = w, *keys_out = w + njobs, *ids_in = w + 2 * njobs, *ids_out = w + 3 * njobs;
    void* temp = w + words;
    t1d_order_keys<<<(unsigned)((njobs + 255) / 256), 256, 0, st>>>(descs, n, keys_in, ids_in);
    if (j2k_cuda_check(ctx, cudaGetLastError(), "decode order keys") != J2K_OK) return nullptr;
    if (j2k_cuda_check(ctx, cub::DeviceRadixSort::SortPairsDescending(temp, tmp, keys_in, keys_out, ids_in, ids_out,
                                                                      n, 0, 32, st),
                       "decode order sort") != J2K_OK)
        return nullptr;
    return ids_out;
}

template <int L>
static j2k_status launch_steps(j2k_ctx* ctx, cudaStream_t st, const j2k_cb_desc* descs,
                               const uint8_t* bytes, const j2k_cb_job* d_jobs, size_t njobs, int32_t* coeff) {
    constexpr size_t smem = lanes_smem_bytes<L>();
    const unsigned grid = (unsigned)((njobs + L * cta_warps<L>() - 1) / (L * cta_warps<L>()));
    static std::atomic<uint64_t> attr_set{0};
    const uint64_t bit = 1ull << (ctx->device & 63);
    if (!(attr_set.load() & bit)) {
        J2K_CUDA(ctx, cudaFuncSetAttribute(t1_decode_steps_kernel<L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem));
        attr_set.fetch_or(bit);
    }
    t1_decode_steps_kernel<L><<<grid, 32 * cta_warps<L>(), smem, st>>>(descs, bytes, d_jobs, (int)njobs, coeff,
                                                                            ctx->d_err);
    J2K_CUDA(ctx, cudaGetLastError());
    return J2K_OK;
}

j2k_status j2k_t1_decode_jobs(j2k_ctx* ctx, const j2k_cb_desc* descs, const uint8_t* bytes,
                              const j2k_cb_job* d_jobs, size_t njobs, int32_t* coeff,
                              cudaStream_t st, int style, const uint32_t* pass_ends, const uint8_t* job_style) {
    if (njobs == 0) return J2K_OK;
    if ((style || job_style) && !pass_ends)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "a styled decode needs the pass ends");
    const bool styled = style || job_style;
    const int L = ctx->t1d_lanes;
    if (L == 0) {  // one warp per block, lane 0 decoding
        const unsigned g = (unsigned)((njobs + kWarps - 1) / kWarps);
        if (styled)
            t1_decode_kernel<true><<<g, kWarps * 32, 0, st>>>(descs, bytes, d_jobs, (int)njobs, coeff, ctx->d_err,
                                                              style, pass_ends, job_style);
        else
            t1_decode_kernel<false><<<g, kWarps * 32, 0, st>>>(descs, bytes, d_jobs, (int)njobs, coeff, ctx->d_err,
                                                               0, nullptr, nullptr);
        J2K_CUDA(ctx, cudaGetLastError());
        return J2K_OK;
    }
    if (!styled && ctx->t1d_steps) {
        switch (L) {
        case 8: return launch_steps<8>(ctx, st, descs, bytes, d_jobs, njobs, coeff);
        case 16: return launch_steps<16>(ctx, st, descs, bytes, d_jobs, njobs, coeff);
        case 32: return launch_steps<32>(ctx, st, descs, bytes, d_jobs, njobs, coeff);
        default: break;
        }
    }
    const uint32_t* ord = nullptr;
    if (ctx->t1d_order && njobs > (size_t)L) {
        ord = decode_order(ctx, st, descs, njobs);
        if (!ord) return J2K_ERR_OUT_OF_MEMORY;
    }
    switch ((styled ? 100 : 0) + L) {
    case 2: return launch_lanes<false, 2>(ctx, st, descs, bytes, d_jobs, njobs, coeff, 0, nullptr, nullptr, ord);
    case 3: return launch_lanes<false, 3>(ctx, st, descs, bytes, d_jobs, njobs, coeff, 0, nullptr, nullptr, ord);
    case 4: return launch_lanes<false, 4>(ctx, st, descs, bytes, d_jobs, njobs, coeff, 0, nullptr, nullptr, ord);
    case 6: return launch_lanes<false, 6>(ctx, st, descs, bytes, d_jobs, njobs, coeff, 0, nullptr, nullptr, ord);
    case 8: return launch_lanes<false, 8>(ctx, st, descs, bytes, d_jobs, njobs, coeff, 0, nullptr, nullptr, ord);
    case 16: return launch_lanes<false, 16>(ctx, st, descs, bytes, d_jobs, njobs, coeff, 0, nullptr, nullptr, ord);
    case 32: return launch_lanes<false, 32>(ctx, st, descs, bytes, d_jobs, njobs, coeff, 0, nullptr, nullptr, ord);
    case 102: return launch_lanes<true, 2>(ctx, st, descs, bytes, d_jobs, njobs, coeff, style, pass_ends, job_style, ord);
    case 103: return launch_lanes<true, 3>(ctx, st, descs, bytes, d_jobs, njobs, coeff, style, pass_ends, job_style, ord);
    case 106: return launch_lanes<true, 6>(ctx, st, descs, bytes, d_jobs, njobs, coeff, style, pass_ends, job_style, ord);
    case 104: return launch_lanes<true, 4>(ctx, st, descs, bytes, d_jobs, njobs, coeff, style, pass_ends, job_style, ord);
    case 108: return launch_lanes<true, 8>(ctx, st, descs, bytes, d_jobs, njobs, coeff, style, pass_ends, job_style, ord);
    case 116: return launch_lanes<true, 16>(ctx, st, descs, bytes, d_jobs, njobs, coeff, style, pass_ends, job_style, ord);
    case 132: return launch_lanes<true, 32>(ctx, st, descs, bytes, d_jobs, njobs, coeff, style, pass_ends, job_style, ord);
    default: return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "tier-1 decoder: blocks per warp must be 0, 2, 3, 4, 6, 8, 16 or 32");
    }
}
