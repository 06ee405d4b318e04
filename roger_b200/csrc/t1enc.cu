// EBCOT tier-1 encoder: context modelling (warp per code-block) + MQ coding (lane per block).
//
// Reference: src/CL/oclbpc.cl:279-746 via src/OCLBPC.cpp:38-50.  The reference kernel computes
// the MSB plane and sigma/neighbourhood state only (its coding actions are empty comments,
// oclbpc.cl:388-443,625-740); the passes, scan order and state variables it documents
// (oclbpc.cl:19-111) are completed here from ITU-T T.800 Annex D (contexts, run-length mode,
// sign coding) and Annex C (MQ coder).
//
// Phase A — one warp per code-block.  Every row of the block is a 64-bit mask (bit x =
// column x) for significance, visited-in-SPP, refined and sign; magnitude bit-planes are sliced
// into masks with __ballot_sync.  Per stripe (4 rows) and pass:
//   * significance propagation membership is the causal fixpoint of
//       N(c,j) = M(c,j) & (E(c,j) | N(c-1,j-1) | N(c-1,j) | N(c-1,j+1) | N(c,j-1)),
//     solved with a carry-propagate run fill along each row (M & (~(M+S) | S)) iterated over
//     the 4 rows; all lanes compute it redundantly (uniform, no divergence);
//   * once the newly significant set is known every context is a function of masks, so lane l
//     forms the ZC/SC/MR/RL labels for stripe columns 2l and 2l+1 in parallel, and a warp
//     prefix sum places the symbols in scan order.
// The output is the exact (context, decision) sequence of the serial coder, one byte per
// symbol (label in bits 0-4, decision in bit 7; sign symbols also carry their context's XOR
// bit in bit 5, so that a raw-coded pass can recover the sign itself).
//
// Phase B — one lane per code-block runs the MQ encoder over its symbol stream (T.800 C.2,
// FLUSH of C.2.9, trailing 0xFF dropped); codeword bytes are written as aligned 32-bit words.
#include <cub/cub.cuh>

#include <algorithm>

#include "j2k_internal.cuh"

namespace {

constexpr int kWarpsPerCta = 8;
constexpr int kRows = 64;
constexpr int kPlaneWords = 32 * kRows;  // per-block bit-plane scratch: 64 rows x 32 planes

struct WarpSmem {
    uint64_t sig[kRows + 2], vis[kRows + 2], ref[kRows + 2], neg[kRows + 2];  // index r+1
    uint64_t bits[kRows];                                                      // current plane
};

// T.800 Table D.1 zero-coding label from (h, v, d) counts
__device__ __forceinline__ int zc_label_calc(int orient, int h, int v, int d) {
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

// (label | xor<<7) of T.800 Tables D.2/D.3 from the horizontal / vertical contributions
__device__ __forceinline__ int sc_code(int hc, int vc) {
    hc = max(-1, min(1, hc));
    vc = max(-1, min(1, vc));
    int x = 0;
    if (hc < 0 || (hc == 0 && vc < 0)) { hc = -hc; vc = -vc; x = 1; }
    int lab = hc == 0 ? (vc ? 10 : 9) : 12 + vc;
    return lab | (x << 7);
}

template <typename T>
__device__ __forceinline__ T dil(T m) { return m | (T)(m << 1) | (T)(m >> 1); }

// 4-bit window of a row mask around this lane's column pair: bit 0 = column c0-1 ...
// bit 3 = column c0+2 (columns outside 0..63 read as 0)
template <typename T>
__device__ __forceinline__ uint32_t win4(T m, int c0) {
    return (uint32_t)(c0 ? (m >> (c0 - 1)) : (T)(m << 1)) & 0xF;
}

// the lane's own columns c0 and c0+1 of a row mask (bit 0 = column c0; columns past the mask
// read as 0): bits 1-2 of win4 without its left-edge case
template <typename T>
__device__ __forceinline__ uint32_t own2(T m, int c0) {
    return (uint32_t)(m >> c0) & 3u;
}

// warp exclusive prefix sum; returns the total in *tot
__device__ __forceinline__ int warp_excl(int v, int lane, int* tot) {
    int inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    *tot = __shfl_sync(0xffffffffu, inc, 31);
    return inc - v;
}

// Context/decision emission for one coded sample: ZC (or SC) from 3-bit neighbour windows.
// zlut: 256-entry zero-coding table of this orientation indexed by the 8 neighbour bits
// (W E N S NW NE SW SE); slut: sign table indexed by (sig W E N S) | (neg W E N S) << 4.
struct Lut {
    const uint8_t* z;
    const uint8_t* s;
};

// One code-block's phase A (bit-plane slicing, the three passes per plane, symbol emission).  MT is
// the row-mask type and CPL the columns per lane: 64-bit masks and two columns per lane for blocks
// wider than 32, 32-bit masks and one column per lane otherwise (all 32 lanes busy, half the mask
// work per stripe).
template <typename MT, int CPL>
__device__ __forceinline__ void phase_a_block(WarpSmem& S, const j2k_cb_job& J, int jid, int lane,
                                              const int32_t* __restrict__ coeff, const uint8_t* zlut,
                                              const uint8_t* slut, uint8_t* __restrict__ syms,
                                              uint32_t* __restrict__ nsyms, uint32_t* __restrict__ pass_end,
                                              uint64_t* __restrict__ planes, j2k_cb_desc* __restrict__ descs,
                                              uint32_t* __restrict__ err, int pad) {
    const int cw = J.cw, ch = J.ch;
    const size_t pitch = J.pitch;
    const int32_t* blk = coeff + J.off;
    const uint8_t* zl = zlut + J.orient * 256;
    const MT colmask = (MT)(cw >= 64 ? ~0ull : ((1ull << cw) - 1));

    // ---- bit-plane slicing: lane p ends up holding plane p of each row and stores it
    uint32_t mor = 0;
    for (int r = 0; r < ch; ++r) {
        int32_t v0 = (lane < cw) ? blk[(size_t)r * pitch + lane] : 0;
        int32_t v1 = (lane + 32 < cw) ? blk[(size_t)r * pitch + lane + 32] : 0;
        uint32_t m0 = v0 < 0 ? (uint32_t)(-(int64_t)v0) : (uint32_t)v0;
        uint32_t m1 = v1 < 0 ? (uint32_t)(-(int64_t)v1) : (uint32_t)v1;
        mor |= m0 | m1;
        uint64_t ng = (uint64_t)__ballot_sync(0xffffffffu, v0 < 0) |
                      ((uint64_t)__ballot_sync(0xffffffffu, v1 < 0) << 32);
        uint32_t any = __reduce_or_sync(0xffffffffu, m0 | m1);
        uint64_t mine = 0;
        for (int p = 0; p < 32 && (any >> p); ++p) {
            uint64_t pm = (uint64_t)__ballot_sync(0xffffffffu, (m0 >> p) & 1) |
                          ((uint64_t)__ballot_sync(0xffffffffu, (m1 >> p) & 1) << 32);
            if (lane == p) mine = pm;
        }
        planes[r * 32 + lane] = mine;  // row-major [row][plane]: one coalesced 256-byte store
        if (lane == 0) S.neg[r + 1] = ng;
    }
    mor = __reduce_or_sync(0xffffffffu, mor);
    const int numbps = mor ? 32 - __clz(mor) : 0;
    for (int r = lane; r < kRows + 2; r += 32) {
        S.sig[r] = 0;
        S.vis[r] = 0;
        S.ref[r] = 0;
        if (r == 0 || r > ch) S.neg[r] = 0;
    }
    j2k_cb_desc d;
    d.offset = (uint32_t)J.out_off;
    d.length = 0;
    d.numbps = (uint8_t)numbps;
    d.npasses = (uint8_t)(numbps ? 3 * numbps - 2 : 0);
    d.orient = J.orient;
    d.band = J.band;
    d.x0 = J.px0;
    d.y0 = J.py0;
    d.cw = J.cw;
    d.ch = J.ch;
    d.comp = J.comp;
    d.reserved = 0;
    if (numbps > 31) {
        if (lane == 0) {
            atomicCAS(err, 0u, (uint32_t)J2K_DEVERR_PLANES);
            nsyms[jid] = 0;
            descs[jid] = d;
        }
        __syncwarp();
        return;
    }
    __syncwarp();
    uint8_t* out = syms + J.sym_off;
    uint32_t* pend = pass_end + (size_t)jid * 92;
    const int cap = (int)J.sym_cap;
    int pos = 0, npass = 0;
    bool ovf = false;
    const int nstripes = (ch + 3) >> 2;
    const int c0 = CPL * lane;
    const bool active = c0 < cw;
    // columns of this lane present: c0 (and c0+1 with two columns per lane)
    const uint32_t ownmask = active ? (CPL == 2 && c0 + 1 < cw ? 3u : 1u) : 0u;

    for (int p = numbps - 1; p >= 0 && !ovf; --p) {
        // current plane into shared (rows beyond ch are zero)
        S.bits[lane] = lane < ch ? planes[lane * 32 + p] : 0;
        S.bits[lane + 32] = lane + 32 < ch ? planes[(lane + 32) * 32 + p] : 0;
        __syncwarp();
        if (p != numbps - 1) {
            // ------------------------- significance propagation pass
            for (int s = 0; s < nstripes && !ovf; ++s) {
                const int r0 = 4 * s;
                MT O[6], N[6], C[4], M[4], E[4], K[4], B[4];
#pragma unroll
                for (int j = 0; j < 6; ++j) O[j] = S.sig[r0 + j];
                bool anyk = false;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const MT V = (r0 + j < ch) ? colmask : (MT)0;
                    C[j] = ~O[j + 1] & V;
                    E[j] = C[j] & dil((MT)(O[j] | O[j + 1] | O[j + 2]));  // dilation distributes over OR
                    anyk |= E[j] != 0;
                }
                if (!anyk) continue;  // no candidate has a significant neighbour: nothing coded
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    B[j] = S.bits[(r0 + j) & 63];
                    M[j] = C[j] & B[j];
                }
                N[0] = N[5] = 0;
                N[1] = N[2] = N[3] = N[4] = 0;
                if ((M[0] | M[1] | M[2] | M[3]) != 0) {  // else no sample becomes significant
                    // Sweeps top to bottom (each row from the row above as just computed); a row's
                    // fill is stable unless the row below, computed after it, seeds one of its
                    // samples outside the runs already filled (row 3's lower neighbour is the next
                    // stripe, not yet coded: always zero).  The fixpoint is the least one either way.
                    do {
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            MT seeds = M[j] & (E[j] | ((N[j] | N[j + 2]) << 1) | N[j]);
                            N[j + 1] = M[j] & (MT)(~(MT)(M[j] + seeds) | seeds);
                        }
                    } while (((M[0] & (MT)(N[2] << 1) & ~N[1]) | (M[1] & (MT)(N[3] << 1) & ~N[2]) |
                              (M[2] & (MT)(N[4] << 1) & ~N[3])) != 0);
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) K[j] = C[j] & (E[j] | ((N[j] | N[j + 1] | N[j + 2]) << 1) | N[j]);
                // per-lane windows
                uint32_t a[6], o[6], ng[6], kk = 0, bb = 0;
#pragma unroll
                for (int j = 0; j < 6; ++j) {
                    o[j] = win4(O[j], c0);
                    a[j] = win4(O[j] | N[j], c0);
                    ng[j] = win4(S.neg[r0 + j], c0);
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    kk |= (own2(K[j], c0) & ownmask) << (2 * j);
                    bb |= own2(B[j], c0) << (2 * j);
                }
                // the newly significant samples are the coded ones whose bit is 1 (N = K & B)
                const uint32_t nn4 = kk & bb;
                int cnt = __popc(kk) + __popc(nn4);
                int tot;
                int off = pos + warp_excl(cnt, lane, &tot);
                if (pos + tot > cap) {
                    ovf = true;
                    break;
                }
                if (cnt) {
#pragma unroll
                    for (int k = 0; k < CPL; ++k)
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const int bitpos = 2 * j + k;
                            if (!((kk >> bitpos) & 1)) continue;
                            const uint32_t up = ((a[j] >> k) & 3) | ((o[j] >> k) & 4);
                            const uint32_t md = ((a[j + 1] >> k) & 1) | ((o[j + 1] >> k) & 4);
                            const uint32_t dn = ((a[j + 2] >> k) & 1) | ((o[j + 2] >> k) & 6);
                            // index: W E N S NW NE SW SE
                            const uint32_t zi = (md & 1) | ((md >> 1) & 2) | ((up & 2) << 1) | ((dn & 2) << 2) |
                                                ((up & 1) << 4) | ((up & 4) << 3) | ((dn & 1) << 6) | ((dn & 4) << 5);
                            const int bit = (bb >> bitpos) & 1;
                            out[off++] = (uint8_t)(zl[zi] | (bit << 7));
                            if (bit) {
                                const uint32_t sg4 = (zi & 15);
                                const uint32_t nw = ng[j + 1] >> k, nu = ng[j] >> k, nd = ng[j + 2] >> k;
                                const uint32_t ng4 = (nw & 1) | ((nw >> 1) & 2) | ((nu & 2) << 1) | ((nd & 2) << 2);
                                const int sc = slut[sg4 | (ng4 << 4)];
                                const int sgn = (ng[j + 1] >> (k + 1)) & 1;
                                out[off++] = (uint8_t)((sc & 31) | ((sc >> 7) << 5) | ((sgn ^ (sc >> 7)) << 7));
                            }
                        }
                }
                pos += tot;
                if (lane == 0) {
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        S.sig[r0 + j + 1] = O[j + 1] | N[j + 1];
                        S.vis[r0 + j + 1] = K[j];
                    }
                }
                __syncwarp();
            }
            if (lane == 0) pend[npass] = (uint32_t)pos;
            ++npass;
            if (pad) {  // the next pass starts on a 16-byte boundary (a coding unit of its own)
                pos = (pos + 15) & ~15;
                ovf |= pos > cap;
            }
            // ------------------------- magnitude refinement pass
            for (int s = 0; s < nstripes && !ovf; ++s) {
                const int r0 = 4 * s;
                MT SG[6], R[4];
                bool anyr = false;
#pragma unroll
                for (int j = 0; j < 6; ++j) SG[j] = S.sig[r0 + j];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    R[j] = SG[j + 1] & ~S.vis[r0 + j + 1];
                    anyr |= R[j] != 0;
                }
                if (!anyr) continue;
                uint32_t rr = 0, rf = 0, nb = 0, bb = 0;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const MT nbm = dil((MT)(SG[j] | SG[j + 2])) | (MT)(SG[j + 1] << 1) | (MT)(SG[j + 1] >> 1);
                    rr |= (own2(R[j], c0) & ownmask) << (2 * j);
                    rf |= own2(S.ref[r0 + j + 1], c0) << (2 * j);
                    nb |= own2(nbm, c0) << (2 * j);
                    bb |= own2(S.bits[(r0 + j) & 63], c0) << (2 * j);
                }
                const int cnt = __popc(rr);
                int tot;
                int off = pos + warp_excl(cnt, lane, &tot);
                if (pos + tot > cap) {
                    ovf = true;
                    break;
                }
                if (cnt) {
#pragma unroll
                    for (int k = 0; k < CPL; ++k)
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const int bitpos = 2 * j + k;
                            if (!((rr >> bitpos) & 1)) continue;
                            const int lab = ((rf >> bitpos) & 1) ? 16 : (((nb >> bitpos) & 1) ? 15 : 14);
                            out[off++] = (uint8_t)(lab | (((bb >> bitpos) & 1) << 7));
                        }
                }
                pos += tot;
                if (lane == 0) {
#pragma unroll
                    for (int j = 0; j < 4; ++j) S.ref[r0 + j + 1] |= R[j];
                }
                __syncwarp();
            }
            if (lane == 0) pend[npass] = (uint32_t)pos;
            ++npass;
            if (pad) {  // the next pass starts on a 16-byte boundary (a coding unit of its own)
                pos = (pos + 15) & ~15;
                ovf |= pos > cap;
            }
        }
        // ------------------------- cleanup pass
        for (int s = 0; s < nstripes && !ovf; ++s) {
            const int r0 = 4 * s;
            const bool full = r0 + 3 < ch;
            MT O[6], C[4], N[4];
            bool anyc = false;
#pragma unroll
            for (int j = 0; j < 6; ++j) O[j] = S.sig[r0 + j];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const MT V = (r0 + j < ch) ? colmask : (MT)0;
                C[j] = V & ~O[j + 1] & ~S.vis[r0 + j + 1];
                N[j] = C[j] & S.bits[(r0 + j) & 63];
                anyc |= C[j] != 0;
            }
            if (!anyc) continue;
            uint32_t a[6], o[6], ng[6], cc = 0, nn4 = 0;
#pragma unroll
            for (int j = 0; j < 6; ++j) {
                o[j] = win4(O[j], c0);
                a[j] = win4((j >= 1 && j <= 4) ? (O[j] | N[j - 1]) : O[j], c0);
                ng[j] = win4(S.neg[r0 + j], c0);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                cc |= (own2(C[j], c0) & ownmask) << (2 * j);
                nn4 |= (own2(N[j], c0) & ownmask) << (2 * j);
            }
            // per column: run-length mode?  (full stripe, 4 candidates, no significant neighbour)
            uint32_t rlmask = 0;  // bit k: column c0+k codes in run-length mode
            int cnt = 0;
#pragma unroll
            for (int k = 0; k < CPL; ++k) {
                const uint32_t colc = (cc >> k) & 0x55;  // bits 0,2,4,6: rows 0..3
                const uint32_t coln = (nn4 >> k) & 0x55;
                bool rl = false;
                if (full && colc == 0x55) {
                    uint32_t q = 0;
#pragma unroll
                    for (int j = 1; j <= 4; ++j) q |= ((a[j] >> k) & 1) | ((o[j] >> k) & 4);
                    q |= ((o[0] >> k) & 7) | ((o[5] >> k) & 7);
                    rl = q == 0;
                }
                if (rl) {
                    rlmask |= 1u << k;
                    if (coln) {
                        const int first = (__ffs(coln) - 1) >> 1;  // row of the first 1
                        int rest = 0;
                        for (int j = first + 1; j < 4; ++j) rest += 1 + ((coln >> (2 * j)) & 1);
                        cnt += 1 + 2 + 1 + rest;
                    } else {
                        cnt += 1;
                    }
                } else {
                    cnt += __popc(colc) + __popc(coln);
                }
            }
            int tot;
            int off = pos + warp_excl(cnt, lane, &tot);
            if (pos + tot > cap) {
                ovf = true;
                break;
            }
            if (cnt) {
#pragma unroll
                for (int k = 0; k < CPL; ++k) {
                    const uint32_t colc = (cc >> k) & 0x55;
                    const uint32_t coln = (nn4 >> k) & 0x55;
                    if (!colc) continue;
                    int jstart = 0;
                    if ((rlmask >> k) & 1) {
                        out[off++] = (uint8_t)(17 | ((coln != 0) << 7));
                        if (!coln) continue;
                        const int first = (__ffs(coln) - 1) >> 1;
                        out[off++] = (uint8_t)(18 | (((first >> 1) & 1) << 7));
                        out[off++] = (uint8_t)(18 | ((first & 1) << 7));
                        // sign of the first significant sample: its four neighbours are insignificant
                        const int sgn = (ng[first + 1] >> (k + 1)) & 1;
                        const int sc = slut[0];
                        out[off++] = (uint8_t)((sc & 31) | ((sc >> 7) << 5) | ((sgn ^ (sc >> 7)) << 7));
                        jstart = first + 1;
                    }
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        if (j < jstart || !((colc >> (2 * j)) & 1)) continue;
                        const uint32_t up = ((a[j] >> k) & 3) | ((o[j] >> k) & 4);
                        const uint32_t md = ((a[j + 1] >> k) & 1) | ((o[j + 1] >> k) & 4);
                        const uint32_t dn = ((a[j + 2] >> k) & 1) | ((o[j + 2] >> k) & 6);
                        const uint32_t zi = (md & 1) | ((md >> 1) & 2) | ((up & 2) << 1) | ((dn & 2) << 2) |
                                            ((up & 1) << 4) | ((up & 4) << 3) | ((dn & 1) << 6) | ((dn & 4) << 5);
                        const int bit = (coln >> (2 * j)) & 1;
                        out[off++] = (uint8_t)(zl[zi] | (bit << 7));
                        if (bit) {
                            const uint32_t nw = ng[j + 1] >> k, nu = ng[j] >> k, nd = ng[j + 2] >> k;
                            const uint32_t ng4 = (nw & 1) | ((nw >> 1) & 2) | ((nu & 2) << 1) | ((nd & 2) << 2);
                            const int sc = slut[(zi & 15) | (ng4 << 4)];
                            const int sgn = (ng[j + 1] >> (k + 1)) & 1;
                            out[off++] = (uint8_t)((sc & 31) | ((sc >> 7) << 5) | ((sgn ^ (sc >> 7)) << 7));
                        }
                    }
                }
            }
            pos += tot;
            if (lane == 0) {
#pragma unroll
                for (int j = 0; j < 4; ++j) S.sig[r0 + j + 1] = O[j + 1] | N[j];
            }
            __syncwarp();
        }
        if (lane == 0) pend[npass] = (uint32_t)pos;
        ++npass;
        if (pad) {
            pos = (pos + 15) & ~15;
            ovf |= pos > cap;
        }
        for (int r = lane; r < kRows + 2; r += 32) S.vis[r] = 0;
        __syncwarp();
    }
    if (ovf) {
        if (lane == 0) atomicCAS(err, 0u, (uint32_t)J2K_DEVERR_SYM_CAPACITY);
        pos = 0;
    }
    if (lane == 0) {
        nsyms[jid] = (uint32_t)pos;
        descs[jid] = d;
    }
    __syncwarp();
}

// MINB: resident CTAs per SM the register budget is cut for (2: no spills; 3: a few spilled
// registers, more warps to hide the ALU chains)
template <int MINB>
__global__ void __launch_bounds__(kWarpsPerCta * 32, MINB)
t1_symbols_kernel(const int32_t* __restrict__ coeff, const j2k_cb_job* __restrict__ jobs,
                  int njobs, const uint32_t* __restrict__ order, uint32_t* __restrict__ queue,
                  uint8_t* __restrict__ syms, uint32_t* __restrict__ nsyms,
                  uint32_t* __restrict__ pass_end, uint64_t* __restrict__ plane_scratch,
                  j2k_cb_desc* __restrict__ descs, uint32_t* __restrict__ err, int pad) {
    __shared__ WarpSmem smem[kWarpsPerCta];
    __shared__ uint8_t zlut[4][256];
    __shared__ uint8_t slut[256];
    for (int i = threadIdx.x; i < 4 * 256; i += blockDim.x) {
        int o = i >> 8, b = i & 255;
        int W = b & 1, E = (b >> 1) & 1, N = (b >> 2) & 1, S = (b >> 3) & 1;
        int d = ((b >> 4) & 1) + ((b >> 5) & 1) + ((b >> 6) & 1) + ((b >> 7) & 1);
        zlut[o][b] = (uint8_t)zc_label_calc(o, W + E, N + S, d);
    }
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        int sg = i & 15, ng = i >> 4;
        auto ct = [&](int k) { return ((sg >> k) & 1) ? (((ng >> k) & 1) ? -1 : 1) : 0; };
        slut[i] = (uint8_t)sc_code(ct(0) + ct(1), ct(2) + ct(3));
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpSmem& S = smem[wid];
    // persistent: each warp pulls code-blocks from the device-side queue until it is empty;
    // its bit-plane scratch slot is reused from block to block
    uint64_t* planes = plane_scratch + (size_t)(blockIdx.x * kWarpsPerCta + wid) * kPlaneWords;
    for (;;) {
    int qi = 0;
    if (lane == 0) qi = (int)atomicAdd(queue, 1u);
    qi = __shfl_sync(0xffffffffu, qi, 0);
    if (qi >= njobs) break;
    const int jid = order ? (int)order[qi] : qi;
    const j2k_cb_job J = jobs[jid];
    if (J.cw == 0 || J.ch == 0 || J.cw > 64 || J.ch > 64 || J.orient > 3 || J.sym_cap % 16 != 0) {
        if (lane == 0) {
            atomicCAS(err, 0u, (uint32_t)J2K_DEVERR_BAD_JOB);
            nsyms[jid] = 0;
        }
        continue;
    }
    if (J.cw <= 32)
        phase_a_block<uint32_t, 1>(S, J, jid, lane, coeff, &zlut[0][0], slut, syms, nsyms, pass_end, planes, descs,
                                   err, pad);
    else
        phase_a_block<uint64_t, 2>(S, J, jid, lane, coeff, &zlut[0][0], slut, syms, nsyms, pass_end, planes, descs,
                                   err, pad);
    }  // queue loop
}

// ---- phase B: MQ encoder, one lane per code-block ------------------------------------------------
//
// The coder is serial per block, so the kernel time is (longest block's symbol count) x
// (latency per symbol).  Blocks are ordered longest-first (a radix sort of the symbol counts)
// so the lanes of a warp finish together and the biggest blocks start first.  Per context the
// state is one packed word in shared memory: Qe (bits 0-15), next-MPS index (16-21), next-LPS
// index (22-27), switch flag (28), MPS (31).  The MPS-without-renormalisation case, the most
// frequent, touches no memory but the state load; the next symbol's state is loaded before the
// current one finishes, and forwarded when both use the same context.

__constant__ uint16_t c_qe[47] = {
    0x5601, 0x3401, 0x1801, 0x0AC1, 0x0521, 0x0221, 0x5601, 0x5401, 0x4801, 0x3801, 0x3001, 0x2401,
    0x1C01, 0x1601, 0x5601, 0x5401, 0x5101, 0x4801, 0x3801, 0x3401, 0x3001, 0x2801, 0x2401, 0x2201,
    0x1C01, 0x1801, 0x1601, 0x1401, 0x1201, 0x1101, 0x0AC1, 0x09C1, 0x08A1, 0x0521, 0x0441, 0x02A1,
    0x0221, 0x0141, 0x0111, 0x0085, 0x0049, 0x0025, 0x0015, 0x0009, 0x0005, 0x0001, 0x5601};
__constant__ uint8_t c_nmps[47] = {1,  2,  3,  4,  5,  38, 7,  8,  9,  10, 11, 12, 13, 29, 15, 16,
                                   17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32,
                                   33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 44, 45, 45, 46};
__constant__ uint8_t c_nlps[47] = {1,  6,  9,  12, 29, 33, 6,  14, 14, 14, 17, 18, 20, 21, 14, 14,
                                   15, 16, 17, 18, 19, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29,
                                   30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 46};

constexpr int kMqThreads = 32;  // one warp per CTA: the longest blocks' warps spread one per SM

// Branch-light MQ encoder state.  The exchange and state transition are predicated so the
// lanes of a warp (each coding a different block) stay converged; only the byte output, about
// one symbol in sixteen, branches.
struct MqEnc {
    uint32_t A, C, B;   // B: pending output byte (may still receive a carry)
    int CT, bp;         // bp: index of B (-1 before the first byte)
    uint32_t* out;      // word-aligned codeword buffer
    int cap;            // bytes
    uint32_t wacc;      // completed bytes waiting for a 32-bit store
    int wn, wbase;
    bool ovf;
    __device__ __forceinline__ void push(uint32_t byte) {
        wacc |= byte << (8 * wn);
        if (++wn == 4) {
            if (wbase + 4 <= cap) out[wbase >> 2] = wacc; else ovf = true;
            wbase += 4;
            wn = 0;
            wacc = 0;
        }
    }
    // T.800 C.2 BYTEOUT in one straight-line form: a carry (C >= 2^27 after a non-0xFF byte)
    // increments the pending byte; a 0xFF byte (before or after the carry) is followed by 7 bits.
    __device__ __forceinline__ void byteout() {
        if (B != 0xFF && C >= 0x8000000u) {
            if (bp >= 0) B += 1;
            C &= 0x7FFFFFF;
        }
        const bool ff = (B == 0xFF);
        const uint32_t v = ff ? (C >> 20) : (C >> 19);
        C &= ff ? 0xFFFFFu : 0x7FFFFu;
        CT = ff ? 7 : 8;
        if (bp >= 0) push(B);
        ++bp;
        B = v & 0xFF;
    }
    // shift by sh (0..15) with at most two byte outputs
    __device__ __forceinline__ void renorm(int sh) {
        int k = min(sh, CT);
        A <<= k;
        C <<= k;
        CT -= k;
        sh -= k;
        if (CT == 0) {
            byteout();
            k = min(sh, CT);
            A <<= k;
            C <<= k;
            CT -= k;
            sh -= k;
            if (CT == 0) {
                byteout();
                A <<= sh;
                C <<= sh;
                CT -= sh;
            }
        }
    }
};

// Warp schedule of the MQ kernel: tier k has warps[k] warps of lanes[k] blocks each.
struct MqSchedule {
    int warps[4] = {0, 0, 0, 0};
    int lanes[4] = {0, 0, 0, 0};
};

// RATE: also record, for every bit-plane k, the bytes produced (bp + 1) when its cleanup pass
// ends (pass 3k; pass ends in symbols from phase A) into plane_bytes[job * 32 + k].
template <int LANES, bool RATE = false>
__global__ void __launch_bounds__(kMqThreads)
t1_mq_kernel(const uint8_t* __restrict__ syms, const j2k_cb_job* __restrict__ jobs, const uint32_t* __restrict__ nsyms,
             const uint32_t* __restrict__ order, int njobs, uint8_t* __restrict__ bytes,
              j2k_cb_desc* __restrict__ descs, uint32_t* __restrict__ err,
              const uint32_t* __restrict__ pend = nullptr, uint32_t* __restrict__ plane_bytes = nullptr,
              MqSchedule sched = MqSchedule{}) {
    __shared__ uint32_t tab[47];
    __shared__ uint32_t cst[32 * kMqThreads];  // contexts 0..18 used; 32 so that a 5-bit index needs no clamp
    for (int i = threadIdx.x; i < 47; i += blockDim.x)
        tab[i] = (uint32_t)c_qe[i] | ((uint32_t)c_nmps[i] << 16) | ((uint32_t)c_nlps[i] << 22) |
                 ((uint32_t)(i == 0 || i == 6 || i == 14) << 28);
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    // warp w takes blocks in longest-first order: the schedule's tiers first (warps with fewer
    // blocks each), then LANES blocks per warp
    const int w = blockIdx.x * (kMqThreads / 32) + wid;
    int gid = -1, wbase = 0, gbase = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (gid < 0 && w < wbase + sched.warps[k]) {
            if (lane >= sched.lanes[k]) return;
            gid = gbase + (w - wbase) * sched.lanes[k] + lane;
        }
        wbase += sched.warps[k];
        gbase += sched.warps[k] * sched.lanes[k];
    }
    if (gid < 0) {
        if (lane >= LANES) return;
        gid = gbase + (w - wbase) * LANES + lane;
    }
    if (gid >= njobs) return;
    const int jid = order ? (int)order[gid] : gid;
    const int t = threadIdx.x;
    uint32_t* st = cst + t;  // context k at st[k * kMqThreads]
    for (int k = 0; k < 32; ++k) st[k * kMqThreads] = tab[0];
    st[0] = tab[4];
    st[17 * kMqThreads] = tab[3];
    st[18 * kMqThreads] = tab[46];
    const j2k_cb_job J = jobs[jid];
    const size_t sym_cap = J.sym_cap, cap_per_block = J.out_cap;
    const int n = (int)min((size_t)nsyms[jid], sym_cap);
    MqEnc e;
    e.A = 0x8000;
    e.C = 0;
    e.B = 0;
    e.CT = 12;
    e.bp = -1;
    e.out = reinterpret_cast<uint32_t*>(bytes + J.out_off);
    e.cap = (int)cap_per_block;
    e.wacc = 0;
    e.wn = 0;
    e.wbase = 0;
    e.ovf = false;
    // Symbols stream in 16-byte chunks with two chunks in flight per lane; the next symbol's
    // context state is loaded one step ahead and forwarded when the current symbol updates it.
    const uint4* sp4 = reinterpret_cast<const uint4*>(syms + J.sym_off);
    const int nchunks = (n + 15) >> 4;
    const uint4 z4 = make_uint4(0, 0, 0, 0);
    uint4 c0 = nchunks > 0 ? __ldcs(sp4) : z4;
    uint4 c1 = nchunks > 1 ? __ldcs(sp4 + 1) : z4;
    int cx = (int)(c0.x & 31);
    uint32_t ent = st[cx * kMqThreads];
    // RATE bookkeeping: next cleanup pass (3 * kp) and the symbol count at which it ends
    int kp = 0, npass = 0;
    uint32_t next_end = 0xFFFFFFFFu;
    const uint32_t* pe = nullptr;
    if (RATE) {
        npass = descs[jid].npasses;
        pe = pend + (size_t)jid * 92;
        next_end = npass > 0 ? pe[0] : 0xFFFFFFFFu;
        while (next_end == 0u) {  // passes with no symbols at all
            plane_bytes[(size_t)jid * 32 + kp] = (uint32_t)(e.bp + 1);
            ++kp;
            next_end = 3 * kp < npass ? pe[3 * kp] : 0xFFFFFFFFu;
        }
    }
    // one symbol: d (bit 7) coded in context cx; the next symbol's context state is loaded now
    // and forwarded if this symbol updates the same context
    auto step = [&](uint32_t sym, uint32_t nsym, bool hit, uint32_t done) {
        const int d = sym >> 7;
        const int ncx = (int)(nsym & 31);
        uint32_t nent = st[ncx * kMqThreads];
        const uint32_t qe = ent & 0xFFFF;
        const int mps = ent >> 31;
        const bool is_mps = d == mps;
        const uint32_t a1 = e.A - qe;
        const bool fast = is_mps && (a1 & 0x8000);
        const bool addc = fast || (is_mps != (a1 < qe));
        e.C += addc ? qe : 0u;
        e.A = addc ? a1 : qe;
        // state transition (not taken on the fast path)
        const int nidx = is_mps ? (ent >> 16) & 63 : (ent >> 22) & 63;
        const uint32_t nmps = (uint32_t)(mps ^ (!is_mps & (int)((ent >> 28) & 1)));
        const uint32_t upd = tab[nidx] | (nmps << 31);
        if (!fast) {
            st[cx * kMqThreads] = upd;
            if (ncx == cx) nent = upd;
        }
        e.renorm(__clz(e.A) - 16);
        cx = ncx;
        ent = nent;
        if (RATE && hit) {
            while (done == next_end) {
                if (kp < 32) plane_bytes[(size_t)jid * 32 + kp] = (uint32_t)(e.bp + 1);
                ++kp;
                next_end = 3 * kp < npass ? pe[3 * kp] : 0xFFFFFFFFu;
            }
        }
    };
    // 4 symbols per unrolled body over a rotating word (a 16-symbol body made the lone-block
    // warps stall on instruction fetch)
    for (int k = 0; k < nchunks; ++k) {
        const uint4 cur = c0;
        c0 = c1;
        c1 = (k + 2 < nchunks) ? __ldcs(sp4 + k + 2) : z4;
        const int m = min(16, n - 16 * k);
        uint32_t wa = cur.x, wb = cur.y, wc = cur.z, wd = cur.w;
        const uint32_t we = c0.x;
#pragma unroll 1
        for (int q = 0; q < 4 && 4 * q < m; ++q) {
            // RATE: only a group that holds a bit-plane end checks symbol by symbol
            const bool hit = RATE && next_end <= (uint32_t)(16 * k + 4 * q + 4);
            const uint32_t base = (uint32_t)(16 * k + 4 * q);
            if (4 * q + 4 <= m) {  // a full group: no per-symbol bound
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    step((wa >> (8 * j)) & 0xFF, j < 3 ? (wa >> (8 * (j + 1))) & 0xFF : wb & 0xFF, hit, base + j + 1);
            } else {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (4 * q + j < m)
                        step((wa >> (8 * j)) & 0xFF, j < 3 ? (wa >> (8 * (j + 1))) & 0xFF : wb & 0xFF, hit,
                             base + j + 1);
            }
            wa = wb;
            wb = wc;
            wc = wd;
            wd = we;
        }
    }
    int len = 0;
    if (n > 0) {
        uint32_t tempc = e.C + e.A;
        e.C |= 0xFFFF;
        if (e.C >= tempc) e.C -= 0x8000;
        e.C <<= e.CT;
        e.byteout();
        e.C <<= e.CT;
        e.byteout();
        len = e.bp + 1;
        if (e.B == 0xFF) len--;
        e.push(e.B);
        uint8_t* bb = bytes + J.out_off;
        for (int k = 0; k < e.wn; ++k) {
            if (e.wbase + k < e.cap) bb[e.wbase + k] = (uint8_t)(e.wacc >> (8 * k));
            else e.ovf = true;
        }
    }
    if (e.ovf || len > (int)cap_per_block) {
        atomicCAS(err, 0u, (uint32_t)J2K_DEVERR_OUT_CAPACITY);
        len = 0;
    }
    descs[jid].length = len;
}

// ---- decoupled MQ coder: probability-state warp + code-register warp ---------------------------
//
// The MQ recurrences split cleanly: the interval register A and the 19 context states never
// read the code register C, and C (with its byte output) only needs, per symbol, the value
// Qe, whether Qe is added to C, and the renormalisation shift.  Warp 0 of each CTA runs the
// A/state recurrence for 32 blocks (one per lane, branch-free) and writes one packed entry
// per symbol (Qe | add<<16 | shift<<17) into a double-buffered shared ring; warp 1 runs the C
// recurrence and the T.800 C.2 byte output one 32-symbol chunk behind.  Each warp carries
// half of the serial chain and the two halves overlap.
constexpr int kPairChunk = 32;

__global__ void __launch_bounds__(64)
t1_mq_pair_kernel(const uint8_t* __restrict__ syms, const j2k_cb_job* __restrict__ jobs, const uint32_t* __restrict__ nsyms,
                  const uint32_t* __restrict__ order, int njobs, uint8_t* __restrict__ bytes,
                   j2k_cb_desc* __restrict__ descs, uint32_t* __restrict__ err) {
    __shared__ uint32_t tab[47];
    __shared__ uint32_t cst[20 * 32];
    __shared__ uint32_t ring[2][kPairChunk][32];
    __shared__ uint32_t finalA[32];
    for (int i = threadIdx.x; i < 47; i += blockDim.x)
        tab[i] = (uint32_t)c_qe[i] | ((uint32_t)c_nmps[i] << 16) | ((uint32_t)c_nlps[i] << 22) |
                 ((uint32_t)(i == 0 || i == 6 || i == 14) << 28);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gid = blockIdx.x * 32 + lane;
    const bool live = gid < njobs;
    const int jid = live ? (order ? (int)order[gid] : gid) : 0;
    const j2k_cb_job J = jobs[jid];
    const size_t sym_cap = J.sym_cap, cap_per_block = J.out_cap;
    const int n = live ? (int)min((size_t)nsyms[jid], sym_cap) : 0;
    int nmax = n;
#pragma unroll
    for (int o = 16; o; o >>= 1) nmax = max(nmax, __shfl_xor_sync(0xffffffffu, nmax, o));
    const int nchunks = (nmax + kPairChunk - 1) / kPairChunk;
    if (warp == 0) {
        // ------------------------------------------------ probability-state warp
        uint32_t* st = cst + lane;  // context k at st[32*k]
        for (int k = 0; k < 19; ++k) st[32 * k] = tab[0];
        st[0] = tab[4];
        st[32 * 17] = tab[3];
        st[32 * 18] = tab[46];
        uint32_t A = 0x8000;
        const uint4* sp4 = reinterpret_cast<const uint4*>(syms + J.sym_off);
        const int nq = (n + 15) >> 4;  // 16-symbol chunks of this lane
        const uint4 z4 = make_uint4(0, 0, 0, 0);
        uint4 q0 = nq > 0 ? __ldcs(sp4) : z4, q1 = nq > 1 ? __ldcs(sp4 + 1) : z4;
        uint4 q2 = nq > 2 ? __ldcs(sp4 + 2) : z4, q3 = nq > 3 ? __ldcs(sp4 + 3) : z4;
        int cx = min((int)(q0.x & 31), 18);
        uint32_t ent = st[32 * cx];
        for (int k = 0; k <= nchunks; ++k) {
            if (k < nchunks) {
                const uint32_t w[9] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w, q2.x};
                const int base = k * kPairChunk;
                uint32_t* rb = &ring[k & 1][0][lane];
#pragma unroll
                for (int j = 0; j < kPairChunk; ++j) {
                    const bool valid = base + j < n;
                    const uint32_t sym = (w[j >> 2] >> (8 * (j & 3))) & 0xFF;
                    const uint32_t nsym = (w[(j + 1) >> 2] >> (8 * ((j + 1) & 3))) & 0xFF;
                    const int ncx = min((int)(nsym & 31), 18);
                    uint32_t nent = st[32 * ncx];
                    const uint32_t qe = valid ? (ent & 0xFFFF) : 0u;
                    const int mps = ent >> 31;
                    const bool is_mps = !valid || ((int)(sym >> 7) == mps);
                    const uint32_t a1 = A - qe;
                    const bool fast = is_mps && (a1 & 0x8000);
                    const bool addc = fast || (is_mps != (a1 < qe));
                    const uint32_t a2 = addc ? a1 : qe;
                    const int sh = __clz(a2) - 16;
                    A = a2 << sh;
                    const int nidx = is_mps ? (ent >> 16) & 63 : (ent >> 22) & 63;
                    const uint32_t nmps = (uint32_t)(mps ^ (!is_mps & (int)((ent >> 28) & 1)));
                    const uint32_t upd = tab[nidx] | (nmps << 31);
                    if (!fast) {
                        st[32 * cx] = upd;
                        if (ncx == cx) nent = upd;
                    }
                    rb[32 * j] = qe | ((uint32_t)addc << 16) | ((uint32_t)sh << 17);
                    cx = ncx;
                    ent = nent;
                }
                // advance the symbol window by two 16-symbol chunks, keeping two in flight
                const int nextq = 2 * (k + 1);
                q0 = q2;
                q1 = q3;
                q2 = nextq + 2 < nq ? __ldcs(sp4 + nextq + 2) : z4;
                q3 = nextq + 3 < nq ? __ldcs(sp4 + nextq + 3) : z4;
            } else {
                finalA[lane] = A;
            }
            __syncthreads();
        }
    } else {
        // ------------------------------------------------ code-register warp
        MqEnc e;
        e.A = 0;
        e.C = 0;
        e.B = 0;
        e.CT = 12;
        e.bp = -1;
        e.out = reinterpret_cast<uint32_t*>(bytes + J.out_off);
        e.cap = (int)cap_per_block;
        e.wacc = 0;
        e.wn = 0;
        e.wbase = 0;
        e.ovf = false;
        for (int k = 0; k <= nchunks; ++k) {
            if (k > 0) {
                const uint32_t* rb = &ring[(k - 1) & 1][0][lane];
#pragma unroll 8
                for (int j = 0; j < kPairChunk; ++j) {
                    const uint32_t en = rb[32 * j];
                    e.C += (en & 0xFFFF) & (0u - ((en >> 16) & 1));
                    int sh = (int)(en >> 17);
                    if (sh < e.CT) {
                        e.C <<= sh;
                        e.CT -= sh;
                    } else {
                        while (sh > 0) {
                            const int kk = min(sh, e.CT);
                            e.C <<= kk;
                            e.CT -= kk;
                            sh -= kk;
                            if (e.CT == 0) e.byteout();
                        }
                    }
                }
            }
            __syncthreads();
        }
        if (!live) return;
        int len = 0;
        if (n > 0) {
            e.A = finalA[lane];
            uint32_t tempc = e.C + e.A;
            e.C |= 0xFFFF;
            if (e.C >= tempc) e.C -= 0x8000;
            e.C <<= e.CT;
            e.byteout();
            e.C <<= e.CT;
            e.byteout();
            len = e.bp + 1;
            if (e.B == 0xFF) len--;
            e.push(e.B);
            uint8_t* bb = bytes + J.out_off;
            for (int k = 0; k < e.wn; ++k) {
                if (e.wbase + k < e.cap) bb[e.wbase + k] = (uint8_t)(e.wacc >> (8 * k));
                else e.ovf = true;
            }
        }
        if (e.ovf || len > (int)cap_per_block) {
            atomicCAS(err, 0u, (uint32_t)J2K_DEVERR_OUT_CAPACITY);
            len = 0;
        }
        descs[jid].length = len;
    }
}

// ---- code-block styles: coding units --------------------------------------------------------
//
// With a code-block style the MQ coder works on units: a run of passes coded serially by one
// lane (context states carried from pass to pass, reset where the style says so, the codeword
// terminated after the passes the style terminates, raw-coded passes written as bits).  When
// the style has both RESET and TERMALL every pass starts from fresh states and a fresh coder,
// so each pass is a unit of its own and the passes of a block code in parallel lanes; otherwise
// a block is one unit.  Unit k of job j is slot j * J2K_PASS_STRIDE + k.  A unit writes its
// segments into a slot of its own (its symbols' range of the symbol buffer, times a factor,
// plus 16 bytes per pass), and a compaction pass then puts each block's units back to back.

__host__ __device__ __forceinline__ bool units_per_pass(int style) {
    return (style & (J2K_CBLK_RESET | J2K_CBLK_TERMALL)) == (J2K_CBLK_RESET | J2K_CBLK_TERMALL);
}

// slot byte offset of the unit that starts at symbol s0 and pass p0 of job j (symbol stream of
// job j at sym_off): slots follow the symbols, so consecutive units never overlap
__device__ __forceinline__ uint64_t seg_slot(uint64_t sym_off, uint32_t s0, int j, int p0, int fac) {
    return (uint64_t)fac * ((sym_off + s0 + 3) & ~(uint64_t)3) + 16ull * ((uint64_t)j * J2K_PASS_STRIDE + p0);
}

// first symbol of pass p of a job whose pass ends are pe: with per-pass units every pass's
// symbols start on a 16-byte boundary (phase A pads them)
__device__ __forceinline__ uint32_t pass_start(const uint32_t* pe, int p, bool per_pass) {
    if (p == 0) return 0u;
    return per_pass ? (pe[p - 1] + 15u) & ~15u : pe[p - 1];
}

// sort keys: symbols of each unit + 1 (0 for slots without a unit); values: slot ids
__global__ void t1_unit_keys_kernel(const j2k_cb_desc* __restrict__ descs, const uint32_t* __restrict__ pend,
                                    int njobs, int style, uint32_t* __restrict__ keys, uint32_t* __restrict__ ids) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= njobs * J2K_PASS_STRIDE) return;
    const int j = i / J2K_PASS_STRIDE, k = i % J2K_PASS_STRIDE;
    const int np = descs[j].npasses;
    const uint32_t* pe = pend + (size_t)j * J2K_PASS_STRIDE;
    uint32_t key = 0;
    if (units_per_pass(style)) {
        // raw passes sort after the MQ ones (bit 31), so that a warp's lanes code alike passes
        if (k < np) key = (pe[k] - pass_start(pe, k, true) + 1u) | (j2k_pass_raw(style, k) ? 0u : 0x80000000u);
    } else if (k == 0 && np > 0) {
        key = pe[np - 1] + 1u;
    }
    keys[i] = key;
    ids[i] = (uint32_t)i;
}

// One lane per unit, units longest first.  ulen[slot] receives the unit's bytes; ends[j *
// stride + p] the unit-relative codeword bytes when pass p ended.
__global__ void __launch_bounds__(128)
t1_mq_units_kernel(const uint8_t* __restrict__ syms, const j2k_cb_job* __restrict__ jobs,
                   const j2k_cb_desc* __restrict__ descs, const uint32_t* __restrict__ pend,
                   const uint32_t* __restrict__ order, const uint32_t* __restrict__ keys, int nslots, int style,
                   int fac, uint8_t* __restrict__ segs, uint32_t* __restrict__ ulen, uint32_t* __restrict__ ends,
                   uint32_t* __restrict__ err) {
    __shared__ uint32_t tab[47];
    __shared__ uint32_t cst[32 * 128];
    for (int i = threadIdx.x; i < 47; i += blockDim.x)
        tab[i] = (uint32_t)c_qe[i] | ((uint32_t)c_nmps[i] << 16) | ((uint32_t)c_nlps[i] << 22) |
                 ((uint32_t)(i == 0 || i == 6 || i == 14) << 28);
    __syncthreads();
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= nslots || keys[gid] == 0) return;  // keys are sorted: the empty slots come last
    const int u = (int)order[gid];
    const int j = u / J2K_PASS_STRIDE, k = u % J2K_PASS_STRIDE;
    const j2k_cb_job J = jobs[j];
    const int np = descs[j].npasses;
    const bool per_pass = units_per_pass(style);
    const int p0 = per_pass ? k : 0, p1 = per_pass ? k + 1 : np;
    const uint32_t* pe = pend + (size_t)j * J2K_PASS_STRIDE;
    uint32_t* eo = ends + (size_t)j * J2K_PASS_STRIDE;
    const uint32_t s0 = p0 ? pe[p0 - 1] : 0u, s1 = pe[p1 - 1];
    if (s1 > J.sym_cap || s0 > s1) {
        atomicCAS(err, 0u, (uint32_t)J2K_DEVERR_BAD_JOB);
        return;
    }
    const uint64_t base = seg_slot(J.sym_off, s0, j, p0, fac);
    const uint64_t lim = seg_slot(J.sym_off, s1, j, p1, fac);
    uint32_t* st = cst + threadIdx.x;  // context c at st[c * 128]
    auto reset_states = [&]() {
        for (int c = 0; c < 32; ++c) st[c * 128] = tab[0];
        st[0] = tab[4];
        st[17 * 128] = tab[3];
        st[18 * 128] = tab[46];
    };
    reset_states();
    MqEnc e;
    e.out = reinterpret_cast<uint32_t*>(segs + base);
    e.cap = (int)(lim - base);
    e.wacc = 0;
    e.wn = 0;
    e.wbase = 0;
    e.ovf = false;
    // raw coder: bits of the byte being filled, bits left in it, the last completed byte (held
    // back one byte so that a final 0xFF can be dropped)
    uint32_t rc = 0;
    int rct = 8, rpend = -1;
    bool rlastff = false, raw = false;
    auto raw_complete = [&](uint32_t b) {
        if (rpend >= 0) e.push((uint32_t)rpend);
        rpend = (int)b;
        rlastff = b == 0xFF;
        rct = rlastff ? 7 : 8;
        rc = 0;
    };
    const uint8_t* sp = syms + J.sym_off;
    for (int p = p0; p < p1; ++p) {
        if (p > p0 && (style & J2K_CBLK_RESET)) reset_states();
        raw = j2k_pass_raw(style, p);
        if (p == p0 || j2k_pass_terminated(style, p - 1, np)) {  // a new segment
            if (raw) {
                rc = 0;
                rct = 8;
                rpend = -1;
                rlastff = false;
            } else {
                e.A = 0x8000;
                e.C = 0;
                e.B = 0;
                e.CT = 12;
                e.bp = -1;
            }
        }
        const uint32_t a = p ? pe[p - 1] : 0u, b = pe[p];
        uint32_t word = 0;
        for (uint32_t i = a; i < b; ++i) {
            if (i == a || (i & 3) == 0) word = __ldcs(reinterpret_cast<const uint32_t*>(sp + (i & ~3u)));
            const uint32_t sym = (word >> (8 * (i & 3))) & 0xFF;
            if (raw) {
                const uint32_t lab = sym & 31;
                const uint32_t bit = ((sym >> 7) ^ ((lab >= 9 && lab <= 13) ? (sym >> 5) : 0u)) & 1u;
                rc = (rc << 1) | bit;
                if (--rct == 0) raw_complete(rc & 0xFF);
            } else {
                const int cx = (int)(sym & 31);
                const int d = (int)(sym >> 7);
                const uint32_t ent = st[cx * 128];
                const uint32_t qe = ent & 0xFFFF;
                const int mps = (int)(ent >> 31);
                const bool is_mps = d == mps;
                const uint32_t a1 = e.A - qe;
                const bool fast = is_mps && (a1 & 0x8000);
                const bool addc = fast || (is_mps != (a1 < qe));
                e.C += addc ? qe : 0u;
                e.A = addc ? a1 : qe;
                if (!fast) {
                    const int nidx = is_mps ? (ent >> 16) & 63 : (ent >> 22) & 63;
                    const uint32_t nmps = (uint32_t)(mps ^ (!is_mps & (int)((ent >> 28) & 1)));
                    st[cx * 128] = tab[nidx] | (nmps << 31);
                }
                e.renorm(__clz(e.A) - 16);
            }
        }
        if (j2k_pass_terminated(style, p, np)) {
            if (raw) {
                if (rct < (rlastff ? 7 : 8)) raw_complete((rc << rct) & 0xFF);
                if (rpend >= 0 && rpend != 0xFF) e.push((uint32_t)rpend);
                rpend = -1;
            } else {  // FLUSH (T.800 C.2.9); a last byte of 0xFF is dropped
                const uint32_t tempc = e.C + e.A;
                e.C |= 0xFFFF;
                if (e.C >= tempc) e.C -= 0x8000;
                e.C <<= e.CT;
                e.byteout();
                e.C <<= e.CT;
                e.byteout();
                if (e.B != 0xFF) e.push(e.B);
            }
            eo[p] = (uint32_t)(e.wbase + e.wn);
        } else {
            eo[p] = (uint32_t)(e.wbase + e.wn) + (raw ? (rpend >= 0) : (uint32_t)(e.bp + 1 > 0));
        }
    }
    // the last partial word
    uint8_t* bb = segs + base;
    for (int q = 0; q < e.wn; ++q) {
        if (e.wbase + q < e.cap) bb[e.wbase + q] = (uint8_t)(e.wacc >> (8 * q));
        else e.ovf = true;
    }
    if (e.ovf) {
        atomicCAS(err, 0u, (uint32_t)J2K_DEVERR_SEG_CAPACITY);
        ulen[u] = 0;
        return;
    }
    ulen[u] = (uint32_t)(e.wbase + e.wn);
}

// Per-pass units (RESET | TERMALL: every pass a codeword segment that starts from fresh context
// states and a fresh coder): one lane per pass, passes longest first, the MQ passes before the
// raw ones.  An MQ pass runs the same loop as t1_mq_kernel (16-byte symbol chunks two in flight,
// four symbols per unrolled body, the next context's state loaded one symbol ahead and
// forwarded), from its 16-byte aligned start, and ends with the FLUSH of T.800 C.2.9 (a last
// 0xFF dropped), however few symbols it has; a raw pass writes its decisions as bits (T.800
// D.6: a byte after 0xFF holds 7, the partial last byte padded with 0s, a last 0xFF dropped).
// Unit bytes go to the pass's slot; ulen / ends as t1_mq_units_kernel.
constexpr int kPassThreads = 128;

__global__ void __launch_bounds__(kPassThreads)
t1_mq_pass_kernel(const uint8_t* __restrict__ syms, const j2k_cb_job* __restrict__ jobs,
                  const j2k_cb_desc* __restrict__ descs, const uint32_t* __restrict__ pend,
                  const uint32_t* __restrict__ order, const uint32_t* __restrict__ keys, int nslots, int style,
                  int fac, uint8_t* __restrict__ segs, uint32_t* __restrict__ ulen, uint32_t* __restrict__ ends,
                  uint32_t* __restrict__ err) {
    __shared__ uint32_t tab[47];
    __shared__ uint32_t cst[32 * kPassThreads];  // 32 contexts per lane: a 5-bit index needs no clamp
    for (int i = threadIdx.x; i < 47; i += blockDim.x)
        tab[i] = (uint32_t)c_qe[i] | ((uint32_t)c_nmps[i] << 16) | ((uint32_t)c_nlps[i] << 22) |
                 ((uint32_t)(i == 0 || i == 6 || i == 14) << 28);
    __syncthreads();
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= nslots || keys[gid] == 0) return;  // keys are sorted: the empty slots come last
    const int u = (int)order[gid];
    const int j = u / J2K_PASS_STRIDE, p = u % J2K_PASS_STRIDE;
    const j2k_cb_job J = jobs[j];
    const uint32_t* pe = pend + (size_t)j * J2K_PASS_STRIDE;
    const uint32_t s0 = pass_start(pe, p, true), s1 = pe[p];
    const uint32_t snext = (s1 + 15u) & ~15u;  // where the next pass's symbols (and slot) start
    if (s1 > J.sym_cap || s0 > s1) {
        atomicCAS(err, 0u, (uint32_t)J2K_DEVERR_BAD_JOB);
        return;
    }
    const int n = (int)(s1 - s0);
    const uint64_t base = seg_slot(J.sym_off, s0, j, p, fac);
    const uint64_t lim = seg_slot(J.sym_off, snext, j, p + 1, fac);
    MqEnc e;
    e.A = 0x8000;
    e.C = 0;
    e.B = 0;
    e.CT = 12;
    e.bp = -1;
    e.out = reinterpret_cast<uint32_t*>(segs + base);
    e.cap = (int)(lim - base);
    e.wacc = 0;
    e.wn = 0;
    e.wbase = 0;
    e.ovf = false;
    const uint4* sp4 = reinterpret_cast<const uint4*>(syms + J.sym_off + s0);
    const int nchunks = (n + 15) >> 4;
    const uint4 z4 = make_uint4(0, 0, 0, 0);
    uint4 c0 = nchunks > 0 ? __ldcs(sp4) : z4;
    uint4 c1 = nchunks > 1 ? __ldcs(sp4 + 1) : z4;
    if (j2k_pass_raw(style, p)) {
        uint32_t rc = 0;
        int rct = 8, rpend = -1;
        bool rlastff = false;
        auto complete = [&](uint32_t b) {
            if (rpend >= 0) e.push((uint32_t)rpend);
            rpend = (int)b;
            rlastff = b == 0xFF;
            rct = rlastff ? 7 : 8;
            rc = 0;
        };
        for (int k = 0; k < nchunks; ++k) {
            const uint4 cur = c0;
            c0 = c1;
            c1 = (k + 2 < nchunks) ? __ldcs(sp4 + k + 2) : z4;
            const uint32_t wv[4] = {cur.x, cur.y, cur.z, cur.w};
            const int m = min(16, n - 16 * k);
            for (int i = 0; i < m; ++i) {
                const uint32_t sym = (wv[i >> 2] >> (8 * (i & 3))) & 0xFF;
                const uint32_t lab = sym & 31;
                const uint32_t bit = ((sym >> 7) ^ ((lab >= 9 && lab <= 13) ? (sym >> 5) : 0u)) & 1u;
                rc = (rc << 1) | bit;
                if (--rct == 0) complete(rc & 0xFF);
            }
        }
        if (rct < (rlastff ? 7 : 8)) complete((rc << rct) & 0xFF);
        if (rpend >= 0 && rpend != 0xFF) e.push((uint32_t)rpend);
    } else {
        uint32_t* st = cst + threadIdx.x;  // context c at st[c * kPassThreads]
        for (int c = 0; c < 32; ++c) st[c * kPassThreads] = tab[0];
        st[0] = tab[4];
        st[17 * kPassThreads] = tab[3];
        st[18 * kPassThreads] = tab[46];
        int cx = (int)(c0.x & 31);
        uint32_t ent = st[cx * kPassThreads];
        auto step = [&](uint32_t sym, uint32_t nsym) {
            const int d = sym >> 7;
            const int ncx = (int)(nsym & 31);
            uint32_t nent = st[ncx * kPassThreads];
            const uint32_t qe = ent & 0xFFFF;
            const int mps = ent >> 31;
            const bool is_mps = d == mps;
            const uint32_t a1 = e.A - qe;
            const bool fast = is_mps && (a1 & 0x8000);
            const bool addc = fast || (is_mps != (a1 < qe));
            e.C += addc ? qe : 0u;
            e.A = addc ? a1 : qe;
            const int nidx = is_mps ? (ent >> 16) & 63 : (ent >> 22) & 63;
            const uint32_t nmps = (uint32_t)(mps ^ (!is_mps & (int)((ent >> 28) & 1)));
            const uint32_t upd = tab[nidx] | (nmps << 31);
            if (!fast) {
                st[cx * kPassThreads] = upd;
                if (ncx == cx) nent = upd;
            }
            e.renorm(__clz(e.A) - 16);
            cx = ncx;
            ent = nent;
        };
        for (int k = 0; k < nchunks; ++k) {
            const uint4 cur = c0;
            c0 = c1;
            c1 = (k + 2 < nchunks) ? __ldcs(sp4 + k + 2) : z4;
            const int m = min(16, n - 16 * k);
            uint32_t wa = cur.x, wb = cur.y, wc = cur.z, wd = cur.w;
            const uint32_t we = c0.x;
#pragma unroll 1
            for (int q = 0; q < 4 && 4 * q < m; ++q) {
                if (4 * q + 4 <= m) {
#pragma unroll
                    for (int jj = 0; jj < 4; ++jj)
                        step((wa >> (8 * jj)) & 0xFF, jj < 3 ? (wa >> (8 * (jj + 1))) & 0xFF : wb & 0xFF);
                } else {
#pragma unroll
                    for (int jj = 0; jj < 4; ++jj)
                        if (4 * q + jj < m) step((wa >> (8 * jj)) & 0xFF, jj < 3 ? (wa >> (8 * (jj + 1))) & 0xFF : wb & 0xFF);
                }
                wa = wb;
                wb = wc;
                wc = wd;
                wd = we;
            }
        }
        // FLUSH (T.800 C.2.9); a last byte of 0xFF is dropped
        const uint32_t tempc = e.C + e.A;
        e.C |= 0xFFFF;
        if (e.C >= tempc) e.C -= 0x8000;
        e.C <<= e.CT;
        e.byteout();
        e.C <<= e.CT;
        e.byteout();
        if (e.B != 0xFF) e.push(e.B);
    }
    uint8_t* bb = segs + base;
    for (int q = 0; q < e.wn; ++q) {
        if (e.wbase + q < e.cap) bb[e.wbase + q] = (uint8_t)(e.wacc >> (8 * q));
        else e.ovf = true;
    }
    if (e.ovf) {
        atomicCAS(err, 0u, (uint32_t)J2K_DEVERR_SEG_CAPACITY);
        ulen[u] = 0;
        return;
    }
    const uint32_t len = (uint32_t)(e.wbase + e.wn);
    ulen[u] = len;
    ends[(size_t)j * J2K_PASS_STRIDE + p] = len;
}

// One warp per code-block: its units' segments back to back into the block's codeword, the
// pass ends made block-relative, and the descriptor's length.
__global__ void t1_units_compact_kernel(const j2k_cb_job* __restrict__ jobs, j2k_cb_desc* __restrict__ descs,
                                        const uint32_t* __restrict__ pend, int njobs, int style, int fac,
                                        const uint8_t* __restrict__ segs, const uint32_t* __restrict__ ulen,
                                        uint32_t* __restrict__ ends, uint8_t* __restrict__ bytes,
                                        uint32_t* __restrict__ err) {
    const int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (j >= njobs) return;
    const j2k_cb_job J = jobs[j];
    const int np = descs[j].npasses;
    const bool per_pass = units_per_pass(style);
    const int nu = np == 0 ? 0 : (per_pass ? np : 1);
    const uint32_t* pe = pend + (size_t)j * J2K_PASS_STRIDE;
    uint32_t* eo = ends + (size_t)j * J2K_PASS_STRIDE;
    uint32_t run = 0;  // bytes of the units before this round of 32
    uint8_t* dst = bytes + J.out_off;
    for (int k0 = 0; k0 < nu; k0 += 32) {
        const int k = k0 + lane;
        const uint32_t len = k < nu ? ulen[(size_t)j * J2K_PASS_STRIDE + k] : 0u;
        int tot;
        const uint32_t off = run + (uint32_t)warp_excl((int)len, lane, &tot);
        if (k < nu) {
            if (off + len > J.out_cap) {
                atomicCAS(err, 0u, (uint32_t)J2K_DEVERR_OUT_CAPACITY);
            } else {
                const int p0 = per_pass ? k : 0, p1 = per_pass ? k + 1 : np;
                for (int p = p0; p < p1; ++p) eo[p] += off;
            }
        }
        // the round's units copied one after another, each by the whole warp
        const bool ok = k < nu && off + len <= J.out_cap;
        const unsigned okm = __ballot_sync(0xffffffffu, ok);
        for (int q = 0; q < 32; ++q) {
            if (!((okm >> q) & 1u)) continue;
            const uint32_t ql = __shfl_sync(0xffffffffu, len, q), qo = __shfl_sync(0xffffffffu, off, q);
            const int kq = k0 + q;
            const int p0 = per_pass ? kq : 0;
            const uint8_t* src = segs + seg_slot(J.sym_off, pass_start(pe, p0, per_pass), j, p0, fac);
            for (uint32_t b = (uint32_t)lane; b < ql; b += 32) dst[qo + b] = src[b];
        }
        run += (uint32_t)tot;
    }
    for (int p = np + lane; p < J2K_PASS_STRIDE; p += 32) eo[p] = 0;
    if (lane == 0) descs[j].length = run <= J.out_cap ? (int32_t)run : 0;
}

__global__ void iota_kernel(uint32_t* v, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = (uint32_t)i;
}

// Squared reconstruction error of every code-block when decoded down to bit-plane k only
// (dist[job * 33 + k]; magnitudes below the last decoded plane at the middle of their interval)
// and with nothing decoded (dist[job * 33 + 32]).  One warp per block, kDistWarps blocks per CTA.
// Each lane keeps one exact 64-bit sum per plane p in registers: a sample of magnitude m with
// top bit b adds its midpoint error at the planes p <= b and m^2 at the planes above b; the
// lanes' sums are then added by shuffles.  Integer sums, so the result (and the truncation
// choices built on it) does not depend on the order of the additions.
constexpr int kDistWarps = 4;
__global__ void __launch_bounds__(kDistWarps * 32)
t1_dist_kernel(const int32_t* __restrict__ coeff, const j2k_cb_job* __restrict__ jobs,
               const j2k_cb_desc* __restrict__ descs, int njobs, double* __restrict__ dist) {
    const int lane = threadIdx.x & 31;
    const int jid = blockIdx.x * kDistWarps + (threadIdx.x >> 5);
    if (jid >= njobs) return;
    const j2k_cb_job J = jobs[jid];
    const int nb = min((int)descs[jid].numbps, 31);  // the same for the whole warp
    unsigned long long acc[31], total = 0;
#pragma unroll
    for (int p = 0; p < 31; ++p) acc[p] = 0;
    if (J.cw <= 64 && J.ch <= 64) {
        for (int y = 0; y < J.ch; ++y) {
            const int32_t* row = coeff + J.off + (size_t)y * J.pitch;
            for (int x = lane; x < J.cw; x += 32) {
                const int32_t v = row[x];
                const uint32_t m = v < 0 ? (uint32_t)(-(int64_t)v) : (uint32_t)v;
                const int b = 31 - __clz(m);  // -1 for m = 0, which adds nothing
                const unsigned long long m2 = (unsigned long long)m * m;
                total += m2;
#pragma unroll
                for (int p = 0; p < 31; ++p) {
                    if (p >= nb) break;
                    // m - (m truncated to plane p + half its interval); |e| < 2^30
                    const int e = (int)(m & ((1u << p) - 1u)) - (int)((1u << p) >> 1);
                    acc[p] += p <= b ? (unsigned long long)((long long)e * e) : m2;
                }
            }
        }
    }
#pragma unroll
    for (int p = 0; p < 31; ++p) {
        if (p >= nb) break;
        unsigned long long s = acc[p];
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        acc[p] = s;
    }
    for (int o = 16; o; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
    if (lane == 0) {
        double* d = dist + (size_t)jid * 33;
        // plane p is the last decoded one after k = nb - 1 - p planes
#pragma unroll
        for (int p = 0; p < 31; ++p)
            if (p < nb) d[nb - 1 - p] = (double)acc[p];
        for (int k = nb; k < 32; ++k) d[k] = 0.0;
        d[32] = (double)total;
    }
}

}  // namespace

// Phase B of a styled encode: units keyed and sorted longest first, coded one lane each, then
// compacted into the blocks' codewords.
static j2k_status encode_styled_units(j2k_ctx* ctx, const j2k_cb_job* d_jobs, size_t njobs, j2k_cb_desc* descs,
                                      uint8_t* bytes, size_t sym_bytes, const uint8_t* syms, const uint32_t* pend,
                                      int style, uint32_t* pass_ends, cudaStream_t st) {
    const size_t nslots = njobs * J2K_PASS_STRIDE;
    if (nslots > 0x7FFFFFFF) return j2k_fail(ctx, J2K_ERR_UNSUPPORTED, "too many code-blocks for a styled encode");
    uint32_t* ub = (uint32_t*)j2k_scratch(ctx, SCR_UNITS, (nslots * (pass_ends ? 5 : 6) + 64) * 4);
    if (!ub) return J2K_ERR_OUT_OF_MEMORY;
    uint32_t* keys_in = ub;
    uint32_t* keys_out = keys_in + nslots;
    uint32_t* ids_in = keys_out + nslots;
    uint32_t* ids_out = ids_in + nslots;
    uint32_t* ulen = ids_out + nslots;
    uint32_t* ends = pass_ends ? pass_ends : ulen + nslots;
    const int fac = std::max(1, ctx->t1_seg_factor);
    // slots end by fac * (sym_bytes + 3) + 16 * nslots (seg_slot of the last unit's end)
    uint8_t* segs = (uint8_t*)j2k_scratch(ctx, SCR_SEGS, (size_t)fac * (sym_bytes + 64) + 16 * nslots + 64);
    if (!segs) return J2K_ERR_OUT_OF_MEMORY;
    const unsigned g = (unsigned)((nslots + 255) / 256);
    t1_unit_keys_kernel<<<g, 256, 0, st>>>(descs, pend, (int)njobs, style, keys_in, ids_in);
    J2K_CUDA(ctx, cudaGetLastError());
    size_t tmp = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp, keys_in, keys_out, ids_in, ids_out, (int)nslots, 0, 32,
                                              st);
    void* tbuf = j2k_scratch(ctx, SCR_MISC, tmp + 16);
    if (!tbuf) return J2K_ERR_OUT_OF_MEMORY;
    J2K_CUDA(ctx, cub::DeviceRadixSort::SortPairsDescending(tbuf, tmp, keys_in, keys_out, ids_in, ids_out,
                                                            (int)nslots, 0, 32, st));
    if (units_per_pass(style))
        t1_mq_pass_kernel<<<(unsigned)((nslots + kPassThreads - 1) / kPassThreads), kPassThreads, 0, st>>>(
            syms, d_jobs, descs, pend, ids_out, keys_out, (int)nslots, style, fac, segs, ulen, ends, ctx->d_err);
    else
        t1_mq_units_kernel<<<(unsigned)((nslots + 127) / 128), 128, 0, st>>>(syms, d_jobs, descs, pend, ids_out,
                                                                             keys_out, (int)nslots, style, fac, segs,
                                                                             ulen, ends, ctx->d_err);
    J2K_CUDA(ctx, cudaGetLastError());
    t1_units_compact_kernel<<<(unsigned)((njobs * 32 + 255) / 256), 256, 0, st>>>(
        d_jobs, descs, pend, (int)njobs, style, fac, segs, ulen, ends, bytes, ctx->d_err);
    J2K_CUDA(ctx, cudaGetLastError());
    return J2K_OK;
}

j2k_status j2k_t1_encode_jobs(j2k_ctx* ctx, const int32_t* coeff, const j2k_cb_job* d_jobs, size_t njobs,
                              j2k_cb_desc* descs, uint8_t* bytes, size_t sym_bytes,
                              const uint32_t* d_order, cudaStream_t st, uint32_t* plane_bytes, double* dist,
                              int style, uint32_t* pass_ends) {
    if (njobs == 0) return J2K_OK;
    if (style && (plane_bytes || dist))
        return j2k_fail(ctx, J2K_ERR_UNSUPPORTED, "rate control with a code-block style");
    if (((uintptr_t)bytes & 15) != 0)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "t1: bytes buffer must be 16-byte aligned");
    uint8_t* syms = (uint8_t*)j2k_scratch(ctx, SCR_SYMS, sym_bytes + 64);
    // persistent phase A: one bit-plane slot per resident warp
    int per_sm = 0;
    const bool occ3 = ctx->t1a_ctas == 3;
    if (occ3)
        J2K_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, t1_symbols_kernel<3>, kWarpsPerCta * 32, 0));
    else
        J2K_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, t1_symbols_kernel<2>, kWarpsPerCta * 32, 0));
    per_sm = std::max(per_sm, 1);
    const size_t ctas = std::min<size_t>((njobs + kWarpsPerCta - 1) / kWarpsPerCta, (size_t)per_sm * ctx->sm_count);
    uint64_t* planes = (uint64_t*)j2k_scratch(ctx, SCR_PLANES, ctas * kWarpsPerCta * kPlaneWords * 8 + 64);
    // meta: queue head | nsyms | pass ends (92 per job) | sort keys/values (3 arrays of njobs)
    size_t meta_words = 16 + njobs * (1 + 92 + 3) + 64;
    uint32_t* meta = (uint32_t*)j2k_scratch(ctx, SCR_T1STATE, meta_words * 4);
    if (!syms || !meta || !planes) return J2K_ERR_OUT_OF_MEMORY;
    uint32_t* queue = meta;
    uint32_t* nsyms = meta + 16;
    uint32_t* pend = nsyms + njobs;
    uint32_t* keys_out = pend + njobs * 92;
    uint32_t* idx_in = keys_out + njobs;
    uint32_t* idx_out = idx_in + njobs;
    J2K_CUDA(ctx, cudaMemsetAsync(queue, 0, 4, st));
    // with per-pass coding units (RESET | TERMALL) every pass's symbols start 16-byte aligned
    const int pad = (style & (J2K_CBLK_RESET | J2K_CBLK_TERMALL)) == (J2K_CBLK_RESET | J2K_CBLK_TERMALL) ? 1 : 0;
    if (occ3)
        t1_symbols_kernel<3><<<(unsigned)ctas, kWarpsPerCta * 32, 0, st>>>(coeff, d_jobs, (int)njobs, d_order, queue,
                                                                          syms, nsyms, pend, planes, descs, ctx->d_err,
                                                                          pad);
    else
        t1_symbols_kernel<2><<<(unsigned)ctas, kWarpsPerCta * 32, 0, st>>>(coeff, d_jobs, (int)njobs, d_order, queue,
                                                                          syms, nsyms, pend, planes, descs, ctx->d_err,
                                                                          pad);
    J2K_CUDA(ctx, cudaGetLastError());
    if (style)
        return encode_styled_units(ctx, d_jobs, njobs, descs, bytes, sym_bytes, syms, pend, style, pass_ends, st);
    // longest-first order for the MQ lanes
    iota_kernel<<<(unsigned)((njobs + 255) / 256), 256, 0, st>>>(idx_in, (int)njobs);
    size_t tmp = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp, nsyms, keys_out, idx_in, idx_out, (int)njobs, 0, 32, st);
    void* tbuf = j2k_scratch(ctx, SCR_MISC, tmp + 16);
    if (!tbuf) return J2K_ERR_OUT_OF_MEMORY;
    J2K_CUDA(ctx, cub::DeviceRadixSort::SortPairsDescending(tbuf, tmp, nsyms, keys_out, idx_in, idx_out,
                                                            (int)njobs, 0, 32, st));
    if (ctx->mq_variant == 1 && !(plane_bytes && dist)) {  // the rate path runs the one-lane coder
        unsigned gp = (unsigned)((njobs + 31) / 32);
        t1_mq_pair_kernel<<<gp, 64, 0, st>>>(syms, d_jobs, nsyms, idx_out, (int)njobs, bytes, descs, ctx->d_err);
        J2K_CUDA(ctx, cudaGetLastError());
        return J2K_OK;
    }
    const int lanes = ctx->mq_lanes;  // active lanes (blocks) per warp: 32, 16 or 8
    // tiers of the schedule, cut to the blocks there are
    MqSchedule sc{};
    size_t left = njobs, warps = 0;
    for (int k = 0; k < J2K_MQ_TIERS && ctx->mq_tier_lanes[k] > 0 && left > 0; ++k) {
        const size_t l = (size_t)ctx->mq_tier_lanes[k];
        const size_t wk = std::min<size_t>((size_t)ctx->mq_tier_warps[k], (left + l - 1) / l);
        sc.warps[k] = (int)wk;
        sc.lanes[k] = (int)l;
        left -= std::min(left, wk * l);
        warps += wk;
    }
    warps += (left + lanes - 1) / lanes;
    unsigned gb = (unsigned)((warps + kMqThreads / 32 - 1) / (kMqThreads / 32));
    const bool rate = plane_bytes && dist;
    // rate control also records the byte positions at every bit-plane end, and the distortion
    // of each truncation point (the coefficients are still in place)
    if (rate) {
        if (lanes == 8)
            t1_mq_kernel<8, true><<<gb, kMqThreads, 0, st>>>(syms, d_jobs, nsyms, idx_out, (int)njobs, bytes, descs,
                                                             ctx->d_err, pend, plane_bytes, sc);
        else if (lanes == 16)
            t1_mq_kernel<16, true><<<gb, kMqThreads, 0, st>>>(syms, d_jobs, nsyms, idx_out, (int)njobs, bytes, descs,
                                                              ctx->d_err, pend, plane_bytes, sc);
        else
            t1_mq_kernel<32, true><<<gb, kMqThreads, 0, st>>>(syms, d_jobs, nsyms, idx_out, (int)njobs, bytes, descs,
                                                              ctx->d_err, pend, plane_bytes, sc);
        J2K_CUDA(ctx, cudaGetLastError());
        t1_dist_kernel<<<(unsigned)((njobs + kDistWarps - 1) / kDistWarps), kDistWarps * 32, 0, st>>>(
            coeff, d_jobs, descs, (int)njobs, dist);
    } else if (lanes == 8)
        t1_mq_kernel<8><<<gb, kMqThreads, 0, st>>>(syms, d_jobs, nsyms, idx_out, (int)njobs, bytes, descs, ctx->d_err,
                                                   nullptr, nullptr, sc);
    else if (lanes == 16)
        t1_mq_kernel<16><<<gb, kMqThreads, 0, st>>>(syms, d_jobs, nsyms, idx_out, (int)njobs, bytes, descs,
                                                    ctx->d_err, nullptr, nullptr, sc);
    else
        t1_mq_kernel<32><<<gb, kMqThreads, 0, st>>>(syms, d_jobs, nsyms, idx_out, (int)njobs, bytes, descs,
                                                    ctx->d_err, nullptr, nullptr, sc);
    J2K_CUDA(ctx, cudaGetLastError());
    return J2K_OK;
}
