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
// symbol (label in bits 0-4, decision in bit 7).
//
// Phase B — one lane per code-block runs the MQ encoder over its symbol stream (T.800 C.2,
// FLUSH of C.2.9, trailing 0xFF dropped); codeword bytes are written as aligned 32-bit words.
#include <cub/cub.cuh>

#include "j2k_internal.cuh"

namespace {

constexpr int kWarpsPerCta = 4;
constexpr int kPlanesShared = 16;   // magnitude planes kept in shared memory; more are sliced from global
constexpr int kRows = 64;
constexpr int kMaxStage = 20;       // symbols per lane per stripe pass (2 columns x 10)

struct WarpSmem {
    uint64_t planes[kPlanesShared][kRows];
    uint64_t sig[kRows + 2], vis[kRows + 2], ref[kRows + 2], neg[kRows + 2];
    uint8_t stage[32][kMaxStage];
};

// T.800 Table D.1 zero-coding labels, index [orient][h][v][d]
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

__device__ __forceinline__ uint64_t dil(uint64_t m) { return m | (m << 1) | (m >> 1); }
__device__ __forceinline__ int bitat(uint64_t m, int c) { return (c < 0 || c > 63) ? 0 : (int)((m >> c) & 1); }

// (label | xor<<7) for the sign context of a sample, T.800 Tables D.2/D.3
__device__ __forceinline__ int sc_code(int hc, int vc) {
    hc = max(-1, min(1, hc));
    vc = max(-1, min(1, vc));
    int x = 0;
    if (hc < 0 || (hc == 0 && vc < 0)) { hc = -hc; vc = -vc; x = 1; }
    int lab = hc == 0 ? (vc ? 10 : 9) : 12 + vc;
    return lab | (x << 7);
}

struct Ctx {
    const int32_t* blk;   // block origin in the coefficient plane
    size_t pitch;
    int cw, ch;
};

// bit-plane row mask for plane p >= kPlanesShared, sliced from global memory
__device__ uint64_t plane_row_global(const Ctx& c, int p, int r, int lane) {
    uint32_t lo = 0, hi = 0;
    int32_t v0 = (lane < c.cw) ? c.blk[(size_t)r * c.pitch + lane] : 0;
    int32_t v1 = (lane + 32 < c.cw) ? c.blk[(size_t)r * c.pitch + lane + 32] : 0;
    uint32_t m0 = v0 < 0 ? (uint32_t)(-(int64_t)v0) : (uint32_t)v0;
    uint32_t m1 = v1 < 0 ? (uint32_t)(-(int64_t)v1) : (uint32_t)v1;
    lo = __ballot_sync(0xffffffffu, (m0 >> p) & 1);
    hi = __ballot_sync(0xffffffffu, (m1 >> p) & 1);
    return (uint64_t)lo | ((uint64_t)hi << 32);
}

__device__ __forceinline__ uint64_t plane_row(const WarpSmem& S, const Ctx& c, int p, int r, int lane) {
    if (r >= c.ch || r < 0) return 0;
    if (p < kPlanesShared) return S.planes[p][r];
    return plane_row_global(c, p, r, lane);
}

// emit staged symbols of all lanes in lane order; returns the warp total
__device__ __forceinline__ int flush_stage(WarpSmem& S, int lane, int cnt, uint8_t* out, int pos,
                                           int cap, bool& ovf) {
    int inc = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    int total = __shfl_sync(0xffffffffu, inc, 31);
    int off = pos + inc - cnt;
    if (pos + total > cap) {
        ovf = true;
        return total;
    }
    for (int k = 0; k < cnt; ++k) out[off + k] = S.stage[lane][k];
    return total;
}

__global__ void __launch_bounds__(kWarpsPerCta * 32)
t1_symbols_kernel(const int32_t* __restrict__ coeff, size_t pitch, const j2k_cb_job* __restrict__ jobs,
                  int njobs, uint8_t* __restrict__ syms, size_t sym_cap, uint32_t* __restrict__ nsyms,
                  uint32_t* __restrict__ pass_end, j2k_cb_desc* __restrict__ descs,
                  size_t cap_per_block, uint32_t* __restrict__ err) {
    __shared__ WarpSmem smem[kWarpsPerCta];
    __shared__ uint8_t zc_lut[4][3][3][5];
    for (int i = threadIdx.x; i < 4 * 45; i += blockDim.x) {
        int o = i / 45, r = i % 45;
        zc_lut[o][r / 15][(r / 5) % 3][r % 5] = (uint8_t)zc_label_calc(o, r / 15, (r / 5) % 3, r % 5);
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int jid = blockIdx.x * kWarpsPerCta + wid;
    if (jid >= njobs) return;
    WarpSmem& S = smem[wid];
    const j2k_cb_job J = jobs[jid];
    if (J.cw == 0 || J.ch == 0 || J.cw > 64 || J.ch > 64 || J.orient > 3) {
        if (lane == 0) {
            atomicCAS(err, 0u, (uint32_t)J2K_DEVERR_BAD_JOB);
            nsyms[jid] = 0;
        }
        return;
    }
    Ctx c{coeff + (size_t)J.y0 * pitch + J.x0, pitch, J.cw, J.ch};
    const int orient = J.orient;
    const uint64_t colmask = c.cw == 64 ? ~0ull : ((1ull << c.cw) - 1);

    // ---- slice magnitudes into bit-plane masks; signs; numbps
    uint32_t mor = 0;
    for (int r = 0; r < c.ch; ++r) {
        int32_t v0 = (lane < c.cw) ? c.blk[(size_t)r * pitch + lane] : 0;
        int32_t v1 = (lane + 32 < c.cw) ? c.blk[(size_t)r * pitch + lane + 32] : 0;
        uint32_t m0 = v0 < 0 ? (uint32_t)(-(int64_t)v0) : (uint32_t)v0;
        uint32_t m1 = v1 < 0 ? (uint32_t)(-(int64_t)v1) : (uint32_t)v1;
        mor |= m0 | m1;
        uint64_t ng = (uint64_t)__ballot_sync(0xffffffffu, v0 < 0) |
                      ((uint64_t)__ballot_sync(0xffffffffu, v1 < 0) << 32);
        if (lane == 0) S.neg[r + 1] = ng;
#pragma unroll 4
        for (int p = 0; p < kPlanesShared; ++p) {
            uint64_t pm = (uint64_t)__ballot_sync(0xffffffffu, (m0 >> p) & 1) |
                          ((uint64_t)__ballot_sync(0xffffffffu, (m1 >> p) & 1) << 32);
            if (lane == 0) S.planes[p][r] = pm;
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) mor |= __shfl_xor_sync(0xffffffffu, mor, o);
    const int numbps = mor ? 32 - __clz(mor) : 0;
    for (int r = lane; r < kRows + 2; r += 32) {
        S.sig[r] = 0;
        S.vis[r] = 0;
        S.ref[r] = 0;
        if (r == 0 || r > c.ch) S.neg[r] = 0;
    }
    __syncwarp();
    j2k_cb_desc d;
    d.offset = (uint32_t)((size_t)jid * cap_per_block);
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
        return;
    }
    uint8_t* out = syms + (size_t)jid * sym_cap;
    uint32_t* pend = pass_end + (size_t)jid * 92;
    const int cap = (int)sym_cap;
    int pos = 0, npass = 0;
    bool ovf = false;
    const int nstripes = (c.ch + 3) >> 2;
    const int c0 = 2 * lane, c1 = 2 * lane + 1;

    for (int p = numbps - 1; p >= 0 && !ovf; --p) {
        if (p != numbps - 1) {
            // ------------------------- significance propagation pass
            for (int s = 0; s < nstripes && !ovf; ++s) {
                const int r0 = 4 * s;
                uint64_t O[6], A[6], B[4], C[4], M[4], E[4], N[6], K[4];
                for (int j = -1; j <= 4; ++j) O[j + 1] = S.sig[r0 + j + 1];
                for (int j = 0; j < 4; ++j) {
                    uint64_t V = (r0 + j < c.ch) ? colmask : 0;
                    B[j] = plane_row(S, c, p, r0 + j, lane);
                    C[j] = ~O[j + 1] & V;
                    M[j] = C[j] & B[j];
                    E[j] = dil(O[j]) | dil(O[j + 1]) | dil(O[j + 2]);
                }
                N[0] = N[1] = N[2] = N[3] = N[4] = N[5] = 0;
                bool changed = true;
                while (changed) {
                    changed = false;
                    for (int j = 0; j < 4; ++j) {
                        uint64_t seeds = M[j] & (E[j] | ((N[j] | N[j + 2]) << 1) | N[j]);
                        uint64_t nn = M[j] & (~(M[j] + seeds) | seeds);
                        if (nn != N[j + 1]) { N[j + 1] = nn; changed = true; }
                    }
                }
                for (int j = 0; j < 4; ++j)
                    K[j] = C[j] & (E[j] | ((N[j] | N[j + 1] | N[j + 2]) << 1) | N[j]);
                A[0] = O[0];
                A[5] = O[5];
                for (int j = 0; j < 4; ++j) A[j + 1] = O[j + 1] | N[j + 1];
                uint64_t NG[6];
                for (int j = -1; j <= 4; ++j) NG[j + 1] = S.neg[r0 + j + 1];
                // contexts for this lane's two columns
                int cnt = 0;
                for (int cc = c0; cc <= c1; ++cc) {
                    if (cc >= c.cw) break;
                    for (int j = 0; j < 4; ++j) {
                        if (!((K[j] >> cc) & 1)) continue;
                        int w_ = bitat(A[j + 1], cc - 1), e_ = bitat(O[j + 1], cc + 1);
                        int n_ = bitat(A[j], cc), s_ = bitat(O[j + 2], cc);
                        int dd = bitat(A[j], cc - 1) + bitat(O[j], cc + 1) + bitat(A[j + 2], cc - 1) +
                                 bitat(O[j + 2], cc + 1);
                        int lab = zc_lut[orient][w_ + e_][n_ + s_][dd];
                        int bit = (int)((B[j] >> cc) & 1);
                        S.stage[lane][cnt++] = (uint8_t)(lab | (bit << 7));
                        if (bit) {
                            int hc = (w_ ? (bitat(NG[j + 1], cc - 1) ? -1 : 1) : 0) +
                                     (e_ ? (bitat(NG[j + 1], cc + 1) ? -1 : 1) : 0);
                            int vc = (n_ ? (bitat(NG[j], cc) ? -1 : 1) : 0) +
                                     (s_ ? (bitat(NG[j + 2], cc) ? -1 : 1) : 0);
                            int sc = sc_code(hc, vc);
                            int sgn = bitat(NG[j + 1], cc);
                            S.stage[lane][cnt++] = (uint8_t)((sc & 31) | ((sgn ^ (sc >> 7)) << 7));
                        }
                    }
                }
                __syncwarp();
                pos += flush_stage(S, lane, cnt, out, pos, cap, ovf);
                __syncwarp();
                if (lane == 0)
                    for (int j = 0; j < 4; ++j) {
                        S.sig[r0 + j + 1] = A[j + 1];
                        S.vis[r0 + j + 1] = K[j];
                    }
                __syncwarp();
            }
            if (lane == 0) pend[npass] = (uint32_t)pos;
            ++npass;
            // ------------------------- magnitude refinement pass
            for (int s = 0; s < nstripes && !ovf; ++s) {
                const int r0 = 4 * s;
                uint64_t SG[6], R[4], B[4], RF[4];
                for (int j = -1; j <= 4; ++j) SG[j + 1] = S.sig[r0 + j + 1];
                for (int j = 0; j < 4; ++j) {
                    R[j] = SG[j + 1] & ~S.vis[r0 + j + 1];
                    B[j] = plane_row(S, c, p, r0 + j, lane);
                    RF[j] = S.ref[r0 + j + 1];
                }
                int cnt = 0;
                for (int cc = c0; cc <= c1; ++cc) {
                    if (cc >= c.cw) break;
                    for (int j = 0; j < 4; ++j) {
                        if (!((R[j] >> cc) & 1)) continue;
                        int lab;
                        if ((RF[j] >> cc) & 1) lab = 16;
                        else {
                            uint64_t nb = dil(SG[j]) | dil(SG[j + 2]) | (SG[j + 1] << 1) | (SG[j + 1] >> 1);
                            lab = ((nb >> cc) & 1) ? 15 : 14;
                        }
                        S.stage[lane][cnt++] = (uint8_t)(lab | (int)(((B[j] >> cc) & 1) << 7));
                    }
                }
                __syncwarp();
                pos += flush_stage(S, lane, cnt, out, pos, cap, ovf);
                __syncwarp();
                if (lane == 0)
                    for (int j = 0; j < 4; ++j) S.ref[r0 + j + 1] = RF[j] | R[j];
                __syncwarp();
            }
            if (lane == 0) pend[npass] = (uint32_t)pos;
            ++npass;
        }
        // ------------------------- cleanup pass
        for (int s = 0; s < nstripes && !ovf; ++s) {
            const int r0 = 4 * s;
            const bool full = r0 + 3 < c.ch;
            uint64_t O[6], A[6], B[4], C[4], N[4], NG[6];
            for (int j = -1; j <= 4; ++j) {
                O[j + 1] = S.sig[r0 + j + 1];
                NG[j + 1] = S.neg[r0 + j + 1];
            }
            for (int j = 0; j < 4; ++j) {
                uint64_t V = (r0 + j < c.ch) ? colmask : 0;
                B[j] = plane_row(S, c, p, r0 + j, lane);
                C[j] = V & ~O[j + 1] & ~S.vis[r0 + j + 1];
                N[j] = C[j] & B[j];
            }
            A[0] = O[0];
            A[5] = O[5];
            for (int j = 0; j < 4; ++j) A[j + 1] = O[j + 1] | N[j];
            int cnt = 0;
            for (int cc = c0; cc <= c1; ++cc) {
                if (cc >= c.cw) break;
                int start = 0;
                if (full && ((C[0] & C[1] & C[2] & C[3]) >> cc) & 1) {
                    uint64_t lm = (cc > 0) ? (1ull << (cc - 1)) : 0;
                    uint64_t rm = (cc + 1 < 64) ? (1ull << (cc + 1)) : 0;
                    uint64_t cm = 1ull << cc;
                    bool quiet = !((A[1] | A[2] | A[3] | A[4]) & lm) && !((O[1] | O[2] | O[3] | O[4]) & rm) &&
                                 !((O[0] | O[5]) & (lm | cm | rm));
                    if (quiet) {
                        int first = -1;
                        for (int j = 0; j < 4; ++j)
                            if (first < 0 && ((N[j] >> cc) & 1)) first = j;
                        S.stage[lane][cnt++] = (uint8_t)(17 | ((first >= 0) << 7));
                        if (first < 0) continue;
                        S.stage[lane][cnt++] = (uint8_t)(18 | (((first >> 1) & 1) << 7));
                        S.stage[lane][cnt++] = (uint8_t)(18 | ((first & 1) << 7));
                        int j = first;
                        int w_ = bitat(A[j + 1], cc - 1), e_ = bitat(O[j + 1], cc + 1);
                        int n_ = bitat(A[j], cc), s_ = bitat(O[j + 2], cc);
                        int hc = (w_ ? (bitat(NG[j + 1], cc - 1) ? -1 : 1) : 0) +
                                 (e_ ? (bitat(NG[j + 1], cc + 1) ? -1 : 1) : 0);
                        int vc = (n_ ? (bitat(NG[j], cc) ? -1 : 1) : 0) +
                                 (s_ ? (bitat(NG[j + 2], cc) ? -1 : 1) : 0);
                        int sc = sc_code(hc, vc);
                        int sgn = bitat(NG[j + 1], cc);
                        S.stage[lane][cnt++] = (uint8_t)((sc & 31) | ((sgn ^ (sc >> 7)) << 7));
                        start = first + 1;
                    }
                }
                for (int j = start; j < 4; ++j) {
                    if (!((C[j] >> cc) & 1)) continue;
                    int w_ = bitat(A[j + 1], cc - 1), e_ = bitat(O[j + 1], cc + 1);
                    int n_ = bitat(A[j], cc), s_ = bitat(O[j + 2], cc);
                    int dd = bitat(A[j], cc - 1) + bitat(O[j], cc + 1) + bitat(A[j + 2], cc - 1) +
                             bitat(O[j + 2], cc + 1);
                    int lab = zc_lut[orient][w_ + e_][n_ + s_][dd];
                    int bit = (int)((B[j] >> cc) & 1);
                    S.stage[lane][cnt++] = (uint8_t)(lab | (bit << 7));
                    if (bit) {
                        int hc = (w_ ? (bitat(NG[j + 1], cc - 1) ? -1 : 1) : 0) +
                                 (e_ ? (bitat(NG[j + 1], cc + 1) ? -1 : 1) : 0);
                        int vc = (n_ ? (bitat(NG[j], cc) ? -1 : 1) : 0) +
                                 (s_ ? (bitat(NG[j + 2], cc) ? -1 : 1) : 0);
                        int sc = sc_code(hc, vc);
                        int sgn = bitat(NG[j + 1], cc);
                        S.stage[lane][cnt++] = (uint8_t)((sc & 31) | ((sgn ^ (sc >> 7)) << 7));
                    }
                }
            }
            __syncwarp();
            pos += flush_stage(S, lane, cnt, out, pos, cap, ovf);
            __syncwarp();
            if (lane == 0)
                for (int j = 0; j < 4; ++j) S.sig[r0 + j + 1] = A[j + 1];
            __syncwarp();
        }
        if (lane == 0) pend[npass] = (uint32_t)pos;
        ++npass;
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

constexpr int kMqThreads = 64;

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

template <int LANES>
__global__ void __launch_bounds__(kMqThreads)
t1_mq_kernel(const uint8_t* __restrict__ syms, size_t sym_cap, const uint32_t* __restrict__ nsyms,
             const uint32_t* __restrict__ order, int njobs, uint8_t* __restrict__ bytes,
             size_t cap_per_block, j2k_cb_desc* __restrict__ descs, uint32_t* __restrict__ err) {
    __shared__ uint32_t tab[47];
    __shared__ uint32_t cst[19 * kMqThreads];
    for (int i = threadIdx.x; i < 47; i += blockDim.x)
        tab[i] = (uint32_t)c_qe[i] | ((uint32_t)c_nmps[i] << 16) | ((uint32_t)c_nlps[i] << 22) |
                 ((uint32_t)(i == 0 || i == 6 || i == 14) << 28);
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane >= LANES) return;
    const int gid = (blockIdx.x * (kMqThreads / 32) + wid) * LANES + lane;
    if (gid >= njobs) return;
    const int jid = order ? (int)order[gid] : gid;
    const int t = threadIdx.x;
    uint32_t* st = cst + t;  // context k at st[k * kMqThreads]
    for (int k = 0; k < 19; ++k) st[k * kMqThreads] = tab[0];
    st[0] = tab[4];
    st[17 * kMqThreads] = tab[3];
    st[18 * kMqThreads] = tab[46];
    const int n = (int)min((size_t)nsyms[jid], sym_cap);
    MqEnc e;
    e.A = 0x8000;
    e.C = 0;
    e.B = 0;
    e.CT = 12;
    e.bp = -1;
    e.out = reinterpret_cast<uint32_t*>(bytes + (size_t)jid * cap_per_block);
    e.cap = (int)cap_per_block;
    e.wacc = 0;
    e.wn = 0;
    e.wbase = 0;
    e.ovf = false;
    // Symbols stream in 16-byte chunks with two chunks in flight per lane; the next symbol's
    // context state is loaded one step ahead and forwarded when the current symbol updates it.
    const uint4* sp4 = reinterpret_cast<const uint4*>(syms + (size_t)jid * sym_cap);
    const int nchunks = (n + 15) >> 4;
    const uint4 z4 = make_uint4(0, 0, 0, 0);
    uint4 c0 = nchunks > 0 ? __ldcs(sp4) : z4;
    uint4 c1 = nchunks > 1 ? __ldcs(sp4 + 1) : z4;
    int cx = min((int)(c0.x & 31), 18);
    uint32_t ent = st[cx * kMqThreads];
    for (int k = 0; k < nchunks; ++k) {
        const uint4 cur = c0;
        c0 = c1;
        c1 = (k + 2 < nchunks) ? __ldcs(sp4 + k + 2) : z4;
        const int m = min(16, n - 16 * k);
        const uint32_t w[5] = {cur.x, cur.y, cur.z, cur.w, c0.x};
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            if (j < m) {
                const uint32_t sym = (w[j >> 2] >> (8 * (j & 3))) & 0xFF;
                const uint32_t nsym = (w[(j + 1) >> 2] >> (8 * ((j + 1) & 3))) & 0xFF;
                const int d = sym >> 7;
                const int ncx = min((int)(nsym & 31), 18);
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
            }
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
        uint8_t* bb = bytes + (size_t)jid * cap_per_block;
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

__global__ void iota_kernel(uint32_t* v, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = (uint32_t)i;
}

}  // namespace

j2k_status j2k_t1_encode_jobs(j2k_ctx* ctx, const int32_t* coeff, size_t pitch,
                              const j2k_cb_job* d_jobs, size_t njobs, j2k_cb_desc* descs,
                              uint8_t* bytes, size_t cap_per_block, size_t sym_cap,
                              cudaStream_t st) {
    if (njobs == 0) return J2K_OK;
    if (cap_per_block % 16 != 0 || sym_cap % 16 != 0)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "t1: capacities must be multiples of 16");
    if (((uintptr_t)bytes & 15) != 0)
        return j2k_fail(ctx, J2K_ERR_INVALID_ARG, "t1: bytes buffer must be 16-byte aligned");
    uint8_t* syms = (uint8_t*)j2k_scratch(ctx, SCR_SYMS, njobs * sym_cap + 64);
    // meta: nsyms | pass ends (92 per job) | sort keys/values (4 arrays of njobs)
    size_t meta_words = njobs * (1 + 92 + 4) + 64;
    uint32_t* meta = (uint32_t*)j2k_scratch(ctx, SCR_T1STATE, meta_words * 4);
    if (!syms || !meta) return J2K_ERR_OUT_OF_MEMORY;
    uint32_t* nsyms = meta;
    uint32_t* pend = meta + njobs;
    uint32_t* keys_out = pend + njobs * 92;
    uint32_t* idx_in = keys_out + njobs;
    uint32_t* idx_out = idx_in + njobs;
    unsigned ga = (unsigned)((njobs + kWarpsPerCta - 1) / kWarpsPerCta);
    t1_symbols_kernel<<<ga, kWarpsPerCta * 32, 0, st>>>(coeff, pitch, d_jobs, (int)njobs, syms, sym_cap,
                                                        nsyms, pend, descs, cap_per_block, ctx->d_err);
    J2K_CUDA(ctx, cudaGetLastError());
    // longest-first order for the MQ lanes
    iota_kernel<<<(unsigned)((njobs + 255) / 256), 256, 0, st>>>(idx_in, (int)njobs);
    size_t tmp = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp, nsyms, keys_out, idx_in, idx_out, (int)njobs, 0, 32, st);
    void* tbuf = j2k_scratch(ctx, SCR_MISC, tmp + 16);
    if (!tbuf) return J2K_ERR_OUT_OF_MEMORY;
    J2K_CUDA(ctx, cub::DeviceRadixSort::SortPairsDescending(tbuf, tmp, nsyms, keys_out, idx_in, idx_out,
                                                            (int)njobs, 0, 32, st));
    const int lanes = ctx->mq_lanes;  // active lanes (blocks) per warp: 32, 16 or 8
    const size_t per_cta = (size_t)lanes * (kMqThreads / 32);
    unsigned gb = (unsigned)((njobs + per_cta - 1) / per_cta);
    if (lanes == 8)
        t1_mq_kernel<8><<<gb, kMqThreads, 0, st>>>(syms, sym_cap, nsyms, idx_out, (int)njobs, bytes, cap_per_block, descs, ctx->d_err);
    else if (lanes == 16)
        t1_mq_kernel<16><<<gb, kMqThreads, 0, st>>>(syms, sym_cap, nsyms, idx_out, (int)njobs, bytes, cap_per_block, descs, ctx->d_err);
    else
        t1_mq_kernel<32><<<gb, kMqThreads, 0, st>>>(syms, sym_cap, nsyms, idx_out, (int)njobs, bytes, cap_per_block, descs, ctx->d_err);
    J2K_CUDA(ctx, cudaGetLastError());
    return J2K_OK;
}
