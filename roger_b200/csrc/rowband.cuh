// Full-row band kernels of the 9/7 lifting (the differentiable 9/7 path).
//
// A level whose width W is a power of two in [64, 1024] is processed in bands of BH rows that
// span the whole width, one CTA per band and image:
//   - a warp holds one row as 32 lanes x SPL = W/32 consecutive samples in registers, so the
//     horizontal steps need two shuffles per step and no halo columns at all: the row ends are
//     the image edges, extended in registers (symmetric: the mirrored sample is the lane's own;
//     adjoint: the neighbour weights 0 outside, 2 at the boundary samples);
//   - a thread holds one column of the band plus 4 halo rows per side (NY = BH + 8 registers),
//     W / NT columns per thread, for the vertical steps;
//   - the two passes meet in shared memory, rows of W words whose 16-byte chunks are permuted
//     per lane (rb_swz) so that both the lanes' row loads and the threads' column accesses are
//     free of bank conflicts.
// Analysis shape (natural rows in, Mallat bands out; columns first): the forward level
// (MODE 3, symmetric) and the transpose of the inverse level (MODE 2, adjoint weights).
// Synthesis shape (Mallat bands in, natural rows out; rows first): the inverse level (MODE 0)
// and the transpose of the forward level (MODE 1).
// Every sample sees the same operations in the same order as in the strip kernels (lift.cuh,
// dwt.cu), so the results are bit-identical; the strip form wastes a fifth of a 1024-wide level
// on its 248-column tiles (half of a 512-wide one) and lifts 24 rows for 16.
//
// Fused epilogues (QB): the relaxed quantiser's forward (QB 1: coefficients y and their noise u
// written, rate partial sums per band) and backward (QB 2: the level's gradient g combined
// with y and u into dL/dy, log-step partial sums per band) run on the band samples a level has
// just produced, and the inverse's first loads (LQ) form y_hat = (y / step + u) * step from y
// and u, so the quantised plane is never written.
//
// Included inside the including file's anonymous namespace, after lift.cuh and philox4 /
// noise_of.

constexpr int RB_HV = 4;  // halo rows per side (four lifting steps)

template <int SPL>
struct RB {
    static constexpr int W = 32 * SPL;                // level width
    static constexpr int NT = 256;                    // threads per CTA (8 warps: 2 band rows each)
    static constexpr int NW = NT / 32;                // warps
    static constexpr int CPT = W >= NT ? W / NT : 1;  // columns per thread (narrow levels: threads < W)
};

// Shared-memory position of sample x of a row: lane l = x / SPL owns chunks 0..SPL/4-1 of its
// segment; chunk q is stored at q ^ s(l), s spreading the 8 lanes of a quarter-warp over the 8
// chunk slots of the 32 banks.
template <int SPL>
__device__ __forceinline__ int rb_swz(int x) {
    constexpr int C = SPL / 4;
    if constexpr (C < 2) {
        return x;
    } else {
        constexpr int SH = C == 8 ? 0 : (C == 4 ? 1 : 2);
        return x ^ ((((x / SPL) >> SH) & (C - 1)) << 2);
    }
}

template <int SPL>
__device__ __forceinline__ void rb_row_load(const float* row, int lane, float (&v)[SPL]) {
    if constexpr (SPL >= 4) {
#pragma unroll
        for (int q = 0; q < SPL / 4; ++q)
            *reinterpret_cast<float4*>(&v[4 * q]) = *reinterpret_cast<const float4*>(&row[rb_swz<SPL>(SPL * lane + 4 * q)]);
    } else {
        *reinterpret_cast<float2*>(&v[0]) = *reinterpret_cast<const float2*>(&row[SPL * lane]);
    }
}
template <int SPL>
__device__ __forceinline__ void rb_row_store(float* row, int lane, const float (&v)[SPL]) {
    if constexpr (SPL >= 4) {
#pragma unroll
        for (int q = 0; q < SPL / 4; ++q)
            *reinterpret_cast<float4*>(&row[rb_swz<SPL>(SPL * lane + 4 * q)]) = *reinterpret_cast<const float4*>(&v[4 * q]);
    } else {
        *reinterpret_cast<float2*>(&row[SPL * lane]) = *reinterpret_cast<const float2*>(&v[0]);
    }
}

// n consecutive floats (n a power of two), vector loads / stores where n allows
template <int N>
__device__ __forceinline__ void rb_gload(const float* p, float (&v)[N]) {
    if constexpr (N >= 4) {
#pragma unroll
        for (int q = 0; q < N / 4; ++q) *reinterpret_cast<float4*>(&v[4 * q]) = __ldcg(reinterpret_cast<const float4*>(p) + q);
    } else if constexpr (N == 2) {
        *reinterpret_cast<float2*>(&v[0]) = __ldcg(reinterpret_cast<const float2*>(p));
    } else {
        v[0] = __ldcg(p);
    }
}
template <int N>
__device__ __forceinline__ void rb_gstore(float* p, const float (&v)[N]) {
    if constexpr (N >= 4) {
#pragma unroll
        for (int q = 0; q < N / 4; ++q) reinterpret_cast<float4*>(p)[q] = *reinterpret_cast<const float4*>(&v[4 * q]);
    } else if constexpr (N == 2) {
        *reinterpret_cast<float2*>(p) = *reinterpret_cast<const float2*>(&v[0]);
    } else {
        p[0] = v[0];
    }
}

// Horizontal steps of one full row (lane l holds x = SPL*l .. SPL*l + SPL-1, the row is W wide).
// MODE 3: forward; 0: inverse; 1: transpose of the forward; 2: transpose of the inverse.
template <int MODE, int SPL>
__device__ __forceinline__ void rb_hlift(float (&v)[SPL], int lane) {
    const bool first = lane == 0, last = lane == 31;
    if constexpr (MODE == 3) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if ((k & 1) == 0) {  // odd samples from their even neighbours; x = W mirrors to W - 2
                float nx = __shfl_down_sync(0xffffffffu, v[0], 1);
                if (last) nx = v[SPL - 2];
#pragma unroll
                for (int j = 1; j < SPL; j += 2) v[j] = KT<97>::op(false, k, v[j], v[j - 1], j + 1 < SPL ? v[j + 1] : nx);
            } else {             // even samples from their odd neighbours; x = -1 mirrors to 1
                float pv = __shfl_up_sync(0xffffffffu, v[SPL - 1], 1);
                if (first) pv = v[1];
#pragma unroll
                for (int j = 0; j < SPL; j += 2) v[j] = KT<97>::op(false, k, v[j], j ? v[j - 1] : pv, v[j + 1]);
            }
        }
#pragma unroll
        for (int j = 0; j < SPL; ++j) v[j] = __fmul_rn(v[j], (j & 1) ? KMUL : KDIV);
    } else if constexpr (MODE == 0) {
#pragma unroll
        for (int j = 0; j < SPL; ++j) v[j] = __fmul_rn(v[j], (j & 1) ? KDIV : KMUL);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if ((k & 1) == 0) {  // even samples from their odd neighbours
                float pv = __shfl_up_sync(0xffffffffu, v[SPL - 1], 1);
                if (first) pv = v[1];
#pragma unroll
                for (int j = 0; j < SPL; j += 2) v[j] = KT<97>::op(true, k, v[j], j ? v[j - 1] : pv, v[j + 1]);
            } else {             // odd samples from their even neighbours
                float nx = __shfl_down_sync(0xffffffffu, v[0], 1);
                if (last) nx = v[SPL - 2];
#pragma unroll
                for (int j = 1; j < SPL; j += 2) v[j] = KT<97>::op(true, k, v[j], v[j - 1], j + 1 < SPL ? v[j + 1] : nx);
            }
        }
    } else {
        constexpr bool FADJ = MODE == 1;
        if constexpr (FADJ) {
#pragma unroll
            for (int j = 0; j < SPL; ++j) v[j] = __fmul_rn(v[j], (j & 1) ? KMUL : KDIV);
        }
        // neighbour weights that differ from 1: x = -1 and x = W (0), x = 0 and x = W-1 (2)
        const float w_out_l = first ? 0.0f : 1.0f, w_out_r = last ? 0.0f : 1.0f;
        const float w_b0 = first ? 2.0f : 1.0f, w_bn = last ? 2.0f : 1.0f;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float c = adj_coef<FADJ>(k);
            if (adj_par<FADJ>(k) == 0) {  // even samples
                const float pv = __shfl_up_sync(0xffffffffu, v[SPL - 1], 1);
#pragma unroll
                for (int j = 0; j < SPL; j += 2) {
                    const float a = j ? v[j - 1] : __fmul_rn(pv, w_out_l);
                    const float b = j == SPL - 2 ? __fmul_rn(v[j + 1], w_bn) : v[j + 1];
                    v[j] = adj_op(c, v[j], a, b);
                }
            } else {                      // odd samples
                const float nx = __shfl_down_sync(0xffffffffu, v[0], 1);
#pragma unroll
                for (int j = 1; j < SPL; j += 2) {
                    const float a = j == 1 ? __fmul_rn(v[0], w_b0) : v[j - 1];
                    const float b = j + 1 < SPL ? v[j + 1] : __fmul_rn(nx, w_out_r);
                    v[j] = adj_op(c, v[j], a, b);
                }
            }
        }
        if constexpr (!FADJ) {
#pragma unroll
            for (int j = 0; j < SPL; ++j) v[j] = __fmul_rn(v[j], (j & 1) ? KDIV : KMUL);
        }
    }
}

// Forward vertical steps of one column (c[r] at absolute row ys + r, ys even), as in the strip
// kernels: step k updates the rows of parity 1 - (k & 1) over the range that stays exact.
template <int NY>
__device__ __forceinline__ void rb_vfwd(float (&c)[NY]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int par = 1 - (k & 1);
#pragma unroll
        for (int r = k + 1; r < NY - k - 1; ++r)
            if ((r & 1) == par) c[r] = KT<97>::op(false, k, c[r], c[r - 1], c[r + 1]);
    }
}

// Operands of the fused quantiser epilogues and loads.
struct RbQ {
    const float* log_steps;  // per QCD band (3L + 1): LL, then HL, LH, HH from the deepest level
    uint64_t seed;           // Philox key = seed + image
    float* u;                // noise plane (Mallat layout and strides of the coefficients)
    const float* y;          // QB 2: the coefficients
    float lam;               // rate weight
    const float* gscale;     // QB 2: the incoming gradient is scaled by (*gscale) * alpha
    float alpha;
    float* part;             // partial sums [image][band][kp]
    int kp;                  // partial slots per image and band
    int levels;              // L
    int level;               // this level (0 = finest)
    int groups;              // Philox counters per Mallat row: ceil(w0 / 4)
};

// Steps and reciprocal steps of every band, as the quantiser kernels form them.
__device__ __forceinline__ void rb_load_steps(const RbQ& q, float* stp, float* rstp) {
    const int nb = 3 * q.levels + 1;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        stp[b] = expf(q.log_steps[b]);
        rstp[b] = __frcp_rn(stp[b]);
    }
}

// One run of N band samples (N a power of two) that a level has produced at Mallat (row, col0)
// of band b, written to p (off: their element offset in the plane, for the y and u planes).
// QB 0: stored as they are.  QB 1 (quantiser forward): stored with their noise u (Philox4x32-10
// keyed by seed + image, counter row * groups + col / 4, word col % 4, as relaxed_quant_k draws
// it); acc += log2(1 + |val / step + u|).  QB 2 (quantiser backward): val is the gradient with
// respect to y_hat and yy, uu the coefficients and noise at the same positions (loaded by the
// caller); dL/dy = G val + drate/dt / step is stored and the log-step partial goes to acc.
template <int QB, int N>
__device__ __forceinline__ void rb_put(float* p, size_t off, const float (&val)[N], int row, int col0, int b,
                                       const RbQ& q, const float* stp, const float* rstp, uint64_t key, float G,
                                       float lamG, float& acc, const float* yy, const float* uu) {
    if constexpr (QB == 0) {
        rb_gstore<N>(p, val);
    } else if constexpr (QB == 1) {
        const float rs = rstp[b];
#pragma unroll
        for (int g = 0; g < (N + 3) / 4; ++g) {  // one Philox call per group of 4 columns
            constexpr int M = N < 4 ? N : 4;
            uint32_t o[4];
            philox4(key, (uint64_t)row * q.groups + (uint64_t)((col0 + 4 * g) >> 2), o);
            float uu[M], vv[M];
#pragma unroll
            for (int i = 0; i < M; ++i) {
                const int k = (col0 + 4 * g + i) & 3;
                uu[i] = noise_of(k == 0 ? o[0] : k == 1 ? o[1] : k == 2 ? o[2] : o[3]);
                vv[i] = val[4 * g + i];
                const float tt = __fadd_rn(__fmul_rn(vv[i], rs), uu[i]);
                acc += __log2f(__fadd_rn(1.0f, fabsf(tt)));
            }
            rb_gstore<M>(p + 4 * g, vv);
            rb_gstore<M>(q.u + off + 4 * g, uu);
        }
    } else {
        const float step = stp[b], rs = rstp[b];
        const float inv_ln2 = 1.4426950408889634f;
        float o[N];
#pragma unroll
        for (int i = 0; i < N; ++i) {
            const float tt = __fadd_rn(__fmul_rn(yy[i], rs), uu[i]);
            const float sg = tt > 0.0f ? 1.0f : (tt < 0.0f ? -1.0f : 0.0f);
            const float drdt = __fdividef(lamG * inv_ln2 * sg, 1.0f + fabsf(tt));
            const float gg = __fmul_rn(G, val[i]);
            o[i] = __fadd_rn(gg, __fmul_rn(drdt, rs));
            acc += gg * uu[i] * step - drdt * yy[i] * rs;
        }
        rb_gstore<N>(p, o);
    }
}

constexpr int RB_BH = 16;  // rows per band

// ---- analysis shape: natural rows in, Mallat bands out -------------------------------------------
// MODE 3: forward level (symmetric extension); MODE 2: transpose of the inverse level (zero
// extension, adjoint weights).  Grid (bands, images).  The level's HL/LH/HH go to their Mallat
// positions in dst, its LL to lld (last: lld is dst itself and the LL is a band of the plane,
// which the QB epilogue then covers too).  Dynamic shared memory: BH rows of W floats.
template <int MODE, int SPL, int QB>
__global__ void __launch_bounds__(RB<SPL>::NT, SPL >= 32 ? (QB == 2 ? 2 : 3) : (SPL == 16 ? (QB == 2 ? 2 : 3) : 4))
rb_ana(const float* __restrict__ in, size_t ipitch, size_t iz, int h, float* __restrict__ dst, size_t dpitch,
       size_t dz, float* __restrict__ lld, size_t llpitch, size_t llz, int last, RbQ q) {
    using G = RB<SPL>;
    constexpr int W = G::W, BH = RB_BH, NY = BH + 2 * RB_HV, H2 = SPL / 2;
    extern __shared__ float4 rb_dyn[];
    float* rbs = reinterpret_cast<float*>(rb_dyn);
    __shared__ float stp[49], rstp[49], red[G::NW][2];
    griddep_launch_dependents();
    griddep_wait();  // launched as a dependent: the previous level's writes are visible from here
    const int t = threadIdx.x, lane = t & 31, wp = t >> 5, img = blockIdx.y;
    const int y0 = blockIdx.x * BH;
    if constexpr (QB != 0) rb_load_steps(q, stp, rstp);
    in += img * iz;
    dst += img * dz;
    lld += img * llz;
    if constexpr (QB != 0) q.u += img * dz;  // the noise and coefficient planes have dst's layout
    if constexpr (QB == 2) q.y += img * dz;
    // 1. the band's columns, 4 halo rows per side, lifted vertically in registers
    const bool inner = y0 - RB_HV >= 0 && y0 + BH + RB_HV <= h;
    auto load_col = [&](int x, float (&c)[NY]) {
        const float* colp = in + x;
#pragma unroll
        for (int r = 0; r < NY; ++r) {
            const int gy = y0 - RB_HV + r;
            if constexpr (MODE == 3) c[r] = __ldcg(colp + (size_t)(inner ? gy : mirror(gy, h)) * ipitch);
            else c[r] = (inner || (gy >= 0 && gy < h)) ? __ldcg(colp + (size_t)gy * ipitch) : 0.0f;
        }
    };
    auto lift_store = [&](int x, float (&c)[NY]) {
        if (h > 1) {
            if constexpr (MODE == 3) {
                rb_vfwd<NY>(c);
            } else {
                const int ys = y0 - RB_HV;
                if (!(ys > 0 && y0 + BH + RB_HV - 1 < h - 1)) vlift<97, 2, true, NY>(c, ys, h);
                else vlift<97, 2, false, NY>(c, ys, h);
            }
        }
#pragma unroll
        for (int r = 0; r < BH; ++r) {
            float v = c[RB_HV + r];
            if (MODE == 3 && h > 1) v = __fmul_rn(v, (r & 1) ? KMUL : KDIV);
            rbs[r * W + rb_swz<SPL>(x)] = v;
        }
    };
    if (W >= G::NT || t < W) {
        // one column at a time: its NY loads are in flight together (loading the next column
        // during the lifting measured slower: register pressure at three CTAs per SM)
#pragma unroll 1
        for (int j = 0; j < G::CPT; ++j) {
            const int x = t + G::NT * j;
            float c[NY];
            load_col(x, c);
            lift_store(x, c);
        }
    }
    __syncthreads();
    // 2. rows: warp wp takes rows wp, wp + NW, ... (all of one parity: NW is even)
    const int wl = W / 2, hl = (h + 1) >> 1;
    const uint64_t key = q.seed + (uint64_t)img;
    float G2 = 1.0f, lamG = q.lam;
    if constexpr (QB == 2) {
        const float s = q.gscale ? *q.gscale : 1.0f;
        G2 = __fmul_rn(s, q.alpha);
        lamG = __fmul_rn(s, q.lam);
    }
    const int bt = 1 + 3 * (q.levels - (q.level + 1));  // this level's HL; LH = bt + 1, HH = bt + 2
    const int bx = H2 * lane;
    float acc_lo = 0.0f, acc_hi = 0.0f;
#pragma unroll 1
    for (int r = wp; r < BH; r += G::NW) {
        const int y = y0 + r;
        if (y >= h) break;
        float v[SPL];
        rb_row_load<SPL>(rbs + r * W, lane, v);
        const int qy = y & 1, sy = (y >> 1) + (qy ? hl : 0);
        const size_t so = (size_t)sy * dpitch;
        // QB 2: the row's coefficients and noise, loaded before the lifting hides their latency
        constexpr int NQ = QB == 2 ? H2 : 1;
        float ylo[NQ], ulo[NQ], yhi[NQ], uhi[NQ];
        if constexpr (QB == 2) {
            rb_gload<H2>(q.y + so + wl + bx, yhi);
            rb_gload<H2>(q.u + so + wl + bx, uhi);
            if (qy || last) {
                rb_gload<H2>(q.y + so + bx, ylo);
                rb_gload<H2>(q.u + so + bx, ulo);
            }
        }
        rb_hlift<MODE, SPL>(v, lane);
        float lo[H2], hi[H2];
#pragma unroll
        for (int i = 0; i < H2; ++i) {
            lo[i] = v[2 * i];
            hi[i] = v[2 * i + 1];
        }
        if (qy) {
            rb_put<QB, H2>(dst + so + bx, so + bx, lo, sy, bx, bt + 1, q, stp, rstp, key, G2, lamG, acc_lo, ylo,
                           ulo);
            rb_put<QB, H2>(dst + so + wl + bx, so + wl + bx, hi, sy, wl + bx, bt + 2, q, stp, rstp, key, G2, lamG,
                           acc_hi, yhi, uhi);
        } else {
            if (QB != 0 && last)
                rb_put<QB, H2>(dst + so + bx, so + bx, lo, sy, bx, 0, q, stp, rstp, key, G2, lamG, acc_lo, ylo, ulo);
            else
                rb_put<0, H2>(lld + (size_t)(y >> 1) * llpitch + bx, 0, lo, 0, 0, 0, q, stp, rstp, key, G2, lamG,
                              acc_lo, lo, lo);
            rb_put<QB, H2>(dst + so + wl + bx, so + wl + bx, hi, sy, wl + bx, bt, q, stp, rstp, key, G2, lamG,
                           acc_hi, yhi, uhi);
        }
    }
    if constexpr (QB != 0) {
        // per band of this CTA, in a fixed order: lanes by a butterfly, then warps in index order
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            acc_lo += __shfl_xor_sync(0xffffffffu, acc_lo, o);
            acc_hi += __shfl_xor_sync(0xffffffffu, acc_hi, o);
        }
        if (lane == 0) {
            red[wp][0] = acc_lo;
            red[wp][1] = acc_hi;
        }
        __syncthreads();
        if (t < 4 && (t != 0 || last)) {  // 0: LL (last level), 1: HL, 2: LH, 3: HH
            const int par = t >> 1, half = t & 1;
            float a = 0.0f;
            for (int w2 = par; w2 < G::NW; w2 += 2) a += red[w2][half];
            const int b = t == 0 ? 0 : bt + t - 1;
            q.part[((size_t)img * (3 * q.levels + 1) + b) * q.kp + blockIdx.x] = a;
        }
    }
}

// ---- synthesis shape: Mallat bands in, natural rows out ------------------------------------------
// MODE 0: inverse level (symmetric extension); MODE 1: transpose of the forward level (zero
// extension, adjoint weights).  The level's details are at their Mallat positions in src, its LL
// in lls (deepest: lls is src itself).  LQ (MODE 0): the details, and the LL of the deepest
// level, are coefficients y with noise u (q.u, the layout of src) and enter as
// y_hat = (y / step + u) * step.  EXTRA as in dwt_syn_fast: 1 out = result - sub and the CTA's sum
// of out^2 to ex.part[image * bands + band]; 2 out = result - (*scale) * alpha * sub.
// Dynamic shared memory: BH + 8 rows of W floats.
template <int MODE, int SPL, bool LQ, int EXTRA>
__global__ void __launch_bounds__(RB<SPL>::NT, SPL >= 32 ? 2 : (SPL == 16 ? 3 : 4))
rb_syn(const float* __restrict__ src, size_t spitch, size_t sz, const float* __restrict__ lls, size_t llpitch,
       size_t llz, int h, float* __restrict__ out, size_t opitch, size_t oz, SynExtra ex, RbQ q, int deepest) {
    using G = RB<SPL>;
    constexpr int W = G::W, BH = RB_BH, NY = BH + 2 * RB_HV, H2 = SPL / 2;
    extern __shared__ float4 rb_dyn[];
    float* rbs = reinterpret_cast<float*>(rb_dyn);
    __shared__ float stp[49], rstp[49], red[G::NW];
    griddep_launch_dependents();
    griddep_wait();  // launched as a dependent: the previous level's writes are visible from here
    const int t = threadIdx.x, lane = t & 31, wp = t >> 5, img = blockIdx.y;
    const int y0 = blockIdx.x * BH;
    if constexpr (LQ) {
        rb_load_steps(q, stp, rstp);
        __syncthreads();
    }
    src += img * sz;
    lls += img * llz;
    out += img * oz;
    const float* up = LQ ? q.u + img * sz : nullptr;
    const int wl = W / 2, hl = (h + 1) >> 1;
    const int bt = 1 + 3 * (q.levels - (q.level + 1));
    const int bx = H2 * lane;
    // 1. the band's rows and 4 halo rows per side (mirrored, or zero outside for MODE 1),
    //    lifted horizontally in registers, natural order into shared memory
#pragma unroll
    for (int r = wp; r < NY; r += G::NW) {
        int gy = y0 - RB_HV + r;
        bool zero = false;
        if (MODE == 0) gy = mirror(gy, h);
        else zero = gy < 0 || gy >= h;
        float v[SPL];
        if (zero) {
#pragma unroll
            for (int j = 0; j < SPL; ++j) v[j] = 0.0f;
        } else {
            const int qy = gy & 1;
            const size_t so = (size_t)((gy >> 1) + (qy ? hl : 0)) * spitch;
            float lo[H2], hi[H2];
            if (qy) rb_gload<H2>(src + so + bx, lo);
            else rb_gload<H2>(lls + (size_t)(gy >> 1) * llpitch + bx, lo);
            rb_gload<H2>(src + so + wl + bx, hi);
            if constexpr (LQ) {
                float u[H2];
                rb_gload<H2>(up + so + wl + bx, u);
                const int bh = qy ? bt + 2 : bt;
#pragma unroll
                for (int i = 0; i < H2; ++i)
                    hi[i] = __fmul_rn(__fadd_rn(__fmul_rn(hi[i], rstp[bh]), u[i]), stp[bh]);
                if (qy || deepest) {
                    rb_gload<H2>(up + so + bx, u);
                    const int bl = qy ? bt + 1 : 0;
#pragma unroll
                    for (int i = 0; i < H2; ++i)
                        lo[i] = __fmul_rn(__fadd_rn(__fmul_rn(lo[i], rstp[bl]), u[i]), stp[bl]);
                }
            }
#pragma unroll
            for (int i = 0; i < H2; ++i) {
                v[2 * i] = lo[i];
                v[2 * i + 1] = hi[i];
            }
            rb_hlift<MODE, SPL>(v, lane);
        }
        rb_row_store<SPL>(rbs + r * W, lane, v);
    }
    __syncthreads();
    // 2. columns: vertical steps in registers, natural-order writes
    float sq = 0.0f, sc = 0.0f;
    if constexpr (EXTRA == 2) sc = __fmul_rn(ex.scale ? *ex.scale : 1.0f, ex.alpha);
    const float* __restrict__ sub = EXTRA != 0 ? ex.sub + img * ex.sub_z : nullptr;
    // the residual operand of a column, fetched one column ahead
    float sb[EXTRA != 0 ? BH : 1], sbn[EXTRA != 0 ? BH : 1];
    auto load_sub = [&](int x, float* d) {
#pragma unroll
        for (int i = 0; i < BH; ++i) d[i] = y0 + i < h ? __ldcg(sub + (size_t)(y0 + i) * ex.sub_pitch + x) : 0.0f;
    };
    if (EXTRA != 0 && (W >= G::NT || t < W)) load_sub(t, sb);
#pragma unroll 1
    for (int j = 0; j < G::CPT; ++j) {
        const int x = t + G::NT * j;
        if (W < G::NT && t >= W) break;
        if (EXTRA != 0 && j + 1 < G::CPT) load_sub(x + G::NT, sbn);
        float c[NY];
#pragma unroll
        for (int r = 0; r < NY; ++r) c[r] = rbs[r * W + rb_swz<SPL>(x)];
        if (h > 1) {
            const int ys = y0 - RB_HV;
            if constexpr (MODE == 1) {
                if (!(ys > 0 && y0 + BH + RB_HV - 1 < h - 1)) vlift<97, 1, true, NY>(c, ys, h);
                else vlift<97, 1, false, NY>(c, ys, h);
            } else {
                vlift<97, 0, false, NY>(c, ys, h);
            }
        }
#pragma unroll
        for (int i = 0; i < BH; ++i) {
            const int y = y0 + i;
            if (y < h) {
                float v = c[RB_HV + i];
                if constexpr (EXTRA == 1) {
                    v = __fsub_rn(v, sb[i]);
                    sq = __fmaf_rn(v, v, sq);
                } else if constexpr (EXTRA == 2) {
                    v = __fsub_rn(v, __fmul_rn(sc, sb[i]));
                }
                out[(size_t)y * opitch + x] = v;
            }
        }
        if constexpr (EXTRA != 0) {
#pragma unroll
            for (int i = 0; i < BH; ++i) sb[i] = sbn[i];
        }
    }
    if constexpr (EXTRA == 1) {
#pragma unroll
        for (int o = 16; o; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
        if (lane == 0) red[wp] = sq;
        __syncthreads();
        // slot layout of the strip kernel's tiles (ceil(w / 248) per 16 rows): this CTA's sum in
        // the first of its part_stride slots, zeros in the others
        const int ps = ex.part_stride > 0 ? ex.part_stride : 1;
        if (t < ps) {
            float a = 0.0f;
            if (t == 0) {
#pragma unroll
                for (int i = 0; i < G::NW; ++i) a += red[i];
            }
            ex.part[((size_t)img * gridDim.x + blockIdx.x) * ps + t] = a;
        }
    }
}
