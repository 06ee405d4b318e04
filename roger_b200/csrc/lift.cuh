// Shared pieces of the lifting kernels: 9/7 constants, whole-sample symmetric extension, the
// 5/3 and 9/7 step traits, the dead-zone (de)quantiser, and the register-lifting strip kernels
// that run the synthesis shape (Mallat bands in, natural order out: the inverse DWT and the
// transpose of the forward DWT) and the analysis shape of the transpose of the inverse DWT.
//
// Strip geometry (all register kernels): a CTA of 256 threads owns a 248-column x 16-row tile
// of the level's output and stages a 256-column x (16 + 2*HV)-row strip in shared memory
// (4 columns of halo on each side, HV = 2 rows for 5/3, 4 for 9/7).  Horizontal lifting runs
// with 8 samples per lane and warp shuffles for the neighbours; vertical lifting runs with one
// thread per column and the whole column in registers.  Each lifting step consumes one sample
// of halo per side, so 4 columns / HV rows suffice for the 2 (5/3) or 4 (9/7) steps.
#pragma once

#include "j2k_internal.cuh"

namespace {

constexpr float P1 = -1.586134342f, U1 = -0.05298011854f, P2 = 0.8829110762f, U2 = 0.4435068522f;
constexpr float KMUL = 1.23017410491400f, KDIV = 0.81289306611596153187273657637352f;

// whole-sample symmetric extension (period 2(n-1)), parity preserving
__device__ __forceinline__ int mirror(int i, int n) {
    if (i >= 0 && i < n) return i;
    if (n == 1) return 0;
    const int p = 2 * (n - 1);
    i %= p;
    if (i < 0) i += p;
    return i >= n ? p - i : i;
}

template <int KERN> struct KT;
template <> struct KT<53> {
    using T = int32_t;
    static constexpr int H = 2, NSTEP = 2;
    __device__ static int par(bool inv, int s) { return inv ? (s & 1) : 1 - (s & 1); }
    __device__ static T op(bool inv, int s, T x, T a, T b) {
        if (!inv) return s == 0 ? x - ((a + b) >> 1) : x + ((a + b + 2) >> 2);
        return s == 0 ? x - ((a + b + 2) >> 2) : x + ((a + b) >> 1);
    }
};
template <> struct KT<97> {
    using T = float;
    static constexpr int H = 4, NSTEP = 4;
    __device__ static int par(bool inv, int s) { return inv ? (s & 1) : 1 - (s & 1); }
    __device__ static T op(bool inv, int s, T x, T a, T b) {
        float c;
        if (!inv) c = s == 0 ? P1 : (s == 1 ? U1 : (s == 2 ? P2 : U2));
        else c = s == 0 ? -U2 : (s == 1 ? -P2 : (s == 2 ? -U1 : -P1));
        return __fadd_rn(x, __fmul_rn(c, __fadd_rn(a, b)));
    }
};

__device__ __forceinline__ int32_t quantize(float v, float step) {
    int32_t m = (int32_t)floorf(__fdiv_rn(fabsf(v), step));
    return v < 0.0f ? -m : m;
}
__device__ __forceinline__ float dequantize(int32_t q, float step) {
    int32_t m = q < 0 ? -q : q;
    float r = m ? __fmul_rn(__fadd_rn((float)m, 0.5f), step) : 0.0f;
    return q < 0 ? -r : r;
}

template <typename T>
__device__ __forceinline__ T bits_as(uint32_t u) {
    if constexpr (sizeof(T) == 4 && T(0.5f) != T(0)) return __uint_as_float(u);
    else return (T)(int32_t)u;
}

struct Steps4 { float ll, hl, lh, hh; };
// element strides between consecutive images of a batch (blockIdx.z selects the image)
struct ZStride { size_t src, dst, ll; };

constexpr int FTW = 248, FNX = 256, STH = 16;

// asynchronous global -> shared copies (sm_80+ cp.async), waited for with cp_async_wait_all
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Programmatic dependent launch (sm_90+): a level kernel lets the next level's grid be launched
// while its own CTAs still run, and waits for the previous level's grid (its writes visible)
// before it reads that level's output.  Both are no-ops for a kernel launched without the
// programmatic-serialisation attribute.
__device__ __forceinline__ void griddep_launch_dependents() {
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

// Launches k<<<g, b, 0, s>>>(args...); with pdl, as a programmatic dependent of the previous
// kernel on the stream (cudaLaunchAttributeProgrammaticStreamSerialization).
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl_smem(void (*k)(KArgs...), dim3 g, dim3 b, size_t smem, cudaStream_t s, bool pdl,
                            Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = g;
    cfg.blockDim = b;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = pdl ? at : nullptr;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, k, args...);
}
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*k)(KArgs...), dim3 g, dim3 b, cudaStream_t s, bool pdl, Args... args) {
    return launch_pdl_smem(k, g, b, 0, s, pdl, args...);
}

// ---- transposed 9/7 steps -----------------------------------------------------------------------
// A forward step updates parity p: x_i += c (x_m(i-1) + x_m(i+1)), m = symmetric mirror.  Its
// transpose updates the other parity with the same coefficient from the neighbours weighted by
// adj_w: 0 outside [0, n), 2 for the boundary samples 0 and n-1 (the mirrored references fold
// back onto them), 1 elsewhere.  Sequences (step k: parity updated, coefficient):
//   transpose of the forward (after the forward scaling): odd U2, even P2, odd U1, even P1
//   transpose of the inverse (then the inverse scaling):  even -P1, odd -U1, even -P2, odd -U2
__device__ __forceinline__ float adj_w(int k, int n) {
    return (k < 0 || k >= n) ? 0.0f : ((k == 0 || k == n - 1) ? 2.0f : 1.0f);
}
template <bool FADJ>
__device__ __forceinline__ constexpr float adj_coef(int k) {
    return FADJ ? (k == 0 ? U2 : k == 1 ? P2 : k == 2 ? U1 : P1) : (k == 0 ? -P1 : k == 1 ? -U1 : k == 2 ? -P2 : -U2);
}
template <bool FADJ>
__device__ __forceinline__ constexpr int adj_par(int k) {  // parity updated by step k
    return FADJ ? ((k & 1) ? 0 : 1) : (k & 1);
}
__device__ __forceinline__ float adj_op(float c, float x, float a, float b) {
    return __fadd_rn(x, __fmul_rn(c, __fadd_rn(a, b)));
}

// Horizontal steps of one strip row held as 8 consecutive samples per lane (v[j] at absolute
// x = xs + j, xs even).  MODE 0: inverse 5/3 or 9/7 (scaling first); 1: transpose of the
// forward 9/7 (forward scaling first); 2: transpose of the inverse 9/7 (inverse scaling last).
// EDGE: apply the adjoint boundary weights (only tiles touching the image edge need them).
template <int KERN, int MODE, bool EDGE>
__device__ __forceinline__ void hlift8(typename KT<KERN>::T (&v)[8], int xs, int n) {
    using T = typename KT<KERN>::T;
    if constexpr (MODE == 0) {
        if constexpr (KERN == 97) {
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = __fmul_rn(v[j], (j & 1) ? KDIV : KMUL);
        }
#pragma unroll
        for (int k = 0; k < KT<KERN>::NSTEP; ++k) {
            if ((k & 1) == 0) {  // even samples from their odd neighbours
                const T pv = __shfl_up_sync(0xffffffffu, v[7], 1);
                v[0] = KT<KERN>::op(true, k, v[0], pv, v[1]);
                v[2] = KT<KERN>::op(true, k, v[2], v[1], v[3]);
                v[4] = KT<KERN>::op(true, k, v[4], v[3], v[5]);
                v[6] = KT<KERN>::op(true, k, v[6], v[5], v[7]);
            } else {             // odd samples from their even neighbours
                const T nx = __shfl_down_sync(0xffffffffu, v[0], 1);
                v[1] = KT<KERN>::op(true, k, v[1], v[0], v[2]);
                v[3] = KT<KERN>::op(true, k, v[3], v[2], v[4]);
                v[5] = KT<KERN>::op(true, k, v[5], v[4], v[6]);
                v[7] = KT<KERN>::op(true, k, v[7], v[6], nx);
            }
        }
    } else {
        constexpr bool FADJ = MODE == 1;
        if constexpr (FADJ) {
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = __fmul_rn(v[j], (j & 1) ? KMUL : KDIV);
        }
        float wt[10];  // weights of absolute positions xs-1 .. xs+8
        if constexpr (EDGE) {
#pragma unroll
            for (int j = 0; j < 10; ++j) wt[j] = adj_w(xs - 1 + j, n);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float c = adj_coef<FADJ>(k);
            if (adj_par<FADJ>(k) == 0) {
                float pv = __shfl_up_sync(0xffffffffu, v[7], 1);
                if constexpr (EDGE) {
#pragma unroll
                    for (int j = 0; j < 8; j += 2) {
                        const float a = __fmul_rn(j ? v[j - 1] : pv, wt[j]), b = __fmul_rn(v[j + 1], wt[j + 2]);
                        v[j] = adj_op(c, v[j], a, b);
                    }
                } else {
                    v[0] = adj_op(c, v[0], pv, v[1]);
                    v[2] = adj_op(c, v[2], v[1], v[3]);
                    v[4] = adj_op(c, v[4], v[3], v[5]);
                    v[6] = adj_op(c, v[6], v[5], v[7]);
                }
            } else {
                float nx = __shfl_down_sync(0xffffffffu, v[0], 1);
                if constexpr (EDGE) {
#pragma unroll
                    for (int j = 1; j < 8; j += 2) {
                        const float a = __fmul_rn(v[j - 1], wt[j]), b = __fmul_rn(j < 7 ? v[j + 1] : nx, wt[j + 2]);
                        v[j] = adj_op(c, v[j], a, b);
                    }
                } else {
                    v[1] = adj_op(c, v[1], v[0], v[2]);
                    v[3] = adj_op(c, v[3], v[2], v[4]);
                    v[5] = adj_op(c, v[5], v[4], v[6]);
                    v[7] = adj_op(c, v[7], v[6], nx);
                }
            }
        }
        if constexpr (!FADJ) {
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = __fmul_rn(v[j], (j & 1) ? KDIV : KMUL);
        }
    }
}

// Vertical steps of one column held in registers (c[r] at absolute row ys + r, ys even).
template <int KERN, int MODE, bool EDGE, int NY>
__device__ __forceinline__ void vlift(typename KT<KERN>::T (&c)[NY], int ys, int n) {
    if constexpr (MODE == 0) {
        if constexpr (KERN == 97) {
#pragma unroll
            for (int r = 0; r < NY; ++r) c[r] = __fmul_rn(c[r], (r & 1) ? KDIV : KMUL);
        }
#pragma unroll
        for (int k = 0; k < KT<KERN>::NSTEP; ++k) {
#pragma unroll
            for (int r = k + 1; r < NY - k - 1; ++r)
                if ((r & 1) == (k & 1)) c[r] = KT<KERN>::op(true, k, c[r], c[r - 1], c[r + 1]);
        }
    } else {
        constexpr bool FADJ = MODE == 1;
        if constexpr (FADJ) {
#pragma unroll
            for (int r = 0; r < NY; ++r) c[r] = __fmul_rn(c[r], (r & 1) ? KMUL : KDIV);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float cf = adj_coef<FADJ>(k);
#pragma unroll
            for (int r = k + 1; r < NY - k - 1; ++r) {
                if ((r & 1) != adj_par<FADJ>(k)) continue;
                float a = c[r - 1], b = c[r + 1];
                if constexpr (EDGE) {
                    a = __fmul_rn(a, adj_w(ys + r - 1, n));
                    b = __fmul_rn(b, adj_w(ys + r + 1, n));
                }
                c[r] = adj_op(cf, c[r], a, b);
            }
        }
        if constexpr (!FADJ) {
#pragma unroll
            for (int r = 0; r < NY; ++r) c[r] = __fmul_rn(c[r], (r & 1) ? KDIV : KMUL);
        }
    }
}

// ---- synthesis strip kernel ---------------------------------------------------------------------
// Reconstructs (MODE 0) or back-propagates through (MODE 1, 9/7 only) one level: the level's
// detail bands sit at their Mallat positions in `src` (pitch spitch), its LL band in `ll_src`
// (or in `src` itself when DEQLL), and the w x h natural-order result goes to `out`.
//   MODE 0: symmetric extension by mirrored loads, inverse steps, bit-identical to dwt_inv_level;
//           DEQ / DEQLL: the detail / LL samples are int32 dead-zone indices, dequantised on load.
//   MODE 1: zero extension and adjoint boundary weights.
// EXTRA 1 (MODE 0, float): out = result - sub, and the CTA's sum of out^2 goes to part[cta].
// EXTRA 2 (MODE 1):        out = result - (*scale) * alpha * sub.
struct SynExtra {
    const float* sub;
    size_t sub_pitch, sub_z;
    const float* scale;
    float alpha;
    float* part;
    int part_stride;  // row-band kernels: slots per CTA (the sum, then zeros; 0 counts as 1)
};

template <int KERN, int MODE, typename TS, bool DEQ, bool DEQLL, int EXTRA>
__global__ void __launch_bounds__(256)
dwt_syn_fast(const TS* __restrict__ src, size_t spitch, const typename KT<KERN>::T* __restrict__ ll_src,
             size_t llpitch, int w, int h, typename KT<KERN>::T* __restrict__ out, size_t opitch, Steps4 st,
             ZStride z, int vec_in, SynExtra ex) {
    using T = typename KT<KERN>::T;
    constexpr int HV = KT<KERN>::H, NY = STH + 2 * HV;
    __shared__ __align__(16) T s[NY][FNX];
    griddep_launch_dependents();
    griddep_wait();  // launched as a dependent: the previous kernel's writes are visible from here
    src += blockIdx.z * z.src;
    ll_src += blockIdx.z * z.ll;
    out += blockIdx.z * z.dst;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, t = threadIdx.x;
    const int x0 = blockIdx.x * FTW, y0 = blockIdx.y * STH;
    const int wl = (w + 1) >> 1, hl = (h + 1) >> 1;
    const bool inner_x = (x0 - 4 >= 0) && (x0 + 252 <= w);
    // the residual operand of this thread's output column, fetched first so that its latency
    // hides behind the lifting
    float sb[EXTRA != 0 ? STH : 1];
    if constexpr (EXTRA != 0) {
        const float* sub = ex.sub + blockIdx.z * ex.sub_z;
        const int x = x0 - 4 + t;
        const bool colok = t >= 4 && t < 252 && x < w;
#pragma unroll
        for (int j = 0; j < STH; ++j)
            sb[j] = (colok && y0 + j < h) ? __ldg(sub + (size_t)(y0 + j) * ex.sub_pitch + x) : 0.0f;
    }
    // 1. the strip's rows y0 - HV + r (mirrored, or zero outside the level for MODE 1), warp w
    //    taking rows w, w + 8, ...: lane l loads the band samples of natural columns
    //    x0 - 4 + 8l .. + 7 straight into registers (low band: LL or LH row, high band: HL or
    //    HH row), raw; all rows' loads are issued before any is used
    constexpr int RI = (NY + 7) / 8;
    uint32_t rl[RI][4], rh[RI][4];
    const int lx = ((x0 - 4) >> 1) + 4 * lane;  // band index of this lane's first low sample
#pragma unroll
    for (int i = 0; i < RI; ++i) {
        const int r = warp + 8 * i;
#pragma unroll
        for (int k = 0; k < 4; ++k) rl[i][k] = rh[i][k] = 0u;
        if (r >= NY) continue;
        int gy = y0 - HV + r;
        if (MODE == 0) gy = mirror(gy, h);
        else if (gy < 0 || gy >= h) continue;
        const int qy = gy & 1;
        const uint32_t* srow = reinterpret_cast<const uint32_t*>(src + (size_t)((gy >> 1) + (qy ? hl : 0)) * spitch);
        const uint32_t* lsrc = (qy == 0 && !DEQLL)
                                   ? reinterpret_cast<const uint32_t*>(ll_src + (size_t)(gy >> 1) * llpitch)
                                   : srow;
        if (inner_x && vec_in) {
            const uint2 l0 = __ldg(reinterpret_cast<const uint2*>(lsrc + lx));
            const uint2 l1 = __ldg(reinterpret_cast<const uint2*>(lsrc + lx + 2));
            const uint2 h0 = __ldg(reinterpret_cast<const uint2*>(srow + wl + lx));
            const uint2 h1 = __ldg(reinterpret_cast<const uint2*>(srow + wl + lx + 2));
            rl[i][0] = l0.x; rl[i][1] = l0.y; rl[i][2] = l1.x; rl[i][3] = l1.y;
            rh[i][0] = h0.x; rh[i][1] = h0.y; rh[i][2] = h1.x; rh[i][3] = h1.y;
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                int ge = x0 - 4 + 8 * lane + 2 * k, go = ge + 1;
                if (MODE == 0) {
                    ge = mirror(ge, w);
                    go = mirror(go, w);
                }
                if (ge >= 0 && ge < w) rl[i][k] = __ldg(lsrc + (ge >> 1));
                if (go >= 0 && go < w) rh[i][k] = __ldg(srow + wl + (go >> 1));
            }
        }
    }
    // 2. horizontal steps on every strip row (the vertical pass needs the halo rows too), written
    //    in natural order: s[r][c] = sample x0 - 4 + c
    {
        const int xs = x0 - 4 + 8 * lane;
        const bool edge_x = !(x0 - 4 > 0 && x0 + 252 < w);
#pragma unroll
        for (int i = 0; i < RI; ++i) {
            const int r = warp + 8 * i;
            if (r >= NY) break;
            T v[8];
            const int qy = r & 1;  // mirroring keeps the parity of y0 - HV + r
            const float sl = qy ? st.lh : st.ll, sh = qy ? st.hh : st.hl;
            const bool lo_raw = qy == 1 || DEQLL;  // LL rows hold values unless DEQLL
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if constexpr (DEQ) {
                    v[2 * k] = lo_raw ? (T)dequantize((int32_t)rl[i][k], sl) : bits_as<T>(rl[i][k]);
                    v[2 * k + 1] = (T)dequantize((int32_t)rh[i][k], sh);
                } else {
                    v[2 * k] = bits_as<T>(rl[i][k]);
                    v[2 * k + 1] = bits_as<T>(rh[i][k]);
                }
            }
            if (w > 1) {
                if (MODE == 1 && edge_x) hlift8<KERN, MODE, true>(v, xs, w);
                else hlift8<KERN, MODE, false>(v, xs, w);
            }
            *reinterpret_cast<uint4*>(&s[r][8 * lane]) = *reinterpret_cast<uint4*>(&v[0]);
            *reinterpret_cast<uint4*>(&s[r][8 * lane + 4]) = *reinterpret_cast<uint4*>(&v[4]);
        }
    }
    __syncthreads();
    // 3. vertical steps, one column per thread, and the natural-order writes
    T c[NY];
#pragma unroll
    for (int r = 0; r < NY; ++r) c[r] = s[r][t];
    if (h > 1) {
        const int ys = y0 - HV;
        const bool edge_y = !(ys > 0 && y0 + STH + HV - 1 < h - 1);
        if (MODE == 1 && edge_y) vlift<KERN, MODE, true, NY>(c, ys, h);
        else vlift<KERN, MODE, false, NY>(c, ys, h);
    }
    const int x = x0 - 4 + t;
    const bool colok = t >= 4 && t < 252 && x < w;
    float sq = 0.0f;
    float sc = 0.0f;
    if constexpr (EXTRA == 2) sc = __fmul_rn(ex.scale ? *ex.scale : 1.0f, ex.alpha);
#pragma unroll
    for (int j = 0; j < STH; ++j) {
        const int y = y0 + j;
        if (colok && y < h) {
            T v = c[HV + j];
            if constexpr (EXTRA == 1) {
                v = __fsub_rn(v, sb[j]);
                sq = __fmaf_rn(v, v, sq);
            } else if constexpr (EXTRA == 2) {
                v = __fsub_rn(v, __fmul_rn(sc, sb[j]));
            }
            out[(size_t)y * opitch + x] = v;
        }
    }
    if constexpr (EXTRA == 1) {
        __shared__ float red[8];
#pragma unroll
        for (int o = 16; o; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
        if (lane == 0) red[warp] = sq;
        __syncthreads();
        if (t == 0) {
            float a = 0.0f;
#pragma unroll
            for (int i = 0; i < 8; ++i) a += red[i];
            ex.part[((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = a;
        }
    }
}

// ---- analysis strip kernel for the transpose of the inverse 9/7 ---------------------------------
// Gradient of a reconstructed level (w x h natural order, `gin`) -> gradients of its subbands:
// details at their Mallat positions in `gdst`, LL into `gll`.  Zero extension, adjoint
// boundary weights; columns first, then rows (the inverse ran rows, then columns).
__global__ void __launch_bounds__(256)
iadj_ana_fast(const float* __restrict__ gin, size_t ipitch, int w, int h, float* __restrict__ gdst, size_t dpitch,
              float* __restrict__ gll, size_t llpitch, ZStride z, int vec_in, int vec_out) {
    constexpr int HV = 4, NY = STH + 2 * HV;
    __shared__ __align__(16) float s[STH][FNX];  // the vertically lifted rows y0 .. y0+STH-1
    griddep_launch_dependents();
    griddep_wait();  // launched as a dependent: the previous kernel's writes are visible from here
    gin += blockIdx.z * z.src;
    gdst += blockIdx.z * z.dst;
    gll += blockIdx.z * z.ll;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, t = threadIdx.x;
    const int x0 = blockIdx.x * FTW, y0 = blockIdx.y * STH;
    (void)vec_in;
    // column t of the strip straight into registers (zero outside the level)
    float c[NY];
    {
        const int gx = x0 - 4 + t;
        const bool colok = gx >= 0 && gx < w;
        const float* colp = gin + (colok ? gx : 0);
#pragma unroll
        for (int r = 0; r < NY; ++r) {
            const int gy = y0 - HV + r;
            c[r] = (colok && gy >= 0 && gy < h) ? __ldg(colp + (size_t)gy * ipitch) : 0.0f;
        }
    }
    if (h > 1) {
        const int ys = y0 - HV;
        if (!(ys > 0 && y0 + STH + HV - 1 < h - 1)) vlift<97, 2, true, NY>(c, ys, h);
        else vlift<97, 2, false, NY>(c, ys, h);
    }
#pragma unroll
    for (int r = HV; r < HV + STH; ++r) s[r - HV][t] = c[r];
    __syncthreads();
    const int wl = (w + 1) >> 1, hl = (h + 1) >> 1;
    const int xs = x0 - 4 + 8 * lane;
    const bool edge_x = !(x0 - 4 > 0 && x0 + 252 < w);
#pragma unroll
    for (int i = 0; i < STH / 8; ++i) {
        const int r = HV + warp + 8 * i;
        const int y = y0 + r - HV;
        if (y >= h) break;
        float v[8];
        *reinterpret_cast<float4*>(&v[0]) = *reinterpret_cast<const float4*>(&s[r - HV][8 * lane]);
        *reinterpret_cast<float4*>(&v[4]) = *reinterpret_cast<const float4*>(&s[r - HV][8 * lane + 4]);
        if (w > 1) {
            if (edge_x) hlift8<97, 2, true>(v, xs, w);
            else hlift8<97, 2, false>(v, xs, w);
        }
        const int qy = y & 1;
        const int sy = (y >> 1) + (qy ? hl : 0);
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int e0 = 8 * lane + 4 * half;
            const int xa = xs + 4 * half;
            if (e0 + 4 <= 4 || e0 >= 252) continue;  // halo columns
#pragma unroll
            for (int qx = 0; qx < 2; ++qx) {
                const float a = v[4 * half + qx], b = v[4 * half + 2 + qx];
                const int sx = (xa >> 1) + (qx ? wl : 0);
                const bool va = xa + qx < w, vb = xa + 2 + qx < w;
                float* p = (qx == 0 && qy == 0) ? gll + (size_t)sy * llpitch + sx : gdst + (size_t)sy * dpitch + sx;
                if (vec_out && va && vb && ((sx & 1) == 0)) {
                    *reinterpret_cast<float2*>(p) = make_float2(a, b);
                } else {
                    if (va) p[0] = a;
                    if (vb) p[1] = b;
                }
            }
        }
    }
}

}  // namespace
