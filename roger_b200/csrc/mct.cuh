// Colour transforms of 8-bit pixels (ITU-T T.800 Annex G: G.2 RCT, G.3 ICT) after the DC level
// shift (-128), shared by the planar split (planar.cu) and the first forward DWT level that reads
// interleaved pixels (dwt.cu).  Every float operation is rounded separately, in the order the CPU
// oracle uses, so both kernels produce the same samples bit for bit.
#pragma once

#include <cstdint>

#include "j2k_internal.cuh"

namespace {

constexpr float YR = 0.299f, YG = 0.587f, YB = 0.114f;
constexpr float BR = -0.16875f, BG = -0.33126f, BB = 0.5f;
constexpr float RR = 0.5f, RG = -0.41869f, RB = -0.08131f;
constexpr float IRV = 1.402f, IGU = -0.34413f, IGV = -0.71414f, IBU = 1.772f;

__device__ __forceinline__ float dot3(float a, float x, float b, float y, float c, float z) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a, x), __fmul_rn(b, y)), __fmul_rn(c, z));
}

// Component c of one pixel held as bytes 0..2 of px (R, G, B; a gray pixel in byte 0 with NC = 1),
// level-shifted and colour-transformed, as type TO: exactly what the planar split stores.
template <typename TO, int NC, int MCT>
__device__ __forceinline__ TO mct_component(uint32_t px, int c) {
    const int r = (int)(px & 0xFF) - 128;
    if constexpr (NC == 1) {
        return (TO)r;
    } else {
        const int g = (int)((px >> 8) & 0xFF) - 128, b = (int)((px >> 16) & 0xFF) - 128;
        if constexpr (MCT == J2K_MCT_RCT) {
            return c == 0 ? (TO)((r + 2 * g + b) >> 2) : (c == 1 ? (TO)(b - g) : (TO)(r - g));
        } else if constexpr (MCT == J2K_MCT_ICT) {
            const float fr = (float)r, fg = (float)g, fb = (float)b;
            return c == 0 ? (TO)dot3(YR, fr, YG, fg, YB, fb)
                          : (c == 1 ? (TO)dot3(BR, fr, BG, fg, BB, fb) : (TO)dot3(RR, fr, RG, fg, RB, fb));
        } else {
            return (TO)(c == 0 ? r : (c == 1 ? g : b));
        }
    }
}

}  // namespace
