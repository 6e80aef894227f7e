// Waiting time of a promoter that switches at a step, from a table of log2 values.
//
// That waiting time is 1 + floor(log2(u) inv) for u = (b + 1) 2^-18 with b the 18 spare bits
// of the gene's normal words (switch_uniform_bits), and log2 is the library's own explicitly
// rounded series (own_log2f), so that the CPU oracle reproduces it.  b takes 2^18 values, so
// the context fills a 1 MB table with own_log2f of every one of them once, on the device and
// with that same function: a lookup returns the same bits as the series for a load instead of
// some 35 instructions.  Without a table (null pointer) the series runs as before.
#pragma once
#include "cle_device.cuh"

namespace scrna {

constexpr int kSwitchLog2Bits = 18;

__device__ __forceinline__ int32_t switch_steps_from_log2(float l2, float inv) {
    float t = __fmul_rn(l2, inv);  // as geom_steps_u
    if (!(t < 1.0e9f)) t = 1.0e9f;
    return 1 + (int32_t)floorf(t);
}

__device__ __forceinline__ int32_t switch_steps(const float* tab, uint32_t b, float inv) {
    const float l2 = tab ? __ldg(tab + b) : own_log2f(switch_uniform_bits(b));
    return switch_steps_from_log2(l2, inv);
}

}  // namespace scrna
