// Correctly rounded quotient lam / k for the integers k = 1..50 of the Poisson inverse CDF,
// without a branch, so that several quotients can be in flight at once.
//
// Markstein's theorem (P. W. Markstein, "Computation of elementary functions on the IBM
// RISC System/6000 processor", IBM J. Res. Develop. 34(1), 1990; also Muller et al.,
// Handbook of Floating-Point Arithmetic, on division with a fused multiply-add): if y is the
// reciprocal 1/k rounded to nearest and q0 is within one ulp of lam / k, then the residual
// r = lam - k q0 is exactly representable (one FMA computes it exactly) and q0 + r y rounded
// once (a second FMA) is lam / k rounded to nearest.  Here q0 = RN(lam y).
//
// Every operation scales exactly by powers of two while its result stays normal, so the
// outcome for lam in [2^-100, 2^100] follows from one binade of lam for each k; the library's
// check (scrna_debug_small_div_check) compares every float lam of [2^-1, 2^2) and the range
// ends against IEEE division for every k.  lam = 0 gives 0.  Callers keep IEEE division
// for lam outside that range (small_div_ok).
#pragma once

namespace scrna {

// 1/k rounded to nearest (IEEE single division of exact operands, folded at compile time).
static __constant__ float kRecipSmall[51] = {
    0.0f,        1.0f / 1,  1.0f / 2,  1.0f / 3,  1.0f / 4,  1.0f / 5,  1.0f / 6,  1.0f / 7,  1.0f / 8,
    1.0f / 9,    1.0f / 10, 1.0f / 11, 1.0f / 12, 1.0f / 13, 1.0f / 14, 1.0f / 15, 1.0f / 16, 1.0f / 17,
    1.0f / 18,   1.0f / 19, 1.0f / 20, 1.0f / 21, 1.0f / 22, 1.0f / 23, 1.0f / 24, 1.0f / 25, 1.0f / 26,
    1.0f / 27,   1.0f / 28, 1.0f / 29, 1.0f / 30, 1.0f / 31, 1.0f / 32, 1.0f / 33, 1.0f / 34, 1.0f / 35,
    1.0f / 36,   1.0f / 37, 1.0f / 38, 1.0f / 39, 1.0f / 40, 1.0f / 41, 1.0f / 42, 1.0f / 43, 1.0f / 44,
    1.0f / 45,   1.0f / 46, 1.0f / 47, 1.0f / 48, 1.0f / 49, 1.0f / 50};

// lam is 0, or in [2^-100, 2^100] (NaN and infinities fail).
__device__ __forceinline__ bool small_div_ok(float lam) {
    return lam == 0.0f || (lam >= 0x1p-100f && lam <= 0x1p100f);
}

// RN(lam / kf) for kf = (float)k, k in 1..50, y = kRecipSmall[k], lam with small_div_ok.
__device__ __forceinline__ float small_div(float lam, float kf, float y) {
    const float q0 = __fmul_rn(lam, y);
    const float r = __fmaf_rn(-q0, kf, lam);
    return __fmaf_rn(r, y, q0);
}

}  // namespace scrna
