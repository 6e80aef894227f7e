// Philox4x32-10 for a counter whose only varying word is c1 (the Euler step), with the part
// of the first three rounds that does not depend on c1 computed once.
//
// Round r maps (c0, c1, c2, c3) to (hi(M1 c2) ^ c1 ^ k0_r, lo(M1 c2), hi(M0 c0) ^ c3 ^ k1_r,
// lo(M0 c0)).  With c0, c2, c3 fixed:
//   round 1: c0 = A ^ c1 with A = hi(M1 c2) ^ k0_0; c1, c2, c3 become constants B, C, D;
//   round 2: the M1 product is of the constant C, so the new c0 (E) and c1 (F) are constants;
//            the M0 product is the first one that depends on the step;
//   round 3: the M0 product is of the constant E: its halves (I, J) are constants.
// Five words carry the rest (A, H = D ^ k1_1, K = F ^ k0_2, L = I ^ k1_2, J), and a draw costs
// 2 products and 3 xors fewer over the first three rounds (34 instead of 40 instructions)
// with the same output bits as philox_rk.
#pragma once
#include <cstdint>

namespace scrna {

struct PhiloxHoist { uint32_t A, H, K, L, J; };

__device__ __forceinline__ PhiloxHoist philox_hoist(uint32_t c0, uint32_t c2, uint32_t c3, const uint32_t* rk0,
                                                    const uint32_t* rk1) {
    const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
    PhiloxHoist h;
    h.A = hi1 ^ rk0[0];
    const uint32_t B = lo1, C = hi0 ^ c3 ^ rk1[0], D = lo0;
    const uint32_t E = __umulhi(0xCD9E8D57u, C) ^ B ^ rk0[1], F = 0xCD9E8D57u * C;
    h.H = D ^ rk1[1];
    const uint32_t I = __umulhi(0xD2511F53u, E);
    h.J = 0xD2511F53u * E;
    h.K = F ^ rk0[2];
    h.L = I ^ rk1[2];
    return h;
}

// philox_rk(c0, c1, c2, c3, rk0, rk1) for the c0, c2, c3 of `h`.
__device__ __forceinline__ uint4 philox_hoisted(const PhiloxHoist& h, uint32_t c1, const uint32_t* rk0,
                                                const uint32_t* rk1) {
    const uint32_t a = h.A ^ c1;                                              // round 1
    const uint32_t c2_2 = __umulhi(0xD2511F53u, a) ^ h.H, c3_2 = 0xD2511F53u * a;  // round 2
    uint32_t c0 = __umulhi(0xCD9E8D57u, c2_2) ^ h.K;                         // round 3
    uint32_t c1r = 0xCD9E8D57u * c2_2;
    uint32_t c2 = c3_2 ^ h.L;
    uint32_t c3 = h.J;
#pragma unroll
    for (int r = 3; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
        const uint32_t n0 = hi1 ^ c1r ^ rk0[r];
        const uint32_t n2 = hi0 ^ c3 ^ rk1[r];
        c0 = n0; c1r = lo1; c2 = n2; c3 = lo0;
    }
    return make_uint4(c0, c1r, c2, c3);
}

}  // namespace scrna
