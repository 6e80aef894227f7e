// Device-side building blocks shared by the CLE kernels: Philox4x32-10, the
// Box-Muller transform on Philox words, probability thresholds and the
// bit-reproducible binomial samplers used for capture and division.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace scrna {

// Random-stream tags (bits 31..24 of counter word 3).  The counter layout is part of
// the library's reproducibility contract: a run is a pure function of (seed, stream).
enum : uint32_t {
    TAG_NORMAL = 1,      // (cell, step, gene_pair)    -> Box-Muller pairs for genes 2k, 2k+1
    TAG_SWITCH = 2,      // (cell, 0, gene), (cell, division step, gene | kDaughterSwitch)
                         //   -> initial / daughter waiting time of a promoter
    TAG_PROMOTER = 3,    // (cell, 0, gene_quad)       -> initial promoter state
    TAG_VOLUME = 4,      // (cell, 0, 0)               -> initial volume
    TAG_MORAN = 5,       // (mother, step, 0)          -> replaced slot
    TAG_PARTITION = 6,   // (cell, step, b<<22|g<<1|s) -> partition bits
    TAG_EFFICIENCY = 7,  // (cell, 0, 0)               -> capture efficiency normal
    TAG_CAPTURE = 8,     // (cell, chunk, gene)        -> capture inverse-CDF uniform
    TAG_TAU = 9          // (cell, step, gene)         -> the four uniforms of a tau-leap update
};

constexpr int kCaptureChunk = 512;
constexpr int64_t kPartitionPopcountMax = 131072;

struct Key { uint32_t k0, k1; };

// Philox4x32-10 (Salmon et al., SC'11): 10 rounds of two 32x32->64 products whose
// high halves are xor'ed with the other counter words and the round key.
__device__ __forceinline__ uint4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                        Key key) {
    uint32_t k0 = key.k0, k1 = key.k1;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    }
    return make_uint4(c0, c1, c2, c3);
}

// Philox4x32-10 with its ten round keys given (round r: key + r (0x9E3779B9, 0xBB67AE85),
// precomputed on the host).  Identical output to philox(); when rk0 / rk1 live in kernel
// parameter space the rounds read them as constant operands instead of recomputing them.
__device__ __forceinline__ uint4 philox_rk(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                           const uint32_t* rk0, const uint32_t* rk1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
        const uint32_t n0 = hi1 ^ c1 ^ rk0[r];
        const uint32_t n2 = hi0 ^ c3 ^ rk1[r];
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    }
    return make_uint4(c0, c1, c2, c3);
}

__device__ __forceinline__ uint32_t tagword(uint32_t tag, uint32_t stream) {
    return (tag << 24) | (stream & 0xFFFFFFu);
}

// FP32 Box-Muller pieces for one pair of words:
//   u1 = 1 - (w0>>9) 2^-23 in (0,1],  h = (w1>>9) 2^-23 - 1/2 in [-1/2,1/2)
//   L = -2 ln u1,  (z0, z1) = sqrt(L) (cos 2 pi h, sin 2 pi h).
// Returned as (L, cos, sin) so callers can fold sqrt(L) into another square root.
struct BM { float L, c, s; };
// 1 + (w >> 9) 2^-23 as the bits 0x3F800000 | (w >> 9), one funnel shift of (0x7F : w) by 9.
__device__ __forceinline__ float one_plus_top23(uint32_t w) { return __uint_as_float(__funnelshift_r(w, 0x7Fu, 9)); }
__device__ __forceinline__ BM box_muller_parts(uint32_t w0, uint32_t w1) {
    const float u1 = 2.0f - one_plus_top23(w0);
    const float h = one_plus_top23(w1) - 1.5f;
    const float th = 6.28318530717958648f * h;
    BM r;
    r.L = -1.38629436111989061f * __log2f(u1);  // -2 ln 2 * log2(u1)
    __sincosf(th, &r.s, &r.c);
    return r;
}

// FP64 Box-Muller (first normal of the pair), same uniforms as above.
__device__ __forceinline__ double box_muller_z0_f64(uint32_t w0, uint32_t w1) {
    const double u1 = (double)(8388608u - (w0 >> 9)) / 8388608.0;
    const double u2 = (double)(w1 >> 9) / 8388608.0;
    const double th = 6.283185307179586 * (u2 - 0.5);
    return sqrt(-2.0 * log(u1)) * cos(th);
}
__device__ __forceinline__ void box_muller_f64(uint32_t w0, uint32_t w1, double* z0, double* z1) {
    const double u1 = (double)(8388608u - (w0 >> 9)) / 8388608.0;
    const double u2 = (double)(w1 >> 9) / 8388608.0;
    const double th = 6.283185307179586 * (u2 - 0.5);
    const double r = sqrt(-2.0 * log(u1));
    double s, c;
    sincos(th, &s, &c);
    *z0 = r * c;
    *z1 = r * s;
}

__device__ __forceinline__ double u53(uint32_t a, uint32_t b) {
    return __dmul_rn(__dadd_rn(__dmul_rn((double)(a >> 5), 67108864.0), (double)(b >> 6)),
                     1.0 / 9007199254740992.0);
}

// Inverse-CDF Binomial(n, p) for n <= kCaptureChunk and p <= 1/2, every operation an
// explicitly rounded IEEE op so that a CPU restatement compiled without FMA contraction
// returns the identical integer:  pmf(0) = (1-p)^n by binary powering, then
// pmf(k+1) = ((pmf(k) (n-k)) / (k+1)) (p/(1-p)); result = smallest k with u < cdf(k).
__device__ __forceinline__ int invcdf_chunk(int n, double p, double u) {
    const double q = __dadd_rn(1.0, -p);
    const double ratio = __ddiv_rn(p, q);
    double base = q, pmf = 1.0;
    for (int e = n; e; e >>= 1) {
        if (e & 1) pmf = __dmul_rn(pmf, base);
        base = __dmul_rn(base, base);
    }
    double cdf = pmf;
    int k = 0;
    while (u >= cdf && k < n) {
        pmf = __dmul_rn(__ddiv_rn(__dmul_rn(pmf, (double)(n - k)), (double)(k + 1)), ratio);
        k += 1;
        cdf = __dadd_rn(cdf, pmf);
    }
    return k;
}

// Binomial(n, p) as a sum of chunks of at most kCaptureChunk trials, each with its own
// uniform (counter (cell, chunk, gene)); p > 1/2 is sampled as n - Binomial(n, 1-p).
__device__ __forceinline__ int64_t binomial_capture(int64_t n, double p, Key key, uint32_t stream,
                                                    uint32_t cell, uint32_t gene) {
    if (n <= 0 || !(p > 0.0)) return 0;
    const bool flip = p > 0.5;
    const double pp = flip ? __dadd_rn(1.0, -p) : p;
    int64_t total = 0;
    const int64_t nch = (n + kCaptureChunk - 1) / kCaptureChunk;
    for (int64_t i = 0; i < nch; ++i) {
        int64_t ni = n - i * kCaptureChunk;
        if (ni > kCaptureChunk) ni = kCaptureChunk;
        const uint4 w = philox(cell, (uint32_t)i, gene, tagword(TAG_CAPTURE, stream), key);
        total += invcdf_chunk((int)ni, pp, u53(w.x, w.y));
    }
    return flip ? n - total : total;
}

// Binomial(n, 1/2) for the division partition: the popcount of n Philox bits.
__device__ __forceinline__ int64_t binomial_half(int64_t n, Key key, uint32_t stream, uint32_t cell,
                                                 uint32_t step, uint32_t gene, uint32_t species) {
    if (n <= 0) return 0;
    if (n > kPartitionPopcountMax) {
        const uint4 w = philox(cell, step, (gene << 1) | species, tagword(TAG_PARTITION, stream), key);
        double z0, z1;
        box_muller_f64(w.x, w.y, &z0, &z1);
        double x = rint(0.5 * (double)n + 0.5 * sqrt((double)n) * z0);
        x = fmin(fmax(x, 0.0), (double)n);
        return (int64_t)x;
    }
    int64_t total = 0, left = n;
    for (uint32_t b = 0; left > 0; ++b) {
        const uint4 w = philox(cell, step, (b << 22) | (gene << 1) | species,
                               tagword(TAG_PARTITION, stream), key);
        const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (left <= 0) break;
            uint32_t x = ws[j];
            if (left < 32) x &= (1u << left) - 1u;
            total += __popc(x);
            left -= 32;
        }
    }
    return total;
}

__device__ __forceinline__ float fsqrt_approx(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// ---- telegraph waiting times ----------------------------------------------------------------
// The reference switches a promoter with probability 1 - exp(-k dt) at every step; the
// number of steps to the next switch is then geometric with stay probability
// exp(-k dt) = 2^(1/inv), inv = -ln2 / (k dt).  It is drawn once per switch as
// 1 + floor(log2(u) inv), u = ((w>>8)+1) 2^-24.  log2 is this library's own: the atanh
// series log2 m = (2/ln 2) atanh z, z = (m-1)/(m+1), m in [sqrt(1/2), sqrt(2)), terms to
// z^11, with every operation explicitly rounded so the CPU oracle reproduces it bit for bit.
__device__ __forceinline__ float own_log2f(float u) {
    const uint32_t b = __float_as_uint(u);
    int e = (int)((b >> 23) & 0xFFu) - 127;
    float m = __uint_as_float((b & 0x7FFFFFu) | 0x3F800000u);
    if (m > 1.41421353816986083984375f) { m = __fmul_rn(m, 0.5f); e += 1; }
    const float z = __fdiv_rn(__fsub_rn(m, 1.0f), __fadd_rn(m, 1.0f));
    const float z2 = __fmul_rn(z, z);
    float q = __fmaf_rn(z2, 1.0f / 11.0f, 1.0f / 9.0f);
    q = __fmaf_rn(z2, q, 1.0f / 7.0f);
    q = __fmaf_rn(z2, q, 1.0f / 5.0f);
    q = __fmaf_rn(z2, q, 1.0f / 3.0f);
    q = __fmaf_rn(z2, q, 1.0f);
    return __fmaf_rn(__fmul_rn(z, q), 2.88539008f, (float)e);
}

__device__ __forceinline__ int32_t geom_steps_u(float u, float inv) {
    float t = __fmul_rn(own_log2f(u), inv);
    if (!(t < 1.0e9f)) t = 1.0e9f;
    return 1 + (int32_t)floorf(t);
}

// Step of the next switch after `step` (saturating), for stay-probability parameter inv
// and a uniform u in (0, 1].
__device__ __forceinline__ int32_t next_switch_u(int64_t step, float u, float inv) {
    const int64_t t = step + geom_steps_u(u, inv);
    return t > 2147483647 ? 2147483647 : (int32_t)t;
}

// Initial and daughter waiting times come from a dedicated switch word w:
// u = ((w>>8)+1) 2^-24.
__device__ __forceinline__ int32_t next_switch(int64_t step, uint32_t w, float inv) {
    return next_switch_u(step, __fmul_rn(__uint2float_rn((w >> 8) + 1u), 5.9604644775390625e-8f), inv);
}

// A promoter that switches at a step draws a waiting time from the spare bits of the
// gene's two normal words of that step (Box-Muller reads only their top 23 bits):
// b = (w0 & 511) << 9 | (w1 & 511), u = (b + 1) 2^-18, so a switch costs no Philox call.
__device__ __forceinline__ uint32_t switch_bits(uint32_t w0, uint32_t w1) {
    return ((w0 & 0x1FFu) << 9) | (w1 & 0x1FFu);
}
__device__ __forceinline__ float switch_uniform_bits(uint32_t b) {
    return __fmul_rn(__uint2float_rn(b + 1u), 3.814697265625e-06f);
}
__device__ __forceinline__ float switch_uniform(uint32_t w0, uint32_t w1) {
    return switch_uniform_bits(switch_bits(w0, w1));
}

__device__ __forceinline__ int32_t sat_step(int64_t t) { return t > 2147483647 ? 2147483647 : (int32_t)t; }

// Switching state of a gene, int2 {x: step of the next switch, y: the waiting time that
// follows it}.  Waiting times are drawn one switch ahead: a promoter switching at step s
// enters state X, stays y steps (drawn earlier, for X) and draws the waiting time after
// its next switch (for !X) from the spare bits of step s.  inv_on parameterises the stay
// while OFF, inv_off while ON.  A fresh promoter (initial state, or a daughter at
// division) draws both from a switch word pair; a gene that never switches has both kNever.
__device__ __forceinline__ int2 fresh_switch(int64_t step, uint32_t w0, uint32_t w1, bool on, float inv_on,
                                             float inv_off) {
    const float u1 = __fmul_rn(__uint2float_rn((w1 >> 8) + 1u), 5.9604644775390625e-8f);
    return make_int2(next_switch(step, w0, on ? inv_off : inv_on), geom_steps_u(u1, on ? inv_on : inv_off));
}
// The switch itself: `on` is the state entered at step s.
__device__ __forceinline__ int2 switch_at(int64_t step, int2 sw, float us, bool on, float inv_on, float inv_off) {
    return make_int2(sat_step(step + sw.y), geom_steps_u(us, on ? inv_on : inv_off));
}

constexpr int32_t kNever = 2147483647;
constexpr uint32_t kDaughterSwitch = 0x800000u;  // counter flag: a daughter's fresh waiting time

__device__ __forceinline__ float frcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ float hill_act(float p, float Kn, float hill_n, int hill_int) {
    float pn;
    if (hill_int == 2) {
        pn = p * p;
    } else if (hill_int > 0) {
        pn = 1.0f;
        for (int i = 0; i < hill_int; ++i) pn *= p;
    } else {
        pn = exp2f(hill_n * __log2f(p));
    }
    // pn / (pn + Kn); an infinite pn gives NaN in the product and fminf returns 1.
    return fminf(pn * frcp_approx(pn + Kn), 1.0f);
}

// One Euler-Maruyama step of (m, p) with collapsed noise (cle.jl:109-120): M first, then P
// with the new M.  z sqrt(dt var) is evaluated as cos(theta) sqrt(L dt var), folding the
// Box-Muller radius sqrt(L) into the variance square root.  m, p >= 0 on entry.
__device__ __forceinline__ void em_update(float& m, float& p, float tx, const BM& bm, float mu_m,
                                          float mu_p, float k_t, float dt) {
    const float Ldt = bm.L * dt;
    const float mo = m, po = p;
    const float var_m = fmaxf(fmaf(mu_m, mo, tx), 0.0f);
    float mn = fmaf(bm.c, fsqrt_approx(Ldt * var_m), fmaf(fmaf(-mu_m, mo, tx), dt, mo));
    mn = fmaxf(mn, 0.0f);
    const float var_p = fmaf(k_t, mn, mu_p * po);
    float pn = fmaf(bm.s, fsqrt_approx(Ldt * var_p), fmaf(fmaf(k_t, mn, -mu_p * po), dt, po));
    pn = fmaxf(pn, 0.0f);
    m = mn;
    p = pn;
}

// ---- gene pairs in packed FP32 ----------------------------------------------------------
// sm_100 adds, multiplies and fused multiply-adds two FP32 values per instruction
// (add/mul/fma .rn.f32x2); each half is rounded exactly as the scalar operation, so the pair
// forms below give the scalar forms' bits gene by gene and the kernels that use them stay
// bit-identical to those that do not.  Minimum, maximum and the special functions have no
// pair form and stay scalar.
__device__ __forceinline__ float2 f2(float x) { return make_float2(x, x); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 max0_2(float2 a) { return make_float2(fmaxf(a.x, 0.0f), fmaxf(a.y, 0.0f)); }

// box_muller_parts of the two genes of one Philox block: gene 0 from (w.x, w.y), gene 1 from
// (w.z, w.w).  2 - a is formed as fma(a, -1, 2): the product is exact, one rounding as the add.
struct BM2 { float2 L, c, s; };
__device__ __forceinline__ BM2 box_muller_parts2(uint4 w) {
    const float2 a = make_float2(one_plus_top23(w.x), one_plus_top23(w.z));
    const float2 b = make_float2(one_plus_top23(w.y), one_plus_top23(w.w));
    const float2 u1 = fma2(a, f2(-1.0f), f2(2.0f));
    const float2 th = mul2(f2(6.28318530717958648f), add2(b, f2(-1.5f)));
    BM2 r;
    r.L = mul2(f2(-1.38629436111989061f), make_float2(__log2f(u1.x), __log2f(u1.y)));
    __sincosf(th.x, &r.s.x, &r.c.x);
    __sincosf(th.y, &r.s.y, &r.c.y);
    return r;
}

// em_update for two genes; mu_m_neg = -mu_m, mu_p_neg = -mu_p.
__device__ __forceinline__ void em_update2(float2& m, float2& p, float2 tx, const BM2& bm, float mu_m,
                                           float mu_m_neg, float mu_p, float mu_p_neg, float k_t, float dt) {
    const float2 Ldt = mul2(bm.L, f2(dt));
    const float2 mo = m, po = p;
    const float2 var_m = max0_2(fma2(f2(mu_m), mo, tx));
    const float2 vm = mul2(Ldt, var_m);
    const float2 mn = max0_2(fma2(bm.c, make_float2(fsqrt_approx(vm.x), fsqrt_approx(vm.y)),
                                  fma2(fma2(f2(mu_m_neg), mo, tx), f2(dt), mo)));
    const float2 var_p = fma2(f2(k_t), mn, mul2(f2(mu_p), po));
    const float2 vp = mul2(Ldt, var_p);
    const float2 pn = max0_2(fma2(bm.s, make_float2(fsqrt_approx(vp.x), fsqrt_approx(vp.y)),
                                  fma2(fma2(f2(k_t), mn, mul2(f2(mu_p_neg), po)), f2(dt), po)));
    m = mn;
    p = pn;
}

// hill_act with hill_int == 2 for two genes.
__device__ __forceinline__ float2 hill2_n2(float2 p, float Kn) {
    const float2 pn = mul2(p, p);
    const float2 d = add2(pn, f2(Kn));
    const float2 r = mul2(pn, make_float2(frcp_approx(d.x), frcp_approx(d.y)));
    return make_float2(fminf(r.x, 1.0f), fminf(r.y, 1.0f));
}

// ---- binomial tau-leap ------------------------------------------------------------------
// exp(x) for x <= 0 from its definition, every operation explicitly rounded so that a CPU
// restatement returns the same bits: x = k ln2 + r, k = rint(x log2 e), |r| <= ln2/2
// (two-constant Cody-Waite reduction), e^r by its Taylor series to r^7 (Horner), then the
// exact scaling by 2^k (in two steps below 2^-126 so a subnormal result rounds once).
__device__ __forceinline__ float own_expf(float x) {
    if (!(x > -104.0f)) return 0.0f;
    if (x > 0.0f) x = 0.0f;
    const float k = rintf(__fmul_rn(x, 1.44269502162933349609375f));
    float r = __fmaf_rn(-k, 0.693145751953125f, x);
    r = __fmaf_rn(-k, 1.428606765330187045e-06f, r);
    float q = __fmaf_rn(r, 1.0f / 5040.0f, 1.0f / 720.0f);
    q = __fmaf_rn(r, q, 1.0f / 120.0f);
    q = __fmaf_rn(r, q, 1.0f / 24.0f);
    q = __fmaf_rn(r, q, 1.0f / 6.0f);
    q = __fmaf_rn(r, q, 0.5f);
    q = __fmaf_rn(r, q, 1.0f);
    q = __fmaf_rn(r, q, 1.0f);
    int ki = (int)k;
    if (ki < -125) {
        q = __fmul_rn(q, __uint_as_float(0x1F800000u));  // 2^-64
        ki += 64;
    }
    return __fmul_rn(q, __uint_as_float((uint32_t)(ki + 127) << 23));
}

// Poisson(lam) by inverse CDF over the first 50 terms (the reference's GPU sampler): the
// number of partial sums of exp(-lam) lam^j / j! that u exceeds, at most 50.  The partial
// sums never decrease, so the loop stops at the first one u does not exceed.
__device__ __forceinline__ float poisson_icdf50(float u, float lam) {
    float term = own_expf(-lam);
    float cdf = term;
    float events = 0.0f;
    for (int k = 1; k <= 50; ++k) {
        if (!(u > cdf)) break;
        events = (float)k;
        term = __fmul_rn(term, __fdiv_rn(lam, (float)k));
        cdf = __fadd_rn(cdf, term);
    }
    return events;
}

// The four uniforms of a tau-leap block: (w >> 9) 2^-23 in [0, 1) (the low 9 bits of words
// 0 and 1 are the telegraph's spare bits, as for the normal words).
__device__ __forceinline__ float tau_uniform(uint32_t w) { return __fmul_rn((float)(w >> 9), 1.1920928955078125e-07f); }

// One tau-leap update of (m, p) (ext/SyntheticscRNAseqCUDAExt.jl:258-275): transcription
// Poisson(lam_tx), mRNA decay min(Poisson(m p_m), m), then translation Poisson(k_t m dt) with
// the new m and protein decay min(Poisson(p p_p), p); counts never go below 0.
__device__ __forceinline__ void tau_update(float& m, float& p, float lam_tx, uint4 w, float k_t, float dt,
                                           float p_dec_m, float p_dec_p) {
    const float n_tx = poisson_icdf50(tau_uniform(w.x), lam_tx);
    const float mp = fmaxf(m, 0.0f);
    const float n_md = fminf(poisson_icdf50(tau_uniform(w.y), __fmul_rn(mp, p_dec_m)), mp);
    const float mn = fmaxf(__fsub_rn(__fadd_rn(m, n_tx), n_md), 0.0f);
    const float n_tl = poisson_icdf50(tau_uniform(w.z), __fmul_rn(__fmul_rn(k_t, mn), dt));
    const float pp = fmaxf(p, 0.0f);
    const float n_pd = fminf(poisson_icdf50(tau_uniform(w.w), __fmul_rn(pp, p_dec_p)), pp);
    m = mn;
    p = fmaxf(__fsub_rn(__fadd_rn(p, n_tl), n_pd), 0.0f);
}

}  // namespace scrna
