/*
 * CPU oracle for the batched CLE path — TEST INFRASTRUCTURE ONLY (see cle_oracle.h).
 *
 * Built with -ffp-contract=off so that every FP64 expression rounds exactly as
 * written, like Julia's broadcasts (which do not contract to FMA).
 */
#include "cle_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---------------------------------------------------------------------------
 * Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
 * as 1, 2, 3", SC'11).  Round: two 32x32->64 multiplies, the high halves
 * xor'ed with the other counter words and the key; key bumped by the Weyl
 * constants between rounds.
 * ------------------------------------------------------------------------- */
#define ORC_LN2 0.69314718055994530942
#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += PHILOX_W0; k1 += PHILOX_W1; }
        uint64_t p0 = (uint64_t)PHILOX_M0 * c0;
        uint64_t p1 = (uint64_t)PHILOX_M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static inline void draw(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t tag,
                        uint32_t stream, uint32_t out[4]) {
    uint32_t ctr[4] = {c0, c1, c2, (tag << 24) | (stream & 0xFFFFFFu)};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    orc_philox4x32_10(ctr, key, out);
}

/* Box-Muller on two 32-bit words (same uniforms as the device code):
 *   u1 = 1 - (w0>>9)*2^-23 in (0,1],  u2 = (w1>>9)*2^-23 in [0,1)
 *   theta = 2*pi*(u2 - 1/2),  r = sqrt(-2 ln u1),  z0 = r cos theta, z1 = r sin theta. */
static inline void box_muller(uint32_t w0, uint32_t w1, double* z0, double* z1) {
    double u1 = (double)(8388608u - (w0 >> 9)) / 8388608.0;
    double u2 = (double)(w1 >> 9) / 8388608.0;
    double th = 6.283185307179586 * (u2 - 0.5);
    double r = sqrt(-2.0 * log(u1));
    *z0 = r * cos(th);
    *z1 = r * sin(th);
}

/* 53-bit uniform in [0,1) from two words. */
static inline double u53(uint32_t a, uint32_t b) {
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

void orc_step_normals(uint64_t seed, uint32_t stream, uint32_t cell, uint32_t step,
                      uint32_t gene, double* zm, double* zp) {
    uint32_t w[4];
    draw(seed, cell, step, gene >> 1, ORC_TAG_NORMAL, stream, w);
    if (gene & 1u) box_muller(w[2], w[3], zm, zp);
    else box_muller(w[0], w[1], zm, zp);
}

/* Probability -> 32-bit threshold: an event fires when the word is < thr. */
static inline uint32_t prob_threshold(double p) {
    if (!(p > 0.0)) return 0u;
    double t = floor(p * 4294967296.0);
    if (t >= 4294967295.0) return 0xFFFFFFFFu;
    return (uint32_t)t;
}

/* ---------------------------------------------------------------------------
 * Binomial samplers (bit-exact with the device code).
 * ------------------------------------------------------------------------- */
#define CAPTURE_CHUNK 512

/* (1-p)^n by binary exponentiation, then the pmf recurrence
 *   pmf(k+1) = ((pmf(k) * (n-k)) / (k+1)) * (p/(1-p)),
 * returning the smallest k with u < cdf(k). Requires p <= 1/2 and n <= 512 so
 * the starting pmf stays a normal double. */
static int64_t invcdf_chunk(int64_t n, double p, double u) {
    double q = 1.0 - p;
    double ratio = p / q;
    double base = q, pmf = 1.0;
    int64_t e = n;
    while (e) { if (e & 1) pmf = pmf * base; base = base * base; e >>= 1; }
    double cdf = pmf;
    int64_t k = 0;
    while (u >= cdf && k < n) {
        pmf = ((pmf * (double)(n - k)) / (double)(k + 1)) * ratio;
        k += 1;
        cdf = cdf + pmf;
    }
    return k;
}

int64_t orc_binomial_invcdf(int64_t n, double p, uint64_t seed, uint32_t stream,
                            uint32_t cell, uint32_t gene) {
    if (n <= 0 || !(p > 0.0)) return 0;
    int flip = p > 0.5;
    double pp = flip ? 1.0 - p : p;
    int64_t total = 0;
    int64_t nchunks = (n + CAPTURE_CHUNK - 1) / CAPTURE_CHUNK;
    for (int64_t i = 0; i < nchunks; ++i) {
        int64_t ni = n - i * CAPTURE_CHUNK;
        if (ni > CAPTURE_CHUNK) ni = CAPTURE_CHUNK;
        uint32_t w[4];
        draw(seed, cell, (uint32_t)i, gene, ORC_TAG_CAPTURE, stream, w);
        total += invcdf_chunk(ni, pp, u53(w[0], w[1]));
    }
    return flip ? n - total : total;
}

#define PARTITION_POPCOUNT_MAX 131072

int64_t orc_binomial_half(int64_t n, uint64_t seed, uint32_t stream, uint32_t cell,
                          uint32_t step, uint32_t gene, uint32_t species) {
    if (n <= 0) return 0;
    if (n > PARTITION_POPCOUNT_MAX) {
        /* Rounded normal approximation (documented: not bit-exact territory). */
        uint32_t w[4];
        draw(seed, cell, step, (gene << 1) | species, ORC_TAG_PARTITION, stream, w);
        double z0, z1;
        box_muller(w[0], w[1], &z0, &z1);
        double x = rint(0.5 * (double)n + 0.5 * sqrt((double)n) * z0);
        if (x < 0) x = 0;
        if (x > (double)n) x = (double)n;
        return (int64_t)x;
    }
    int64_t total = 0, left = n;
    for (uint32_t b = 0; left > 0; ++b) {
        uint32_t w[4];
        draw(seed, cell, step, (b << 22) | (gene << 1) | species, ORC_TAG_PARTITION, stream, w);
        for (int j = 0; j < 4 && left > 0; ++j) {
            uint32_t x = w[j];
            if (left < 32) x &= (1u << left) - 1u;
            total += __builtin_popcount(x);
            left -= 32;
        }
    }
    return total;
}

/* ---------------------------------------------------------------------------
 * Telegraph waiting times.  log2 by the atanh series (log2 m = (2/ln 2) atanh z,
 * z = (m-1)/(m+1), m in [sqrt(1/2), sqrt(2)), terms to z^11), every operation an
 * explicitly rounded FP32 op so the device computes the identical value.
 * ------------------------------------------------------------------------- */
static inline float f_of_bits(uint32_t b) { float f; memcpy(&f, &b, 4); return f; }
static inline uint32_t bits_of_f(float f) { uint32_t b; memcpy(&b, &f, 4); return b; }

float orc_log2f(float u) {
    uint32_t b = bits_of_f(u);
    int e = (int)((b >> 23) & 0xFFu) - 127;
    float m = f_of_bits((b & 0x7FFFFFu) | 0x3F800000u);
    if (m > 1.41421353816986083984375f) { m = m * 0.5f; e += 1; }
    float z = (m - 1.0f) / (m + 1.0f);
    float z2 = z * z;
    float q = fmaf(z2, 1.0f / 11.0f, 1.0f / 9.0f);
    q = fmaf(z2, q, 1.0f / 7.0f);
    q = fmaf(z2, q, 1.0f / 5.0f);
    q = fmaf(z2, q, 1.0f / 3.0f);
    q = fmaf(z2, q, 1.0f);
    return fmaf(z * q, 2.88539008f, (float)e);
}

/* Geometric number of steps (>= 1) until the next switch for stay probability
 * 2^(1/inv): 1 + floor(log2(u) * inv) for a uniform u in (0, 1]. */
int32_t orc_geom_steps_u(float u, float inv) {
    float t = orc_log2f(u) * inv;
    if (!(t < 1.0e9f)) t = 1.0e9f;
    return 1 + (int32_t)floorf(t);
}

/* Initial and daughter waiting times: u = ((w>>8)+1) 2^-24 from a dedicated switch word. */
int32_t orc_geom_steps(uint32_t w, float inv) {
    return orc_geom_steps_u((float)((w >> 8) + 1u) * 5.9604644775390625e-8f, inv);
}

/* Waiting time drawn when a promoter switches at a step: the 9 low bits of each of the
 * gene's two normal words of that step (Box-Muller reads only their top 23 bits),
 * u = (((w0 & 511) << 9 | (w1 & 511)) + 1) 2^-18. */
float orc_switch_uniform(uint32_t w0, uint32_t w1) {
    uint32_t b = ((w0 & 0x1FFu) << 9) | (w1 & 0x1FFu);
    return (float)(b + 1u) * 3.814697265625e-06f;
}

static inline int32_t clamp_step(int64_t t) { return t > 2147483647 ? 2147483647 : (int32_t)t; }

/* Switching state of one gene: the step of the next switch and the waiting time that
 * follows it.  Waiting times are drawn one switch ahead: a promoter switching at step s
 * enters state X, stays kn steps (drawn earlier, for X) and draws the waiting time after
 * its next switch (for !X) from the spare bits of step s.  A fresh promoter (initial state
 * or a daughter) draws both from one switch word pair.  Never switching: both INT32_MAX. */
typedef struct { int32_t ns, kn; } sw_t;

static inline void fresh_switch(sw_t* sw, int64_t step, const uint32_t w[4], int on, float inv_on,
                                float inv_off) {
    sw->ns = clamp_step(step + orc_geom_steps(w[0], on ? inv_off : inv_on));
    sw->kn = orc_geom_steps(w[1], on ? inv_on : inv_off);
}

/* ---------------------------------------------------------------------------
 * CLE
 * ------------------------------------------------------------------------- */
typedef struct {
    int G;
    double* Apos;  /* [G*G] row-major, precompute_hill_matrices (network.jl:206-219) */
    double* Aneg;
    /* Nonzero columns of each row of Apos / Aneg, ascending: row i's are
     * pos_col[pos_ptr[i] .. pos_ptr[i+1]-1].  The row sums run over these only; the
     * skipped terms are +0 * finite >= 0 = +0 and s + (+0) = s for the nonnegative partial
     * sums, so the result is bit-identical to the dense loop of cle.jl:84-86. */
    int32_t* pos_ptr;
    int32_t* pos_col;
    double* pos_val;
    int32_t* neg_ptr;
    int32_t* neg_col;
    double* neg_val;
    float* inv_on;      /* 1 / log2(stay probability OFF) = -ln2 / (k_on dt) */
    float* inv_off;     /* 1 / log2(stay probability ON)  = -ln2 / (k_off dt) */
    uint32_t* thr_init;
    uint8_t* tel;       /* switching active: isfinite(k_on) (tauleap_binomial.jl:86) */
    uint8_t* init_rand; /* both rates finite: random initial state (tauleap_binomial.jl:69) */
    int bursty;
} prep_t;

static void prep_build(const orc_net* net, double dt, prep_t* pp) {
    int G = net->G;
    pp->G = G;
    pp->Apos = (double*)calloc((size_t)G * G, sizeof(double));
    pp->Aneg = (double*)calloc((size_t)G * G, sizeof(double));
    for (int i = 0; i < G; ++i)
        for (int j = 0; j < G; ++j) {
            if (i == j) continue;
            double a = net->A[(size_t)i * G + j] * net->basals[i];
            pp->Apos[(size_t)i * G + j] = a > 0.0 ? a : 0.0;
            pp->Aneg[(size_t)i * G + j] = -a > 0.0 ? -a : 0.0;
        }
    pp->pos_ptr = (int32_t*)calloc((size_t)G + 1, 4);
    pp->neg_ptr = (int32_t*)calloc((size_t)G + 1, 4);
    size_t npos = 0, nneg = 0;
    for (size_t k = 0; k < (size_t)G * G; ++k) {
        npos += pp->Apos[k] != 0.0;
        nneg += pp->Aneg[k] != 0.0;
    }
    pp->pos_col = (int32_t*)malloc((npos ? npos : 1) * 4);
    pp->neg_col = (int32_t*)malloc((nneg ? nneg : 1) * 4);
    pp->pos_val = (double*)malloc((npos ? npos : 1) * sizeof(double));
    pp->neg_val = (double*)malloc((nneg ? nneg : 1) * sizeof(double));
    npos = nneg = 0;
    for (int i = 0; i < G; ++i) {
        pp->pos_ptr[i] = (int32_t)npos;
        pp->neg_ptr[i] = (int32_t)nneg;
        for (int j = 0; j < G; ++j) {
            if (pp->Apos[(size_t)i * G + j] != 0.0) {
                pp->pos_col[npos] = j;
                pp->pos_val[npos++] = pp->Apos[(size_t)i * G + j];
            }
            if (pp->Aneg[(size_t)i * G + j] != 0.0) {
                pp->neg_col[nneg] = j;
                pp->neg_val[nneg++] = pp->Aneg[(size_t)i * G + j];
            }
        }
    }
    pp->pos_ptr[G] = (int32_t)npos;
    pp->neg_ptr[G] = (int32_t)nneg;
    pp->inv_on = (float*)calloc(G, 4);
    pp->inv_off = (float*)calloc(G, 4);
    pp->thr_init = (uint32_t*)calloc(G, 4);
    pp->tel = (uint8_t*)calloc(G, 1);
    pp->init_rand = (uint8_t*)calloc(G, 1);
    pp->bursty = 0;
    for (int g = 0; g < G; ++g) {
        double kon = net->k_on[g], koff = net->k_off[g];
        if (isfinite(kon) || isfinite(koff)) pp->bursty = 1;
        pp->tel[g] = isfinite(kon) ? 1 : 0;
        pp->init_rand[g] = (isfinite(kon) && isfinite(koff)) ? 1 : 0;
        pp->inv_on[g] = (float)(-ORC_LN2 / (kon * dt));
        pp->inv_off[g] = (float)(-ORC_LN2 / (koff * dt));
        if (pp->init_rand[g]) pp->thr_init[g] = prob_threshold(kon / (kon + koff));
    }
}

static void prep_free(prep_t* pp) {
    free(pp->Apos); free(pp->Aneg); free(pp->pos_ptr); free(pp->pos_col); free(pp->pos_val);
    free(pp->neg_ptr); free(pp->neg_col); free(pp->neg_val); free(pp->inv_on); free(pp->inv_off);
    free(pp->thr_init); free(pp->tel); free(pp->init_rand);
}

typedef struct {
    double k_t, Kn, hill_n, mu_m, mu_p, dt, sqrt_dt;
} coef_t;

/* Regulatory input of every gene from the protein levels p: Hill fractions (cle.jl:79-82),
 * reg = A_pos*act + A_neg*rep over the nonzero columns of each row (cle.jl:84-86), then the
 * cooperative / redundant corrections (cle.jl:89-106). */
static void regulation(const orc_net* net, const prep_t* pp, const coef_t* cf, const double* p, double* act,
                       double* rep, double* reg) {
    int G = net->G;
    /* Hill fractions */
    for (int g = 0; g < G; ++g) {
        double pn = pow(p[g], cf->hill_n);
        double den = pn + cf->Kn;
        act[g] = pn / den;
        rep[g] = cf->Kn / den;
    }
    /* reg = A_pos*act + A_neg*rep (cle.jl:84-86), over the nonzero columns of each row */
    for (int i = 0; i < G; ++i) {
        double s1 = 0.0, s2 = 0.0;
        for (int k = pp->pos_ptr[i]; k < pp->pos_ptr[i + 1]; ++k) s1 = s1 + pp->pos_val[k] * act[pp->pos_col[k]];
        for (int k = pp->neg_ptr[i]; k < pp->neg_ptr[i + 1]; ++k) s2 = s2 + pp->neg_val[k] * rep[pp->neg_col[k]];
        reg[i] = s1 + s2;
    }
    /* cooperative / redundant corrections (cle.jl:89-106) */
    for (int e = 0; e < net->n_coop; ++e) {
        double prod = 1.0;
        for (int k = net->coop_ptr[e]; k < net->coop_ptr[e + 1]; ++k) prod = prod * act[net->coop_src[k]];
        int t = net->coop_target[e];
        reg[t] = reg[t] + net->coop_strength[e] * net->basals[t] * prod;
    }
    for (int e = 0; e < net->n_redun; ++e) {
        double prod = 1.0;
        for (int k = net->redun_ptr[e]; k < net->redun_ptr[e + 1]; ++k)
            prod = prod * (1.0 - act[net->redun_src[k]]);
        int t = net->redun_target[e];
        reg[t] = reg[t] + net->redun_strength[e] * net->basals[t] * (1.0 - prod);
    }
}

/* One Euler-Maruyama step for one cell (cle.jl:78-121; population form cle.jl:185-234
 * when vol > 0).  m, p, on are this cell's G-vectors; act/rep/reg are scratch. */
static void cell_step(const orc_net* net, const prep_t* pp, const coef_t* cf, uint64_t seed,
                      uint32_t stream, uint32_t cell, uint32_t step, double vol, double* m,
                      double* p, uint8_t* on, sw_t* sw, double* act, double* rep, double* reg) {
    int G = net->G;
    /* telegraph switching before the transcription update (tauleap_binomial.jl:111-121):
     * the per-step Bernoulli(1 - exp(-k dt)) switch is sampled as its geometric waiting
     * time (one switch ahead, see sw_t), from the spare bits of the gene's normal words
     * of the switch step. */
    if (pp->bursty) {
        for (int g = 0; g < G; ++g) {
            if (!pp->tel[g] || (int64_t)step != sw[g].ns) continue;
            on[g] ^= 1;
            uint32_t w[4];
            draw(seed, cell, step, (uint32_t)(g >> 1), ORC_TAG_NORMAL, stream, w);
            float u = (g & 1) ? orc_switch_uniform(w[2], w[3]) : orc_switch_uniform(w[0], w[1]);
            sw[g].ns = clamp_step((int64_t)step + sw[g].kn);
            sw[g].kn = orc_geom_steps_u(u, on[g] ? pp->inv_on[g] : pp->inv_off[g]);
        }
    }
    regulation(net, pp, cf, p, act, rep, reg);
    /* M then P update with the new M (cle.jl:109-120) */
    for (int g = 0; g < G; ++g) {
        uint32_t w[4];
        double zm, zp;
        /* one Philox block serves genes 2k (words 0,1) and 2k+1 (words 2,3) */
        draw(seed, cell, step, (uint32_t)(g >> 1), ORC_TAG_NORMAL, stream, w);
        if (g & 1) box_muller(w[2], w[3], &zm, &zp);
        else box_muller(w[0], w[1], &zm, &zp);

        double tx = reg[g] + net->basals[g];
        if (vol > 0.0) tx = tx * vol;
        if (pp->bursty && !on[g]) tx = 0.0;
        double mg = m[g], pg = p[g];
        double var_m = tx + cf->mu_m * (mg > 0.0 ? mg : 0.0);
        if (!(var_m > 0.0)) var_m = 0.0;
        double nm = zm * cf->sqrt_dt * sqrt(var_m);
        mg = mg + (tx - cf->mu_m * mg) * cf->dt + nm;
        if (!(mg > 0.0)) mg = 0.0;
        double var_p = cf->k_t * (mg > 0.0 ? mg : 0.0) + cf->mu_p * (pg > 0.0 ? pg : 0.0);
        if (!(var_p > 0.0)) var_p = 0.0;
        double np_ = zp * cf->sqrt_dt * sqrt(var_p);
        pg = pg + (cf->k_t * mg - cf->mu_p * pg) * cf->dt + np_;
        if (!(pg > 0.0)) pg = 0.0;
        m[g] = mg;
        p[g] = pg;
    }
}

/* Initial promoter states (tauleap_binomial.jl:64-76) and first switch times. */
static void init_promoters(const prep_t* pp, uint64_t seed, uint32_t stream, uint32_t cell,
                           uint8_t* on, sw_t* sw) {
    int G = pp->G;
    for (int g0 = 0; g0 < G; g0 += 4) {
        uint32_t w[4];
        int any = 0;
        for (int g = g0; g < G && g < g0 + 4; ++g) any |= pp->init_rand[g];
        if (any) draw(seed, cell, 0, (uint32_t)(g0 >> 2), ORC_TAG_PROMOTER, stream, w);
        for (int g = g0; g < G && g < g0 + 4; ++g)
            on[g] = pp->init_rand[g] ? (w[g - g0] < pp->thr_init[g]) : 1;
    }
    for (int g = 0; g < G; ++g) {
        sw[g].ns = sw[g].kn = 2147483647;
        if (!pp->tel[g]) continue;
        uint32_t w[4];
        draw(seed, cell, 0, (uint32_t)g, ORC_TAG_SWITCH, stream, w);
        fresh_switch(&sw[g], 0, w, on[g], pp->inv_on[g], pp->inv_off[g]);
    }
}


/* ---------------------------------------------------------------------------
 * GPU binomial tau-leap (ext/SyntheticscRNAseqCUDAExt.jl:215-399, population :531-651),
 * in FP32 like the reference's kernels.  Every FP32 operation below is one IEEE operation
 * (this file is compiled without FMA contraction; fmaf is the fused one), so the library's
 * device code, written with the same explicitly rounded operations, returns the same bits.
 * ------------------------------------------------------------------------- */

/* exp(x) for x <= 0 from its definition: x = k ln2 + r with k = rint(x log2 e) and |r| <=
 * ln2/2 (two-constant Cody-Waite reduction), e^r by its Taylor series to r^7 (Horner), then
 * the exact scaling by 2^k (in two steps below 2^-126, so subnormal results round once). */
float orc_expf(float x) {
    if (!(x > -104.0f)) return 0.0f;
    if (x > 0.0f) x = 0.0f;
    const float k = rintf(x * 1.44269502162933349609375f);
    float r = fmaf(-k, 0.693145751953125f, x);       /* ln2 high part: 11 significant bits */
    r = fmaf(-k, 1.428606765330187045e-06f, r);        /* ln2 - high part */
    float q = fmaf(r, 1.0f / 5040.0f, 1.0f / 720.0f);
    q = fmaf(r, q, 1.0f / 120.0f);
    q = fmaf(r, q, 1.0f / 24.0f);
    q = fmaf(r, q, 1.0f / 6.0f);
    q = fmaf(r, q, 0.5f);
    q = fmaf(r, q, 1.0f);
    q = fmaf(r, q, 1.0f);
    int ki = (int)k;
    if (ki < -125) {
        q = q * f_of_bits(0x1F800000u); /* 2^-64, exact: q >= 2^-1 */
        ki += 64;
    }
    return q * f_of_bits((uint32_t)(ki + 127) << 23);
}

/* Poisson(lam) by inverse CDF over the first 50 terms (ext:21-31): the number of partial
 * sums of exp(-lam) lam^j / j! (j < k) that the uniform u exceeds, at most 50. */
float orc_poisson_icdf(float u, float lam) {
    float term = orc_expf(-lam);
    float cdf = term;
    float events = 0.0f;
    for (int k = 1; k <= 50; ++k) {
        if (!(u > cdf)) break; /* the partial sums never decrease: no later term counts */
        events = (float)k;
        term = term * (lam / (float)k);
        cdf = cdf + term;
    }
    return events;
}

/* The four uniforms of a (cell, step, gene) tau-leap block: (w >> 9) 2^-23 in [0, 1). */
static inline float tau_uniform(uint32_t w) { return (float)(w >> 9) * 1.1920928955078125e-07f; }

typedef struct {
    float k_t, dt, p_dec_m, p_dec_p;
} tcoef_t;

/* One tau-leap step for one cell (ext:250-275; population form ext:586-612 when vol > 0:
 * Hill of the concentration p / V, transcription scaled by V).  m, p hold counts. */
static void tau_cell_step(const orc_net* net, const prep_t* pp, const coef_t* cf, const tcoef_t* tc,
                          uint64_t seed, uint32_t stream, uint32_t cell, uint32_t step, double vol, double* m,
                          double* p, uint8_t* on, sw_t* sw, double* conc, double* act, double* rep, double* reg) {
    int G = net->G;
    if (pp->bursty) {
        for (int g = 0; g < G; ++g) {
            if (!pp->tel[g] || (int64_t)step != sw[g].ns) continue;
            on[g] ^= 1;
            uint32_t w[4];
            draw(seed, cell, step, (uint32_t)g, ORC_TAG_TAU, stream, w);
            float u = orc_switch_uniform(w[0], w[1]);
            sw[g].ns = clamp_step((int64_t)step + sw[g].kn);
            sw[g].kn = orc_geom_steps_u(u, on[g] ? pp->inv_on[g] : pp->inv_off[g]);
        }
    }
    const float vf = (float)vol;
    for (int g = 0; g < G; ++g) conc[g] = vol > 0.0 ? (double)((float)p[g] / vf) : p[g];
    regulation(net, pp, cf, conc, act, rep, reg);
    for (int g = 0; g < G; ++g) {
        uint32_t w[4];
        draw(seed, cell, step, (uint32_t)g, ORC_TAG_TAU, stream, w);
        float M = (float)m[g], P = (float)p[g];
        float tx = (float)(reg[g] + net->basals[g]);
        tx = tx > 0.0f ? tx : 0.0f;
        if (vol > 0.0) tx = tx * vf;
        float lam = tx * tc->dt;
        if (pp->bursty && !on[g]) lam = 0.0f;
        const float n_tx = orc_poisson_icdf(tau_uniform(w[0]), lam);
        const float mp = M > 0.0f ? M : 0.0f;
        float n_md = orc_poisson_icdf(tau_uniform(w[1]), mp * tc->p_dec_m);
        n_md = n_md < mp ? n_md : mp;
        M = (M + n_tx) - n_md;
        M = M > 0.0f ? M : 0.0f;
        const float n_tl = orc_poisson_icdf(tau_uniform(w[2]), (tc->k_t * M) * tc->dt);
        const float pp_ = P > 0.0f ? P : 0.0f;
        float n_pd = orc_poisson_icdf(tau_uniform(w[3]), pp_ * tc->p_dec_p);
        n_pd = n_pd < pp_ ? n_pd : pp_;
        P = (P + n_tl) - n_pd;
        P = P > 0.0f ? P : 0.0f;
        m[g] = M;
        p[g] = P;
    }
}

static int simulate_impl(const orc_net* net, const orc_kin* kin, const orc_pop* pop,
                         const orc_opts* opt, double* M, double* P, double* V, uint8_t* prom,
                         int nthreads, int tau) {
    int G = net->G;
    int64_t N = opt->cell_num;
    if (G <= 0 || N <= 0 || !(opt->dt > 0.0)) return 1;
    if (pop && N < 2 && pop->exclude_mother) return 1;
    if (pop && pop->div_check_interval <= 0) return 1;
    int64_t n_steps = opt->n_steps > 0 ? opt->n_steps : (int64_t)ceil(opt->T / opt->dt);

    prep_t pp;
    prep_build(net, opt->dt, &pp);
    coef_t cf;
    cf.k_t = kin->k_t;
    cf.Kn = pow(kin->K_d, kin->n);
    cf.hill_n = kin->n;
    /* plain CLE: decay includes dilution (cle.jl:60-61); population: intrinsic only (cle.jl:166-167) */
    cf.mu_m = pop ? kin->mu_m : kin->mu_m + kin->dilution;
    cf.mu_p = pop ? kin->mu_p : kin->mu_p + kin->dilution;
    cf.dt = opt->dt;
    cf.sqrt_dt = sqrt(opt->dt);
    /* tau-leap: FP32 rates; decay probabilities 1 - exp(-mu dt), with dilution unless a
     * population makes it emergent (ext:240-241, ext:574-575) */
    tcoef_t tc;
    tc.k_t = (float)kin->k_t;
    tc.dt = (float)opt->dt;
    tc.p_dec_m = (float)(1.0 - exp(-(pop ? kin->mu_m : kin->mu_m + kin->dilution) * opt->dt));
    tc.p_dec_p = (float)(1.0 - exp(-(pop ? kin->mu_p : kin->mu_p + kin->dilution) * opt->dt));

    /* initial condition: ceil of the steady state (cle.jl:49-53, kinetics.jl:65-70, ext:230-236);
     * tau-leap populations: max(1, round(steady state x V)) per cell (ext:560-566) */
    double* m0 = (double*)malloc(sizeof(double) * G);
    double* p0 = (double*)malloc(sizeof(double) * G);
    double* mss = (double*)malloc(sizeof(double) * G);
    double* pss = (double*)malloc(sizeof(double) * G);
    for (int g = 0; g < G; ++g) {
        mss[g] = net->basals[g] / (kin->mu_m + kin->dilution);
        pss[g] = kin->k_t * mss[g] / (kin->mu_p + kin->dilution);
        m0[g] = ceil(mss[g]);
        p0[g] = ceil(pss[g]);
    }
    uint64_t seed = opt->seed;
    uint32_t stream = opt->stream;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif

    if (!pop) {
        /* cells are independent: cell-major loop, parallel over cells */
#pragma omp parallel
        {
            double* m = (double*)malloc(sizeof(double) * G);
            double* p = (double*)malloc(sizeof(double) * G);
            double* act = (double*)malloc(sizeof(double) * G);
            double* rep = (double*)malloc(sizeof(double) * G);
            double* reg = (double*)malloc(sizeof(double) * G);
            double* conc = (double*)malloc(sizeof(double) * G);
            uint8_t* on = (uint8_t*)malloc(G);
            sw_t* ns = (sw_t*)malloc(sizeof(sw_t) * G);
#pragma omp for schedule(static)
            for (int64_t c = 0; c < N; ++c) {
                memcpy(m, m0, sizeof(double) * G);
                memcpy(p, p0, sizeof(double) * G);
                const uint32_t gc = (uint32_t)(opt->cell_offset + c);
                init_promoters(&pp, seed, stream, gc, on, ns);
                for (int64_t s = 1; s <= n_steps; ++s) {
                    if (tau)
                        tau_cell_step(net, &pp, &cf, &tc, seed, stream, gc, (uint32_t)s, 0.0, m, p, on, ns, conc,
                                      act, rep, reg);
                    else
                        cell_step(net, &pp, &cf, seed, stream, gc, (uint32_t)s, 0.0, m, p, on, ns, act, rep, reg);
                }
                for (int g = 0; g < G; ++g) {
                    M[(size_t)g * N + c] = m[g];
                    P[(size_t)g * N + c] = p[g];
                    if (prom) prom[(size_t)g * N + c] = on[g];
                }
            }
            free(m); free(p); free(act); free(rep); free(reg); free(conc); free(on); free(ns);
        }
    } else {
        /* population: cells in lockstep, state cell-major [c][g] for the step loop */
        double* Ms = (double*)malloc(sizeof(double) * G * N);
        double* Ps = (double*)malloc(sizeof(double) * G * N);
        uint8_t* On = (uint8_t*)malloc((size_t)G * N);
        sw_t* Ns = (sw_t*)malloc(sizeof(sw_t) * G * N);
        double* Vs = (double*)malloc(sizeof(double) * N);
        double growth_factor = exp(pop->growth_rate * opt->dt);
        for (int64_t c = 0; c < N; ++c) {
            memcpy(Ms + c * G, m0, sizeof(double) * G);
            memcpy(Ps + c * G, p0, sizeof(double) * G);
            init_promoters(&pp, seed, stream, (uint32_t)c, On + c * G, Ns + c * G);
            uint32_t w[4];
            draw(seed, (uint32_t)c, 0, 0, ORC_TAG_VOLUME, stream, w);
            Vs[c] = pop->V_lo + (pop->V_hi - pop->V_lo) * u53(w[0], w[1]); /* cle.jl:158-159 */
            if (tau)
                for (int g = 0; g < G; ++g) {
                    const double mi = rint(mss[g] * Vs[c]), pi = rint(pss[g] * Vs[c]);
                    Ms[c * G + g] = mi > 1.0 ? mi : 1.0;
                    Ps[c * G + g] = pi > 1.0 ? pi : 1.0;
                }
        }
        int64_t* dividers = (int64_t*)malloc(sizeof(int64_t) * N);
        double* dM = (double*)malloc(sizeof(double) * G * N);
        double* dP = (double*)malloc(sizeof(double) * G * N);
        uint8_t* dOn = (uint8_t*)malloc((size_t)G * N);
        sw_t* dNs = (sw_t*)malloc(sizeof(sw_t) * G * N);
        double* dV = (double*)malloc(sizeof(double) * N);
        for (int64_t s = 1; s <= n_steps; ++s) {
#pragma omp parallel
            {
                double* act = (double*)malloc(sizeof(double) * G);
                double* rep = (double*)malloc(sizeof(double) * G);
                double* reg = (double*)malloc(sizeof(double) * G);
                double* conc = (double*)malloc(sizeof(double) * G);
#pragma omp for schedule(static)
                for (int64_t c = 0; c < N; ++c) {
                    if (tau)
                        tau_cell_step(net, &pp, &cf, &tc, seed, stream, (uint32_t)c, (uint32_t)s, Vs[c], Ms + c * G,
                                      Ps + c * G, On + c * G, Ns + c * G, conc, act, rep, reg);
                    else
                        cell_step(net, &pp, &cf, seed, stream, (uint32_t)c, (uint32_t)s, Vs[c],
                                  Ms + c * G, Ps + c * G, On + c * G, Ns + c * G, act, rep, reg);
                    Vs[c] = Vs[c] * growth_factor; /* cle.jl:237 */
                }
                free(act); free(rep); free(reg); free(conc);
            }
            if (s % pop->div_check_interval != 0) continue;
            /* division (cle.jl:240-273) */
            int64_t nd = 0;
            for (int64_t c = 0; c < N; ++c)
                if (Vs[c] > pop->V_div) dividers[nd++] = c;
            for (int64_t k = 0; k < nd; ++k) {
                int64_t c = dividers[k];
                for (int g = 0; g < G; ++g) {
                    double* mm = Ms + c * G + g;
                    double* pq = Ps + c * G + g;
                    if (pop->partition == 1) {
                        double hm = *mm / 2.0, hp = *pq / 2.0;
                        *mm = hm; dM[k * G + g] = hm;
                        *pq = hp; dP[k * G + g] = hp;
                    } else {
                        int64_t mi = (int64_t)rint(*mm);
                        int64_t mmth = mi > 0 ? orc_binomial_half(mi, seed, stream, (uint32_t)c,
                                                                  (uint32_t)s, (uint32_t)g, 0) : 0;
                        *mm = (double)mmth; dM[k * G + g] = (double)(mi - mmth);
                        int64_t pi = (int64_t)rint(*pq);
                        int64_t pmth = pi > 0 ? orc_binomial_half(pi, seed, stream, (uint32_t)c,
                                                                  (uint32_t)s, (uint32_t)g, 1) : 0;
                        *pq = (double)pmth; dP[k * G + g] = (double)(pi - pmth);
                    }
                    dOn[k * G + g] = On[c * G + g];
                    /* the daughter's switching is independent of the mother's: fresh waiting time */
                    dNs[k * G + g].ns = dNs[k * G + g].kn = 2147483647;
                    if (pp.tel[g]) {
                        uint32_t w[4];
                        draw(seed, (uint32_t)c, (uint32_t)s, (uint32_t)g | 0x800000u, ORC_TAG_SWITCH, stream, w);
                        fresh_switch(&dNs[k * G + g], s, w, dOn[k * G + g], pp.inv_on[g], pp.inv_off[g]);
                    }
                }
                Vs[c] = Vs[c] / 2.0;
                dV[k] = Vs[c];
            }
            for (int64_t k = 0; k < nd; ++k) {
                int64_t c = dividers[k];
                uint32_t w[4];
                draw(seed, (uint32_t)c, (uint32_t)s, 0, ORC_TAG_MORAN, stream, w);
                int64_t r;
                if (pop->exclude_mother) {
                    r = (int64_t)(((uint64_t)w[0] * (uint64_t)(N - 1)) >> 32);
                    if (r >= c) r += 1;
                } else {
                    r = (int64_t)(((uint64_t)w[0] * (uint64_t)N) >> 32);
                }
                memcpy(Ms + r * G, dM + k * G, sizeof(double) * G);
                memcpy(Ps + r * G, dP + k * G, sizeof(double) * G);
                memcpy(On + r * G, dOn + k * G, (size_t)G);
                memcpy(Ns + r * G, dNs + k * G, sizeof(sw_t) * G);
                Vs[r] = dV[k];
            }
        }
        for (int64_t c = 0; c < N; ++c) {
            for (int g = 0; g < G; ++g) {
                M[(size_t)g * N + c] = Ms[c * G + g];
                P[(size_t)g * N + c] = Ps[c * G + g];
                if (prom) prom[(size_t)g * N + c] = On[c * G + g];
            }
            if (V) V[c] = Vs[c];
        }
        free(Ms); free(Ps); free(On); free(Ns); free(dNs); free(Vs); free(dividers); free(dM); free(dP);
        free(dOn); free(dV);
    }
    free(m0); free(p0); free(mss); free(pss);
    prep_free(&pp);
    return 0;
}

int orc_cle_simulate(const orc_net* net, const orc_kin* kin, const orc_pop* pop, const orc_opts* opt,
                     double* M, double* P, double* V, uint8_t* prom, int nthreads) {
    return simulate_impl(net, kin, pop, opt, M, P, V, prom, nthreads, 0);
}

int orc_tauleap_simulate(const orc_net* net, const orc_kin* kin, const orc_pop* pop, const orc_opts* opt,
                         double* M, double* P, double* V, uint8_t* prom, int nthreads) {
    return simulate_impl(net, kin, pop, opt, M, P, V, prom, nthreads, 1);
}

/* ---------------------------------------------------------------------------
 * Capture (capture.jl:25-47)
 * ------------------------------------------------------------------------- */
void orc_capture_efficiency(int64_t N, double efficiency, double efficiency_std,
                            int32_t mean_correction, uint64_t seed, uint32_t stream,
                            double* eff) {
    double mu_log = log(efficiency);
    if (mean_correction) mu_log = mu_log - efficiency_std * efficiency_std / 2.0;
    for (int64_t c = 0; c < N; ++c) {
        uint32_t w[4];
        draw(seed, (uint32_t)c, 0, 0, ORC_TAG_EFFICIENCY, stream, w);
        double z0, z1;
        box_muller(w[0], w[1], &z0, &z1);
        double p = exp(mu_log + efficiency_std * z0);
        if (p < 0.0) p = 0.0;
        if (p > 1.0) p = 1.0;
        eff[c] = p;
    }
}

void orc_capture_counts(int64_t N, int32_t G, const double* X, const double* eff,
                        uint64_t seed, uint32_t stream, int32_t* Y, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < N; ++c) {
        for (int g = 0; g < G; ++g) {
            double x = rint(X[(size_t)g * N + c]);
            int64_t n = x > 0.0 ? (int64_t)x : 0;
            double p = eff[c];
            int64_t y = 0;
            if (n > 0 && p != 0.0) y = orc_binomial_invcdf(n, p, seed, stream, (uint32_t)c, (uint32_t)g);
            Y[(size_t)g * N + c] = (int32_t)y;
        }
    }
}
