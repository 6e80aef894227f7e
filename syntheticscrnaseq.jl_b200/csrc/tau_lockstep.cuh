// Binomial tau-leap update of the genes of one thread unit (a quad or a pair), with the
// Poisson draws either in lock step or one after another.  Each draw is the 50-term inverse CDF of poisson_icdf50 (the
// reference's GPU sampler, ext/SyntheticscRNAseqCUDAExt.jl:21-39) with the same operations
// in the same order, and its quotients lam / k are the correctly rounded ones (small_div.cuh,
// or IEEE division outside its range), so every count is bit-identical to poisson_icdf50's;
// only the schedule changes.
//
// Lock step: of a gene's four draws, translation needs the new mRNA count and the other three
// only the state at the start of the step.  The unit's transcription and mRNA-decay draws
// share one loop, then its translation and protein-decay draws a second: near the steady
// state the two draws of a loop have about the same Poisson mean (transcription balances
// mRNA decay, translation protein decay), so few terms are spent on chains that have stopped.
// Each chain's count is the last k whose preceding partial sum u exceeds, and a loop ends
// (checked every second term) when u exceeds no chain's partial sum or after 50 terms.  A
// loop issues 2 QG x its longest chain's terms instead of the sum of its chains' terms, in
// exchange for 2 QG independent chains in flight.
#pragma once

#include "cle_device.cuh"
#include "small_div.cuh"

namespace scrna {

// poisson_icdf50 with the branch-free quotient (same result).
__device__ __forceinline__ float poisson_icdf50_fast(float u, float lam) {
    if (!small_div_ok(lam)) return poisson_icdf50(u, lam);
    float term = own_expf(-lam);
    float cdf = term;
    float events = 0.0f;
    for (int k = 1; k <= 50; ++k) {
        if (!(u > cdf)) break;
        const float kf = (float)k;
        events = kf;
        term = __fmul_rn(term, small_div(lam, kf, kRecipSmall[k]));
        cdf = __fadd_rn(cdf, term);
    }
    return events;
}

template <int C>
__device__ __forceinline__ void poisson_icdf50_lockstep(const float (&u)[C], const float (&lam)[C],
                                                        float (&events)[C]) {
    bool ok = true;
#pragma unroll
    for (int c = 0; c < C; ++c) ok &= small_div_ok(lam[c]);
    if (!ok) {
#pragma unroll
        for (int c = 0; c < C; ++c) events[c] = poisson_icdf50(u[c], lam[c]);
        return;
    }
    float term[C], cdf[C];
    bool any = false;
#pragma unroll
    for (int c = 0; c < C; ++c) {
        term[c] = own_expf(-lam[c]);
        cdf[c] = term[c];
        events[c] = 0.0f;
        any |= u[c] > cdf[c];
    }
    // A stopped chain keeps adding terms: they are >= 0 and rounding is monotone, so its
    // partial sum never falls back below u and its count stays where it stopped.
    for (int k = 1; k <= 50 && any; k += 2) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const float kf = (float)(k + h);
            const float y = kRecipSmall[k + h];
#pragma unroll
            for (int c = 0; c < C; ++c) {
                events[c] = u[c] > cdf[c] ? kf : events[c];
                term[c] = __fmul_rn(term[c], small_div(lam[c], kf, y));
                cdf[c] = __fadd_rn(cdf[c], term[c]);
            }
        }
        any = false;
#pragma unroll
        for (int c = 0; c < C; ++c) any |= u[c] > cdf[c];
    }
}

// One tau-leap step of the first `ng` genes of a unit of QG (4 or 2) genes (tau_update per
// gene: transcription Poisson(lam_tx), mRNA decay min(Poisson(m p_m), m), translation
// Poisson(k_t m' dt) with the new m', protein decay min(Poisson(p p_p), p); counts never
// below 0).  w[i] holds gene i's four words; in lock step a slot without a gene passes u = 0
// (no events) and keeps m = p = 0.
template <int QG>
__device__ __forceinline__ void tau_update_unit(float (&m)[QG], float (&p)[QG], const float (&lam_tx)[QG],
                                                const uint4 (&w)[QG], int ng, bool lockstep, float k_t, float dt,
                                                float p_dec_m, float p_dec_p) {
    if (!lockstep) {
#pragma unroll
        for (int i = 0; i < QG; ++i) {
            if (i >= ng) break;
            const float n_tx = poisson_icdf50_fast(tau_uniform(w[i].x), lam_tx[i]);
            const float mp = fmaxf(m[i], 0.0f);
            const float n_md = fminf(poisson_icdf50_fast(tau_uniform(w[i].y), __fmul_rn(mp, p_dec_m)), mp);
            const float mn = fmaxf(__fsub_rn(__fadd_rn(m[i], n_tx), n_md), 0.0f);
            const float n_tl = poisson_icdf50_fast(tau_uniform(w[i].z), __fmul_rn(__fmul_rn(k_t, mn), dt));
            const float pp = fmaxf(p[i], 0.0f);
            const float n_pd = fminf(poisson_icdf50_fast(tau_uniform(w[i].w), __fmul_rn(pp, p_dec_p)), pp);
            m[i] = mn;
            p[i] = fmaxf(__fsub_rn(__fadd_rn(p[i], n_tl), n_pd), 0.0f);
        }
        return;
    }
    // transcription and mRNA decay of the unit's genes
    float ua[2 * QG], la[2 * QG], na[2 * QG];
#pragma unroll
    for (int i = 0; i < QG; ++i) {
        ua[2 * i] = tau_uniform(w[i].x);
        la[2 * i] = lam_tx[i];
        ua[2 * i + 1] = tau_uniform(w[i].y);
        la[2 * i + 1] = __fmul_rn(fmaxf(m[i], 0.0f), p_dec_m);
    }
    poisson_icdf50_lockstep<2 * QG>(ua, la, na);
    // translation with the new mRNA counts, and protein decay
    float ub[2 * QG], lb[2 * QG], nb[2 * QG];
#pragma unroll
    for (int i = 0; i < QG; ++i) {
        const float n_md = fminf(na[2 * i + 1], fmaxf(m[i], 0.0f));
        m[i] = fmaxf(__fsub_rn(__fadd_rn(m[i], na[2 * i]), n_md), 0.0f);
        ub[2 * i] = tau_uniform(w[i].z);
        lb[2 * i] = __fmul_rn(__fmul_rn(k_t, m[i]), dt);
        ub[2 * i + 1] = tau_uniform(w[i].w);
        lb[2 * i + 1] = __fmul_rn(fmaxf(p[i], 0.0f), p_dec_p);
    }
    poisson_icdf50_lockstep<2 * QG>(ub, lb, nb);
#pragma unroll
    for (int i = 0; i < QG; ++i) {
        const float n_pd = fminf(nb[2 * i + 1], fmaxf(p[i], 0.0f));
        p[i] = fmaxf(__fsub_rn(__fadd_rn(p[i], nb[2 * i]), n_pd), 0.0f);
    }
}

}  // namespace scrna
