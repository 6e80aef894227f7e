/*
 * CPU oracle for the batched CLE path — TEST INFRASTRUCTURE ONLY.
 *
 * This is an FP64 restatement of the reference Julia CLE, used by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker.
 * Nothing in the shipped library links, loads or calls it.
 *
 * Reference lines it follows (paths inside Msturroc/SyntheticscRNAseq.jl):
 *   src/algorithms/cle.jl:46-129      plain CLE (Hill, A_pos/A_neg GEMMs, coop/redun, M then P update)
 *   src/algorithms/cle.jl:143-283     population CLE (volume growth, division, Moran replacement)
 *   src/network.jl:112-219            Hill functions, A_eff = A[i,j]*beta_i split into +/- parts
 *   src/kinetics.jl:65-70             deterministic steady state used as the initial condition
 *   src/algorithms/tauleap_binomial.jl:64-76,111-121,134-137 and
 *   scripts/generate_figures.jl:124-131  telegraph init / switching / transcription gating
 *   ext/SyntheticscRNAseqCUDAExt.jl:641-651  binomial partition of rounded counts at division
 *   src/capture.jl:25-47              LogNormal-Binomial capture
 *
 * Parity status: the reference is Julia, which is not installed here, so the
 * reference itself cannot be run.  The reference has no golden vectors; its
 * tests are statistical (closed-form moments with tolerance bands).  The
 * oracle is pinned against those bands (tests/test_oracle_moments.py) and its
 * Philox generator against the published Philox4x32-10 known-answer vectors.
 * Random streams are this project's own counter-based Philox streams, so
 * sample-level parity with Julia's MersenneTwister is not possible; the
 * oracle and the CUDA library consume identical increments.
 */
#ifndef SCRNA_CLE_ORACLE_H
#define SCRNA_CLE_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* GeneNetwork (src/network.jl:55-63). A is row-major: A[i*G+j] = effect of
 * protein j on gene i. Edge sources are 0-based and stored CSR-style. */
typedef struct {
    int32_t G;
    const double* basals;        /* [G] */
    const double* A;             /* [G*G] row-major */
    int32_t n_coop;
    const int32_t* coop_target;  /* [n_coop] */
    const int32_t* coop_ptr;     /* [n_coop+1] */
    const int32_t* coop_src;     /* [coop_ptr[n_coop]] */
    const double* coop_strength; /* [n_coop] */
    int32_t n_redun;
    const int32_t* redun_target;
    const int32_t* redun_ptr;
    const int32_t* redun_src;
    const double* redun_strength;
    const double* k_on;          /* [G], +inf = constitutive */
    const double* k_off;         /* [G] */
} orc_net;

/* KineticParams (src/kinetics.jl:25-32). */
typedef struct { double k_t, K_d, n, mu_m, mu_p, dilution; } orc_kin;

/* PopulationConfig (src/population.jl:27-34) + partition / Moran mode. */
typedef struct {
    double growth_rate, V_div, V_lo, V_hi;
    int32_t div_check_interval;
    int32_t partition;        /* 0 = binomial (ext:641-651), 1 = halve (cle.jl:249-261) */
    int32_t exclude_mother;   /* 1 = slot != mother (cle.jl:265-268), 0 = any (ext:509) */
} orc_pop;

typedef struct {
    double dt, T;
    int64_t cell_num;
    uint64_t seed;
    uint32_t stream;
    int64_t n_steps;          /* <=0: ceil(T/dt) as cle.jl:56; >0: run exactly this many steps */
    int64_t cell_offset;      /* global index of cell 0 (plain CLE only) */
} orc_opts;

/* Random-stream tags (bits 31..24 of Philox counter word 3). */
enum {
    ORC_TAG_NORMAL = 1, ORC_TAG_SWITCH = 2, ORC_TAG_PROMOTER = 3, ORC_TAG_VOLUME = 4,
    ORC_TAG_MORAN = 5, ORC_TAG_PARTITION = 6, ORC_TAG_EFFICIENCY = 7, ORC_TAG_CAPTURE = 8,
    ORC_TAG_TAU = 9
};

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* The two N(0,1) increments (z_m, z_p) of one (cell, step, gene). */
void orc_step_normals(uint64_t seed, uint32_t stream, uint32_t cell, uint32_t step,
                      uint32_t gene, double* zm, double* zp);

/* Simulate. M, P are [G][N] (index g*N + c). V may be NULL without population.
 * prom ([G][N], 0/1) may be NULL. Returns 0 on success. */
int orc_cle_simulate(const orc_net* net, const orc_kin* kin, const orc_pop* pop,
                     const orc_opts* opt, double* M, double* P, double* V,
                     uint8_t* prom, int nthreads);

/* GPU binomial tau-leap (ext/SyntheticscRNAseqCUDAExt.jl:215-399, population ext:531-651) in
 * FP32 as the reference's kernels compute it, with the CPU path's cooperative / redundant
 * edges and telegraph gating (tauleap_binomial.jl:84-137); same arguments and outputs as
 * orc_cle_simulate, M and P hold molecule counts. */
int orc_tauleap_simulate(const orc_net* net, const orc_kin* kin, const orc_pop* pop,
                         const orc_opts* opt, double* M, double* P, double* V,
                         uint8_t* prom, int nthreads);

/* exp(x) (x <= 0) and the 50-term Poisson inverse CDF of the tau-leap, bit-exact with the
 * library's device code. */
float orc_expf(float x);
float orc_poisson_icdf(float u, float lam);

/* Per-cell capture efficiency (capture.jl:30-36); mean_correction=1 subtracts sigma^2/2. */
void orc_capture_efficiency(int64_t N, double efficiency, double efficiency_std,
                            int32_t mean_correction, uint64_t seed, uint32_t stream,
                            double* eff);

/* Binomial capture of X ([G][N]) with per-cell efficiencies (capture.jl:37-44).
 * Y is [G][N] int32. Bit-exact restatement of the library's inverse-CDF sampler. */
void orc_capture_counts(int64_t N, int32_t G, const double* X, const double* eff,
                        uint64_t seed, uint32_t stream, int32_t* Y, int nthreads);

/* Binomial(n, p) by chunked inverse CDF given the chunk uniforms' Philox counter base. */
int64_t orc_binomial_invcdf(int64_t n, double p, uint64_t seed, uint32_t stream,
                            uint32_t cell, uint32_t gene);

/* log2 of u in [2^-24, 1] by the explicitly rounded FP32 atanh series, and the
 * geometric telegraph waiting time 1 + floor(log2(u) * inv) (>= 1 steps) for a uniform
 * u in (0, 1]: from a switch word, u = ((w>>8)+1) 2^-24 (initial and daughter waiting
 * times); at a switch step, u = orc_switch_uniform of the gene's two normal words. */
float orc_log2f(float u);
int32_t orc_geom_steps_u(float u, float inv);
int32_t orc_geom_steps(uint32_t w, float inv);
float orc_switch_uniform(uint32_t w0, uint32_t w1);

/* Binomial(n, 1/2) partition draw (popcount of n Philox bits). */
int64_t orc_binomial_half(int64_t n, uint64_t seed, uint32_t stream, uint32_t cell,
                          uint32_t step, uint32_t gene, uint32_t species);

#ifdef __cplusplus
}
#endif
#endif
