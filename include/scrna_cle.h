/*
 * scrna_cle.h — C ABI of the B200 batched Chemical Langevin Equation library
 * (libscrna_cle.so, sm_100a).
 *
 * The library replaces the GPU CLE of Msturroc/SyntheticscRNAseq.jl
 * (ext/SyntheticscRNAseqCUDAExt.jl) behind the package's own Julia interface.
 * Every entry point below names the reference function it stands in for.
 * Conventions:
 *   - All functions return an int status (SCRNA_OK == 0, negative on error);
 *     scrna_last_error() returns a thread-local message for the last failure.
 *   - Host arrays follow Julia: matrices are column-major.  The interaction
 *     matrix A is G x G with A[i + j*G] = effect of protein j on gene i
 *     (src/network.jl:44-45).  Edge gene indices are `index_base`-based
 *     (1 for Julia callers, 0 for C callers).
 *   - Output matrices are cells x G (or cells x 2G for SCRNA_READOUT_BOTH),
 *     column-major, exactly the Matrix{Float64} the reference returns
 *     (src/algorithms/cle.jl:123-129).  Count matrices are cells x G int32.
 *   - The caller owns host buffers; the library owns device memory and frees
 *     it in the matching *_destroy call.
 *   - A context is bound to one device and one CUDA stream; calls on one
 *     context must not run concurrently from several threads.
 */
#ifndef SCRNA_CLE_H
#define SCRNA_CLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SCRNA_ABI_VERSION 1

enum scrna_status {
    SCRNA_OK = 0,
    SCRNA_EINVAL = -1,    /* bad argument (reference: @assert / error(), src/network.jl:66-68) */
    SCRNA_ENOMEM = -2,    /* device or host allocation failed, or admission refused */
    SCRNA_ECUDA = -3,     /* CUDA runtime error */
    SCRNA_ETIMEOUT = -4,  /* wait ran out of time */
    SCRNA_EBUSY = -5,     /* queue full / request still running */
    SCRNA_ENOTSUP = -6,   /* configuration not supported by this build */
    SCRNA_ECANCELED = -7  /* request was cancelled */
};

enum scrna_readout { SCRNA_READOUT_MRNA = 0, SCRNA_READOUT_PROTEIN = 1, SCRNA_READOUT_BOTH = 2 };

/* Division partition: binomial split of rounded counts (ext/SyntheticscRNAseqCUDAExt.jl:641-651)
 * or deterministic halving (src/algorithms/cle.jl:249-261). */
enum scrna_partition { SCRNA_PARTITION_BINOMIAL = 0, SCRNA_PARTITION_HALVE = 1 };

/* Arithmetic of a run: the FP32 path (its tensor-core contraction at large dense G takes
 * BF16 inputs, or FP16 inputs with SCRNA_PRECISION_FP32_F16), or the plain FP64
 * one-kernel-per-step path kept as the comparison baseline. */
enum scrna_precision {
    SCRNA_PRECISION_FP32 = 0, SCRNA_PRECISION_FP64_PLAIN = 1, SCRNA_PRECISION_FP32_F16 = 2
};

/* Kernel family for the FP32 precision.  AUTO picks the register path for sparse
 * networks (the lane-per-gene-unit kernel when the network fits it, G <= 512, block tiles
 * otherwise) and the tensor-core path for dense ones (>= 5 % of the G x G edges over >= 256
 * genes; at up to 256 genes from 8,192 cells) and for networks the register path cannot hold
 * (more than 512 genes, or tables beyond shared memory).  BLOCK and WARP force one
 * register-path kernel (both give identical results).  TENSOR is the fused tcgen05
 * contraction + Euler step; TENSOR_LIBRARY the same step with the contraction done by a
 * library GEMM (cuBLASLt) and a separate update kernel, kept for comparison. */
enum scrna_path {
    SCRNA_PATH_AUTO = 0, SCRNA_PATH_REGISTER = 1, SCRNA_PATH_TENSOR = 2,
    SCRNA_PATH_BLOCK = 3, SCRNA_PATH_WARP = 4, SCRNA_PATH_TENSOR_LIBRARY = 5
};

typedef struct scrna_ctx scrna_ctx;
typedef struct scrna_net scrna_net;
typedef struct scrna_state scrna_state;

/* KineticParams (src/kinetics.jl:25-32). */
typedef struct {
    double k_t, K_d, n, mu_m, mu_p, dilution;
} scrna_kinetics;

/* PopulationConfig (src/population.jl:27-34) plus the partition and Moran modes.
 * exclude_mother = 1 picks the replaced slot among the other N-1 cells
 * (src/algorithms/cle.jl:265-268); 0 picks any cell (ext/SyntheticscRNAseqCUDAExt.jl:509). */
typedef struct {
    int64_t cell_num;
    double growth_rate;
    double V_div;
    double V_init_lo, V_init_hi;
    int32_t div_check_interval;
    int32_t partition;        /* enum scrna_partition */
    int32_t exclude_mother;
    int32_t reserved;
    double growth_noise;      /* accepted for interface parity; the CLE ignores it (cle.jl:237) */
} scrna_population;

/* CaptureModel (src/population.jl:57-61).  mean_correction = 1 uses the reference's
 * mu_log = log(efficiency) - sigma^2/2 (src/capture.jl:30); 0 uses mu_log = log(efficiency). */
typedef struct {
    double efficiency, efficiency_std;
    int32_t readout;          /* SCRNA_READOUT_MRNA or SCRNA_READOUT_PROTEIN */
    int32_t mean_correction;
} scrna_capture;

/* CLE(dt) (src/algorithms/cle.jl:21-23) plus the simulate keywords (cle.jl:34-39). */
typedef struct {
    double dt;
    double T;
    int64_t cell_num;         /* ignored when a population config is given (pop.cell_num wins) */
    int32_t readout;          /* enum scrna_readout */
    int32_t precision;        /* enum scrna_precision */
    uint64_t seed;            /* Philox key */
    uint32_t stream;          /* Philox stream id (24 bits); distinct per network in a batch */
    int32_t path;             /* enum scrna_path */
    int64_t n_steps;          /* <= 0: ceil(T/dt) (cle.jl:56); > 0: exactly this many steps */
    int64_t cell_offset;      /* global index of cell 0 (cell sharding across GPUs) */
} scrna_cle_opts;

/* ---- library / context ---------------------------------------------------- */
const char* scrna_last_error(void);
int scrna_version(void);
int scrna_ctx_create(int device, scrna_ctx** out);
int scrna_ctx_destroy(scrna_ctx* ctx);
/* Use the caller's cudaStream_t (passed as void*) for all work of this context. */
int scrna_ctx_set_stream(scrna_ctx* ctx, void* cuda_stream);
int scrna_ctx_synchronize(scrna_ctx* ctx);
/* Number of kernels this context has launched so far. */
int64_t scrna_ctx_launch_count(const scrna_ctx* ctx);
/* Bytes this context's calls have copied host -> device (network tables, per-run gene
 * tables) and device -> host (results) so far.  No counterpart in the reference: it lets a
 * caller account for the transfers of an end-to-end call. */
int scrna_ctx_transfer_bytes(const scrna_ctx* ctx, int64_t* h2d, int64_t* d2h);

/* ---- networks ---------------------------------------------------------------
 * Uploads a GeneNetwork (src/network.jl:55-63): basals, A, cooperative and
 * redundant edges (network.jl:16-34), telegraph rates k_on/k_off (+Inf =
 * constitutive).  Edge e has target coop_target[e] and sources
 * coop_src[coop_ptr[e] .. coop_ptr[e+1]-1]; strengths are the raw edge
 * strengths (the library multiplies by basals[target] as cle.jl:96,103 do). */
int scrna_net_create(scrna_ctx* ctx, int32_t G, const double* basals, const double* A_colmajor,
                     int32_t n_coop, const int32_t* coop_target, const int32_t* coop_ptr,
                     const int32_t* coop_src, const double* coop_strength,
                     int32_t n_redun, const int32_t* redun_target, const int32_t* redun_ptr,
                     const int32_t* redun_src, const double* redun_strength,
                     const double* k_on, const double* k_off, int32_t index_base,
                     scrna_net** out);
int scrna_net_destroy(scrna_net* net);
int32_t scrna_net_genes(const scrna_net* net);

/* ---- simulate -----------------------------------------------------------------
 * Replaces simulate(net, CLE(dt), kin, Val(:gpu); cell_num, T, readout)
 * (ext/SyntheticscRNAseqCUDAExt.jl:48-117) and, with pop != NULL,
 * simulate(net, CLE(dt), kin, Val(:gpu), pop; T, readout) (ext:409-529).
 * `out` (host, cells x G or cells x 2G, column-major) receives the readout.
 * With cap != NULL, `counts` (host, cells x G int32) receives the captured
 * counts (src/capture.jl:25-47) and `efficiencies` (host, cells, nullable) the
 * per-cell capture efficiencies.  Blocks until the results are on the host. */
int scrna_cle_simulate(scrna_ctx* ctx, const scrna_net* net, const scrna_kinetics* kin,
                       const scrna_population* pop, const scrna_capture* cap,
                       const scrna_cle_opts* opts, double* out, int32_t* counts,
                       double* efficiencies);

/* Replaces simulate_gpu_batch(networks, CLE(dt), kin; cell_num, T, readout)
 * (ext/SyntheticscRNAseqCUDAExt.jl:132-213; stub src/SyntheticscRNAseq.jl:75-76).
 * Unlike the reference, networks may differ in G and in cell count, and each may
 * carry its own population config (pops[b] nullable; pops itself nullable).
 * All B networks run in one persistent launch fed by a device work queue.
 * kins: B entries, or 1 entry shared by all.  cell_nums: per network cell
 * counts (ignored for networks with a population config).  Network b uses
 * Philox stream opts->stream + b.  outs[b] / counts[b] as in scrna_cle_simulate. */
int scrna_cle_simulate_batch(scrna_ctx* ctx, int32_t B, const scrna_net* const* nets,
                             const scrna_kinetics* kins, int32_t n_kins,
                             const int64_t* cell_nums, const scrna_population* const* pops,
                             const scrna_capture* cap, const scrna_cle_opts* opts,
                             double* const* outs, int32_t* const* counts);

/* ---- binomial tau-leap --------------------------------------------------------------
 * Replace the GPU BinomialTauLeap methods of the reference:
 *   simulate(net, BinomialTauLeap(dt), kin, Val(:gpu); cell_num, T, readout)
 *     (ext/SyntheticscRNAseqCUDAExt.jl:215-284),
 *   simulate(net, BinomialTauLeap(dt), kin, Val(:gpu), pop; T, readout) (ext:531-663),
 *   simulate_gpu_batch(networks, BinomialTauLeap(dt), kin[s]; ...) (ext:290-399, ext:666-837).
 * Same arguments as the CLE entry points (opts->dt is the tau-leap step).  Per step and gene,
 * as the reference computes it in FP32: transcription Poisson(max(reg + beta, 0) dt (x V)),
 * mRNA decay min(Poisson(m (1 - exp(-mu_m dt))), m), translation Poisson(k_t m dt) with the new
 * m, protein decay likewise; Poisson by inverse CDF over 50 terms (ext:21-39).  Additions as
 * in the CLE: cooperative / redundant edges and telegraph gating (tauleap_binomial.jl:84-137).
 * With a population: Hill of the concentration P / V, transcription x V, decay without
 * dilution, initial counts max(1, round(steady state x V)), and the readout is M / V, P / V
 * (capture counts are drawn from the molecule counts).  Paths: the block-tile register kernel
 * (REGISTER, BLOCK; up to 512 genes with its tables within shared memory) or the tensor form
 * (TENSOR, TENSOR_LIBRARY; any G, populations included): the state cell-major in device memory
 * and the draws over gene pairs; SCRNA_PATH_WARP is rejected.  At SCRNA_PRECISION_FP32 the
 * tensor form's regulation is the register path's FP32 arithmetic for every network that path
 * holds (and sparse ones beyond it), so both give the same counts bit for bit; AUTO takes the
 * tensor form beyond 128 genes (where it is faster) or when the register path cannot hold the
 * network.  Dense networks beyond the register path take the regulation from a BF16 GEMM, and
 * SCRNA_PRECISION_FP32_F16 from an FP16 GEMM. */
int scrna_tauleap_simulate(scrna_ctx* ctx, const scrna_net* net, const scrna_kinetics* kin,
                           const scrna_population* pop, const scrna_capture* cap,
                           const scrna_cle_opts* opts, double* out, int32_t* counts,
                           double* efficiencies);
int scrna_tauleap_simulate_batch(scrna_ctx* ctx, int32_t B, const scrna_net* const* nets,
                                 const scrna_kinetics* kins, int32_t n_kins,
                                 const int64_t* cell_nums, const scrna_population* const* pops,
                                 const scrna_capture* cap, const scrna_cle_opts* opts,
                                 double* const* outs, int32_t* const* counts);
int scrna_tauleap_run_device(scrna_ctx* ctx, const scrna_net* net, const scrna_kinetics* kin,
                             const scrna_population* pop, const scrna_capture* cap,
                             const scrna_cle_opts* opts, scrna_state* st);

/* Replaces apply_capture(X, capture; rng) (src/capture.jl:25-47): X is a host
 * cells x G column-major Float64 matrix of molecule values.  Y (host, cells x G
 * int32) gets the captured counts, eff (host, cells, nullable) the efficiencies. */
int scrna_apply_capture(scrna_ctx* ctx, int64_t N, int32_t G, const double* X,
                        const scrna_capture* cap, uint64_t seed, uint32_t stream, int32_t* Y,
                        double* eff);

/* ---- device-resident runs ------------------------------------------------------
 * A state object keeps one network's simulation state and outputs in device
 * memory so repeated runs touch no host memory.  scrna_cle_run_device enqueues
 * a whole run on the context stream and returns without waiting;
 * scrna_state_read copies the readout / counts / efficiencies to the host. */
int scrna_state_create(scrna_ctx* ctx, const scrna_net* net, int64_t cell_num, int32_t readout,
                       int32_t with_capture, scrna_state** out);
int scrna_state_destroy(scrna_state* st);
int scrna_cle_run_device(scrna_ctx* ctx, const scrna_net* net, const scrna_kinetics* kin,
                         const scrna_population* pop, const scrna_capture* cap,
                         const scrna_cle_opts* opts, scrna_state* st);
int scrna_state_read(scrna_ctx* ctx, scrna_state* st, double* out, int32_t* counts,
                     double* efficiencies);
/* Device pointers of the state's FP32 mRNA / protein arrays (for tests): [G][N] after a
 * run on the block kernel, [N][G] (cell-major) after a run on the lane kernel. */
int scrna_state_device_ptrs(scrna_state* st, void** d_mrna, void** d_protein);
/* Copies the raw simulation state of the last run to the host: mRNA and protein as
 * [G][N] float32 (FP32 path) or float64 (FP64 baseline path, then pass doubles),
 * promoter states [G][N] uint8 and volumes [N] float64 (population runs).
 * Any pointer may be NULL. */
int scrna_state_read_raw(scrna_ctx* ctx, scrna_state* st, void* mrna, void* protein,
                         uint8_t* promoter, double* volume);

/* ---- autotuning ---------------------------------------------------------------------
 * No counterpart in the reference.  The register path has several kernel variants that
 * compute the same sums in the same order (block tiles; the lane kernel with 2 or 4 genes
 * per lane and 2, 4 or 8 warps per block), so they give bit-identical results and differ
 * only in speed.  With autotuning on (the default; environment SCRNA_AUTOTUNE=0/1/2 sets a
 * new context's mode), the first run of a network shape (device, G, in-edges per gene,
 * cooperative/redundant terms, telegraph genes, Hill exponent 2, power-of-two bucket of the
 * cell count) measures the variants for a few steps and keeps the fastest in memory and in
 * a JSON cache file (SCRNA_AUTOTUNE_CACHE, else $XDG_CACHE_HOME or ~/.cache
 * /scrna_b200/autotune.json), which later runs and processes read.  Applies to the AUTO,
 * REGISTER and WARP paths of scrna_cle_simulate, scrna_cle_run_device (a measurement there
 * waits for the device) and the batch call; the server uses cached choices only (a request
 * stream's shapes mostly occur once, and measuring would stall the running requests).  The fused tensor-core step's tile
 * width (160, 192 or 224 genes; the same contraction order, so identical results) is tuned
 * the same way per (device, G, operand type, telegraph genes, Hill exponent 2, cell bucket). */
typedef struct {
    int32_t kernel;          /* 0 block tiles, 1 lane kernel, 2 the fused tensor-core step */
    int32_t genes_per_lane;  /* lane kernel: 2 or 4; tensor-core step: genes per tile (160, 192, 224) */
    int32_t block_warps;     /* lane kernel with cells within one warp: 2, 4 or 8 (0: default) */
    int32_t found;           /* lookups: 1 if the key was in the cache */
    double us_per_step;      /* measured time of one Euler step of the whole run */
} scrna_tune_choice;

/* mode 0: static choice; 1: cached or measured choice; 2: cached choice only, no measurement.
 * cache_path NULL keeps the current file; "" keeps choices in memory only. */
int scrna_ctx_set_autotune(scrna_ctx* ctx, int32_t mode, const char* cache_path);
/* The kernel variant the context's last register-path run used (found = 1 if tuned). */
int scrna_autotune_last_choice(const scrna_ctx* ctx, scrna_tune_choice* out);
/* Cache key of a network shape ("<device>|G..|e..|t..|b..|h..|N.."); device as "sm100x148". */
int scrna_autotune_key(const char* device, int32_t G, int32_t in_edges, int32_t n_terms, int32_t bursty,
                       int32_t hill2, int64_t cell_num, char* out, int32_t out_len);
/* Cache file access (host only, no device needed): lookup sets out->found; store adds or
 * replaces one entry, keeping the entries other processes wrote, by an atomic rename. */
int scrna_autotune_cache_lookup(const char* path, const char* key, scrna_tune_choice* out);
int scrna_autotune_cache_store(const char* path, const char* key, const scrna_tune_choice* choice);

/* ---- validation reductions and count-matrix output ---------------------------------
 * Computed on the device from a state's last results; only summaries cross to the host.
 * source 0: the readout (cells x G, or x 2G for BOTH), source 1: the captured counts.
 * scrna_state_moments: per column mean and unbiased variance (FP64, two passes); the
 *   host-side comparison is compare_moments (src/validate.jl:70-77).
 * scrna_state_ks: per column the two-sample Kolmogorov-Smirnov statistic between two
 *   states' samples, with the tie order of ks_statistic (src/validate.jl:14-41).
 * scrna_state_histogram: counts of the values of one column rounded to integers and clamped
 *   to [0, nbins-1] (the empirical distribution compared with telegraph_pmf,
 *   src/analytical.jl:35-95).
 * scrna_state_write_mtx: writes dir/matrix.mtx (MatrixMarket coordinate integer general,
 *   genes x cells, 1-based, entries in cell order: the layout read_10x_mtx of
 *   experiments/compare_real_scrnaseq.jl:69-93 reads), dir/genes.tsv ("id<TAB>name" per gene,
 *   names from gene_names or gene<k>) and dir/barcodes.tsv (<prefix><k>, prefix "cell" if
 *   NULL) from the captured counts, compacting the nonzeros on the device 65,536 cells at a
 *   time.  The directory must exist. */
int scrna_state_moments(scrna_ctx* ctx, scrna_state* st, int32_t source, double* mean, double* var);
int scrna_state_ks(scrna_ctx* ctx, scrna_state* a, scrna_state* b, int32_t source, double* D);
int scrna_state_histogram(scrna_ctx* ctx, scrna_state* st, int32_t source, int32_t column, int32_t nbins,
                          int64_t* hist);
int scrna_state_write_mtx(scrna_ctx* ctx, scrna_state* st, const char* dir, const char* const* gene_names,
                          const char* barcode_prefix);

/* ---- continuation and checkpoints ---------------------------------------------------
 * A run of the register path (CLE or tau-leap) is a pure function of its inputs and of
 * increments keyed by (seed, stream, cell, step, gene), and its state is exact between
 * launches, so a run continued from step T1 to T2 equals one run of T2 steps bit for bit.
 * A tau-leap run of the tensor form at FP32 precision leaves the same state (for networks the
 * register path holds), so it continues and checkpoints the same way; other tensor-path runs
 * keep no state to continue.
 * The reference's nearest counterpart returns the final population state for inspection
 * (simulate_with_state, src/algorithms/tauleap_binomial.jl:270-324).
 * scrna_cle_resume / scrna_tauleap_resume: continue the run `st` holds (from a run on this
 * state or scrna_state_restore) to the total step count of opts (T or n_steps, counted from
 * step 1); same network, kinetics, population mode, seed, stream, cells and readout as the
 * run being continued; the readout and capture are written at the end as for a full run.
 * scrna_state_steps_done: steps the held run has done (0 if none).
 * scrna_state_checkpoint: with buf NULL sets *bytes to the size needed; else writes the held
 * run's state (header "SCRNACK1", G, flags, N, steps, divisions; M, P float32, promoter
 * uint8, switching int32 pairs, all [G][N]; volumes float64 with a population) into buf.
 * scrna_state_restore: loads a checkpoint into a state created for the same G and N. */
int scrna_cle_resume(scrna_ctx* ctx, const scrna_net* net, const scrna_kinetics* kin,
                     const scrna_population* pop, const scrna_capture* cap, const scrna_cle_opts* opts,
                     scrna_state* st);
int scrna_tauleap_resume(scrna_ctx* ctx, const scrna_net* net, const scrna_kinetics* kin,
                         const scrna_population* pop, const scrna_capture* cap, const scrna_cle_opts* opts,
                         scrna_state* st);
int scrna_state_steps_done(const scrna_state* st, int64_t* steps);
int scrna_state_checkpoint(scrna_ctx* ctx, scrna_state* st, void* buf, size_t capacity, size_t* bytes);
int scrna_state_restore(scrna_ctx* ctx, scrna_state* st, const void* buf, size_t bytes);

/* ---- serving loop ---------------------------------------------------------------------
 * A request server with continuous batching (no counterpart in the reference, which runs
 * one simulate call at a time).  Submitted requests wait in a FIFO queue until their device
 * footprint fits the HBM budget, then join the running set at the next chunk boundary: every
 * chunk advances all running requests by up to `chunk_steps` Euler steps in shared
 * persistent launches.  Requests keep their state on the device between chunks; results are
 * identical to scrna_cle_simulate on the same inputs, alone or in any mix.  Population
 * dynamics are not served (SCRNA_ENOTSUP). */
typedef struct scrna_server scrna_server;

typedef struct {
    const scrna_net* net;
    scrna_kinetics kin;
    scrna_cle_opts opts;      /* cell_num, T or n_steps, readout, seed, stream, dt */
    int32_t with_capture;
    int32_t reserved;
    scrna_capture capture;
} scrna_request;

enum scrna_request_state {
    SCRNA_REQ_QUEUED = 0, SCRNA_REQ_RUNNING = 1, SCRNA_REQ_DONE = 2, SCRNA_REQ_FAILED = 3,
    SCRNA_REQ_CANCELLED = 4
};

typedef struct {
    int64_t submitted, completed, failed, queued, running;
    int64_t units_done;       /* cell-gene-steps of completed requests */
    int64_t bytes_in_use;     /* device footprint of admitted requests */
    double busy_s;            /* wall time the worker spent with work in flight */
    int64_t chunks;           /* chunk launches issued */
} scrna_server_stats;

/* hbm_budget_bytes <= 0: 80 % of the free device memory at creation. */
int scrna_server_create(scrna_ctx* ctx, int64_t hbm_budget_bytes, int32_t chunk_steps, scrna_server** out);
int scrna_server_destroy(scrna_server* srv);
/* Non-blocking.  The network handle must stay alive until the request completes. */
int scrna_submit(scrna_server* srv, const scrna_request* req, uint64_t* ticket);
int scrna_poll(scrna_server* srv, uint64_t ticket, int32_t* state);
/* Waits up to timeout_ms (< 0: forever) for the request, copies its results to the host
 * (out: cells x G (x2) column-major; counts/efficiencies with capture, nullable) and
 * releases it.  Returns SCRNA_ETIMEOUT if it is not done in time (the request stays). */
int scrna_wait(scrna_server* srv, uint64_t ticket, int32_t timeout_ms, double* out, int32_t* counts,
               double* efficiencies, double* latency_s);
int scrna_cancel(scrna_server* srv, uint64_t ticket);
int scrna_server_get_stats(scrna_server* srv, scrna_server_stats* stats);
/* Trace of the server's most recent chunks (up to 4,096, oldest first): per chunk the
 * worker's clock (seconds since the server was created) when its launches were issued and
 * when they had finished, the requests and kernel groups it ran, and its cell·gene·steps.
 * With recs NULL sets *n to the number held; else copies min(capacity, held) records. */
typedef struct {
    double t_start, t_end;
    int32_t requests, groups;
    int64_t units;
} scrna_chunk_record;
int scrna_server_trace(scrna_server* srv, scrna_chunk_record* recs, int32_t capacity, int32_t* n);

/* ---- scratch-free run ---------------------------------------------------------------
 * This entry point has no counterpart in the reference.  It is for callers that
 * cannot allocate device memory when they run a simulation (the allocator is owned
 * by another component, a serving loop must not synchronise on cudaMalloc/cudaFree,
 * or device memory is budgeted up front).  It runs the block-tile FP32 register kernel
 * of scrna_cle_run_device, optionally with population and capture, and calls no
 * cudaMalloc, cudaFree or other allocating routine: all working memory comes from
 * one file-scope device array of about 16.0 MB, held until the process exits.
 * Limits per call: 65,536 cells, 512 genes and 262,144 cell-genes; larger runs are
 * rejected with SCRNA_EINVAL.  opts->path must be AUTO, REGISTER or BLOCK (others:
 * SCRNA_ENOTSUP).
 *   d_out    device pointer, cells x G (x2 for SCRNA_READOUT_BOTH) float64, column-major
 *   d_counts device pointer, cells x G int32 (required with cap, else ignored)
 *   d_eff    device pointer, cells float64 (required with cap, else ignored)
 * The call only enqueues work on the context stream; synchronise before reading.  It
 * leaves the calling thread's current device as it found it.
 * First call per device: under CUDA's default lazy module loading, the array's memory
 * is mapped on a device by the first call there (which looks up the array's device
 * address and may synchronise the device).  Make that first call during set-up, before
 * the caller can no longer allocate and before any stream capture.
 * All calls share the one array, which keeps the last call's contents: calls whose work
 * overlaps on the GPU (other streams or contexts on the same device) race and corrupt
 * each other's results. */
int scrna_cle_simulate_noalloc(scrna_ctx* ctx, const scrna_net* net, const scrna_kinetics* kin,
                               const scrna_population* pop, const scrna_capture* cap,
                               const scrna_cle_opts* opts, double* d_out, int32_t* d_counts,
                               double* d_eff);

/* ---- page-locked host buffers -----------------------------------------------------
 * Page-locked (pinned) host memory for result arrays: a device-to-host copy into it runs
 * at the link's DMA rate instead of through the driver's staging of pageable memory.
 * No counterpart in the reference (Julia returns Arrays in pageable memory); the Python
 * layer keeps a pool of these blocks for the arrays that simulate() returns.
 * scrna_host_alloc: *p = bytes of portable pinned memory (SCRNA_ECUDA if refused).
 * scrna_host_free: releases a block from scrna_host_alloc (NULL is a no-op). */
int scrna_host_alloc(size_t bytes, void** p);
int scrna_host_free(void* p);

/* ---- diagnostics ----------------------------------------------------------------
 * Runs Philox4x32-10 on the device for n counters (host arrays ctr[4n], key[2]) and
 * returns the words in out[4n]; used to check the device generator against the
 * published known-answer vectors. */
int scrna_debug_philox(scrna_ctx* ctx, int32_t n, const uint32_t* ctr, const uint32_t* key,
                       uint32_t* out);
/* C[M x N] (FP32, row-major) = A[M x K] * B[N x K]^T on device pointers, A and B 16-bit
 * (dtype 0 BF16, 1 FP16) row-major with K a multiple of 64, by the library's hand-written
 * tcgen05 GEMM (the contraction of the dense path); synchronous.  No counterpart in the
 * reference: it checks the tensor-core kernel against another GEMM. */
int scrna_debug_tc_gemm(scrna_ctx* ctx, const void* A, const void* B, float* C, int64_t M, int32_t N,
                        int32_t K, int32_t dtype);
/* The same GEMM with its TMA producer stopping before its load number `withhold` (>= 0) in
 * every CTA, so the MMA issuer's and the epilogue's bounded waits (2 s each) run out: returns
 * SCRNA_ETIMEOUT after the kernel has left through its normal exit (TMEM released), and the
 * context stays usable.  No counterpart in the reference: it tests the failure path of the
 * tensor-core pipeline without faulting or hanging the GPU. */
int scrna_debug_tc_gemm_withhold(scrna_ctx* ctx, const void* A, const void* B, float* C, int64_t M, int32_t N,
                                 int32_t K, int32_t dtype, int32_t withhold);
/* Compares the tau-leap's branch-free quotient lam / k (the Poisson inverse CDF's terms,
 * ext/SyntheticscRNAseqCUDAExt.jl:21-39) with IEEE division for every float lam whose bit
 * pattern lies in [lo, hi) and is in the quotient's range (0 or 2^-100..2^100), for every
 * k = 1..50; returns the number of differing quotients and the first (lam bits, k) that
 * differs.  No counterpart in the reference: it checks the library's own arithmetic. */
int scrna_debug_small_div_check(scrna_ctx* ctx, uint32_t lo, uint32_t hi, int64_t* mismatches,
                                uint32_t* first_bad_lam, int32_t* first_bad_k);
/* Measures the sustained issue rate of the FP32 FMA pipe and of the special-function
 * unit (MUFU) pipe with two microkernels; results in operations per second. */
int scrna_measure_pipe_peaks(scrna_ctx* ctx, double* fma_ops_per_s, double* sfu_ops_per_s,
                             double* int_ops_per_s);
/* Measures the throughput of the library's Philox4x32-10 generator (round keys from kernel
 * parameters, as the CLE kernels use it) with a microkernel: generator calls per second. */
int scrna_measure_philox_rate(scrna_ctx* ctx, double* calls_per_s);

#ifdef __cplusplus
}
#endif
#endif /* SCRNA_CLE_H */
