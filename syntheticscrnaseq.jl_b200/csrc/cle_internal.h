// Internal structures shared by the host side of the library (capi.cu) and the
// kernels.  Not part of the public ABI.
#pragma once
#include <cstddef>
#include <cstdint>

namespace scrna {

// Per-gene record, rebuilt for every run (thresholds depend on dt, initial values on
// the kinetics).  32 bytes, read by the kernels with two 16-byte loads.
struct GeneRec {
    float beta;        // basal rate beta_g
    float cneg;        // sum_j max(-A_eff[g,j], 0): the repression constant of the one-GEMM form
    float inv_on;      // -ln2 / (k_on dt): waiting-time parameter while OFF (-0: switch next step)
    float inv_off;     // -ln2 / (k_off dt): waiting-time parameter while ON (-inf: never)
    int32_t slot;      // regulator slot of this gene (-1 when no edge reads its protein)
    int32_t in_begin;  // additive in-edges [in_begin, in_end) in the edge table
    int32_t in_end;
    int32_t na_range;  // cooperative/redundant edges targeting g: begin << 16 | count
};
struct GeneInit {
    float m0, p0;       // ceil of the steady state (cle.jl:49-53)
    uint32_t thr_init;  // initial ON when word < thr_init (k_on/(k_on+k_off))
    int32_t init_rand;  // 1: initial promoter state drawn (both rates finite)
};

// Cooperative (kind 0) / redundant (kind 1) edge with coefficient s*beta_target and
// sources na_src[src_begin, src_end) (as regulator slots).
struct NonAdd {
    int32_t kind;
    float coef;
    int32_t src_begin;
    int32_t src_end;
};

// Tables of the warp kernel.  A gene's in-edges are {source slot, weight bits}: its
// additive edges, then one edge {n_reg + 3 + j, coef_j} per cooperative / redundant term
// j targeting it; padding is {slot n_reg (constant 0), weight 0}.  A term names regulator
// slots as sources; a padded source names a constant slot (n_reg + 1 holding 1 for a
// cooperative term, n_reg holding 0 for a redundant one).
constexpr int kLaneEdges = 8;  // in-edges per gene (additive + terms)
constexpr int kLaneTerms = 2;  // terms evaluated per lane
constexpr int kLaneSrc = 3;    // sources per term
constexpr size_t kMaxDynamicSmem = 227 * 1024;  // opt-in shared memory of one block (sm_100a)
struct LaneTerm {
    float coef;
    int32_t kind;
    int32_t src[kLaneSrc];
    int32_t pad[3];
};

// Device-resident network tables (owned by scrna_net).
struct NetDev {
    int32_t G = 0;
    int32_t n_reg = 0;      // regulator slots
    int32_t n_in = 0;       // additive edges
    int32_t n_na = 0;       // cooperative + redundant edges
    int32_t n_na_src = 0;
    int32_t n_quads = 0;
    float2* in_edge = nullptr;   // {w, slot bits}, grouped by target gene
    NonAdd* na = nullptr;
    int32_t* na_src = nullptr;
    int32_t* reg_gene = nullptr; // gene of each regulator slot
    double* in_w64 = nullptr;    // FP64 additive weights (baseline path)
    double* na_coef64 = nullptr; // FP64 s*beta_target (baseline path)
    double* beta64 = nullptr;    // FP64 basals (baseline path)
    int2* lane_in = nullptr;     // [G][kLaneEdges] padded in-edges (small networks), or null
    LaneTerm* lane_term = nullptr;  // [n_na] terms with padded sources (with lane_in)
    int32_t lane_gpl = 0;        // genes per lane of the warp kernel (2 or 4)
    int32_t lane_emax = 0;       // in-edges per gene the warp kernel runs (2, 4 or 8)
    int32_t lane_tmax = 0;       // terms per lane the warp kernel evaluates (0, 1 or 2)
    bool bursty = false;         // any gene switches (finite k_on)
};

// Arguments of the fused FP32 register-path kernel.
struct FusedArgs {
    int32_t G, n_quads, n_reg, n_in, n_na, n_na_src;
    int64_t N;              // cells of this network
    int64_t cell_offset;    // global index of cell 0 (Philox counter)
    int32_t step_begin;     // first step of this launch (1-based)
    int32_t step_end;       // last step of this launch (inclusive)
    int32_t first;          // 1: initialise state from GeneInit instead of reading it
    int32_t last;           // 1: write readout / capture after the last step
    int32_t check;          // 1: step_end is a division check step
    int32_t epoch;          // division epoch of this launch's prologue
    float k_t, Kn, hill_n, mu_m, mu_p, dt;
    int32_t hill_int;       // >0: integer Hill exponent (repeated products)
    uint32_t key0, key1, stream;
    uint32_t rk0[10], rk1[10];  // Philox round keys of (key0, key1)
    // population
    double growth_factor, V_div, V_lo, V_hi;
    int32_t partition, exclude_mother;
    // tables
    const GeneRec* genes;
    const GeneInit* ginit;
    const float2* in_edge;
    const NonAdd* na;
    const int32_t* na_src;
    const uint8_t* quad_tel;     // per quad: any gene switches (finite k_on)
    const int2* lane_in;         // [G][kLaneEdges] padded in-edges (warp kernel)
    const LaneTerm* lane_term;   // [n_na] terms with padded sources (warp kernel)
    // state: [G][N] for the block kernel, [N][G] (cell-major) for the lane kernel (also the
    // division scratch below), so a warp's loads and stores of a cell's genes are adjacent
    float* M;
    float* P;
    uint8_t* prom;
    int2* NS;               // switching state {next switch step, waiting time after it}
    double* V;
    // division scratch (two parities)
    float* dM[2];
    float* dP[2];
    uint8_t* dprom[2];
    int2* dNS[2];
    double* dV[2];
    unsigned long long* owner[2];
    // outputs
    double* out;            // readout, cells x G (x2) column-major, nullable
    int32_t readout;
    int32_t* counts;        // cells x G, nullable
    double* eff;            // cells, nullable
    int32_t capture_species;
    double cap_mu_log, cap_sigma;
    int32_t lane_nw1;       // lane kernel: warps per block when a cell fits in one warp (0 = 4)
    // binomial tau-leap (block kernel with TAU): FP32 decay probabilities 1 - exp(-mu dt),
    // FP64 basals and steady-state denominators for a population's initial counts
    float p_dec_m, p_dec_p;
    const double* beta64;
    double ss_mu_m, ss_mu_p, k_t64;
    // tau-leap draw schedule (same counts either way): 1 = the Poisson draws of a gene quad in
    // lock step, 0 = one draw after another
    int32_t tau_lockstep;
    // own_log2f of every 18-bit switch uniform (switch_table.cuh), or null
    const float* log2_tab;
};

// Step range and division flags of one launch (or one queued work item).
struct TileCtl {
    int32_t step_begin, step_end, first, last, check, epoch;
};

// One item of a persistent launch's work queue: a cell tile of network `arg` (index into
// the launch's FusedArgs array) advanced through a step range.
struct TileWork {
    int32_t arg;
    int32_t tile;
    TileCtl ctl;
};

// Philox round keys shared by every network of one queued launch (a batch call has one
// seed): passed as a kernel parameter, so the rounds read them as constant operands.
struct KeySchedule {
    uint32_t rk0[10], rk1[10];
};

// Launch shape of the fused kernel chosen for a network: quads per thread (UPT),
// warps per block (NW, so 32 cells x NW warps) and dynamic shared memory.
struct FusedLaunch {
    int upt;     // gene units per thread
    int nw;      // warps per block
    size_t smem;
    int qg = 4;  // genes per unit: 4 (the CLE), 4 or 2 (the tau-leap)
};

// Arguments of the plain FP64 one-kernel-per-step baseline.
struct PlainArgs {
    int32_t G, n_quads;
    int64_t N, cell_offset;
    int32_t step;
    double k_t, Kn, hill_n, mu_m, mu_p, dt, sqrt_dt;
    uint32_t key0, key1, stream;
    const GeneRec* genes;
    const float2* in_edge;   // weights used in double
    const double* in_w64;    // FP64 weights (A_pos/A_neg split) of the additive edges
    const NonAdd* na;
    const double* na_coef64;
    const int32_t* na_src;
    const int32_t* reg_gene;
    const uint8_t* quad_tel;
    const double* beta64;
    double* M;
    const double* Pold;
    double* Pnew;
    uint8_t* prom;
    int2* NS;
};

}  // namespace scrna
