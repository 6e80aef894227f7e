// Host-side objects behind the C ABI handles (scrna_ctx, scrna_net, scrna_state),
// shared by the translation units of the library.  Not part of the public ABI.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <functional>
#include <map>
#include <string>
#include <vector>

#include "../../include/scrna_cle.h"
#include "cle_internal.h"

struct cublasLtContext;

namespace scrna {
int fail(int code, const char* fmt, ...);
}  // namespace scrna

struct scrna_net;
struct scrna_state;
struct scrna_ctx;

#define CU(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return scrna::fail(SCRNA_ECUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// ---- device buffers -----------------------------------------------------------------------
namespace scrna {
struct DevBuf {
    void* p = nullptr;
    size_t n = 0;
    ~DevBuf() { if (p) cudaFree(p); }
    cudaError_t ensure(size_t bytes) {
        if (bytes <= n) return cudaSuccess;
        if (p) { cudaFree(p); p = nullptr; n = 0; }
        cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
        if (e == cudaSuccess) n = bytes;
        return e;
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
};
}  // namespace scrna
using scrna::DevBuf;
using scrna::NetDev;
using scrna::NonAdd;

struct scrna_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::atomic<int64_t> launches{0};
    // bytes the library copied host -> device and device -> host for this context's networks,
    // per-run tables and results (scrna_ctx_transfer_bytes)
    std::atomic<int64_t> h2d_bytes{0}, d2h_bytes{0};
    int sm_count = 0;
    // states reused by the synchronous simulate calls (most recent last)
    std::vector<scrna_state*> state_cache;
    // cuBLASLt handle and workspace of the tensor-core path (created on first use)
    void* lt_handle = nullptr;
    scrna::DevBuf lt_workspace;
    scrna::DevBuf tc_err;        // error flag of the tcgen05 kernels (one int)
    scrna::DevBuf log2_tab;      // own_log2f of the 2^18 switch uniforms (switch_table.cuh)
    bool log2_tab_ready = false;
    // autotuning of the register-path kernel (tune.cu): mode 0 off, 1 measure on a miss,
    // 2 cache only; cache file (empty: memory only); choices made on this context
    int tune_mode = 1;
    std::string tune_path;
    char tune_arch[32] = "sm100";
    std::map<std::string, scrna_tune_choice> tune_mem;
    scrna_tune_choice tune_last{};
};

struct scrna_net {
    scrna_ctx* ctx = nullptr;
    int32_t G = 0;
    std::vector<double> basals;
    std::vector<double> A;  // row-major A[i*G+j]
    std::vector<double> k_on, k_off;
    // host tables
    std::vector<int32_t> reg_slot;   // gene -> slot or -1
    std::vector<int32_t> reg_gene;   // slot -> gene
    std::vector<int32_t> in_begin, in_end;
    std::vector<float2> in_edge;
    std::vector<double> in_w64;
    std::vector<double> cneg64;
    std::vector<int32_t> na_begin, na_count;
    std::vector<NonAdd> na;
    std::vector<double> na_coef64;
    std::vector<int32_t> na_src;
    NetDev dev;
    DevBuf b_tables;  // the network's upload-time tables (NetDev's pointers) in one allocation
    // per-run tables cached for the last (kinetics, dt, population mode)
    DevBuf b_genes, b_ginit, b_quad_tel;
    // tensor-core path: W = A_eff as 16-bit [G][Kp] (K-major), nonadd sources compacted
    int32_t t_kp = 0;
    int32_t t_dtype = -1;              // 0 bf16, 1 fp16
    int32_t t_n_src = 0;               // distinct genes read by cooperative/redundant edges
    DevBuf t_w16, t_na, t_na_src, t_src_gene, t_src_of_gene;
    DevBuf t_slot_of_gene;             // gene -> regulator slot or -1 (the tau-leap's exact regulation)
    bool cache_valid = false;
    double c_dt = 0, c_kin[6] = {0};
    bool c_pop = false;
};

struct scrna_state {
    scrna_ctx* ctx = nullptr;
    int32_t G = 0;
    int64_t N = 0;
    int32_t readout = 1;
    bool capture = false;
    DevBuf M, P, prom, NS, V, out, counts, eff;
    DevBuf dM[2], dP[2], dprom[2], dNS[2], dV[2], owner[2];
    DevBuf M64, P64a, P64b;  // FP64 baseline state
    // tensor-core path state, cell-major [N][G]
    DevBuf tM, tP, tprom, tNS, tact16, tact32[2], treg;
    int t_ld = 0;  // row stride of the cell-major tensor-path state
    bool last_tensor = false;
    bool last_cell_major = false;  // the lane kernel ran: M, P, prom, NS are [N][G]
    bool have_counts = false;
    bool last_plain = false;
    bool last_pop = false;
    const double* p64_final = nullptr;
    // continuation of register-path runs (scrna_cle_resume, checkpoints): the state holds the
    // end of a run of `steps_done` steps with `epoch` divisions, by the CLE or the tau-leap
    bool has_register_state = false;
    bool last_tau = false;
    int64_t steps_done = 0;
    int32_t epoch = 0;
};


namespace scrna {
// Register-path kernel chosen for a network.
struct KernelChoice {
    bool warp;
    int gpl, emax, tmax, nwarps;
    int nw1;  // lane kernel: warps per block when a cell fits in one warp (0: the default 4)
    FusedLaunch block;
    size_t smem;
};
int set_device(scrna_ctx* ctx);
int ensure_gene_tables(scrna_net* n, const scrna_kinetics* kin, double dt, bool pop);
int validate_run(const scrna_net* net, const scrna_kinetics* kin, const scrna_population* pop,
                 const scrna_capture* cap, const scrna_cle_opts* o);
int64_t n_steps_of(const scrna_cle_opts* o);
int state_alloc(scrna_state* st, bool pop, bool plain);
void fill_fused_args(scrna_net* net, const scrna_kinetics* kin, const scrna_population* pop,
                     const scrna_capture* cap, const scrna_cle_opts* o, scrna_state* st, FusedArgs* out);
KernelChoice choose_kernel(const scrna_net* net, int path);
void tune_init_ctx(scrna_ctx* ctx);
// The context's table of switch-uniform log2 values, filled on first use; null if it cannot
// be allocated (the kernels then evaluate the series).
const float* switch_log2_table(scrna_ctx* ctx);
// Tile width of the fused tensor-core step (slices of 32 genes: 5, 6 or 7): 7 with autotuning
// off, else the cached or measured fastest (measure(S, &us_per_step)); *measured tells
// whether measurement launches ran.
int tc_choose_slices(scrna_ctx* ctx, int G, int64_t N, bool bursty, int dtype, bool hill2,
                     const std::function<int(int, double*)>& measure, int* S, bool* measured);
int choose_kernel_tuned(scrna_ctx* ctx, scrna_net* net, const scrna_kinetics* kin, const scrna_cle_opts* o,
                        scrna_state* st, KernelChoice* out, const FusedArgs* base = nullptr,
                        cudaStream_t stream = nullptr, bool may_measure = true);
// Converts a state's M, P, promoter and switching arrays between gene-major [G][N] and
// cell-major [N][G] (the lane kernel's layout).
int state_relayout(scrna_ctx* ctx, scrna_state* st, bool to_cell_major);
int resume_register_run(scrna_ctx* ctx, scrna_net* net, const scrna_kinetics* kin, const scrna_population* pop,
                        const scrna_capture* cap, const scrna_cle_opts* o, scrna_state* st, bool tau);
int fused_max_quads();
// The register path takes the network (gene count and shared-memory tables).
bool register_path_holds(const NetDev& d);
// The automatic path's choice of the tensor path for a network of N cells.
bool auto_tensor(const scrna_net* net, bool tau, int64_t N);
// The tau-leap's tensor form with the register path's exact FP32 regulation (no GEMM).
bool tau_tensor_exact(const scrna_net* n, int dtype);
// Copies a tensor-form tau-leap state into the register path's gene-major buffers.
int tensor_state_to_register(scrna_ctx* ctx, scrna_state* st);
cudaError_t fused_queue_launch(const FusedArgs* args, const TileWork* items, int n_items, int* counter, int upt,
                               int nw, size_t smem, bool pop, int grid, TileCtl shared_ctl, int use_shared,
                               cudaStream_t st);
// ks: round keys shared by every network of the launch (NULL: each network's own, computed
// in the rounds)
cudaError_t warpcell_queue_launch(const FusedArgs* args, const TileWork* items, int n_items, int* counter, int gpl,
                                  int emax, int tmax, bool pop, size_t smem, int grid, int nwarps,
                                  TileCtl shared_ctl, int use_shared, const KeySchedule* ks, cudaStream_t st);
int warpcell_cells_per_block_host(int G, int gpl, int nw1);
int warpcell_block_warps_host(int G, int gpl, int nw1);
int warpcell_wpc_host(int G, int gpl);
size_t warpcell_smem(int G, int gpl, int n_reg, int n_terms, int nw1);
int tensor_prepare_net(scrna_net* n, int dtype);
cudaError_t tensor_terms_launch(int dtype, int64_t N, int G, int Kp, int n_terms, int n_src, const NonAdd* na,
                                const int32_t* na_src, const float* act32, void* act16, cudaStream_t st);
int tc_run(scrna_ctx* ctx, scrna_net* n, const scrna_kinetics* kin, const scrna_capture* cap,
           const scrna_cle_opts* o, scrna_state* st, int dtype);
int tensor_run(scrna_ctx* ctx, scrna_net* n, const scrna_kinetics* kin, const scrna_capture* cap,
               const scrna_cle_opts* o, scrna_state* st, int dtype, bool tau = false,
               const scrna_population* pop = nullptr);
int batch_simulate(scrna_ctx* ctx, int32_t B, const scrna_net* const* nets, const scrna_kinetics* kins,
                   int32_t n_kins, const int64_t* cell_nums, const scrna_population* const* pops,
                   const scrna_capture* cap, const scrna_cle_opts* opts, double* const* outs,
                   int32_t* const* counts, bool tau);
void fill_tau_args(const scrna_net* net, const scrna_kinetics* kin, const scrna_population* pop,
                   const scrna_cle_opts* o, FusedArgs* a);
int tau_lockstep_default();
void gene_tables_host(const scrna_net* n, const scrna_kinetics* kin, double dt, GeneRec* gr, GeneInit* gi,
                      uint8_t* qt);
cudaError_t tau_queue_launch(const FusedArgs* args, const TileWork* items, int n_items, int* counter, int upt, int nw,
                             size_t smem, bool pop, int grid, TileCtl shared_ctl, int use_shared, int qg,
                             cudaStream_t st);
FusedLaunch tau_plan(int G, int n_reg, int n_in, int n_na, int n_na_src, int qg);
int tau_genes_per_unit(int G, int n_reg, int n_in, int n_na, int n_na_src, int64_t N);
}  // namespace scrna
