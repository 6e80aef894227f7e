// Launch planning and dispatch of the fused register-path kernel (the kernel
// template is in cle_fused.cuh; each quads-per-thread variant is compiled in its
// own translation unit).
#include <cstdlib>
#include <type_traits>

#include "cle_internal.h"
#include "cle_warpcell.cuh"
#include <cuda_runtime.h>

namespace scrna {

template <int UPT, bool POP, bool TAU, int QG = 4>
cudaError_t fused_launch_t(const FusedArgs& a, int nw, size_t smem, cudaStream_t st);

size_t fused_smem_bytes_host(int G, int n_reg, int n_in, int n_na, int n_na_src, int n_quads) {
    size_t b = (size_t)2 * n_reg * 32 * sizeof(float);
    b += (size_t)G * sizeof(GeneRec);
    b += (size_t)n_in * sizeof(float2);
    b += (size_t)n_na * sizeof(NonAdd);
    b += (size_t)n_na_src * sizeof(int32_t);
    b += (size_t)n_quads;
    return (b + 15) & ~(size_t)15;
}

FusedLaunch fused_plan(int G, int n_reg, int n_in, int n_na, int n_na_src, int n_quads) {
    FusedLaunch L{};
    int upt = 1;
    while (upt < 8 && (n_quads + upt - 1) / upt > (upt <= 2 ? 8 : 16)) upt *= 2;
    L.upt = upt;
    L.nw = (n_quads + upt - 1) / upt;
    L.smem = fused_smem_bytes_host(G, n_reg, n_in, n_na, n_na_src, n_quads);
    return L;
}

int fused_max_quads() { return 8 * 16; }

// Whether the register path can run a network: at most 512 genes and its tables (in gene
// quads, the smallest layout of every kernel of the path) within a block's shared memory.
bool register_path_holds(const NetDev& d) {
    return d.n_quads <= fused_max_quads() &&
           fused_plan(d.G, d.n_reg, d.n_in, d.n_na, d.n_na_src, d.n_quads).smem <= kMaxDynamicSmem;
}

cudaError_t fused_launch(const FusedArgs& a, const FusedLaunch& L, bool pop, cudaStream_t st) {
    switch (L.upt * 2 + (pop ? 1 : 0)) {
        case 2: return fused_launch_t<1, false, false>(a, L.nw, L.smem, st);
        case 3: return fused_launch_t<1, true, false>(a, L.nw, L.smem, st);
        case 4: return fused_launch_t<2, false, false>(a, L.nw, L.smem, st);
        case 5: return fused_launch_t<2, true, false>(a, L.nw, L.smem, st);
        case 8: return fused_launch_t<4, false, false>(a, L.nw, L.smem, st);
        case 9: return fused_launch_t<4, true, false>(a, L.nw, L.smem, st);
        case 16: return fused_launch_t<8, false, false>(a, L.nw, L.smem, st);
        case 17: return fused_launch_t<8, true, false>(a, L.nw, L.smem, st);
        default: return cudaErrorInvalidValue;
    }
}

// ---- lane-per-gene-unit variant (networks up to 512 genes) ---------------------------------
template <int GPL, int EMAX, int TMAX, bool POP>
cudaError_t warpcell_launch_t(const FusedArgs& a, cudaStream_t st);
template <int GPL, int EMAX, int TMAX, bool POP>
cudaError_t warpcell_queue_launch_t(const FusedArgs* args, const TileWork* items, int n_items, int* counter,
                                    size_t smem, int grid, int nwarps, TileCtl shared_ctl, int use_shared,
                                    const KeySchedule* ks, cudaStream_t st);
template <int UPT, bool POP, bool TAU, int QG = 4>
cudaError_t fused_queue_launch_t(const FusedArgs* args, const TileWork* items, int n_items, int* counter,
                                 int nw, size_t smem, int grid, TileCtl shared_ctl, int use_shared, cudaStream_t st);

int warpcell_max_genes() { return kWarpcellMaxGenes; }
int warpcell_emax_class(int max_in) { return max_in <= 2 ? 2 : max_in <= 4 ? 4 : 8; }

// Genes per lane for a network: a cost model of issue slots per cell-gene-step, ~20 per
// lane and step plus ~80 per gene, over the lanes a cell occupies (idle lanes included).
int warpcell_pick_gpl(int G, bool bursty, int emax) {
    (void)bursty;
    if (emax > 4) return 2;  // 8 padded in-edges per gene: only gene pairs fit in registers
    double best = 1e30;
    int pick = 2;
    for (int gpl : {2, 4}) {
        const int w = warpcell_wpc(G, gpl);
        const double lanes = w == 1 ? 32.0 / warpcell_cells_per_warp(G, gpl) : 32.0 * w;
        const double cost = lanes * (20.0 + 80.0 * gpl) / G;
        if (cost < best) { best = cost; pick = gpl; }
    }
    return pick;
}

size_t warpcell_smem(int G, int gpl, int n_reg, int n_terms, int nw1) {
    return warpcell_smem_bytes(G, gpl, n_reg, n_terms, nw1);
}
int warpcell_cells_per_block_host(int G, int gpl, int nw1) { return warpcell_cells_per_block(G, gpl, nw1); }
int warpcell_block_warps_host(int G, int gpl, int nw1) { return warpcell_block_warps(G, gpl, nw1); }
int warpcell_wpc_host(int G, int gpl) { return warpcell_wpc(G, gpl); }

template <int V>
using IntC = std::integral_constant<int, V>;

// Calls f(IntC<GPL>, IntC<EMAX>, IntC<TMAX>, bool_constant<POP>) for the runtime shape
// (gene quads take at most 4 in-edges per gene).
template <class F>
static cudaError_t warpcell_dispatch(int gpl, int emax, int tmax, bool pop, F&& f) {
    auto by_k = [&](auto g, auto r) -> cudaError_t {
        switch (tmax * 2 + (pop ? 1 : 0)) {
            case 0: return f(g, r, IntC<0>{}, std::false_type{});
            case 1: return f(g, r, IntC<0>{}, std::true_type{});
            case 2: return f(g, r, IntC<1>{}, std::false_type{});
            case 3: return f(g, r, IntC<1>{}, std::true_type{});
            case 4: return f(g, r, IntC<2>{}, std::false_type{});
            case 5: return f(g, r, IntC<2>{}, std::true_type{});
            default: return cudaErrorInvalidValue;
        }
    };
    switch (gpl * 16 + emax) {
        case 34: return by_k(IntC<2>{}, IntC<2>{});
        case 36: return by_k(IntC<2>{}, IntC<4>{});
        case 40: return by_k(IntC<2>{}, IntC<8>{});
        case 66: return by_k(IntC<4>{}, IntC<2>{});
        case 68: return by_k(IntC<4>{}, IntC<4>{});
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t warpcell_launch(const FusedArgs& a, int gpl, int emax, int tmax, bool pop, cudaStream_t st) {
    return warpcell_dispatch(gpl, emax, tmax, pop, [&](auto g, auto r, auto k, auto p) {
        return warpcell_launch_t<decltype(g)::value, decltype(r)::value, decltype(k)::value, decltype(p)::value>(a, st);
    });
}

cudaError_t warpcell_queue_launch(const FusedArgs* args, const TileWork* items, int n_items, int* counter, int gpl,
                                  int emax, int tmax, bool pop, size_t smem, int grid, int nwarps,
                                  TileCtl shared_ctl, int use_shared, const KeySchedule* ks, cudaStream_t st) {
    return warpcell_dispatch(gpl, emax, tmax, pop, [&](auto g, auto r, auto k, auto p) {
        return warpcell_queue_launch_t<decltype(g)::value, decltype(r)::value, decltype(k)::value, decltype(p)::value>(
            args, items, n_items, counter, smem, grid, nwarps, shared_ctl, use_shared, ks, st);
    });
}

cudaError_t fused_queue_launch(const FusedArgs* args, const TileWork* items, int n_items, int* counter, int upt,
                               int nw, size_t smem, bool pop, int grid, TileCtl shared_ctl, int use_shared,
                               cudaStream_t st) {
    switch (upt * 2 + (pop ? 1 : 0)) {
        case 2: return fused_queue_launch_t<1, false, false>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        case 3: return fused_queue_launch_t<1, true, false>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        case 4: return fused_queue_launch_t<2, false, false>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        case 5: return fused_queue_launch_t<2, true, false>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        case 8: return fused_queue_launch_t<4, false, false>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        case 9: return fused_queue_launch_t<4, true, false>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        case 16: return fused_queue_launch_t<8, false, false>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        case 17: return fused_queue_launch_t<8, true, false>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        default: return cudaErrorInvalidValue;
    }
}

// Binomial tau-leap variant of the block-tile kernel (cle_fused.cuh, TAU), in gene quads or
// gene pairs per thread unit (same counts).  The plan is fused_plan's over units of qg genes.
FusedLaunch tau_plan(int G, int n_reg, int n_in, int n_na, int n_na_src, int qg) {
    while (qg < 4 && (G + qg - 1) / qg > fused_max_quads()) qg *= 2;  // at most 8 units a thread, 16 warps a block
    FusedLaunch L = fused_plan(G, n_reg, n_in, n_na, n_na_src, (G + qg - 1) / qg);
    L.qg = qg;
    return L;
}

// Genes per thread unit of the tau-leap for a network of G genes over N cells (every choice gives
// the same counts; SCRNA_TAU_GENES_PER_THREAD=1, 2 or 4 forces one).  Single genes when they give
// a tile more warps than pairs do, or the same warps in a launch of at least 4 warps per SM
// sub-partition; pairs otherwise, where the 4 chains of a pair's lock-step loops hide latency
// that a launch of few warps cannot.  Measured on a B200 (ms; quads / pairs / single genes):
// 5 genes x 5,000 cells 8.8 / 5.5 / 3.7; 10 telegraph genes x 20,000 cells 26.1 / 18.1 / 17.7;
// 100 regulated genes x 20,000 cells 78 / 41 / 39, x 2,000 cells 25 / 8.3 / 9.5.
int tau_genes_per_unit(int G, int n_reg, int n_in, int n_na, int n_na_src, int64_t N) {
    if (const char* e = std::getenv("SCRNA_TAU_GENES_PER_THREAD")) {
        const int q = std::atoi(e);
        return q == 1 || q == 4 ? q : 2;
    }
    const FusedLaunch one = tau_plan(G, n_reg, n_in, n_na, n_na_src, 1);
    const FusedLaunch two = tau_plan(G, n_reg, n_in, n_na, n_na_src, 2);
    // larger units where the tables, with one telegraph-flag byte per unit, outgrow shared memory
    if (two.smem > kMaxDynamicSmem) return 4;
    if (one.smem > kMaxDynamicSmem) return two.qg;
    if (one.qg != 1) return two.qg;  // too many genes for single-gene units
    if (one.nw > two.nw) return 1;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        sms = 148;
    const int64_t warps = (N + 31) / 32 * one.nw;
    return warps >= (int64_t)sms * 4 * 4 ? 1 : 2;
}

template <int QG>
static cudaError_t tau_launch_q(const FusedArgs& a, const FusedLaunch& L, bool pop, cudaStream_t st) {
    switch (L.upt * 2 + (pop ? 1 : 0)) {
        case 2: return fused_launch_t<1, false, true, QG>(a, L.nw, L.smem, st);
        case 3: return fused_launch_t<1, true, true, QG>(a, L.nw, L.smem, st);
        case 4: return fused_launch_t<2, false, true, QG>(a, L.nw, L.smem, st);
        case 5: return fused_launch_t<2, true, true, QG>(a, L.nw, L.smem, st);
        case 8: return fused_launch_t<4, false, true, QG>(a, L.nw, L.smem, st);
        case 9: return fused_launch_t<4, true, true, QG>(a, L.nw, L.smem, st);
        case 16: return fused_launch_t<8, false, true, QG>(a, L.nw, L.smem, st);
        case 17: return fused_launch_t<8, true, true, QG>(a, L.nw, L.smem, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t tau_launch(const FusedArgs& a, const FusedLaunch& L, bool pop, cudaStream_t st) {
    return L.qg == 1 ? tau_launch_q<1>(a, L, pop, st)
         : L.qg == 2 ? tau_launch_q<2>(a, L, pop, st)
                     : tau_launch_q<4>(a, L, pop, st);
}

template <int QG>
static cudaError_t tau_queue_launch_q(const FusedArgs* args, const TileWork* items, int n_items, int* counter,
                                      int upt, int nw, size_t smem, bool pop, int grid, TileCtl shared_ctl,
                                      int use_shared, cudaStream_t st) {
    switch (upt * 2 + (pop ? 1 : 0)) {
        case 2: return fused_queue_launch_t<1, false, true, QG>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        case 3: return fused_queue_launch_t<1, true, true, QG>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        case 4: return fused_queue_launch_t<2, false, true, QG>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        case 5: return fused_queue_launch_t<2, true, true, QG>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        case 8: return fused_queue_launch_t<4, false, true, QG>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        case 9: return fused_queue_launch_t<4, true, true, QG>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        case 16: return fused_queue_launch_t<8, false, true, QG>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        case 17: return fused_queue_launch_t<8, true, true, QG>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t tau_queue_launch(const FusedArgs* args, const TileWork* items, int n_items, int* counter, int upt, int nw,
                             size_t smem, bool pop, int grid, TileCtl shared_ctl, int use_shared, int qg,
                             cudaStream_t st) {
    if (qg == 1)
        return tau_queue_launch_q<1>(args, items, n_items, counter, upt, nw, smem, pop, grid, shared_ctl, use_shared, st);
    if (qg == 2)
        return tau_queue_launch_q<2>(args, items, n_items, counter, upt, nw, smem, pop, grid, shared_ctl, use_shared, st);
    return tau_queue_launch_q<4>(args, items, n_items, counter, upt, nw, smem, pop, grid, shared_ctl, use_shared, st);
}

}  // namespace scrna
