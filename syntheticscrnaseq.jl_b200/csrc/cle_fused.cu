// Launch planning and dispatch of the fused register-path kernel (the kernel
// template is in cle_fused.cuh; each quads-per-thread variant is compiled in its
// own translation unit).
#include "cle_internal.h"
#include <cuda_runtime.h>

namespace scrna {

template <int UPT, bool POP>
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

cudaError_t fused_launch(const FusedArgs& a, const FusedLaunch& L, bool pop, cudaStream_t st) {
    switch (L.upt * 2 + (pop ? 1 : 0)) {
        case 2: return fused_launch_t<1, false>(a, L.nw, L.smem, st);
        case 3: return fused_launch_t<1, true>(a, L.nw, L.smem, st);
        case 4: return fused_launch_t<2, false>(a, L.nw, L.smem, st);
        case 5: return fused_launch_t<2, true>(a, L.nw, L.smem, st);
        case 8: return fused_launch_t<4, false>(a, L.nw, L.smem, st);
        case 9: return fused_launch_t<4, true>(a, L.nw, L.smem, st);
        case 16: return fused_launch_t<8, false>(a, L.nw, L.smem, st);
        case 17: return fused_launch_t<8, true>(a, L.nw, L.smem, st);
        default: return cudaErrorInvalidValue;
    }
}

// ---- warp-per-cell-group variant for small networks ---------------------------------------
template <int GPL, int NREG, bool POP>
cudaError_t warpcell_launch_t(const FusedArgs& a, cudaStream_t st);
template <int GPL, int NREG, bool POP>
cudaError_t warpcell_queue_launch_t(const FusedArgs* args, const TileWork* items, int n_items, int* counter,
                                    size_t smem, int grid, TileCtl shared_ctl, int use_shared, cudaStream_t st);
template <int UPT, bool POP>
cudaError_t fused_queue_launch_t(const FusedArgs* args, const TileWork* items, int n_items, int* counter,
                                 int nw, size_t smem, int grid, TileCtl shared_ctl, int use_shared, cudaStream_t st);

int warpcell_max_genes() { return 32; }
int warpcell_max_regs() { return 16; }
int warpcell_nreg_class(int n_reg) { return n_reg <= 4 ? 4 : n_reg <= 8 ? 8 : 16; }

// Genes per lane for a network: a cost model of issue slots per cell-gene-step
// (Philox calls per gene, plus lanes left idle by the cell packing).
int warpcell_pick_gpl(int G, bool bursty) {
    double best = 1e30;
    int pick = 2;
    for (int gpl : {2, 4}) {
        const int lpc = (G + gpl - 1) / gpl;
        const int cpw = 32 / lpc;
        const double philox = 0.5 + (bursty ? 0.02 : 0.0);
        const double waste = 32.0 * gpl / ((double)G * cpw);
        const double cost = (48.0 + 42.0 * philox) * waste;
        if (cost < best) { best = cost; pick = gpl; }
    }
    return pick;
}

size_t warpcell_smem(int G, int gpl, int n_reg, int n_na, int n_na_src) {
    const int lpc = (G + gpl - 1) / gpl;
    const int cpw = 32 / lpc;
    const int nreg = warpcell_nreg_class(n_reg);
    size_t b = (size_t)4 * 2 * (cpw + 1) * (nreg + 1) * sizeof(float);
    b += (size_t)n_na * sizeof(NonAdd) + (size_t)n_na_src * sizeof(int32_t);
    return (b + 15) & ~(size_t)15;
}

#define SCRNA_WARP_DISPATCH(CALL)                                        \
    switch ((gpl == 4 ? 100 : 0) + nreg * 2 + (pop ? 1 : 0)) {           \
        case 8: return CALL(2, 4, false);                                \
        case 9: return CALL(2, 4, true);                                 \
        case 16: return CALL(2, 8, false);                               \
        case 17: return CALL(2, 8, true);                                \
        case 32: return CALL(2, 16, false);                              \
        case 33: return CALL(2, 16, true);                               \
        case 108: return CALL(4, 4, false);                              \
        case 109: return CALL(4, 4, true);                               \
        case 116: return CALL(4, 8, false);                              \
        case 117: return CALL(4, 8, true);                               \
        case 132: return CALL(4, 16, false);                             \
        case 133: return CALL(4, 16, true);                              \
        default: return cudaErrorInvalidValue;                           \
    }

cudaError_t warpcell_launch(const FusedArgs& a0, const float* wdense, int gpl, bool pop, cudaStream_t st) {
    FusedArgs a = a0;
    a.wdense = wdense;
    const int nreg = warpcell_nreg_class(a.n_reg);
#define CALL(G_, R_, P_) warpcell_launch_t<G_, R_, P_>(a, st)
    SCRNA_WARP_DISPATCH(CALL)
#undef CALL
}

cudaError_t warpcell_queue_launch(const FusedArgs* args, const TileWork* items, int n_items, int* counter, int gpl,
                                  int nreg, bool pop, size_t smem, int grid, TileCtl shared_ctl, int use_shared,
                                  cudaStream_t st) {
#define CALL(G_, R_, P_) \
    warpcell_queue_launch_t<G_, R_, P_>(args, items, n_items, counter, smem, grid, shared_ctl, use_shared, st)
    SCRNA_WARP_DISPATCH(CALL)
#undef CALL
}

cudaError_t fused_queue_launch(const FusedArgs* args, const TileWork* items, int n_items, int* counter, int upt,
                               int nw, size_t smem, bool pop, int grid, TileCtl shared_ctl, int use_shared,
                               cudaStream_t st) {
    switch (upt * 2 + (pop ? 1 : 0)) {
        case 2: return fused_queue_launch_t<1, false>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        case 3: return fused_queue_launch_t<1, true>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        case 4: return fused_queue_launch_t<2, false>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        case 5: return fused_queue_launch_t<2, true>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        case 8: return fused_queue_launch_t<4, false>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        case 9: return fused_queue_launch_t<4, true>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        case 16: return fused_queue_launch_t<8, false>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        case 17: return fused_queue_launch_t<8, true>(args, items, n_items, counter, nw, smem, grid, shared_ctl, use_shared, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace scrna
