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

}  // namespace scrna
