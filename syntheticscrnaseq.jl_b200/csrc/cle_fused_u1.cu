// Instantiations of the fused register-path kernel with 1 gene quad(s) per thread.
#include "cle_fused.cuh"

namespace scrna {
template cudaError_t fused_launch_t<1, false>(const FusedArgs&, int, size_t, cudaStream_t);
template cudaError_t fused_launch_t<1, true>(const FusedArgs&, int, size_t, cudaStream_t);
}  // namespace scrna
