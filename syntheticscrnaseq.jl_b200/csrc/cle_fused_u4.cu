// Instantiations of the fused register-path kernel with 4 gene quad(s) per thread.
#include "cle_fused.cuh"

namespace scrna {
template cudaError_t fused_launch_t<4, false>(const FusedArgs&, int, size_t, cudaStream_t);
template cudaError_t fused_launch_t<4, true>(const FusedArgs&, int, size_t, cudaStream_t);
}  // namespace scrna
