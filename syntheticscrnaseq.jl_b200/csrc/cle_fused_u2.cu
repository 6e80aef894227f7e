// Instantiations of the fused register-path kernel with 2 gene quad(s) per thread.
#include "cle_fused.cuh"

namespace scrna {
template cudaError_t fused_launch_t<2, false, false>(const FusedArgs&, int, size_t, cudaStream_t);
template cudaError_t fused_launch_t<2, true, false>(const FusedArgs&, int, size_t, cudaStream_t);
template cudaError_t fused_queue_launch_t<2, false, false>(const FusedArgs*, const TileWork*, int, int*, int, size_t, int, TileCtl, int,
                                                     cudaStream_t);
template cudaError_t fused_queue_launch_t<2, true, false>(const FusedArgs*, const TileWork*, int, int*, int, size_t, int, TileCtl, int,
                                                    cudaStream_t);
}  // namespace scrna
