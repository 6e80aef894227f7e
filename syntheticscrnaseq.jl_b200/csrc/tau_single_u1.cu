// Instantiations of the block-tile kernel's binomial tau-leap variant as single genes, 1 gene(s) per thread.
#include "cle_fused.cuh"

namespace scrna {
template cudaError_t fused_launch_t<1, false, true, 1>(const FusedArgs&, int, size_t, cudaStream_t);
template cudaError_t fused_launch_t<1, true, true, 1>(const FusedArgs&, int, size_t, cudaStream_t);
template cudaError_t fused_queue_launch_t<1, false, true, 1>(const FusedArgs*, const TileWork*, int, int*, int, size_t,
                                                              int, TileCtl, int, cudaStream_t);
template cudaError_t fused_queue_launch_t<1, true, true, 1>(const FusedArgs*, const TileWork*, int, int*, int, size_t,
                                                             int, TileCtl, int, cudaStream_t);
}  // namespace scrna
