// Instantiations of the block-tile kernel's binomial tau-leap variant in gene pairs, 8 pair(s) per thread.
#include "cle_fused.cuh"

namespace scrna {
template cudaError_t fused_launch_t<8, false, true, 2>(const FusedArgs&, int, size_t, cudaStream_t);
template cudaError_t fused_launch_t<8, true, true, 2>(const FusedArgs&, int, size_t, cudaStream_t);
template cudaError_t fused_queue_launch_t<8, false, true, 2>(const FusedArgs*, const TileWork*, int, int*, int, size_t,
                                                              int, TileCtl, int, cudaStream_t);
template cudaError_t fused_queue_launch_t<8, true, true, 2>(const FusedArgs*, const TileWork*, int, int*, int, size_t,
                                                             int, TileCtl, int, cudaStream_t);
}  // namespace scrna
