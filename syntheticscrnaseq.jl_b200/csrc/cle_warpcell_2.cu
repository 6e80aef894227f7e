// Instantiations of the warp-per-cell-group kernel with 2 genes per lane.
#include "cle_warpcell.cuh"

namespace scrna {
template cudaError_t warpcell_launch_t<2, 4, false>(const FusedArgs&, cudaStream_t);
template cudaError_t warpcell_queue_launch_t<2, 4, false>(const FusedArgs*, const TileWork*, int, int*, size_t, int, TileCtl, int,
                                                              cudaStream_t);
template cudaError_t warpcell_launch_t<2, 4, true>(const FusedArgs&, cudaStream_t);
template cudaError_t warpcell_queue_launch_t<2, 4, true>(const FusedArgs*, const TileWork*, int, int*, size_t, int, TileCtl, int,
                                                              cudaStream_t);
template cudaError_t warpcell_launch_t<2, 8, false>(const FusedArgs&, cudaStream_t);
template cudaError_t warpcell_queue_launch_t<2, 8, false>(const FusedArgs*, const TileWork*, int, int*, size_t, int, TileCtl, int,
                                                              cudaStream_t);
template cudaError_t warpcell_launch_t<2, 8, true>(const FusedArgs&, cudaStream_t);
template cudaError_t warpcell_queue_launch_t<2, 8, true>(const FusedArgs*, const TileWork*, int, int*, size_t, int, TileCtl, int,
                                                              cudaStream_t);
template cudaError_t warpcell_launch_t<2, 16, false>(const FusedArgs&, cudaStream_t);
template cudaError_t warpcell_queue_launch_t<2, 16, false>(const FusedArgs*, const TileWork*, int, int*, size_t, int, TileCtl, int,
                                                              cudaStream_t);
template cudaError_t warpcell_launch_t<2, 16, true>(const FusedArgs&, cudaStream_t);
template cudaError_t warpcell_queue_launch_t<2, 16, true>(const FusedArgs*, const TileWork*, int, int*, size_t, int, TileCtl, int,
                                                              cudaStream_t);
}  // namespace scrna
