// Instantiations of the warp-per-cell-group kernel: 4 genes per lane, 4 padded in-edges per gene.
#include "cle_warpcell.cuh"

SCRNA_WARPCELL_INSTANTIATE_ALL(4, 4)
