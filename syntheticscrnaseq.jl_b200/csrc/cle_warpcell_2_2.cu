// Instantiations of the warp-per-cell-group kernel: 2 genes per lane, 2 padded in-edges per gene.
#include "cle_warpcell.cuh"

SCRNA_WARPCELL_INSTANTIATE_ALL(2, 2)
