// Instantiations of the warp-per-cell-group kernel: 4 genes per lane, up to 16 regulator slots.
#include "cle_warpcell.cuh"

SCRNA_WARPCELL_INSTANTIATE_ALL(4, 16)
