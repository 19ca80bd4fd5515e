// Kernel instantiations for the i16s population storage (StoreI16S).
#define LBM_TILE_MINB 4
#include "aa_store_impl.cuh"

LBM_DEFINE_STORAGE_OPS(storage_ops_i16s, StoreI16S, "i16s")
