// Kernel instantiations for the f64 population storage (StoreF64).
#define LBM_TILE_MINB 2
#include "aa_store_impl.cuh"

LBM_DEFINE_STORAGE_OPS(storage_ops_f64, StoreF64, "f64")
