// Kernel instantiations for the f32 population storage (StoreF32).
#define LBM_TILE_MINB 4
#include "aa_store_impl.cuh"

LBM_DEFINE_STORAGE_OPS(storage_ops_f32, StoreF32, "f32")
