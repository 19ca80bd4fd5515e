// Kernel instantiations for the f32s population storage (StoreF32S).
#define LBM_TILE_MINB 4
#include "aa_store_impl.cuh"

LBM_DEFINE_STORAGE_OPS(storage_ops_f32s, StoreF32S, "f32s")
