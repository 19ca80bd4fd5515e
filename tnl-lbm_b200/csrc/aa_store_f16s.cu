// Kernel instantiations for the f16s population storage (StoreF16S).
#define LBM_TILE_MINB 4
#include "aa_store_impl.cuh"

LBM_DEFINE_STORAGE_OPS(storage_ops_f16s, StoreF16S, "f16s")
