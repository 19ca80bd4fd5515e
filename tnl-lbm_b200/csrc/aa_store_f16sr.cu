// Kernel instantiations for the f16sr population storage (StoreF16SR).
#define LBM_TILE_MINB 4
#include "aa_store_impl.cuh"

LBM_DEFINE_STORAGE_OPS(storage_ops_f16sr, StoreF16SR, "f16sr")
