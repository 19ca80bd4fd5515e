// Kernel instantiations for the bf16sr population storage (StoreBF16SR).
#define LBM_TILE_MINB 4
#include "aa_store_impl.cuh"

LBM_DEFINE_STORAGE_OPS(storage_ops_bf16sr, StoreBF16SR, "bf16sr")
