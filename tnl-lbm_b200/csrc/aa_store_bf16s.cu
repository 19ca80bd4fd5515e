// Kernel instantiations for the bf16s population storage (StoreBF16S).
#define LBM_TILE_MINB 4
#include "aa_store_impl.cuh"

LBM_DEFINE_STORAGE_OPS(storage_ops_bf16s, StoreBF16S, "bf16s")
